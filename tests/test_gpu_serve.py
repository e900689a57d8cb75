"""Served hopper cases: each result is the same alone and in the mix.

Requests arrive while others run (on a clock that advances one unit per
step chunk, so admission is reproducible), are admitted into the running
batch, and leave when done.  Every case must end in exactly the state it
reaches when it is served alone -- the same batch kernels, its own step
numbering and rebuild cadence -- so the comparison is bit for bit.
"""
import numpy as np
import pytest

from mfix_dem import configs, load_library
from mfix_dem.serve import DemServer

pytestmark = pytest.mark.gpu


def _build(req):
    return configs.hopper_case(req["n"], friction=req["friction"], outlet_d=req["outlet_d"], seed=req["seed"],
                               spacing=0.98)


REQS = [
    {"rid": 0, "arrival": 0.0, "n": 3000, "friction": 0.3, "outlet_d": 8, "seed": 5, "steps": 200},
    {"rid": 1, "arrival": 2.0, "n": 5000, "friction": 0.5, "outlet_d": 6, "seed": 6, "steps": 100},
    {"rid": 2, "arrival": 3.0, "n": 2000, "friction": 0.2, "outlet_d": 10, "seed": 7, "steps": 150},
    {"rid": 3, "arrival": 5.0, "n": 4000, "friction": 0.4, "outlet_d": 9, "seed": 8, "steps": 75},
]


def _serve(reqs):
    srv = DemServer(load_library(), _build, _build(REQS[0]), hbm_budget_bytes=2 << 30, max_systems=8,
                    builders=0)
    out = srv.run(reqs, clock=lambda: float(srv.chunks_done), keep_state=True, idle_sleep=0.0)
    srv.close()
    return out


def test_served_results_same_alone_and_in_the_mix():
    mix = _serve(REQS)
    assert [r.rid for r in mix["results"]] == [0, 1, 2, 3]
    # the mix really overlapped: request 1 was admitted while request 0 ran
    r0, r1 = mix["results"][0], mix["results"][1]
    assert r1.admitted < r0.finished
    assert mix["p99_s"] >= mix["p50_s"] > 0
    for req, got in zip(REQS, mix["results"]):
        alone = _serve([dict(req, arrival=0.0)])["results"][0]
        assert got.stats["n_normal"] == alone.stats["n_normal"]
        for k in ("pos", "vel", "omega", "state"):
            assert np.array_equal(got.state[k], alone.state[k]), (req["rid"], k)
        assert got.stats["steps_done"] == req["steps"]


def test_batch_memory_is_its_footprint():
    """The device memory a batch handle takes is what dem_batch_footprint
    counts for its limits (the same arrays, the same sizes): dem_memory_info
    reports it exactly, and the device's free memory drops by it (within the
    allocation granularity); served cases then stay within the pair room."""
    import torch
    from mfix_dem.serve import footprint, limits_for_budget
    from mfix_dem.system import BatchSystem
    lib = load_library()
    _, prm, arr, walls, _ = _build(REQS[1])
    lim, per = limits_for_budget(lib, prm, walls[0].shape[0], 2 << 30, 8)
    f = footprint(lib, prm, lim)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    b = BatchSystem(lib, prm, lim)
    m = b.memory_info()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    try:
        for k in ("array_bytes", "pair_bytes", "pair_capacity"):
            assert m[k] == f[k], k
        used = free0 - free1
        assert abs(used - f["bytes"]) <= 0.05 * f["bytes"] + (64 << 20), (used, f["bytes"])
        sid = b.add(prm, arr["pos"].shape[1])
        b.set_walls(sid, *walls)
        b.upload_state(sid, arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                       arr["state"], arr["phase"])
        b.start([sid])
        b.step(50)
        m2 = b.memory_info()
        assert 0 < m2["pairs"] <= m2["pair_capacity"] == f["pair_capacity"]
    finally:
        b.close()
