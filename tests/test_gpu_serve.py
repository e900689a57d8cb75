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
