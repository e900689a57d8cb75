"""Host logic of the DEM server (admission, retirement, latency accounting)
against a CPU model of the batch handle; no kernel runs here."""
import numpy as np
import pytest

from mfix_dem import abi, configs, load_library
from mfix_dem.serve import DemServer
from mfix_dem.system import DemError


class FakeBatch:
    """Particle capacity only; every started system advances by the steps."""

    def __init__(self, capacity):
        self.capacity = capacity
        self.used = {}
        self.steps = {}
        self.started = set()
        self.next = 0
        self.max_live = 0

    def set_graphs(self, on):
        pass

    def memory_info(self):
        # the pair room never binds here: admission is by particle ranges
        return {"pairs": 0, "pair_capacity": 1 << 40}

    def add(self, prm, n):
        if sum(self.used.values()) + n > self.capacity:
            raise DemError(abi.DEM_ERR_CAPACITY, "dem_sys_add", "full")
        sid = self.next
        self.next += 1
        self.used[sid] = n
        self.steps[sid] = 0
        self.max_live = max(self.max_live, len(self.used))
        return sid

    def set_walls(self, sid, v, nrm):
        pass

    def upload_state(self, sid, *a):
        pass

    def start(self, sids):
        self.started.update(sids)

    def step(self, k):
        for s in self.started:
            self.steps[s] += k

    def stats(self, sid):
        return {"n_normal": self.used[sid], "steps_done": self.steps[sid]}

    def download_state(self, sid):
        return {"steps": self.steps[sid]}

    def remove(self, sid):
        del self.used[sid]
        self.started.discard(sid)

    def close(self):
        pass


TEMPLATE = configs.hopper_case(2000)


def _build(req):
    n = req["n"]
    arr = {k: None for k in ("vel", "omega", "radius", "pmass", "omoi", "state", "phase")}
    arr["pos"] = np.zeros((3, n))
    return (None, TEMPLATE[1], arr, (np.zeros((1, 3, 3)), np.zeros((1, 3))), {})


def _server(capacity):
    return DemServer(load_library(), _build, TEMPLATE, hbm_budget_bytes=1 << 30, max_systems=8, builders=0,
                     batch=FakeBatch(capacity))


def test_admission_overlaps_and_respects_capacity():
    reqs = [{"rid": k, "arrival": float(k), "n": 1000, "steps": 100} for k in range(6)]
    srv = _server(capacity=2500)          # two requests fit at a time
    out = srv.run(reqs, clock=lambda: float(srv.chunks_done), idle_sleep=0.0, keep_state=True)
    res = out["results"]
    assert [r.rid for r in res] == list(range(6))
    assert srv.batch.max_live == 2
    for r in res:
        assert r.stats["steps_done"] == 100 and r.state["steps"] == 100
        assert r.finished >= r.admitted >= r.arrival
    # the third request waited for a slot
    assert res[2].admitted >= res[0].finished
    assert out["p99_s"] >= out["p50_s"] > 0
    assert out["particle_steps"] == 6 * 1000 * 100


def test_request_larger_than_budget_is_an_error():
    srv = _server(capacity=500)
    with pytest.raises(RuntimeError):
        srv.run([{"rid": 0, "arrival": 0.0, "n": 1000, "steps": 25}], clock=lambda: 0.0, idle_sleep=0.0)


def test_steps_must_be_whole_chunks():
    srv = _server(capacity=5000)
    with pytest.raises(ValueError):
        srv.run([{"rid": 0, "arrival": 0.0, "n": 100, "steps": 30}], clock=lambda: 0.0)


def test_limits_fill_the_budget_by_the_library_footprint():
    """The server's limits: the footprint the library counts for them is
    within the budget and within one particle row of it; the bytes per
    particle cover the state and the pair-list room."""
    from mfix_dem.serve import footprint, limits_for_budget
    lib = load_library()
    _, prm, _, walls, _ = TEMPLATE
    for budget, nsys in ((1 << 30, 8), (4 << 30, 16), (40 * 10**9, 64)):
        lim, per = limits_for_budget(lib, prm, walls[0].shape[0], budget, nsys, pairs_per_particle=6)
        f = footprint(lib, prm, lim)
        assert f["bytes"] <= budget < f["bytes"] + 64 * per + 1
        assert f["pair_capacity"] == 6 * lim.max_particles + 1024
        # state and histories (> 500 B), plus 6 pairs of > 100 B each
        assert 500 + 6 * 100 < per < 3000
        # the pair-list room is the one term that grows with pairs_per_particle
        lim8 = abi.DemBatchLimits.from_buffer_copy(lim)
        lim8.pairs_per_particle = 8
        assert footprint(lib, prm, lim8)["bytes"] > f["bytes"]


def test_request_footprint_grows_with_the_case():
    srv = _server(capacity=10**6)
    small, big = _build({"n": 10_000}), _build({"n": 100_000})
    fs, fb = srv.request_footprint(small), srv.request_footprint(big)
    assert fs < fb
    # the difference is 90,000 particles at the server's bytes per particle
    assert abs((fb - fs) - 90_000 * srv.bytes_per_particle) < 0.01 * (fb - fs)
