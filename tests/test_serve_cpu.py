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


def _build(req):
    n = req["n"]
    arr = {k: None for k in ("vel", "omega", "radius", "pmass", "omoi", "state", "phase")}
    arr["pos"] = np.zeros((3, n))
    return (None, None, arr, (np.zeros((1, 3, 3)), np.zeros((1, 3))), {})


def _server(capacity):
    tmpl = configs.hopper_case(2000)
    return DemServer(load_library(), _build, tmpl, hbm_budget_bytes=1 << 30, max_systems=8, builders=0,
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
