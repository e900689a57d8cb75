"""The launch-shape autotuner changes no result.

A handle tuned partway (dem_autotune after 10 steps) must reach the same
state, bit for bit, as an untuned handle over the same steps; tuning a batch
likewise.  The chosen shapes are among the candidates."""
import numpy as np
import pytest

from mfix_dem import GpuSystem
from cases import make_system, settling_case
from test_gpu_batch import _add, _batch, _cases, _compare

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results():
    case, prm, arr, walls = settling_case(n_side=(8, 20, 8), spacing=0.98, jitter=0.03, coll="HERTZ",
                                          mew_r=0.01, seed=77)
    a = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    b = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    a.step(10)
    b.step(10)
    t = b.autotune(reps=3)
    assert t["pair_threads"] in (64, 128, 256) and t["pair_blocks_per_sm"] in (2, 4, 8, 16)
    assert t["gather_threads"] in (64, 128, 256) and t["neigh_threads"] in (32, 64, 128)
    assert t["pair_ms"] > 0 and t["gather_ms"] > 0 and t["neigh_ms"] > 0
    a.step(50)
    b.step(50)
    sa, sb = a.download_state(), b.download_state()
    for k in ("pos", "vel", "omega", "state"):
        assert np.array_equal(sa[k], sb[k]), k
    pa, pb = a.download_pairs(), b.download_pairs()
    for x, y in zip(pa, pb):
        assert np.array_equal(x, y)
    # set_tuning round trip
    b.set_tuning({"pair_threads": 128, "pair_blocks_per_sm": 4, "gather_threads": 64, "neigh_threads": 32})
    g = b.get_tuning()
    assert (g["pair_threads"], g["pair_blocks_per_sm"], g["gather_threads"], g["neigh_threads"]) == (128, 4, 64, 32)
    a.close()
    b.close()


def test_autotune_batch_keeps_results():
    cases = _cases(seeds=(51, 52, 53))
    bt = _batch(cases)
    ids = [_add(bt, c) for c in cases]
    bt.start(ids)
    bt.step(5)
    bt.autotune(reps=2)
    bt.step(45)
    from test_gpu_batch import _alone
    for sid, case in zip(ids, cases):
        g = _alone(case, 50)
        _compare(bt, sid, g)
        g.close()
    bt.close()
