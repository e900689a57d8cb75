"""Batch handles: many independent systems in one handle.

Every system of a batch must give exactly the results it gives in a handle
of its own -- positions, velocities, spins, states, the pair list and its
tangential history -- whatever else shares the batch, and when systems join
or leave between steps.  The FP64 path is compared bit for bit; the split
path (compiled with FMA contraction) within 1e-12 relative.
"""
import numpy as np
import pytest

from mfix_dem import GpuBatch, GpuSystem, abi, load_library
from mfix_dem import params as P
from cases import make_system, settling_case

pytestmark = pytest.mark.gpu

SPLIT_TOL = 1e-12


def _cases(seeds=(11, 12, 13), **kw):
    a = settling_case(n_side=(6, 20, 6), seed=seeds[0], kn=1000.0, mew=0.1, **kw)
    b = settling_case(n_side=(5, 12, 4), seed=seeds[1], kn=1500.0, mew=0.3, spacing=0.98, **kw)
    c = settling_case(n_side=(8, 16, 8), seed=seeds[2], kn=600.0, mew=0.2, vmax=0.2, **kw)
    return [a, b, c]


def _entry(case):
    _, prm, arr, walls = case
    return prm, arr["pos"].shape[1], walls[0].shape[0]


def _batch(cases, max_systems=None, slack=1.0):
    lim = P.batch_limits(load_library(), [_entry(c) for c in cases], max_systems=max_systems, slack=slack)
    return GpuBatch(cases[0][1], lim)


def _add(bt, case):
    _, prm, arr, walls = case
    sid = bt.add(prm, arr["pos"].shape[1])
    bt.set_walls(sid, *walls)
    bt.upload_state(sid, arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                    arr["state"], arr["phase"])
    return sid


def _alone(case, steps):
    _, prm, arr, walls = case
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    if steps:
        g.step(steps)
    return g


def _compare(bt, sid, g, tol=0.0):
    sb, sg = bt.download_state(sid), g.download_state()
    assert np.array_equal(sb["state"], sg["state"])
    for k in ("pos", "vel", "omega"):
        if tol == 0.0:
            assert np.array_equal(sb[k], sg[k]), (k, float(np.max(np.abs(sb[k] - sg[k]))))
        else:
            scale = max(float(np.max(np.abs(sg[k]))), 1e-300)
            assert float(np.max(np.abs(sb[k] - sg[k]))) <= tol * scale, k
    nib, nbb, pfb = bt.download_pairs(sid)
    nig, nbg, pfg = g.download_pairs()
    assert np.array_equal(nib, nig)
    assert np.array_equal(nbb, nbg)
    if tol == 0.0:
        assert np.array_equal(pfb, pfg)
    else:
        assert float(np.max(np.abs(pfb - pfg), initial=0.0)) <= tol * max(float(np.max(np.abs(pfg), initial=0.0)), 1e-300)
    st = bt.stats(sid)
    assert st["n_normal"] == g.stats()["n_normal"]
    assert st["n_pairs"] == nbg.shape[0]


def test_batch_matches_each_system_alone():
    cases = _cases()
    bt = _batch(cases)
    ids = [_add(bt, c) for c in cases]
    bt.start(ids)
    bt.step(60)  # rebuilds at NN = 1, 25, 50
    for sid, case in zip(ids, cases):
        g = _alone(case, 60)
        _compare(bt, sid, g)
        assert bt.info(sid)["next_nn"] == 61
        g.close()
    bt.close()


def test_systems_join_and_leave_between_steps():
    a, b, c = _cases(seeds=(21, 22, 23))
    d = settling_case(n_side=(4, 10, 4), seed=24, kn=800.0, mew=0.4, spacing=0.98)
    bt = _batch([a, b, c, d], max_systems=4, slack=1.0)
    ia, ib = _add(bt, a), _add(bt, b)
    bt.start([ia, ib])
    bt.step(30)
    ic = _add(bt, c)          # joins at A's and B's NN = 31, its own NN = 1
    bt.start([ic])
    bt.step(20)
    bt.remove(ib)             # B leaves; D takes free space
    idd = _add(bt, d)
    bt.start([idd])
    bt.step(30)
    for sid, case, steps in ((ia, a, 80), (ic, c, 50), (idd, d, 30)):
        g = _alone(case, steps)
        _compare(bt, sid, g)
        g.close()
    bt.close()


def test_batch_hertz_periodic_adams_bashforth():
    cases = _cases(seeds=(31, 32, 33), coll="HERTZ", intg="ADAMS_BASHFORTH", mew_r=0.02,
                   periodic=(True, False, True))
    bt = _batch(cases)
    ids = [_add(bt, c) for c in cases]
    bt.start(ids)
    bt.step(55)
    for sid, case in zip(ids, cases):
        g = _alone(case, 55)
        _compare(bt, sid, g)
        g.close()
    bt.close()


def test_batch_split_precision():
    cases = _cases(seeds=(41, 42, 43), coll="HERTZ", precision=abi.DEM_PREC_SPLIT)
    bt = _batch(cases)
    ids = [_add(bt, c) for c in cases]
    bt.start(ids)
    bt.step(40)
    for sid, case in zip(ids, cases):
        g = _alone(case, 40)
        _compare(bt, sid, g, tol=SPLIT_TOL)
        g.close()
    bt.close()


def test_batch_refuses_single_system_calls():
    cases = _cases()[:1]
    bt = _batch(cases)
    _add(bt, cases[0])
    with pytest.raises(Exception):
        bt._call("step", bt._h, 1, 1)
    with pytest.raises(Exception):
        bt.step(1)  # a system with particles has not been started
    bt.close()


def test_extent_grows_and_shrinks_with_long_rows():
    """The step kernels of a batch cover the extent of the live systems'
    ranges.  A small system (its range ends inside a 64-particle block, so
    padding slots follow it) runs alone; a system with rows of a few hundred
    neighbours (three large spheres among small ones) joins past it, runs,
    and leaves from the top of the extent; a third joins where it was.
    Each system matches its own handle bit for bit."""
    from cases import bimodal_case
    a = settling_case(n_side=(5, 10, 5), seed=41, kn=900.0, mew=0.2)
    big = bimodal_case()
    c = settling_case(n_side=(4, 10, 4), seed=43, kn=700.0, mew=0.3, spacing=0.98)
    bt = _batch([a, big, c], max_systems=3, slack=1.0)
    ia = _add(bt, a)
    bt.start([ia])
    bt.step(30)
    ib = _add(bt, big)
    bt.start([ib])
    bt.step(30)
    g = _alone(big, 30)
    _compare(bt, ib, g)
    g.close()
    bt.remove(ib)
    bt.step(25)
    ic = _add(bt, c)
    bt.start([ic])
    bt.step(30)
    for sid, case, steps in ((ia, a, 115), (ic, c, 30)):
        g = _alone(case, steps)
        _compare(bt, sid, g)
        g.close()
    bt.close()
