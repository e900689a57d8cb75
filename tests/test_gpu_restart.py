"""Restart on the GPU: a whole-state snapshot restored into a fresh handle,
and the RES restart file, continue bit for bit like the uninterrupted run
(and like the oracle's)."""
import numpy as np
import pytest

from cases import make_system, settling_case
from mfix_dem.restart import restore, snapshot

pytestmark = pytest.mark.gpu


def _gpu(prm, n):
    from mfix_dem import GpuSystem
    return GpuSystem(prm, n)


def _case():
    return settling_case(n_side=(6, 14, 6), spacing=0.99, jitter=0.05, coll="HERTZ", intg="ADAMS_BASHFORTH",
                         nsn=10, mew_r=0.01)


def _same(a, b):
    sa, sb = a.download_state(), b.download_state()
    for k in ("pos", "vel", "omega", "state"):
        assert np.array_equal(sa[k], sb[k]), k
    for x, y in zip(a.download_pairs(), b.download_pairs()):
        assert np.array_equal(x, y)
    for x, y in zip(a.download_wall_history(), b.download_wall_history()):
        assert np.array_equal(x, y)


def test_snapshot_restore_matches_uninterrupted_and_oracle():
    from oracle_ffi import OracleSystem
    case, prm, arr, walls = _case()
    a = make_system(_gpu, prm, arr, walls)
    a.step(40)
    o = make_system(OracleSystem, prm, arr, walls)
    o.step(40)
    b = make_system(_gpu, prm, arr, walls)
    b.step(20)
    snap = snapshot(b)
    assert (snap["walls"][0] > 0).any() and np.abs(snap["pairs"][2]).max() > 0
    c = _gpu(prm, arr["pos"].shape[1])
    c.set_walls(*walls)
    restore(c, snap, arr["radius"], arr["pmass"], arr["omoi"], arr["phase"])
    c.step(20)
    _same(a, c)
    _same(o, c)


def test_res_file_restart(tmp_path):
    """WRITE_RES0_DES at a rebuild step, READ_RES0_DES into a fresh handle
    (pairs and PFT from the file; the wall and Adams-Bashforth histories,
    which the format does not hold, from the snapshot): the run continues
    bit for bit.  Reading without the pair section and rebuilding gives the
    same pair list."""
    case, prm, arr, walls = _case()
    n = arr["pos"].shape[1]
    a = make_system(_gpu, prm, arr, walls)
    a.step(40)
    b = make_system(_gpu, prm, arr, walls)
    b.step(20)
    snap = snapshot(b)
    path = tmp_path / "settle_DES.RES"
    b.write_res0_des(path, ro_sol=[case.ro_s0[0]], vtp_findex=4)
    c = _gpu(prm, n)
    c.set_walls(*walls)
    info = c.read_res0_des(path, restore_pairs=True)
    assert info.n_particles == n and info.vtp_findex == 4 and info.n_pairs == len(snap["pairs"][1])
    c.desgrid_pic()
    c.upload_wall_history(*snap["walls"])
    acc, racc, _ = snap["ab2"]
    c.set_ab2_history(acc, racc, first_pass=False)
    c.nn = snap["nn"]
    c.step(20)
    _same(a, c)
    d = _gpu(prm, n)
    d.set_walls(*walls)
    d.read_res0_des(path, restore_pairs=False)
    d.init_neighbors()
    ni, nb, _ = d.download_pairs()
    assert np.array_equal(ni, snap["pairs"][0]) and np.array_equal(nb, snap["pairs"][1])
