"""Restart equivalence on the oracle: a run interrupted at a rebuild step,
snapshotted (state, pair list with PFT_NEIGHBOR, wall-contact history,
Adams-Bashforth history) and restored into a fresh system continues bit for
bit like the uninterrupted run (the reference's restart test demands the
same of a RES restart)."""
import numpy as np
import pytest

from cases import make_system, settling_case
from mfix_dem.restart import restore, snapshot
from oracle_ffi import OracleSystem


@pytest.mark.parametrize("coll,intg", [("LSD", "EULER"), ("HERTZ", "ADAMS_BASHFORTH")])
def test_snapshot_restore_continues_bitwise(coll, intg):
    case, prm, arr, walls = settling_case(n_side=(4, 10, 4), spacing=0.99, jitter=0.05, coll=coll, intg=intg,
                                          nsn=10, mew_r=0.01 if coll == "HERTZ" else 0.0)
    a = make_system(OracleSystem, prm, arr, walls)
    a.step(40)
    b = make_system(OracleSystem, prm, arr, walls)
    b.step(20)
    snap = snapshot(b)
    fid, _ = snap["walls"]
    assert (fid > 0).any()                        # wall contacts carry history
    assert np.abs(snap["pairs"][2]).max() > 0     # so do pair contacts
    c = OracleSystem(prm, arr["pos"].shape[1])
    c.set_walls(*walls)
    restore(c, snap, arr["radius"], arr["pmass"], arr["omoi"], arr["phase"])
    c.step(20)
    sa, sc = a.download_state(), c.download_state()
    for k in ("pos", "vel", "omega", "state"):
        assert np.array_equal(sa[k], sc[k]), k
    for x, y in zip(a.download_pairs(), c.download_pairs()):
        assert np.array_equal(x, y)
    for x, y in zip(a.download_wall_history(), c.download_wall_history()):
        assert np.array_equal(x, y)


def test_histories_matter():
    """Control: restoring the particles and pairs but not the wall-contact and
    Adams-Bashforth histories (what the RES format holds) changes the run."""
    case, prm, arr, walls = settling_case(n_side=(4, 10, 4), spacing=0.99, jitter=0.05, coll="HERTZ",
                                          intg="ADAMS_BASHFORTH", nsn=10)
    a = make_system(OracleSystem, prm, arr, walls)
    a.step(40)
    b = make_system(OracleSystem, prm, arr, walls)
    b.step(20)
    snap = snapshot(b)
    c = OracleSystem(prm, arr["pos"].shape[1])
    c.set_walls(*walls)
    st = snap["state"]
    c.upload_state(st["pos"], st["vel"], st["omega"], arr["radius"], arr["pmass"], arr["omoi"], st["state"],
                   arr["phase"])
    c.desgrid_pic()
    c.upload_pairs(*snap["pairs"])
    c.nn = snap["nn"]
    c.step(20)
    assert not np.array_equal(a.download_state()["vel"], c.download_state()["vel"])
