"""Outflow boundaries on the oracle (MASS_OUTFLOW_DEM, UPDATE_EXIT_DES_VEL,
mass_outflow_dem.f): particles crossing the floor of a box are marked
EXITING while they straddle it and deleted once their centre is past it;
the deletions force a neighbour search."""
import numpy as np
import pytest

from cases import make_system
from mfix_dem import abi
from oracle_ffi import OracleSystem
from outflow_cases import outflow_case


def _run(mass_outflow, intg="EULER", steps=(100, 100, 100, 100)):
    case, prm, arr, walls, bc = outflow_case(mass_outflow, intg=intg)
    s = make_system(OracleSystem, prm, arr, walls)
    s.set_outflow_bcs([bc])
    seen_exit = 0
    for k in steps:
        s.step(k)
        st = s.download_state()
        ex = st["state"] == abi.DEM_STATE_EXITING
        seen_exit = max(seen_exit, int(ex.sum()))
        # straddling particles: centre above the floor by at most a radius
        if ex.any():
            y = st["pos"][1, ex]
            assert np.all(y > 0.0) and np.all(y <= arr["radius"][ex] + 1e-3)
            vy = st["vel"][1, ex]
            if mass_outflow:
                assert np.allclose(st["vel"][:, ex], np.array([[0.0], [-2.0], [0.0]]) + 0 * vy)
            else:
                assert np.all(st["vel"][0, ex] == 0.0) and np.all(st["vel"][2, ex] == 0.0) and np.all(vy < 0.0)
        gone = st["state"] == abi.DEM_STATE_NONEXISTENT
        assert np.all(st["pos"][:, gone] == 0.0)
    return s, seen_exit


@pytest.mark.parametrize("mass_outflow", [False, True])
def test_box_empties_through_outflow(mass_outflow):
    s, seen_exit = _run(mass_outflow)
    st = s.stats()
    assert seen_exit > 0
    assert st["n_outflow_removed"] > 0
    assert st["n_outflow_removed"] + st["n_normal"] + int((s.download_state()["state"] == 3).sum()) == 100
    assert st["n_rogue_removed"] == 0          # nothing leaks out as rogue


def test_adams_bashforth_and_no_bc_control():
    s, seen_exit = _run(False, intg="ADAMS_BASHFORTH")
    assert s.stats()["n_outflow_removed"] > 0
    # without the boundary the same particles leave as rogue particles
    case, prm, arr, walls, bc = outflow_case(False)
    t = make_system(OracleSystem, prm, arr, walls)
    t.step(400)
    assert t.stats()["n_outflow_removed"] == 0 and t.stats()["n_rogue_removed"] > 0


def test_rejects_overlapping_boxes():
    case, prm, arr, walls, bc = outflow_case(False)
    s = make_system(OracleSystem, prm, arr, walls)
    with pytest.raises(Exception):
        s.set_outflow_bcs([bc, bc])
