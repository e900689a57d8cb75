"""Mass-inflow boundaries on the oracle (MASS_INFLOW_DEM, SEED_NEW_PARTICLE,
mass_inflow_dem.f): particles are seeded ENTERING in successive layout
windows at the boundary's rate, move with the boundary velocity and turn
NORMAL once clear of the plane by more than their radius."""
import numpy as np
import pytest

from cases import make_system
from mfix_dem import abi
from mfix_dem.system import DemError
from oracle_ffi import OracleSystem
from inflow_cases import inflow_case


def _injection_steps(dt, pi_factor, steps, mi_time=0.0):
    """The steps (0-based) at which MASS_INFLOW_DEM seeds, with the same
    floating-point updates of S_TIME and DEM_MI_TIME."""
    s_time, out = 0.0, []
    for k in range(steps):
        if not (mi_time > s_time):
            out.append(k)
            mi_time = mi_time + pi_factor * dt
        s_time = s_time + dt
    return out


def test_seeding_rate_windows_and_entering():
    case, prm, arr, walls, bc, _ = inflow_case()
    n0 = int((arr["state"] == abi.DEM_STATE_NORMAL).sum())
    s = make_system(OracleSystem, prm, arr, walls)
    s.set_inflow_bcs([bc], seed=5)
    steps = 500
    s.step(steps)
    inj = _injection_steps(prm.dtsolid, bc.pi_factor, steps)
    st = s.stats()
    assert st["n_inflow_added"] == 2 * len(inj)
    vac, mi_time = s.inflow_state(0)
    assert vac == (2 * len(inj)) % bc.occupants + 1
    assert mi_time == pytest.approx(len(inj) * bc.pi_factor * prm.dtsolid)
    d = s.download_state()
    new = np.arange(arr["pos"].shape[1]) >= n0
    seeded = new & (d["state"] != abi.DEM_STATE_NONEXISTENT)
    assert int(seeded.sum()) == 2 * len(inj)
    # the first free slots, in index order
    assert np.all(np.flatnonzero(seeded) == n0 + np.arange(2 * len(inj)))
    # ENTERING ones have not cleared the plane; NORMAL ones did
    top = case.domain_hi[1]
    r = 0.45e-3
    ent = d["state"] == abi.DEM_STATE_ENTERING
    nor = seeded & (d["state"] == abi.DEM_STATE_NORMAL)
    assert ent.any() and nor.any()
    # the test runs on the cells of the last DESGRID_PIC (every 10 steps here)
    assert np.all(d["pos"][1, ent] > top - r - 11 * 2.0 * prm.dtsolid - 1e-12)
    assert np.all(d["pos"][1, nor] < top - r)
    # ENTERING particles keep the boundary velocity
    assert np.all(d["vel"][:, ent] == np.array([[0.0], [-2.0], [0.0]]))
    # seeded inside the layout's band
    assert np.all(d["pos"][0, seeded] >= 0.5e-3 + r - 1e-12)
    assert np.all(d["pos"][0, seeded] <= case.domain_hi[0] - 0.5e-3 - r + 1e-12)


def test_queued_numbers_place_the_first_seeds():
    case, prm, arr, walls, bc, _ = inflow_case()
    n0 = int((arr["state"] == abi.DEM_STATE_NORMAL).sum())
    s = make_system(OracleSystem, prm, arr, walls)
    s.set_inflow_bcs([bc], seed=5)
    rnd = [0.25, 0.75, 0.5]
    s.push_inflow_random(rnd)
    s.step(1)
    d = s.download_state()
    P, Q, _ = bc._keep
    dd, w = 0.9e-3, bc.window
    for k in range(2):
        x = P[k] + (0.5 * dd + (w - dd) * rnd[0])
        z = Q[k] + (0.5 * dd + (w - dd) * rnd[1])
        # one step at the boundary velocity from the seeding plane
        assert d["pos"][0, n0 + k] == x and d["pos"][2, n0 + k] == z
        assert d["pos"][1, n0 + k] == pytest.approx(bc.offset, abs=1e-8)
        assert d["state"][n0 + k] == abi.DEM_STATE_ENTERING


def test_capacity_exhausted():
    case, prm, arr, walls, bc, _ = inflow_case(spare=3)
    s = make_system(OracleSystem, prm, arr, walls)
    s.set_inflow_bcs([bc])
    with pytest.raises(DemError) as e:
        s.step(30)
    assert e.value.code == abi.DEM_ERR_CAPACITY


def test_bad_arguments():
    case, prm, arr, walls, bc, _ = inflow_case()
    s = make_system(OracleSystem, prm, arr, walls)
    bc.vacancy = 0
    with pytest.raises(DemError):
        s.set_inflow_bcs([bc])
    bc.vacancy = 1
    bc.plane = ord("Q")
    with pytest.raises(DemError):
        s.set_inflow_bcs([bc])


def test_inflow_with_outflow_floor_conserves_count():
    case, prm, arr, walls, bc, obc = inflow_case(outflow=True, spare=200)
    n0 = int((arr["state"] == abi.DEM_STATE_NORMAL).sum())
    s = make_system(OracleSystem, prm, arr, walls)
    s.set_inflow_bcs([bc], seed=3)
    s.set_outflow_bcs([obc])
    s.step(400)
    st = s.stats()
    d = s.download_state()
    alive = int((d["state"] != abi.DEM_STATE_NONEXISTENT).sum())
    assert st["n_inflow_added"] > 0 and st["n_outflow_removed"] > 0
    assert alive == n0 + st["n_inflow_added"] - st["n_outflow_removed"] - st["n_rogue_removed"]
