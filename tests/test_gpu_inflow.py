"""Mass-inflow boundaries on the GPU against the oracle: seeded particles,
states, positions, velocities and pair lists bit for bit while a box fills
through its top (MASS_INFLOW_DEM), alone and with an outflow floor."""
import numpy as np
import pytest

from cases import make_system
from gpu_util import compare_pairs, compare_state
from inflow_cases import inflow_case
from mfix_dem import abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("intg,outflow", [("EULER", False), ("ADAMS_BASHFORTH", False), ("EULER", True),
                                          ("ADAMS_BASHFORTH", True)])
def test_inflow_matches_oracle(intg, outflow):
    from mfix_dem import GpuSystem
    from oracle_ffi import OracleSystem
    case, prm, arr, walls, bc, obc = inflow_case(intg=intg, outflow=outflow, spare=220)
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    g.set_inflow_bcs([bc], seed=9)
    o.set_inflow_bcs([bc], seed=9)
    if outflow:
        g.set_outflow_bcs([obc]); o.set_outflow_bcs([obc])
    for _ in range(5):
        g.step(100); o.step(100)
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
        assert g.inflow_state(0) == o.inflow_state(0)
    sg, so = g.stats(), o.stats()
    assert sg["n_inflow_added"] == so["n_inflow_added"] > 0
    assert sg["n_outflow_removed"] == so["n_outflow_removed"]
    if outflow:
        assert sg["n_outflow_removed"] > 0


def test_queued_numbers_match_oracle():
    from mfix_dem import GpuSystem
    from oracle_ffi import OracleSystem
    case, prm, arr, walls, bc, _ = inflow_case()
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    rnd = np.random.default_rng(4).random(3 * 40)
    for s in (g, o):
        s.set_inflow_bcs([bc], seed=1)
        s.push_inflow_random(rnd)
    g.step(60); o.step(60)
    compare_state(g, o, exact=True)
    assert g.stats()["n_inflow_added"] == o.stats()["n_inflow_added"] > 0


def test_restart_file_carries_the_inflow_state(tmp_path):
    """dem_write_res0_des writes the inflow records (DEM_MI_TIME, VACANCY and
    the layout); dem_read_res0_des into a handle with the same boundaries
    installed restores DEM_MI_TIME and VACANCY.  (The uniform numbers the
    boundaries draw are not part of the file: a restarted run seeds from its
    own generator or from the numbers its driver queues.)  A file without the
    inflow section, read into a handle with inflow boundaries, is refused."""
    from mfix_dem import GpuSystem
    from mfix_dem import restart
    from mfix_dem._lib import load
    case, prm, arr, walls, bc, _ = inflow_case()
    a = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    a.set_inflow_bcs([bc], seed=2)
    a.step(60)
    path = tmp_path / "inflow.RES"
    a.write_res0_des(path, ro_sol=[case.ro_s0[0]])
    rec = restart.res_read_inflow(load(), path, no_k=False)
    vac, mi_time = a.inflow_state(0)
    assert len(rec) == 1 and rec[0]["vacancy"] == vac and rec[0]["mi_time"] == mi_time
    P, Q, _ = bc._keep
    assert np.array_equal(rec[0]["p"], P) and np.array_equal(rec[0]["q"], Q)
    assert rec[0]["occupants"] == bc.occupants and rec[0]["window"] == bc.window
    b = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    b.set_inflow_bcs([bc], seed=2)
    b.read_res0_des(path, restore_pairs=True)
    assert b.inflow_state(0) == (vac, mi_time)
    # a file written by a handle with no inflow boundaries (DEM_BCMI = 0)
    from mfix_dem.system import DemError
    c = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    plain = tmp_path / "plain.RES"
    c.write_res0_des(plain, ro_sol=[case.ro_s0[0]])
    with pytest.raises(DemError) as e:
        b.read_res0_des(plain, restore_pairs=True)
    assert e.value.code == abi.DEM_ERR_STATE
    assert b.inflow_state(0) == (vac, mi_time)
