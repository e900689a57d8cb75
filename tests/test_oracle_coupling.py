"""CPU checks of the oracle's CFD-DEM coupling (GARG_2012 / Gidaspow / mean
fields) on small cases."""
import numpy as np

from cases import coupled_case, make_coupled
from oracle_ffi import OracleSystem


def test_mean_fields_are_physical_and_deterministic():
    ct = coupled_case()
    s = make_coupled(OracleSystem, ct)
    s.comp_mean_fields()
    ep, rop = s.get_mean_fields()
    case, prm, arr, walls, info, grid, fields = ct
    gi, gj, gk = grid.imax + 2, grid.jmax + 2, grid.kmax + 2
    ep3 = ep.reshape(gk, gj, gi)[1:-1, 1:-1, 1:-1]
    assert np.all(ep3 > 0.0) and np.all(ep3 <= 1.0)
    assert ep3.min() < 0.9            # the bed is there
    s2 = make_coupled(OracleSystem, ct)
    s2.comp_mean_fields()
    ep2, rop2 = s2.get_mean_fields()
    assert np.array_equal(ep, ep2) and np.array_equal(rop, rop2)


def test_drag_opposes_gravity():
    """The upward gas flow gives every particle an upward drag of the order of
    its weight (Gidaspow: Ergun in the bed, Wen-Yu above it)."""
    ct = coupled_case()
    case, prm, arr, walls, info, grid, fields = ct
    s = make_coupled(OracleSystem, ct)
    s.comp_mean_fields()
    s.calc_force()
    fc0, _ = s.download_forces()
    s.drag_gs_des0()
    fc1, _ = s.download_forces()
    drag_y = fc1[1] - fc0[1]
    weight = arr["pmass"] * 9.81
    assert np.all(drag_y > 0.0)
    assert 0.1 < drag_y.mean() / weight.mean() < 10.0
    s.cfnewvalues()
    s.step_coupled(5, 2)
