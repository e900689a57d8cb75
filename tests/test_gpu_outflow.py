"""Outflow boundaries on the GPU against the oracle: states, positions,
velocities and pair lists bit for bit while the box empties through its
floor (MASS_OUTFLOW_DEM, UPDATE_EXIT_DES_VEL)."""
import numpy as np
import pytest

from cases import make_system
from gpu_util import compare_pairs, compare_state
from outflow_cases import outflow_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mass_outflow,intg", [(False, "EULER"), (True, "EULER"), (False, "ADAMS_BASHFORTH"),
                                               (True, "ADAMS_BASHFORTH")])
def test_outflow_matches_oracle(mass_outflow, intg):
    from mfix_dem import GpuSystem
    from oracle_ffi import OracleSystem
    case, prm, arr, walls, bc = outflow_case(mass_outflow, intg=intg)
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    g.set_outflow_bcs([bc]); o.set_outflow_bcs([bc])
    for _ in range(4):
        g.step(100); o.step(100)
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
    sg, so = g.stats(), o.stats()
    assert sg["n_outflow_removed"] == so["n_outflow_removed"] > 0
    assert sg["n_rogue_removed"] == so["n_rogue_removed"] == 0
