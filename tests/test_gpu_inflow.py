"""Mass-inflow boundaries on the GPU against the oracle: seeded particles,
states, positions, velocities and pair lists bit for bit while a box fills
through its top (MASS_INFLOW_DEM), alone and with an outflow floor."""
import numpy as np
import pytest

from cases import make_system
from gpu_util import compare_pairs, compare_state
from inflow_cases import inflow_case

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
