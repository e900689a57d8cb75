"""Split-precision path (FP32 contact forces, FP64 history and integration)
against the FP64 path and the oracle.

Tolerances: the per-step force error max|F_split - F_fp64| / max|F_fp64| must
stay at or below 1e-5; trajectories of a contact-dense bed must stay within
1e-6 relative of the FP64 oracle over 30 steps; pair lists are identical
(they do not depend on the force precision).
"""
import numpy as np
import pytest

from cases import settling_case, make_system
from gpu_util import compare_pairs, rel_err

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _gpu(prm, arr, walls):
    from mfix_dem import GpuSystem
    return make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)


@pytest.mark.parametrize("coll", ["LSD", "HERTZ"])
def test_split_force_error_within_tolerance(coll):
    from mfix_dem import abi
    case, prm, arr, walls = settling_case(n_side=(8, 12, 8), spacing=0.97, jitter=0.02, coll=coll,
                                          mew_r=0.02, polydisperse=0.0, vmax=0.3,
                                          precision=abi.DEM_PREC_SPLIT)
    g = _gpu(prm, arr, walls)
    errs = []
    for _ in range(5):
        errs.append(g.force_error())
        g.step(7)
    assert max(errs) <= FORCE_TOL, errs
    assert g.stats()["n_contacts"] > 0


def test_split_trajectory_tracks_fp64_oracle():
    from mfix_dem import abi
    from oracle_ffi import OracleSystem
    case, prm, arr, walls = settling_case(n_side=(8, 12, 8), spacing=0.97, jitter=0.02, coll="HERTZ",
                                          polydisperse=0.0, precision=abi.DEM_PREC_SPLIT, nsn=10)
    g = _gpu(prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)  # the oracle is FP64 whatever the flag says
    g.step(30); o.step(30)
    sg, so = g.download_state(), o.download_state()
    assert rel_err(sg["pos"], so["pos"]) <= 1e-6
    assert rel_err(sg["vel"], so["vel"]) <= 1e-3
    compare_pairs(g, o)
