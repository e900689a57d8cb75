"""Hopper cone walls on the GPU against the oracle.

Spheres placed against the slanted facets of a hopper-discharge case's cone
(tests/cases.py::hopper_wall_case) hit them within the first steps: the facet
binning of the cone to DES cells (TRI_BOX_OVERLAP, stl_preproc_des_mod.f:
135-349, stl_functions_des_mod.f:280-536), the closest-point contacts and
the per-particle facet history slots (GET/UPDATE/REMOVE_COLLISION,
calc_collision_wall_mod.f:651-792) must give the oracle's results bit for
bit: state, wall-history slots and their tangential histories, contact
counts.
"""
import numpy as np
import pytest

from cases import hopper_wall_case, make_system
from gpu_util import compare_pairs, compare_state

pytestmark = pytest.mark.gpu


def test_hopper_cone_walls_match_oracle():
    from mfix_dem import GpuSystem
    from oracle_ffi import OracleSystem
    case, prm, arr, walls = hopper_wall_case()
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    for _ in range(6):
        g.step(50); o.step(50)
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
        fg, pg = g.download_wall_history()
        fo, po = o.download_wall_history()
        assert np.array_equal(fg, fo)
        assert np.array_equal(pg, po)
        sg, so = g.stats(), o.stats()
        assert sg["n_wall_contacts"] == so["n_wall_contacts"]
        assert sg["n_contacts"] == so["n_contacts"]
    assert so["n_wall_contacts"] > 500


def test_hopper_cone_walls_split_precision():
    """The same spheres in split precision: the wall terms stay FP64 and the
    per-step force error against the FP64 path stays within 1e-5."""
    from mfix_dem import GpuSystem, abi
    case, prm, arr, walls = hopper_wall_case(precision=abi.DEM_PREC_SPLIT)
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    errs = []
    for _ in range(4):
        g.step(40)
        errs.append(g.force_error())
    assert max(errs) <= 1e-5, errs
    assert g.stats()["n_wall_contacts"] > 500
