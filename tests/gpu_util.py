"""Helpers for the GPU parity tests (CUDA library vs the CPU oracle)."""
import numpy as np

from mfix_dem import GpuSystem
from oracle_ffi import OracleSystem
from cases import make_system

# Tolerance of the FP64 path against the oracle: per-particle positions and
# velocities within 1e-10 relative, measured normwise per array
# (max |a - b| / max |b|).  The FP64 kernels reproduce the serial reference's
# operation order, so the observed difference is normally exactly zero.
REL_TOL = 1e-10


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / scale)


def pair_both(prm, arr, walls):
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    return g, o


def compare_state(g, o, exact=False):
    sg, so = g.download_state(), o.download_state()
    errs = {k: rel_err(sg[k], so[k]) for k in ("pos", "vel", "omega")}
    assert np.array_equal(sg["state"], so["state"])
    if exact:
        for k in ("pos", "vel", "omega"):
            assert np.array_equal(sg[k], so[k]), (k, errs[k])
    for k, e in errs.items():
        assert e <= REL_TOL, (k, e)
    return errs


def compare_pairs(g, o):
    nig, nbg, pfg = g.download_pairs()
    nio, nbo, pfo = o.download_pairs()
    assert np.array_equal(nig, nio), "NEIGHBOR_INDEX differs"
    assert np.array_equal(nbg, nbo), "NEIGHBORS differs"
    return rel_err(pfg, pfo) if len(pfo) else 0.0
