"""dem_get_stats_noalloc against dem_get_stats.

The no-allocation entry point keeps its partial sums in a static device
array shared by every call on the device; two calls in a row must each give
the statistics of dem_get_stats (same kernels, same block-ordered sums, so
the agreement is expected to be exact; the test allows 1e-12 relative).
"""
import numpy as np
import pytest

from mfix_dem import GpuSystem
from cases import settling_case, make_system

pytestmark = pytest.mark.gpu

TOL = 1e-12
KEYS_EXACT = ("n_normal", "n_pairs", "n_contacts", "n_wall_contacts", "n_rogue_removed", "steps_done")
KEYS_FLOAT = ("mean_vel", "gran_temp", "kinetic_energy", "bed_height", "s_time")


def _check(a, b):
    for k in KEYS_EXACT:
        assert a[k] == b[k], (k, a[k], b[k])
    for k in KEYS_FLOAT:
        x = np.atleast_1d(np.asarray(a[k], dtype=np.float64))
        y = np.atleast_1d(np.asarray(b[k], dtype=np.float64))
        scale = max(float(np.max(np.abs(y))), 1e-300)
        assert float(np.max(np.abs(x - y))) <= TOL * scale, (k, x, y)


def test_noalloc_stats_match_get_stats_twice():
    # 16,000 spheres in contact with the walls and with each other: 63
    # partial-sum blocks, so the block-ordered total is exercised
    case, prm, arr, walls = settling_case(n_side=(20, 40, 20), spacing=0.98, jitter=0.03,
                                        box=(22e-3, 60e-3, 22e-3))
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    g.step(5)
    ref = g.stats()
    assert ref["n_normal"] == arr["pos"].shape[1]
    assert ref["n_contacts"] > 0 and ref["kinetic_energy"] > 0
    first = g.stats_noalloc()
    second = g.stats_noalloc()
    _check(first, ref)
    _check(second, ref)
    # after more steps the shared scratch holds the previous call's sums;
    # the next two calls must still follow the new state
    g.step(5)
    ref2 = g.stats()
    assert ref2["kinetic_energy"] != ref["kinetic_energy"]
    _check(g.stats_noalloc(), ref2)
    _check(g.stats_noalloc(), ref2)
    g.close()
