"""Particle output through the handle: the .vtp of a stepped system holds
the device state of its NORMAL particles."""
import numpy as np
import pytest

from cases import make_system, settling_case
from test_vtp_cpu import _parse

pytestmark = pytest.mark.gpu


def test_write_vtp_matches_state(tmp_path):
    from mfix_dem import GpuSystem
    case, prm, arr, walls = settling_case(n_side=(6, 12, 6))
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    g.step(30)
    path = tmp_path / "settle_DES_00001.vtp"
    n = g.write_vtp(path, time=1.5, angular_velocity=True)
    st = g.download_state()
    sel = np.nonzero(st["state"] == 1)[0]
    npts, a, _ = _parse(path)
    assert n == npts == len(sel)
    assert np.array_equal(a["coordinates"], st["pos"][:, sel].T.astype(np.float32))
    assert np.array_equal(a["Velocity"], st["vel"][:, sel].T.astype(np.float32))
    assert np.array_equal(a["Angular_velocity"], st["omega"][:, sel].T.astype(np.float32))
    assert np.array_equal(a["Diameter"], (2.0 * arr["radius"][sel]).astype(np.float32))
