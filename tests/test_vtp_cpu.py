"""Particle output (.vtp) on the host: the file parsed back -- XML header,
appended big-endian Float32 arrays at the offsets the header states -- as
WRITE_VTP_FILE lays it out (model/des/vtp_mod.f:705-2906), and the VTK
region selection of SETUP_VTK_REGION_PARTICLES (vtp_mod.f:2925-3172)."""
import ctypes as C
import re
import struct

import numpy as np
import pytest

from mfix_dem import abi, load_library
from mfix_dem.system import _bp, _dp, _ip


def _write(path, pos, vel, omega, radius, state, phase, **kw):
    lib = load_library()
    o = abi.vtp_options(**kw)
    n = C.c_int64()
    rc = lib.dem_vtp_write(str(path).encode(), C.byref(o), len(radius), _dp(pos), _dp(vel), _dp(omega),
                           _dp(radius), _bp(state), _ip(phase), C.byref(n))
    assert rc == 0
    return int(n.value)


def _parse(path):
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b"<AppendedData encoding=\"raw\">\n_")
    text = head.decode()
    assert 'byte_order="BigEndian"' in text and 'type="PolyData"' in text
    npts = int(re.search(r'NumberOfPoints="(\d+)"', text).group(1))
    arrays = {}
    for m in re.finditer(r'<DataArray type="Float32" Name="([^"]+)"(?: NumberOfComponents="(\d)")? '
                         r'format="appended" offset="(\d+)"', text):
        name, nc, off = m.group(1), int(m.group(2) or 1), int(m.group(3))
        nbytes = struct.unpack(">i", rest[off:off + 4])[0]
        assert nbytes == 4 * nc * npts
        a = np.frombuffer(rest[off + 4:off + 4 + nbytes], dtype=">f4").astype(np.float32)
        arrays[name] = a.reshape(npts, nc) if nc > 1 else a
    assert rest.endswith(b"</AppendedData>\n</VTKFile>\n")
    return npts, arrays, text


def _case(n=500, seed=3):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1e-2, (3, n))
    vel = rng.normal(0, 0.2, (3, n))
    omega = rng.normal(0, 20.0, (3, n))
    radius = rng.uniform(2e-4, 5e-4, n)
    state = np.full(n, abi.DEM_STATE_NORMAL, np.int8)
    state[::17] = abi.DEM_STATE_NONEXISTENT
    state[5] = abi.DEM_STATE_NORMAL_GHOST
    state[6] = abi.DEM_STATE_ENTERING
    phase = rng.integers(1, 3, n).astype(np.int32)
    return pos, vel, omega, radius, state, phase


def test_whole_domain(tmp_path):
    pos, vel, omega, radius, state, phase = _case()
    path = tmp_path / "run_DES_00000.vtp"
    n = _write(path, pos, vel, omega, radius, state, phase, time=0.125, angular_velocity=True)
    sel = np.nonzero(state == 1)[0]
    npts, a, text = _parse(path)
    assert n == npts == len(sel)
    assert "Time = 0.125" in text
    assert np.array_equal(a["coordinates"], pos[:, sel].T.astype(np.float32))
    assert np.array_equal(a["Diameter"], (2.0 * radius[sel]).astype(np.float32))
    assert np.array_equal(a["Velocity"], vel[:, sel].T.astype(np.float32))
    assert np.array_equal(a["Angular_velocity"], omega[:, sel].T.astype(np.float32))
    # array order and offsets as the reference lays them out
    offs = [int(x) for x in re.findall(r'offset="(\d+)"', text)]
    assert offs == [0, 4 + 12 * npts, 8 + 16 * npts, 12 + 28 * npts]


@pytest.mark.parametrize("mode", ["C", "P", "I"])
def test_region_selection(tmp_path, mode):
    pos, vel, omega, radius, state, phase = _case()
    lo, hi = np.array([2e-3, 1e-3, 3e-3]), np.array([7e-3, 8e-3, 9e-3])
    path = tmp_path / f"r{mode}.vtp"
    n = _write(path, pos, vel, omega, radius, state, phase, box=(lo, hi), select_mode=mode, phases=[2])
    p1, p2 = pos - radius, pos + radius
    if mode == "C":
        inside = np.all((lo[:, None] <= pos) & (pos <= hi[:, None]), axis=0)
    elif mode == "P":
        inside = np.all((lo[:, None] <= p1) & (p2 <= hi[:, None]), axis=0)
    else:
        inside = np.all(~((hi[:, None] <= p1) | (p2 <= lo[:, None])), axis=0)
    sel = np.nonzero((state == 1) & (phase == 2) & inside)[0]
    npts, a, _ = _parse(path)
    assert n == npts == len(sel) > 0
    assert np.array_equal(a["coordinates"], pos[:, sel].T.astype(np.float32))
    assert "Angular_velocity" not in a


def test_empty(tmp_path):
    pos, vel, omega, radius, state, phase = _case(n=10)
    state[:] = abi.DEM_STATE_NONEXISTENT
    path = tmp_path / "e.vtp"
    assert _write(path, pos, vel, omega, radius, state, phase) == 0
    npts, a, _ = _parse(path)
    assert npts == 0 and a["Diameter"].size == 0
