"""The DEM restart-file (RES) codec on the host: the records against a
plain restatement of WRITE_RES0_DES's layout (model/des/write_res0_des.f:44-208,
write_res1_des_mod.f, out_bin_512.f, out_bin_512i.f), and the round trip.
No device is needed: dem_res_write / dem_res_read are host code of the
library."""
import math
import struct

import numpy as np
import pytest

from mfix_dem import abi, load_library
from mfix_dem.restart import res_read, res_write

REC = 512


def _case(n=300, seed=5, no_k=False):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1e-2, (3, n))
    vel = rng.normal(0, 0.1, (3, n))
    omega = rng.normal(0, 10.0, (3, n))
    if no_k:
        pos[2] = 0.5e-3; vel[2] = 0.0; omega[:2] = 0.0
    radius = rng.uniform(4e-4, 6e-4, n)
    state = np.full(n, abi.DEM_STATE_NORMAL, np.int8)
    state[[q for q in (3, 50, 51, 299) if q < n]] = abi.DEM_STATE_NONEXISTENT
    state[7] = abi.DEM_STATE_NORMAL_GHOST
    state[11] = abi.DEM_STATE_EXITING
    phase = rng.integers(1, 3, n).astype(np.int32)
    # a CSR pair list with empty rows and entries that touch removed slots
    rows = [sorted(set(rng.integers(0, n, rng.integers(0, 5)).tolist())) if i % 7 else [] for i in range(n)]
    nb = np.array([j + 1 for r in rows for j in r], np.int32)
    ends = np.cumsum([len(r) for r in rows]).astype(np.int32) + 1
    pft = rng.normal(0, 1e-6, (len(nb), 3))
    return pos, vel, omega, radius, state, phase, ends, nb, pft, rows


def _info(ro=(2500.0, 1200.0)):
    info = abi.DemResInfo()
    info.vtp_findex, info.tecplot_findex, info.dtsolid = 17, 3, 2.5e-6
    for m, r in enumerate(ro):
        info.ro_sol[m] = r
    return info


def _records(path):
    raw = open(path, "rb").read()
    assert len(raw) % REC == 0
    return [raw[i:i + REC] for i in range(0, len(raw), REC)]


class _Reader:
    """WRITE_RES0_DES read back record by record (serial layout)."""

    def __init__(self, recs):
        self.recs, self.k = recs, 0

    def _next(self):
        r = self.recs[self.k]
        self.k += 1
        return r

    def i(self):
        return struct.unpack(">i", self._next()[:4])[0]

    def d(self):
        return struct.unpack(">d", self._next()[:8])[0]

    def arr(self, n, kind):
        w, fmt = (64, ">d") if kind == "d" else (128, ">i")
        size = struct.calcsize(fmt)
        out = []
        nrec = max(1, math.ceil(n / w))
        for r in range(nrec):
            rec = self._next()
            m = min(w, n - r * w)
            out += [struct.unpack(fmt, rec[size * q:size * (q + 1)])[0] for q in range(m)]
            assert rec[size * m:] == bytes(REC - size * m)       # padding
        return np.array(out)


@pytest.mark.parametrize("no_k", [False, True])
def test_records_follow_write_res0_des(tmp_path, no_k):
    lib = load_library()
    pos, vel, omega, radius, state, phase, ends, nb, pft, rows = _case(no_k=no_k)
    n = len(radius)
    path = tmp_path / "case_DES.RES"
    info = _info()
    res_write(lib, path, info, no_k, pos, vel, omega, radius, state, phase, ends, nb, pft)
    r = _Reader(_records(path))
    exists = (state != 0) & (state < 101)
    slots = np.nonzero(exists)[0]
    keep = [(i, j) for i, row in enumerate(rows) for j in row if exists[i] and exists[j]]
    flat = [(i, j, c) for c, (i, j) in enumerate((i, j) for i, row in enumerate(rows) for j in row)]
    kept = [c for i, j, c in flat if exists[i] and exists[j]]
    dimn = 2 if no_k else 3
    assert r.d() == float(np.float32(1.2))             # VERSION = 1.2 (a REAL(4) literal)
    assert r.i() == len(slots)                          # particles
    assert r.i() == 0                                   # ghosts
    assert r.i() == len(keep)                           # pairs
    assert (r.i(), r.i(), r.d()) == (17, 3, 2.5e-6)     # VTP_FINDEX, TECPLOT_FINDEX, DTSOLID
    for c in range(dimn):
        assert np.array_equal(r.arr(len(slots), "d"), pos[c, slots])
    assert np.array_equal(r.arr(len(slots), "i"), slots + 1)         # iGLOBAL_ID
    assert np.array_equal(r.arr(len(slots), "i"), state[slots])
    for c in range(dimn):
        assert np.array_equal(r.arr(len(slots), "d"), vel[c, slots])
    for c in range(1 if no_k else 3):                    # OMEGA_NEW(:,1) only in 2D
        assert np.array_equal(r.arr(len(slots), "d"), omega[c, slots])
    assert np.array_equal(r.arr(len(slots), "d"), radius[slots])
    assert np.array_equal(r.arr(len(slots), "d"), np.array([2500.0, 1200.0])[phase[slots] - 1])
    assert np.array_equal(r.arr(len(slots), "i"), phase[slots])      # PIJK(:,5)
    assert r.i() == 0                                                 # DES_USR_VAR_SIZE
    assert np.array_equal(r.arr(len(slots), "d"), np.zeros(len(slots)))   # RESIDENCE_TIME
    assert np.array_equal(r.arr(len(keep), "i"), [j + 1 for _, j in keep])   # NEIGHBORS (global ids)
    assert np.array_equal(r.arr(len(keep), "i"), [i + 1 for i, _ in keep])   # owners
    for c in range(dimn):
        assert np.array_equal(r.arr(len(keep), "d"), pft[kept, c])
    assert r.i() == 0                                                 # DEM_BCMI
    assert r.k == len(r.recs)


def test_round_trip_packs_particles_and_maps_pairs(tmp_path):
    lib = load_library()
    pos, vel, omega, radius, state, phase, ends, nb, pft, rows = _case()
    path = tmp_path / "rt_DES.RES"
    res_write(lib, path, _info(), False, pos, vel, omega, radius, state, phase, ends, nb, pft)
    out = res_read(lib, path, 320, False)
    exists = (state != 0) & (state < 101)
    slots = np.nonzero(exists)[0]
    m = len(slots)
    assert out["info"].n_particles == m and out["info"].dtsolid == 2.5e-6
    for k, a in (("pos", pos), ("vel", vel), ("omega", omega)):
        assert np.array_equal(out[k][:, :m], a[:, slots])
        assert not out[k][:, m:].any()
    assert np.array_equal(out["radius"][:m], radius[slots])
    assert np.array_equal(out["state"][:m], state[slots]) and not out["state"][m:].any()
    assert np.array_equal(out["phase"][:m], phase[slots])
    new_of = {int(s) + 1: q + 1 for q, s in enumerate(slots)}
    keep = [(i, j, c) for c, (i, j) in enumerate((i, j) for i, row in enumerate(rows) for j in row)
            if exists[i] and exists[j]]
    assert np.array_equal(out["owner"], [new_of[i + 1] for i, _, _ in keep])
    assert np.array_equal(out["neighbor"], [new_of[j + 1] for _, j, _ in keep])
    assert np.array_equal(out["pft"], pft[[c for _, _, c in keep]])


def test_reader_rejects_old_versions_and_small_capacity(tmp_path):
    lib = load_library()
    pos, vel, omega, radius, state, phase, ends, nb, pft, rows = _case(n=40)
    path = tmp_path / "v_DES.RES"
    res_write(lib, path, _info(), False, pos, vel, omega, radius, state, phase, ends, nb, pft)
    with pytest.raises(OSError):
        res_read(lib, path, 10, False)                  # more particles than slots
    raw = bytearray(open(path, "rb").read())
    raw[:8] = struct.pack(">d", 1.1)                    # before PIJK(:,5) was stored
    open(path, "wb").write(bytes(raw))
    with pytest.raises(OSError):
        res_read(lib, path, 40, False)


def test_empty_system(tmp_path):
    lib = load_library()
    n = 5
    z = np.zeros((3, n))
    st = np.zeros(n, np.int8)
    path = tmp_path / "e_DES.RES"
    res_write(lib, path, _info(), False, z, z, z, np.zeros(n), st, np.ones(n, np.int32),
              np.ones(n, np.int32), np.zeros(0, np.int32), np.zeros((0, 3)))
    recs = _records(path)
    # header 7 records, 3+1+1+3+3+1+1+1 arrays of one record each, 1 scalar,
    # 1 array, 2+3 pair arrays, 1 scalar
    assert len(recs) == 7 + 14 + 1 + 1 + 5 + 1
    out = res_read(lib, path, n, False)
    assert out["info"].n_particles == 0 and out["info"].n_pairs == 0
