"""Restart: whole-state snapshots of a system and the RES record codec.

`snapshot` / `restore` carry everything a DEM step depends on -- particle
state, the pair list with PFT_NEIGHBOR, the wall-contact history and the
Adams-Bashforth history -- through the C ABI's download/upload calls, so a
restored system continues bit for bit.  The RES file (`write_res0_des` on a
system, `res_write` / `res_read` here on host arrays) is the reference's
restart format (model/des/write_res0_des.f), which holds particles and pairs
but neither of the two histories.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .system import DemSystem, _bp, _dp, _ip


def snapshot(s: DemSystem, first_pass: bool = False) -> dict:
    """Everything `restore` needs, as host arrays.  Take it after a step whose
    NN is a multiple of NEIGHBOR_SEARCH_N (or any step with a periodic axis):
    the pair list and the DES cells then describe the current positions, as
    they do when the reference restarts (MAKE_ARRAYS_DES rebuilds both).
    first_pass is the Adams-Bashforth FIRST_PASS flag (False once stepped)."""
    st = s.download_state()
    ni, nb, pf = s.download_pairs()
    fid, wpf = s.download_wall_history()
    acc, racc = s.get_ab2_history()
    return {"state": st, "pairs": (ni, nb, pf), "walls": (fid, wpf), "ab2": (acc, racc, first_pass),
            "nn": s.nn}


def restore(s: DemSystem, snap: dict, radius, pmass, omoi, phase) -> DemSystem:
    """Loads a snapshot into a system created with the same parameters and
    walls; radius/pmass/omoi/phase are the constant particle arrays."""
    st = snap["state"]
    s.upload_state(st["pos"], st["vel"], st["omega"], radius, pmass, omoi, st["state"], phase)
    s.desgrid_pic()
    s.upload_pairs(*snap["pairs"])
    s.upload_wall_history(*snap["walls"])
    acc, racc, first = snap["ab2"]
    s.set_ab2_history(acc, racc, first_pass=first)
    s.nn = snap["nn"]
    return s


def res_write(lib, path, info: abi.DemResInfo, no_k: bool, pos, vel, omega, radius, state, phase,
              neighbor_index=None, neighbors=None, pft=None):
    """The RES codec on host arrays (DES arrays in Fortran layout)."""
    n = int(np.asarray(radius).shape[0])
    f = lambda a, sh: np.ascontiguousarray(a, dtype=np.float64).reshape(sh)  # noqa: E731
    pos, vel, omega = f(pos, (3, n)), f(vel, (3, n)), f(omega, (3, n))
    radius = f(radius, (n,))
    state = np.ascontiguousarray(state, dtype=np.int8)
    phase = np.ascontiguousarray(phase, dtype=np.int32)
    P = 0 if neighbors is None else int(len(neighbors))
    ni = None if neighbor_index is None else np.ascontiguousarray(neighbor_index, dtype=np.int32)
    nb = None if neighbors is None else np.ascontiguousarray(neighbors, dtype=np.int32)
    pf = None if pft is None else f(pft, (max(P, 0), 3))
    rc = lib.dem_res_write(str(path).encode(), C.byref(info), n, 1 if no_k else 0, _dp(pos), _dp(vel), _dp(omega),
                           _dp(radius), _bp(state), _ip(phase), _ip(ni), _ip(nb), _dp(pf), P)
    if rc:
        raise OSError(f"dem_res_write failed ({abi.ERROR_NAMES.get(rc, rc)})")


def res_read(lib, path, max_pip: int, no_k: bool, pairs: bool = True) -> dict:
    """Reads a RES file into max_pip slots; returns the arrays, the info and,
    with pairs, (owner, neighbour) 1-based local indices and PFT (P,3)."""
    info = abi.DemResInfo()
    rc = lib.dem_res_read(str(path).encode(), C.byref(info), 0, 1 if no_k else 0, *([None] * 10), 0)
    if rc:
        raise OSError(f"dem_res_read failed ({abi.ERROR_NAMES.get(rc, rc)})")
    n, P = int(max_pip), int(info.n_pairs)
    out = {k: np.zeros((3, n)) for k in ("pos", "vel", "omega")}
    out.update(radius=np.zeros(n), ro_sol=np.zeros(n), state=np.zeros(n, np.int8), phase=np.zeros(n, np.int32))
    own = np.zeros(max(P, 1), np.int32) if pairs else None
    nbr = np.zeros(max(P, 1), np.int32)
    pft = np.zeros((max(P, 1), 3))
    rc = lib.dem_res_read(str(path).encode(), C.byref(info), n, 1 if no_k else 0, _dp(out["pos"]), _dp(out["vel"]),
                          _dp(out["omega"]), _dp(out["radius"]), _dp(out["ro_sol"]), _bp(out["state"]),
                          _ip(out["phase"]), _ip(own), _ip(nbr), _dp(pft), max(P, 1))
    if rc:
        raise OSError(f"dem_res_read failed ({abi.ERROR_NAMES.get(rc, rc)})")
    out["info"] = info
    if pairs:
        out["owner"], out["neighbor"], out["pft"] = own[:P].copy(), nbr[:P].copy(), pft[:P].copy()
    return out


def res_read_inflow(lib, path, no_k: bool, max_bc: int = 8, max_occ: int = 4096) -> list:
    """The mass-inflow records at the end of a RES file: one dict per
    boundary with mi_time, vacancy, occupants, window, offset, l_index and
    the W, H, P, Q arrays."""
    mi = (abi.DemResInflow * max(max_bc, 1))()
    nbc = C.c_int32()
    w = np.zeros((max_bc, max_occ), np.int32)
    hh = np.zeros((max_bc, max_occ), np.int32)
    p = np.zeros((max_bc, max_occ))
    q = np.zeros((max_bc, max_occ))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rc = lib.dem_res_read_inflow(str(path).encode(), 1 if no_k else 0, C.byref(nbc), C.cast(mi, C.c_void_p),
                                 max_bc, ip(w), ip(hh), dp(p), dp(q), max_occ)
    if rc:
        raise OSError(f"dem_res_read_inflow failed ({abi.ERROR_NAMES.get(rc, rc)})")
    out = []
    for b in range(min(nbc.value, max_bc)):
        r = mi[b]
        o = int(r.occupants)
        out.append(dict(mi_time=r.mi_time, vacancy=r.vacancy, occupants=o, window=r.window, offset=r.offset,
                        l_index=r.l_index, w=w[b, :o].copy(), h=hh[b, :o].copy(), p=p[b, :o].copy(),
                        q=q[b, :o].copy()))
    return out
