"""Host-side mirror of the DES_TIME_STEP call sequence over the C ABI.

`DemSystem` wraps one dem_handle of the CUDA library (include/dem_b200.h).
Its methods are named after the reference routines they replace
(model/des/des_time_march.f:293-460) and take/return numpy arrays in the
Fortran layouts of the DES arrays: per-particle vectors are (3, MAX_PIP)
arrays whose memory is the (MAX_PIP,3) column-major Fortran array, indices
are 1-based where the reference stores indices.

The same class drives any library that exports the ABI under another
prefix (the test suite points it at the CPU restatement with prefix "orc_").
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import abi


class DemError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        self.code = code
        name = abi.ERROR_NAMES.get(code, str(code))
        super().__init__(f"{where}: {name}: {msg}")


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


def _bp(a):
    return a.ctypes.data_as(C.POINTER(C.c_int8)) if a is not None else None


def _f64(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


class DemSystem:
    """One DEM case resident on the device (or in the CPU restatement)."""

    def __init__(self, lib, params: abi.DemParams, max_pip: int, prefix: str = "dem_"):
        self._lib = lib
        self._pre = prefix
        self.params = params
        self.n = int(max_pip)
        h = C.c_void_p()
        self._call("create", C.byref(params), C.c_int32(self.n), C.byref(h))
        self._h = h
        self.nn = 0  # last DES_TIME_STEP index executed

    # ------------------------------------------------------------------
    def _fn(self, name):
        return getattr(self._lib, self._pre + name)

    def _call(self, name, *args):
        rc = self._fn(name)(*args)
        if rc != 0:
            msg = ""
            if getattr(self, "_h", None) is not None:
                raw = self._fn("last_error")(self._h)
                msg = raw.decode() if raw else ""
            raise DemError(rc, self._pre + name, msg)
        return rc

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._fn("destroy")(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------
    def set_walls(self, vertex: np.ndarray, norm_face: np.ndarray):
        """VERTEX(3,3,F) as a (F,3,3) [f,c,v] array, NORM_FACE(3,F) as (F,3)."""
        vertex = np.ascontiguousarray(vertex, dtype=np.float64)
        norm_face = np.ascontiguousarray(norm_face, dtype=np.float64)
        nf = vertex.shape[0]
        self._call("set_walls", self._h, _dp(vertex), _dp(norm_face), C.c_int32(nf))

    def upload_state(self, pos, vel, omega, radius=None, pmass=None, omoi=None, state=None, phase=None):
        """dem_upload_state; after a first full upload, radius, pmass, omoi,
        state and phase may be None (the handle keeps its own)."""
        n = self.n
        pos = _f64(pos, (3, n)); vel = _f64(vel, (3, n)); omega = _f64(omega, (3, n))
        radius = None if radius is None else _f64(radius, (n,))
        pmass = None if pmass is None else _f64(pmass, (n,))
        omoi = None if omoi is None else _f64(omoi, (n,))
        state = None if state is None else np.ascontiguousarray(state, dtype=np.int8)
        phase = None if phase is None else np.ascontiguousarray(phase, dtype=np.int32)
        self._call("upload_state", self._h, _dp(pos), _dp(vel), _dp(omega), _dp(radius), _dp(pmass), _dp(omoi),
                   _bp(state), _ip(phase), C.c_int32(n))

    def download_state(self, out=None):
        """DES_POS_NEW, DES_VEL_NEW, OMEGA_NEW, PARTICLE_STATE; `out` may hold
        preallocated (e.g. pinned) arrays under the same keys."""
        n = self.n
        if out is not None:
            pos, vel, omega, state = out["pos"], out["vel"], out["omega"], out["state"]
        else:
            pos = np.empty((3, n)); vel = np.empty((3, n)); omega = np.empty((3, n))
            state = np.empty(n, dtype=np.int8)
        self._call("download_state", self._h, _dp(pos), _dp(vel), _dp(omega), _bp(state), C.c_int32(n))
        return {"pos": pos, "vel": vel, "omega": omega, "state": state}

    def download_forces(self):
        n = self.n
        fc = np.empty((3, n)); tow = np.empty((3, n))
        self._call("download_forces", self._h, _dp(fc), _dp(tow), C.c_int32(n))
        return fc, tow

    def set_ab2_history(self, acc_old=None, rot_acc_old=None, first_pass=True):
        n = self.n
        a = None if acc_old is None else _f64(acc_old, (3, n))
        r = None if rot_acc_old is None else _f64(rot_acc_old, (3, n))
        self._call("set_ab2_history", self._h, _dp(a), _dp(r), C.c_int32(1 if first_pass else 0), C.c_int32(n))

    def get_ab2_history(self):
        n = self.n
        a = np.empty((3, n)); r = np.empty((3, n))
        self._call("get_ab2_history", self._h, _dp(a), _dp(r), C.c_int32(n))
        return a, r

    def pair_count(self) -> int:
        v = C.c_int64()
        self._call("pair_count", self._h, C.byref(v))
        return int(v.value)

    def download_pairs(self):
        """NEIGHBOR_INDEX (1-based end pointers), NEIGHBORS (1-based), PFT (P,3)."""
        n = self.n
        P = self.pair_count()
        ni = np.empty(n, dtype=np.int32)
        nb = np.empty(max(P, 1), dtype=np.int32)
        pf = np.empty((max(P, 1), 3))
        self._call("download_pairs", self._h, _ip(ni), _ip(nb), _dp(pf), C.c_int64(max(P, 1)), C.c_int32(n))
        return ni, nb[:P].copy(), pf[:P].copy()

    def upload_pairs(self, neighbor_index, neighbors, pft):
        n = self.n
        ni = np.ascontiguousarray(neighbor_index, dtype=np.int32)
        nb = np.ascontiguousarray(neighbors, dtype=np.int32)
        pf = np.ascontiguousarray(pft, dtype=np.float64).reshape(-1, 3)
        P = nb.shape[0]
        self._call("upload_pairs", self._h, _ip(ni), _ip(nb), _dp(pf), C.c_int64(P), C.c_int32(n))

    def download_wall_history(self):
        n = self.n
        cm = self.params.collision_array_max or 8
        fid = np.empty((n, cm), dtype=np.int32)
        pf = np.empty((n, cm, 3))
        self._call("download_wall_history", self._h, _ip(fid), _dp(pf), C.c_int32(n))
        return fid, pf

    def upload_wall_history(self, facet_id, pft):
        n = self.n
        cm = self.params.collision_array_max or 8
        fid = np.ascontiguousarray(facet_id, dtype=np.int32).reshape(n, cm)
        pf = np.ascontiguousarray(pft, dtype=np.float64).reshape(n, cm, 3)
        self._call("upload_wall_history", self._h, _ip(fid), _dp(pf), C.c_int32(n))

    def set_outflow_bcs(self, bcs):
        """The DEM outflow boundaries (abi.DemOutflowBC, e.g. from
        params.outflow_bc); an empty list removes them."""
        arr = (abi.DemOutflowBC * max(len(bcs), 1))(*bcs)
        self._call("set_outflow_bcs", self._h, C.cast(arr, C.c_void_p), C.c_int32(len(bcs)))

    def set_inflow_bcs(self, bcs, seed: int = 0):
        """The DEM mass-inflow boundaries (abi.DemInflowBC, e.g. from
        params.inflow_bc); `seed` starts the handle's generator of the
        uniform numbers MASS_INFLOW_DEM draws.  An empty list removes them."""
        arr = (abi.DemInflowBC * max(len(bcs), 1))(*bcs)
        self._call("set_inflow_bcs", self._h, C.cast(arr, C.c_void_p), C.c_int32(len(bcs)), C.c_uint64(seed))

    def push_inflow_random(self, r):
        """Queue uniform numbers for the inflow boundaries (three per
        boundary per step, in boundary order), used before the generator."""
        a = np.ascontiguousarray(r, dtype=np.float64).ravel()
        self._call("push_inflow_random", self._h, _dp(a), C.c_int64(a.size))

    def inflow_state(self, bc: int):
        """(DEM_MI%VACANCY, DEM_MI_TIME) of inflow boundary `bc` (0-based)."""
        v = C.c_int32()
        t = C.c_double()
        self._call("get_inflow_state", self._h, C.c_int32(bc), C.byref(v), C.byref(t))
        return int(v.value), float(t.value)

    def download_cells(self):
        cells = np.empty(self.n, dtype=np.int32)
        self._call("download_cells", self._h, _ip(cells), C.c_int32(self.n))
        return cells

    # ---- stages ------------------------------------------------------
    def desgrid_pic(self):
        self._call("desgrid_pic", self._h)

    def neighbour(self):
        self._call("neighbour", self._h)

    def calc_force(self):
        self._call("calc_force", self._h)

    def cfnewvalues(self):
        self._call("cfnewvalues", self._h)

    def init_neighbors(self):
        """MAKE_ARRAYS_DES tail: DESGRID_PIC + NEIGHBOUR on the uploaded state."""
        self._call("init_neighbors", self._h)

    def set_dtsolid(self, dt: float):
        """DTSOLID of the following steps (a coupled driver's shortened last
        DEM step of a fluid step, and its restore)."""
        self._call("set_dtsolid", self._h, C.c_double(float(dt)))

    def step(self, nsteps: int = 1, nn_first: Optional[int] = None):
        """DES_TIME_STEP(NN) for the next nsteps values of NN."""
        first = self.nn + 1 if nn_first is None else nn_first
        self._call("step", self._h, C.c_int32(first), C.c_int32(nsteps))
        self.nn = first + nsteps - 1

    def stats(self) -> dict:
        s = abi.DemStats()
        self._call("get_stats", self._h, C.byref(s))
        return s.as_dict()

    def stats_noalloc(self) -> dict:
        """Same statistics through dem_get_stats_noalloc (static scratch,
        no allocation; CUDA library only)."""
        s = abi.DemStats()
        self._call("get_stats_noalloc", self._h, C.byref(s))
        return s.as_dict()

    # ---- coupling ----------------------------------------------------
    def set_gas_fields(self, grid: abi.DemFluidGrid, ep_g, u_g, v_g, w_g, p_force=None):
        ep_g = np.ascontiguousarray(ep_g, dtype=np.float64)
        u_g = np.ascontiguousarray(u_g, dtype=np.float64)
        v_g = np.ascontiguousarray(v_g, dtype=np.float64)
        w_g = np.ascontiguousarray(w_g, dtype=np.float64)
        pf = None if p_force is None else np.ascontiguousarray(p_force, dtype=np.float64)
        self._keep = (ep_g, u_g, v_g, w_g, pf)
        self._call("set_gas_fields", self._h, C.byref(grid), _dp(ep_g), _dp(u_g), _dp(v_g), _dp(w_g), _dp(pf))
        self._ncell = ep_g.shape[0]

    def get_mean_fields(self):
        ep = np.empty(self._ncell); rop = np.empty(self._ncell)
        self._call("get_mean_fields", self._h, _dp(ep), _dp(rop))
        return ep, rop

    def comp_mean_fields(self):
        self._call("comp_mean_fields", self._h)

    def calc_des_bedheight(self) -> np.ndarray:
        """CALC_DES_BEDHEIGHT per solids phase from the last mean fields."""
        out = np.zeros(self.params.n_phases)
        self._call("calc_des_bedheight", self._h, _dp(out))
        return out

    def drag_gs_des0(self):
        self._call("drag_gs_des0", self._h)

    def drag_gs_gas0(self):
        """DRAG_GS_GAS0: returns F_GDS (ncells), DRAG_AM (ncells),
        DRAG_BM (3, ncells) and F_GP (max_pip)."""
        f_gds = np.empty(self._ncell); am = np.empty(self._ncell)
        bm = np.empty((3, self._ncell)); f_gp = np.empty(self.n)
        self._call("drag_gs_gas0", self._h, _dp(f_gds), _dp(am), _dp(bm), _dp(f_gp))
        return f_gds, am, bm, f_gp

    def drag_gs_des1(self):
        self._call("drag_gs_des1", self._h)

    def drag_gs_gas1(self):
        """DRAG_GS_GAS1 without a filter: returns F_GDS (ncells), DRAG_BM
        (3, ncells) and F_GP (max_pip)."""
        f_gds = np.empty(self._ncell); bm = np.empty((3, self._ncell)); f_gp = np.empty(self.n)
        self._call("drag_gs_gas1", self._h, _dp(f_gds), _dp(bm), _dp(f_gp))
        return f_gds, bm, f_gp

    def step_coupled(self, nsteps: int = 1, nn_first: Optional[int] = None):
        first = self.nn + 1 if nn_first is None else nn_first
        self._call("step_coupled", self._h, C.c_int32(first), C.c_int32(nsteps))
        self.nn = first + nsteps - 1

    # ---- CUDA-only ---------------------------------------------------
    def write_vtp(self, path, time=0.0, angular_velocity=False, box=None, select_mode="C", phases=None) -> int:
        """WRITE_VTP_FILE for particle data; box = (lo, hi) of the VTK
        region, phases = 1-based phases to keep.  Returns the particle count."""
        o = abi.vtp_options(time, angular_velocity, box, select_mode, phases)
        n = C.c_int64()
        self._call("write_vtp", self._h, str(path).encode(), C.byref(o), C.byref(n))
        return int(n.value)

    def write_res0_des(self, path, ro_sol, vtp_findex=0, tecplot_findex=0, dtsolid=None):
        """WRITE_RES0_DES: the DEM restart file of this system.  ro_sol is
        RO_SOL per phase (the density the particles were generated with)."""
        info = abi.DemResInfo()
        info.vtp_findex, info.tecplot_findex = int(vtp_findex), int(tecplot_findex)
        info.dtsolid = self.params.dtsolid if dtsolid is None else float(dtsolid)
        for m, r in enumerate(ro_sol):
            info.ro_sol[m] = float(r)
        self._call("write_res0_des", self._h, str(path).encode(), C.byref(info))

    def read_res0_des(self, path, restore_pairs=True) -> abi.DemResInfo:
        """READ_RES0_DES into this system; with restore_pairs the pair list
        and its history come from the file, else call init_neighbors."""
        info = abi.DemResInfo()
        self._call("read_res0_des", self._h, str(path).encode(), C.c_int32(1 if restore_pairs else 0),
                   C.byref(info))
        return info

    def set_graphs(self, on: bool):
        self._call("set_graphs", self._h, C.c_int32(1 if on else 0))

    def set_profiling(self, on):
        """False/True, or 2 to time the parts of the force step as well."""
        self._call("set_profiling", self._h, C.c_int32(int(on)))

    def profile(self):
        """{class: (ms, launches)} since profiling was switched on."""
        ms = (C.c_double * 9)()
        nl = (C.c_int64 * 9)()
        self._call("get_profile", self._h, ms, nl)
        names = ("force", "neighbor", "desgrid", "integrate", "coupling", "other", "walls", "pairs", "gather")
        return {k: (float(ms[i]), int(nl[i])) for i, k in enumerate(names)}

    def memory_info(self) -> dict:
        """dem_memory_info: device bytes the handle holds (array_bytes,
        pair_bytes, scratch_bytes), its pair capacity and its pairs."""
        m = abi.DemMemory()
        self._call("memory_info", self._h, C.byref(m))
        return m.as_dict()

    def launch_count(self) -> int:
        v = C.c_int64()
        self._call("launch_count", self._h, C.byref(v))
        return int(v.value)

    def set_stream(self, stream_ptr: int):
        self._call("set_stream", self._h, C.c_void_p(stream_ptr))

    def autotune(self, reps: int = 5) -> dict:
        """Picks the launch shapes of the hot kernels by timing them on the
        current state (dem_autotune); returns the chosen shapes and times."""
        t = abi.DemTuning()
        self._call("autotune", self._h, C.c_int32(int(reps)), C.byref(t))
        return t.as_dict()

    def get_tuning(self) -> dict:
        t = abi.DemTuning()
        self._call("get_tuning", self._h, C.byref(t))
        return t.as_dict()

    def set_tuning(self, tuning: dict):
        t = abi.DemTuning()
        for k in ("pair_threads", "pair_blocks_per_sm", "gather_threads", "neigh_threads"):
            setattr(t, k, int(tuning[k]))
        self._call("set_tuning", self._h, C.byref(t))

    def force_error(self) -> float:
        v = C.c_double()
        self._call("force_error", self._h, C.byref(v))
        return float(v.value)


class BatchSystem:
    """A batch handle of the CUDA library: many independent DEM systems
    stepped together (dem_batch_create and the dem_sys_* calls).

    Systems are added with their own parameters and particle capacity and
    addressed by the id `add` returns; arrays use the same layouts as
    DemSystem, with as many rows as the system's particle count."""

    def __init__(self, lib, common: abi.DemParams, limits: abi.DemBatchLimits):
        self._lib = lib
        self._pre = "dem_"
        self.common = common
        self.limits = limits
        self.n_of = {}
        h = C.c_void_p()
        self._call("batch_create", C.byref(common), C.byref(limits), C.byref(h))
        self._h = h

    _fn = DemSystem._fn
    _call = DemSystem._call
    close = DemSystem.close
    __del__ = DemSystem.__del__
    __enter__ = DemSystem.__enter__
    __exit__ = DemSystem.__exit__

    def add(self, params: abi.DemParams, max_pip: int) -> int:
        sid = C.c_int32()
        self._call("sys_add", self._h, C.byref(params), C.c_int32(int(max_pip)), C.byref(sid))
        self.n_of[sid.value] = int(max_pip)
        return sid.value

    def remove(self, sid: int):
        self._call("sys_remove", self._h, C.c_int32(sid))
        self.n_of.pop(sid, None)

    def set_walls(self, sid: int, vertex: np.ndarray, norm_face: np.ndarray):
        vertex = np.ascontiguousarray(vertex, dtype=np.float64)
        norm_face = np.ascontiguousarray(norm_face, dtype=np.float64)
        self._call("sys_set_walls", self._h, C.c_int32(sid), _dp(vertex), _dp(norm_face),
                   C.c_int32(vertex.shape[0]))

    def upload_state(self, sid: int, pos, vel, omega, radius, pmass, omoi, state, phase):
        n = np.asarray(radius).shape[0]
        pos = _f64(pos, (3, n)); vel = _f64(vel, (3, n)); omega = _f64(omega, (3, n))
        radius = _f64(radius, (n,)); pmass = _f64(pmass, (n,)); omoi = _f64(omoi, (n,))
        state = np.ascontiguousarray(state, dtype=np.int8)
        phase = np.ascontiguousarray(phase, dtype=np.int32)
        self._call("sys_upload_state", self._h, C.c_int32(sid), _dp(pos), _dp(vel), _dp(omega), _dp(radius),
                   _dp(pmass), _dp(omoi), _bp(state), _ip(phase), C.c_int32(n))
        self.n_of[sid] = n

    def download_state(self, sid: int):
        n = self.n_of[sid]
        pos = np.empty((3, n)); vel = np.empty((3, n)); omega = np.empty((3, n))
        state = np.empty(n, dtype=np.int8)
        self._call("sys_download_state", self._h, C.c_int32(sid), _dp(pos), _dp(vel), _dp(omega), _bp(state),
                   C.c_int32(n))
        return {"pos": pos, "vel": vel, "omega": omega, "state": state}

    def start(self, sids):
        ids = np.ascontiguousarray(list(sids), dtype=np.int32)
        self._call("sys_start", self._h, _ip(ids), C.c_int32(ids.shape[0]))

    def step(self, nsteps: int = 1):
        self._call("batch_step", self._h, C.c_int32(int(nsteps)))

    def stats(self, sid: int) -> dict:
        s = abi.DemStats()
        self._call("sys_get_stats", self._h, C.c_int32(sid), C.byref(s))
        return s.as_dict()

    def download_pairs(self, sid: int):
        n = self.n_of[sid]
        P = int(self.stats(sid)["n_pairs"])
        ni = np.empty(n, dtype=np.int32)
        nb = np.empty(max(P, 1), dtype=np.int32)
        pf = np.empty((max(P, 1), 3))
        self._call("sys_download_pairs", self._h, C.c_int32(sid), _ip(ni), _ip(nb), _dp(pf),
                   C.c_int64(max(P, 1)), C.c_int32(n))
        return ni, nb[:P].copy(), pf[:P].copy()

    def total_stats(self) -> dict:
        """dem_get_stats over the whole handle (all systems together)."""
        s = abi.DemStats()
        self._call("get_stats", self._h, C.byref(s))
        return s.as_dict()

    def info(self, sid: int) -> dict:
        s = abi.DemSysStatus()
        self._call("sys_info", self._h, C.c_int32(sid), C.byref(s))
        return {"capacity": s.capacity, "started": bool(s.started), "next_nn": s.next_nn,
                "particle_offset": s.particle_offset, "steps_done": s.steps_done, "s_time": s.s_time}

    def launch_count(self) -> int:
        v = C.c_int64()
        self._call("launch_count", self._h, C.byref(v))
        return int(v.value)

    def set_profiling(self, on):
        """False/True, or 2 to time the parts of the force step as well."""
        self._call("set_profiling", self._h, C.c_int32(int(on)))

    profile = DemSystem.profile
    pair_count = DemSystem.pair_count
    set_stream = DemSystem.set_stream
    set_graphs = DemSystem.set_graphs
    memory_info = DemSystem.memory_info
    autotune = DemSystem.autotune
    get_tuning = DemSystem.get_tuning
    set_tuning = DemSystem.set_tuning
