"""ctypes mirror of include/dem_b200.h (structs, constants, signatures).

The structures here must match the C header field for field; the tests check
sizeof() against the library's own view through dem_abi_version and a
round-trip of dem_params.
"""
import ctypes as C

DEM_ABI_VERSION = 2
DEM_MAX_PHASES = 8

DEM_COLL_LSD = 0
DEM_COLL_HERTZ = 1
DEM_INTG_EULER = 0
DEM_INTG_AB2 = 1
DEM_PREC_FP64 = 0
DEM_PREC_SPLIT = 1

DEM_INTERP_GARG = 0
DEM_INTERP_NONE = 1
DEM_DRAG_GIDASPOW = 0
DEM_DRAG_SINGLE_SPHERE = 1

DEM_STATE_NONEXISTENT = 0
DEM_STATE_NORMAL = 1
DEM_STATE_ENTERING = 2
DEM_STATE_EXITING = 3
DEM_STATE_RIGID = 10
DEM_STATE_NORMAL_GHOST = 101

DEM_OK = 0
DEM_ERR_ARG = 1
DEM_ERR_CUDA = 2
DEM_ERR_ZERO_DISTANCE = 3
DEM_ERR_PAIR_OVERFLOW = 4
DEM_ERR_WALL_SLOTS = 5
DEM_ERR_ROGUE = 6
DEM_ERR_NONFINITE = 7
DEM_ERR_STATE = 8
DEM_ERR_TIMEOUT = 9
DEM_ERR_CAPACITY = 10

ERROR_NAMES = {
    0: "DEM_OK", 1: "DEM_ERR_ARG", 2: "DEM_ERR_CUDA", 3: "DEM_ERR_ZERO_DISTANCE",
    4: "DEM_ERR_PAIR_OVERFLOW", 5: "DEM_ERR_WALL_SLOTS", 6: "DEM_ERR_ROGUE",
    7: "DEM_ERR_NONFINITE", 8: "DEM_ERR_STATE", 9: "DEM_ERR_TIMEOUT",
    10: "DEM_ERR_CAPACITY",
}

_M2 = DEM_MAX_PHASES * DEM_MAX_PHASES


class DemParams(C.Structure):
    _fields_ = [
        ("n_phases", C.c_int32),
        ("coll_model", C.c_int32),
        ("intg_method", C.c_int32),
        ("neighbor_search_n", C.c_int32),
        ("force_precision", C.c_int32),
        ("remove_rogue", C.c_int32),
        ("no_k", C.c_int32),
        ("periodic", C.c_int32 * 3),
        ("dg_imax", C.c_int32),
        ("dg_jmax", C.c_int32),
        ("dg_kmax", C.c_int32),
        ("collision_array_max", C.c_int32),
        ("reserved_i", C.c_int32 * 6),
        ("factor_rlm", C.c_double),
        ("dtsolid", C.c_double),
        ("grav", C.c_double * 3),
        ("kn", C.c_double),
        ("kt", C.c_double),
        ("kn_w", C.c_double),
        ("kt_w", C.c_double),
        ("mew", C.c_double),
        ("mew_w", C.c_double),
        ("mew_r", C.c_double),
        ("mew_rw", C.c_double),
        ("max_radius", C.c_double),
        ("dg_xstart", C.c_double),
        ("dg_ystart", C.c_double),
        ("dg_zstart", C.c_double),
        ("dg_dxinv", C.c_double),
        ("dg_dyinv", C.c_double),
        ("dg_dzinv", C.c_double),
        ("domain_lo", C.c_double * 3),
        ("domain_hi", C.c_double * 3),
        ("des_etan", C.c_double * _M2),
        ("des_etat", C.c_double * _M2),
        ("hert_kn", C.c_double * _M2),
        ("hert_kt", C.c_double * _M2),
        ("des_etan_wall", C.c_double * DEM_MAX_PHASES),
        ("des_etat_wall", C.c_double * DEM_MAX_PHASES),
        ("hert_kwn", C.c_double * DEM_MAX_PHASES),
        ("hert_kwt", C.c_double * DEM_MAX_PHASES),
        ("reserved_d", C.c_double * 8),
    ]


class DemStats(C.Structure):
    _fields_ = [
        ("n_normal", C.c_int64),
        ("n_pairs", C.c_int64),
        ("n_contacts", C.c_int64),
        ("n_wall_contacts", C.c_int64),
        ("n_rogue_removed", C.c_int64),
        ("steps_done", C.c_int64),
        ("mean_vel", C.c_double * 3),
        ("gran_temp", C.c_double * 3),
        ("kinetic_energy", C.c_double),
        ("max_overlap_ratio", C.c_double),
        ("bed_height", C.c_double),
        ("s_time", C.c_double),
        ("n_outflow_removed", C.c_int64),
        ("n_inflow_added", C.c_int64),
        ("n_candidate_lists", C.c_int64),
        ("n_builds_filtered", C.c_int64),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            if name == "reserved":
                continue
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class DemFluidGrid(C.Structure):
    _fields_ = [
        ("imax", C.c_int32),
        ("jmax", C.c_int32),
        ("kmax", C.c_int32),
        ("drag_model", C.c_int32),
        ("interp_scheme", C.c_int32),
        ("reserved_i", C.c_int32),
        ("dx", C.c_double),
        ("dy", C.c_double),
        ("dz", C.c_double),
        ("ro_g", C.c_double),
        ("mu_g", C.c_double),
        ("ep_star", C.c_double),
        ("ur_f_gs", C.c_double),
        ("ro_s", C.c_double * DEM_MAX_PHASES),
        ("usr_d_p0", C.c_double),
        ("reserved", C.c_double * 5),
    ]


class DemTuning(C.Structure):
    _fields_ = [
        ("pair_threads", C.c_int32),
        ("pair_blocks_per_sm", C.c_int32),
        ("gather_threads", C.c_int32),
        ("neigh_threads", C.c_int32),
        ("pair_ms", C.c_double),
        ("gather_ms", C.c_double),
        ("neigh_ms", C.c_double),
        ("reserved", C.c_double * 4),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class DemBatchLimits(C.Structure):
    _fields_ = [
        ("max_particles", C.c_int32),
        ("max_systems", C.c_int32),
        ("max_cells", C.c_int32),
        ("max_search_cells", C.c_int32),
        ("max_facets", C.c_int32),
        ("max_facet_bins", C.c_int32),
        ("pairs_per_particle", C.c_int32),
        ("reserved", C.c_int32 * 9),
    ]


class DemMemory(C.Structure):
    _fields_ = [
        ("array_bytes", C.c_int64),
        ("pair_bytes", C.c_int64),
        ("scratch_bytes", C.c_int64),
        ("pair_capacity", C.c_int64),
        ("pairs", C.c_int64),
        ("reserved", C.c_int64 * 3),
    ]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


class DemSysStatus(C.Structure):
    _fields_ = [
        ("capacity", C.c_int32),
        ("started", C.c_int32),
        ("next_nn", C.c_int32),
        ("particle_offset", C.c_int32),
        ("steps_done", C.c_int64),
        ("s_time", C.c_double),
        ("reserved", C.c_double * 6),
    ]


class DemResInfo(C.Structure):
    _fields_ = [
        ("version", C.c_double),
        ("dtsolid", C.c_double),
        ("vtp_findex", C.c_int32),
        ("tecplot_findex", C.c_int32),
        ("n_particles", C.c_int32),
        ("n_pairs", C.c_int32),
        ("ro_sol", C.c_double * DEM_MAX_PHASES),
        ("reserved", C.c_double * 4),
    ]


class DemVtpOptions(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("angular_velocity", C.c_int32),
        ("use_box", C.c_int32),
        ("select_mode", C.c_int32),
        ("phase_mask", C.c_uint32),
        ("box_lo", C.c_double * 3),
        ("box_hi", C.c_double * 3),
        ("reserved", C.c_double * 4),
    ]


class DemOutflowBC(C.Structure):
    _fields_ = [
        ("plane", C.c_int32),
        ("mass_outflow", C.c_int32),
        ("dg_lo", C.c_int32 * 3),
        ("dg_hi", C.c_int32 * 3),
        ("reserved_i", C.c_int32 * 4),
        ("face", C.c_double),
        ("vel", (C.c_double * 3) * DEM_MAX_PHASES),
        ("reserved_d", C.c_double * 4),
    ]


class DemInflowBC(C.Structure):
    _fields_ = [
        ("plane", C.c_int32),
        ("occupants", C.c_int32),
        ("vacancy", C.c_int32),
        ("pi_count", C.c_int32),
        ("polydisperse", C.c_int32),
        ("n_layout", C.c_int32),
        ("dg_lo", C.c_int32 * 3),
        ("dg_hi", C.c_int32 * 3),
        ("l_index", C.c_int32),
        ("reserved_i", C.c_int32 * 3),
        ("offset", C.c_double),
        ("window", C.c_double),
        ("face", C.c_double),
        ("pi_factor", C.c_double),
        ("mi_time", C.c_double),
        ("start_time", C.c_double),
        ("end_time", C.c_double),
        ("p", C.POINTER(C.c_double)),
        ("q", C.POINTER(C.c_double)),
        ("poly_layout", C.POINTER(C.c_int32)),
        ("w_cell", C.POINTER(C.c_int32)),
        ("h_cell", C.POINTER(C.c_int32)),
        ("d_p0", C.c_double * DEM_MAX_PHASES),
        ("ro_s0", C.c_double * DEM_MAX_PHASES),
        ("vel", (C.c_double * 3) * DEM_MAX_PHASES),
        ("reserved_d", C.c_double * 4),
    ]


class DemResInflow(C.Structure):
    _fields_ = [
        ("mi_time", C.c_double),
        ("window", C.c_double),
        ("offset", C.c_double),
        ("vacancy", C.c_int32),
        ("occupants", C.c_int32),
        ("l_index", C.c_int32),
        ("reserved", C.c_int32),
    ]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I8 = C.POINTER(C.c_int8)

# name -> (restype, argtypes); prefix is substituted ("dem_" or "orc_")
SIGNATURES = {
    "create": (C.c_int, [C.POINTER(DemParams), C.c_int32, C.POINTER(C.c_void_p)]),
    "destroy": (C.c_int, [_P]),
    "last_error": (C.c_char_p, [_P]),
    "set_walls": (C.c_int, [_P, _D, _D, C.c_int32]),
    "upload_state": (C.c_int, [_P, _D, _D, _D, _D, _D, _D, _I8, _I32, C.c_int32]),
    "download_state": (C.c_int, [_P, _D, _D, _D, _I8, C.c_int32]),
    "download_forces": (C.c_int, [_P, _D, _D, C.c_int32]),
    "set_ab2_history": (C.c_int, [_P, _D, _D, C.c_int32, C.c_int32]),
    "get_ab2_history": (C.c_int, [_P, _D, _D, C.c_int32]),
    "pair_count": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "download_pairs": (C.c_int, [_P, _I32, _I32, _D, C.c_int64, C.c_int32]),
    "upload_pairs": (C.c_int, [_P, _I32, _I32, _D, C.c_int64, C.c_int32]),
    "download_wall_history": (C.c_int, [_P, _I32, _D, C.c_int32]),
    "set_outflow_bcs": (C.c_int, [_P, C.c_void_p, C.c_int32]),
    "set_inflow_bcs": (C.c_int, [_P, C.c_void_p, C.c_int32, C.c_uint64]),
    "push_inflow_random": (C.c_int, [_P, _D, C.c_int64]),
    "get_inflow_state": (C.c_int, [_P, C.c_int32, _I32, _D]),
    "upload_wall_history": (C.c_int, [_P, _I32, _D, C.c_int32]),
    "download_cells": (C.c_int, [_P, _I32, C.c_int32]),
    "desgrid_pic": (C.c_int, [_P]),
    "neighbour": (C.c_int, [_P]),
    "calc_force": (C.c_int, [_P]),
    "cfnewvalues": (C.c_int, [_P]),
    "init_neighbors": (C.c_int, [_P]),
    "step": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "get_stats": (C.c_int, [_P, C.POINTER(DemStats)]),
    "set_gas_fields": (C.c_int, [_P, C.POINTER(DemFluidGrid), _D, _D, _D, _D, _D]),
    "get_mean_fields": (C.c_int, [_P, _D, _D]),
    "comp_mean_fields": (C.c_int, [_P]),
    "set_dtsolid": (C.c_int, [_P, C.c_double]),
    "calc_des_bedheight": (C.c_int, [_P, _D]),
    "drag_gs_des0": (C.c_int, [_P]),
    "drag_gs_gas0": (C.c_int, [_P, _D, _D, _D, _D]),
    "drag_gs_des1": (C.c_int, [_P]),
    "drag_gs_gas1": (C.c_int, [_P, _D, _D, _D]),
    "step_coupled": (C.c_int, [_P, C.c_int32, C.c_int32]),
}

# entry points only the CUDA library has
DEM_ONLY = {
    "abi_version": (C.c_int, []),
    "launch_count": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "set_stream": (C.c_int, [_P, C.c_void_p]),
    "force_error": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "set_profiling": (C.c_int, [_P, C.c_int32]),
    "set_graphs": (C.c_int, [_P, C.c_int32]),
    "get_profile": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "get_stats_noalloc": (C.c_int, [_P, C.POINTER(DemStats)]),
    "autotune": (C.c_int, [_P, C.c_int32, C.POINTER(DemTuning)]),
    "get_tuning": (C.c_int, [_P, C.POINTER(DemTuning)]),
    "set_tuning": (C.c_int, [_P, C.POINTER(DemTuning)]),
    # batches of independent systems
    "params_cells": (C.c_int, [C.POINTER(DemParams), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "batch_create": (C.c_int, [C.POINTER(DemParams), C.POINTER(DemBatchLimits), C.POINTER(C.c_void_p)]),
    "sys_add": (C.c_int, [_P, C.POINTER(DemParams), C.c_int32, C.POINTER(C.c_int32)]),
    "sys_remove": (C.c_int, [_P, C.c_int32]),
    "sys_set_walls": (C.c_int, [_P, C.c_int32, _D, _D, C.c_int32]),
    "sys_upload_state": (C.c_int, [_P, C.c_int32, _D, _D, _D, _D, _D, _D, _I8, _I32, C.c_int32]),
    "sys_download_state": (C.c_int, [_P, C.c_int32, _D, _D, _D, _I8, C.c_int32]),
    "sys_start": (C.c_int, [_P, _I32, C.c_int32]),
    "batch_step": (C.c_int, [_P, C.c_int32]),
    "batch_footprint": (C.c_int, [C.POINTER(DemParams), C.POINTER(DemBatchLimits), C.POINTER(DemMemory)]),
    "memory_info": (C.c_int, [_P, C.POINTER(DemMemory)]),
    # particle output
    "write_vtp": (C.c_int, [_P, C.c_char_p, C.POINTER(DemVtpOptions), C.POINTER(C.c_int64)]),
    "vtp_write": (C.c_int, [C.c_char_p, C.POINTER(DemVtpOptions), C.c_int32, _D, _D, _D, _D, _I8, _I32,
                            C.POINTER(C.c_int64)]),
    # restart files
    "write_res0_des": (C.c_int, [_P, C.c_char_p, C.POINTER(DemResInfo)]),
    "read_res0_des": (C.c_int, [_P, C.c_char_p, C.c_int32, C.POINTER(DemResInfo)]),
    "res_write": (C.c_int, [C.c_char_p, C.POINTER(DemResInfo), C.c_int32, C.c_int32, _D, _D, _D, _D, _I8, _I32,
                            _I32, _I32, _D, C.c_int64]),
    "res_read_inflow": (C.c_int, [C.c_char_p, C.c_int32, _I32, C.c_void_p, C.c_int32, _I32, _I32, _D, _D, C.c_int32]),
    "res_read": (C.c_int, [C.c_char_p, C.POINTER(DemResInfo), C.c_int32, C.c_int32, _D, _D, _D, _D, _D, _I8, _I32,
                           _I32, _I32, _D, C.c_int64]),
    "sys_get_stats": (C.c_int, [_P, C.c_int32, C.POINTER(DemStats)]),
    "sys_download_pairs": (C.c_int, [_P, C.c_int32, _I32, _I32, _D, C.c_int64, C.c_int32]),
    "sys_info": (C.c_int, [_P, C.c_int32, C.POINTER(DemSysStatus)]),
}

DEM_STATS_NOALLOC_MAX_PARTICLES = 1 << 23


def bind(lib, prefix, extra=None):
    """Set restype/argtypes for every entry point present in `lib`."""
    table = dict(SIGNATURES)
    if extra:
        table.update(extra)
    for name, (res, args) in table.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
    return lib


def vtp_options(time=0.0, angular_velocity=False, box=None, select_mode="C", phases=None) -> DemVtpOptions:
    """A dem_vtp_options for one VTK region of particle data."""
    o = DemVtpOptions()
    o.time = float(time)
    o.angular_velocity = 1 if angular_velocity else 0
    o.select_mode = ord(select_mode)
    if box is not None:
        o.use_box = 1
        for c in range(3):
            o.box_lo[c], o.box_hi[c] = float(box[0][c]), float(box[1][c])
    if phases:
        o.phase_mask = sum(1 << (int(m) - 1) for m in phases)
    return o
