"""Keyword-level set-up of a DEM case: the derived tables MFiX computes before
the DEM loop, restated for the host side of this library.

A Fortran driver already holds these values in its module globals and passes
them to dem_create().  Python users build them here from the same keywords:

- reference particle size/mass per phase, GET_REF_PARTICLE_SIZE_AND_MASS
  (model/check_data/check_solids_dem.f:1135-1223);
- LSD and Hertz spring/damping tables and DTSOLID, CHECK_SOLIDS_DEM_COLL_LSD
  (check_solids_dem.f:519-782) and CHECK_SOLIDS_DEM_COLL_HERTZ (798-1122);
- DES grid sizing, CHECK_GEOMETRY (model/check_data/check_geometry.f:133-190)
  and DESGRID_INIT (model/des/desgrid_mod.f:571-604, 833-850);
- particle mass and inverse moment of inertia, MAKE_ARRAYS_DES
  (model/des/make_arrays_des.f:241-244).

Keyword defaults follow model/des/des_init_namelist.f.  Several of them are
REAL(4) literals in the reference and are reproduced as such (float32 values
widened to double): FACTOR_RLM = 1.2 (line 1169) and KT_FAC = KT_W_FAC =
0.28571428571429 (lines 1215, 1237).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import abi

PI = 4.0 * math.atan(1.0)          # parse_line.f:563
UNDEFINED = 9.87654321e31          # param1_mod.f:20
FLT_HUGE = float(np.finfo(np.float32).max)


def f32(x: float) -> float:
    """A Fortran default-REAL literal widened to DOUBLE PRECISION."""
    return float(np.float32(x))


FACTOR_RLM_DEFAULT = f32(1.2)
KT_FAC_DEFAULT = f32(0.28571428571429)


def xpow3(x):
    """x**3.0d0 through the reference's pow wrapper (model/xpow.c): an
    integral exponent 3 is evaluated by binary powering as x*(x*x)."""
    return x * (x * x)


@dataclass
class DemCase:
    """The DEM keywords of one case (des_init_namelist.f names in comments)."""
    n_phases: int = 1
    d_p0: Sequence[float] = (1e-3,)             # D_P0(M)
    ro_s0: Sequence[float] = (2500.0,)          # RO_S0(M)
    coll_model: str = "LSD"                      # DES_COLL_MODEL
    intg_method: str = "EULER"                   # DES_INTG_METHOD
    kn: float = UNDEFINED                        # KN
    kn_w: float = UNDEFINED                      # KN_W
    kt_fac: Optional[float] = None               # KT_FAC (default f32 2/7)
    kt_w_fac: Optional[float] = None             # KT_W_FAC
    des_etat_fac: Optional[float] = None         # DES_ETAT_FAC (default 1/2)
    des_etat_w_fac: Optional[float] = None       # DES_ETAT_W_FAC
    des_en_input: Optional[np.ndarray] = None    # (M,M) restitution
    des_en_wall_input: Optional[Sequence[float]] = None
    des_et_input: Optional[np.ndarray] = None    # Hertz tangential restitution
    des_et_wall_input: Optional[Sequence[float]] = None
    e_young: Sequence[float] = ()                # E_YOUNG(M)
    v_poisson: Sequence[float] = ()              # V_POISSON(M)
    ew_young: float = UNDEFINED                  # Ew_YOUNG
    vw_poisson: float = UNDEFINED                # Vw_POISSON
    mew: float = 0.0                             # MEW
    mew_w: float = 0.0                           # MEW_W
    mew_r: float = 0.0                           # MEW_R
    mew_rw: float = 0.0                          # MEW_RW
    grav: Sequence[float] = (0.0, -9.81, 0.0)    # GRAVITY_X/Y/Z
    domain_lo: Sequence[float] = (0.0, 0.0, 0.0)
    domain_hi: Sequence[float] = (1.0, 1.0, 1.0)
    fluid_cells: Sequence[int] = (1, 1, 1)       # IMAX, JMAX, KMAX
    no_k: bool = False
    periodic: Sequence[bool] = (False, False, False)
    desgridsearch: Sequence[Optional[int]] = (None, None, None)
    neighbor_search_n: int = 25                  # NEIGHBOR_SEARCH_N
    factor_rlm: float = FACTOR_RLM_DEFAULT       # FACTOR_RLM
    dtsolid_factor: float = 50.0                 # DTSOLID_FACTOR
    dtsolid: Optional[float] = None              # DTSOLID (None = derived)
    collision_array_max: int = 8                 # COLLISION_ARRAY_MAX
    remove_rogue: bool = True                    # REMOVE_ROGUE_PARTICLES
    force_precision: int = abi.DEM_PREC_FP64


def particle_props(radius: np.ndarray, rho: np.ndarray):
    """PVOL, PMASS, OMOI as MAKE_ARRAYS_DES computes them
    (make_arrays_des.f:241-244): PVOL = (4/3)*PI*R**3.0d0, PMASS = PVOL*RO,
    OMOI = 2.5/(PMASS*R**2)."""
    radius = np.asarray(radius, dtype=np.float64)
    pvol = ((4.0 / 3.0) * PI) * xpow3(radius)
    pmass = pvol * np.asarray(rho, dtype=np.float64)
    with np.errstate(divide="ignore"):
        omoi = 2.5 / (pmass * (radius * radius))
    return pvol, pmass, omoi


def ref_size_and_mass(case: DemCase, radius, pmass, phase, state):
    """GET_REF_PARTICLE_SIZE_AND_MASS (check_solids_dem.f:1135-1223): the
    minimum of the phase's nominal and actual NORMAL particle sizes/masses.
    `phase` is 1-based."""
    M = case.n_phases
    ref_r = np.zeros(M)
    ref_m = np.zeros(M)
    for m in range(M):
        d = case.d_p0[m]
        ref_r[m] = 0.5 * d
        ref_m[m] = (PI / 6.0) * (d * d * d) * case.ro_s0[m]
    normal = np.asarray(state) == abi.DEM_STATE_NORMAL
    ph = np.asarray(phase) - 1
    for m in range(M):
        sel = normal & (ph == m)
        if sel.any():
            ref_r[m] = min(ref_r[m], float(np.min(radius[sel])))
            ref_m[m] = min(ref_m[m], float(np.min(pmass[sel])))
    return ref_r, ref_m


def _sym(x, M, name):
    if x is None:
        raise ValueError(f"Required input not specified: {name}")
    a = np.asarray(x, dtype=np.float64)
    if a.ndim == 0:
        return np.full((M, M), float(a))
    return a


def contact_constants(case: DemCase, ref_r, ref_m, p: abi.DemParams):
    """Fills the contact tables of `p` and returns TCOLL.

    LSD: check_solids_dem.f:519-782.  Hertz: check_solids_dem.f:798-1122.
    Tables are stored in the particle-agnostic form the force routines use.
    """
    M, S = case.n_phases, abi.DEM_MAX_PHASES
    en = _sym(case.des_en_input, M, "DES_EN_INPUT")
    enw = np.asarray(case.des_en_wall_input if case.des_en_wall_input is not None
                     else [None] * M, dtype=object)
    if any(v is None for v in enw):
        raise ValueError("Required input not specified: DES_EN_WALL_INPUT")
    enw = enw.astype(np.float64)
    tcoll = UNDEFINED
    if case.coll_model.upper() == "LSD":
        if case.kn == UNDEFINED or case.kn_w == UNDEFINED:
            raise ValueError("Required input not specified: KN / KN_W")
        kt_fac = KT_FAC_DEFAULT if case.kt_fac is None else case.kt_fac
        kt_w_fac = KT_FAC_DEFAULT if case.kt_w_fac is None else case.kt_w_fac
        etat_fac = 0.5 if case.des_etat_fac is None else case.des_etat_fac
        etat_w_fac = 0.5 if case.des_etat_w_fac is None else case.des_etat_w_fac
        p.kn, p.kn_w = case.kn, case.kn_w
        p.kt = kt_fac * case.kn
        p.kt_w = kt_w_fac * case.kn_w
        for m in range(M):
            mass_m = ref_m[m]
            for l in range(m, M):
                e = en[m, l]
                mass_l = ref_m[l]
                meff = mass_m * mass_l / (mass_m + mass_l)
                if e != 0.0:
                    etan = 2.0 * math.sqrt(case.kn * meff) * abs(math.log(e))
                    etan = etan / math.sqrt(PI * PI + (math.log(e) * math.log(e)))
                    tc = PI / math.sqrt(case.kn / meff - ((etan / meff) * (etan / meff)) / 4.0)
                else:
                    etan = 2.0 * math.sqrt(case.kn * meff)
                    tc = PI / math.sqrt(case.kn / meff)
                tcoll = min(tc, tcoll)
                etan = etan / math.sqrt(meff)
                p.des_etan[m * S + l] = p.des_etan[l * S + m] = etan
                p.des_etat[m * S + l] = p.des_etat[l * S + m] = etat_fac * etan
            e = enw[m]
            meff = mass_m
            if e != 0.0:
                etan = 2.0 * math.sqrt(case.kn_w * meff) * abs(math.log(e))
                etan = etan / math.sqrt(PI * PI + (math.log(e) * math.log(e)))
            else:
                etan = 2.0 * math.sqrt(case.kn_w * meff)
            etan = etan / math.sqrt(meff)
            p.des_etan_wall[m] = etan
            p.des_etat_wall[m] = etat_w_fac * etan
    elif case.coll_model.upper() == "HERTZ":
        et = _sym(case.des_et_input, M, "DES_ET_INPUT")
        if case.des_et_wall_input is None:
            raise ValueError("Required input not specified: DES_ET_WALL_INPUT")
        etw = np.asarray(case.des_et_wall_input, dtype=np.float64)
        if case.ew_young == UNDEFINED or case.vw_poisson == UNDEFINED:
            raise ValueError("Required input not specified: Ew_YOUNG / Vw_POISSON")
        E = np.asarray(case.e_young, dtype=np.float64)
        nu = np.asarray(case.v_poisson, dtype=np.float64)
        gw = 0.5 * case.ew_young / (1.0 + case.vw_poisson)
        G = [0.5 * E[m] / (1.0 + nu[m]) for m in range(M)]
        for m in range(M):
            mass_m = ref_m[m]
            for l in range(m, M):
                e, t = en[m, l], et[m, l]
                mass_l = ref_m[l]
                meff = (mass_m * mass_l) / (mass_m + mass_l)
                red = (2.0 / 7.0) * meff
                reff = ref_r[m] * ref_r[l] / (ref_r[m] + ref_r[l])
                eeff = E[m] * E[l] / (E[m] * (1.0 - nu[l] * nu[l]) + E[l] * (1.0 - nu[m] * nu[m]))
                geff = G[m] * G[l] / (G[m] * (2.0 - nu[l]) + G[l] * (2.0 - nu[m]))
                hkn = (4.0 / 3.0) * math.sqrt(reff) * eeff
                hkt = 8.0 * math.sqrt(reff) * geff
                if e != 0.0:
                    etan = math.sqrt(5.0) * math.sqrt(hkn * meff) * abs(math.log(e))
                    etan = etan / math.sqrt(PI * PI + (math.log(e) * math.log(e)))
                    tc = PI / math.sqrt(hkn / meff - ((etan / meff) * (etan / meff)) / 5.0)
                else:
                    etan = math.sqrt(5.0) * math.sqrt(hkn * meff)
                    tc = PI / math.sqrt(hkn / meff)
                if t != 0.0:
                    etat = math.sqrt(5.0) * math.sqrt(hkt * red) * abs(math.log(t))
                    etat = etat / math.sqrt(PI * PI + (math.log(t) * math.log(t)))
                else:
                    etat = math.sqrt(5.0) * math.sqrt(hkt * red)
                tcoll = min(tc, tcoll)
                etan = etan / math.sqrt(hkn * meff)
                etat = etat / math.sqrt(hkt * meff)
                hkn = hkn / math.sqrt(reff)
                hkt = hkt / math.sqrt(reff)
                p.hert_kn[m * S + l] = p.hert_kn[l * S + m] = hkn
                p.hert_kt[m * S + l] = p.hert_kt[l * S + m] = hkt
                p.des_etan[m * S + l] = p.des_etan[l * S + m] = etan
                p.des_etat[m * S + l] = p.des_etat[l * S + m] = etat
            e, t = enw[m], etw[m]
            meff = mass_m
            red = (2.0 / 7.0) * meff
            reff = ref_r[m]
            eeff = E[m] * case.ew_young / (E[m] * (1.0 - case.vw_poisson * case.vw_poisson)
                                          + case.ew_young * (1.0 - nu[m] * nu[m]))
            geff = G[m] * gw / (G[m] * (2.0 - case.vw_poisson) + gw * (2.0 - nu[m]))
            hkwn = (4.0 / 3.0) * math.sqrt(reff) * eeff
            hkwt = 8.0 * math.sqrt(reff) * geff
            if e != 0.0:
                etan = math.sqrt(5.0) * math.sqrt(hkwn * meff) * abs(math.log(e))
                etan = etan / math.sqrt(PI * PI + (math.log(e) * math.log(e)))
            else:
                etan = math.sqrt(5.0) * math.sqrt(hkwn * meff)
            if t != 0.0:
                etat = math.sqrt(5.0) * math.sqrt(hkwt * red) * abs(math.log(t))
                etat = etat / math.sqrt(PI * PI + (math.log(t) * math.log(t)))
            else:
                etat = math.sqrt(5.0) * math.sqrt(hkwt * red)
            p.des_etan_wall[m] = etan / math.sqrt(hkwn * meff)
            p.des_etat_wall[m] = etat / math.sqrt(hkwt * meff)
            p.hert_kwn[m] = hkwn / math.sqrt(reff)
            p.hert_kwt[m] = hkwt / math.sqrt(reff)
    else:
        raise ValueError(f"unknown DES_COLL_MODEL {case.coll_model}")
    return tcoll


def desgrid_geometry(case: DemCase, max_radius: float):
    """DES grid cells per axis and origin/inverse width for one rank.

    CHECK_GEOMETRY (check_geometry.f:133-190): WIDTH = 3*max diameter, capped
    by the smallest fluid cell; DESGRIDSEARCH_?MAX = max(int(LENGTH/WIDTH),1)
    unless given.  DESGRID_INIT (desgrid_mod.f:833-850): dg_xstart is the west
    face of the first interior fluid cell and dg_dxinv = cells/(xend-xstart),
    with xend accumulated face by face over the fluid cells.
    """
    max_diam = 2.0 * max_radius
    width = 3.0 * max_diam
    lo, hi = case.domain_lo, case.domain_hi
    ncell, starts, invs = [], [], []
    for ax in range(3):
        length = hi[ax] - lo[ax]
        nfl = case.fluid_cells[ax]
        dfl = length / nfl
        if ax == 2 and case.no_k:
            ncell.append(1)
            starts.append(lo[2])
            invs.append(1.0 / (hi[2] - lo[2]))
            continue
        w = min(width, dfl)
        n = case.desgridsearch[ax]
        if n is None:
            n = max(int(length / w), 1)
        if length / float(n) < max_diam:
            raise ValueError("The des search grid is too fine (cell smaller than the max diameter)")
        xend = lo[ax]
        for _ in range(nfl):
            xend = xend + dfl
        ncell.append(n)
        starts.append(lo[ax])
        invs.append(n / (xend - lo[ax]))
    return ncell, starts, invs


def build_params(case: DemCase, radius, pmass, phase, state):
    """dem_params for a case, plus a dict of derived scalars (tcoll, ...)."""
    p = abi.DemParams()
    M = case.n_phases
    if not (1 <= M <= abi.DEM_MAX_PHASES):
        raise ValueError("n_phases out of range")
    p.n_phases = M
    p.coll_model = abi.DEM_COLL_HERTZ if case.coll_model.upper() == "HERTZ" else abi.DEM_COLL_LSD
    intg = case.intg_method.upper()
    p.intg_method = abi.DEM_INTG_AB2 if intg in ("ADAMS_BASHFORTH", "AB2") else abi.DEM_INTG_EULER
    p.neighbor_search_n = case.neighbor_search_n
    p.force_precision = case.force_precision
    p.remove_rogue = 1 if case.remove_rogue else 0
    p.no_k = 1 if case.no_k else 0
    for a in range(3):
        p.periodic[a] = 1 if case.periodic[a] else 0
        p.grav[a] = case.grav[a]
        p.domain_lo[a] = case.domain_lo[a]
        p.domain_hi[a] = case.domain_hi[a]
    p.collision_array_max = case.collision_array_max
    p.factor_rlm = case.factor_rlm
    p.mew, p.mew_w, p.mew_r, p.mew_rw = case.mew, case.mew_w, case.mew_r, case.mew_rw

    # MAX_RADIUS: largest nominal radius (check_solids_common_discrete.f:176-181)
    max_radius = max(0.5 * d for d in case.d_p0[:M])
    normal = np.asarray(state) == abi.DEM_STATE_NORMAL
    if normal.any():
        max_radius = max(max_radius, float(np.max(np.asarray(radius)[normal])))
    p.max_radius = max_radius

    ref_r, ref_m = ref_size_and_mass(case, np.asarray(radius), np.asarray(pmass), phase, state)
    tcoll = contact_constants(case, ref_r, ref_m, p)
    p.dtsolid = case.dtsolid if case.dtsolid is not None else tcoll / case.dtsolid_factor

    ncell, starts, invs = desgrid_geometry(case, max_radius)
    p.dg_imax, p.dg_jmax, p.dg_kmax = ncell
    p.dg_xstart, p.dg_ystart, p.dg_zstart = starts
    p.dg_dxinv, p.dg_dyinv, p.dg_dzinv = invs
    for ax in range(3):
        if case.periodic[ax] and ncell[ax] < 3:
            raise ValueError("periodic axes need at least 3 DES grid cells")
    return p, {"tcoll": tcoll, "ref_radius": ref_r, "ref_mass": ref_m, "max_radius": max_radius}


# ---------------------------------------------------------------------------
# Wall geometry in the Fortran layout VERTEX(3,3,F), NORM_FACE(3,F).

def _facets(tris, norms):
    F = len(tris)
    vertex = np.zeros((F, 3, 3))   # [f, c, v] -> offset v + 3c + 9f
    norm = np.zeros((F, 3))
    for f, (t, nrm) in enumerate(zip(tris, norms)):
        for v in range(3):
            for c in range(3):
                vertex[f, c, v] = t[v][c]
        norm[f] = nrm
    return vertex, norm


def default_walls(lo, hi, periodic=(False, False, False), no_k=False):
    """CONVERT_DEFAULT_WALLS_TO_STL (stl_preproc_des_mod.f:973-1046): one large
    triangle per non-periodic domain face, normals pointing into the domain."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    xl, yl, zl = x1 - x0, y1 - y0, z1 - z0
    tris, norms = [], []
    if not periodic[0]:
        tris.append([(x0, y0, z0), (x0, y1 + yl, z0), (x0, y0, z1 + zl)]); norms.append((1.0, 0.0, 0.0))
        tris.append([(x1, y0, z0), (x1, y1 + yl, z0), (x1, y0, z1 + zl)]); norms.append((-1.0, 0.0, 0.0))
    if not periodic[1]:
        tris.append([(x0, y0, z0), (x1 + xl, y0, z0), (x0, y0, z1 + zl)]); norms.append((0.0, 1.0, 0.0))
        tris.append([(x0, y1, z0), (x1 + xl, y1, z0), (x0, y1, z1 + zl)]); norms.append((0.0, -1.0, 0.0))
    if not periodic[2] and not no_k:
        tris.append([(x0, y0, z0), (x1 + xl, y0, z0), (x0, y1 + yl, z0)]); norms.append((0.0, 0.0, 1.0))
        tris.append([(x0, y0, z1), (x1 + xl, y0, z1), (x0, y1 + yl, z1)]); norms.append((0.0, 0.0, -1.0))
    return _facets(tris, norms)


def _facet_normal(t, toward):
    """Unit normal of triangle t (cross product of its edges), oriented to
    have a positive component along `toward`."""
    a, b, c = (np.asarray(v, dtype=float) for v in t)
    n = np.cross(b - a, c - a)
    n = n / np.linalg.norm(n)
    if float(np.dot(n, np.asarray(toward, dtype=float))) < 0.0:
        n = -n
    return tuple(float(x) for x in n)


def hopper_walls(lo, hi, half_angle_deg=30.0, outlet_diam=0.012, y_out=None, n_seg=64):
    """Box walls with a conical hopper bottom, triangulated.

    The cone has its axis along y through the box centre, its wall at
    `half_angle_deg` from the axis, an outlet of diameter `outlet_diam` at
    height y_out (default 5 % of the box height above its floor) and its rim
    on the circle inscribed in the box cross-section.  A flat plate at the rim
    height closes the corners between the rim and the box walls.  The x, z
    and top faces are the default box walls; the floor below the outlet is
    open, so particles that leave through the outlet end up outside the
    domain and are removed as rogue by the neighbour build.  Each facet's
    normal is its own (cross product), pointing into the particle region.
    n_seg must be a multiple of 8 so that the plate reaches the box corners.
    """
    if n_seg % 8:
        raise ValueError("n_seg must be a multiple of 8")
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    cx, cz = 0.5 * (x0 + x1), 0.5 * (z0 + z1)
    hx, hz = 0.5 * (x1 - x0), 0.5 * (z1 - z0)
    R = min(hx, hz)
    r_out = 0.5 * outlet_diam
    t = math.tan(math.radians(half_angle_deg))
    h_cone = (R - r_out) / t
    if y_out is None:
        y_out = y0 + 0.05 * (y1 - y0)
    y_top = y_out + h_cone
    xl, yl, zl = x1 - x0, y1 - y0, z1 - z0
    tris, norms = [], []
    # x faces, top face and z faces (one large triangle each, as the default walls)
    tris.append([(x0, y0, z0), (x0, y1 + yl, z0), (x0, y0, z1 + zl)]); norms.append((1.0, 0.0, 0.0))
    tris.append([(x1, y0, z0), (x1, y1 + yl, z0), (x1, y0, z1 + zl)]); norms.append((-1.0, 0.0, 0.0))
    tris.append([(x0, y1, z0), (x1 + xl, y1, z0), (x0, y1, z1 + zl)]); norms.append((0.0, -1.0, 0.0))
    tris.append([(x0, y0, z0), (x1 + xl, y0, z0), (x0, y1 + yl, z0)]); norms.append((0.0, 0.0, 1.0))
    tris.append([(x0, y0, z1), (x1 + xl, y0, z1), (x0, y1 + yl, z1)]); norms.append((0.0, 0.0, -1.0))

    def rim(a, r, y):
        return (cx + r * math.cos(a), y, cz + r * math.sin(a))

    def square(a):
        c, s_ = math.cos(a), math.sin(a)
        k = min(hx / abs(c) if abs(c) > 1e-15 else math.inf, hz / abs(s_) if abs(s_) > 1e-15 else math.inf)
        return (cx + k * c, y_top, cz + k * s_)

    for s_ in range(n_seg):
        a0 = 2 * math.pi * s_ / n_seg
        a1 = 2 * math.pi * (s_ + 1) / n_seg
        am = 0.5 * (a0 + a1)
        P0t, P1t = rim(a0, R, y_top), rim(a1, R, y_top)
        P0b, P1b = rim(a0, r_out, y_out), rim(a1, r_out, y_out)
        # cone wall: the particle side is toward the axis and up
        inward = (-math.cos(am), math.tan(math.radians(half_angle_deg)), -math.sin(am))
        for tri in ([P0b, P1b, P1t], [P0b, P1t, P0t]):
            tris.append(tri); norms.append(_facet_normal(tri, inward))
        # plate between the rim and the box walls
        Q0, Q1 = square(a0), square(a1)
        for tri in ([P0t, P1t, Q1], [P0t, Q1, Q0]):
            if np.linalg.norm(np.cross(np.subtract(tri[1], tri[0]), np.subtract(tri[2], tri[0]))) > 1e-18:
                tris.append(tri); norms.append((0.0, 1.0, 0.0))
    return _facets(tris, norms), {"y_out": y_out, "y_top": y_top, "r_out": r_out, "R": R}


def batch_limits(lib, entries, max_systems=None, slack=1.0, bins_per_cell=8):
    """dem_batch_limits for a batch holding `entries` = [(params, max_pip,
    n_facets), ...] at once (times `slack` for later arrivals).  The cell
    needs come from the library's own grid sizing (dem_params_cells)."""
    import ctypes as C
    des = srch = parts = facets = 0
    for prm, n, nf in entries:
        a, b = C.c_int32(), C.c_int32()
        rc = lib.dem_params_cells(C.byref(prm), C.byref(a), C.byref(b))
        if rc != 0:
            raise ValueError("invalid system parameters")
        des += a.value
        srch += b.value
        parts += ((int(n) + 63) // 64) * 64
        facets += int(nf)
    lim = abi.DemBatchLimits()
    lim.max_particles = int(parts * slack) + 64
    lim.max_systems = int(max_systems if max_systems is not None else max(1, len(entries)))
    lim.max_cells = int(des * slack) + 1
    lim.max_search_cells = int(srch * slack) + 1
    lim.max_facets = int(facets * slack) + 1
    lim.max_facet_bins = int(des * slack * bins_per_cell) + 1
    return lim


def _nint(v: float) -> int:
    """Fortran NINT: nearest integer, halves away from zero."""
    return int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5))


def outflow_bc(prm, plane: str, lo, hi, face: float, mass_outflow: bool = False, vel=None):
    """A dem_outflow_bc for a boundary whose extents are BC_X_w..BC_X_e,
    BC_Y_s..BC_Y_n, BC_Z_b..BC_Z_t = lo..hi: its DES-cell box as SET_BC_DEM_MO
    builds it (set_bc_dem_mo.f:79-101) with IofBCPOS/JofBCPOS/KofBCPOS
    (desgrid_mod.f:428-455: NINT of the position in DES cells, 1-based with
    one ghost layer), `face` the plane the distance is measured from and
    `vel` the BC_U_s/V_s/W_s per phase for MASS_OUTFLOW."""
    from . import abi
    b = abi.DemOutflowBC()
    b.plane = ord(plane)
    b.mass_outflow = 1 if mass_outflow else 0
    start = (prm.dg_xstart, prm.dg_ystart, prm.dg_zstart)
    inv = (prm.dg_dxinv, prm.dg_dyinv, prm.dg_dzinv)
    for a in range(3):
        if a == 2 and prm.no_k:
            b.dg_lo[2] = b.dg_hi[2] = 1
            continue
        b.dg_lo[a] = _nint((lo[a] - start[a]) * inv[a]) + 2 - 1
        b.dg_hi[a] = _nint((hi[a] - start[a]) * inv[a]) + 2 - 1 + 1
    b.face = float(face)
    for m, v in enumerate(vel or []):
        for c in range(3):
            b.vel[m][c] = float(v[c])
    return b


def inflow_bc(prm, plane: str, lo, hi, d_p0, ro_s0, vel, pi_count: int, pi_factor: float,
              min_radius: float, max_radius: float, face=None, phases=(1,), mi_time: float = 0.0,
              start_time: float = 0.0, end_time: float = 1.0e30, layout_seed: int = 0):
    """A dem_inflow_bc for a boundary with extents lo..hi (BC_X_w/BC_Y_s/BC_Z_b ..
    BC_X_e/BC_Y_n/BC_Z_t) on plane `plane`.

    The seeding layout follows LAYOUT_DEM_MI_NS/_EW (layout_mi_dem.f:96-420)
    for a boundary with no excluded cells and no STL facets across it: WMAX x
    HMAX windows of width WINDOW = min(PLEN/WMAX, QLEN/HMAX), centred on the
    boundary, OFFSET one largest diameter off the plane; the windows are
    visited in a seeded random order (the reference draws that permutation
    with RANDOM_NUMBER).  The DES-cell box of the entering test is
    SET_DEM_BCMI_IJK's (set_bc_dem_mi.f:466-522).  d_p0, ro_s0 and vel are per
    phase (vel: BC_U_s, BC_V_s, BC_W_s); `phases` are the 1-based phases
    injected (one entry: monodisperse; several: a DEM_BC_POLY_LAYOUT of 10000
    slots split equally).  `face` defaults to the plane's coordinate.  The
    returned structure keeps its layout arrays alive."""
    import numpy as np
    from . import abi
    b = abi.DemInflowBC()
    b.plane = ord(plane)
    normal = {"N": 1, "S": 1, "E": 0, "W": 0, "T": 2, "B": 2}[plane]
    pa, qa = {1: (0, 2), 0: (1, 2), 2: (0, 1)}[normal]
    do_k = not prm.no_k
    max_dia = max(float(d_p0[m - 1]) for m in phases)
    plen = float(hi[pa] - lo[pa])
    wmax = int(math.floor(float(np.float32(plen / max_dia))))
    if qa == 2 and not do_k:
        qlen = max_dia
    else:
        qlen = float(hi[qa] - lo[qa])
    hmax = int(math.floor(float(np.float32(qlen / max_dia))))
    if wmax < 1 or hmax < 1:
        raise ValueError("inflow boundary narrower than the largest diameter")
    shift = -1.0 if plane in ("N", "E", "T") else 1.0
    b.offset = float(lo[normal]) + max_dia * shift
    window = min(plen / wmax, qlen / hmax)
    b.window = window
    mp0 = float(lo[pa]) + 0.5 * (plen - wmax * window)
    mesh_p = [mp0 + (lc - 1) * window for lc in range(1, wmax + 1)]
    if qa == 2 and not do_k:
        mesh_q = [0.0]
    else:
        mq0 = float(lo[qa]) + 0.5 * (qlen - hmax * window)
        mesh_q = [mq0 + (lc - 1) * window for lc in range(1, hmax + 1)]
    occ = wmax * hmax
    perm = np.random.default_rng(layout_seed).permutation(occ)  # RAND_MAP, 0-based
    P = np.zeros(occ)
    Q = np.zeros(occ)
    lc = 0
    for h in range(hmax):
        for w in range(wmax):
            ll = perm[lc]
            P[ll] = mesh_p[w]
            Q[ll] = mesh_q[h] if len(mesh_q) > h else mesh_q[0]
            lc += 1
    b.occupants = occ
    b.vacancy = 1
    b.pi_count = int(pi_count)
    b.pi_factor = float(pi_factor)
    b.mi_time = float(mi_time)
    b.start_time = float(start_time)
    b.end_time = float(end_time)
    if len(phases) > 1:
        layout = np.repeat(np.asarray(phases, dtype=np.int32), -(-10000 // len(phases)))[:10000].copy()
        b.polydisperse = 1
    else:
        layout = np.asarray([phases[0]], dtype=np.int32)
        b.polydisperse = 0
    b.n_layout = int(layout.size)
    P = np.ascontiguousarray(P)
    Q = np.ascontiguousarray(Q)
    b.p = P.ctypes.data_as(C.POINTER(C.c_double))
    b.q = Q.ctypes.data_as(C.POINTER(C.c_double))
    b.poly_layout = layout.ctypes.data_as(C.POINTER(C.c_int32))
    b._keep = (P, Q, layout)
    for m in range(len(d_p0)):
        b.d_p0[m] = float(d_p0[m])
        b.ro_s0[m] = float(ro_s0[m])
        for c in range(3):
            b.vel[m][c] = float(vel[m][c])
    # SET_DEM_BCMI_IJK: IofbcPOS is NINT-based, IofPOS FLOOR-based; 1-based
    # with one ghost layer (interior 2..dg_imax+1)
    start = (prm.dg_xstart, prm.dg_ystart, prm.dg_zstart)
    inv = (prm.dg_dxinv, prm.dg_dyinv, prm.dg_dzinv)
    nmax = (prm.dg_imax, prm.dg_jmax, prm.dg_kmax)
    for a in range(3):
        if a == 2 and not do_k:
            b.dg_lo[2] = b.dg_hi[2] = 1
            continue
        if a == normal:
            ofpos = lambda x: int(math.floor((x - start[a]) * inv[a])) + 2
            if shift < 0:   # 'N', 'E', 'T'
                b.dg_lo[a] = ofpos(lo[a] + min_radius)
                b.dg_hi[a] = ofpos(hi[a] + max_radius)
            else:
                b.dg_lo[a] = ofpos(lo[a] - max_radius)
                b.dg_hi[a] = ofpos(hi[a] - min_radius)
        else:
            b.dg_lo[a] = max(_nint((lo[a] - start[a]) * inv[a]) + 1 - 1, 2)
            b.dg_hi[a] = min(_nint((hi[a] - start[a]) * inv[a]) + 1 + 1, nmax[a] + 1)
    b.face = float(lo[normal] if face is None else face)
    return b
