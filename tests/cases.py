"""Small DEM cases shared by the oracle and GPU parity tests.

Each builder returns (params, arrays, walls) where arrays holds the DES
arrays in Fortran layout ((3, n) for vectors, 1-based phases).
"""
import math

import numpy as np

from mfix_dem import abi
from mfix_dem import params as P


def state_arrays(pos, vel, omega, radius, rho, phase=None):
    n = pos.shape[1]
    _, pmass, omoi = P.particle_props(radius, rho)
    st = np.full(n, abi.DEM_STATE_NORMAL, dtype=np.int8)
    ph = np.ones(n, np.int32) if phase is None else np.asarray(phase, np.int32)
    return {"pos": pos, "vel": vel, "omega": omega, "radius": np.asarray(radius, float),
            "pmass": pmass, "omoi": omoi, "state": st, "phase": ph}


def dem01_case(intg, kn, en):
    """DEM01 (tests/dem/DEM01/mfix.dat): one 0.2 m sphere dropped from
    y = 0.5 m in a 1 m box, LSD, default walls, one DES cell."""
    case = P.DemCase(d_p0=(0.2,), ro_s0=(2600.0,), coll_model="LSD", intg_method=intg,
                     kn=kn, kn_w=kn, des_en_input=en, des_en_wall_input=[en],
                     grav=(0.0, -9.80665, 0.0), neighbor_search_n=99, desgridsearch=(1, 1, 1))
    arr = state_arrays(np.array([[0.6], [0.5], [0.6]]), np.zeros((3, 1)), np.zeros((3, 1)),
                       np.array([0.1]), np.array([2600.0]))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    return case, prm, arr, walls


def dem03_case(en, en_w):
    """DEM03 (tests/dem/DEM03/mfix.dat): two 1 mm spheres (rho 2e4 and 1e4,
    phases 1 and 2) stacked between the bottom and top walls of a 1 x 1.8 mm
    x 1 m box, each overlapping its wall and the other; LSD KN = KN_W = 1e3,
    KT_FAC = KT_W_FAC = 1, DES_ETAT_FAC = DES_ETAT_W_FAC = 1, no friction,
    Adams-Bashforth, one DES cell."""
    case = P.DemCase(n_phases=2, d_p0=(1e-3, 1e-3), ro_s0=(2.0e4, 1.0e4), coll_model="LSD",
                     intg_method="ADAMS_BASHFORTH", kn=1.0e3, kn_w=1.0e3, kt_fac=1.0, kt_w_fac=1.0,
                     des_etat_fac=1.0, des_etat_w_fac=1.0, des_en_input=en, des_en_wall_input=[en_w, en_w],
                     mew=0.0, mew_w=0.0, grav=(0.0, -9.80665, 0.0), domain_hi=(1.0, 0.0018, 1.0),
                     neighbor_search_n=99, desgridsearch=(1, 1, 1))
    pos = np.array([[0.5, 0.5], [0.00045, 0.00135], [0.5, 0.5]])
    arr = state_arrays(pos, np.zeros((3, 2)), np.zeros((3, 2)), np.array([0.0005, 0.0005]),
                       np.array([2.0e4, 1.0e4]), phase=[1, 2])
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    return case, prm, arr, walls


def dem05_case(model, particle_input):
    """DEM05 (tests/dem/DEM05/mfix.dat): 93 spheres of 5 mm in a 0.5 x 0.1 x
    0.5 m box without gravity: 31 phase-1 spheres (rho 4000) strike the floor
    at impact angles 0-65 degrees, 31 strike fixed phase-2 targets (rho
    5000; particles 63-93, reset every step by USR2_DES); Adams-Bashforth,
    friction 0.092, elastic (e_n = e_t = 1).  model: "LSD" (KN = KN_W =
    1.72e7, KT_FAC = 1.48/1.72) or "HERTZ" (E = 380e9 / 70e9, wall 70e9,
    nu = 0.23 / 0.25, wall 0.25)."""
    a = np.asarray(particle_input, dtype=np.float64).reshape(-1, 8)
    n = a.shape[0]
    kw = dict(n_phases=2, d_p0=(5.0e-3, 5.0e-3), ro_s0=(4.0e3, 5.0e3), intg_method="ADAMS_BASHFORTH",
              des_en_input=1.0, des_en_wall_input=[1.0, 1.0], mew=0.092, mew_w=0.092,
              grav=(0.0, 0.0, 0.0), domain_hi=(0.5, 0.1, 0.5), fluid_cells=(5, 1, 5))
    if model == "LSD":
        case = P.DemCase(coll_model="LSD", kn=1.72e7, kn_w=1.72e7, kt_fac=1.48 / 1.72, kt_w_fac=1.48 / 1.72, **kw)
    else:
        case = P.DemCase(coll_model="HERTZ", e_young=(380.0e9, 70.0e9), v_poisson=(0.23, 0.25),
                         ew_young=70.0e9, vw_poisson=0.25, des_et_input=1.0, des_et_wall_input=[1.0, 1.0], **kw)
    phase = np.where(a[:, 4] > 4500.0, 2, 1)
    arr = state_arrays(a[:, 0:3].T.copy(), a[:, 5:8].T.copy(), np.zeros((3, n)), a[:, 3].copy(), a[:, 4].copy(),
                       phase=phase)
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    return case, prm, arr, walls


def settling_case(n_side=(6, 20, 6), d=1e-3, rho=2500.0, box=(12e-3, 60e-3, 12e-3),
                  spacing=1.1, jitter=0.04, vmax=0.1, seed=1000, coll="LSD", intg="EULER",
                  kn=1000.0, en=0.9, mew=0.1, nsn=25, polydisperse=0.0, mew_r=0.0,
                  periodic=(False, False, False), precision=abi.DEM_PREC_FP64):
    """Dry granular settling: spheres on a cubic lattice of spacing `spacing`*d
    with seeded jitter and velocities, default box walls, gravity -9.81 in y.
    The 4,000-sphere LSD instance of this builder (n_side=(10,40,10)) is the
    reference-runnable settling workload; smaller n_side are parity cases."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = n_side
    n = nx * ny * nz
    a = spacing * d
    # order: y fastest, then x, then z (the DES cell key order, j fastest)
    kk, ii, jj = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    x0 = np.array(box) * 0.0
    pos = np.empty((3, n))
    pos[0] = (ii.ravel() + 0.5) * a + (box[0] - nx * a) * 0.5
    pos[1] = (jj.ravel() + 0.5) * a + 0.5 * a * 0.0 + 1e-5
    pos[2] = (kk.ravel() + 0.5) * a + (box[2] - nz * a) * 0.5
    pos += rng.uniform(-jitter * d, jitter * d, size=pos.shape)
    vel = rng.uniform(-vmax, vmax, size=(3, n))
    omega = np.zeros((3, n))
    if polydisperse > 0:
        diam = np.clip(d * np.exp(rng.normal(0.0, polydisperse, n)), 0.5 * d, 2.0 * d)
        diam = np.minimum(diam, a * 0.95)
    else:
        diam = np.full(n, d)
    radius = 0.5 * diam
    arr = state_arrays(pos, vel, omega, radius, np.full(n, rho))
    dmax = float(np.max(diam))
    kw = {}
    if coll == "HERTZ":
        kw = dict(e_young=(1e7,), v_poisson=(0.3,), ew_young=1e7, vw_poisson=0.3,
                  des_et_input=en, des_et_wall_input=[en])
    case = P.DemCase(d_p0=(dmax,), ro_s0=(rho,), coll_model=coll, intg_method=intg,
                     kn=kn, kn_w=kn, des_en_input=en, des_en_wall_input=[en],
                     mew=mew, mew_w=mew, mew_r=mew_r, mew_rw=mew_r,
                     grav=(0.0, -9.81, 0.0), domain_hi=box, fluid_cells=(1, 1, 1),
                     neighbor_search_n=nsn, periodic=periodic, force_precision=precision, **kw)
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi, periodic=periodic)
    return case, prm, arr, walls


def make_system(cls, prm, arr, walls, **kw):
    s = cls(prm, arr["pos"].shape[1], **kw)
    s.set_walls(*walls)
    s.upload_state(arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"],
                   arr["omoi"], arr["state"], arr["phase"])
    s.init_neighbors()
    return s


def coupled_case(cells=(8, 24, 8), n=1500, **kw):
    """A small CFD-DEM case on a cells[0] x cells[1] x cells[2] grid of 1 mm cells."""
    from mfix_dem import configs
    return configs.coupled(n=n, cells=cells, **kw)


def make_coupled(cls, case_tuple, **kw):
    case, prm, arr, walls, info, grid, fields = case_tuple
    s = make_system(cls, prm, arr, walls, **kw)
    s.set_gas_fields(grid, fields["ep_g"], fields["u_g"], fields["v_g"], fields["w_g"])
    return s


def hopper_wall_case(n=1500, d=2e-3, rho=2500.0, friction=0.4, outlet_d=8, seed=44, precision=abi.DEM_PREC_FP64):
    """Spheres against the cone of a hopper-discharge case (the 20 x 60 x 20 cm
    box with a 30 degree conical bottom, mfix_dem.configs.hopper_case): each
    sits off a random interior point of a random cone facet, at a gap from
    the facet's plane drawn from [-0.01, 0.05] mm (some overlap it at the
    start), moving toward it at up to 0.5 m/s with a random tangential
    velocity up to 0.5 m/s, so wall contacts with tangential history and
    Coulomb slip start within a few steps, on the slanted facets binned by
    TRI_BOX_OVERLAP.  Spheres closer than a diameter to an earlier one are
    dropped."""
    from mfix_dem import configs
    box = configs.HOPPER_BOX
    (vertex, norm), geo = P.hopper_walls((0.0, 0.0, 0.0), box, half_angle_deg=30.0, outlet_diam=outlet_d * d)
    rng = np.random.default_rng(seed)
    axis = np.array([0.5 * box[0], 0.0, 0.5 * box[2]])
    r = 0.5 * d
    cone = np.array([f for f in range(vertex.shape[0]) if 0.1 < abs(norm[f, 1]) < 0.99])
    pos, vel = [], []
    for _ in range(20 * n):
        if len(pos) >= n:
            break
        f = cone[rng.integers(cone.shape[0])]
        a, b, c = vertex[f].T                 # vertex[f][c][v]: a column per vertex
        u, v = rng.uniform(0.1, 0.8, 2)
        if u + v > 0.9:
            u, v = 0.9 - v, 0.9 - u
        q = a + u * (b - a) + v * (c - a)
        nrm = np.cross(b - a, c - a)
        nrm /= np.linalg.norm(nrm)
        to_axis = axis - q
        to_axis[1] = 0.0
        if nrm @ to_axis < 0:                 # orient toward the inside of the cone
            nrm = -nrm
        x = q + nrm * (r + rng.uniform(-1e-5, 5e-5))
        if x[1] < geo["y_out"] + 2 * d or x[1] > geo["y_top"] - 2 * d:
            continue
        if pos and np.min(np.linalg.norm(np.asarray(pos) - x, axis=1)) < d * 1.001:
            continue
        tang = rng.uniform(-0.5, 0.5, 3)
        tang -= (tang @ nrm) * nrm
        pos.append(x)
        vel.append(-nrm * rng.uniform(0.0, 0.5) + tang)
    pos, vel = np.asarray(pos), np.asarray(vel)
    n = pos.shape[0]
    case = P.DemCase(d_p0=(d,), ro_s0=(rho,), coll_model="HERTZ", intg_method="EULER",
                     des_en_input=0.85, des_en_wall_input=[0.85], des_et_input=0.85, des_et_wall_input=[0.85],
                     e_young=(1e7,), v_poisson=(0.3,), ew_young=1e7, vw_poisson=0.3,
                     mew=friction, mew_w=friction, grav=(0.0, -9.81, 0.0), domain_hi=box,
                     fluid_cells=(1, 1, 1), remove_rogue=True, force_precision=precision, neighbor_search_n=25)
    arr = state_arrays(pos.T.copy(), vel.T.copy(), np.zeros((3, n)), np.full(n, r), np.full(n, rho))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    return case, prm, arr, (vertex, norm)


def bimodal_case(periodic=(False, False, False), seed=77, coll="LSD"):
    """Three 8 mm spheres among ~11,000 1 mm spheres in a 24 mm box (36 x 24
    x 36 mm when x and z are periodic, which needs three DES cells): the
    first two large ones have the lowest indices, so their half-list rows
    hold every small neighbour (a few hundred, past any fixed row length),
    and the last has the highest, so hundreds of rows end in it (a long
    incoming list).  Small spheres on a lattice of spacing 1.02 d with
    jitter, none overlapping a large one; LSD, default walls."""
    rng = np.random.default_rng(seed)
    d, D = 1e-3, 8e-3
    box = (36e-3, 24e-3, 36e-3) if periodic[0] else (24e-3, 24e-3, 24e-3)
    a = 1.02 * d
    axes = []
    for L in box:
        m = int(L // a)
        axes.append((np.arange(m) + 0.5) * a + 0.5 * (L - m * a))
    small = np.stack(np.meshgrid(*axes, indexing="ij"), 0).reshape(3, -1)
    # with periodic x and z the first large sphere straddles the periodic
    # faces, so its neighbours come through the image shift
    big = (np.array([[1.0, 12.0, 1.0], [18.0, 12.0, 18.0], [12.0, 12.0, 30.0]]) if periodic[0] else
           np.array([[6.0, 12.0, 6.0], [18.0, 12.0, 18.0], [12.0, 12.0, 12.0]])).T * 1e-3
    sep = small[:, :, None] - big[:, None, :]
    for ax in range(3):
        if periodic[ax]:
            sep[ax] -= box[ax] * np.round(sep[ax] / box[ax])
    dist = np.sqrt((sep ** 2).sum(axis=0)).min(axis=1)
    small = small[:, dist > 0.5 * (D + d) * 1.01]
    small = small + rng.uniform(-0.01 * d, 0.01 * d, size=small.shape)
    pos = np.concatenate([big[:, :2], small, big[:, 2:]], axis=1)
    n = pos.shape[1]
    radius = np.full(n, 0.5 * d)
    radius[[0, 1, n - 1]] = 0.5 * D
    vel = rng.uniform(-0.05, 0.05, size=(3, n))
    arr = state_arrays(pos, vel, np.zeros((3, n)), radius, np.full(n, 2500.0))
    kw = {}
    if coll == "HERTZ":
        kw = dict(e_young=(1e7,), v_poisson=(0.3,), ew_young=1e7, vw_poisson=0.3,
                  des_et_input=0.9, des_et_wall_input=[0.9])
    case = P.DemCase(d_p0=(D,), ro_s0=(2500.0,), coll_model=coll, intg_method="EULER",
                     kn=1000.0, kn_w=1000.0, des_en_input=0.9, des_en_wall_input=[0.9],
                     mew=0.2, mew_w=0.2, grav=(0.0, -9.81, 0.0), domain_hi=box, fluid_cells=(1, 1, 1),
                     neighbor_search_n=25, periodic=periodic,
                     desgridsearch=(3, 2, 3) if periodic[0] else (None, None, None), **kw)
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi, periodic=periodic)
    return case, prm, arr, walls
