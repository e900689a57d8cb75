"""Seeded synthetic DEM workloads (no dataset is involved in the reference's
DEM benchmarks; these follow the shapes the workloads are specified with).

- `settling_4k`      4,000 monodisperse 1 mm spheres, LSD, 12x60x12 mm box,
                     lattice 1.1 d with +-0.04 d jitter (the CPU-runnable case).
- `hertz_rsa_1m`     1,000,000 lognormal spheres (median 1 mm, sigma 0.25,
                     clipped 0.5-2 mm), Hertz E=1e7, periodic x/z, bottom
                     wall, random sequential placement at 40 % solids.
- `coupled_500k`     500,000 spheres of 0.5 mm in a 64x256x64 fluid grid.
- `batched_256`      256 independent settling columns (the 4,000-sphere box
                     scaled in height to each count), counts lognormal in
                     [2,000, 200,000] summing to about 6,000,000, kn
                     U[200, 2000] N/m and friction U[0.1, 0.5] per system.

Particles are numbered in DES-cell order (k, then i, then j fastest, the
order of DG_FUNIJK), which is a free choice of the input and gives the
neighbour gathers spatial locality.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from . import params as P

SEED_BASE = 1000


def _rsa_numba():
    import numba as nb

    @nb.njit(cache=False)
    def rsa(diam, lo, hi, periodic, cell, ncell, seed, max_attempts, grow):
        n = diam.shape[0]
        pos = np.zeros((n, 3))
        cap = 64
        grid = -np.ones((ncell[0] * ncell[1] * ncell[2], cap), dtype=np.int64)
        gcnt = np.zeros(ncell[0] * ncell[1] * ncell[2], dtype=np.int64)
        np.random.seed(seed)
        y_top = hi[1]
        L = hi - lo
        placed = 0
        for i in range(n):
            r = 0.5 * diam[i]
            ok = False
            att = 0
            while not ok:
                att += 1
                if att > max_attempts:
                    y_top = y_top + grow
                    att = 0
                x = np.empty(3)
                for a in range(3):
                    if a == 1:
                        x[a] = lo[1] + r + np.random.random() * (min(y_top, hi[1] + 1e9) - lo[1] - 2 * r)
                    elif periodic[a]:
                        x[a] = lo[a] + np.random.random() * L[a]
                    else:
                        x[a] = lo[a] + r + np.random.random() * (L[a] - 2 * r)
                ci = np.empty(3, dtype=np.int64)
                for a in range(3):
                    ci[a] = int((x[a] - lo[a]) / cell[a])
                    if ci[a] < 0:
                        ci[a] = 0
                    if ci[a] >= ncell[a]:
                        ci[a] = ncell[a] - 1
                ok = True
                for dk in range(-1, 2):
                    if not ok:
                        break
                    for di in range(-1, 2):
                        if not ok:
                            break
                        for dj in range(-1, 2):
                            c0 = ci[0] + di
                            c1 = ci[1] + dj
                            c2 = ci[2] + dk
                            if periodic[0]:
                                c0 = (c0 + ncell[0]) % ncell[0]
                            if periodic[2]:
                                c2 = (c2 + ncell[2]) % ncell[2]
                            if c0 < 0 or c0 >= ncell[0] or c1 < 0 or c1 >= ncell[1] or c2 < 0 or c2 >= ncell[2]:
                                continue
                            g = (c2 * ncell[0] + c0) * ncell[1] + c1
                            for s in range(gcnt[g]):
                                j = grid[g, s]
                                d2 = 0.0
                                for a in range(3):
                                    d = x[a] - pos[j, a]
                                    if periodic[a]:
                                        if d > 0.5 * L[a]:
                                            d -= L[a]
                                        elif d < -0.5 * L[a]:
                                            d += L[a]
                                    d2 += d * d
                                rr = r + 0.5 * diam[j]
                                if d2 < rr * rr:
                                    ok = False
                                    break
                            if not ok:
                                break
                if ok:
                    g = (ci[2] * ncell[0] + ci[0]) * ncell[1] + ci[1]
                    if gcnt[g] >= cap:
                        ok = False
                        continue
                    for a in range(3):
                        pos[i, a] = x[a]
                    grid[g, gcnt[g]] = i
                    gcnt[g] += 1
                    placed += 1
        return pos, y_top

    return rsa


def random_sequential_placement(diam, lo, hi, periodic, seed, region_top, max_attempts=4000, grow_frac=0.005):
    """Places spheres (largest first) uniformly at random without overlap in
    [lo, (hi.x, region_top, hi.z)], raising the region top by grow_frac of its
    height whenever max_attempts consecutive tries fail.  Returns positions
    (in the input order of `diam`) and the final region top."""
    order = np.argsort(-diam, kind="stable")
    d_sorted = diam[order]
    lo = np.asarray(lo, float)
    hi_reg = np.asarray(hi, float).copy()
    hi_reg[1] = region_top
    dmax = float(d_sorted[0])
    ncell = np.maximum(((np.asarray(hi, float) - lo) / dmax).astype(np.int64), 1)
    cell = (np.asarray(hi, float) - lo) / ncell
    rsa = _rsa_numba()
    pos_sorted, top = rsa(d_sorted, lo, hi_reg, np.asarray(periodic, np.bool_), cell, ncell,
                          int(seed) % (2**31), max_attempts, grow_frac * (region_top - lo[1]))
    pos = np.empty_like(pos_sorted)
    pos[order] = pos_sorted
    return pos, float(top)


def _sort_by_des_cell(prm, pos):
    """Permutation that orders particles by DG_FUNIJK cell (j fastest)."""
    li = np.floor((pos[:, 0] - prm.dg_xstart) * prm.dg_dxinv).astype(np.int64)
    lj = np.floor((pos[:, 1] - prm.dg_ystart) * prm.dg_dyinv).astype(np.int64)
    lk = np.floor((pos[:, 2] - prm.dg_zstart) * prm.dg_dzinv).astype(np.int64)
    key = (lk * (prm.dg_imax + 2) + li) * (prm.dg_jmax + 2) + lj
    return np.argsort(key, kind="stable")


def _arrays(pos, vel, omega, radius, rho):
    n = pos.shape[0]
    _, pmass, omoi = P.particle_props(radius, rho)
    return {
        "pos": np.ascontiguousarray(pos.T), "vel": np.ascontiguousarray(vel.T),
        "omega": np.ascontiguousarray(omega.T), "radius": radius, "pmass": pmass, "omoi": omoi,
        "state": np.full(n, abi.DEM_STATE_NORMAL, np.int8), "phase": np.ones(n, np.int32),
    }


def hertz_rsa(n=1_000_000, box=(0.1, 0.4, 0.1), solids=0.40, seed=SEED_BASE + 1,
              precision=abi.DEM_PREC_FP64, nsn=25, cache_dir=None, inflate=1.0):
    """1M polydisperse Hertzian spheres: lognormal d (median 1 mm, sigma
    0.25, clipped to [0.5, 2] mm), rho 2500, E 1e7, nu 0.3, e_n = e_t = 0.85,
    mu 0.3, mu_r 0.01, periodic x/z, flat bottom wall; random sequential
    placement with the region height set for `solids` volume fraction.
    The placement is cached as .npz in `cache_dir` when given."""
    rng = np.random.default_rng(seed)
    d = np.clip(1e-3 * np.exp(rng.normal(0.0, 0.25, n)), 0.5e-3, 2.0e-3)
    vol = float(np.sum((math.pi / 6.0) * d ** 3))
    top = vol / (solids * box[0] * box[2])
    cache = None
    if cache_dir is not None:
        from pathlib import Path
        cache = Path(cache_dir) / f"hertz_rsa_{n}_{seed}_{box[0]:.4g}_{box[2]:.4g}_{solids:.3f}.npz"
    if cache is not None and cache.exists():
        z = np.load(cache)
        pos, top_final = z["pos"], float(z["top"])
    else:
        pos, top_final = random_sequential_placement(d, (0, 0, 0), box, (True, False, True), seed, top)
        if cache is not None:
            cache.parent.mkdir(parents=True, exist_ok=True)
            np.savez(cache, pos=pos, top=top_final)
    vel = np.zeros((n, 3)); omega = np.zeros((n, 3))
    # inflate > 1 grows every sphere after placement, which turns the
    # near-contacts of the random packing into overlapping contacts
    radius = 0.5 * d * inflate
    case = P.DemCase(d_p0=(2e-3 * inflate,), ro_s0=(2500.0,), coll_model="HERTZ", intg_method="EULER",
                     des_en_input=0.85, des_en_wall_input=[0.85], des_et_input=0.85, des_et_wall_input=[0.85],
                     e_young=(1e7,), v_poisson=(0.3,), ew_young=1e7, vw_poisson=0.3,
                     mew=0.3, mew_w=0.3, mew_r=0.01, mew_rw=0.01, grav=(0.0, -9.81, 0.0),
                     domain_hi=box, fluid_cells=(1, 1, 1), periodic=(True, False, True),
                     neighbor_search_n=nsn, force_precision=precision)
    arr = _arrays(pos, vel, omega, radius, np.full(n, 2500.0))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    perm = _sort_by_des_cell(prm, pos)
    arr = _arrays(pos[perm], vel[perm], omega[perm], radius[perm], np.full(n, 2500.0))
    walls = P.default_walls(case.domain_lo, case.domain_hi, periodic=case.periodic)
    info.update({"region_top": top, "region_top_final": top_final,
                 "solids_fraction": vol / (box[0] * box[2] * top_final)})
    return case, prm, arr, walls, info


def settling(n_side=(10, 40, 10), d=1e-3, rho=2500.0, box=(12e-3, 60e-3, 12e-3), spacing=1.1,
             jitter=0.04, vmax=0.1, seed=SEED_BASE, kn=1000.0, en=0.9, mew=0.1,
             precision=abi.DEM_PREC_FP64):
    """Dry settling: cubic lattice of spacing `spacing`*d, jitter +-`jitter`*d,
    velocities U(+-vmax); LSD kn = kn_w, kt = 2/7 kn, e_n, friction mew;
    default box walls; dt = t_coll/50.  n_side=(10,40,10) is the 4,000-sphere
    case."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = n_side
    n = nx * ny * nz
    a = spacing * d
    kk, ii, jj = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    pos = np.empty((n, 3))
    pos[:, 0] = (ii.ravel() + 0.5) * a + (box[0] - nx * a) * 0.5
    pos[:, 1] = (jj.ravel() + 0.5) * a
    pos[:, 2] = (kk.ravel() + 0.5) * a + (box[2] - nz * a) * 0.5
    pos += rng.uniform(-jitter * d, jitter * d, size=pos.shape)
    vel = rng.uniform(-vmax, vmax, size=(n, 3))
    omega = np.zeros((n, 3))
    radius = np.full(n, 0.5 * d)
    case = P.DemCase(d_p0=(d,), ro_s0=(rho,), coll_model="LSD", kn=kn, kn_w=kn,
                     des_en_input=en, des_en_wall_input=[en], mew=mew, mew_w=mew,
                     grav=(0.0, -9.81, 0.0), domain_hi=box, fluid_cells=(1, 1, 1),
                     force_precision=precision)
    arr = _arrays(pos, vel, omega, radius, np.full(n, rho))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    return case, prm, arr, walls, info


def _smooth_noise(rng, shape, sigma_cells, std):
    """Gaussian noise with a Gaussian correlation of sigma_cells, scaled to std."""
    from scipy.ndimage import gaussian_filter
    a = gaussian_filter(rng.normal(0.0, 1.0, shape), sigma=sigma_cells, mode="wrap")
    s = a.std()
    return a * (std / s if s > 0 else 0.0)


def coupled(n=500_000, cells=(64, 256, 64), dx=1e-3, d=0.5e-3, rho=2600.0, kn=500.0, en=0.9, mew=0.1,
            u_sup=1.0, u_std=0.1, corr_cells=4, ro_g=1.2, mu_g=1.8e-5, spacing=1.1, seed=SEED_BASE + 2,
            nsn=25, interp="GARG_2012"):
    """CFD-DEM coupling: n spheres of diameter d on a jittered cubic lattice
    (spacing `spacing`*d) filling the bottom of a cells[0] x cells[1] x cells[2]
    fluid grid of cell size dx, LSD contact, default walls; frozen gas with
    superficial velocity u_sup in y plus seeded Gaussian perturbations (std
    u_std, correlation corr_cells cells) on every component; the interstitial
    velocity is the superficial one divided by the initial void fraction.
    `interp` is DES_INTERP_SCHEME: "GARG_2012" or "NONE".
    Returns (case, prm, arr, walls, info, grid, fields)."""
    rng = np.random.default_rng(seed)
    box = (cells[0] * dx, cells[1] * dx, cells[2] * dx)
    a = spacing * d
    nx, nz = int(box[0] / a), int(box[2] / a)
    ny = int(math.ceil(n / (nx * nz)))
    kk, ii, jj = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    pos = np.empty((nx * ny * nz, 3))
    pos[:, 0] = (ii.ravel() + 0.5) * a
    pos[:, 1] = (jj.ravel() + 0.5) * a
    pos[:, 2] = (kk.ravel() + 0.5) * a
    pos = pos[np.argsort(pos[:, 1] * 1e6 + pos[:, 2] * 1e3 + pos[:, 0], kind="stable")][:n]
    pos += rng.uniform(-0.04 * d, 0.04 * d, size=pos.shape)
    vel = np.zeros((n, 3)); omega = np.zeros((n, 3))
    radius = np.full(n, 0.5 * d)
    case = P.DemCase(d_p0=(d,), ro_s0=(rho,), coll_model="LSD", kn=kn, kn_w=kn, des_en_input=en,
                     des_en_wall_input=[en], mew=mew, mew_w=mew, grav=(0.0, -9.81, 0.0),
                     domain_hi=box, fluid_cells=cells, neighbor_search_n=nsn)
    arr = _arrays(pos, vel, omega, radius, np.full(n, rho))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    perm = _sort_by_des_cell(prm, pos)
    arr = _arrays(pos[perm], vel[perm], omega[perm], radius[perm], np.full(n, rho))
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    # fluid fields on MFiX IJK (one ghost layer, i fastest)
    gi, gj, gk = cells[0] + 2, cells[1] + 2, cells[2] + 2
    vs_cell = np.zeros((gk, gj, gi))
    ci = np.clip((pos[:, 0] / dx).astype(int) + 1, 1, cells[0])
    cj = np.clip((pos[:, 1] / dx).astype(int) + 1, 1, cells[1])
    ck = np.clip((pos[:, 2] / dx).astype(int) + 1, 1, cells[2])
    np.add.at(vs_cell, (ck, cj, ci), (math.pi / 6.0) * d ** 3)
    ep = 1.0 - np.minimum(1.0, vs_cell / dx ** 3)
    ep = np.maximum(ep, 0.35)
    shape = (gk, gj, gi)
    u = _smooth_noise(rng, shape, corr_cells, u_std)
    v = u_sup + _smooth_noise(rng, shape, corr_cells, u_std)
    w = _smooth_noise(rng, shape, corr_cells, u_std)
    fields = {"ep_g": ep.ravel().copy(), "u_g": (u / ep).ravel().copy(), "v_g": (v / ep).ravel().copy(),
              "w_g": (w / ep).ravel().copy()}
    grid = abi.DemFluidGrid()
    grid.imax, grid.jmax, grid.kmax = cells
    grid.drag_model = 0
    grid.interp_scheme = {"GARG_2012": abi.DEM_INTERP_GARG, "NONE": abi.DEM_INTERP_NONE}[interp]
    grid.dx = grid.dy = grid.dz = dx
    grid.ro_g, grid.mu_g = ro_g, mu_g
    grid.ep_star = 0.42
    grid.ur_f_gs = 1.0
    grid.ro_s[0] = rho
    return case, prm, arr, walls, info, grid, fields


def batched_counts(n_sys=256, total=6_000_000, lo=2_000, hi=200_000, sigma=1.0, seed=SEED_BASE + 3):
    """Per-system particle counts: lognormal, clipped to [lo, hi], median
    chosen so that the clipped counts sum to about `total`; multiples of 100
    (10 x 10 lattice columns)."""
    rng = np.random.default_rng(seed)
    raw = rng.lognormal(mean=0.0, sigma=sigma, size=n_sys)
    a, b = float(lo), float(hi)
    for _ in range(80):
        m = 0.5 * (a + b)
        if np.clip(m * raw, lo, hi).sum() < total:
            a = m
        else:
            b = m
    counts = np.clip(np.round(0.5 * (a + b) * raw / 100.0) * 100.0, lo, hi).astype(np.int64)
    return counts, rng


def batched(n_sys=256, total=6_000_000, lo=2_000, hi=200_000, sigma=1.0, seed=SEED_BASE + 3,
            precision=abi.DEM_PREC_SPLIT):
    """Independent dry settling systems for one batch handle.  System s has
    counts[s] = 100 * ny spheres of 1 mm on a 10 x ny x 10 lattice of spacing
    1.1 d (jitter +-0.04 d, velocities U(+-0.1 m/s)) in a 12 x (60 ny / 40) x
    12 mm box with walls, LSD with its own kn and friction, e_n = 0.9, and
    dt = t_coll/50 of its own kn.  Returns (systems, info) where systems is a
    list of (case, prm, arr, walls, info) tuples."""
    counts, rng = batched_counts(n_sys, total, lo, hi, sigma, seed)
    kn = rng.uniform(200.0, 2000.0, n_sys)
    mew = rng.uniform(0.1, 0.5, n_sys)
    systems = []
    for s in range(n_sys):
        ny = int(counts[s] // 100)
        box = (12e-3, 60e-3 * ny / 40.0, 12e-3)
        systems.append(settling(n_side=(10, ny, 10), box=box, seed=seed * 1000 + s, kn=float(kn[s]),
                                mew=float(mew[s]), precision=precision))
    info = {"n_systems": n_sys, "n_particles": int(counts.sum()), "min_count": int(counts.min()),
            "max_count": int(counts.max()), "median_count": int(np.median(counts))}
    return systems, info


HOPPER_BOX = (0.2, 0.6, 0.2)


def hopper_case(n, friction=0.4, outlet_d=8, seed=SEED_BASE + 4, d=2e-3, rho=2500.0,
                precision=abi.DEM_PREC_SPLIT, jitter=0.04, spacing=1.1, half_angle=30.0):
    """One hopper-discharge case: a 20 x 60 x 20 cm box with a conical bottom
    (half-angle 30 degrees) and an outlet of `outlet_d` particle diameters,
    `n` spheres of d = 2 mm filled on a lattice of spacing 1.1 d with +-0.04 d
    jitter above the cone, Hertz E = 1e7 Pa, nu = 0.3, e_n = e_t = 0.85,
    friction `friction` with particles and walls.  Particles that fall out
    through the outlet leave the domain and are removed as rogue."""
    box = HOPPER_BOX
    (vertex, norm), geo = P.hopper_walls((0.0, 0.0, 0.0), box, half_angle_deg=half_angle,
                                         outlet_diam=outlet_d * d)
    rng = np.random.default_rng(seed)
    a = spacing * d
    m = int((min(box[0], box[2]) - a) // a)          # lattice sites per row across the box
    layers = -(-n // (m * m))
    y_base = geo["y_top"] + a
    if y_base + layers * a > box[1] - a:
        raise ValueError("hopper fill does not fit in the box")
    kk, ii, jj = np.meshgrid(np.arange(m), np.arange(m), np.arange(layers), indexing="ij")
    pos = np.empty((m * m * layers, 3))
    pos[:, 0] = (ii.ravel() + 0.5) * a + 0.5 * (box[0] - m * a)
    pos[:, 1] = y_base + jj.ravel() * a
    pos[:, 2] = (kk.ravel() + 0.5) * a + 0.5 * (box[2] - m * a)
    pos = pos[np.argsort(pos[:, 1], kind="stable")][:n]      # the n lowest sites
    pos += rng.uniform(-jitter * d, jitter * d, size=pos.shape)
    vel = np.zeros((n, 3))
    omega = np.zeros((n, 3))
    radius = np.full(n, 0.5 * d)
    case = P.DemCase(d_p0=(d,), ro_s0=(rho,), coll_model="HERTZ", intg_method="EULER",
                     des_en_input=0.85, des_en_wall_input=[0.85], des_et_input=0.85, des_et_wall_input=[0.85],
                     e_young=(1e7,), v_poisson=(0.3,), ew_young=1e7, vw_poisson=0.3,
                     mew=friction, mew_w=friction, grav=(0.0, -9.81, 0.0), domain_hi=box,
                     fluid_cells=(1, 1, 1), remove_rogue=True, force_precision=precision)
    arr = _arrays(pos, vel, omega, radius, np.full(n, rho))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    perm = _sort_by_des_cell(prm, pos)
    arr = _arrays(pos[perm], vel[perm], omega[perm], radius[perm], np.full(n, rho))
    info.update(geo)
    info.update({"n": n, "friction": friction, "outlet_d": outlet_d})
    return case, prm, arr, (vertex, norm), info


def hopper_requests(n_req, rate, seed=SEED_BASE + 4, n_lo=5_000, n_hi=500_000, steps=20_000):
    """A Poisson request stream of hopper cases: arrival times (s) with mean
    rate `rate`, particle counts log-uniform in [n_lo, n_hi], friction
    U[0.2, 0.6], outlet U{6..10} diameters, `steps` DES steps each."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_req))
    n = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), n_req)).astype(np.int64)
    mu = rng.uniform(0.2, 0.6, n_req)
    outlet = rng.integers(6, 11, n_req)
    return [{"rid": k, "arrival": float(t[k]), "n": int(n[k]), "friction": float(mu[k]),
             "outlet_d": int(outlet[k]), "seed": int(seed * 1000 + k), "steps": int(steps)}
            for k in range(n_req)]
