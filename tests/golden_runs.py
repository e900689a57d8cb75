"""The reference's regression runs DEM02, DEM04 and the homogeneous cooling
system, as case builders plus drivers that step any system with the
library's host interface (the CPU oracle or the CUDA library) and record
what the reference's user routines record.

DEM02 (tests/dem/DEM02): a 0.2 m sphere bouncing on the floor of the default
STL box (Adams-Bashforth); USR2_DES (usr2_des.f) keeps the maximum height of
each bounce, max(y before, y after) at the step where v_y turns from
positive to negative.
DEM04 (tests/dem/DEM04): a 1 mm sphere launched along a rough floor at
0.1 m/s slides until it rolls; WRITE_USR1 (write_usr1.f, called every DEM
step because USR_DT = 1e-8) records, at the first step where the slip
velocity v_x + omega_z*r is COMPARE-equal to 1e-6 or negative, the scaled
time |MEW*g/u0|*t and the scaled velocities |v_x/u0| and |omega_z*r/u0|.
Homogeneous cooling (legacy_tests/dem-tests/homogeneous-cooling-system): 195
elastic frictionless 1 cm spheres (CGS units) in a fully periodic 8 cm cube
with a neighbour search every step; USR0_DES/USR2_DES (usr0_des.f,
usr2_des.f) print DES_GRANULAR_TEMPERATURE's mean granular temperature,
kinetic energy and mean velocity every 0.05 s of solids time.
"""
import math

import numpy as np

from cases import dem01_case, state_arrays
from mfix_dem import params as P


def pure_granular_steps(prm, tstop):
    """FACTOR = CEILING(real((TSTOP-TIME)/DTSOLID)) with TIME = 0
    (des_time_march.f, DES_TIME_INIT): the number of DES steps of a pure
    granular run, the quotient rounded to single precision first."""
    return math.ceil(float(np.float32(tstop / prm.dtsolid)))


# ---- DEM02 ---------------------------------------------------------------
def dem02_case(kn, en):
    """DEM02's deck is DEM01's with Adams-Bashforth, MEW = MEW_W = 0 and
    KN = KN_W, DES_EN_INPUT = DES_EN_WALL_INPUT from the sweep."""
    return dem01_case("ADAMS_BASHFORTH", kn, en)


def dem02_heights(s, prm, tstop=10.0, last_bounce=50, max_bounce=50):
    """MAX_HEIGHT(0:k) of USR2_DES, stepping until bounce `last_bounce` is
    recorded or TSTOP is reached."""
    st = s.download_state()
    ypos_o, yvel_o = float(st["pos"][1, 0]), float(st["vel"][1, 0])
    heights = [ypos_o]
    count = 0
    for nn in range(1, pure_granular_steps(prm, tstop) + 1):
        s.step(1, nn)
        st = s.download_state()
        y, v = float(st["pos"][1, 0]), float(st["vel"][1, 0])
        if v < 0.0 and yvel_o > 0.0 and count < max_bounce:
            count += 1
            heights.append(max(ypos_o, y))
            if count >= last_bounce:
                break
        yvel_o, ypos_o = v, y
    return heights


# ---- DEM04 ---------------------------------------------------------------
GRAV_DEFAULT = -9.80665   # GRAVITY keyword default, m/s^2


def dem04_case(mew):
    """tests/dem/DEM04/mfix.dat with MEW = MEW_W = mew."""
    case = P.DemCase(d_p0=(1.0e-3,), ro_s0=(1.0e4,), coll_model="LSD", intg_method="ADAMS_BASHFORTH",
                     kn=1.0e4, kn_w=1.0e4, kt_fac=1.0, kt_w_fac=1.0, des_etat_fac=1.0, des_etat_w_fac=1.0,
                     des_en_input=1.0, des_en_wall_input=[1.0], mew=mew, mew_w=mew,
                     grav=(0.0, GRAV_DEFAULT, 0.0), neighbor_search_n=99, desgridsearch=(1, 1, 1))
    arr = state_arrays(np.array([[0.001], [0.0005], [0.5]]), np.array([[0.1], [0.0], [0.0]]), np.zeros((3, 1)),
                       np.array([0.0005]), np.array([1.0e4]))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    return case, prm, arr, walls


def compare(v1, v2, tol_com=1.0e-4, small=1.0e-15):
    """COMPARE of toleranc_mod.f:138-162."""
    if abs(v1) <= small:
        return abs(v2) <= small
    return abs(v2 / v1 - 1.0) <= tol_com


def dem04_roll(s, prm, mew, tstop=0.02):
    """(scaled time, |v_x/u0|, |omega_z*r/u0|) at the end of slip, or None."""
    st = s.download_state()
    u0 = float(st["vel"][0, 0])
    r = 0.0005
    t = 0.0
    for nn in range(1, pure_granular_steps(prm, tstop) + 1):
        s.step(1, nn)
        t = t + prm.dtsolid
        st = s.download_state()
        vx, wz = float(st["vel"][0, 0]), float(st["omega"][2, 0])
        slip = vx + wz * r
        if compare(abs(slip), 1.0e-6) or slip < 0.0:
            return abs(mew * GRAV_DEFAULT / u0) * t, abs(vx / u0), abs(wz * r / u0)
    return None


# ---- homogeneous cooling ---------------------------------------------------
def hcs_case(particle_input):
    """homogeneous-cooling-system/mfix.dat: CGS, 8 cm fully periodic cube,
    4x4x4 fluid and DES-search cells, LSD KN = KN_W = 1e6, e = 1, no
    friction, no gravity, NEIGHBOR_SEARCH_N = 1, Euler."""
    a = np.asarray(particle_input, dtype=np.float64)
    case = P.DemCase(d_p0=(1.0,), ro_s0=(1.0,), coll_model="LSD", intg_method="EULER",
                     kn=1.0e6, kn_w=1.0e6, des_en_input=1.0, des_en_wall_input=[1.0], mew=0.0, mew_w=0.0,
                     grav=(0.0, 0.0, 0.0), domain_hi=(8.0, 8.0, 8.0), fluid_cells=(4, 4, 4),
                     periodic=(True, True, True), desgridsearch=(4, 4, 4), neighbor_search_n=1)
    arr = state_arrays(a[:, 0:3].T.copy(), a[:, 5:8].T.copy(), np.zeros((3, a.shape[0])), a[:, 3].copy(),
                       a[:, 4].copy())
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi, periodic=case.periodic)
    return case, prm, arr, walls


def granular_temperature(st, pmass):
    """DES_GRANULAR_TEMPERATURE (des_granular_temperature.f:33-191) for
    existing particles: mean velocity, kinetic energy, and USR0_DES's
    (1/3)*sum(GLOBAL_GRAN_TEMP) and (1/3)*sum(DES_VEL_AVG)."""
    keep = st["state"] != 0
    v = st["vel"][:, keep]
    m = pmass[keep]
    n = v.shape[1]
    ke = 0.0
    avg = np.zeros(3)
    for ll in range(n):
        sq = v[0, ll] ** 2 + v[1, ll] ** 2 + v[2, ll] ** 2
        ke = ke + m[ll] / 2.0 * sq
        avg = avg + v[:, ll]
    avg = avg / float(n)
    gt = np.zeros(3)
    for ll in range(n):
        gt = gt + (v[:, ll] - avg) ** 2
    gt = gt / float(n)
    third = float(np.float32(1.0) / np.float32(3.0))
    return third * float(np.sum(gt)), ke, third * float(np.sum(avg))


def hcs_rows(s, prm, pmass, tstop=5.0, usr_dt=0.05):
    """(S_TIME, granular temperature, kinetic energy, mean velocity) at the
    start and at each USR2_DES output (S_TIME + 0.1*DTSOLID past the next
    multiple of USR_DT; the first call only arms the timer) up to TSTOP.
    The output steps follow from the accumulated S_TIME alone, so the
    system is stepped in chunks between them."""
    outs = []
    usr_time = 0.0
    t = 0.0
    for nn in range(1, pure_granular_steps(prm, tstop) + 1):
        t = t + prm.dtsolid
        if usr_time == 0.0:
            usr_time = usr_dt
            continue
        over = t + 0.1 * prm.dtsolid
        if over >= usr_time:
            usr_time = (int(over / usr_dt) + 1) * usr_dt
            outs.append((nn, t))
    rows = [(0.0,) + granular_temperature(s.download_state(), pmass)]
    done = 0
    for nn, t in outs:
        s.step(nn - done, done + 1)
        done = nn
        rows.append((t,) + granular_temperature(s.download_state(), pmass))
    return rows


# ---- DEM06 ----------------------------------------------------------------
# tests/dem/DEM06: one 0.1 mm sphere (rho 2000) released at rest at
# y = 92.5 mm in a 10 x 100 x 10 mm column of gas rising at 0.4 m/s (rho_g
# 1.2, mu_g 1.8e-5; 5 x 20 x 5 fluid cells of 2 x 5 x 2 mm), one-way coupled, with the
# user drag law of usr_drag.f (DEM_DRAG_SINGLE_SPHERE); fluid steps of 1 ms
# each hold CEILING(DT/DTSOLID) DEM steps, the last shortened to land on the
# fluid time.  The gas is uniform and hydrostatic: V_G = 0.4 on every face,
# EP_G = 1 and P_FORCE = -grad(P_g) = (0, RO_g*9.80665, 0) (CALC_PG_GRAD,
# calc_pg_grad.f:70-72), the buoyancy the table's own solution includes.
DEM06_CELLS = (5, 20, 5)


def dem06_case(interp="NONE"):
    from mfix_dem import abi
    case = P.DemCase(d_p0=(1.0e-4,), ro_s0=(2.0e3,), coll_model="LSD", intg_method="EULER",
                     kn=0.1, kn_w=0.1, des_en_input=1.0, des_en_wall_input=[1.0], mew=0.0, mew_w=0.0,
                     grav=(0.0, GRAV_DEFAULT, 0.0), domain_hi=(0.01, 0.10, 0.01), fluid_cells=DEM06_CELLS,
                     desgridsearch=DEM06_CELLS)
    arr = state_arrays(np.array([[0.005], [0.0925], [0.005]]), np.zeros((3, 1)), np.zeros((3, 1)),
                       np.array([5.0e-5]), np.array([2.0e3]))
    prm, info = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    walls = P.default_walls(case.domain_lo, case.domain_hi)
    grid = abi.DemFluidGrid()
    grid.imax, grid.jmax, grid.kmax = DEM06_CELLS
    grid.drag_model = abi.DEM_DRAG_SINGLE_SPHERE
    grid.interp_scheme = abi.DEM_INTERP_NONE if interp == "NONE" else abi.DEM_INTERP_GARG
    grid.dx, grid.dy, grid.dz = 2.0e-3, 5.0e-3, 2.0e-3
    grid.ro_g, grid.mu_g = 1.2, 1.8e-5
    grid.ep_star = 0.42
    grid.ur_f_gs = 1.0
    grid.ro_s[0] = 2.0e3
    grid.usr_d_p0 = 1.0e-4
    nc = (DEM06_CELLS[0] + 2) * (DEM06_CELLS[1] + 2) * (DEM06_CELLS[2] + 2)
    pf = np.zeros((nc, 3))
    pf[:, 1] = 1.2 * -GRAV_DEFAULT
    fields = {"ep_g": np.ones(nc), "u_g": np.zeros(nc), "v_g": np.full(nc, 0.4), "w_g": np.zeros(nc),
              "p_force": pf}
    return case, prm, arr, walls, grid, fields


def dem06_rows(s, prm, tstop=0.35, dt=1.0e-3, usr_dt=0.01):
    """(TIME, y, v_y) at t = 0 and after the fluid step reaching each
    multiple of USR_DT (TIME + 0.1*DT past it), stepping the coupled DEM
    with the sub-steps of DES_TIME_MARCH (des_time_march.f, DES_TIME_INIT
    FACTOR = CEILING(real(DT/DTSOLID)), DES_TIME_STEP's shortened last
    step, DES_TIME_END's restore)."""
    st = s.download_state()
    rows = [(0.0, float(st["pos"][1, 0]), float(st["vel"][1, 0]))]
    dts = prm.dtsolid
    time = 0.0
    usr_time = usr_dt
    nfluid = int(round(tstop / dt))
    for _ in range(nfluid):
        s_time = time
        dtsolid = dts
        factor = math.ceil(float(np.float32(dt / dtsolid)))
        for nn in range(1, factor + 1):
            if s_time >= time + dt:
                break
            if s_time + dtsolid > time + dt:
                dtsolid = time + dt - s_time
                s.set_dtsolid(dtsolid)
            s.step_coupled(1, nn)
            s_time = s_time + dtsolid
        if dtsolid != dts:
            s.set_dtsolid(dts)
        time = time + dt
        if time + 0.1 * dt >= usr_time:
            usr_time = (int((time + 0.1 * dt) / usr_dt) + 1) * usr_dt
            st = s.download_state()
            rows.append((time, float(st["pos"][1, 0]), float(st["vel"][1, 0])))
    return rows
