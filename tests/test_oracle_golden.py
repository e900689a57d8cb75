"""Pins the CPU oracle to the reference's own regression tables.

DEM01 (tests/dem/DEM01 in MFiX): a 0.2 m sphere falls onto the bottom wall
of the default STL box; 38 runs sweep DES_INTG_METHOD (EULER, ADAMS_BASHFORTH),
KN = KN_W and the restitution coefficient.  DEM03 (tests/dem/DEM03): two
particles of different density stacked and compressed between the bottom
and top walls (particle-particle and particle-wall contacts, Adams-Bashforth,
two solids phases); 6 runs sweep the restitution coefficients.  DEM05
(tests/dem/DEM05): oblique impacts of 5 mm spheres on the floor and on fixed
target spheres (sliding and sticking tangential contact with friction,
spins), LSD and Hertz; the tables give rebound angles, spins and tangential
restitution at the end of the run to 4 decimals.  The AUTOTEST
tables print MFiX's values with 8 decimals at the first DEM step past each
output time; the oracle must reproduce every printed value to within the
print resolution (5e-9, plus a small allowance for the rounding of the last
digit).  DEM02 (bounce heights on the floor), DEM04 (slip to roll on a rough
floor) and the homogeneous cooling system (fully periodic, a neighbour
search every step) are described at their tests below.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import golden_runs as G
from cases import dem01_case, dem03_case, dem05_case, make_system
from oracle_ffi import OracleSystem

GOLD = Path(__file__).resolve().parent / "golden"


def _dem01_runs():
    return json.loads((GOLD / "dem01.json").read_text())["runs"]


@pytest.mark.parametrize("run_idx", range(38))
def test_dem01_matches_mfix_table(run_idx):
    run = _dem01_runs()[run_idx]
    case, prm, arr, walls = dem01_case(run["intg"], run["kn"], run["en"])
    s = make_system(OracleSystem, prm, arr, walls)
    # pure granular run: FACTOR = CEILING(real((TSTOP-TIME)/DTSOLID)), des_time_march.f:129
    tstop = 0.5
    factor = math.ceil(float(np.float32(tstop / prm.dtsolid)))
    times, ys, vs = [0.0], [0.5], [0.0]
    t = 0.0
    for nn in range(1, factor + 1):
        s.step(1, nn)
        t = t + prm.dtsolid
        st = s.download_state()
        times.append(t)
        ys.append(st["pos"][1, 0])
        vs.append(st["vel"][1, 0])
    times = np.asarray(times)
    assert len(run["rows"]) == 101
    for tg, yg, vg in run["rows"]:
        k = int(np.argmin(np.abs(times - tg)))
        assert abs(times[k] - tg) <= 5e-9 + 1e-12
        assert abs(ys[k] - yg) <= 5e-9 + 1e-12, (tg, ys[k], yg)
        assert abs(vs[k] - vg) <= 5e-9 + 1e-12, (tg, vs[k], vg)


def _dem03_runs():
    return json.loads((GOLD / "dem03.json").read_text())["runs"]


def _run_pure_granular(s, prm, tstop, record):
    """DES steps of a pure granular run up to TSTOP: FACTOR =
    CEILING(real((TSTOP-TIME)/DTSOLID)) (des_time_march.f:129); returns the
    times and record(state) after every step."""
    factor = math.ceil(float(np.float32(tstop / prm.dtsolid)))
    times, vals = [0.0], [record(s.download_state())]
    t = 0.0
    for nn in range(1, factor + 1):
        s.step(1, nn)
        t = t + prm.dtsolid
        times.append(t)
        vals.append(record(s.download_state()))
    return np.asarray(times), vals


@pytest.mark.parametrize("run_idx", range(6))
def test_dem03_matches_mfix_table(run_idx):
    run = _dem03_runs()[run_idx]
    assert run["intg"] == "ADAMS_BASHFORTH" and run["kn"] == 1000.0
    case, prm, arr, walls = dem03_case(run["en"], run["en_w"])
    s = make_system(OracleSystem, prm, arr, walls)
    times, ys = _run_pure_granular(s, prm, 1.0e-3, lambda st: (st["pos"][1, 0], st["pos"][1, 1]))
    assert len(run["rows"]) > 100
    for tg, y1, y2 in run["rows"]:
        k = int(np.argmin(np.abs(times - tg)))
        assert abs(times[k] - tg) <= 5e-9 + 1e-12
        assert abs(ys[k][0] - y1) <= 5e-9 + 1e-12, (tg, ys[k][0], y1)
        assert abs(ys[k][1] - y2) <= 5e-9 + 1e-12, (tg, ys[k][1], y2)


def _dem05():
    return json.loads((GOLD / "dem05.json").read_text())


@pytest.mark.parametrize("model", ["LSD", "HERTZ"])
def test_dem05_matches_mfix_table(model):
    d = _dem05()
    tab = d["models"][0 if model == "LSD" else 1]
    assert ("LINEAR" in tab["model"]) == (model == "LSD")
    case, prm, arr, walls = dem05_case(model, d["particle_input"])
    s = make_system(OracleSystem, prm, arr, walls)
    v0 = arr["vel"]
    init_vt = np.sqrt(v0[0] ** 2 + v0[2] ** 2)
    pi = 4.0 * math.atan(1.0)
    init_angle = np.abs(np.arctan(init_vt[:62] / v0[1, :62])) * 180.0 / pi
    factor = math.ceil(float(np.float32(0.0025 / prm.dtsolid)))
    for nn in range(1, factor + 1):
        s.step(1, nn)
        # USR2_DES (end of every DES_TIME_STEP): targets 63-93 held at y =
        # 0.0475 under particles 32-62, at rest
        st = s.download_state()
        pos, vel, om = st["pos"], st["vel"], st["omega"]
        pos[0, 62:93] = pos[0, 31:62]
        pos[2, 62:93] = pos[2, 31:62]
        pos[1, 62:93] = 0.0475
        vel[:, 62:93] = 0.0
        om[:, 62:93] = 0.0
        s.upload_state(pos, vel, om, arr["radius"], arr["pmass"], arr["omoi"], st["state"], arr["phase"])
    st = s.download_state()
    vel, om = st["vel"], st["omega"]
    vxz = np.sqrt(vel[0] ** 2 + vel[2] ** 2)
    rxz = np.sqrt(om[0] ** 2 + om[2] ** 2)
    tol = 5e-5 + 1e-9
    for lc in range(1, 32):
        pp, pw = lc + 30, lc - 1          # NP = LC+31 and NP = LC, 0-based
        ang, a_pp, a_pw = tab["alpha"][lc - 1]
        assert abs(init_angle[pw] - ang) <= tol
        assert abs(math.atan(vxz[pp] / vel[1, pp]) * 180.0 / pi - a_pp) <= tol, (lc, "alpha pp")
        assert abs(math.atan(vxz[pw] / vel[1, pw]) * 180.0 / pi - a_pw) <= tol, (lc, "alpha pw")
        _, o_pp, o_pw = tab["omega"][lc - 1]
        assert abs(rxz[pp] - o_pp) <= tol, (lc, "omega pp", rxz[pp], o_pp)
        assert abs(rxz[pw] - o_pw) <= tol, (lc, "omega pw", rxz[pw], o_pw)
        if lc >= 2:
            _, c_pp, c_pw = tab["coeff"][lc - 2]
            assert abs(vxz[pp] / init_vt[pp] - c_pp) <= tol, (lc, "coeff pp")
            assert abs(vxz[pw] / init_vt[pw] - c_pw) <= tol, (lc, "coeff pw")


# ---- DEM02, DEM04, homogeneous cooling -------------------------------------
# Tables extracted by tests/golden/extract_goldens.py; drivers in golden_runs.py.
PRINT_8 = 5e-9 + 1e-12   # half a unit of the 8th decimal (F15.8 columns)


def _load(name):
    return json.loads((GOLD / name).read_text())


@pytest.mark.parametrize("run_idx", range(18))
def test_dem02_bounce_heights_match_mfix_table(run_idx):
    """Every bounce height MFiX printed (POST_HEIGHT.dat: KN = KN_W in
    {5e4, 5e5, 5e6}, e = 1.0 ... 0.5, Adams-Bashforth) to its 8 decimals."""
    run = _load("dem02.json")["runs"][run_idx]
    assert run["intg"] == "ADAMS_BASHFORTH" and run["en"] == run["en_w"] and run["kn"] == run["kn_w"]
    case, prm, arr, walls = G.dem02_case(run["kn"], run["en"])
    s = make_system(OracleSystem, prm, arr, walls)
    last = run["rows"][-1][0]
    h = G.dem02_heights(s, prm, last_bounce=last)
    assert len(h) == last + 1
    for k, hk in run["rows"]:
        assert abs(h[k] - hk) <= PRINT_8, (k, h[k], hk)


@pytest.mark.parametrize("run_idx", range(9))
def test_dem04_slip_to_roll_matches_mfix_table(run_idx):
    """The end of slip of a sphere launched along the floor (MEW = MEW_W =
    0.2 ... 1.0): the scaled time matches MFiX's table to its 8 decimals.
    The scaled velocities agree within 2e-5 (the AUTOTEST tolerance of the
    reference is 1e-6 absolute or 5 % relative); at the end of slip the
    sphere sits in the floor by mg/KN_W, 1e-5 of its radius, the size of
    that difference, which therefore looks like a lever-arm convention of
    the build that printed the table (this restatement uses DISTMOD,
    calc_collision_wall_mod.f:476,606)."""
    mew, t_nd, tvel, avel = _load("dem04.json")["rows"][run_idx]
    case, prm, arr, walls = G.dem04_case(mew)
    s = make_system(OracleSystem, prm, arr, walls)
    r = G.dem04_roll(s, prm, mew)
    assert r is not None, "no end of slip within TSTOP"
    assert abs(r[0] - t_nd) <= PRINT_8, (r[0], t_nd)
    assert abs(r[1] - tvel) <= 2e-5, (r[1], tvel)
    assert abs(r[2] - avel) <= 2e-5, (r[2], avel)


def _sig5(x, ref):
    """x printed with G11.5 (5 significant digits) reads as ref."""
    if ref == 0.0:
        return abs(x) < 5e-6
    e = math.floor(math.log10(abs(ref)))
    return abs(x - ref) <= 0.5 * 10.0 ** (e - 4) + 1e-12


HCS_EXACT_ROWS = 31   # output times up to 1.5 s


def test_homogeneous_cooling_matches_mfix_table():
    """195 elastic spheres in a fully periodic cube, a neighbour search every
    step (legacy_tests/dem-tests/homogeneous-cooling-system): the pairs across
    the periodic faces come from the minimum image here and from ghost
    copies (DES_PAR_EXCHANGE) in MFiX.  Every printed value of the first 31
    outputs (t <= 1.5 s: solids time, granular temperature, kinetic energy,
    mean velocity) matches to its 5 significant digits.  The system is
    chaotic, so later rows are compared as statistics: the mean velocity
    (momentum) stays exact to print, the kinetic energy between collisions
    returns to the same maximum, and the mean granular temperature over the
    remaining rows agrees within 1 %."""
    d = _load("hcs.json")
    case, prm, arr, walls = G.hcs_case(d["particle_input"])
    s = make_system(OracleSystem, prm, arr, walls)
    rows = np.asarray(G.hcs_rows(s, prm, arr["pmass"]))
    gold = np.asarray(d["rows"])
    assert rows.shape == gold.shape == (101, 4)
    for i in range(HCS_EXACT_ROWS):
        for c in range(4):
            assert _sig5(rows[i, c], gold[i, c]), (i, c, rows[i, c], gold[i, c])
    for i in range(rows.shape[0]):
        assert _sig5(rows[i, 0], gold[i, 0]) and _sig5(rows[i, 3], gold[i, 3]), i
    assert _sig5(rows[:, 2].max(), gold[:, 2].max())
    tail = slice(HCS_EXACT_ROWS, None)
    assert abs(rows[tail, 1].mean() / gold[tail, 1].mean() - 1.0) <= 0.01


@pytest.mark.parametrize("run_idx,interp", [(0, "NONE"), (1, "GARG_2012")])
def test_dem06_terminal_velocity_matches_mfix_table(run_idx, interp):
    """DEM06's one-way coupled runs (DES_INTERP_ON = .F., i.e. the
    unfiltered NONE scheme, and GARG_2012): a 0.1 mm sphere falling against
    a 0.4 m/s upflow with the case's user drag (Schiller-Naumann,
    DEM_DRAG_SINGLE_SPHERE), DRAG_GS_DES1/DRAG_GS_DES0 with the buoyancy
    term P_FORCE*PVOL, DEM sub-steps inside 1 ms fluid steps.  Positions
    and velocities match MFiX's table within 1e-6 absolute, the tolerance
    of the reference's own runtest (numdiff -a 1e-6).  The gas here is the
    exact uniform hydrostatic state; MFiX solves it, and its two runs
    differ from each other by up to 2.2e-7 in velocity, the size of the
    remaining difference (4.4e-7 in v, 1.4e-7 in y)."""
    d = _load("dem06.json")
    run = d["runs"][run_idx]
    assert run["oneway"] and run["scheme"] == interp
    case, prm, arr, walls, grid, f = G.dem06_case(interp)
    s = make_system(OracleSystem, prm, arr, walls)
    s.set_gas_fields(grid, f["ep_g"], f["u_g"], f["v_g"], f["w_g"], f["p_force"])
    rows = G.dem06_rows(s, prm)
    assert len(rows) == len(run["rows"]) == 36
    for (t, y, v), (tg, yg, vg) in zip(rows, run["rows"]):
        assert abs(t - tg) <= PRINT_8
        assert abs(y - yg) <= 1e-6, (t, y, yg)
        assert abs(v - vg) <= 1e-6, (t, v, vg)
