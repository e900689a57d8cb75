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
digit).
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

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
