"""The reference's regression tables on the CUDA path.

DEM02 (bounce heights), DEM03 (two stacked, compressed particles), DEM04
(slip to roll on a rough floor), DEM05 (oblique impacts on the floor and on
fixed targets, LSD and Hertz) and the homogeneous cooling system (fully
periodic, a neighbour search every step) run on the GPU beside the oracle:
the GPU results must equal the oracle's bit for bit, and both must reproduce
MFiX's printed values (tests/test_oracle_golden.py states the tolerances).
"""
import json
import math

import numpy as np
import pytest

import golden_runs as G
from mfix_dem import GpuSystem
from cases import dem03_case, dem05_case, make_system
from oracle_ffi import OracleSystem
from test_oracle_golden import GOLD, HCS_EXACT_ROWS, PRINT_8, _sig5

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("run_idx", [0, 3, 5])
def test_dem03_gpu_equals_oracle_and_table(run_idx):
    run = json.loads((GOLD / "dem03.json").read_text())["runs"][run_idx]
    case, prm, arr, walls = dem03_case(run["en"], run["en_w"])
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    factor = math.ceil(float(np.float32(1.0e-3 / prm.dtsolid)))
    t, times, ys = 0.0, [0.0], [arr["pos"][1].copy()]
    for nn in range(1, factor + 1):
        g.step(1, nn)
        o.step(1, nn)
        sg, so = g.download_state(), o.download_state()
        for k in ("pos", "vel", "omega"):
            assert np.array_equal(sg[k], so[k]), (nn, k)
        t = t + prm.dtsolid
        times.append(t)
        ys.append(sg["pos"][1].copy())
    times = np.asarray(times)
    for tg, y1, y2 in run["rows"]:
        k = int(np.argmin(np.abs(times - tg)))
        assert abs(ys[k][0] - y1) <= 5e-9 + 1e-12 and abs(ys[k][1] - y2) <= 5e-9 + 1e-12


@pytest.mark.parametrize("model", ["LSD", "HERTZ"])
def test_dem05_gpu_equals_oracle(model):
    d = json.loads((GOLD / "dem05.json").read_text())
    case, prm, arr, walls = dem05_case(model, d["particle_input"])
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    factor = math.ceil(float(np.float32(0.0025 / prm.dtsolid)))
    for nn in range(1, factor + 1):
        for s in (g, o):
            s.step(1, nn)
            st = s.download_state()
            pos, vel, om = st["pos"], st["vel"], st["omega"]
            pos[0, 62:93] = pos[0, 31:62]
            pos[2, 62:93] = pos[2, 31:62]
            pos[1, 62:93] = 0.0475
            vel[:, 62:93] = 0.0
            om[:, 62:93] = 0.0
            s.upload_state(pos, vel, om, arr["radius"], arr["pmass"], arr["omoi"], st["state"], arr["phase"])
        if nn % 500 == 0 or nn == factor:
            sg, so = g.download_state(), o.download_state()
            for k in ("pos", "vel", "omega"):
                assert np.array_equal(sg[k], so[k]), (nn, k)
    # the wall histories agree too
    fg, pg = g.download_wall_history()
    fo, po = o.download_wall_history()
    assert np.array_equal(fg, fo) and np.array_equal(pg, po)


def _gpu(prm, arr, walls):
    return make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)


@pytest.mark.parametrize("run_idx", [1, 5, 6, 9])
def test_dem02_gpu_equals_oracle_and_table(run_idx):
    run = json.loads((GOLD / "dem02.json").read_text())["runs"][run_idx]
    case, prm, arr, walls = G.dem02_case(run["kn"], run["en"])
    last = run["rows"][-1][0]
    hg = G.dem02_heights(_gpu(prm, arr, walls), prm, last_bounce=last)
    ho = G.dem02_heights(make_system(OracleSystem, prm, arr, walls), prm, last_bounce=last)
    assert hg == ho
    for k, hk in run["rows"]:
        assert abs(hg[k] - hk) <= PRINT_8, (k, hg[k], hk)


@pytest.mark.parametrize("run_idx", range(9))
def test_dem04_gpu_equals_oracle(run_idx):
    mew, t_nd, tvel, avel = json.loads((GOLD / "dem04.json").read_text())["rows"][run_idx]
    case, prm, arr, walls = G.dem04_case(mew)
    rg = G.dem04_roll(_gpu(prm, arr, walls), prm, mew)
    ro = G.dem04_roll(make_system(OracleSystem, prm, arr, walls), prm, mew)
    assert rg == ro and rg is not None
    assert abs(rg[0] - t_nd) <= PRINT_8


def test_homogeneous_cooling_gpu_equals_oracle_and_table():
    """The fully periodic cooling system for the whole 5 s (155,528 steps,
    a pair-list build every step): the GPU rows equal the oracle's exactly,
    and the first 31 match MFiX's table to its 5 printed digits."""
    d = json.loads((GOLD / "hcs.json").read_text())
    case, prm, arr, walls = G.hcs_case(d["particle_input"])
    g = _gpu(prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    rg = np.asarray(G.hcs_rows(g, prm, arr["pmass"]))
    ro = np.asarray(G.hcs_rows(o, prm, arr["pmass"]))
    assert np.array_equal(rg, ro)
    sg, so = g.download_state(), o.download_state()
    for k in ("pos", "vel", "omega"):
        assert np.array_equal(sg[k], so[k]), k
    gold = np.asarray(d["rows"])
    for i in range(HCS_EXACT_ROWS):
        for c in range(4):
            assert _sig5(rg[i, c], gold[i, c]), (i, c, rg[i, c], gold[i, c])


@pytest.mark.parametrize("interp", ["NONE", "GARG_2012"])
def test_dem06_gpu_matches_oracle(interp):
    """DEM06 on the GPU: the same rows as the oracle within 1e-12 relative
    (the drag calls pow, whose last bit can differ between CUDA and the host
    libm), hence within the table's 1e-6 (tests/test_oracle_golden.py)."""
    from gpu_util import rel_err
    d = json.loads((GOLD / "dem06.json").read_text())
    run = d["runs"][0 if interp == "NONE" else 1]
    case, prm, arr, walls, grid, f = G.dem06_case(interp)
    out = []
    for s in (_gpu(prm, arr, walls), make_system(OracleSystem, prm, arr, walls)):
        s.set_gas_fields(grid, f["ep_g"], f["u_g"], f["v_g"], f["w_g"], f["p_force"])
        out.append(np.asarray(G.dem06_rows(s, prm)))
    rg, ro = out
    assert rel_err(rg[:, 1], ro[:, 1]) <= 1e-12 and rel_err(rg[:, 2], ro[:, 2]) <= 1e-12
    gold = np.asarray(run["rows"])
    assert np.max(np.abs(rg[:, 1:] - gold[:, 1:])) <= 1e-6
