"""Pins the CPU oracle to the reference's own regression tables.

DEM01 (tests/dem/DEM01 in MFiX): a 0.2 m sphere falls onto the bottom wall
of the default STL box; 38 runs sweep DES_INTG_METHOD (EULER, ADAMS_BASHFORTH),
KN = KN_W and the restitution coefficient.  The AUTOTEST tables print MFiX's
position and velocity with 8 decimals at the first DEM step past each output
time; the oracle must reproduce every printed value to within the print
resolution (5e-9, plus a small allowance for the rounding of the last digit).
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from cases import dem01_case, make_system
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
