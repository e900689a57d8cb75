"""Extracts the reference's DEM regression tables into small JSON fixtures.

Run in a container that holds the MFiX sources (default root below); the
fixtures it writes are committed so the tests run without the reference:

    python tests/golden/extract_goldens.py [/path/to/mfix]

Sources (relative to the MFiX root):
  tests/dem/DEM01/AUTOTEST/POST_POS.dat, POST_VEL.dat   free fall + wall bounce
  tests/dem/DEM01/particle_input.dat
  tests/dem/DEM02..DEM05 AUTOTEST tables and particle inputs (see below)
Only the MFiX-computed columns are kept, with each run's keyword header.
"""
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def parse_table(path):
    """Blocks of (header keywords, numeric rows) from a WRITE_USR1 table."""
    blocks, cur = [], None
    for line in open(path):
        m = re.search(r"Time Stepping Scheme: (\S+)", line)
        if m:
            cur = {"intg": m.group(1), "rows": []}
            blocks.append(cur)
            continue
        if cur is None:
            continue
        for key, pat in (("kn", r"\bKN =\s+(\S+)"), ("kn_w", r"\bKN_W =\s+(\S+)"),
                         ("en", r"DES_EN_INPUT =\s+(\S+)"), ("en_w", r"DES_EN_WALL_INPUT =\s+(\S+)")):
            m = re.search(pat, line)
            if m:
                cur[key] = float(m.group(1))
                break
        else:
            t = line.split()
            if t and all(re.match(r"^-?\d+(\.\d+)?([eEdD][-+]?\d+)?$", x) for x in t):
                cur["rows"].append([float(x.replace("D", "E").replace("d", "e")) for x in t])
    return blocks


def main(root):
    root = Path(root)
    out = {}
    d1 = root / "tests/dem/DEM01"
    pos = parse_table(d1 / "AUTOTEST/POST_POS.dat")
    vel = parse_table(d1 / "AUTOTEST/POST_VEL.dat")
    runs = []
    for bp, bv in zip(pos, vel):
        runs.append({
            "intg": bp["intg"], "kn": bp["kn"], "kn_w": bp["kn_w"], "en": bp["en"],
            # columns: time, MFiX y position, MFiX y velocity
            "rows": [[rp[0], rp[3], rv[3]] for rp, rv in zip(bp["rows"], bv["rows"])],
        })
    out["DEM01"] = {
        "particle_input": (d1 / "particle_input.dat").read_text().split(),
        "runs": runs,
    }
    (HERE / "dem01.json").write_text(json.dumps(out["DEM01"]))
    print("wrote dem01.json:", len(runs), "runs")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
