"""Extracts the reference's DEM regression tables into small JSON fixtures.

Run where the MFiX sources are checked out, passing their root; the
fixtures it writes are committed so the tests run without the reference:

    python tests/golden/extract_goldens.py /path/to/mfix

Sources (relative to the MFiX root):
  tests/dem/DEM01/AUTOTEST/POST_POS.dat, POST_VEL.dat   free fall + wall bounce
  tests/dem/DEM01/particle_input.dat
  tests/dem/DEM03/AUTOTEST/POST_POS1.dat, POST_POS2.dat   two stacked particles
  tests/dem/DEM03/particle_input.dat
  tests/dem/DEM05/AUTOTEST/POST_ALPHA.dat, POST_OMEGA.dat, POST_COEFF.dat   oblique impacts
  tests/dem/DEM05/particle_input.dat
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


def parse_model_blocks(path):
    """DEM05 tables: per collision model, rows (impact angle, particle-
    particle value, particle-wall value)."""
    blocks, cur = [], None
    for line in open(path):
        m = re.search(r"Collision model: (.+)", line)
        if m:
            cur = {"model": m.group(1).strip(), "rows": []}
            blocks.append(cur)
            continue
        if cur is None:
            continue
        t = line.split()
        if len(t) == 3 and all(re.match(r"^-?\d+\.\d+$", x) for x in t):
            cur["rows"].append([float(x) for x in t])
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

    # DEM03: two stacked, compressed particles (pair and wall contacts, AB2)
    d3 = root / "tests/dem/DEM03"
    p1 = parse_table(d3 / "AUTOTEST/POST_POS1.dat")
    p2 = parse_table(d3 / "AUTOTEST/POST_POS2.dat")
    runs3 = []
    for b1, b2 in zip(p1, p2):
        runs3.append({
            "intg": b1["intg"], "kn": b1["kn"], "kn_w": b1["kn_w"], "en": b1["en"], "en_w": b1["en_w"],
            # columns: time, MFiX y position of particle 1, of particle 2
            "rows": [[r1[0], r1[2], r2[2]] for r1, r2 in zip(b1["rows"], b2["rows"])],
        })
    out["DEM03"] = {"particle_input": (d3 / "particle_input.dat").read_text().split(), "runs": runs3}
    (HERE / "dem03.json").write_text(json.dumps(out["DEM03"]))
    print("wrote dem03.json:", len(runs3), "runs")

    # DEM05: oblique impacts on the floor and on fixed target particles
    d5 = root / "tests/dem/DEM05"
    tables = {k: parse_model_blocks(d5 / f"AUTOTEST/POST_{k.upper()}.dat") for k in ("alpha", "omega", "coeff")}
    models = []
    for i, b in enumerate(tables["alpha"]):
        models.append({"model": b["model"], "alpha": b["rows"], "omega": tables["omega"][i]["rows"],
                       "coeff": tables["coeff"][i]["rows"]})
    out["DEM05"] = {"particle_input": (d5 / "particle_input.dat").read_text().split(), "models": models}
    (HERE / "dem05.json").write_text(json.dumps(out["DEM05"]))
    print("wrote dem05.json:", [(m["model"], len(m["alpha"]), len(m["omega"]), len(m["coeff"])) for m in models])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_goldens.py <reference checkout>")
    main(sys.argv[1])
