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
  tests/dem/DEM02/AUTOTEST/POST_HEIGHT.dat   bounce heights on the floor
  tests/dem/DEM04/AUTOTEST/POST_TIME.dat, POST_TVEL.dat, POST_AVEL.dat
                                             slip-to-roll on a rough wall
  tests/dem/DEM06/AUTOTEST/POST_POS.dat, POST_VEL.dat   drag, terminal velocity
  legacy_tests/dem-tests/homogeneous-cooling-system/AUTOTEST/POST_GT.dat
  legacy_tests/dem-tests/homogeneous-cooling-system/particle_input.dat
                                             fully periodic cooling (NSN = 1)
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


def parse_dem06_blocks(path):
    """DEM06 tables: per run, its coupling flags and rows (time, RK4
    reference value, MFiX value)."""
    blocks, cur = [], None
    for line in open(path):
        m = re.search(r"DES_ONEWAY_COUPLED =\s+(\S)", line)
        if m:
            cur = {"oneway": m.group(1) == "T", "rows": []}
            blocks.append(cur)
            continue
        if cur is None:
            continue
        m = re.search(r"DES_INTERP_ON =\s+(\S)(?:\s+DES_INTERP_SCHEME = (\S+))?", line)
        if m:
            cur["interp_on"] = m.group(1) == "T"
            cur["scheme"] = m.group(2) or "NONE"
            continue
        m = re.search(r"DES_INTERP_WIDTH =\s+(\S+)", line)
        if m:
            cur["width"] = float(m.group(1))
        t = line.split()
        if len(t) == 4 and all(re.match(r"^-?\d+\.\d+$", x) for x in t):
            cur["rows"].append([float(t[0]), float(t[1]), float(t[2])])
    return blocks


def parse_rows(path, ncol):
    """Numeric rows of exactly ncol columns (Fortran E or F format)."""
    rows = []
    for line in open(path):
        t = line.split()
        if len(t) == ncol:
            try:
                rows.append([float(x.replace("D", "E")) for x in t])
            except ValueError:
                pass
    return rows


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

    # DEM02: maximum height of each bounce of a sphere on the floor (AB2)
    d2 = root / "tests/dem/DEM02"
    runs2 = []
    for b in parse_table(d2 / "AUTOTEST/POST_HEIGHT.dat"):
        # columns: bounce number, MFiX maximum height
        runs2.append({"intg": b["intg"], "kn": b["kn"], "kn_w": b["kn_w"], "en": b["en"], "en_w": b["en_w"],
                      "rows": [[int(r[0]), r[2]] for r in b["rows"]]})
    dem02 = {"particle_input": (d2 / "particle_input.dat").read_text().split(), "runs": runs2}
    (HERE / "dem02.json").write_text(json.dumps(dem02))
    print("wrote dem02.json:", len(runs2), "runs")

    # DEM04: a sphere sliding on the floor until it rolls (AB2, friction sweep)
    d4 = root / "tests/dem/DEM04"
    cols = {k: parse_rows(d4 / f"AUTOTEST/POST_{k}.dat", 4) for k in ("TIME", "TVEL", "AVEL")}
    # columns: MEW, MFiX scaled time, MFiX scaled translational and angular velocity
    rows4 = [[t[0], t[2], v[2], a[2]] for t, v, a in zip(cols["TIME"], cols["TVEL"], cols["AVEL"])]
    dem04 = {"particle_input": (d4 / "particle_input.dat").read_text().split(), "rows": rows4}
    (HERE / "dem04.json").write_text(json.dumps(dem04))
    print("wrote dem04.json:", len(rows4), "runs")

    # DEM06: one sphere reaching terminal velocity in a uniform upflow
    d6 = root / "tests/dem/DEM06"
    pos6 = parse_dem06_blocks(d6 / "AUTOTEST/POST_POS.dat")
    vel6 = parse_dem06_blocks(d6 / "AUTOTEST/POST_VEL.dat")
    runs6 = []
    for bp, bv in zip(pos6, vel6):
        # columns: time, MFiX y position, MFiX y velocity
        runs6.append({"oneway": bp["oneway"], "interp_on": bp.get("interp_on"), "scheme": bp.get("scheme"),
                      "width": bp.get("width"),
                      "rows": [[rp[0], rp[2], rv[2]] for rp, rv in zip(bp["rows"], bv["rows"])]})
    dem06 = {"particle_input": (d6 / "particle_input.dat").read_text().split(), "runs": runs6}
    (HERE / "dem06.json").write_text(json.dumps(dem06))
    print("wrote dem06.json:", [(r["oneway"], r["scheme"], len(r["rows"])) for r in runs6])

    # homogeneous cooling: 195 elastic spheres in a fully periodic cube
    dh = root / "legacy_tests/dem-tests/homogeneous-cooling-system"
    hcs = {"particle_input": parse_rows(dh / "particle_input.dat", 8),
           # columns: solids time, granular energy, kinetic energy, mean speed
           "rows": parse_rows(dh / "AUTOTEST/POST_GT.dat", 4)}
    (HERE / "hcs.json").write_text(json.dumps(hcs))
    print("wrote hcs.json:", len(hcs["particle_input"]), "particles,", len(hcs["rows"]), "rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_goldens.py <reference checkout>")
    main(sys.argv[1])
