"""GPU parity: the CUDA library against the CPU oracle on the same inputs.

Integer outputs (DES cells, NEIGHBOR_INDEX, NEIGHBORS, wall facet slots)
must be identical.  FP64 state must agree within 1e-10 relative (normwise
per array) over the first 100 steps; the FP64 kernels keep the serial
reference's operation order, and the exact-equality checks below show that
the agreement is in fact bitwise.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from cases import dem01_case, settling_case, make_system
from gpu_util import REL_TOL, compare_pairs, compare_state, pair_both, rel_err

pytestmark = pytest.mark.gpu


def test_cells_and_pairs_match_oracle():
    case, prm, arr, walls = settling_case(n_side=(6, 20, 6))
    g, o = pair_both(prm, arr, walls)
    assert np.array_equal(g.download_cells(), o.download_cells())
    compare_pairs(g, o)
    assert g.pair_count() > 0


def test_force_matches_oracle_bitwise():
    case, prm, arr, walls = settling_case(n_side=(6, 20, 6), spacing=0.98, jitter=0.03)
    g, o = pair_both(prm, arr, walls)
    g.calc_force(); o.calc_force()
    fg, tg = g.download_forces()
    fo, to = o.download_forces()
    assert np.abs(fo).max() > 0
    assert np.array_equal(fg, fo), rel_err(fg, fo)
    assert np.array_equal(tg, to), rel_err(tg, to)
    # per-stage integration matches too
    g.cfnewvalues(); o.cfnewvalues()
    compare_state(g, o, exact=True)
    assert rel_err(g.download_pairs()[2], o.download_pairs()[2]) == 0.0


@pytest.mark.parametrize("coll,intg,mew_r,poly", [
    ("LSD", "EULER", 0.0, 0.0),
    ("LSD", "ADAMS_BASHFORTH", 0.0, 0.0),
    ("HERTZ", "EULER", 0.01, 0.25),
    ("HERTZ", "ADAMS_BASHFORTH", 0.01, 0.25),
])
def test_100_steps_match_oracle(coll, intg, mew_r, poly):
    case, prm, arr, walls = settling_case(n_side=(6, 16, 6), spacing=1.0, jitter=0.04, coll=coll,
                                          intg=intg, mew_r=mew_r, polydisperse=poly, nsn=10)
    g, o = pair_both(prm, arr, walls)
    for chunk in range(4):
        g.step(25); o.step(25)
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
    fg, pg = g.download_wall_history()
    fo, po = o.download_wall_history()
    assert np.array_equal(fg, fo)
    assert np.array_equal(pg[fg > 0], po[fo > 0])
    sg, so = g.stats(), o.stats()
    assert sg["n_contacts"] == so["n_contacts"]
    assert sg["n_wall_contacts"] == so["n_wall_contacts"]
    assert sg["n_pairs"] == so["n_pairs"]


def test_dem01_golden_on_gpu():
    gold = json.loads((Path(__file__).resolve().parent / "golden" / "dem01.json").read_text())
    from mfix_dem import GpuSystem
    for run in gold["runs"][::7]:
        case, prm, arr, walls = dem01_case(run["intg"], run["kn"], run["en"])
        g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
        factor = math.ceil(float(np.float32(0.5 / prm.dtsolid)))
        t, times, ys = 0.0, [0.0], [0.5]
        for nn in range(1, factor + 1):
            g.step(1, nn)
            t = t + prm.dtsolid
            times.append(t)
            ys.append(g.download_state()["pos"][1, 0])
        times = np.asarray(times)
        for tg, yg, vg in run["rows"]:
            k = int(np.argmin(np.abs(times - tg)))
            assert abs(ys[k] - yg) <= 5e-9 + 1e-12


def test_periodic_matches_oracle():
    case, prm, arr, walls = settling_case(n_side=(10, 10, 10), box=(12e-3, 40e-3, 12e-3), spacing=1.1,
                                          periodic=(True, False, True), nsn=5, vmax=0.3)
    g, o = pair_both(prm, arr, walls)
    for _ in range(4):
        g.step(10); o.step(10)
        compare_state(g, o, exact=True)
        compare_pairs(g, o)


def test_rogue_particles_removed_like_oracle():
    case, prm, arr, walls = settling_case(n_side=(6, 10, 6))
    # push two particles far outside the domain: they land in ghost cells
    arr = dict(arr)
    pos = arr["pos"].copy()
    pos[0, 50] = -0.5
    pos[1, 120] = 2.0
    arr["pos"] = pos
    g, o = pair_both(prm, arr, walls)
    compare_pairs(g, o)
    sg, so = g.download_state(), o.download_state()
    assert np.array_equal(sg["state"], so["state"])
    assert sg["state"][50] == 0 and sg["state"][120] == 0
    g.step(20); o.step(20)
    compare_state(g, o, exact=True)


def test_narrow_des_grid_matches_oracle():
    """DES cells narrower than the search diameter 2*FACTOR_RLM*MAX_RADIUS:
    the reference scans all 27 cells.  (With the default sizing of 3 max
    diameters the cells are wider and the reference scans only the nearer
    2x2x2 cells, desgrid_mod.f:1116-1152; the other tests cover that.)"""
    from mfix_dem import params as P
    case, prm, arr, walls = settling_case(n_side=(8, 20, 8), box=(12e-3, 60e-3, 12e-3), spacing=1.0, nsn=5)
    case.desgridsearch = (11, 55, 11)
    prm, _ = P.build_params(case, arr["radius"], arr["pmass"], arr["phase"], arr["state"])
    assert not (1.0 > 2.0 * prm.max_radius * prm.factor_rlm * prm.dg_dxinv)
    g, o = pair_both(prm, arr, walls)
    compare_pairs(g, o)
    for _ in range(3):
        g.step(10); o.step(10)
        compare_state(g, o, exact=True)
        compare_pairs(g, o)


def test_dense_overlapping_bed_matches_oracle():
    """Initial overlaps everywhere (lattice spacing 0.97 d): every pair is a
    contact from the first step, Hertz with rolling friction, AB2."""
    case, prm, arr, walls = settling_case(n_side=(8, 12, 8), spacing=0.97, jitter=0.01, coll="HERTZ",
                                          intg="ADAMS_BASHFORTH", mew_r=0.02, polydisperse=0.0, nsn=7)
    g, o = pair_both(prm, arr, walls)
    for _ in range(3):
        g.step(11); o.step(11)
        compare_state(g, o, exact=True)
        compare_pairs(g, o)
    assert g.stats()["n_contacts"] == o.stats()["n_contacts"] > 0


@pytest.mark.parametrize("coll,intg,periodic", [("HERTZ", "EULER", (False, False, False)),
                                                ("LSD", "ADAMS_BASHFORTH", (True, False, True))])
def test_graph_replay_matches_eager_and_oracle(coll, intg, periodic):
    """dem_step replays whole NEIGHBOR_SEARCH_N periods as CUDA graphs; the
    result must not differ from launching step by step, nor from the oracle."""
    from mfix_dem import GpuSystem
    from oracle_ffi import OracleSystem
    kw = dict(n_side=(10, 10, 10), box=(12e-3, 40e-3, 12e-3), spacing=1.0, coll=coll, intg=intg,
              periodic=periodic, nsn=5, vmax=0.3)
    case, prm, arr, walls = settling_case(**kw)
    g1 = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    g2 = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    g2.set_graphs(False)
    o = make_system(OracleSystem, prm, arr, walls)
    for s in (g1, g2, o):
        s.step(1)
        s.step(33)
    l0 = g1.launch_count()
    g1.step(10); g2.step(10); o.step(10)
    assert g1.launch_count() > l0
    compare_state(g1, o, exact=True)
    compare_state(g2, o, exact=True)
    compare_pairs(g1, o)
    assert g1.stats()["n_contacts"] == o.stats()["n_contacts"]


def test_periodic_particles_reach_a_wall_between_builds():
    """A periodic system re-places its particles every step: spheres falling
    from a DES cell without facets into the floor's cells between two
    rebuilds must meet the floor as the oracle's (unscreened) wall test has
    them do."""
    from mfix_dem import GpuSystem
    from oracle_ffi import OracleSystem
    from cases import make_system, settling_case
    case, prm, arr, walls = settling_case(n_side=(3, 1, 3), spacing=3.0, jitter=0.05, vmax=0.01, seed=21,
                                          periodic=(True, False, True), nsn=2000)
    h = 1.0 / prm.dg_dyinv
    arr["pos"][1] = 1.5 * h + 0.1e-3 * np.arange(arr["pos"].shape[1]) / arr["pos"].shape[1]
    arr["vel"][1] = -3.0
    g = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    o = make_system(OracleSystem, prm, arr, walls)
    steps = int(2.0 * h / (3.0 * prm.dtsolid)) + 50
    for _ in range(4):
        g.step(steps // 4); o.step(steps // 4)
        compare_state(g, o, exact=True)
    d = o.download_state()
    assert np.all(d["pos"][1] > 0.0)            # the floor held them
    assert o.stats()["n_wall_contacts"] >= 0


@pytest.mark.parametrize("periodic", [(False, False, False), (True, False, True)])
def test_long_rows_and_long_incoming_lists_match_oracle(periodic):
    """Large spheres among small ones: rows of a few hundred neighbours (past
    the 16 slots the count pass keeps and the 128 keys a warp ranks, so the
    fill pass takes its one-lane insertion path) and an incoming list of a
    few hundred pairs (past the 16 the transpose sorts in registers); with
    periodic x and z the first large sphere straddles the periodic faces.
    Cells, NEIGHBOR_INDEX / NEIGHBORS and the state stay bit-identical to the
    oracle through a rebuild."""
    from cases import bimodal_case
    case, prm, arr, walls = bimodal_case(periodic=periodic)
    g, o = pair_both(prm, arr, walls)
    ni = np.asarray(o.download_pairs()[0])
    rows = np.diff(np.concatenate([[1], ni]))
    assert rows.max() > 128
    assert np.array_equal(g.download_cells(), o.download_cells())
    compare_pairs(g, o)
    g.step(30); o.step(30)
    compare_state(g, o, exact=True)
    assert compare_pairs(g, o) == 0.0


@pytest.mark.parametrize("periodic", [(False, False, False), (True, False, True)])
def test_pair_builds_from_the_candidate_list_match_oracle(periodic):
    """Between two grid scans a pair build filters the candidate list (the
    pairs within the search radius plus a skin of 0.3 FACTOR_RLM MAX_RADIUS
    when the list was made) until the particles may have moved half the
    skin; then a build scans the grid and makes a new list.  Spheres at up to
    5 m/s, rebuilt every 5 steps for 300 steps under captured periods:
    builds of both kinds, and NEIGHBOR_INDEX / NEIGHBORS and the state stay
    the oracle's, bit for bit, after every fifth build."""
    case, prm, arr, walls = settling_case(n_side=(8, 12, 8), spacing=1.0, jitter=0.03, coll="HERTZ",
                                          intg="EULER", nsn=5, vmax=3.0, periodic=periodic)
    g, o = pair_both(prm, arr, walls)
    for _ in range(12):
        g.step(25); o.step(25)
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
    st = g.stats()
    assert st["n_builds_filtered"] > 10
    assert st["n_candidate_lists"] >= 2


def test_upload_of_the_moving_state_only():
    """dem_upload_state with only positions, velocities and spins (the
    other arrays NULL) keeps the handle's radius, mass, inertia, state and
    phase: a run that re-sends its own moving state every step stays
    bit-identical to one that does not.  The first upload needs every
    array."""
    from mfix_dem import GpuSystem
    from mfix_dem.system import DemError
    from mfix_dem import abi
    case, prm, arr, walls = settling_case(n_side=(6, 16, 6), spacing=0.98, jitter=0.03)
    fresh = GpuSystem(prm, arr["pos"].shape[1])
    with pytest.raises(DemError) as e:
        fresh.upload_state(arr["pos"], arr["vel"], arr["omega"])
    assert e.value.code == abi.DEM_ERR_ARG
    fresh.close()
    a = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    b = make_system(lambda p, n: GpuSystem(p, n), prm, arr, walls)
    for k in range(40):
        a.step(1)
        b.step(1)
        s = b.download_state()
        b.upload_state(s["pos"], s["vel"], s["omega"])
    sa, sb = a.download_state(), b.download_state()
    for key in ("pos", "vel", "omega", "state"):
        assert np.array_equal(sa[key], sb[key]), key
    assert a.stats()["n_contacts"] == b.stats()["n_contacts"] > 0


def test_motion_only_uploads_move_the_bound_not_the_list():
    """A motion-only upload that moves the particles adds the largest move
    to the displacement bound: small moves keep the candidate list (the
    build after each filters it), a move past half the skin makes the next
    build scan the grid for a new list.  The oracle gets the same uploads;
    state and NEIGHBOR_INDEX / NEIGHBORS stay its own, bit for bit."""
    case, prm, arr, walls = settling_case(n_side=(8, 12, 8), spacing=1.0, jitter=0.03, coll="HERTZ",
                                          intg="EULER", nsn=5, vmax=0.1)
    g, o = pair_both(prm, arr, walls)
    rng = np.random.default_rng(7)
    skin = 0.3 * prm.factor_rlm * float(arr["radius"].max())
    for shift, new_list in ((0.02, 0), (0.02, 0), (0.6, 1), (0.02, 0)):
        st0 = g.stats()
        s = o.download_state()
        # every particle moves by at most shift * skin
        pos = s["pos"] + rng.uniform(-1.0, 1.0, s["pos"].shape) * (shift * skin / np.sqrt(3.0))
        g.upload_state(pos, s["vel"], s["omega"])
        o.upload_state(pos, s["vel"], s["omega"])
        g.step(5); o.step(5)  # one or two builds
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
        st1 = g.stats()
        assert st1["n_candidate_lists"] - st0["n_candidate_lists"] == new_list, shift
        assert st1["n_builds_filtered"] - st0["n_builds_filtered"] >= 1 - new_list, shift


@pytest.mark.parametrize("periodic", [(False, False, False), (True, False, True)])
def test_candidate_lists_at_multi_tile_sizes_match_oracle(periodic):
    """4,096 spheres at up to 5 m/s (scans of more than one tile, whose
    scratch the list build and the transpose of the new pair list both
    use), rebuilt every 5 steps for 200 steps: candidate lists made and
    filtered, and the state and NEIGHBOR_INDEX / NEIGHBORS stay the
    oracle's, bit for bit."""
    case, prm, arr, walls = settling_case(n_side=(16, 16, 16), box=(20e-3, 40e-3, 20e-3), spacing=1.0,
                                          jitter=0.03, coll="HERTZ", intg="EULER", nsn=5, vmax=3.0,
                                          periodic=periodic)
    g, o = pair_both(prm, arr, walls)
    for _ in range(8):
        g.step(25); o.step(25)
        compare_state(g, o, exact=True)
        assert compare_pairs(g, o) == 0.0
    st = g.stats()
    assert st["n_builds_filtered"] > 10
    assert st["n_candidate_lists"] >= 2
