#!/usr/bin/env python3
"""bench.py -- DEM particle step throughput on B200.

Workload (`--workload dense`, the headline): 1,000,000 polydisperse
Hertzian spheres (lognormal d, median 1 mm, sigma 0.25, clipped to 0.5-2 mm;
rho 2500; E 1e7, nu 0.3; e_n = e_t = 0.85; friction 0.3, rolling friction
0.01) in a 0.1 x 0.4 x 0.1 m box, periodic in x and z with a flat bottom
wall, placed by seeded random sequential placement at 40 % solids and then
every diameter grown by 1.15 (61 % solids, about two contacts per particle),
so that the bed carries contacts like a settled bed.  `--workload rsa40`
is the placement as placed (40 % solids, no contacts within the timed
steps).  One step = one DES_TIME_STEP (contact forces, walls, integration,
and the neighbour rebuild every NEIGHBOR_SEARCH_N = 25 steps).  The timed
window of K steps ends on a rebuild step, so it holds ceil(K / 25) rebuilds:
at least their natural rate.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  N > 1 runs N independent replicas of the system, one
per GPU (the DEM step of one system does not shard without a halo exchange);
value is the sum over replicas, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "mfix-cfd-dem_b200"))
CACHE = ROOT / "mfix-cfd-dem_b200" / "_cache"

METRIC = "particle-steps/s"
PROFILE_TRAFFIC = ROOT / "profiles" / "force_traffic.json"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000, help="particles per system")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-sample", type=int, default=1_000_000, help="particles in the CPU sample")
    ap.add_argument("--cpu-steps", type=int, default=200, help="timed steps of the CPU sample (about 10 s)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision leg")
    ap.add_argument("--serve-graphs", type=int, default=1,
                    help="served leg: replay aligned periods as CUDA graphs (1) or step launch by launch (0)")
    ap.add_argument("--batch-systems", type=int, default=256, help="systems of the batched leg (0 = skip)")
    ap.add_argument("--batch-total", type=int, default=6_000_000, help="particles of the batched leg")
    ap.add_argument("--serve-rates", default="5,10,20,50,100,200",
                    help="request rates (1/s) of the served leg ('' = skip)")
    ap.add_argument("--serve-requests", type=int, default=30, help="requests per rate")
    ap.add_argument("--serve-steps", type=int, default=20000, help="DES steps per served case")
    ap.add_argument("--serve-budget-gb", type=float, default=40.0, help="HBM budget of the server")
    ap.add_argument("--serve-profile", action="store_true",
                    help="only the per-chunk cost of a fixed served mix (three hopper cases), by kernel class")
    ap.add_argument("--workload", default="dense", choices=["dense", "rsa40"],
                    help="dense: the placement with every diameter grown by --inflate; rsa40: as placed")
    ap.add_argument("--inflate", type=float, default=1.15,
                    help="diameter growth after placement of the dense workload")
    ap.add_argument("--no-rsa40", action="store_true", help="skip the FP64 leg on the bed as placed")
    a = ap.parse_args()
    if a.workload == "rsa40":
        a.inflate = 1.0
    return a


def workload_name(inflate):
    return "hertz_rsa_1m" if inflate == 1.0 else f"hertz_rsa_1m_dense_x{inflate:g}"


def timed_window(warm_min, steps, nsn):
    """First NN of a window of `steps` steps that starts after at least
    warm_min warm-up steps and ends on a neighbour-search step (NN a multiple
    of nsn), and the number of rebuilds inside it: ceil(steps / nsn), the
    natural rate or above it."""
    end = -(-(warm_min + steps) // nsn) * nsn
    nn0 = end - steps + 1
    rebuilds = sum(1 for nn in range(nn0, end + 1) if nn % nsn == 0)
    return nn0, rebuilds


def bench_config(args, info, prm):
    """The `config` object shared by both arms."""
    return {"workload": workload_name(args.inflate), "n_particles_requested": args.n,
            "inflate": args.inflate, "contact": "hertz", "integrator": "euler", "periodic": "xz",
            "neighbor_search_n": int(prm.neighbor_search_n),
            "solids_fraction": round(float(info.get("solids_fraction")) * args.inflate ** 3, 4),
            "dtsolid": prm.dtsolid, "steps_timed": args.steps}


def workload(n, precision, inflate=1.0):
    from mfix_dem import abi, configs
    prec = abi.DEM_PREC_SPLIT if precision == "split" else abi.DEM_PREC_FP64
    scale = (n / 1_000_000) ** 0.5
    box = (0.1 * scale, 0.4, 0.1 * scale)
    return configs.hertz_rsa(n=n, box=box, precision=prec, cache_dir=CACHE, inflate=inflate)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x, ws, device):
    """The largest of the ranks' values of x (a time): the job's time is its
    slowest replica's.  Every rank calls it at the same point."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms.  Started
    before the timed region (nvidia-smi needs a moment to report); the
    samples kept are those from the last one before the region to the first
    one after it."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def start(self, wait_s=10.0):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
            return
        end = time.monotonic() + wait_s
        while not self.lines and time.monotonic() < end:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def begin(self):
        self.t0 = time.monotonic()

    def end(self):
        self.t1 = time.monotonic()

    def stop(self):
        if self.proc is None:
            return None
        t1 = self.t1 if self.t1 is not None else time.monotonic()
        deadline = time.monotonic() + 1.0
        while time.monotonic() < deadline and not any(t > t1 for t, _ in self.lines):
            time.sleep(0.02)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        t0 = self.t0 if self.t0 is not None else 0.0
        before = [i for i, (t, _) in enumerate(self.lines) if t <= t0]
        after = [i for i, (t, _) in enumerate(self.lines) if t >= t1]
        lo = before[-1] if before else 0
        hi = after[0] if after else len(self.lines) - 1
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, ln in self.lines[lo:hi + 1]:
            parts = [q.strip() for q in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "timed_s": round(t1 - t0, 4)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(n_normal, n_pairs, periodic=True, n_torque=None):
    # per step: N*(64 read + 48 write + 4 CSR) for positions and velocities,
    # T*(32 read + 24 write) for the spins of the T particles with a torque
    # (in contact with a particle or a wall: at most 2 per contact and 1 per
    # wall contact; under Euler the others keep theirs untouched, all of
    # them otherwise), P*(4 id + 24 PFT read + 24 PFT write), and for a
    # periodic system the DES cell and facet flag the integration writes
    # (N*5)
    t = n_normal if n_torque is None else min(n_normal, n_torque)
    return n_normal * (121 if periodic else 116) + t * 56 + n_pairs * 52


def torqued(stats, integrator):
    """The particles whose spin the integration must read and write: with
    Euler at most two per particle contact and one per wall contact, with
    Adams-Bashforth all."""
    if integrator != "euler":
        return None
    return 2 * int(stats["n_contacts"]) + int(stats["n_wall_contacts"])


def cpu_sample(args, threads=None):
    """The oracle in its OpenMP mode on a bounded sample of the workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_ffi import OracleSystem
    threads = threads or os.cpu_count() or 1
    case, prm, arr, walls, info = workload(args.cpu_sample, "fp64", args.inflate)
    o = OracleSystem(prm, arr["pos"].shape[1], openmp=True, threads=threads, native=True)
    o.set_walls(*walls)
    o.upload_state(arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                   arr["state"], arr["phase"])
    o.init_neighbors()
    o.step(1, 1)  # warm-up (includes the first rebuild)
    t0 = time.perf_counter()
    o.step(args.cpu_steps, 2)
    dt = time.perf_counter() - t0
    n = int(o.stats()["n_normal"])
    return {"value": n * args.cpu_steps / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{n} particles of the same workload (box scaled to keep density and bed height), "
                      f"{args.cpu_steps} steps incl. {args.cpu_steps // 25} neighbour rebuilds, OpenMP oracle "
                      f"(-O3 -march=native), {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    t_all = time.perf_counter()
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_ffi import OracleSystem
    threads = os.cpu_count() or 1
    case, prm, arr, walls, info = workload(args.cpu_sample, "fp64", args.inflate)
    o = OracleSystem(prm, arr["pos"].shape[1], openmp=True, threads=threads, native=True)
    o.set_walls(*walls)
    o.upload_state(arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                   arr["state"], arr["phase"])
    o.init_neighbors()
    # the same window placement as the GPU arm: W warm-up steps or more, and
    # K timed steps ending on a rebuild step
    nsn = int(prm.neighbor_search_n)
    nn0, rebuilds = timed_window(max(args.warmup, 1), args.steps, nsn)
    o.step(nn0 - 1, 1)
    t0 = time.perf_counter()
    o.step(args.steps, nn0)
    dt = time.perf_counter() - t0
    n = int(o.stats()["n_normal"])
    value = n * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": bench_config(args, info, prm) | {"n_particles": n, "precision": "fp64",
                                                   "timed_window_nn": [nn0, nn0 + args.steps - 1],
                                                   "rebuilds_timed": rebuilds},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{n} particles of the {workload_name(args.inflate)} workload, "
                                   f"{args.steps} timed steps incl. {rebuilds} neighbour rebuilds, OpenMP "
                                   "C++ restatement of the Fortran reference (-O3 -march=native; the "
                                   "Fortran reference cannot be compiled here)"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t_all,
    }
    print(json.dumps(line), flush=True)


def _timed_run(args, prec, stream, barrier, ws, local, with_e2e):
    """Builds one system for `prec`, runs W warm-up steps, then K timed steps
    bracketed by CUDA events on the library's stream; returns the figures."""
    import torch
    from mfix_dem import GpuSystem
    case, prm, arr, walls, info = workload(args.n, prec, args.inflate)
    n = arr["pos"].shape[1]
    g = GpuSystem(prm, n)
    g.set_stream(stream.cuda_stream)
    g.set_walls(*walls)
    g.upload_state(arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                   arr["state"], arr["phase"])
    g.init_neighbors()
    # warm-up: at least W steps and at least three periods, so that both
    # CUDA graphs of a period (the buffer parities alternate) are captured;
    # the timed window then ends on a rebuild step
    nsn = int(prm.neighbor_search_n)
    nn0, rebuilds = timed_window(max(args.warmup, 3 * nsn), args.steps, nsn)
    warm = nn0 - 1
    g.step(5, 1)
    tuning = g.autotune(reps=3)  # before the graphs are captured (a new shape drops them)
    g.step(warm - 5, 6)
    torch.cuda.synchronize()
    ferr0 = g.force_error() if prec == "split" else None
    clocks = ClockSampler(local)
    clocks.start()
    p0 = g.pair_count()
    l0 = g.launch_count()
    f0 = g.stats()["n_builds_filtered"]
    barrier()
    torch.cuda.synchronize()
    clocks.begin()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    g.step(args.steps, warm + 1)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = g.launch_count() - l0
    p1 = g.pair_count()
    st = g.stats()
    # kernel times: a second pass of the same length with CUDA events around
    # every kernel class, launched step by step (events cannot sit inside the
    # graphs the timed pass replays)
    g.set_profiling(True)
    ep0 = torch.cuda.Event(enable_timing=True)
    ep1 = torch.cuda.Event(enable_timing=True)
    ep0.record(stream)
    g.step(args.steps, warm + args.steps + 1)
    ep1.record(stream)
    torch.cuda.synchronize()
    ms_eager = ep0.elapsed_time(ep1)
    prof = g.profile()
    # the parts of the force step, timed on a short extra pass (their
    # events split the step, so they are not used for the roofline)
    g.set_profiling(2)
    g.step(10, warm + 2 * args.steps + 1)
    parts = {k: v[0] / v[1] for k, v in g.profile().items() if k in ("walls", "pairs", "gather") and v[1]}
    g.set_profiling(False)
    ferr1 = g.force_error() if prec == "split" else None
    ms = max_over_ranks(ms, ws, "cuda")
    n_normal = int(st["n_normal"])
    value = ws * n_normal * args.steps / (ms / 1e3)

    # roofline of the dominant kernel class (contact forces + fused integration)
    f_ms, f_n = prof["force"]
    peak, peak_kind = measured_peak()
    p_avg = 0.5 * (p0 + p1)
    bytes_launch = algorithmic_bytes(n_normal, p_avg, n_torque=torqued(st, "euler"))
    achieved = bytes_launch / (f_ms / f_n / 1e3) / 1e9 if f_n else None
    traffic = None
    if PROFILE_TRAFFIC.exists():
        tr = json.loads(PROFILE_TRAFFIC.read_text())
        key = f"{workload_name(args.inflate)}:{prec}"
        traffic = tr.get(key)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": "force step (k_walls + k_pairs + k_gather with fused integration)",
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_launch,
                "avg_launch_ms": f_ms / f_n if f_n else None,
                "share_of_step": f_ms / ms_eager if ms_eager else None,
                "ms_per_step_eager": ms_eager / args.steps,
                "kernel_ms": {k: v[0] for k, v in prof.items() if v[1]},
                "force_parts_ms_per_launch": parts}
    out = {"value": value, "ms": ms, "n": n, "n_normal": n_normal, "pairs": int(p1), "launches": int(launches),
           "warmup": warm, "tuning": tuning, "window": [warm + 1, warm + args.steps], "rebuilds_timed": rebuilds,
           "rebuilds_timed_filtered": int(st["n_builds_filtered"] - f0),
           "candidate_list": {"lists_made": int(st["n_candidate_lists"]),
                              "builds_filtered": int(st["n_builds_filtered"])},
           "roofline": roofline, "clocks": clk, "contacts": int(st["n_contacts"]), "prm": prm, "info": info,
           "force_error": None if ferr0 is None else [ferr0, ferr1]}

    # e2e: per step, H2D of the particle arrays from pinned host memory, one
    # DES_TIME_STEP through the C ABI, D2H of the new positions/velocities/spins
    if with_e2e and args.e2e_steps > 0:
        def pinned(a):
            t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.int8: torch.int8,
                                            np.int32: torch.int32}[a.dtype.type], pin_memory=True)
            t.numpy()[...] = a
            return t.numpy()
        nn_e0, e2e_rebuilds = timed_window(warm + 2 * args.steps + 10, args.e2e_steps, nsn)
        g.step(nn_e0 - (warm + 2 * args.steps + 11), warm + 2 * args.steps + 11)
        st_now = g.download_state()
        # the driver's moving state goes in every step (positions, velocities,
        # spins); radius, mass, inertia, state and phase stay on the device
        hin = {"pos": pinned(st_now["pos"]), "vel": pinned(st_now["vel"]), "omega": pinned(st_now["omega"]),
               "state": pinned(st_now["state"])}
        hout = {"pos": hin["pos"], "vel": hin["vel"], "omega": hin["omega"], "state": hin["state"]}
        nn0 = nn_e0
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.e2e_steps):
            g.upload_state(hin["pos"], hin["vel"], hin["omega"])
            g.step(1, nn0 + k)
            g.download_state(out=hout)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        ems = max_over_ranks(ems, ws, "cuda")
        out["e2e"] = {"value": ws * n_normal * args.e2e_steps / (ems / 1e3), "unit": METRIC,
                      "h2d_bytes_per_step": n * 9 * 8, "d2h_bytes_per_step": n * (9 * 8 + 1),
                      "steps": args.e2e_steps, "rebuilds_timed": e2e_rebuilds,
                      "note": "each step: dem_upload_state of DES_POS_NEW, DES_VEL_NEW and OMEGA_NEW from pinned host "
                              "arrays (the per-particle constants stay on the device), dem_step, dem_download_state "
                              "of positions, velocities, spins and states"}
    g.close()
    return out


def _batched_run(args, prec, stream, systems, info, barrier):
    """The batched workload: every system of `systems` in one batch handle.
    Warm-up up to the first period boundary (NN = 26), autotune, then K steps
    (a multiple of NEIGHBOR_SEARCH_N, replayed as captured periods) timed with
    CUDA events on the library's stream, and an eager pass with kernel-class
    timing for the roofline."""
    import torch
    from mfix_dem import GpuBatch, abi, load_library
    from mfix_dem import params as P
    entries = [(s[1], s[2]["pos"].shape[1], s[3][0].shape[0]) for s in systems]
    lim = P.batch_limits(load_library(), entries, max_systems=len(systems))
    bt = GpuBatch(systems[0][1], lim)
    bt.set_stream(stream.cuda_stream)
    ids = []
    for case, prm, arr, walls, _ in systems:
        sid = bt.add(prm, arr["pos"].shape[1])
        bt.set_walls(sid, *walls)
        bt.upload_state(sid, arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                        arr["state"], arr["phase"])
        ids.append(sid)
    bt.start(ids)
    nsn = int(systems[0][1].neighbor_search_n)
    warm = max(args.warmup, 3 * nsn)
    warm = ((warm + nsn - 1) // nsn) * nsn  # NN = m*N + 1 next, both period graphs captured
    # tune first (a new launch shape drops the captured graphs), then warm up
    bt.step(5)
    tuning = bt.autotune(reps=3)
    bt.step(warm - 5)
    # at least four periods: one period is ~15 ms, short enough for a host
    # hiccup (clock sampling, the per-period pair-count read) to show
    steps = max(((args.steps + nsn - 1) // nsn) * nsn, 4 * nsn)
    torch.cuda.synchronize()
    p0 = bt.pair_count()
    l0 = bt.launch_count()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    clocks.begin()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    bt.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks.end()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = bt.launch_count() - l0
    p1 = bt.pair_count()
    st = bt.total_stats()
    bt.set_profiling(True)
    bt.step(steps)
    torch.cuda.synchronize()
    prof = bt.profile()
    bt.set_profiling(2)
    bt.step(10)
    parts = {k: v[0] / v[1] for k, v in bt.profile().items() if k in ("walls", "pairs", "gather") and v[1]}
    bt.set_profiling(False)
    n_normal = int(st["n_normal"])
    f_ms, f_n = prof["force"]
    peak, peak_kind = measured_peak()
    bytes_launch = algorithmic_bytes(n_normal, 0.5 * (p0 + p1), periodic=False, n_torque=torqued(st, "euler"))
    achieved = bytes_launch / (f_ms / f_n / 1e3) / 1e9 if f_n else None
    final = {sid: bt.download_state(sid)["pos"] for sid in ids}
    bt.close()
    return {"value": n_normal * steps / (ms / 1e3), "ms_per_step": ms / steps, "steps": steps, "warmup": warm,
            "n_normal": n_normal, "pairs": int(p1), "gpu_launches": int(launches), "tuning": tuning,
            "clocks": clk,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": None,
                         "kernel": "force step over all systems (walls + pairs + gather with fused integration)",
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_launch,
                         "avg_launch_ms": f_ms / f_n if f_n else None,
                         "kernel_ms": {k: v[0] for k, v in prof.items() if v[1]},
                         "force_parts_ms_per_launch": parts},
            "final_pos": final}


def run_batched(args, stream, barrier, ws, rank):
    """Split-precision and FP64 runs of the same batch; the split run's
    trajectory error is max over systems of max|x_split - x_fp64| / max|x_fp64|
    after the same steps.  With N ranks the systems are spread by a greedy
    size balance (mfix_dem.partition), one batch handle per GPU; the job's
    time is the slowest rank's and its particle-steps the sum over ranks."""
    from mfix_dem import abi, configs
    from mfix_dem.partition import gather_metrics, partition_work
    out = {}
    for prec in ("split", "fp64"):
        systems, info = configs.batched(n_sys=args.batch_systems, total=args.batch_total,
                                        precision=abi.DEM_PREC_SPLIT if prec == "split" else abi.DEM_PREC_FP64)
        part = partition_work([s[2]["pos"].shape[1] for s in systems], ws)
        mine = [systems[i] for i in part[rank]]
        r = _batched_run(args, prec, stream, mine, info, barrier)
        m = gather_metrics({"ms": r["ms_per_step"] * r["steps"], "ps": r["value"] * r["ms_per_step"] * r["steps"] / 1e3},
                           ws, "cuda")
        r["rank_particle_steps_per_s"] = r["value"]
        r["ms_per_step"] = max(m["ms"]) / r["steps"]
        r["value"] = sum(m["ps"]) / (max(m["ms"]) / 1e3)
        r["partition"] = {"ranks": ws, "systems_per_rank": [len(p) for p in part],
                          "particles_per_rank": [sum(systems[i][2]["pos"].shape[1] for i in p) for p in part]}
        out[prec] = r
        out["info"] = info
    err = 0.0
    for sid, xs in out["split"]["final_pos"].items():
        xd = out["fp64"]["final_pos"][sid]
        err = max(err, float(np.max(np.abs(xs - xd)) / max(np.max(np.abs(xd)), 1e-300)))
    for prec in ("split", "fp64"):
        out[prec].pop("final_pos")
    out["trajectory_rel_err"] = max(gather_metrics({"e": err}, ws, "cuda")["e"])
    return out


def run_served(args, barrier, ws, rank):
    """Poisson streams of hopper-discharge cases served with continuous
    batching (mfix_dem.serve.DemServer); per rate: p50/p99 latency from
    arrival to completion and the aggregate particle-steps/s.  With N ranks
    each request goes, in arrival order, to the rank with the least
    particle-steps assigned so far (mfix_dem.partition); each rank serves its
    share on its own GPU and the latencies are gathered."""
    from mfix_dem import configs, load_library
    from mfix_dem.partition import gather_list, gather_metrics, partition_requests
    from mfix_dem.serve import DemServer

    def build(req):
        return configs.hopper_case(req["n"], friction=req["friction"], outlet_d=req["outlet_d"], seed=req["seed"])

    rates = [float(r) for r in args.serve_rates.split(",") if r.strip()]
    out = []
    template = build({"n": 5000, "friction": 0.4, "outlet_d": 8, "seed": 1})
    for k, rate in enumerate(rates):
        reqs_all = configs.hopper_requests(args.serve_requests, rate, seed=configs.SEED_BASE + 4 + 100 * k,
                                           steps=args.serve_steps)
        reqs = partition_requests(reqs_all, ws)[rank]
        srv = DemServer(load_library(), build, template, hbm_budget_bytes=int(args.serve_budget_gb * 1e9),
                        max_systems=64, graphs=bool(args.serve_graphs))
        server_bytes = srv.footprint["bytes"]
        barrier()
        res = srv.run(reqs)
        srv.close()
        lat = gather_list([r.latency for r in res["results"]], ws, "cuda")
        # particles that left through the outlet (deleted as rogue)
        gone = sum(r.n - int(r.stats["n_normal"]) for r in res["results"])
        m = gather_metrics({"work": res["particle_steps"], "span": res["span_s"], "busy": res["busy_s"],
                            "chunks": res["chunks"], "gone": float(gone)}, ws, "cuda")
        span = max(m["span"])
        out.append({"rate_per_s": rate, "requests": len(reqs_all), "p50_s": float(np.percentile(lat, 50)),
                    "p99_s": float(np.percentile(lat, 99)), "mean_s": float(np.mean(lat)),
                    "particle_steps_per_s": sum(m["work"]) / span if span > 0 else 0.0,
                    "span_s": span, "gpu_busy_s": max(m["busy"]), "chunks": int(sum(m["chunks"])),
                    "particles_discharged": int(sum(m["gone"])), "server_footprint_gb": server_bytes / 1e9,
                    "ranks": ws})
    return out


def serve_profile(args):
    """Per-chunk cost of the served pattern: three hopper cases (20k, 60k and
    150k particles) admitted together and run 500 steps (20 chunks of 25),
    on servers of two sizes (40 GB / 64 system slots and 4 GB / 8 slots),
    once with graph replay (wall time per chunk) and once eagerly with the
    kernel classes timed by CUDA events (ms per chunk and launches)."""
    import torch
    from mfix_dem import configs, load_library
    from mfix_dem.serve import DemServer
    torch.cuda.set_device(0)
    cases = {}

    def build(req):
        if req["n"] not in cases:
            cases[req["n"]] = configs.hopper_case(req["n"], friction=req["friction"], outlet_d=req["outlet_d"],
                                                  seed=req["seed"])
        return cases[req["n"]]

    template = configs.hopper_case(5000)
    out = []
    for budget, msys, prof in ((40, 64, False), (4, 8, False), (40, 64, True), (4, 8, True)):
        reqs = [dict(rid=k, arrival=0.0, n=n, friction=0.4, outlet_d=8, seed=k, steps=500)
                for k, n in enumerate((20_000, 60_000, 150_000))]
        srv = DemServer(load_library(), build, template, hbm_budget_bytes=int(budget * 1e9), max_systems=msys,
                        graphs=True, builders=0)
        if prof:
            srv.batch.set_profiling(1)
        res = srv.run(reqs)
        row = {"budget_gb": budget, "system_slots": msys, "timed_classes": prof, "chunks": res["chunks"],
               "ms_per_chunk": 1e3 * res["busy_s"] / res["chunks"], "particles": 230_000,
               "server_footprint_gb": srv.footprint["bytes"] / 1e9}
        if prof:
            row["classes_ms_per_chunk"] = {k: v[0] / res["chunks"] for k, v in srv.batch.profile().items() if v[1]}
            row["launches_per_chunk"] = {k: v[1] / res["chunks"] for k, v in srv.batch.profile().items() if v[1]}
        srv.close()
        out.append(row)
    print(json.dumps({"serve_profile": out}), flush=True)


def run_ours(args):
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    stream = torch.cuda.Stream()
    main = _timed_run(args, args.precision, stream, barrier, ws, local, with_e2e=True)
    other = None
    if args.precision == "fp64" and not args.no_split:
        other = _timed_run(args, "split", stream, barrier, ws, local, with_e2e=False)
    rsa40 = None
    if args.inflate != 1.0 and not args.no_rsa40:
        import copy
        a40 = copy.copy(args)
        a40.inflate = 1.0
        rsa40 = _timed_run(a40, "fp64", stream, barrier, ws, local, with_e2e=False)

    batched = None
    if args.batch_systems > 0:
        batched = run_batched(args, stream, barrier, ws, rank)

    served = None
    if args.serve_rates.strip():
        served = run_served(args, barrier, ws, rank)

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            cpu = cpu_sample(args)
        except Exception as ex:  # reported, not fatal
            cpu = {"error": str(ex)}

    if rank == 0:
        prm, info = main["prm"], main["info"]
        line = {
            "metric": METRIC, "value": main["value"], "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": main["warmup"], "warmup_requested": args.warmup, "ms_per_step": main["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": bench_config(args, main["info"], main["prm"]) | {
                       "n_particles": main["n_normal"], "n_pairs": main["pairs"],
                       "pairs_per_particle": main["pairs"] / max(main["n_normal"], 1),
                       "precision": args.precision,
                       "contacts_last_step": main["contacts"],
                       "timed_window_nn": main["window"], "rebuilds_timed": main["rebuilds_timed"],
                       "rebuilds_timed_from_candidate_list": main["rebuilds_timed_filtered"],
                       "candidate_list_since_start": main["candidate_list"],
                       "l2": "inputs larger than L2 (state and pair arrays ~%.0f MB)" % (
                           (main["n"] * 3 * 32 * 2 + main["pairs"] * 100) / 1e6),
                       "parallelism": f"replicas x{ws}"},
            "roofline": main["roofline"],
            "tuning": main["tuning"],
            "cpu_baseline": cpu,
            "clocks": main["clocks"],
            "e2e": main.get("e2e"),
            "gpu_launches": main["launches"],
        }
        if other is not None:
            line["split"] = {"value": other["value"], "ms_per_step": other["ms"] / args.steps,
                             "speedup_vs_fp64": other["value"] / main["value"],
                             "force_rel_error_first_last": other["force_error"],
                             "force_error_note": ("max over particles and components of |F_split - F_fp64| / "
                                                  "max |F_fp64| on one state, before and after the timed "
                                                  "steps; contacts within 1e-4 of the onset of slip, where "
                                                  "the friction law turns the tangential force "
                                                  "(calc_force_dem.f:330-342), take the FP64 test's branch"),
                             "contacts_last_step": other["contacts"], "rebuilds_timed": other["rebuilds_timed"],
                             "rebuilds_timed_from_candidate_list": other["rebuilds_timed_filtered"],
                             "roofline": other["roofline"], "gpu_launches": other["launches"],
                             "tuning": other["tuning"],
                             "clocks": other["clocks"]}
        if rsa40 is not None:
            line["rsa40"] = {"workload": workload_name(1.0), "precision": "fp64",
                             "note": "the placement as placed (40 % solids): no contacts within the timed steps",
                             "value": rsa40["value"], "ms_per_step": rsa40["ms"] / args.steps,
                             "contacts_last_step": rsa40["contacts"], "n_pairs": rsa40["pairs"],
                             "rebuilds_timed": rsa40["rebuilds_timed"],
                             "rebuilds_timed_from_candidate_list": rsa40["rebuilds_timed_filtered"],
                             "roofline": rsa40["roofline"],
                             "gpu_launches": rsa40["launches"], "clocks": rsa40["clocks"]}
        if batched is not None:
            b = batched
            line["batched"] = {
                "workload": f"batched_{b['info']['n_systems']}", "config": b["info"],
                "value": b["split"]["value"], "unit": METRIC, "precision": "split",
                "ms_per_step": b["split"]["ms_per_step"], "steps": b["split"]["steps"],
                "warmup": b["split"]["warmup"], "roofline": b["split"]["roofline"],
                "tuning": b["split"]["tuning"], "gpu_launches": b["split"]["gpu_launches"],
                "clocks": b["split"]["clocks"],
                "fp64": {"value": b["fp64"]["value"], "ms_per_step": b["fp64"]["ms_per_step"],
                         "roofline": b["fp64"]["roofline"], "tuning": b["fp64"]["tuning"],
                         "clocks": b["fp64"]["clocks"]},
                "speedup_split_vs_fp64_batched": b["split"]["value"] / b["fp64"]["value"],
                "speedup_vs_plain_fp64_single": b["split"]["value"] / main["value"],
                "trajectory_rel_err_vs_fp64": b["trajectory_rel_err"],
                "n_pairs": b["split"]["pairs"]}
        if served is not None:
            from mfix_dem import configs as _cfg
            dt = float(_cfg.hopper_case(5000)[1].dtsolid)
            line["served"] = {
                "workload": "hopper_discharge_poisson", "precision": "split", "integration": "fp64",
                "steps_per_case": args.serve_steps, "particles_per_case": "log-uniform 5,000-500,000",
                "hbm_budget_gb": args.serve_budget_gb,
                "admission": "footprint counted by the library (dem_batch_footprint): limits sized to the budget, "
                             "a case admitted when its particle/cell/facet ranges and its pair-list room are free",
                "physical_time_per_case_s": dt * args.serve_steps,
                "note": "latency = completion - arrival (case built on the host after arrival), wall clock; at "
                        "DTSOLID %.3g s the steps per case cover %.3g s, in which the fill (starting at rest "
                        "about 0.19 m above the outlet) falls under a millimetre: no particle reaches the "
                        "outlet, which would take about 0.2 s (~%d k steps) per case" % (
                            dt, dt * args.serve_steps, int(0.2 / dt / 1000)),
                "rates": served}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.serve_profile:
        serve_profile(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
