#!/usr/bin/env python3
"""bench.py -- DEM particle step throughput on B200.

Workload: 1,000,000 polydisperse Hertzian spheres (lognormal d, median 1 mm,
sigma 0.25, clipped to 0.5-2 mm; rho 2500; E 1e7, nu 0.3; e_n = e_t = 0.85;
friction 0.3, rolling friction 0.01) in a 0.1 x 0.4 x 0.1 m box, periodic in x
and z with a flat bottom wall, seeded random sequential placement at 40 %
solids.  One step = one DES_TIME_STEP (contact forces, walls, integration, and
the neighbour rebuild every NEIGHBOR_SEARCH_N = 25 steps).

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
    ap.add_argument("--cpu-sample", type=int, default=125_000, help="particles in the CPU sample")
    ap.add_argument("--cpu-steps", type=int, default=25)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision leg")
    ap.add_argument("--inflate", type=float, default=1.0,
                    help="grow every sphere by this factor after placement (contact-dense variant)")
    return ap.parse_args()


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


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
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
                "samples": len(sm)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(n_normal, n_pairs):
    # per step: N*(96 read + 72 write + 4 CSR) + P*(4 id + 24 PFT read + 24 PFT write)
    return n_normal * 172 + n_pairs * 52


def cpu_sample(args, threads=None):
    """The oracle in its OpenMP mode on a bounded sample of the workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_ffi import OracleSystem
    threads = threads or os.cpu_count() or 1
    case, prm, arr, walls, info = workload(args.cpu_sample, args.precision if args.precision == "fp64" else "fp64")
    o = OracleSystem(prm, arr["pos"].shape[1], openmp=True, threads=threads)
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
                      f"{args.cpu_steps} steps incl. one neighbour rebuild, OpenMP oracle, {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    t_all = time.perf_counter()
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle_ffi import OracleSystem
    threads = os.cpu_count() or 1
    case, prm, arr, walls, info = workload(args.cpu_sample, "fp64")
    o = OracleSystem(prm, arr["pos"].shape[1], openmp=True, threads=threads)
    o.set_walls(*walls)
    o.upload_state(arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                   arr["state"], arr["phase"])
    o.init_neighbors()
    o.step(max(args.warmup, 1), 1)
    t0 = time.perf_counter()
    o.step(args.steps, max(args.warmup, 1) + 1)
    dt = time.perf_counter() - t0
    n = int(o.stats()["n_normal"])
    value = n * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "hertz_rsa_1m (sampled)", "n_particles": n, "periodic": "xz",
                   "contact": "hertz", "integrator": "euler"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{n} particles of the 1M workload (same density/bed height), "
                                   f"{args.steps} timed steps, OpenMP C++ restatement of the Fortran "
                                   "reference (the Fortran reference cannot be compiled here)"},
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
    g.step(args.warmup, 1)
    torch.cuda.synchronize()
    ferr0 = g.force_error() if prec == "split" else None
    clocks = ClockSampler(local)
    p0 = g.pair_count()
    l0 = g.launch_count()
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    g.step(args.steps, args.warmup + 1)
    ev1.record(stream)
    torch.cuda.synchronize()
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
    g.step(args.steps, args.warmup + args.steps + 1)
    ep1.record(stream)
    torch.cuda.synchronize()
    ms_eager = ep0.elapsed_time(ep1)
    prof = g.profile()
    g.set_profiling(False)
    ferr1 = g.force_error() if prec == "split" else None
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    n_normal = int(st["n_normal"])
    value = ws * n_normal * args.steps / (ms / 1e3)

    # roofline of the dominant kernel class (contact forces + fused integration)
    f_ms, f_n = prof["force"]
    peak, peak_kind = measured_peak()
    p_avg = 0.5 * (p0 + p1)
    bytes_launch = algorithmic_bytes(n_normal, p_avg)
    achieved = bytes_launch / (f_ms / f_n / 1e3) / 1e9 if f_n else None
    traffic = None
    if PROFILE_TRAFFIC.exists():
        tr = json.loads(PROFILE_TRAFFIC.read_text())
        key = f"{'hertz_rsa_1m' if args.inflate == 1.0 else 'hertz_rsa_1m_inflated'}:{prec}"
        traffic = tr.get(key)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "kernel": "force step (k_walls + k_pairs + k_gather with fused integration)",
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": bytes_launch,
                "avg_launch_ms": f_ms / f_n if f_n else None,
                "share_of_step": f_ms / ms_eager if ms_eager else None,
                "ms_per_step_eager": ms_eager / args.steps,
                "kernel_ms": {k: v[0] for k, v in prof.items() if v[1]}}
    out = {"value": value, "ms": ms, "n": n, "n_normal": n_normal, "pairs": int(p1), "launches": int(launches),
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
        st_now = g.download_state()
        hin = {"pos": pinned(st_now["pos"]), "vel": pinned(st_now["vel"]), "omega": pinned(st_now["omega"]),
               "radius": pinned(arr["radius"]), "pmass": pinned(arr["pmass"]), "omoi": pinned(arr["omoi"]),
               "state": pinned(st_now["state"]), "phase": pinned(arr["phase"])}
        hout = {"pos": hin["pos"], "vel": hin["vel"], "omega": hin["omega"], "state": hin["state"]}
        nn0 = args.warmup + 2 * args.steps + 1
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.e2e_steps):
            g.upload_state(hin["pos"], hin["vel"], hin["omega"], hin["radius"], hin["pmass"], hin["omoi"],
                           hin["state"], hin["phase"])
            g.step(1, nn0 + k)
            g.download_state(out=hout)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if ws > 1:
            import torch.distributed as dist
            t = torch.tensor([ems], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        out["e2e"] = {"value": ws * n_normal * args.e2e_steps / (ems / 1e3), "unit": METRIC,
                      "h2d_bytes_per_step": n * (9 * 8 + 3 * 8 + 1 + 4), "d2h_bytes_per_step": n * (9 * 8 + 1),
                      "steps": args.e2e_steps,
                      "note": "each step: dem_upload_state from pinned host arrays, dem_step, dem_download_state"}
    g.close()
    return out


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

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            cpu = cpu_sample(args)
        except Exception as ex:  # reported, not fatal
            cpu = {"error": str(ex)}

    if rank == 0:
        prm, info = main["prm"], main["info"]
        wl = "hertz_rsa_1m" if args.inflate == 1.0 else f"hertz_rsa_1m_inflated_{args.inflate:g}"
        line = {
            "metric": METRIC, "value": main["value"], "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": wl, "n_particles": main["n_normal"], "n_pairs": main["pairs"],
                       "pairs_per_particle": main["pairs"] / max(main["n_normal"], 1),
                       "precision": args.precision, "contact": "hertz", "integrator": "euler",
                       "periodic": "xz", "neighbor_search_n": int(prm.neighbor_search_n),
                       "solids_fraction": info.get("solids_fraction"), "dtsolid": prm.dtsolid,
                       "contacts_last_step": main["contacts"],
                       "l2": "inputs larger than L2 (state and pair arrays ~%.0f MB)" % (
                           (main["n"] * 3 * 32 * 2 + main["pairs"] * 100) / 1e6),
                       "parallelism": f"replicas x{ws}"},
            "roofline": main["roofline"],
            "cpu_baseline": cpu,
            "clocks": main["clocks"],
            "e2e": main.get("e2e"),
            "gpu_launches": main["launches"],
        }
        if other is not None:
            line["split"] = {"value": other["value"], "ms_per_step": other["ms"] / args.steps,
                             "speedup_vs_fp64": other["value"] / main["value"],
                             "force_rel_error_first_last": other["force_error"],
                             "roofline": other["roofline"], "gpu_launches": other["launches"],
                             "clocks": other["clocks"]}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
