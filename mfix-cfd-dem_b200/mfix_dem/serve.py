"""Serving DEM cases with continuous batching (no counterpart in the
reference, which runs one case per process).

`DemServer` keeps one batch handle resident on the device.  Its limits are
sized from the HBM budget with the library's own count of the arrays a
batch allocates (dem_batch_footprint): cell, facet and bin ranges for
`max_systems` cases of the template's box, pair-list room of
`pairs_per_particle` per particle, and the rest of the budget to particles.
Requests arrive over time; each is built on the host (in worker threads),
admitted into the batch as soon as its footprint fits -- its particle, cell,
facet and bin ranges are taken from the free ranges of the limits, and the
pairs of the running cases plus its own estimate fit the pair-list room --
and then steps with everything else already running.  Admission and
retirement happen between chunks of NEIGHBOR_SEARCH_N steps; a finished case
is downloaded and removed, and its ranges go to the next arrivals.
Because every system of a batch keeps its own step numbering and rebuild
cadence, a case's result does not depend on what else was running
(tests/test_gpu_serve.py checks it against the case served alone).

Latency of a request = completion time - arrival time, on the server's clock.
"""
from __future__ import annotations

import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import abi
from . import params as P
from .system import BatchSystem, DemError


def footprint(lib, prm, lim) -> dict:
    """dem_batch_footprint: device bytes of a batch handle with limits lim
    (array_bytes, pair_bytes, pair_capacity)."""
    import ctypes as C
    m = abi.DemMemory()
    rc = lib.dem_batch_footprint(C.byref(prm), C.byref(lim), C.byref(m))
    if rc != 0:
        raise ValueError("invalid batch limits")
    d = m.as_dict()
    d["bytes"] = d["array_bytes"] + d["pair_bytes"]
    return d


def limits_for_budget(lib, prm, n_facets: int, budget_bytes: int, max_systems: int, pairs_per_particle: int = 6):
    """Batch limits whose footprint fits budget_bytes: the cell, facet and
    bin ranges of max_systems systems like `prm` (with n_facets facets), and
    the particle capacity the rest of the budget pays for.  The footprint is
    affine in the particle capacity, so two evaluations give the bytes per
    particle (its arrays and its pair-list room).  Returns (limits,
    bytes_per_particle)."""
    per = P.batch_limits(lib, [(prm, 64, n_facets)], max_systems=1)
    lim = abi.DemBatchLimits()
    lim.max_systems = int(max_systems)
    lim.max_cells = int(per.max_cells) * max_systems
    lim.max_search_cells = int(per.max_search_cells) * max_systems
    lim.max_facets = int(per.max_facets) * max_systems
    lim.max_facet_bins = int(per.max_facet_bins) * max_systems
    lim.pairs_per_particle = int(pairs_per_particle)
    step = 1 << 20
    lim.max_particles = 64
    f0 = footprint(lib, prm, lim)["bytes"]
    lim.max_particles = 64 + step
    per_particle = (footprint(lib, prm, lim)["bytes"] - f0) / step
    n = int((budget_bytes - f0) // per_particle) + 64
    n = min(n, (1 << 27) - 64) // 64 * 64
    if n < 64:
        raise ValueError(f"{budget_bytes} bytes do not hold the cell ranges of {max_systems} systems")
    lim.max_particles = n
    assert footprint(lib, prm, lim)["bytes"] <= budget_bytes
    return lim, per_particle


@dataclass
class Result:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    stats: dict
    state: Optional[dict] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class _Running:
    req: dict
    sid: int
    admitted: float
    done: int = 0


class DemServer:
    """Continuous-batching loop over one batch handle.

    build(req) -> (case, prm, arr, walls, info) makes a request's case on the
    host; `template` is one such case, whose DES grid sizes every admitted
    case must not exceed (all requests of a server share the box).
    """

    def __init__(self, lib, build: Callable, template, hbm_budget_bytes: int, max_systems: int = 64,
                 chunk: int = 25, builders: int = 2, graphs: bool = False, batch=None, pairs_per_particle: int = 6):
        self.lib = lib
        self.build = build
        self.chunk = int(chunk)
        self.pairs_per_particle = int(pairs_per_particle)
        _, prm, arr, walls, _ = template
        lim, self.bytes_per_particle = limits_for_budget(lib, prm, walls[0].shape[0], hbm_budget_bytes,
                                                         max_systems, pairs_per_particle)
        self.limits = lim
        self.footprint = footprint(lib, prm, lim)
        # `batch` replaces the device batch (the CPU tests pass a model of it)
        self.batch = batch if batch is not None else BatchSystem(lib, prm, lim)
        self.batch.set_graphs(graphs)
        self.pool = ThreadPoolExecutor(max_workers=builders) if builders > 0 else None
        self.chunks_done = 0

    def close(self):
        if self.pool is not None:
            self.pool.shutdown(wait=False)
        self.batch.close()

    def request_footprint(self, case) -> int:
        """Device bytes a case takes: the footprint of a batch holding it
        alone (its particle, cell, facet and bin ranges and its pair-list
        room)."""
        _, prm, arr, walls, _ = case
        lim = P.batch_limits(self.lib, [(prm, arr["pos"].shape[1], walls[0].shape[0])], max_systems=1)
        lim.pairs_per_particle = self.pairs_per_particle
        return footprint(self.lib, prm, lim)["bytes"]

    def _admit(self, req, case, now, pairs_pending: int) -> Optional[_Running]:
        _, prm, arr, walls, _ = case
        bt = self.batch
        # the pairs of the running cases (last build), those admitted in this
        # round and this case's estimate must fit the pair-list room
        mem = bt.memory_info()
        if mem["pairs"] + pairs_pending + self.pairs_per_particle * arr["pos"].shape[1] > mem["pair_capacity"]:
            return None
        try:
            sid = bt.add(prm, arr["pos"].shape[1])
        except DemError as e:
            if e.code == abi.DEM_ERR_CAPACITY:
                return None
            raise
        try:
            bt.set_walls(sid, *walls)
        except DemError as e:
            bt.remove(sid)
            if e.code == abi.DEM_ERR_CAPACITY:
                return None
            raise
        bt.upload_state(sid, arr["pos"], arr["vel"], arr["omega"], arr["radius"], arr["pmass"], arr["omoi"],
                        arr["state"], arr["phase"])
        return _Running(req=req, sid=sid, admitted=now)

    def run(self, requests, clock: Optional[Callable[[], float]] = None, keep_state: bool = False,
            idle_sleep: float = 0.0005) -> dict:
        """Serves `requests` (dicts with rid, arrival [s], n, steps, ...) to
        completion.  `clock` returns seconds (default: wall time from the
        start of the call); steps of a request must be a multiple of the
        chunk."""
        if clock is None:
            t0 = time.perf_counter()
            clock = lambda: time.perf_counter() - t0  # noqa: E731
        for r in requests:
            if r["steps"] % self.chunk:
                raise ValueError("steps per request must be a multiple of the chunk")
        pend = deque(sorted(requests, key=lambda r: r["arrival"]))
        building = deque()   # (req, future or case), arrival order
        running: dict[int, _Running] = {}
        results: list[Result] = []
        bt = self.batch
        chunks = 0
        busy = 0.0
        while pend or building or running:
            now = clock()
            while pend and pend[0]["arrival"] <= now:
                r = pend.popleft()
                building.append((r, self.pool.submit(self.build, r) if self.pool else self.build(r)))
            # admit every built request that fits, in arrival order
            new = []
            keep = deque()
            pending = 0
            for r, fut in building:
                if self.pool is not None and not fut.done():
                    keep.append((r, fut))
                    continue
                case = fut.result() if self.pool is not None else fut
                rec = self._admit(r, case, now, pending)
                if rec is None:
                    keep.append((r, case if self.pool is None else fut))
                    continue
                pending += self.pairs_per_particle * r["n"]
                running[rec.sid] = rec
                new.append(rec.sid)
            building = keep
            if not running and not new and building and all(
                    self.pool is None or f.done() for _, f in building):
                raise RuntimeError(f"request {building[0][0]['rid']} does not fit the server's budget")
            if new:
                bt.start(new)
            if running:
                t_a = clock()
                bt.step(self.chunk)
                busy += clock() - t_a
                chunks += 1
                self.chunks_done += 1
                now = clock()
                for sid, rec in list(running.items()):
                    rec.done += self.chunk
                    if rec.done >= rec.req["steps"]:
                        state = bt.download_state(sid) if keep_state else None
                        st = bt.stats(sid)
                        bt.remove(sid)
                        del running[sid]
                        results.append(Result(rid=rec.req["rid"], n=rec.req["n"], steps=rec.req["steps"],
                                              arrival=rec.req["arrival"], admitted=rec.admitted,
                                              finished=now, stats=st, state=state))
            elif pend and not building:
                wait = pend[0]["arrival"] - clock()
                if wait > 0 and idle_sleep > 0:
                    time.sleep(min(wait, 0.05))
            elif idle_sleep > 0:
                time.sleep(idle_sleep)
        lat = np.array([r.latency for r in results]) if results else np.zeros(1)
        work = float(sum(r.n * r.steps for r in results))
        span = max(r.finished for r in results) - min(r.arrival for r in results) if results else 0.0
        return {"results": sorted(results, key=lambda r: r.rid),
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(np.mean(lat)), "particle_steps": work,
                "particle_steps_per_s": work / span if span > 0 else 0.0, "span_s": span,
                "chunks": chunks, "busy_s": busy}
