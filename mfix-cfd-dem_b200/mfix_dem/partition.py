"""Independent DEM systems spread over GPUs: one batch handle (or server) per
rank, systems assigned by a greedy size balance, no data-path collective.

The systems of a batch (and the requests of a served stream) do not
interact, so each rank steps its own share; only the metrics are gathered at
the end (times, particle-steps, latencies).  The assignment is a pure
function of the work list, so every rank computes the same partition
without communicating.

    part = partition_work(work, n_ranks)     # list of index lists, one per rank
    mine = part[rank]
    ...
    totals = gather_metrics({"ms": t, "particle_steps": ps}, world_size)
"""
from __future__ import annotations

import heapq
from typing import Dict, List, Sequence


def partition_work(work: Sequence[float], n_ranks: int) -> List[List[int]]:
    """Longest-processing-time-first greedy balance: items in decreasing
    `work` (ties by index) go to the rank with the least work so far (ties
    by rank).  Returns each rank's item indices in ascending order.  The
    largest load is at most 4/3 of the optimum (Graham's bound)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be positive")
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    out: List[List[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    return [sorted(x) for x in out]


def loads(work: Sequence[float], part: List[List[int]]) -> List[float]:
    """Total work of each rank's share."""
    return [float(sum(work[i] for i in p)) for p in part]


def partition_requests(requests: Sequence[dict], n_ranks: int) -> List[List[dict]]:
    """A served stream split over ranks in arrival order: each request goes
    to the rank whose assigned particle-steps are the least so far (ties by
    rank), so the shares stay balanced while the stream is open (a
    request's rank is fixed when it arrives, from the earlier arrivals
    only)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be positive")
    heap = [(0.0, r) for r in range(n_ranks)]
    out: List[List[dict]] = [[] for _ in range(n_ranks)]
    for req in sorted(requests, key=lambda r: (r["arrival"], r["rid"])):
        load, r = heapq.heappop(heap)
        out[r].append(req)
        heapq.heappush(heap, (load + float(req["n"]) * float(req["steps"]), r))
    return out


def gather_metrics(local: Dict[str, float], world_size: int, device="cpu") -> Dict[str, List[float]]:
    """Every rank's values of `local` (same keys on every rank), gathered to
    all ranks with one all_gather of a float64 vector (torch.distributed;
    a single rank returns its own)."""
    keys = sorted(local)
    if world_size <= 1:
        return {k: [float(local[k])] for k in keys}
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local[k]) for k in keys], dtype=torch.float64, device=device)
    bufs = [torch.empty_like(t) for _ in range(world_size)]
    dist.all_gather(bufs, t)
    return {k: [float(b[j].item()) for b in bufs] for j, k in enumerate(keys)}


def gather_list(values: Sequence[float], world_size: int, device="cpu") -> List[float]:
    """Concatenation over ranks of a per-rank list of floats of any length
    (two collectives: the lengths, then the padded values)."""
    if world_size <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    n = torch.tensor([len(values)], dtype=torch.int64, device=device)
    ns = [torch.empty_like(n) for _ in range(world_size)]
    dist.all_gather(ns, n)
    m = max(int(x.item()) for x in ns)
    t = torch.zeros(max(m, 1), dtype=torch.float64, device=device)
    if len(values):
        t[: len(values)] = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    bufs = [torch.empty_like(t) for _ in range(world_size)]
    dist.all_gather(bufs, t)
    out: List[float] = []
    for b, k in zip(bufs, ns):
        out.extend(float(x) for x in b[: int(k.item())].tolist())
    return out
