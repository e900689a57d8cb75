"""The multi-process paths of bench.py on CPU: two gloo ranks agree on the
slowest rank's time, and the reference arm under torchrun with two ranks
prints one line from rank 0 while rank 1 exits without work."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _rank_main(rank, port, out):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        out[rank] = bench.max_over_ranks(1.5 + rank, 2, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    import torch.multiprocessing as mp
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(port, out), nprocs=2, join=True)
        assert out[0] == out[1] == 2.5


def test_reference_arm_two_ranks(tmp_path):
    port = 30500 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "3", "--warmup", "1", "--cpu-sample", "60000"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
