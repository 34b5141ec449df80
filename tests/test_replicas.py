"""bench.py's multi-process path on CPU: world_size-2 gloo ranks.

The path does not shard across GPUs (replicas only): every rank runs the
same workload on its own GPU and the job's time is the max over ranks.
Here the rank plumbing (rendezvous, max-over-ranks, barriers) runs as gloo
ranks without a GPU, and the reference arm under torchrun must print exactly
one JSON line (rank 0) while the other rank exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(None)
    m = bench.dist_max(float(10 * (r + 1)), w)
    bench.dist_barrier(w)
    dist.destroy_process_group()
    q.put((r, w, m))


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 2, 20.0), (1, 2, 20.0)]


def test_reference_arm_under_torchrun_prints_once():
    from oracle import ref_available
    if not ref_available("avx", 4):
        pytest.skip("reference not built")
    port = _free_port()
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                        "--master-port", str(port), "bench.py", "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "Gint/s" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
