"""World-size-2 gloo test of bench.py's multi-rank host logic (on CPU).

On N GPUs each rank solves its own spin/k-point problem; the only collectives
are the max-over-ranks device time and the sum of CG iterations.  Both are
exercised here with the gloo backend, without a GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    t, it = bench.combine_ranks(100.0 + 50.0 * rank, 30 + rank, world, device="cpu")
    q.put((rank, t, it))
    dist.destroy_process_group()


def test_combine_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, it in res:
        assert t == 150.0 and it == 61.0


def test_combine_ranks_single():
    import bench

    assert bench.combine_ranks(12.5, 7, 1) == (12.5, 7.0)


def test_bench_spawns_its_own_ranks():
    """`bench.py --gpus 2` without torchrun starts one process per rank itself (RANK,
    LOCAL_RANK, WORLD_SIZE, MASTER_* set); the reference arm then runs on rank 0 alone and
    reports n_gpus = 2.  The CPU arm needs no GPU, so this runs here."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--workload", "dense_832", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout  # rank 0 alone prints
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2
