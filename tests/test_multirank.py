"""The N > 1 path of bench.py on CPU ranks (gloo): every rank solves its own
replica (replicas only, no data-path collective), the timing is the max over
ranks and rank 0 alone prints the JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    class A:
        pass
    r, w, local = bench.dist_setup(A())
    bench.barrier(w)
    m = bench.max_over_ranks(float(10 + r), w)
    q.put((r, w, m))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 11.0), (1, 2, 11.0)]


def test_reference_arm_two_ranks():
    """`bench.py --impl reference` under torchrun with two ranks: rank 0
    times the CPU path and prints one line, rank 1 exits without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=2", "--master-addr=127.0.0.1",
           f"--master-port={free_port()}", "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--config", "cfg0"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port"
