"""Multi-rank plumbing on CPU (gloo, world size 2).

The time step does not shard across GPUs here: N GPUs run N independent
replicas, lined up by a barrier, timed as the maximum over ranks.  These
tests exercise that host logic without a GPU.
"""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from sparc2_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    m = rep.max(1.0 + rank)
    rate = rep.aggregate_rate(1000.0, 0.5 * (rank + 1))
    q.put((rank, m, rate))
    rep.close()


def test_max_over_ranks_and_whole_job_rate():
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
    assert [r[1] for r in res] == [2.0, 2.0]          # max over ranks
    assert [r[2] for r in res] == [2000.0, 2000.0]    # 2 ranks * 1000 / 1 s


def _failing_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from sparc2_b200.replicas import Replicas
    rep = Replicas("gloo", timeout_s=10)
    if rank == 1:
        raise SystemExit(3)        # leaves between steps, before the barrier
    try:
        rep.barrier()
        q.put((rank, "passed"))
    except Exception:
        q.put((rank, "error"))


def test_a_rank_that_leaves_ends_the_others_barrier_with_an_error():
    """Failure on the host: a rank exits between steps; the surviving rank's
    next collective ends with an error (peer gone or the short process-group
    timeout) instead of waiting for good."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    assert q.get(timeout=120) == (0, "error")
    for p in procs:
        p.join(timeout=60)
    assert procs[1].exitcode == 3
    assert procs[0].exitcode == 0


def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port"
