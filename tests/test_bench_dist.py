"""bench.py's multi-rank plumbing on CPU: two gloo ranks (the GPU runs use one
process per GPU over NCCL with the same code).  Replicas only: the group
carries the barrier and the maximum of the per-rank timings, and the
reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    r, w = bench.setup_dist(ws, backend="gloo")
    bench.barrier()
    t = bench.max_over_ranks(1.0 + rank)       # rank 1 is the slower one
    rate = bench.whole_job_rate(1000.0, w, t)  # 1000 units per rank
    bench.barrier()
    bench._dist.destroy_process_group()
    q.put((r, w, t, rate))


def test_two_gloo_ranks_max_timing_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for r, (rank, ws, t, rate) in enumerate(out):
        assert (rank, ws) == (r, 2)
        assert t == 2.0                 # max over ranks, identical on both
        assert rate == 1000.0 * 2 / 2.0


def _ref_worker(rank, ws, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    class A:  # the reference arm must not run (or print) on rank 1
        steps = 1
        warmup = 0

    if rank == 1:
        q.put(bench.run_reference_arm(A, 1, ws))
    else:
        q.put(0)


def test_reference_arm_is_rank0_only():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_worker, args=(1, 2, _free_port(), q))
    p.start()
    p.join(60)
    assert p.exitcode == 0 and q.get(timeout=5) == 0
