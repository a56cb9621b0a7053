"""The multi-rank plumbing of bench.py on CPU: two gloo ranks with different
step times agree on the slowest one, and the whole-job rate counts every
rank's replica against it (no GPU; 127.0.0.1 rendezvous)."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = [10.0, 12.5][rank]
        slowest = bench.max_over_ranks(ms, world, device="cpu")
        out[rank] = (slowest, bench.job_rate(1000, world, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_slowest_step():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0] == res[1]
    slowest, rate = res[0]
    assert slowest == 12.5
    assert abs(rate - 1000 * 2 / 12.5e-3) <= 1e-9 * rate


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.job_rate(500, 1, 2.0) == 500 / 2e-3
