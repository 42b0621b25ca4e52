"""The multi-GPU path of bench.py on CPU: two gloo ranks over 127.0.0.1.

With N GPUs each rank tracks its own bunch (independent replicas: the path
has no data exchange), and the whole-job number is the sum of all ranks'
macroparticle-steps over the slowest rank's time.  This checks that
reduction and the reference arm's rank handling with world size 2, without
a GPU.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r ran (r + 1) * 1000 macroparticle-steps in 0.5 + r seconds
        t, w = bench.over_ranks(dist, torch, 0.5 + rank, (rank + 1) * 1000, "cpu")
        dist.barrier()
        out.put((rank, t, w))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_over_ranks_max_time_sum_work():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(world))
    for _, t, w in res:
        assert t == 1.5  # the slowest rank's time
        assert w == 3000.0  # every rank's work


def test_over_ranks_single_process_passthrough():
    import bench
    assert bench.over_ranks(None, torch, 2.0, 7, "cpu") == (2.0, 7)


def test_reference_arm_other_ranks_do_no_work(capsys):
    """Under torchrun only rank 0 runs and prints the reference arm."""
    import argparse
    import bench
    bench.run_reference(argparse.Namespace(gpus=2, steps=1, warmup=3), rank=1)
    assert capsys.readouterr().out == ""
