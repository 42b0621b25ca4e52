"""One bunch split over two processes by particle range (the reference's
MPI bunch decomposition): the ranks exchange moment sums, valid counts and
the charge density through a sum-allreduce (sb2_propagator_set_allreduce).

CPU: the shard ranges and a two-rank gloo sum through the host-staged
callback types (untyped double, typed double and float).  GPU: two
processes (gloo, host-staged exchanges; both on the one GPU: their kernels
never wait on each other, the ranks meet on the host) against the whole
bunch in one process -- coordinates within 1e-10 relative (the deposit's
summation order differs; 1e-6 in mixed precision, whose FP32 charge grid is
exchanged as float), ids, masks, discards and the bunch's total and real
numbers exact.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import ROOT, SIG_C0, fodo_cell, gaussian_bunch, product_lattice, rel_l2, ring_cell


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges_cover_the_bunch():
    from synergia2_b200.sharding import shard_range
    for n, w in ((10, 3), (7, 7), (100, 1), (5, 8)):
        rs = [shard_range(n, r, w) for r in range(w)]
        assert rs[0][0] == 0 and rs[-1][1] == n
        assert all(rs[k][1] == rs[k + 1][0] for k in range(w - 1))
        assert max(h - l for l, h in rs) - min(h - l for l, h in rs) <= 1


def _cpu_rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import ctypes
        from synergia2_b200 import _lib
        arr = np.full(5, rank + 1.0)

        def fn(a):
            dist.all_reduce(torch.from_numpy(a), op=dist.ReduceOp.SUM)

        def cb(ctx, data, count, host):
            fn(np.ctypeslib.as_array(data, shape=(int(count),)))
            return 0
        c = _lib.ALLREDUCE_FN(cb)
        rc = c(None, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 5, 1)
        # the typed callback type: a float32 and a float64 buffer
        seen = []

        def tcb(ctx, data, count, dtype, host):
            dt = np.dtype(np.float32 if dtype == 1 else np.float64)
            seen.append(dt.name)
            fn(np.frombuffer((ctypes.c_char * (int(count) * dt.itemsize)).from_address(data), dtype=dt))
            return 0
        t = _lib.ALLREDUCE_TYPED_FN(tcb)
        a32 = np.full(3, rank + 0.5, dtype=np.float32)
        a64 = np.full(4, rank + 0.25)
        rc32 = t(None, a32.ctypes.data, 3, 1, 1)
        rc64 = t(None, a64.ctypes.data, 4, 0, 1)
        q.put((rank, rc + rc32 + rc64, arr.tolist(), a32.tolist(), a64.tolist(), seen))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_allreduce_callback_sums_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_cpu_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(90)
    assert all(p.exitcode == 0 for p in ps)
    for _ in range(2):
        _, rc, vals, v32, v64, seen = q.get(timeout=5)
        assert rc == 0 and vals == [3.0] * 5
        assert v32 == [2.0] * 3 and v64 == [1.5] * 4 and seen == ["float32", "float64"]


def _spec(case):
    if case.startswith("fodo"):
        return fodo_cell(), 8, SIG_C0
    return ring_cell(radius=0.004), 16, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4]


def _sc_opts(syn, case):
    opts = syn.Space_charge_3d_open_hockney_options(16, 16, 32)
    if case.endswith("mixed"):
        opts.precision = syn.precision_t.mixed
    return opts


def _gpu_rank(rank, world, port, case, n, q):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import synergia2_b200 as syn
        from synergia2_b200.sharding import attach, shard_range
        spec, steps, sig = _spec(case)
        p = gaussian_bunch(n, sig, 95)
        lo, hi = shard_range(n, rank, world)
        lat, ref = product_lattice(spec)
        prop = syn.Propagator(lat, syn.Split_operator_stepper(_sc_opts(syn, case), steps))
        dtypes = set()
        orig = dist.all_reduce

        def seen(t, *a, **k):
            dtypes.add(str(t.dtype))
            return orig(t, *a, **k)
        dist.all_reduce = seen
        attach(prop)
        b = syn.Bunch(ref, hi - lo, 1e11)  # real_num of the whole bunch on every shard
        b.set_particles(np.asfortranarray(p[lo:hi]))
        prop.propagate(b, 2)
        gp, gm, gd = b.get_particles()
        q.put((rank, gp, gm, gd, b.get_total_num(), b.get_real_num(), sorted(dtypes)))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.timeout(300)
@pytest.mark.parametrize("case", ["fodo", "ring", "fodo_mixed", "ring_mixed"])
def test_sharded_bunch_matches_whole_bunch(syn, case):
    n = 60000
    spec, steps, sig = _spec(case)
    p = gaussian_bunch(n, sig, 95)
    lat, ref = product_lattice(spec)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(_sc_opts(syn, case), steps))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 2)
    wp, wm, wd = b.get_particles()

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_gpu_rank, args=(r, 2, port, case, n, q)) for r in range(2)]
    for pr in ps:
        pr.start()
    res = sorted(q.get(timeout=240) for _ in range(2))
    for pr in ps:
        pr.join(60)
    assert all(pr.exitcode == 0 for pr in ps)
    sp = np.concatenate([r[1] for r in res])
    sm = np.concatenate([r[2] for r in res])
    sd = np.concatenate([r[3] for r in res])
    assert np.array_equal(sp[:, 6], wp[:, 6]) and np.array_equal(sm, wm) and np.array_equal(sd, wd)
    if case.startswith("ring"):
        assert 0 < int(wm.sum()) < n  # losses happened
    mixed = case.endswith("mixed")
    for r in res:
        assert r[4] == b.get_total_num()
        assert r[5] == b.get_real_num()
        # the charge grid crosses as float32 in mixed precision only
        assert r[6] == (["torch.float32", "torch.float64"] if mixed else ["torch.float64"])
    for j in range(6):
        assert rel_l2(sp[:, j], wp[:, j]) <= (1e-6 if mixed else 1e-10), j


def _nccl_rank(port, n, case, q):
    """World size 1 over NCCL: the device-buffer exchange (the library's
    stream handed to the collective) runs for real on the one GPU."""
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    torch.cuda.set_device(0)
    import datetime
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        import synergia2_b200 as syn
        from synergia2_b200.sharding import attach
        calls = [0]
        dtypes = set()
        orig = dist.all_reduce

        def counted(t, *a, **k):
            calls[0] += 1
            dtypes.add(str(t.dtype))
            return orig(t, *a, **k)
        dist.all_reduce = counted
        spec, steps, sig = _spec(case)
        p = gaussian_bunch(n, sig, 96)
        lat, ref = product_lattice(spec)
        prop = syn.Propagator(lat, syn.Split_operator_stepper(_sc_opts(syn, case), steps))
        attach(prop)
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.propagate(b, 2)
        gp, gm, gd = b.get_particles()
        q.put((dist.get_backend(), calls[0], gp, gm, gd, b.get_total_num(), b.get_real_num(), sorted(dtypes)))
        del prop
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.timeout(300)
@pytest.mark.parametrize("case", ["ring", "ring_mixed"])
def test_nccl_device_exchange_world_one_matches_whole_bunch(syn, case):
    """The NCCL branch of sharding.attach (device buffers, the collective
    ordered on the library's stream, no host synchronisation) at world size
    1 against the same bunch without an exchange: ring cell with losses, two
    turns; ids, masks, discards, total and real numbers exact, coordinates
    within 1e-10 (the deposit's summation order; 1e-6 in mixed precision,
    where the FP32 charge grid goes through NCCL as float32)."""
    n = 40000
    spec, steps, sig = _spec(case)
    p = gaussian_bunch(n, sig, 96)
    lat, ref = product_lattice(spec)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(_sc_opts(syn, case), steps))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 2)
    wp, wm, wd = b.get_particles()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pr = ctx.Process(target=_nccl_rank, args=(_free_port(), n, case, q))
    pr.start()
    backend, calls, gp, gm, gd, total, real, dtypes = q.get(timeout=240)
    pr.join(60)
    assert pr.exitcode == 0
    assert backend == "nccl" and calls > 0
    mixed = case.endswith("mixed")
    assert dtypes == (["torch.float32", "torch.float64"] if mixed else ["torch.float64"])
    assert np.array_equal(gp[:, 6], wp[:, 6]) and np.array_equal(gm, wm) and np.array_equal(gd, wd)
    assert 0 < int(wm.sum()) < n
    assert total == b.get_total_num() and real == b.get_real_num()
    for j in range(6):
        assert rel_l2(gp[:, j], wp[:, j]) <= (1e-6 if mixed else 1e-10), j


@pytest.mark.gpu
def test_device_exchange_failure_is_reported(syn):
    """A device-buffer exchange whose collective fails makes the propagate
    call return the library's error, not a silent result."""
    n = 5000
    p = gaussian_bunch(n, SIG_C0, 97)
    lat, ref = product_lattice(fodo_cell())
    prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 8))

    def broken(ptr, count):
        raise RuntimeError("collective failed")
    prop.set_allreduce(broken, on_host=False)
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    with pytest.raises(syn.SB2Error, match="allreduce callback failed"):
        prop.propagate(b, 1)
