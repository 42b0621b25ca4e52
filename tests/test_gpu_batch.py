"""CUDA-graph turns, concurrent batches of jobs, and the continuous-batching
server.

Tolerances: FP64 runs agree with the direct (un-batched, graph-free) runs to
1e-10 relative (only the deposit's atomic summation order differs); mixed
precision runs to 1e-6 relative (that order difference can flip an FP32
rounding of the spectrum).
"""
import numpy as np
import pytest

from helpers import MP, SIG_C0, elem, fodo_cell, gaussian_bunch, product_lattice, rel_l2

pytestmark = pytest.mark.gpu


def _job(syn, k1, n, shape, seed, precision, graphs):
    lat, ref = product_lattice(fodo_cell(k1))
    opts = syn.Space_charge_3d_open_hockney_options(*shape)
    opts.precision = precision
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 8))
    if graphs:
        prop.set_graphs(True)
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(gaussian_bunch(n, SIG_C0, seed))
    return prop, b


def test_graph_turns_match_direct(syn, monkeypatch):
    monkeypatch.setenv("SB2_CELL_SORT", "0")
    out = []
    for graphs in (False, True):
        prop, b = _job(syn, 0.6, 60000, (16, 16, 32), 81, syn.precision_t.fp64, graphs)
        prop.propagate(b, 4)
        out.append(b.get_particles())
        if graphs:
            captures, replays = prop.graph_stats()
            assert captures >= 1 and replays >= 2, (captures, replays)
    (a, am, _), (g, gm, _) = out
    assert np.array_equal(am, gm) and np.array_equal(a[:, 6], g[:, 6])
    for j in range(6):
        assert rel_l2(g[:, j], a[:, j]) <= 1e-10, j


def test_batch_jobs_match_alone(syn, monkeypatch):
    """Quad-strength scan: jobs with their own k1, grid and bunch size run
    concurrently give the same result as each run alone."""
    monkeypatch.setenv("SB2_CELL_SORT", "0")
    specs = [(0.45, 30000, (16, 16, 32), 1), (0.6, 80000, (32, 32, 64), 2), (0.75, 20000, (16, 16, 64), 3),
             (0.55, 50000, (16, 32, 32), 4)]
    alone = []
    for k1, n, shape, seed in specs:
        prop, b = _job(syn, k1, n, shape, seed, syn.precision_t.fp64, True)
        prop.propagate(b, 3)
        alone.append(b.get_particles()[0])
    batch = syn.Batch()
    keep = []
    for k1, n, shape, seed in specs:
        prop, b = _job(syn, k1, n, shape, seed, syn.precision_t.fp64, True)
        keep.append((prop, b, batch.add(prop, b)))
    batch.run({slot: 3 for _, _, slot in keep})
    for (prop, b, slot), ref_parts in zip(keep, alone):
        p = b.get_particles()[0]
        assert np.array_equal(p[:, 6], ref_parts[:, 6])
        for j in range(6):
            assert rel_l2(p[:, j], ref_parts[:, j]) <= 1e-10, (slot, j)


def _stream(syn, njobs=6):
    from synergia2_b200.serving import JobSpec
    rng = np.random.default_rng(5)
    jobs = []
    for i in range(njobs):
        k1 = float(rng.uniform(0.4, 0.8))
        lattice = fodo_cell(k1)
        n = int(rng.integers(20000, 60000))
        shape = [(16, 16, 32), (32, 32, 64)][i % 2]
        jobs.append(JobSpec(job_id=i, lattice=lattice, steps_per_turn=8, n=n, grid=shape,
                            turns=int(rng.integers(1, 5)), sigmas=tuple(SIG_C0), seed=100 + i,
                            arrival=0.002 * i))
    return jobs


def test_served_results_same_alone_and_in_mix(syn):
    """Each served job gives the same particles when it is the only job on
    the GPU and when it shares the device with the rest of the stream."""
    from synergia2_b200.serving import Server, summarize
    jobs = _stream(syn)
    alone, _ = Server(hbm_budget=8 << 30, max_active=1, keep_particles=True).run(jobs, realtime=False)
    srv = Server(hbm_budget=8 << 30, max_active=16, keep_particles=True)
    mixed_res, wall = srv.run(jobs, realtime=True)
    assert srv.max_inflight >= 2  # jobs overlapped on the device
    a = {r.job_id: r for r in alone}
    m = {r.job_id: r for r in mixed_res}
    assert set(a) == set(m) == {j.job_id for j in jobs}
    for jid in a:
        pa, pm = a[jid].particles, m[jid].particles
        assert np.array_equal(pa[:, 6], pm[:, 6])
        for j in range(6):
            assert rel_l2(pm[:, j], pa[:, j]) <= 1e-6, (jid, j)
        assert np.allclose(m[jid].emittance, a[jid].emittance, rtol=1e-6, atol=0)
    s = summarize(mixed_res, wall)
    assert s["latency_p50_s"] > 0 and s["latency_p99_s"] >= s["latency_p50_s"]


def test_admission_respects_memory_budget(syn):
    from synergia2_b200.serving import Server, footprint_bytes
    jobs = _stream(syn, 5)
    budget = max(footprint_bytes(j) for j in jobs) + 1024  # one job at a time
    srv = Server(hbm_budget=budget, max_active=16)
    peak = [0]
    orig = srv._admit

    def admit(spec, now):
        orig(spec, now)
        peak[0] = max(peak[0], srv.used)
        assert len(srv.active) == 1
    srv._admit = admit
    res, _ = srv.run(jobs, realtime=False)
    assert len(res) == len(jobs) and peak[0] <= budget


def test_batch_launch_query_matches_run(syn, monkeypatch):
    """The asynchronous form (launch, then poll) gives the same particles as
    the blocking batch run, and a slot refuses a second launch while its
    turns are in flight."""
    monkeypatch.setenv("SB2_CELL_SORT", "0")
    specs = [(0.5, 40000, (16, 16, 32), 11), (0.7, 70000, (32, 32, 64), 12)]
    ref = []
    b0 = syn.Batch()
    keep0 = []
    for k1, n, shape, seed in specs:
        prop, b = _job(syn, k1, n, shape, seed, syn.precision_t.fp64, True)
        keep0.append((prop, b, b0.add(prop, b)))
    b0.run({slot: 2 for _, _, slot in keep0})
    ref = [b.get_particles()[0] for _, b, _ in keep0]
    batch = syn.Batch()
    keep = []
    for k1, n, shape, seed in specs:
        prop, b = _job(syn, k1, n, shape, seed, syn.precision_t.fp64, True)
        keep.append((prop, b, batch.add(prop, b)))
    for _, _, slot in keep:
        batch.launch(slot, 2)
    with pytest.raises(syn.SB2Error, match="in flight"):
        batch.launch(keep[0][2], 1)
    pending = {slot for _, _, slot in keep}
    while pending:
        pending = {s for s in pending if not batch.query(s)}
    for (prop, b, slot), r in zip(keep, ref):
        p = b.get_particles()[0]
        assert np.array_equal(p[:, 6], r[:, 6])
        for j in range(6):
            assert rel_l2(p[:, j], r[:, j]) <= 1e-10, (slot, j)


def _lockstep_specs():
    # quad-strength scan: own k1, bunch size and grid per job (two grid shapes)
    return [(0.45, 30000, (16, 16, 32), 11), (0.6, 80000, (32, 32, 64), 12), (0.75, 20000, (16, 16, 32), 13),
            (0.55, 50000, (32, 32, 64), 14), (0.7, 5000, (16, 16, 32), 15)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_lockstep_batch_matches_alone(syn, precision, tol):
    """Jobs advanced in lockstep (one work-list launch per kernel kind and
    grid shape per step for all of them) give each job's result alone: ids
    and masks exact; coordinates within the deposit-order tolerance (FP64
    1e-10; mixed precision 1e-6, an FP32 rounding of the charge grid or the
    spectrum can flip)."""
    prec = getattr(syn.precision_t, precision)
    specs = _lockstep_specs()
    alone = []
    for k1, n, shape, seed in specs:
        prop, b = _job(syn, k1, n, shape, seed, prec, False)
        prop.propagate(b, 3)
        alone.append(b.get_particles())
    batch = syn.Batch()
    keep = []
    for k1, n, shape, seed in specs:
        prop, b = _job(syn, k1, n, shape, seed, prec, False)
        keep.append((prop, b, batch.add(prop, b)))
    batch.run_lockstep([slot for _, _, slot in keep], 2)
    batch.run_lockstep([slot for _, _, slot in keep], 1)  # a second call continues from the first
    for (prop, b, slot), (ap, am, _) in zip(keep, alone):
        p, m, _ = b.get_particles()
        assert np.array_equal(p[:, 6], ap[:, 6]) and np.array_equal(m, am)
        for j in range(6):
            assert rel_l2(p[:, j], ap[:, j]) <= tol, (slot, j)
        assert b.get_total_num() == int(am.sum())


def test_lockstep_batch_ring_losses_exact(syn):
    """Ring cells with apertures in lockstep: lost sets, discards, counts and
    real numbers equal the jobs run alone."""
    from helpers import ring_cell
    out = []
    for lockstep in (False, True):
        batch = syn.Batch()
        keep = []
        for i, (n, shape) in enumerate(((40000, (16, 16, 32)), (25000, (16, 16, 32)), (60000, (32, 32, 64)))):
            lat, ref = product_lattice(ring_cell(radius=0.004 + 0.001 * i))
            prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(*shape), 16))
            b = syn.Bunch(ref, n, 1e11)
            b.set_particles(gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 20 + i))
            if lockstep:
                keep.append((prop, b, batch.add(prop, b)))
            else:
                prop.propagate(b, 2)
                keep.append((prop, b, None))
        if lockstep:
            batch.run_lockstep([slot for _, _, slot in keep], 2)
        out.append([(b.get_particles(), b.counts()) for _, b, _ in keep])
    for ((ap, am, ad), ac), ((lp, lm, ld), lc) in zip(out[0], out[1]):
        assert np.array_equal(am, lm) and np.array_equal(ad, ld) and 0 < int(am.sum()) < len(am)
        assert ac == lc
        alive = am.astype(bool)
        for j in range(6):
            assert rel_l2(lp[alive, j], ap[alive, j]) <= 1e-10, j


def test_lockstep_rejects_jobs_out_of_step(syn):
    """Jobs whose turns have different step counts cannot share launches."""
    batch = syn.Batch()
    a = _job(syn, 0.6, 10000, (16, 16, 32), 1, syn.precision_t.fp64, False)
    lat, ref = product_lattice(fodo_cell(0.6))
    p2 = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 4))
    b2 = syn.Bunch(ref, 10000, 1e11)
    b2.set_particles(gaussian_bunch(10000, SIG_C0, 2))
    s1, s2 = batch.add(*a), batch.add(p2, b2)
    with pytest.raises(syn.SB2Error, match="lockstep"):
        batch.run_lockstep([s1, s2], 1)


def test_lockstep_rejects_shared_propagator_or_bunch(syn):
    """The list launches advance all jobs at once, so two jobs of one
    lockstep call cannot share a propagator (its grids and sort scratch) or
    a bunch."""
    p1, b1 = _job(syn, 0.6, 10000, (16, 16, 32), 1, syn.precision_t.fp64, False)
    p2, b2 = _job(syn, 0.7, 10000, (16, 16, 32), 2, syn.precision_t.fp64, False)
    for pair in (((p1, b1), (p1, b2)), ((p1, b1), (p2, b1))):
        batch = syn.Batch()
        s1, s2 = batch.add(*pair[0]), batch.add(*pair[1])
        with pytest.raises(syn.SB2Error, match="own propagator and bunch"):
            batch.run_lockstep([s1, s2], 1)


def test_graph_turns_inside_propagate_steps(syn):
    """propagate_steps with CUDA-graph turns (the working copy cell-sorted):
    the steps that fall in one turn are one graph (the partial turns at either
    end and the whole turns between), and the result equals the same steps
    without graphs (ids and masks exact, coordinates to the deposit-order
    tolerance 1e-10).  prepare_steps captures those graphs ahead and leaves the
    bunch as it was, so the call itself only replays."""
    n = 60000
    p = gaussian_bunch(n, SIG_C0, 83)
    lat, ref = product_lattice(fodo_cell())
    out = []
    for graphs in (False, True):
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 8))
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.propagate_steps(b, 0, 5)
        if graphs:
            prop.set_graphs(True)
            before = b.get_particles()
            state = bytes(b.get_state())
            prop.prepare_steps(b, 5, 21)
            for x, y in zip(before, b.get_particles()):
                assert np.array_equal(x, y)
            assert bytes(b.get_state()) == state
            c0, r0 = prop.graph_stats()
            assert c0 >= 3 and r0 == 0  # steps 5-7, a whole turn, steps 24-25
        prop.propagate_steps(b, 5, 21)  # graphs: steps 5-7, turns 8-15 and 16-23, steps 24-25
        if graphs:
            assert prop.graph_stats() == (c0, r0 + 4)
        out.append((b.get_particles(), b.counts()))
    ((a, am, ad), ac), ((g, gm, gd), gc) = out
    assert np.array_equal(am, gm) and np.array_equal(ad, gd) and np.array_equal(a[:, 6], g[:, 6]) and ac == gc
    for j in range(6):
        assert rel_l2(g[:, j], a[:, j]) <= 1e-10, j


def test_prepare_steps_with_diagnostics_from_the_first_call(syn):
    """prepare_steps on a bunch never propagated, with per-turn diagnostics
    on: the first propagate_steps call (which also records the initial state)
    only replays, and its particles and diagnostics equal the same call
    without graphs."""
    n = 40000
    p = gaussian_bunch(n, SIG_C0, 84)
    lat, ref = product_lattice(fodo_cell())
    out = []
    for graphs in (False, True):
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 8))
        prop.set_diagnostics(8)
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        if graphs:
            prop.set_graphs(True)
            prop.prepare_steps(b, 0, 19)
            c0, r0 = prop.graph_stats()
        prop.propagate_steps(b, 0, 19)  # graphs: two whole turns, then steps 16-18
        if graphs:
            assert prop.graph_stats() == (c0, r0 + 3)
        out.append((b.get_particles()[0], prop.diagnostics()))
    (a, da), (g, dg) = out
    assert np.array_equal(a[:, 6], g[:, 6])
    for j in range(6):
        assert rel_l2(g[:, j], a[:, j]) <= 1e-10, j
    assert list(da["s"]) == list(dg["s"]) and len(da["s"]) == 3  # the initial state and two turn ends
    for key in ("mean", "std"):
        assert np.allclose(np.asarray(dg[key]), np.asarray(da[key]), rtol=1e-8, atol=1e-13), key
