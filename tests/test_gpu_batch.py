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
