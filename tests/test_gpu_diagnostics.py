"""Per-turn bunch diagnostics on the device (Diagnostics_full2::do_update,
bunch/diagnostics_full2.cc:16-37; calculate_emittances,
diagnostics_full2_host.cc).

The records are checked against numpy on the particles read back at the
same points (initial state, end of the run): mean, second moments, min/max
and emittances to 1e-10 relative (only summation order differs).  Turning
diagnostics on splits the fused particle pass at turn ends and must not
change the particles; CUDA-graph turns give the same records.
"""
import numpy as np
import pytest

from helpers import SIG_C0, fodo_cell, gaussian_bunch, product_lattice, rel_l2

pytestmark = pytest.mark.gpu


def _numpy_record(p, m, total):
    live = p[m.astype(bool), :6]
    mean = live.sum(0) / total
    d = live - mean
    mom2 = d.T @ d / total
    emit = [np.sqrt(max(np.linalg.det(mom2[2 * k:2 * k + 2, 2 * k:2 * k + 2]), 0.0)) for k in range(3)]
    return mean, mom2, emit, live[:, [0, 2, 4]].min(0), live[:, [0, 2, 4]].max(0), np.sqrt(np.linalg.det(mom2[:4, :4]))


def _run(syn, graphs, diag, p, turns=3, shape=(16, 16, 32)):
    lat, ref = product_lattice(fodo_cell())
    prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(*shape), 8))
    if graphs:
        prop.set_graphs(True)
    if diag:
        prop.set_diagnostics(16)
    b = syn.Bunch(ref, p.shape[0], 1e11)
    b.set_particles(p)
    prop.propagate(b, turns)
    return prop, b


@pytest.mark.parametrize("graphs", [False, True])
def test_diagnostics_records_match_numpy(syn, graphs):
    n = 60000
    p = gaussian_bunch(n, SIG_C0, 91)
    prop, b = _run(syn, graphs, True, p)
    d = prop.diagnostics()
    assert len(d["num_particles"]) == 4  # initial + 3 turns
    assert list(d["turns"]) == [0, 1, 2, 3]
    assert np.allclose(d["s"], [0.0, 10.0, 20.0, 30.0])
    checks = [(0, p, np.ones(n, np.uint8))]
    gp, gm, _ = b.get_particles()
    checks.append((3, gp, gm))
    for k, parts, masks in checks:
        mean, mom2, emit, mn, mx, exy = _numpy_record(parts, masks, int(d["num_particles"][k]))
        assert d["num_particles"][k] == masks.sum()
        sd = np.sqrt(np.diag(mom2))
        # summation order differs: relative 1e-10, plus 1e-12 of the spread
        # for entries near zero (means, uncorrelated cross moments)
        assert np.all(np.abs(d["mean"][k] - mean) <= 1e-10 * np.abs(mean) + 1e-12 * sd)
        assert np.all(np.abs(d["mom2"][k] - mom2) <= 1e-10 * np.abs(mom2) + 1e-12 * np.outer(sd, sd))
        assert np.array_equal(d["min"][k], mn) and np.array_equal(d["max"][k], mx)
        assert np.allclose([d["emitx"][k], d["emity"][k], d["emitz"][k]], emit, rtol=1e-9)
        assert abs(d["emitxy"][k] / exy - 1) < 1e-8
        assert np.allclose(d["std"][k], np.sqrt(np.diag(mom2)), rtol=1e-10)
        assert np.allclose(np.diag(d["corr"][k]), 1.0, rtol=1e-12)


def test_diagnostics_do_not_change_tracking(syn):
    p = gaussian_bunch(40000, SIG_C0, 92)
    _, b0 = _run(syn, False, False, p)
    _, b1 = _run(syn, False, True, p)
    a, _, _ = b0.get_particles()
    c, _, _ = b1.get_particles()
    assert np.array_equal(a[:, 6], c[:, 6])
    for j in range(6):
        assert rel_l2(c[:, j], a[:, j]) <= 1e-10, j


def test_diagnostics_graphs_match_direct(syn, monkeypatch):
    monkeypatch.setenv("SB2_CELL_SORT", "0")
    p = gaussian_bunch(40000, SIG_C0, 93)
    pd, _ = _run(syn, False, True, p)
    pg, _ = _run(syn, True, True, p)
    a, g = pd.diagnostics(), pg.diagnostics()
    assert np.array_equal(a["turns"], g["turns"])
    for key in ("emitx", "emity", "emitz"):
        assert np.allclose(a[key], g[key], rtol=1e-10, atol=0), key
    sd = a["std"]
    assert np.all(np.abs(a["mean"] - g["mean"]) <= 1e-10 * np.abs(a["mean"]) + 1e-12 * sd)


def test_loss_records_cover_every_lost_particle(syn):
    """Diagnostics_loss (bunch.h:727-740): every particle an aperture
    discards is recorded once, with its coordinates at the aperture (the
    coordinates it keeps afterwards, lost particles being frozen), and with
    the repetition and path length of the bunch reference there."""
    from helpers import ring_cell
    n = 30000
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 94)
    lat, ref = product_lattice(ring_cell(radius=0.004))
    prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 16))
    prop.set_loss_diagnostics(n)
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 2)
    gp, gm, gd = b.get_particles()
    rec = prop.losses()
    lost = np.where(gm == 0)[0]
    assert 0 < len(lost) < n
    ids = rec[:, 6].astype(np.int64)
    assert np.array_equal(np.sort(ids), lost)
    assert np.array_equal(rec[:, :6], gp[ids, :6])
    assert set(np.unique(rec[:, 7])) <= {0.0, 1.0}
    assert np.all((rec[:, 8] >= 0) & (rec[:, 8] <= 16.0 + 1e-9)) and np.all(rec[:, 9] <= 8.0 + 1e-9)
    with pytest.raises(syn.SB2Error, match="CUDA-graph"):
        prop.set_graphs(True)


def test_gpu_step_counts_match_per_step_calls(syn):
    """Per-step count records (reg_diag_per_step): the counts after every
    step of one fused propagate call equal the counts read after each of
    the same steps run one call at a time (ring cell with losses)."""
    from helpers import gaussian_bunch, product_lattice, ring_cell
    n = 20000
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 41)
    lat, ref = product_lattice(ring_cell(radius=0.004))
    a = syn.Propagator(lat, syn.Split_operator_stepper(None, 16))
    b = syn.Propagator(lat, syn.Split_operator_stepper(None, 16))
    ns = a.num_steps()
    ba, bb = syn.Bunch(ref, n, 1e11), syn.Bunch(ref, n, 1e11)
    ba.set_particles(p)
    bb.set_particles(p)
    a.set_step_counts(4 * ns)
    a.propagate(ba, 2)
    recs = a.step_counts()
    assert len(recs) == 2 * ns
    seen = []
    for k in range(2 * ns):
        b.propagate_steps(bb, k, 1)
        c = bb.counts()
        seen.append((c["local_num"], c["total_num"], c["real_num"]))
    assert recs == seen
    assert recs[-1][0] < n  # particles were lost along the way
    assert np.array_equal(ba.get_particles()[1], bb.get_particles()[1])


def test_gpu_step_counts_with_space_charge_and_graph_refusal(syn):
    """One record per step with space charge; records continue across calls;
    CUDA-graph turns refuse records into a pageable host buffer (the records
    then come by copies that a graph would replay to the same addresses)."""
    from helpers import SIG_C0, fodo_cell, gaussian_bunch, product_lattice
    n = 20000
    lat, ref = product_lattice(fodo_cell())
    prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 8))
    bunch = syn.Bunch(ref, n, 1e11)
    bunch.set_particles(gaussian_bunch(n, SIG_C0, 42))
    prop.set_step_counts(20)
    prop.propagate_steps(bunch, 0, 5)
    prop.propagate_steps(bunch, 5, 7)
    recs = prop.step_counts()
    assert len(recs) == 12 and all(r == (n, n, 1e11) for r in recs)
    prop.set_step_counts(0)
    import ctypes
    pageable = np.zeros(4 * ctypes.sizeof(syn._lib.sb2_step_counts), np.uint8)
    L = syn.lib()
    syn.check(L.sb2_propagator_set_step_counts(prop.h, ctypes.c_void_p(pageable.ctypes.data), 4))
    with pytest.raises(syn.SB2Error, match="pageable"):
        prop.set_graphs(True)
    syn.check(L.sb2_propagator_set_step_counts(prop.h, None, 0))
    prop.set_graphs(True)
    with pytest.raises(syn.SB2Error, match="pageable"):
        syn.check(L.sb2_propagator_set_step_counts(prop.h, ctypes.c_void_p(pageable.ctypes.data), 4))


def test_gpu_step_counts_with_graph_turns(syn):
    """Per-step records into pinned memory with CUDA-graph turns (ring cell
    with losses, space charge): the records equal the same steps launched
    directly, the turns replay graphs (the records go to a device-side
    cursor, so turns stay alike), and the bunches agree."""
    from helpers import gaussian_bunch, product_lattice, ring_cell
    n = 30000
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 43)
    lat, ref = product_lattice(ring_cell(radius=0.004))
    out = []
    for graphs in (False, True):
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32),
                                                               16))
        ns = prop.num_steps()
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.set_step_counts(4 * ns)
        if graphs:
            prop.set_graphs(True)
        prop.propagate_steps(b, 0, 3 * ns + 5)
        if graphs:
            captures, replays = prop.graph_stats()
            assert replays >= 1 and captures <= 3, (captures, replays)
        out.append((prop.step_counts(), b.get_particles()))
    (ra, (pa, ma, _)), (rg, (pg, mg, _)) = out
    assert len(ra) == len(rg) == 3 * ns + 5 and ra == rg
    assert ra[-1][0] < n  # particles were lost along the way
    assert np.array_equal(ma, mg) and np.array_equal(pa[:, 6], pg[:, 6])


def test_gpu_fp64_peak_probe(syn):
    """The FP64 FMA probe behind the particle passes' FP64 roofline returns
    a plausible rate for a B200 (tens of TFLOP/s)."""
    import ctypes
    v = ctypes.c_double()
    syn.check(syn.lib().sb2_fp64_peak_probe(ctypes.byref(v), None))
    assert 5.0 < v.value < 200.0, v.value
