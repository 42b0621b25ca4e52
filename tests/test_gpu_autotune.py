"""The project's autotuner over the particle-pass launch shapes, the
re-sort interval, the FFT radix plan and the deposit tile chunk
(sb2_propagator_autotune): it leaves the bunch and the propagator's records
untouched, applies the fastest configuration, and every configuration
computes the same results."""
import numpy as np
import pytest

from helpers import SIG_C0, fodo_cell, gaussian_bunch, product_lattice, rel_l2, ring_cell

pytestmark = pytest.mark.gpu

CONFIGS = [dict(light_shape=1, full_occ=2, full_ppt=1, quad_variant=1, ctas_per_sm=8),
           dict(light_shape=2, full_occ=2, full_ppt=2, quad_variant=0, ctas_per_sm=4),
           dict(light_shape=0, full_occ=3, full_ppt=1, quad_variant=1, ctas_per_sm=12),
           dict(light_shape=3, full_occ=2, full_ppt=1, quad_variant=1, ctas_per_sm=4)]


def test_gpu_launch_shapes_give_identical_tracks(syn):
    """Ring cell with losses, no collective operator: every launch shape
    gives bit-identical particles, masks and counts."""
    n = 20000
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 51)
    lat, ref = product_lattice(ring_cell(radius=0.004))
    out = []
    for cfg in CONFIGS:
        prop = syn.Propagator(lat, syn.Split_operator_stepper(None, 16))
        prop.set_tune(**cfg)
        assert {k: prop.get_tune()[k] for k in cfg} == cfg
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.propagate(b, 2)
        out.append((b.get_particles(), b.counts()))
    for (parts, c) in out[1:]:
        assert np.array_equal(parts[0], out[0][0][0]) and np.array_equal(parts[1], out[0][0][1])
        assert c == out[0][1]


def test_gpu_launch_shapes_with_space_charge(syn):
    """FODO with space charge: every launch shape and re-sort interval agrees
    to the deposit's atomic-order rounding."""
    n = 30000
    p = gaussian_bunch(n, SIG_C0, 52)
    lat, ref = product_lattice(fodo_cell())
    out = []
    for cfg, si in zip(CONFIGS, (4, 2, 8, 1)):
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 8))
        prop.set_tune(sort_interval=si, **cfg)
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.propagate(b, 2)
        out.append(b.get_particles()[0])
    for parts in out[1:]:
        assert np.array_equal(parts[:, 6], out[0][:, 6])
        for j in range(6):
            assert rel_l2(parts[:, j], out[0][:, j]) <= 1e-12, j


@pytest.mark.parametrize("grid", [(16, 16, 32), (8, 32, 64)])
def test_gpu_fft_plans_and_deposit_chunks_agree(syn, grid):
    """Both FFT radix plans (the doubled lengths 16, 32 and 128 are not powers
    of 8, so the plans differ there) and every deposit chunk give the same
    particles to the FFT's and the deposit's rounding."""
    n = 40000
    p = gaussian_bunch(n, SIG_C0, 54)
    lat, ref = product_lattice(fodo_cell())
    out = []
    for plan, chunk in ((0, 4), (1, 4), (0, 8), (1, 8), (0, 0)):
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(*grid), 8))
        prop.set_tune(fft_plan=plan, deposit_chunk=chunk)
        assert prop.get_tune()["fft_plan"] == plan and prop.get_tune()["deposit_chunk"] == chunk
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.propagate(b, 2)
        out.append(b.get_particles()[0])
    for parts in out[1:]:
        assert np.array_equal(parts[:, 6], out[0][:, 6])
        for j in range(6):
            assert rel_l2(parts[:, j], out[0][:, j]) <= 1e-12, j


def test_gpu_autotune_leaves_state_and_applies_best(syn):
    """autotune: trials cover every knob, the fastest is applied, the bunch
    (particles, state), per-turn diagnostics and step records are unchanged,
    and propagation afterwards matches an untuned propagator."""
    n = 50000
    p = gaussian_bunch(n, SIG_C0, 53)
    lat, ref = product_lattice(fodo_cell())
    mk = lambda: syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(16, 16, 32), 8))
    prop, plain = mk(), mk()
    b, c = syn.Bunch(ref, n, 1e11), syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    c.set_particles(p)
    prop.set_diagnostics(8)
    prop.set_step_counts(64)
    prop.propagate(b, 1)
    plain.propagate(c, 1)
    before = b.get_particles()
    st0 = b.get_state()
    nrec, ndiag = len(prop.step_counts()), len(prop.diagnostics()["s"])
    best, log = prop.autotune(b, steps=8)
    assert len(log) >= 10
    assert {r["light_shape"] for r in log} == {0, 1, 2, 3} and {r["ctas_per_sm"] for r in log} == {4, 8, 12}
    assert {r["sort_interval"] for r in log} == {2, 4, 8}
    assert {r["fft_plan"] for r in log} == {0, 1} and {r["deposit_chunk"] for r in log} == {4, 8}
    fastest = min(log, key=lambda r: r["ms"])
    assert best == {k: fastest[k] for k in best} == prop.get_tune()
    after = b.get_particles()
    for x, y in zip(before, after):
        assert np.array_equal(x, y)
    st1 = b.get_state()
    assert bytes(st0) == bytes(st1)
    assert len(prop.step_counts()) == nrec and len(prop.diagnostics()["s"]) == ndiag
    prop.propagate(b, 1)
    plain.propagate(c, 1)
    bp, cp_ = b.get_particles()[0], c.get_particles()[0]
    for j in range(6):
        assert rel_l2(bp[:, j], cp_[:, j]) <= 1e-12, j
    assert len(prop.step_counts()) == nrec + plain.num_steps()


def test_gpu_tune_validation(syn):
    lat, ref = product_lattice(fodo_cell())
    prop = syn.Propagator(lat, syn.Split_operator_stepper(None, 8))
    with pytest.raises(syn.SB2Error, match="ctas_per_sm"):
        prop.set_tune(ctas_per_sm=13)
    with pytest.raises(syn.SB2Error, match="full_occ"):
        prop.set_tune(full_occ=1)
    with pytest.raises(syn.SB2Error, match="fft_plan"):
        prop.set_tune(fft_plan=2)
    with pytest.raises(syn.SB2Error, match="deposit_chunk"):
        prop.set_tune(deposit_chunk=6)
