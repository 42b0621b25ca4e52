"""GPU parity of the 3D open-boundary Hockney space-charge solver.

FP64 tolerances (written in each test):
  * charge density, potential and fields: 1e-10 relative L2 against the
    oracle on the same particles (the deposit's summation order and the FFT
    algorithm are the only differences);
  * kicked coordinates: the kick itself (xp, yp, dpop change) within 1e-9
    relative of the oracle's kick, positions bit-identical;
  * known answers of the reference's own tests: rod-bunch line-charge kick
    and Gaussian-sphere field.
"""
import math

import numpy as np
import pytest

from helpers import MP, SIG_C0, fodo_cell, gaussian_bunch, oracle_lattice, product_lattice, rel_l2

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-10


def sc_both(syn, orc, parts, shape, time_step, real_num=1e11, green_fn=1, fixed=None, value=2.5 + MP, masks=None):
    gx, gy, gz = shape
    opts = syn.Space_charge_3d_open_hockney_options(gx, gy, gz)
    opts.green_fn = green_fn
    if fixed is not None:
        opts.set_fixed_domain(*fixed)
    fm = syn.Four_momentum(MP, value)
    ref = syn.Reference_particle(1, fm)
    b = syn.Bunch(ref, parts.shape[0], real_num)
    b.set_particles(parts, masks)
    sc = syn.Space_charge_3d_open_hockney(opts)
    sc.apply(b, time_step)
    gp, gm, _ = b.get_particles()
    g = sc.last()
    oopts = orc.SCOptions.make(gx, gy, gz, green_fn=green_fn, fixed=fixed)
    op, o = orc.sc_apply(oopts, parts, time_step, real_num, masks=masks, value=value, kind=orc.REF_TOTAL_ENERGY)
    return gp, g, op, o


@pytest.mark.parametrize("shape", [(16, 16, 32), (32, 16, 64), (8, 32, 16), (8, 8, 256), (8, 256, 16)])
@pytest.mark.parametrize("green_fn", [1, 0])
def test_sc_fields_match_oracle(syn, orc, shape, green_fn):
    n = 200000
    p = gaussian_bunch(n, SIG_C0, 21)
    ts = 1.25 / (0.96 * 299792458.0)
    gp, g, op, o = sc_both(syn, orc, p, shape, ts, green_fn=green_fn)
    assert np.allclose(g["left"], o["left"], rtol=1e-13, atol=0)
    assert np.allclose(g["h"], o["h"], rtol=1e-13, atol=0)
    assert rel_l2(g["rho"], o["rho"]) <= FIELD_TOL
    assert rel_l2(g["phi"], o["phi"]) <= FIELD_TOL
    for c in ("ex", "ey", "ez"):
        assert rel_l2(g[c], o[c]) <= FIELD_TOL, c
    assert abs(g["fn_norm"] / o["fn_norm"] - 1) <= 1e-13
    assert abs(g["factor"] / o["factor"] - 1) <= 1e-13
    # positions untouched, kicks agree
    for j in (0, 2, 4, 6):
        assert np.array_equal(gp[:, j], op[:, j])
    for j in (1, 3, 5):
        kick_g = gp[:, j] - p[:, j]
        kick_o = op[:, j] - p[:, j]
        assert rel_l2(kick_g, kick_o) <= 1e-9, j


def test_sc_fixed_domain_and_masks(syn, orc):
    n = 100000
    p = gaussian_bunch(n, SIG_C0, 22)
    m = np.ones(n, np.uint8)
    m[::5] = 0
    fixed = ((0.0, 0.0, 0.0), (8e-3, 8e-3, 2.4))
    gp, g, op, o = sc_both(syn, orc, p, (16, 16, 16), 1e-8, fixed=fixed, masks=m)
    assert rel_l2(g["rho"], o["rho"]) <= FIELD_TOL
    for c in ("ex", "ey", "ez"):
        assert rel_l2(g[c], o[c]) <= FIELD_TOL
    dead = ~m.astype(bool)
    assert np.array_equal(gp[dead], p[dead])


def test_sc_rod_bunch_line_charge(syn):
    """collective/tests/test_space_charge_3d_open_hockney_mpi.cc:8-107 at the
    reference's size (2,000,009 particles, 256 x 256 x 64, fixed domain):
    probe kick vs 2 N r_p / (L beta^2 gamma^3) * D / r to 1e-3 relative
    (the reference allows 0.01 absolute)."""
    from test_oracle import rod_bunch
    for gamma in (61.0 / 60.0, 61.0 / 11.0):
        p, beta = rod_bunch(250001, gamma)
        probe = 80e-6
        opts = syn.Space_charge_3d_open_hockney_options(256, 256, 64)
        opts.set_fixed_domain([0, 0, 0], [probe * 4, probe * 4, 0.1 / beta])
        ref = syn.Reference_particle(1, syn.Four_momentum(MP, MP * gamma))
        b = syn.Bunch(ref, p.shape[0], 5.0e9)
        b.set_particles(p)
        syn.Space_charge_3d_open_hockney(opts).apply(b, 0.1 / (beta * 299792458.0))
        out = b.get_particles()[0]
        bg = beta * gamma
        rp = syn.pconstants.rp
        expected = ((2.0 * 5.0e9 * rp) / (0.1 * bg * bg * gamma)) * (0.1 / probe)
        assert abs(out[0, 1] - expected) < 0.01
        assert abs(out[0, 1] / expected - 1) < 1e-3


def test_sc_degenerate_domain_error(syn):
    """space_charge_3d_open_hockney.cc:512-516: all sigmas below 1e-10."""
    ref = syn.Reference_particle(1, syn.Four_momentum(MP, MP + 2.5))
    b = syn.Bunch(ref, 1000, 1e10)
    sc = syn.Space_charge_3d_open_hockney(syn.Space_charge_3d_open_hockney_options(8, 8, 8))
    with pytest.raises(syn.SB2Error, match="neglible extent"):
        sc.apply(b, 1e-9)


def test_propagate_with_space_charge_matches_oracle(syn, orc):
    """FODO cell, split operator with 8 kicks per cell, adaptive domain,
    linear Green function, 2 turns (16 kicks): last solve's fields within
    1e-10 of the oracle's, coordinates within 1e-12 relative (the deposit
    order moves them by ~1e-14, measured at full size in
    test_gpu_parity_scale.py), ids and masks exact."""
    n, shape, turns = 100000, (16, 16, 32), 2
    p = gaussian_bunch(n, SIG_C0, 31)
    lat, ref = product_lattice(fodo_cell())
    opts = syn.Space_charge_3d_open_hockney_options(*shape)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 8))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, turns)
    gp, gm, _ = b.get_particles()
    g = prop.sc_last()
    sim = orc.Sim(oracle_lattice(fodo_cell()), n, 1e11, stepper=orc.STEPPER_SPLIT, num=8,
                  sc=orc.SCOptions.make(*shape), value=2.5 + MP)
    sim.set_particles(p)
    sim.propagate(turns)
    op, om, _ = sim.get_particles()
    o = sim.sc_last(shape)
    assert np.array_equal(gm, om) and np.array_equal(gp[:, 6], op[:, 6])
    for c in ("rho", "ex", "ey", "ez"):
        assert rel_l2(g[c], o[c]) <= FIELD_TOL, c
    for j in range(6):
        assert rel_l2(gp[:, j], op[:, j]) <= 1e-12, j


def test_bunch_moments_and_emittance(syn):
    n = 100000
    p = gaussian_bunch(n, SIG_C0, 41)
    ref = syn.Reference_particle(1, syn.Four_momentum(MP, MP + 2.5))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    mean, mom2, emit = b.moments()
    assert np.allclose(mean, p[:, :6].mean(0), rtol=0, atol=1e-12)
    c = np.cov(p[:, :6].T, bias=True)
    assert np.allclose(mom2, c, rtol=1e-9, atol=1e-30)
    ex = math.sqrt(c[0, 0] * c[1, 1] - c[0, 1] ** 2)
    assert abs(emit[0] / ex - 1) < 1e-9


def test_populate_gaussian_statistics(syn):
    n = 1 << 20
    ref = syn.Reference_particle(1, syn.Four_momentum(MP, MP + 2.5))
    b = syn.Bunch(ref, n, 1e11)
    b.populate_gaussian(SIG_C0, seed=3)
    p, m, _ = b.get_particles()
    assert m.all() and np.array_equal(p[:, 6], np.arange(n))
    sd = p[:, :6].std(0)
    assert np.allclose(sd, SIG_C0, rtol=5e-3)
    b2 = syn.Bunch(ref, n, 1e11)
    b2.populate_gaussian(SIG_C0, seed=3)
    assert np.array_equal(b2.get_particles()[0], p)


def test_cell_sorted_working_copy_matches_unsorted(syn, monkeypatch):
    """The propagator's cell-ordered working copy is invisible to callers:
    particles come back in their original order (ids, masks) and agree with
    a run without it to the FP64 tolerance of the deposit order."""
    n, shape = 50000, (16, 16, 32)
    p = gaussian_bunch(n, SIG_C0, 61)
    p[::97, 0] += 0.05  # a few particles outside the domain
    out = []
    for sort in ("1", "0"):
        monkeypatch.setenv("SB2_CELL_SORT", sort)
        lat, ref = product_lattice(fodo_cell())
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(*shape), 8))
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        prop.propagate(b, 1)
        out.append(b.get_particles())
    (a, am, ad), (u, um, ud) = out
    assert np.array_equal(a[:, 6], np.arange(n)) and np.array_equal(am, um) and np.array_equal(ad, ud)
    for j in range(6):
        assert rel_l2(a[:, j], u[:, j]) <= 1e-10, j


def test_working_copy_persists_between_calls(syn, monkeypatch):
    """An owned bunch stays in its cell-ordered working copy between
    propagate calls (no re-sort from the caller's order at every call): 15
    steps in five calls give the caller's order back and agree with an
    unsorted run to the FP64 tolerance of the deposit order."""
    n, shape = 50000, (16, 16, 32)
    p = gaussian_bunch(n, SIG_C0, 62)
    out = []
    for sort in ("1", "0"):
        monkeypatch.setenv("SB2_CELL_SORT", sort)
        lat, ref = product_lattice(fodo_cell())
        prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(*shape), 8))
        b = syn.Bunch(ref, n, 1e11)
        b.set_particles(p)
        for k in range(5):
            prop.propagate_steps(b, 3 * k, 3)
        out.append(b.get_particles())
    (a, am, ad), (u, um, ud) = out
    assert np.array_equal(a[:, 6], np.arange(n)) and np.array_equal(am, um) and np.array_equal(ad, ud)
    for j in range(6):
        assert rel_l2(a[:, j], u[:, j]) <= 1e-10, j


def test_wrapped_bunch_arrays_current_after_each_call(syn, monkeypatch):
    """A bunch over caller-owned device arrays (sb2_bunch_wrap) has its
    particles back in those arrays, in the caller's order, when a propagate
    call returns."""
    import ctypes
    import torch
    monkeypatch.setenv("SB2_CELL_SORT", "1")
    n, shape = 30000, (16, 16, 32)
    p = gaussian_bunch(n, SIG_C0, 63)
    lat, ref = product_lattice(fodo_cell())
    opts = syn.Space_charge_3d_open_hockney_options(*shape)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 8))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 1)
    expect = b.get_particles()[0]

    L = syn.lib()
    dparts = torch.tensor(np.ascontiguousarray(p.T), device="cuda")  # (7, n): column-major N x 7
    dmask = torch.ones(n, dtype=torch.uint8, device="cuda")
    ddisc = torch.zeros(n, dtype=torch.uint8, device="cuda")
    h = ctypes.c_void_p()
    syn.check(L.sb2_bunch_wrap(1, MP, MP + 2.5, 0, ctypes.c_void_p(dparts.data_ptr()), n,
                               ctypes.c_void_p(dmask.data_ptr()), ctypes.c_void_p(ddisc.data_ptr()), n, 1e11,
                               ctypes.byref(h)))
    try:
        prop2 = syn.Propagator(lat, syn.Split_operator_stepper(opts, 8))
        syn.check(L.sb2_propagator_propagate(prop2.h, h, 1, None))
        torch.cuda.synchronize()
        got = dparts.cpu().numpy().T
        assert np.array_equal(got[:, 6], np.arange(n))
        assert dmask.cpu().numpy().all()
        for j in range(6):
            assert rel_l2(got[:, j], expect[:, j]) <= 1e-10, j
    finally:
        L.sb2_bunch_destroy(h)


def test_c3_size_ring_properties(syn):
    """The ring configuration at full size (16,777,216 macroparticles,
    128 x 128 x 256 grid, 16 kicks per cell, circular aperture), one turn:
    size-independent properties -- ids stay a permutation of 0..N-1 in the
    caller's order, lost particles are exactly the masked-out ones and the
    bunch counters agree with the masks; and on the turn's final particles
    the mixed-precision field is within 1e-5 relative L2 of the FP64 field."""
    from helpers import ring_cell
    n, shape = 16777216, (128, 128, 256)
    lat, ref = product_lattice(ring_cell() * 24)
    opts = syn.Space_charge_3d_open_hockney_options(*shape)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 384))
    b = syn.Bunch(ref, n, 1e11)
    b.populate_gaussian([2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], seed=3)
    prop.propagate(b, 1)
    gp, gm, gd = b.get_particles()
    assert np.array_equal(gp[:, 6], np.arange(n))
    c = b.counts()
    assert c["local_num"] == int(gm.sum()) == c["total_num"]
    assert np.array_equal(gd.astype(bool) & ~gm.astype(bool), gd.astype(bool))  # discarded => masked
    fields = []
    for prec in (syn.precision_t.fp64, syn.precision_t.mixed):
        o = syn.Space_charge_3d_open_hockney_options(*shape)
        o.precision = prec
        bb = syn.Bunch(ref, n, 1e11)
        bb.set_particles(gp, gm)
        sc = syn.Space_charge_3d_open_hockney(o)
        sc.apply(bb, 0.5 / (0.96 * 299792458.0))
        fields.append(sc.last())
        del sc, bb
    num = sum(float(((fields[1][k] - fields[0][k]) ** 2).sum()) for k in ("ex", "ey", "ez"))
    den = sum(float((fields[0][k] ** 2).sum()) for k in ("ex", "ey", "ez"))
    assert np.sqrt(num / den) <= 1e-5


@pytest.mark.parametrize("green_fn,fixed", [(0, None), (1, ((0.0, 0.0, 0.0), (1.2e-2, 1.2e-2, 3.0)))])
def test_split_operator_elements_with_space_charge(syn, orc, green_fn, fixed):
    """Split_operator_stepper_elements (split_operator_stepper_elements.cc:
    4-47: kicks per element) with space charge, pointlike Green function and
    adaptive domain, or linear Green function and a fixed domain: two turns
    of the ring cell (bends, thin sextupoles, apertures) within 1e-10 of the
    oracle; lost sets exact."""
    from helpers import ring_cell
    n, shape = 40000, (16, 16, 32)
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 33)
    spec = ring_cell(radius=0.006)
    lat, ref = product_lattice(spec)
    opts = syn.Space_charge_3d_open_hockney_options(*shape)
    opts.green_fn = green_fn
    if fixed is not None:
        opts.set_fixed_domain(*fixed)
    prop = syn.Propagator(lat, syn.Split_operator_stepper_elements(opts, 2))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 2)
    gp, gm, gd = b.get_particles()
    sim = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT_ELEMENTS, num=2,
                  sc=orc.SCOptions.make(*shape, green_fn=green_fn, fixed=fixed), value=2.5 + MP)
    sim.set_particles(p)
    sim.propagate(2)
    op, om, od = sim.get_particles()
    assert np.array_equal(gm, om) and np.array_equal(gd, od) and np.array_equal(gp[:, 6], op[:, 6])
    assert 0 < int(gm.sum()) < n
    alive = gm.astype(bool)
    for j in range(6):
        assert rel_l2(gp[alive, j], op[alive, j]) <= 1e-10, j
    c = b.counts()
    nv, nt, rn = sim.counts()
    assert c["total_num"] == nt and c["real_num"] == rn
