"""GPU parity of the element maps and apertures against the oracle.

The FP64 map kernels run without FMA contraction and with IEEE sqrt/div, so
drift, quadrupole (Yoshida), thin multipole and sextupole maps are compared
bit for bit with the oracle; the sector bend calls asin/sin/cos, whose CUDA
and libm results may differ in the last bit, so it is held to 1e-12
relative.  Particle ids and lost-particle sets must match exactly.
"""
import json
import math
import os

import numpy as np
import pytest

from helpers import (MP, ROOT, SIG_C0, elem, fodo_cell, gaussian_bunch, oracle_lattice, product_lattice,
                     ring_cell)

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "madx_tracks.json")))["cases"]


def run_both(syn, orc, spec, parts, stepper, num, turns, value=2.5 + MP, kind=0, masks=None, real_num=1e11):
    n = parts.shape[0]
    lat, ref = product_lattice(spec, value=value, kind=kind)
    if stepper == "indep":
        st, ok = syn.Independent_stepper_elements(num), orc.STEPPER_INDEP_ELEMENTS
    elif stepper == "split":
        st, ok = syn.Split_operator_stepper(None, num), orc.STEPPER_SPLIT
    else:
        st, ok = syn.Split_operator_stepper_elements(None, num), orc.STEPPER_SPLIT_ELEMENTS
    prop = syn.Propagator(lat, st)
    b = syn.Bunch(ref, n, real_num)
    b.set_particles(parts, masks)
    prop.propagate(b, turns)
    gp, gm, gd = b.get_particles()
    sim = orc.Sim(oracle_lattice(spec, value=value, kind=kind), n, real_num, stepper=ok, num=num,
                  value=value, kind=kind)
    sim.set_particles(parts, masks)
    sim.propagate(turns)
    op, om, od = sim.get_particles()
    return (gp, gm, gd, b, prop), (op, om, od, sim)


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_gpu_madx_golden(syn, orc, case):
    """The reference's MAD-X element tests through the GPU path: within the
    reference's tolerances of MAD-X and bit-identical to the oracle."""
    p = np.zeros((16, 7), order="F")
    p[:, :6] = np.array(case["initial"])
    p[:, 6] = np.arange(16)
    (gp, gm, _, _, _), (op, _, _, _) = run_both(syn, orc, case["lattice"], p, "indep", 1, 1,
                                                value=case["p0"], kind=1, real_num=1e10)
    exp = np.array(case["expected"])
    tol = np.array(case["tol"])
    assert np.all(np.abs(gp[:, :6] - exp) <= tol)
    if case["name"] in ("solenoid", "rfc") or case["name"].startswith("cfsbend"):
        # CUDA's sin/cos/asin/log vs libm: last-bit differences
        scale = np.max(np.abs(op[:, :6]), axis=0)
        assert np.all(np.abs(gp[:, :6] - op[:, :6]) <= 1e-12 * scale)
    else:
        assert np.array_equal(gp, op)
    assert gm.all()


def test_gpu_fodo_no_space_charge_bit_exact(syn, orc):
    """FODO cell, split-operator stepper with 8 steps and no collective
    operator, 3 turns: every coordinate bit-identical to the oracle."""
    n = 20000
    p = gaussian_bunch(n, SIG_C0, 11)
    (gp, gm, gd, b, _), (op, om, od, sim) = run_both(syn, orc, fodo_cell(), p, "split", 8, 3)
    assert np.array_equal(gp, op)
    assert np.array_equal(gm, om) and gm.all()
    st_g, sn_g = b.design_state()
    st_o, sn_o = sim.design_state()
    assert np.array_equal(st_g, st_o) and sn_g == sn_o


def test_gpu_ring_losses_exact(syn, orc):
    """Ring cell (sector bends, thin sextupoles, r = 4 mm circular aperture
    on every element) with a bunch wide enough to lose particles: lost sets,
    ids, discards and the n_valid / n_total / real_num bookkeeping match the
    oracle exactly; surviving coordinates within 1e-12 relative."""
    n = 30000
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 5)
    (gp, gm, gd, b, _), (op, om, od, sim) = run_both(syn, orc, ring_cell(radius=0.004), p, "split", 16, 2)
    assert np.array_equal(gm, om)
    assert np.array_equal(gd, od)
    assert 0 < int(gm.sum()) < n
    assert np.array_equal(gp[:, 6], op[:, 6])
    scale = np.max(np.abs(op[:, :6]), axis=0)
    alive = om.astype(bool)
    err = np.max(np.abs(gp[alive, :6] - op[alive, :6]), axis=0) / scale
    assert np.all(err <= 1e-12), err
    c = b.counts()
    nv, nt, rn = sim.counts()
    assert c["local_num"] == nv and c["total_num"] == nt
    assert c["real_num"] == rn


def test_gpu_finite_aperture_discards_nan(syn, orc):
    """Finite_aperture (aperture_operation.h:54-86) drops NaN/Inf particles
    and particles with (1+dpop)^2 < xp^2 + yp^2."""
    n = 1000
    p = gaussian_bunch(n, SIG_C0, 2)
    p[3, 0] = np.nan
    p[7, 1] = np.inf
    p[11, 1] = 2.0  # xp > 1 + dpop
    (gp, gm, gd, b, _), (op, om, od, _) = run_both(syn, orc, fodo_cell(), p, "split", 4, 1)
    assert not gm[3] and not gm[7] and not gm[11]
    assert np.array_equal(gm, om)
    assert b.get_total_num() == n - 3


def test_gpu_masked_particles_frozen(syn, orc):
    """Masked-out particles are not propagated (masks checked per particle,
    gsv size 1 on the GPU build)."""
    n = 512
    p = gaussian_bunch(n, SIG_C0, 9)
    m = np.ones(n, np.uint8)
    m[::7] = 0
    (gp, gm, _, b, _), (op, om, _, _) = run_both(syn, orc, fodo_cell(), p, "split", 8, 1, masks=m)
    assert np.array_equal(gp[~m.astype(bool)], p[~m.astype(bool)])
    assert np.array_equal(gp, op) and np.array_equal(gm, om)


@pytest.mark.parametrize("elem_def,tol", [
    (elem("sbend", "b", l=2.0, angle=math.pi / 24), 2.0e-17),
    (elem("drift", "d", l=10.0), 2.0e-17),
    (elem("quadrupole", "q", l=4.0, k1=1 / 10), 2.0e-17),
    (elem("sextupole", "s", l=0.5, k2=0.25), 2.0e-17),
    (elem("quadrupole", "q", l=4.0, k1=1 / 10, tilt=math.pi / 4), 2.0e-17),
])
def test_gpu_zero_particle(syn, orc, elem_def, tol):
    """libFF/tests/test_zeroparticle_propagate.cc: a particle at 0 stays at 0
    and the design particle's cdt * beta equals the element length."""
    n = 8
    p = np.zeros((n, 7), order="F")
    p[:, 6] = np.arange(n)
    value = 0.8 + MP
    (gp, _, _, b, _), (op, _, _, sim) = run_both(syn, orc, [elem_def], p, "indep", 1, 1, value=value, real_num=1e9)
    assert np.all(np.abs(gp[0, :4]) < tol)
    st, _ = b.design_state()
    gamma = value / MP
    beta = math.sqrt(1 - 1 / gamma ** 2)
    L = elem_def["double"]["l"]
    assert abs(1 - st[4] * beta / L) < 1.0e-7
    assert np.allclose(gp, op, rtol=0, atol=1e-15)


def test_gpu_thin_elements_and_edge_apertures(syn, orc):
    """Thin multipole (MAD-X knl/ksl and MAD8 kNl forms, tilt), thin
    sextupole, element apertures from aperture_type (independent_operator.cc:
    41-72), elliptical and rectangular apertures."""
    spec = [elem("drift", "d0", l=0.3),
            elem("multipole", "m1", knl=[0.0, 0.02, 1.5], ksl=[0.0, 0.0, 0.3], tilt=0.1),
            elem("multipole", "m2", k1l=0.01, k2l=-0.5, t2=0.05),
            elem("quadrupole", "q", l=0.4, k1=0.7, aperture_type="elliptical",
                 elliptical_aperture_horizontal_radius=0.004, elliptical_aperture_vertical_radius=0.003),
            elem("sextupole", "s", l=0.0, k2=3.0, k2s=0.5),
            elem("drift", "d1", l=0.6, aperture_type="rectangular", rectangular_aperture_width=0.008,
                 rectangular_aperture_height=0.006)]
    n = 20000
    p = gaussian_bunch(n, [2e-3, 2e-4, 2e-3, 2e-4, 0.3, 1e-3], 4)
    (gp, gm, gd, b, _), (op, om, od, sim) = run_both(syn, orc, spec, p, "split", 3, 2)
    assert np.array_equal(gm, om) and np.array_equal(gd, od)
    assert 0 < int(gm.sum()) < n
    assert np.array_equal(gp, op)


def test_gpu_quad_multipole_errors(syn, orc):
    """Quadrupole with a_n / b_n multipole errors (cf_kick, ff_quadrupole.h:
    22-35, 362-391) and offsets."""
    spec = [elem("quadrupole", "q", l=0.8, k1=0.5, b2=0.3, a3=0.1, hoffset=1e-4, voffset=-2e-4, tilt=0.02,
                 yoshida_steps=3), elem("drift", "d", l=1.0)]
    n = 5000
    p = gaussian_bunch(n, SIG_C0, 8)
    (gp, gm, _, _, _), (op, om, _, _) = run_both(syn, orc, spec, p, "indep", 2, 1)
    assert np.array_equal(gp, op)


def test_gpu_yoshida_sextupole_thick(syn, orc):
    n = 5000
    p = gaussian_bunch(n, SIG_C0, 6)
    spec = [elem("sextupole", "s", l=0.7, k2=2.0, k2s=0.3, tilt=0.1), elem("drift", "d", l=0.5)]
    (gp, _, _, b, _), (op, _, _, sim) = run_both(syn, orc, spec, p, "indep", 3, 2)
    assert np.array_equal(gp, op)
    assert np.array_equal(b.design_state()[0], sim.design_state()[0])


def test_gpu_empty_bunch(syn):
    lat, ref = product_lattice(fodo_cell())
    prop = syn.Propagator(lat, syn.Split_operator_stepper(None, 8))
    b = syn.Bunch(ref, 0, 1e11)
    prop.propagate(b, 2)
    assert b.get_total_num() == 0


def test_gpu_unsupported_element_is_reported(syn):
    lat, ref = product_lattice([elem("elens", "el", l=0.0, current=1.0, eenergy=0.01, radius=1e-3)])
    prop = syn.Propagator(lat, syn.Independent_stepper_elements(1))
    b = syn.Bunch(ref, 16, 1e10)
    with pytest.raises(syn.SB2Error, match="elens"):
        prop.propagate(b, 1)


def test_gpu_octupole_and_kickers_sliced(syn, orc):
    """Thick and thin octupoles and kickers (FF_octupole, FF_kicker through
    FF_patterned_propagator) cut into slices by the split-operator stepper,
    including a drift-kick-drift ('simple') kicker and one whose design
    particle is timed by a drift: bit-identical to the oracle after two
    turns."""
    spec = [elem("drift", "d0", l=0.3),
            elem("octupole", "o1", l=0.6, k3=40.0, k3s=5.0, tilt=0.2),
            elem("hkicker", "h1", l=0.4, kick=2e-4),
            elem("octupole", "o2", l=0.0, k3=3.0),
            elem("vkicker", "v1", l=0.0, kick=-1e-4),
            elem("kicker", "k1", l=0.5, hkick=1e-4, vkick=-2e-4, tilt=0.1, simple=1.0),
            elem("kicker", "k2", l=0.5, hkick=-1e-4, vkick=1e-4, cdt_use_drift=1.0),
            elem("drift", "d1", l=0.7)]
    n = 20000
    p = gaussian_bunch(n, [2e-3, 2e-4, 2e-3, 2e-4, 0.3, 1e-3], 12)
    (gp, gm, _, b, _), (op, om, _, sim) = run_both(syn, orc, spec, p, "split", 5, 2)
    assert np.array_equal(gm, om)
    assert np.array_equal(gp, op)
    assert np.array_equal(b.design_state()[0], sim.design_state()[0])


def test_gpu_solenoid_sliced(syn, orc):
    """Solenoid (FF_solenoid) cut into slices by the split-operator stepper:
    entry and exit edge kicks only on the end slices; within 1e-12 of the
    oracle (CUDA's sin/cos vs libm)."""
    spec = [elem("drift", "d0", l=0.2), elem("solenoid", "s1", l=1.3, ks=0.4), elem("drift", "d1", l=0.5),
            elem("solenoid", "s2", l=0.6, ks=0.0)]
    n = 10000
    p = gaussian_bunch(n, [2e-3, 2e-4, 2e-3, 2e-4, 0.3, 1e-3], 14)
    (gp, gm, _, b, _), (op, om, _, sim) = run_both(syn, orc, spec, p, "split", 4, 2)
    assert np.array_equal(gm, om) and np.array_equal(gp[:, 6], op[:, 6])
    scale = np.max(np.abs(op[:, :6]), axis=0)
    assert np.all(np.abs(gp[:, :6] - op[:, :6]) <= 1e-12 * scale)


def test_gpu_rfcavity_accelerates_with_space_charge(syn, orc):
    """A thick rf cavity (FF_rfcavity: half drift, thin_rfcavity_unit, half
    drift) with a second harmonic in a FODO cell with space charge: the
    bunch's reference momentum changes at every pass, the kick factor and
    every later map follow it; two turns agree with the oracle to 1e-10
    (CUDA's sin vs libm and the deposit order), ids and masks exact."""
    spec = fodo_cell() + [elem("rfcavity", "rf", l=0.4, volt=0.8, lag=0.3, freq=53.0, h2_str=0.2, h2_phase=0.1)]
    n, shape = 30000, (16, 16, 32)
    p = gaussian_bunch(n, SIG_C0, 15)
    lat, ref = product_lattice(spec)
    opts = syn.Space_charge_3d_open_hockney_options(*shape)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 9))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 2)
    gp, gm, _ = b.get_particles()
    sim = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT, num=9, sc=orc.SCOptions.make(*shape),
                  value=2.5 + MP)
    sim.set_particles(p)
    sim.propagate(2)
    op, om, _ = sim.get_particles()
    assert np.array_equal(gm, om) and np.array_equal(gp[:, 6], op[:, 6])
    from helpers import rel_l2
    for j in range(6):
        assert rel_l2(gp[:, j], op[:, j]) <= 1e-10, j


def _close_to_oracle(gp, gm, op, om, rel=1e-12):
    assert np.array_equal(gm, om) and np.array_equal(gp[:, 6], op[:, 6])
    alive = om.astype(bool)
    scale = np.max(np.abs(op[alive, :6]), axis=0)
    err = np.max(np.abs(gp[alive, :6] - op[alive, :6]), axis=0) / scale
    assert np.all(err <= rel), err


def test_gpu_cf_sbend_sliced_with_faces(syn, orc):
    """Combined-function sector bends (FF_sbend with k1..k4(s): PropSbendCF,
    bend_yoshida6 with thin_cf_kick_5) with entry/exit face angles in a
    focusing cell, cut into slices by the split-operator stepper so that
    only the end slices carry the edges, two turns.  The bend map computes
    x as the difference of two numbers of the size of the bend radius, so
    last-bit differences (CUDA's asin/sin/cos/log vs libm) grow along the
    lattice: the GPU must stay within 4x the oracle's own spread under a
    one-ulp change of the initial coordinates, and that spread itself below
    1e-8 relative.  The design particle (host side in both) is exact."""
    spec = [elem("quadrupole", "qf", l=0.5, k1=0.6), elem("drift", "d0", l=0.4),
            elem("sbend", "b1", l=1.5, angle=0.12, k1=0.05, k2=0.8, k2s=-0.4, e1=0.03, e2=0.05),
            elem("drift", "d1", l=0.6), elem("quadrupole", "qd", l=0.5, k1=-0.6), elem("drift", "d2", l=0.4),
            elem("sbend", "b2", l=1.0, angle=0.08, k1s=0.02, k3=3.0, k4=-10.0, k4s=5.0), elem("drift", "d3", l=0.6)]
    n = 20000
    p = gaussian_bunch(n, SIG_C0, 21)
    (gp, gm, _, b, _), (op, om, _, sim) = run_both(syn, orc, spec, p, "split", 6, 2)
    assert np.array_equal(gm, om) and np.array_equal(gp[:, 6], op[:, 6])
    q = p.copy()
    q[:, :6] *= 1.0 + 2.0 ** -52
    sim2 = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT, num=6, value=2.5 + MP)
    sim2.set_particles(q)
    sim2.propagate(2)
    oq = sim2.get_particles()[0]
    scale = np.max(np.abs(op[:, :6]), axis=0)
    spread = np.max(np.abs(oq[:, :6] - op[:, :6]), axis=0)
    assert np.all(spread <= 1e-8 * scale), spread / scale
    err = np.max(np.abs(gp[:, :6] - op[:, :6]), axis=0)
    assert np.all(err <= 4.0 * spread + 1e-15 * scale), (err / scale, spread / scale)
    assert np.array_equal(b.design_state()[0], sim.design_state()[0])  # both on the host (libm)


def test_gpu_sbend_multipole_moments_use_cf_path(syn, orc):
    """An sbend with b_n / a_n moments (ff_sbend.h:790-828: scaled by angle
    * n! into the combined-function strengths) runs the combined-function
    integrator, here with space charge in the same passes: one turn agrees
    with the oracle to 1e-10 (libm vs CUDA and the deposit order), ids and
    masks exact."""
    spec = [elem("quadrupole", "q", l=0.4, k1=0.5),
            elem("sbend", "b", l=2.0, angle=0.1, b1=0.05, a2=0.3, b3=2.0),
            elem("drift", "d", l=1.0)]
    n, shape = 30000, (16, 16, 32)
    p = gaussian_bunch(n, SIG_C0, 22)
    lat, ref = product_lattice(spec)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(syn.Space_charge_3d_open_hockney_options(*shape), 4))
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 1)
    gp, gm, _ = b.get_particles()
    sim = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT, num=4, sc=orc.SCOptions.make(*shape),
                  value=2.5 + MP)
    sim.set_particles(p)
    sim.propagate(1)
    op, om, _ = sim.get_particles()
    assert np.array_equal(gm, om) and np.array_equal(gp[:, 6], op[:, 6])
    from helpers import rel_l2
    for j in range(6):
        assert rel_l2(gp[:, j], op[:, j]) <= 1e-10, j
    assert np.array_equal(b.design_state()[0], sim.design_state()[0])


def test_gpu_sbend_both_k_and_moments_is_an_error(syn):
    """ff_sbend.h:815-819: k_n and a/b moments of the same order are
    forbidden together."""
    lat, ref = product_lattice([elem("sbend", "b", l=1.0, angle=0.1, k1=0.2, b1=0.1)])
    prop = syn.Propagator(lat, syn.Independent_stepper_elements(1))
    b = syn.Bunch(ref, 16, 1e10)
    with pytest.raises(syn.SB2Error, match="forbidden in sbends"):
        prop.propagate(b, 1)


def test_gpu_nllens_matches_oracle(syn, orc):
    """Thin nonlinear lens (FF_nllens) between two 0.5 um drifts: the
    golden file's 32 points plus random ones and a particle on the cut
    (y = 0, |x| > cnll), whose angles become NaN and which the Finite
    aperture at the end of the operator then removes.  Within 1e-12 of the
    oracle (CUDA's atan and log vs libm); masks and ids exact."""
    import json
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "nllens_track.json")))
    knll, cnll, d = g["knll"], g["cnll"], g["drift"]
    spec = [elem("drift", "d1", l=d), elem("nllens", "nll", l=0.0, knll=knll, cnll=cnll), elem("drift", "d2", l=d)]
    init = np.array(g["initial"])
    rng = np.random.default_rng(6)
    n = 32 + 200 + 1
    p = np.zeros((n, 7), order="F")
    p[:32, :6] = init
    p[32:232, 0] = rng.uniform(-6e-3, 6e-3, 200)
    p[32:232, 2] = rng.uniform(-6e-3, 6e-3, 200)
    p[232, 0] = 1.5 * cnll  # on the cut
    p[:, 6] = np.arange(n)
    (gp, gm, _, _, _), (op, om, _, _) = run_both(syn, orc, spec, p, "indep", 1, 1, real_num=1e10)
    assert np.array_equal(gm, om) and not gm[232] and gm[:232].all()
    assert np.array_equal(gp[:, 6], op[:, 6])
    alive = om.astype(bool)
    scale = np.max(np.abs(op[alive, :4]), axis=0)
    assert np.all(np.abs(gp[alive, :4] - op[alive, :4]) <= 1e-12 * scale)


def test_gpu_nllens_with_length_is_an_error(syn):
    lat, ref = product_lattice([elem("nllens", "nll", l=0.2, knll=1e-6, cnll=1e-2)])
    prop = syn.Propagator(lat, syn.Independent_stepper_elements(1))
    b = syn.Bunch(ref, 16, 1e10)
    with pytest.raises(syn.SB2Error, match="non-zero length"):
        prop.propagate(b, 1)


def test_gpu_dipedge_bit_exact(syn, orc):
    """Dipole edges (FF_dipedge, MAD-X tmfrng), linear and with the
    second-order terms, around a quadrupole and a drift, split-operator
    stepper, two turns: bit-identical to the oracle, design particle too."""
    spec = [elem("dipedge", "de1", l=0.0, e1=0.12, h=0.8, hgap=0.03, fint=0.4),
            elem("quadrupole", "q", l=0.5, k1=0.3),
            elem("dipedge", "de2", l=0.0, e1=-0.05, h=0.8, hgap=0.03, fint=0.4, second_order=1.0),
            elem("drift", "d", l=0.7)]
    n = 20000
    p = gaussian_bunch(n, [2e-3, 2e-4, 2e-3, 2e-4, 0.3, 1e-3], 23)
    (gp, gm, _, b, _), (op, om, _, sim) = run_both(syn, orc, spec, p, "split", 4, 2)
    assert np.array_equal(gm, om)
    assert np.array_equal(gp, op)
    assert np.array_equal(b.design_state()[0], sim.design_state()[0])


def test_gpu_matrix_element_bit_exact(syn, orc):
    """MAD-X MATRIX elements (FF_matrix): one linear with kicks, one with a
    second-order tensor held in device memory, between drifts, two turns:
    bit-identical to the oracle; the design particle is not moved by them."""
    from test_matrix_element import BOOSTER, matrix_attrs
    g = np.random.default_rng(10)
    rm = np.eye(6) + 0.05 * g.standard_normal((6, 6))
    tm = np.zeros((6, 6, 6))
    tm[0, 0, 0], tm[1, 0, 2], tm[3, 2, 3], tm[4, 5, 5], tm[5, 1, 4] = 2.0, -3.0, 0.5, 10.0, 0.25
    spec = [elem("drift", "d0", l=0.3), elem("matrix", "m1", **matrix_attrs(BOOSTER, kick=[1e-5, 0, -2e-5, 0, 0, 0])),
            elem("drift", "d1", l=0.3), elem("matrix", "m2", **matrix_attrs(rm, tm=tm))]
    n = 5000
    p = gaussian_bunch(n, [1e-4, 1e-5, 1e-4, 1e-5, 0.01, 1e-5], 24)
    (gp, gm, _, b, _), (op, om, _, sim) = run_both(syn, orc, spec, p, "indep", 1, 2)
    assert np.array_equal(gm, om)
    assert np.array_equal(gp, op)
    assert np.array_equal(b.design_state()[0], sim.design_state()[0])
