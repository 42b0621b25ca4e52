"""The per-operator boundary: sb2_libff_apply (LibFF_operation::apply_impl,
simulation/independent_operation.h:45-60 -> FF_element::apply,
libFF/ff_element.h:25-67) and sb2_aperture_apply (Aperture_operation<AP>::
apply_impl, simulation/aperture_operation.h:14-24 -> Bunch::apply_aperture,
bunch/bunch_particles.h:484-524).  These are the bodies of the reference-side
LibFF / Aperture operation shims.

Each half step is driven the way Independent_operator::apply_impl
(simulation/independent_operator.cc:94-133) drives it: one LibFF operation over
the half step's slices, then the Finite and the Circular aperture of its last
slice.  Tolerances: FODO maps bit-identical; ring maps (sector bends call
CUDA's asin/sin/cos) within 1e-12 of each column's scale; discard counts of
every aperture call, lost sets, masks and discard flags exact.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from helpers import MP, ROOT, SIG_C0, fodo_cell, gaussian_bunch, oracle_lattice, product_lattice, ring_cell

SIG_RING = [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4]


def _bunch_with_bad_particles(n, sig, seed):
    p = gaussian_bunch(n, sig, seed)
    p[3, 0] = np.nan      # non-finite: Finite_aperture
    p[7, 1] = np.inf
    p[11, 1] = 2.0        # (1 + dpop)^2 < xp^2 + yp^2: Finite_aperture
    return p


def _oracle_by_operations(orc, spec, p, nsteps, turns):
    """The oracle driven operation by operation, slices from its own stepper."""
    sim = orc.Sim(oracle_lattice(spec), p.shape[0], 1e11, stepper=orc.STEPPER_SPLIT, num=nsteps, value=2.5 + MP)
    sim.set_particles(p)
    counts = []
    for _ in range(turns):
        for s in range(sim.num_steps()):
            for op in (0, 1):
                sl = sim.step_slices(s, op)
                sim.libff_apply(sl)
                last = int(sl[-1, 0])
                for ap in ("finite", "circular"):
                    counts.append(sim.aperture_apply(last, ap))
    return sim, counts


def test_oracle_operations_equal_its_stepper(orc):
    """CPU: the oracle's per-operation entry points, driven as
    Independent_operator drives them, give exactly the oracle stepper's
    particles (ring cell with losses and non-finite particles)."""
    n, nsteps, turns = 4000, 8, 2
    spec = ring_cell(radius=0.006)
    p = _bunch_with_bad_particles(n, SIG_RING, 71)
    ops, counts = _oracle_by_operations(orc, spec, p, nsteps, turns)
    ref = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT, num=nsteps, value=2.5 + MP)
    ref.set_particles(p)
    ref.propagate(turns)
    a, am, ad = ops.get_particles()
    b, bm, bd = ref.get_particles()
    assert np.array_equal(a, b, equal_nan=True) and np.array_equal(am, bm) and np.array_equal(ad, bd)
    assert sum(counts) == n - int(am.sum()) and sum(counts) > 3


def _product_by_operations(syn, spec, p, nsteps, turns, slicer):
    lat, ref = product_lattice(spec)
    b = syn.Bunch(ref, p.shape[0], 1e11)
    b.set_particles(p)
    counts = []
    for _ in range(turns):
        for s in range(slicer.num_steps()):
            for op in (0, 1):
                sl = slicer.step_slices(s, op)
                syn.LibFF_operation(lat, sl).apply(b)
                last = int(sl[-1, 0])
                for ap in ("finite", "circular"):
                    counts.append(syn.Aperture_operation(lat, last, ap).apply(b))
    return b, counts


def _compare(gp, gm, gd, op, om, od, exact):
    assert np.array_equal(gm, om) and np.array_equal(gd, od)
    assert np.array_equal(gp[:, 6], op[:, 6])
    alive = om.astype(bool)
    if exact:
        assert np.array_equal(gp[alive], op[alive])
    else:
        scale = np.max(np.abs(op[alive, :6]), axis=0)
        err = np.max(np.abs(gp[alive, :6] - op[alive, :6]), axis=0) / scale
        assert np.all(err <= 1e-12), err


@pytest.mark.gpu
@pytest.mark.parametrize("lattice", ["fodo", "ring"])
def test_gpu_operations_match_oracle(syn, orc, lattice):
    """Python mirror (LibFF_operation / Aperture_operation) over the C ABI,
    slice lists from the product's own stepper, against the oracle driven the
    same way: per-call discard counts, lost sets and coordinates; the design
    reference particle ends where the oracle's does."""
    n, nsteps, turns = 20000, 8, 2
    spec = fodo_cell() if lattice == "fodo" else ring_cell(radius=0.006)
    sig = SIG_C0 if lattice == "fodo" else SIG_RING
    p = _bunch_with_bad_particles(n, sig, 72)
    lat, _ = product_lattice(spec)
    slicer = syn.Propagator(lat, syn.Split_operator_stepper(None, nsteps))
    b, gcounts = _product_by_operations(syn, spec, p, nsteps, turns, slicer)
    sim, ocounts = _oracle_by_operations(orc, spec, p, nsteps, turns)
    assert gcounts == ocounts
    gp, gm, gd = b.get_particles()
    op, om, od = sim.get_particles()
    _compare(gp, gm, gd, op, om, od, exact=lattice == "fodo")
    assert b.get_local_num() == int(om.sum())
    st_g, _ = b.design_state()
    st_o, _ = sim.design_state()
    if lattice == "fodo":
        assert np.array_equal(st_g, st_o)
    else:
        assert np.allclose(st_g, st_o, rtol=0, atol=1e-15)
    if lattice == "ring":
        assert sum(gcounts) > 3  # losses beyond the three bad particles


@pytest.mark.gpu
def test_gpu_operations_equal_propagator(syn):
    """The per-operation calls and the fused propagator are the same
    physics: FODO without space charge, bit-identical particles."""
    n, nsteps, turns = 20000, 8, 2
    p = _bunch_with_bad_particles(n, SIG_C0, 73)
    lat, ref = product_lattice(fodo_cell())
    prop = syn.Propagator(lat, syn.Split_operator_stepper(None, nsteps))
    b1, _ = _product_by_operations(syn, fodo_cell(), p, nsteps, turns, prop)
    b2 = syn.Bunch(ref, n, 1e11)
    b2.set_particles(p)
    prop.propagate(b2, turns)
    a, am, ad = b1.get_particles()
    c, cm, cd = b2.get_particles()
    assert np.array_equal(am, cm) and np.array_equal(ad, cd)
    assert np.array_equal(a, c, equal_nan=True)


def _build_shim(tmp_path):
    exe = str(tmp_path / "shim_driver")
    lib = os.path.join(ROOT, "synergia2_b200")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "shim_driver.cc"), "-L", lib, "-lsb2",
                    "-Wl,-rpath," + lib, "-o", exe], check=True)
    return exe


def test_shim_driver_compiles_against_the_c_abi(tmp_path):
    assert os.path.exists(_build_shim(tmp_path))


def _write(path, p, m):
    with open(path, "wb") as f:
        np.array([p.shape[0]], np.int64).tofile(f)
        np.asfortranarray(p).ravel(order="F").tofile(f)
        np.ascontiguousarray(m, np.uint8).tofile(f)


def _read(path):
    with open(path, "rb") as f:
        n = int(np.fromfile(f, np.int64, 1)[0])
        p = np.fromfile(f, np.float64, 7 * n).reshape((n, 7), order="F")
        m = np.fromfile(f, np.uint8, n)
        d = np.fromfile(f, np.uint8, n)
    return p, m, d


@pytest.mark.gpu
@pytest.mark.parametrize("lattice", ["fodo", "ring"])
def test_gpu_shim_driver_matches_oracle(tmp_path, orc, lattice):
    """A C++ caller shaped like the reference-side shims (tests/cxx/
    shim_driver.cc: LibFF_b200_operation and Aperture_operation bodies over
    the C ABI) against the oracle's stepper."""
    exe = _build_shim(tmp_path)
    n, nsteps, turns = 30000, 16, 2
    spec = fodo_cell() if lattice == "fodo" else ring_cell(radius=0.006)
    sig = SIG_C0 if lattice == "fodo" else SIG_RING
    p = _bunch_with_bad_particles(n, sig, 74)
    _write(str(tmp_path / "in.bin"), p, np.ones(n, np.uint8))
    r = subprocess.run([exe, lattice, str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), str(turns), str(nsteps)],
                       check=True, capture_output=True, text=True)
    gcounts = json.loads(r.stdout)["discards"]
    gp, gm, gd = _read(str(tmp_path / "out.bin"))
    sim = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT, num=nsteps, value=2.5 + MP)
    sim.set_particles(p)
    sim.propagate(turns)
    op, om, od = sim.get_particles()
    _compare(gp, gm, gd, op, om, od, exact=lattice == "fodo")
    assert sum(gcounts) == n - int(om.sum())
