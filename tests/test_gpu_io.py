"""Particle I/O and checkpoint/resume through the device-resident bunch:
Bunch::write_openpmd_file / read_openpmd_file, write_file / read_file,
syn::checkpoint_save / checkpoint_load (simulation/checkpoint.cc:18-140),
and the stream-ordered snapshot they read through."""
import numpy as np
import pytest

from helpers import MP, SIG_C0, elem, fodo_cell, gaussian_bunch, product_lattice, rel_l2, ring_cell

pytestmark = pytest.mark.gpu


def _fodo_prop(syn, sc_shape=None, steps=8):
    lat, ref = product_lattice(fodo_cell())
    opts = None if sc_shape is None else syn.Space_charge_3d_open_hockney_options(*sc_shape)
    return syn.Propagator(lat, syn.Split_operator_stepper(opts, steps)), ref


def _same_state(a, b):
    for f in ("design_set", "turns_done", "n_valid", "n_total", "real_num"):
        assert getattr(a, f) == getattr(b, f), f
    for r in ("ref", "design"):
        assert bytes(getattr(a, r)) == bytes(getattr(b, r)), r


def test_gpu_snapshot_matches_checkout(syn):
    """A snapshot taken while the bunch sits in its cell-ordered working copy
    (after a space-charge turn) holds the bunch at that point in the
    caller's order although a second turn is queued behind it at once, and
    the working copy stays in use (the next turn gives the same result as
    without a snapshot).  Two bunches run the same turns here, so their
    coordinates agree to the deposit's atomic-order rounding."""
    import torch
    n = 40000
    p = gaussian_bunch(n, SIG_C0, 31)
    prop, ref = _fodo_prop(syn, (16, 16, 32))
    a = syn.Bunch(ref, n, 1e11)
    b = syn.Bunch(ref, n, 1e11)
    a.set_particles(p)
    b.set_particles(p)
    s = torch.cuda.Stream()
    prop.propagate(a, 1, s.cuda_stream)
    prop.propagate(b, 1, s.cuda_stream)
    snap = a.snapshot(s.cuda_stream)
    prop.propagate(a, 1, s.cuda_stream)        # queued behind the snapshot
    sp, sm, sd, st = snap.wait()
    s.synchronize()
    bp, bm, bd = b.get_particles()             # b settled after one turn
    assert np.array_equal(sm, bm) and np.array_equal(sd, bd) and np.array_equal(sp[:, 6], bp[:, 6])
    for j in range(6):
        assert rel_l2(sp[:, j], bp[:, j]) <= 1e-13, j
    assert st.turns_done == 1 and st.n_valid == n
    prop.propagate(b, 1, s.cuda_stream)
    s.synchronize()
    ap, _, _ = a.get_particles()
    bp, _, _ = b.get_particles()
    for j in range(6):
        assert rel_l2(ap[:, j], bp[:, j]) <= 1e-13, j


def test_gpu_checkpoint_resume_exact_without_space_charge(syn, tmp_path):
    """Ring cell with apertures (losses), no collective operator: 2 turns,
    checkpoint, load, 2 more turns is bit-identical to 4 straight turns,
    particles, masks, discards, reference and design particles and counts."""
    n = 20000
    p = gaussian_bunch(n, [2e-3, 1e-4, 2e-3, 1e-4, 0.3, 1e-4], 32)
    lat, ref = product_lattice(ring_cell(radius=0.004))
    prop = syn.Propagator(lat, syn.Split_operator_stepper(None, 16))
    a = syn.Bunch(ref, n, 1e11)
    a.set_particles(p)
    prop.propagate(a, 4)
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 2)
    path = syn.checkpoint_save(prop, b, str(tmp_path))
    assert path.endswith("cp_state.json")
    prop2, c = syn.checkpoint_load(str(tmp_path))
    prop2.propagate(c, 2)
    ap, am, ad = a.get_particles()
    cp_, cm, cd = c.get_particles()
    assert 0 < int(am.sum()) < n
    assert np.array_equal(ap, cp_) and np.array_equal(am, cm) and np.array_equal(ad, cd)
    _same_state(a.get_state(), c.get_state())


def test_gpu_checkpoint_resume_with_space_charge(syn, tmp_path):
    """FODO with space charge: resumed turns agree with the uninterrupted run
    to 1e-12 (the deposit's atomic order differs with the particle order of
    the working copy); counts and reference particles exact."""
    n = 30000
    p = gaussian_bunch(n, SIG_C0, 33)
    prop, ref = _fodo_prop(syn, (16, 16, 32))
    a = syn.Bunch(ref, n, 1e11)
    a.set_particles(p)
    prop.propagate(a, 3)
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 1)
    syn.checkpoint_save(prop, b, str(tmp_path))
    prop2, c = syn.checkpoint_load(str(tmp_path))
    assert prop2.stepper.collective_options.shape == [16, 16, 32]
    prop2.propagate(c, 2)
    ap, am, _ = a.get_particles()
    cp_, cm, _ = c.get_particles()
    assert np.array_equal(am, cm) and np.array_equal(ap[:, 6], cp_[:, 6])
    for j in range(6):
        assert rel_l2(ap[:, j], cp_[:, j]) <= 1e-12, j
    _same_state(a.get_state(), c.get_state())


def test_gpu_checkpoint_async_while_propagating(syn, tmp_path):
    """wait=False: the files are written by a host thread while more turns
    are queued on the same stream; the checkpoint holds the state at the
    moment it was queued."""
    import torch
    n = 30000
    p = gaussian_bunch(n, SIG_C0, 34)
    prop, ref = _fodo_prop(syn, (16, 16, 32))
    s = torch.cuda.Stream()
    b = syn.Bunch(ref, n, 1e11)
    b.set_particles(p)
    prop.propagate(b, 1, s.cuda_stream)
    ref_p, ref_m, _ = b.get_particles()
    ref_state = b.get_state()
    pending = syn.checkpoint_save(prop, b, str(tmp_path), stream=s.cuda_stream, wait=False)
    prop.propagate(b, 2, s.cuda_stream)
    pending.join()
    s.synchronize()
    _, c = syn.checkpoint_load(str(tmp_path))
    cp_, cm, _ = c.get_particles()
    assert np.array_equal(cp_, ref_p) and np.array_equal(cm, ref_m)
    _same_state(c.get_state(), ref_state)
    assert b.get_state().turns_done == 3


def test_gpu_openpmd_and_npz_files(syn, tmp_path):
    """write_openpmd_file / read_openpmd_file and write_file / read_file
    through device bunches: coordinates, ids and masks come back exactly; the
    openPMD reader sets the bunch reference particle from gamma_ref."""
    n = 5000
    p = gaussian_bunch(n, SIG_C0, 35)
    prop, ref = _fodo_prop(syn)
    a = syn.Bunch(ref, n, 1e11)
    m = np.ones(n, np.uint8)
    m[::97] = 0
    a.set_particles(p, m)
    prop.propagate(a, 1)
    f = str(tmp_path / "bunch.json")
    a.write_openpmd_file(f)
    fm = syn.Four_momentum(MP)
    fm.set_total_energy(MP + 1.0)  # a different energy: the file's gamma_ref wins
    b = syn.Bunch(syn.Reference_particle(1, fm), n, 1e11)
    b.read_openpmd_file(f)
    ap, am, _ = a.get_particles()
    bp, bm, _ = b.get_particles()
    assert np.array_equal(ap, bp) and np.array_equal(am, bm)
    sa, sb = a.get_state(), b.get_state()
    assert sb.ref.gamma == sa.ref.gamma and abs(sb.ref.momentum - sa.ref.momentum) <= 1e-15 * sa.ref.momentum
    g = str(tmp_path / "bunch.npz")
    a.write_file(g)
    c = syn.Bunch(ref, n, 1e11)
    c.read_file(g)
    cp_, cm, _ = c.get_particles()
    assert np.array_equal(ap, cp_) and np.array_equal(am, cm)
    with pytest.raises(ValueError, match="HDF5"):
        a.write_file(str(tmp_path / "bunch.h5"))
