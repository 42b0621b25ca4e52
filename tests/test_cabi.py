"""CPU tests of the C ABI: the library loads, exports every function that
include/sb2.h declares, and the host-side logic (options, slicing) works
without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from helpers import MP, ROOT, fodo_cell, oracle_lattice, product_lattice, ring_cell

HEADER = os.path.join(ROOT, "include", "sb2.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sb2_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "sb2_propagator_propagate" in names and "sb2_sc3d_apply" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(syn):
    L = syn.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_binding_covers_header(syn):
    from synergia2_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES), \
        set(declared_functions()) ^ set(_lib.SIGNATURES)


def test_options_defaults_mirror_reference(syn):
    """Space_charge_3d_open_hockney_options(gridx, gridy, gridz)
    (implemented_collective_options.h:81-95)."""
    o = syn.Space_charge_3d_open_hockney_options(32, 32, 64)
    assert o.shape == [32, 32, 64]
    assert o.doubled_shape == [64, 64, 128]
    assert o.green_fn == syn.green_fn_t.linear
    assert o.n_sigma == 8.0 and o.kick_scale == 1.0
    assert o.comm_group_size == 4 and o.domain_fixed == 0
    o.set_fixed_domain([0, 0, 0], [1e-3, 1e-3, 0.1])
    assert o.domain_fixed == 1 and o.size == [1e-3, 1e-3, 0.1]


def test_invalid_options_rejected_on_cpu(syn):
    lat, _ = product_lattice(fodo_cell())
    o = syn.Space_charge_3d_open_hockney_options(16, 16, 32)
    o.doubled_shape = [40, 32, 64]
    with pytest.raises(syn.SB2Error, match="doubled_shape"):
        syn.Propagator(lat, syn.Split_operator_stepper(o, 8))
    o = syn.Space_charge_3d_open_hockney_options(16, 16, 32)
    o.periodic_z = 1
    with pytest.raises(syn.SB2Error, match="periodic_z not yet implemented"):
        syn.Propagator(lat, syn.Split_operator_stepper(o, 8))


def _slices_equal(prop, sim, nsteps, nops):
    for k in range(nsteps):
        for op in range(nops):
            a = prop.step_slices(k, op)
            b = sim.step_slices(k, op)
            if a is None or b is None:
                assert a is None and b is None
                continue
            assert a.shape == b.shape, (k, op)
            assert np.array_equal(a, b), (k, op, a, b)


@pytest.mark.parametrize("num_steps", [1, 8, 13, 40])
def test_split_operator_slicing_matches_oracle_fodo(syn, orc, num_steps):
    """Split_operator_stepper slices (split_operator_stepper.cc:14-82),
    host logic only, against the oracle's restatement."""
    spec = fodo_cell()
    lat, _ = product_lattice(spec)
    o = syn.Space_charge_3d_open_hockney_options(8, 8, 8)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(o, num_steps))
    sim = orc.Sim(oracle_lattice(spec), 1, 1.0, stepper=orc.STEPPER_SPLIT, num=num_steps,
                  sc=orc.SCOptions.make(8, 8, 8), value=2.5 + MP)
    assert prop.num_steps() == sim.num_steps() == num_steps
    _slices_equal(prop, sim, num_steps, 2)


@pytest.mark.parametrize("stepper", ["split", "split_elements", "indep_elements"])
def test_ring_slicing_matches_oracle(syn, orc, stepper):
    spec = ring_cell()
    lat, _ = product_lattice(spec)
    o = syn.Space_charge_3d_open_hockney_options(8, 8, 8)
    if stepper == "split":
        st, kind, num = syn.Split_operator_stepper(o, 16), orc.STEPPER_SPLIT, 16
    elif stepper == "split_elements":
        st, kind, num = syn.Split_operator_stepper_elements(o, 3), orc.STEPPER_SPLIT_ELEMENTS, 3
    else:
        st, kind, num = syn.Independent_stepper_elements(2), orc.STEPPER_INDEP_ELEMENTS, 2
    prop = syn.Propagator(lat, st)
    sim = orc.Sim(oracle_lattice(spec), 1, 1.0, stepper=kind, num=num,
                  sc=orc.SCOptions.make(8, 8, 8) if stepper != "indep_elements" else None, value=2.5 + MP)
    assert prop.num_steps() == sim.num_steps()
    _slices_equal(prop, sim, prop.num_steps(), 2)


def test_lattice_length_and_errors(syn):
    lat, _ = product_lattice(ring_cell())
    assert abs(lat.get_length() - 8.0) < 1e-12
    bad = syn.Lattice("x")
    bad.append(syn.Lattice_element("drift", "d"))
    with pytest.raises(syn.SB2Error, match="no reference particle"):
        syn.Propagator(bad, syn.Independent_stepper_elements(1))
