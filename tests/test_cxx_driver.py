"""A C++ caller of the C ABI (tests/cxx/fodo_driver.cc, the shape of the
reference's examples/fodo_cxx driver): it compiles and links against
include/sb2.h and libsb2.so (CPU), and on a GPU its result agrees with the
same run through the Python mirror."""
import json
import os
import subprocess

import numpy as np
import pytest

from helpers import ROOT, fodo_cell, product_lattice

SRC = os.path.join(ROOT, "tests", "cxx", "fodo_driver.cc")
LIBDIR = os.path.join(ROOT, "synergia2_b200")


def _build(tmp_path):
    exe = str(tmp_path / "fodo_driver")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lsb2", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def test_cxx_driver_compiles_against_the_c_abi(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_cxx_driver_matches_python_mirror(tmp_path, syn, mixed):
    exe = _build(tmp_path)
    n, turns = 200000, 2
    args = [exe, str(n), str(turns)] + (["mixed"] if mixed else [])
    out = json.loads(subprocess.run(args, check=True, capture_output=True, text=True).stdout)
    lat, ref = product_lattice(fodo_cell(), value=2.5, kind=2)
    opts = syn.Space_charge_3d_open_hockney_options(32, 32, 64)
    if mixed:
        opts.precision = syn.precision_t.mixed
    prop = syn.Propagator(lat, syn.Split_operator_stepper(opts, 8))
    b = syn.Bunch(ref, n, 1e11)
    b.populate_gaussian([1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4], 1)
    prop.propagate(b, turns)
    mean, mom2, emit = b.moments()
    assert out["total_num"] == b.get_total_num()
    sd = np.sqrt(np.diag(mom2))
    # run to run, only the deposit's summation order differs: FP64 sums in
    # the drop-in, an FP32 charge grid (merged from neighbouring tiles in any
    # order) in mixed precision
    tol = 1e-8 if mixed else 1e-12
    assert np.all(np.abs(np.array(out["mean"]) - mean) <= tol * sd)
    assert np.allclose(out["emit"], emit, rtol=1e-7 if mixed else 1e-9, atol=0)
