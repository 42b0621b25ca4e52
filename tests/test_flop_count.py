"""The oracle's operation counting (orc_flops_*): algorithmic FP64 work per
macroparticle, counted by running the oracle's own particle code on a
counting scalar.  The FP64 roofline of the particle passes divides these
counts by measured launch times."""
import json
import os
import sys

import numpy as np
import pytest

from helpers import MP, ROOT, elem, fodo_cell, gaussian_bunch, oracle_lattice

SIG = [1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4]


def _sim(orc, spec, n=512, sc=None, num=1, seed=3):
    p = gaussian_bunch(n, SIG, seed)
    sim = orc.Sim(oracle_lattice(spec), n, 1e11, stepper=orc.STEPPER_SPLIT, num=num, sc=sc, value=2.5 + MP)
    sim.set_particles(p)
    return sim


def test_drift_unit_count(orc):
    """drift_unit (ff_algorithm.h:47-79) by hand: 1 + 4 adds for the
    longitudinal momentum, 2 for x and y, 2 for D2, 1 for E2, 2 for cdt (10);
    3 squares, 4 products for the slopes, 3 for D2, 1 for p, 2 for E2, 1 for
    p^2, 2 for cdt (16); 2 divisions; 2 square roots.  Every half step ends
    with a finite (1 add, 3 mul, 2 sub) and a circular aperture (2 sub,
    2 mul, 1 add)."""
    sim = _sim(orc, [elem("drift", "d", l=1.0)])
    recs = sim.count_flops(0, 0, 1)
    assert [r[1] for r in recs] == ["I", "I"]  # no collective operator
    first = recs[0][2]
    assert first["drift"] == {"add": 10, "mul": 16, "div": 2, "sqrt": 2, "fn": 0}
    assert first["aperture"] == {"add": 6, "mul": 5, "div": 0, "sqrt": 0, "fn": 0}


def test_yoshida_quadrupole_count(orc):
    """A thick quadrupole slice: yoshida6 with 4 steps of 10 drift units and
    9 thin quadrupole kicks (8 flops each), plus the offset subtractions and
    additions of the particle loop."""
    sim = _sim(orc, [elem("quadrupole", "q", l=0.5, k1=0.6)])
    first = sim.count_flops(0, 0, 1)[0][2]
    quad = sum(first["quadrupole"].values())
    assert quad == 4 * (10 * 30 + 9 * 8) + 4
    assert first["quadrupole"]["div"] == 4 * 10 * 2 and first["quadrupole"]["sqrt"] == 4 * 10 * 2


def test_counting_leaves_results_unchanged(orc):
    """The counted body runs on copies: a FODO cell with space charge gives
    bit-identical particles with and without counting."""
    sc = orc.SCOptions.make(16, 16, 32)
    a = _sim(orc, fodo_cell(), n=3000, sc=sc, num=8)
    b = _sim(orc, fodo_cell(), n=3000, sc=sc, num=8)
    a.propagate_steps(0, 8)
    recs = b.count_flops(17, 0, 8)
    assert len(recs) == 24
    pa, ma, _ = a.get_particles()
    pb, mb, _ = b.get_particles()
    assert np.array_equal(pa, pb) and np.array_equal(ma, mb)
    kick = recs[1][2]
    assert sum(kick["sc_kick"].values()) == 128 and sum(kick["sc_domain"].values()) == 9
    assert sum(kick["sc_deposit"].values()) == 56


def test_uninstrumented_element_raises(orc):
    sim = _sim(orc, [elem("solenoid", "s", l=0.5, ks=0.3)])
    with pytest.raises(RuntimeError, match="instrumented"):
        sim.count_flops(0, 0, 1)


def test_committed_table_matches_oracle(orc):
    """profiles/fp64_flops_per_particle.json is what oracle/count_flops.py
    computes now."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import count_flops as cf
    finally:
        sys.path.pop(0)
    table = json.load(open(cf.OUT))
    for name, spec in cf.WORKLOADS.items():
        _, steps = cf.count_workload(spec)
        passes = cf.passes_of(steps)
        got = table["workloads"][name]
        assert [p["flops"] for p in passes] == [p["flops"] for p in got["passes"]]
        assert [p["variant"] for p in passes] == [p["variant"] for p in got["passes"]]
    c1 = table["workloads"]["fodo_c1"]
    assert (c1["light_passes"], c1["full_passes"]) == (6, 2)
