"""Dipole edge (FF_dipedge, dipedge_unit ff_algorithm.h:1284-1316 after MAD-X
tmfrng) in the oracle: the known answer of the reference's
libFF/tests/print_dipedge_map.py (MAD-X R43 of dipedge e1 = 0,
h = 1.216203238, hgap = 0.029, fint = 0.5 at E = mp + 2.5 MeV) and the
second-order terms against a numpy restatement."""
import math

import numpy as np
import pytest

from helpers import MP, elem, oracle_lattice

MADX_R43 = 0.04291315480354536  # print_dipedge_map.py, from MAD-X's map of print_dipedge_map.madx


def _track(orc, attrs, p, value=MP + 0.0025):
    spec = [elem("dipedge", "dedge30", **attrs)]
    n = p.shape[0]
    sim = orc.Sim(oracle_lattice(spec, value=value), n, 1e10, stepper=orc.STEPPER_INDEP_ELEMENTS, num=1, value=value)
    sim.set_particles(p)
    sim.propagate(1)
    return sim.get_particles()[0]


def test_dipedge_madx_r43(orc):
    p = np.zeros((3, 7), order="F")
    p[:, 2] = [1e-6, -2e-6, 3e-7]
    p[:, 6] = np.arange(3)
    out = _track(orc, dict(l=0.0, e1=0.0, h=1.216203238, hgap=0.029, fint=0.5), p)
    assert np.allclose(out[:, 3] / p[:, 2], MADX_R43, rtol=1e-12, atol=0)
    assert np.array_equal(out[:, 2], p[:, 2]) and np.all(out[:, [0, 1, 4, 5]] == 0)


def test_dipedge_second_order(orc):
    e1, h, hgap, fint = 0.12, 0.8, 0.03, 0.4
    g = np.random.default_rng(8)
    n = 50
    p = np.zeros((n, 7), order="F")
    for j, s in zip(range(4), (2e-3, 2e-4, 2e-3, 2e-4)):
        p[:, j] = g.standard_normal(n) * s
    p[:, 6] = np.arange(n)
    out = _track(orc, dict(l=0.0, e1=e1, h=h, hgap=hgap, fint=fint, second_order=1.0), p)
    corr = 2 * h * hgap * fint
    t, sec, sn = math.tan(e1), 1 / math.cos(e1), math.sin(e1)
    re21, re43 = h * t, -h * math.tan(e1 - corr * sec * (1 + sn * sn))
    hh = h / 2
    te = [-hh * t * t, hh * sec * sec, 0.0, hh * t * t, 0.0, -hh * t * t, hh * t * t, 0.0, -hh * t * t, -hh * sec * sec]
    te[4] = hh * h * t ** 3 + (h * sec) ** 2 * (t / 2)
    x, xp, y, yp = p[:, 0], p[:, 1], p[:, 2], p[:, 3]
    ex = x + te[0] * x * x + te[1] * y * y
    exp_ = xp + re21 * x + te[2] * x * x + te[4] * y * y + 2 * te[3] * x * xp + 2 * te[5] * y * yp
    ey = y + 2 * te[6] * x * y
    eyp = yp + re43 * y + 2 * te[7] * x * y + 2 * te[8] * x * yp + 2 * te[9] * y * xp
    for j, e in zip(range(4), (ex, exp_, ey, eyp)):
        assert np.allclose(out[:, j], e, rtol=1e-13, atol=1e-19), j
