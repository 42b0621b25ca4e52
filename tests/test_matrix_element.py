"""MAD-X MATRIX element (FF_matrix, matrix_unit ff_algorithm.h:2439-2700) in
the oracle: the reference's simulation/tests/test_matrix_prop.py checks
that particles leave a matrix element as the linear map times their
coordinates (its booster one-turn map); here also the kicks and the
second-order tensor, against numpy."""
import numpy as np
import pytest

from helpers import MP, elem, oracle_lattice

BOOSTER = np.array([
    [-0.2360913935508699, -32.676028880719926, 0, 0, 0.00015078471867412094, 3.940712863966235],
    [0.02871519571777345, -0.26124972905688154, 0, 0, 6.410405557641018e-07, -0.09022913657323245],
    [0, 0, 0.36246234212348744, -4.883667648489127, 0, 0],
    [0, 0, 0.17702195094897383, 0.3737867616380023, 0, 0],
    [-0.1303165086379494, 5.56865106574654, 0, 0, 0.9967905427138485, 303.41542490997386],
    [2.1217926701948382e-07, 0.00023439092605032628, 0, 0, -4.660146993258213e-05, 0.9890119639891961]])


def matrix_attrs(rm, kick=None, tm=None):
    a = {"l": 0.0}
    for i in range(6):
        for j in range(6):
            if rm[i, j] != (1.0 if i == j else 0.0):
                a["rm%d%d" % (i + 1, j + 1)] = float(rm[i, j])
    if kick is not None:
        for i in range(6):
            a["kick%d" % (i + 1)] = float(kick[i])
    if tm is not None:
        for idx in zip(*np.nonzero(tm)):
            a["tm%d%d%d" % tuple(i + 1 for i in idx)] = float(tm[idx])
    return a


def ring_bunch():
    """8 particles on a transverse ring x 5 longitudinal positions."""
    p = []
    for cdt in (-0.2, -0.1, 0.0, 0.1, 0.2):
        for k in range(8):
            a = 2 * np.pi * k / 8
            p.append([1e-3 * np.cos(a), 0.0, 1e-3 * np.sin(a), 0.0, cdt, 1e-4 * cdt])
    out = np.zeros((len(p), 7), order="F")
    out[:, :6] = p
    out[:, 6] = np.arange(len(p))
    return out


def track(orc, attrs, p):
    spec = [elem("matrix", "m", **attrs)]
    sim = orc.Sim(oracle_lattice(spec, value=MP + 0.4), p.shape[0], 4e10, stepper=orc.STEPPER_INDEP_ELEMENTS, num=1,
                  value=MP + 0.4)
    sim.set_particles(p)
    sim.propagate(1)
    return sim.get_particles()[0], sim.design_state()[0]


def test_matrix_linear_booster_map(orc):
    p = ring_bunch()
    out, design = track(orc, matrix_attrs(BOOSTER), p)
    assert np.allclose(out[:, :6], p[:, :6] @ BOOSTER.T, rtol=1e-14, atol=1e-18)
    assert np.array_equal(design, np.zeros(6))


def test_matrix_kick_and_tensor(orc):
    g = np.random.default_rng(9)
    rm = np.eye(6) + 0.1 * g.standard_normal((6, 6))
    kick = 1e-4 * g.standard_normal(6)
    tm = np.zeros((6, 6, 6))
    tm[0, 0, 0], tm[1, 0, 2], tm[3, 2, 3], tm[4, 5, 5], tm[5, 1, 4] = 2.0, -3.0, 0.5, 10.0, 0.25
    p = ring_bunch()
    out, _ = track(orc, matrix_attrs(rm, kick, tm), p)
    v = p[:, :6]
    expect = kick + v @ rm.T + np.einsum("ijl,nj,nl->ni", tm, v, v)
    assert np.allclose(out[:, :6], expect, rtol=1e-13, atol=1e-18)


def test_matrix_length_is_an_error(orc):
    with pytest.raises(RuntimeError, match="non-zero length"):
        track(orc, {"l": 0.5, "rm12": 1.0}, ring_bunch())
