"""Thin nonlinear lens (FF_nllens, nllens_unit ff_algorithm.h:1180-1270).

The reference's only data for this element, track_nllensone.npy (copied to
tests/golden/nllens_track.json), holds the analytic Danilov-Nagaitsev kick:
with z = (x + i y)/cnll, the angles change by -knll/cnll (Re, -Im) of
z/(1 - z^2) + asin(z)/(1 - z^2)^(3/2) on the principal branch.  The
reference's nllens_unit computes asin(z)/(1 - z^2) with a square root of
1 - z^2 whose imaginary part is never negative, which moves these angles by
up to 17%; no reference test reads the file.  The oracle and the GPU path
follow the reference's arithmetic; these tests pin that against an
independent numpy restatement, and record what the file holds."""
import cmath
import json
import math
import os

import numpy as np
import pytest

from helpers import MP, ROOT, elem, oracle_lattice

G = json.load(open(os.path.join(ROOT, "tests", "golden", "nllens_track.json")))
KNLL, CNLL = G["knll"], G["cnll"]


def live_kick(x, y):
    """The reference's arithmetic, restated with Python complex numbers."""
    z = complex(x / CNLL, y / CNLL)
    c = 1 - z * z
    root = complex(math.sqrt(0.5 * (c.real + abs(c))), math.sqrt(0.5 * (-c.real + abs(c))))
    co = 1j * z + root
    theta = math.atan(co.imag / co.real) + (0.0 if co.real > 0 else math.pi)
    df = z / (root * root) + complex(theta, -math.log(abs(co))) / (root * root)
    k = -KNLL / CNLL
    return k * df.real, -k * df.imag


def analytic_kick(x, y):
    z = complex(x / CNLL, y / CNLL)
    root = cmath.sqrt(1 - z * z)
    df = z / (root * root) + (-1j * cmath.log(1j * z + root)) / root ** 3
    k = -KNLL / CNLL
    return k * df.real, -k * df.imag


def channel():
    d = G["drift"]
    return [elem("drift", "d1", l=d), elem("nllens", "nll", l=0.0, knll=KNLL, cnll=CNLL), elem("drift", "d2", l=d)]


def test_golden_file_is_the_analytic_kick():
    init, fin = np.array(G["initial"]), np.array(G["final"])
    for r0, r1 in zip(init, fin):
        dxp, dyp = analytic_kick(r0[0], r0[2])
        assert abs(dxp - r1[1]) <= 1e-18 and abs(dyp - r1[3]) <= 1e-18
    worst = max(abs(live_kick(r[0], r[2])[0] - f[1]) / abs(f[1]) for r, f in zip(init, fin) if f[1] != 0)
    assert worst > 0.05  # the reference's arithmetic is not what the file holds


def test_oracle_nllens_follows_the_reference_arithmetic(orc):
    init = np.array(G["initial"])
    g = np.random.default_rng(5)
    extra = np.column_stack([g.uniform(-6e-3, 6e-3, 64), np.zeros(64), g.uniform(-6e-3, 6e-3, 64)])
    pts = np.vstack([init[:, [0, 1, 2]], extra])
    n = pts.shape[0]
    p = np.zeros((n, 7), order="F")
    p[:, 0], p[:, 2], p[:, 6] = pts[:, 0], pts[:, 2], np.arange(n)
    sim = orc.Sim(oracle_lattice(channel(), value=MP + 2.5), n, 1e10, stepper=orc.STEPPER_INDEP_ELEMENTS, num=1,
                  value=MP + 2.5)
    sim.set_particles(p)
    sim.propagate(1)
    out = sim.get_particles()[0]
    # Python's complex division and abs() round differently from the
    # reference's real arithmetic (~1e-12); the two formulas differ by 17%
    for i in range(n):
        dxp, dyp = live_kick(p[i, 0], p[i, 2])
        assert out[i, 1] == pytest.approx(dxp, rel=1e-9, abs=1e-20)
        assert out[i, 3] == pytest.approx(dyp, rel=1e-9, abs=1e-20)
    # the drifts move x, y by xp * 0.5 um only
    assert np.max(np.abs(out[:, 0] - p[:, 0])) < 1e-9


def test_oracle_nllens_errors(orc):
    with pytest.raises(RuntimeError, match="non-zero length"):
        spec = [elem("nllens", "nll", l=0.1, knll=KNLL, cnll=CNLL)]
        orc.Sim(oracle_lattice(spec), 4, 1e10, stepper=orc.STEPPER_INDEP_ELEMENTS, num=1,
                value=MP + 2.5).propagate(1)
