"""Sector bends at a momentum other than the design one, against the
closed-form circle (restating the physics checks of the reference's
simulation/tests/test_higher_momentum_bend.py and
test_rfcavity_plus_cfbend.py): a particle on the design orbit entering a
bend of radius R0 = L / angle with momentum p follows a circle of radius
R = R0 p / p0, so at the exit x = R0 (sqrt(2 R / R0 - 1) - 1) and its path
time differs by R acos((R - R0) / R) / beta - L / beta0.  The GPU path also
agrees with the oracle."""
import math

import numpy as np
import pytest

from helpers import MP, elem, oracle_lattice, product_lattice

pytestmark = pytest.mark.gpu


def _circle(p0, p, beta0, beta, length=math.pi / 2, angle=math.pi / 2):
    r0 = length / angle
    r = r0 * p / p0
    x = r0 * (math.sqrt(2 * (r / r0) - 1)) - r0
    dct = r * math.acos((r - r0) / r) / beta - length / beta0
    return x, dct


def _run(syn, orc, spec, lat_value, lat_kind, bunch_value, bunch_kind):
    lat, _ = product_lattice(spec, value=lat_value, kind=lat_kind)
    fm = syn.Four_momentum(MP)
    if bunch_kind == 0:
        fm.set_total_energy(bunch_value)
    else:
        fm.set_momentum(bunch_value)
    prop = syn.Propagator(lat, syn.Independent_stepper_elements(1))
    b = syn.Bunch(syn.Reference_particle(1, fm), 16, 4.0e10)
    p = np.zeros((16, 7), order="F")
    p[:, 6] = np.arange(16)
    b.set_particles(p)
    prop.propagate(b, 1)
    gp = b.get_particles()[0]
    sim = orc.Sim(oracle_lattice(spec, value=lat_value, kind=lat_kind), 16, 4.0e10, stepper=orc.STEPPER_INDEP_ELEMENTS,
                  num=1, value=bunch_value, kind=bunch_kind)
    sim.set_particles(p)
    sim.propagate(1)
    op = sim.get_particles()[0]
    scale = np.maximum(np.max(np.abs(op[:, :6]), axis=0), 1e-300)
    # x and cdt are differences of O(1) quantities (the circle): last-bit
    # differences of CUDA's asin/sin/cos show at ~1e-12 of these 1e-4 offsets
    assert np.all(np.abs(gp[:, :6] - op[:, :6]) <= 1e-10 * scale)
    return gp, b.get_state()


@pytest.mark.parametrize("k1,tol", [(None, 1e-9), (1e-20, 1e-9), (3.2e-6, 2.5e-6)])
def test_gpu_bend_at_higher_momentum(syn, orc, k1, tol):
    """test_higher_momentum_bend.py: the bunch 0.1 MeV above the lattice
    energy through an angle = L = pi/2 bend.  The pure dipole and the
    combined-function integrator with a negligible k1 follow the circle to
    1e-9; k1 = 3.2e-6 bends the orbit by ~2e-6 of the offsets."""
    attrs = dict(l=math.pi / 2, angle=math.pi / 2)
    if k1 is not None:
        attrs["k1"] = k1
    e0 = MP + 0.8
    gp, st = _run(syn, orc, [elem("sbend", "b", **attrs)], e0, 0, e0 + 0.0001, 0)
    x, dct = _circle(st.design.momentum, st.ref.momentum, st.design.beta, st.ref.beta)
    assert gp[0, 5] == 0.0
    assert gp[0, 0] == pytest.approx(x, rel=tol)
    assert gp[0, 4] == pytest.approx(dct, rel=tol)


def test_gpu_rfcavity_then_cf_bend(syn, orc):
    """test_rfcavity_plus_cfbend.py: a thin rf cavity (0.2 MV, lag 1/12)
    raises the bunch energy by 0.2e-3 sin(pi/6) GeV, then a combined-
    function bend (k1 = 3.2e-6) takes the particle on the larger circle;
    energy, x and path time within the reference's 1e-6."""
    p0 = 0.75 * MP
    spec = [elem("rfcavity", "rfc", l=0.0, volt=0.2, harmon=1.0, lag=1.0 / 12.0),
            elem("sbend", "b", l=math.pi / 2, angle=math.pi / 2, k1=3.2e-6)]
    gp, st = _run(syn, orc, spec, p0, 1, p0, 1)
    e_old = math.sqrt(p0 * p0 + MP * MP)
    assert st.ref.energy - e_old == pytest.approx(0.0002 * math.sin(math.pi / 6), rel=1e-6)
    assert gp[0, 5] == 0.0
    x, dct = _circle(p0, st.ref.momentum, st.design.beta, st.ref.beta)
    assert gp[0, 0] == pytest.approx(x, rel=1e-6)
    assert gp[0, 4] == pytest.approx(dct, rel=1e-6)
