"""Shared test helpers: lattice specifications of the benchmark configurations,
seeded synthetic bunches, and builders that turn one specification into the
product's objects and the oracle's."""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

MP = 0.938272046
KINETIC = 2.5  # GeV, proton bunches of the FODO / ring configurations
REAL_NUM = 1e11


def elem(etype, name, **attrs):
    d = {"type": etype, "name": name, "double": {}, "string": {}, "vector": {}}
    for k, v in attrs.items():
        if isinstance(v, str):
            d["string"][k] = v
        elif isinstance(v, (list, tuple)):
            d["vector"][k] = list(v)
        else:
            d["double"][k] = float(v)
    return d


def fodo_cell(k1=0.6):
    """QF L=0.5 k1=+k1, drift 4.5, QD L=0.5 k1=-k1, drift 4.5 (10 m)."""
    return [elem("quadrupole", "qf", l=0.5, k1=k1), elem("drift", "d1", l=4.5),
            elem("quadrupole", "qd", l=0.5, k1=-k1), elem("drift", "d2", l=4.5)]


def ring_cell(k1=0.55, k2l=0.2, radius=0.05, ncells=24):
    """One cell of the 24-cell ring: QF 0.5, SF thin, D 0.75, B 2.0, D 0.75,
    QD 0.5, SD thin, D 0.75, B 2.0, D 0.75 = 8.0 m; two sector bends of
    2 pi / (2 * ncells); circular aperture radius on every element."""
    ang = 2 * math.pi / (2 * ncells)
    r = dict(circular_aperture_radius=radius)
    return [elem("quadrupole", "qf", l=0.5, k1=k1, **r), elem("sextupole", "sf", l=0.0, k2=k2l, **r),
            elem("drift", "d1", l=0.75, **r), elem("sbend", "b1", l=2.0, angle=ang, **r),
            elem("drift", "d2", l=0.75, **r), elem("quadrupole", "qd", l=0.5, k1=-k1, **r),
            elem("sextupole", "sd", l=0.0, k2=-k2l, **r), elem("drift", "d3", l=0.75, **r),
            elem("sbend", "b2", l=2.0, angle=ang, **r), elem("drift", "d4", l=0.75, **r)]


def gaussian_bunch(n, sigmas, seed):
    """Seeded 6D uncorrelated Gaussian (numpy Philox), ids 0..n-1."""
    g = np.random.Generator(np.random.Philox(seed))
    p = np.zeros((n, 7), order="F")
    for j in range(6):
        p[:, j] = g.standard_normal(n) * sigmas[j]
    p[:, 6] = np.arange(n)
    return p


SIG_C0 = [1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4]


def product_lattice(spec, value=KINETIC + MP, kind=0, name="lattice"):
    import synergia2_b200 as syn
    fm = syn.Four_momentum(MP)
    if kind == 0:
        fm.set_total_energy(value)
    elif kind == 1:
        fm.set_momentum(value)
    else:
        fm.set_kinetic_energy(value)
    ref = syn.Reference_particle(1, fm)
    lat = syn.Lattice(name)
    for e in spec:
        le = syn.Lattice_element(e["type"], e["name"])
        for k, v in e.get("double", {}).items():
            le.set_double_attribute(k, v)
        for k, v in e.get("string", {}).items():
            le.set_string_attribute(k, v)
        for k, v in e.get("vector", {}).items():
            le.set_vector_attribute(k, v)
        lat.append(le)
    lat.set_reference_particle(ref)
    return lat, ref


def oracle_lattice(spec, value=KINETIC + MP, kind=0):
    from oracle import oracle as O
    return O.Lattice(spec, value=value, kind=kind)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
