"""Particle files and checkpoint serialisation on the host (no GPU):
Bunch::write_openpmd_file / read_openpmd_file (bunch/bunch.cc:189-600) as an
openPMD JSON series, Bunch::write_file / read_file (bunch_particles.cc:
677-702) as .npz, and the checkpoint's state round trips."""
import json
import math

import numpy as np
import pytest

from synergia2_b200 import _lib, particle_io
from synergia2_b200 import checkpoint as cp

from helpers import MP, gaussian_bunch


def _bunch(n=257, seed=3):
    p = gaussian_bunch(n, [1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4], seed)
    m = np.ones(n, np.uint8)
    m[[3, n // 3, n - 2]] = 0
    p[n // 3, 1] = np.nan  # particles a Finite_aperture dropped
    p[n - 2, 0] = np.inf
    return p, m


def test_openpmd_json_round_trip(tmp_path):
    p, m = _bunch()
    f = str(tmp_path / "b.json")
    g = 3.664472432
    beta = math.sqrt(1 - 1 / g ** 2)
    particle_io.write_openpmd_json(f, p, m, MP, beta, g)
    q, mq, mass, b2, g2 = particle_io.read_openpmd_json(f)
    finite = np.isfinite(p)
    assert np.array_equal(q[finite], p[finite])            # doubles survive the text form exactly
    assert np.all(np.isnan(q[~finite]))                    # non-finite values come back as NaN
    assert np.array_equal(mq, m)
    assert abs(mass - MP) <= 1e-15 * MP and b2 == beta and g2 == g


def test_openpmd_json_layout(tmp_path):
    """The records and attributes the reference's reader looks up
    (bunch.cc:201-300): software synergia3, species bunch_particles with
    mass [kg], beta_ref, gamma_ref, position/moments x y z and id, masks as
    species bunch_particles_masks; strict JSON (no NaN tokens)."""
    p, m = _bunch(20)
    f = str(tmp_path / "b.json")
    particle_io.write_openpmd_json(f, p, m, MP, 0.9, 2.3, iteration=4)
    text = open(f).read()
    doc = json.loads(text, parse_constant=lambda c: pytest.fail("non-JSON constant " + c))
    assert doc["attributes"]["software"]["value"] == "synergia3"
    assert doc["attributes"]["openPMD"]["value"] == "1.1.0"
    assert doc["attributes"]["basePath"]["value"] == "/data/%T/"
    sp = doc["data"]["4"]["particles"]["bunch_particles"]
    assert abs(sp["attributes"]["mass"]["value"] * particle_io.KG_TO_GEV - MP) < 1e-15
    for rec in ("position", "moments"):
        for c in "xyz":
            comp = sp[rec][c]
            assert comp["datatype"] == "DOUBLE" and len(comp["data"]) == 20
            assert comp["attributes"]["unitSI"]["value"] == 1.0
        assert len(sp[rec]["attributes"]["unitDimension"]["value"]) == 7
    assert sp["position"]["z"]["data"][5] == p[5, 4]       # z is cdt
    assert sp["moments"]["z"]["data"][5] == p[5, 5]        # moments z is dpop
    assert sp["id"]["data"] == list(p[:, 6])
    mk = doc["data"]["4"]["particles"]["bunch_particles_masks"]["id"]
    assert mk["datatype"] == "UCHAR" and mk["data"] == list(m)


def test_openpmd_partial_and_last_iteration(tmp_path):
    p, m = _bunch(50)
    f = str(tmp_path / "b.json")
    particle_io.write_openpmd_json(f, p, m, MP, 0.9, 2.3, num_part=10, offset=5)
    q, mq, *_ = particle_io.read_openpmd_json(f)
    assert q.shape == (10, 7) and np.array_equal(q[:, 6], p[5:15, 6])
    with pytest.raises(ValueError):
        particle_io.write_openpmd_json(f, p, m, MP, 0.9, 2.3, num_part=10, offset=45)
    # a series with two iterations reads the last one, as the reference does
    doc = json.load(open(f))
    doc["data"]["7"] = json.loads(json.dumps(doc["data"]["0"]))
    doc["data"]["7"]["particles"]["bunch_particles"]["id"]["data"] = [float(i) for i in range(100, 110)]
    json.dump(doc, open(f, "w"))
    q, *_ = particle_io.read_openpmd_json(f)
    assert q[0, 6] == 100.0
    q, *_ = particle_io.read_openpmd_json(f, iteration=0)
    assert q[0, 6] == p[5, 6]


def test_openpmd_rejects_other_software(tmp_path):
    p, m = _bunch(5)
    f = str(tmp_path / "b.json")
    particle_io.write_openpmd_json(f, p, m, MP, 0.9, 2.3)
    doc = json.load(open(f))
    doc["attributes"]["software"]["value"] = "someone-else"
    json.dump(doc, open(f, "w"))
    with pytest.raises(ValueError, match="synergia3"):
        particle_io.read_openpmd_json(f)


def test_npz_round_trip_and_extensions(tmp_path):
    p, m = _bunch(64)
    f = str(tmp_path / "b.npz")
    particle_io.write_npz(f, p, m)
    q, mq = particle_io.read_npz(f)
    assert np.array_equal(q, p, equal_nan=True) and np.array_equal(mq, m)
    with np.load(f) as z:
        assert set(z.files) == {"particles", "particles_masks"} and z["particles"].flags["C_CONTIGUOUS"]
    with pytest.raises(ValueError, match="HDF5"):
        particle_io.check_extension("x.h5", (".npz",))
    with pytest.raises(ValueError):
        particle_io.check_extension("x.txt", (".npz",))


def test_bunch_state_struct_round_trip():
    st = _lib.sb2_bunch_state()
    st.ref.charge, st.ref.mass, st.ref.gamma = 1, MP, 3.5
    st.ref.state[4] = 0.25
    st.design.s_n = 7.5
    st.turns_done, st.n_valid, st.n_total, st.real_num = 4, 99, 100, 1e11
    d = json.loads(json.dumps(cp._struct_to_dict(st)))
    back = cp._dict_to_struct(d, _lib.sb2_bunch_state())
    assert bytes(back) == bytes(st)


def test_sc_options_round_trip():
    import synergia2_b200 as syn
    o = syn.Space_charge_3d_open_hockney_options(16, 32, 64)
    o.n_sigma = 6.5
    o.precision = syn.precision_t.mixed
    d = json.loads(json.dumps(cp._struct_to_dict(o._o)))
    o2 = syn.Space_charge_3d_open_hockney_options(*d["shape"])
    cp._dict_to_struct(d, o2._o)
    assert bytes(o2._o) == bytes(o._o)
