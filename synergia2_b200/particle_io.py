"""Particle files: the reference's Bunch::write_openpmd_file /
read_openpmd_file (bunch/bunch.cc:189-320, 466-600) and Bunch::write_file /
read_file (bunch/bunch.h:600-650, bunch_particles.cc:677-702).

openPMD.  The reference writes one openPMD series through openPMD-api, whose
backend follows the file extension; this module writes and reads the JSON
representation of that series (openPMD standard 1.1.0, the layout of
openPMD-api's JSON backend: groups as objects, attributes as
{"datatype", "value"} pairs under "attributes", datasets as
{"datatype", "data"}), with the reference's records:

  /data/<iteration>/particles/bunch_particles
      attributes mass [kg], beta_ref, gamma_ref
      position/{x, y, z} = x, y, cdt;  moments/{x, y, z} = xp, yp, dpop;  id
  /data/<iteration>/particles/bunch_particles_masks
      id = the uint8 masks

and the series attribute software = "synergia3", which is what the
reference's reader checks before it accepts a file.  JSON has no NaN or
infinity: non-finite coordinates (particles a Finite_aperture dropped) are
written as null and read back as NaN.

write_file / read_file.  The reference writes HDF5 datasets "particles"
(N x 7, row-major) and "particles_masks"; no HDF5 library is available to
this package, so the same two datasets go into a NumPy .npz archive.

All functions here work on host arrays (N x 7 particles, N masks); the
Bunch methods that call them take the arrays from the device with one
copy (Bunch.snapshot).
"""
import datetime
import json
import math

import numpy as np

C_LIGHT = 299792458.0
E_CHARGE = 1.602176565e-19
KG_TO_GEV = 1.0e-9 * C_LIGHT * C_LIGHT / E_CHARGE  # physical_constants.h:122

SOFTWARE = "synergia3"
SOFTWARE_VERSION = "synergia2_b200"
SPECIES = "bunch_particles"
MASK_SPECIES = "bunch_particles_masks"


def _attr(dtype, value):
    return {"datatype": dtype, "value": value}


def _finite_list(a):
    return [v if math.isfinite(v) else None for v in a.tolist()]


def _component(data, dtype="DOUBLE", unit_si=1.0):
    data = np.asarray(data)
    values = _finite_list(data.astype(np.float64)) if dtype == "DOUBLE" else data.astype(int).tolist()
    return {"attributes": {"unitSI": _attr("DOUBLE", unit_si)}, "datatype": dtype, "data": values}


def _record(components, unit_dimension):
    rec = {"attributes": {"timeOffset": _attr("FLOAT", 0.0), "unitDimension": _attr("ARR_DBL_7", unit_dimension)}}
    rec.update(components)
    return rec


def _scalar_record(data, dtype, unit_dimension):
    rec = _component(data, dtype)
    rec["attributes"]["timeOffset"] = _attr("FLOAT", 0.0)
    rec["attributes"]["unitDimension"] = _attr("ARR_DBL_7", unit_dimension)
    return rec


def write_openpmd_json(filename, parts, masks, mass_gev, beta_ref, gamma_ref, iteration=0, num_part=-1, offset=0):
    """Bunch::write_openpmd_file (bunch.cc:466-600) for a JSON series.
    num_part = -1 writes all particles; otherwise rows offset..offset+num_part."""
    parts = np.asarray(parts, dtype=np.float64)
    masks = np.asarray(masks, dtype=np.uint8)
    n = parts.shape[0]
    if num_part == -1:
        lo, hi = 0, n
    else:
        lo, hi = int(offset), int(offset) + int(num_part)
        if num_part < 0 or offset < 0 or hi > n:
            raise ValueError("invalid num_part or offset for write_openpmd_file")
    p, m = parts[lo:hi], masks[lo:hi]
    length = [1.0, 0, 0, 0, 0, 0, 0]
    none = [0.0] * 7
    species = {
        "attributes": {"mass": _attr("DOUBLE", mass_gev / KG_TO_GEV), "beta_ref": _attr("DOUBLE", float(beta_ref)),
                       "gamma_ref": _attr("DOUBLE", float(gamma_ref))},
        "position": _record({"x": _component(p[:, 0]), "y": _component(p[:, 2]), "z": _component(p[:, 4])}, length),
        "moments": _record({"x": _component(p[:, 1]), "y": _component(p[:, 3]), "z": _component(p[:, 5])}, none),
        "id": _scalar_record(p[:, 6], "DOUBLE", none),
    }
    mask_species = {"attributes": {}, "id": _scalar_record(m, "UCHAR", none)}
    series = {
        "attributes": {
            "basePath": _attr("STRING", "/data/%T/"),
            "date": _attr("STRING", datetime.datetime.now().astimezone().strftime("%Y-%m-%d %H:%M:%S %z")),
            "iterationEncoding": _attr("STRING", "groupBased"),
            "iterationFormat": _attr("STRING", "/data/%T/"),
            "meshesPath": _attr("STRING", "meshes/"),
            "openPMD": _attr("STRING", "1.1.0"),
            "openPMDextension": _attr("UINT", 0),
            "particlesPath": _attr("STRING", "particles/"),
            "software": _attr("STRING", SOFTWARE),
            "softwareVersion": _attr("STRING", SOFTWARE_VERSION),
        },
        "data": {
            str(int(iteration)): {
                "attributes": {"dt": _attr("DOUBLE", 1.0), "time": _attr("DOUBLE", 0.0),
                               "timeUnitSI": _attr("DOUBLE", 1.0)},
                "particles": {SPECIES: species, MASK_SPECIES: mask_species},
            }
        },
    }
    with open(filename, "w") as f:
        json.dump(series, f, allow_nan=False)


def _values(ds):
    return np.array([np.nan if v is None else v for v in ds["data"]], dtype=np.float64)


def read_openpmd_json(filename, iteration=None):
    """Bunch::read_openpmd_file (bunch.cc:189-320) for a JSON series written
    by synergia3: the last iteration unless `iteration` is given.  Returns
    (parts N x 7, masks N, mass [GeV], beta_ref, gamma_ref)."""
    with open(filename) as f:
        series = json.load(f)
    attrs = series.get("attributes", {})
    software = attrs.get("software", {}).get("value")
    if software is None:
        raise ValueError("Could not determine which software generated the input")
    if software != SOFTWARE:
        raise ValueError("openPMD input written by %r: only synergia3 series are read" % software)
    its = series["data"]
    key = str(iteration) if iteration is not None else max(its, key=int)
    parts_grp = its[key]["particles"]
    sp = parts_grp[SPECIES]
    ids = _values(sp["id"])
    n = len(ids)
    parts = np.zeros((n, 7), order="F")
    for col, (rec, comp) in enumerate([("position", "x"), ("moments", "x"), ("position", "y"), ("moments", "y"),
                                       ("position", "z"), ("moments", "z")]):
        parts[:, col] = _values(sp[rec][comp])
    parts[:, 6] = ids
    masks = np.array(parts_grp[MASK_SPECIES]["id"]["data"], dtype=np.uint8) if MASK_SPECIES in parts_grp \
        else np.ones(n, np.uint8)
    mass = sp["attributes"]["mass"]["value"] * KG_TO_GEV
    return parts, masks, mass, sp["attributes"]["beta_ref"]["value"], sp["attributes"]["gamma_ref"]["value"]


def write_npz(filename, parts, masks, num_part=-1, offset=0):
    """Bunch::write_file (bunch_particles.cc:677-702): datasets "particles"
    (rows offset..offset+num_part, N x 7 row-major) and "particles_masks"."""
    parts = np.asarray(parts, dtype=np.float64)
    masks = np.asarray(masks, dtype=np.uint8)
    n = parts.shape[0]
    if num_part == -1:
        lo, hi = 0, n
    else:
        lo, hi = int(offset), int(offset) + int(num_part)
        if num_part < 0 or offset < 0 or hi > n:
            raise ValueError("invalid num_part or offset for bunch_particles_t::write_file()")
    np.savez(filename, particles=np.ascontiguousarray(parts[lo:hi]), particles_masks=masks[lo:hi])


def read_npz(filename):
    """Bunch::read_file: (parts N x 7, masks N)."""
    with np.load(filename) as z:
        return np.asfortranarray(z["particles"]), np.array(z["particles_masks"], dtype=np.uint8)


def check_extension(filename, allowed):
    low = filename.lower()
    if low.endswith((".h5", ".hdf5")):
        raise ValueError("HDF5 is not available to this package: write %s instead" % " or ".join(allowed))
    if not low.endswith(allowed):
        raise ValueError("unsupported particle file %r (expected %s)" % (filename, ", ".join(allowed)))
