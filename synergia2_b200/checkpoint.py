"""Checkpoint and resume: syn::checkpoint_save / checkpoint_load / resume
(simulation/checkpoint.h, checkpoint.cc:18-140, checkpoint_json.cc).

The reference writes one JSON document, cp_state.json, with the keys
"propagator" (the serialised Propagator: lattice, stepper) and "simulator"
(one serialised Bunch_simulator per rank), and stores the particles of each
bunch in HDF5 (bunch_particles.cc:721-750).  Here cp_state.json keeps the
same two keys -- "propagator": lattice (reference particle, elements with
their attributes), stepper kind, its step count and the space-charge
options field by field; "simulator": one entry per bunch with its size,
real_num and the full sb2_bunch_state (reference and design particles,
turns done, counts) -- and the particles, masks and discards of each bunch
go to an .npz archive beside it.

The particle data leaves the GPU through Bunch.snapshot: one stream-ordered
copy (after a device-side scatter back to the caller's order when the bunch
is in its cell-ordered working copy).  With wait=False the files are written
by a host thread once the copy has landed, while the caller keeps queueing
turns on the same stream.

Diagnostics buffers, CUDA graph caches and the collective hook of a
propagator are run-time settings, not checkpointed state: set them again on
the loaded propagator.
"""
import json
import os
import threading

import numpy as np

from . import _lib

STATE_FILE = "cp_state.json"


def _refpart_spec(ref):
    charge, mass, value, kind = ref._spec()
    return {"charge": charge, "mass": mass, "value": value, "kind": kind}


def _refpart_from(spec):
    from . import Four_momentum, Reference_particle
    fm = Four_momentum(spec["mass"])
    fm._kind, fm._value = spec["kind"], spec["value"]
    return Reference_particle(spec["charge"], fm)


def _struct_to_dict(st):
    out = {}
    for name, _ in st._fields_:
        v = getattr(st, name)
        if hasattr(v, "_fields_"):
            out[name] = _struct_to_dict(v)
        elif hasattr(v, "__len__"):
            out[name] = list(v)
        else:
            out[name] = v
    return out


def _dict_to_struct(d, st):
    for name, _ in st._fields_:
        v = getattr(st, name)
        if hasattr(v, "_fields_"):
            _dict_to_struct(d[name], v)
        elif hasattr(v, "__len__"):
            for i, x in enumerate(d[name]):
                v[i] = x
        else:
            setattr(st, name, d[name])
    return st


def propagator_state(prop):
    """The "propagator" entry: everything needed to rebuild the Propagator."""
    lat = prop.lattice
    stepper = prop.stepper
    opts = stepper.collective_options
    return {
        "lattice": {
            "name": lat.name,
            "reference_particle": None if lat.reference_particle is None else _refpart_spec(lat.reference_particle),
            "elements": [{"type": e.type, "name": e.name, "double": dict(e.double), "string": dict(e.string),
                          "vector": {k: list(v) for k, v in e.vector.items()}} for e in lat.elements],
        },
        "stepper": {"class": type(stepper).__name__, "num": stepper.num,
                    "collective": None if opts is None else _struct_to_dict(opts._o)},
    }


def propagator_from_state(d):
    import synergia2_b200 as syn
    L = d["lattice"]
    lat = syn.Lattice(L["name"])
    if L["reference_particle"] is not None:
        lat.set_reference_particle(_refpart_from(L["reference_particle"]))
    for e in L["elements"]:
        el = syn.Lattice_element(e["type"], e["name"])
        for k, v in e["double"].items():
            el.set_double_attribute(k, v)
        for k, v in e["string"].items():
            el.set_string_attribute(k, v)
        for k, v in e["vector"].items():
            el.set_vector_attribute(k, v)
        lat.append(el)
    S = d["stepper"]
    opts = None
    if S["collective"] is not None:
        shape = S["collective"]["shape"]
        opts = syn.Space_charge_3d_open_hockney_options(*shape)
        _dict_to_struct(S["collective"], opts._o)
    cls = getattr(syn, S["class"])
    stepper = cls(S["num"]) if S["class"] == "Independent_stepper_elements" else cls(opts, S["num"])
    return syn.Propagator(lat, stepper)


class PendingCheckpoint:
    """A checkpoint whose files are still being written (wait=False)."""

    def __init__(self, thread, result):
        self._thread, self._result = thread, result

    def join(self):
        self._thread.join()
        if "error" in self._result:
            raise self._result["error"]
        return self._result["path"]


def checkpoint_save(propagator, bunch, directory=".", stream=None, wait=True):
    """syn::checkpoint_save(prop, sim): cp_state.json + cp_particles_0.npz in
    `directory`.  The particles are snapshotted on `stream` behind the work
    already queued there; wait=False returns a PendingCheckpoint at once."""
    os.makedirs(directory, exist_ok=True)
    snap = bunch.snapshot(stream)
    prop_d = propagator_state(propagator)
    ref_d = _refpart_spec(bunch.reference_particle)
    n = bunch.n
    result = {}

    def finish():
        try:
            parts, masks, discards, st = snap.wait()
            pfile = "cp_particles_0.npz"
            np.savez(os.path.join(directory, pfile), parts=parts, masks=masks, discards=discards)
            doc = {"propagator": prop_d,
                   "simulator": [{"bunch": {"total_num": n, "reference_particle": ref_d,
                                            "state": _struct_to_dict(st), "particles_file": pfile}}]}
            path = os.path.join(directory, STATE_FILE)
            tmp = path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(doc, f)
            os.replace(tmp, path)
            result["path"] = path
        except Exception as ex:  # reported by join()
            result["error"] = ex

    if wait:
        finish()
        if "error" in result:
            raise result["error"]
        return result["path"]
    t = threading.Thread(target=finish, daemon=True)
    t.start()
    return PendingCheckpoint(t, result)


def checkpoint_load(directory="."):
    """syn::checkpoint_load(): (Propagator, Bunch) from the most recent
    checkpoint in `directory`, the bunch restored exactly (particles, masks,
    discards, reference and design particles, turns done, counts)."""
    import synergia2_b200 as syn
    with open(os.path.join(directory, STATE_FILE)) as f:
        doc = json.load(f)
    prop = propagator_from_state(doc["propagator"])
    B = doc["simulator"][0]["bunch"]
    st = _dict_to_struct(B["state"], _lib.sb2_bunch_state())
    bunch = syn.Bunch(_refpart_from(B["reference_particle"]), B["total_num"], st.real_num)
    with np.load(os.path.join(directory, B["particles_file"])) as z:
        bunch.set_particles(np.asfortranarray(z["parts"]), z["masks"])
        bunch.set_discards(z["discards"])
    bunch.set_state(st)
    return prop, bunch


def resume(turns, directory=".", stream=None):
    """syn::resume(): load the most recent checkpoint and propagate `turns`
    more turns; returns (Propagator, Bunch)."""
    prop, bunch = checkpoint_load(directory)
    prop.propagate(bunch, turns, stream)
    return prop, bunch
