"""synergia2_b200 — B200-native space-charge + tracking step of Synergia.

Python mirror of the reference's own Python API for this path (class and
method names as in synergia.foundation / lattice / collective / simulation /
bunch), driving the sm_100a library libsb2.so through its C ABI
(include/sb2.h).  Particles live on the GPU; host arrays cross only in
get_particles / set_particles.

    import synergia2_b200 as syn
    ref = syn.Reference_particle(1, syn.Four_momentum(syn.pconstants.mp, syn.pconstants.mp + 2.5))
    lat = syn.Lattice("fodo"); ...; lat.set_reference_particle(ref)
    sc = syn.Space_charge_3d_open_hockney_options(64, 64, 128)
    prop = syn.Propagator(lat, syn.Split_operator_stepper(sc, 8))
    bunch = syn.Bunch(ref, 4194304, 1e11)
    bunch.populate_gaussian([1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4], seed=1)
    prop.propagate(bunch, 100)
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import SB2Error, check, lib

__all__ = ["Batch", "pconstants", "Four_momentum", "Reference_particle", "Lattice_element", "Lattice", "Bunch",
           "Space_charge_3d_open_hockney_options", "Space_charge_3d_open_hockney", "Split_operator_stepper",
           "Split_operator_stepper_elements", "Independent_stepper_elements", "Propagator", "SB2Error",
           "green_fn_t", "precision_t", "BunchSnapshot", "checkpoint_save", "checkpoint_load", "resume"]


class pconstants:
    """foundation/physical_constants.h (PDG 2012)."""
    mp = proton_mass = 0.938272046
    me = electron_mass = 0.510998928e-3
    e = 1.602176565e-19
    c = 299792458.0
    mu0 = 4 * math.pi * 1.0e-7
    epsilon0 = 1.0 / (c * c * mu0)
    rp = e / (4 * math.pi * epsilon0 * mp * 1.0e9)
    proton_charge = 1


class green_fn_t:
    pointlike = _lib.SB2_GREEN_POINTLIKE
    linear = _lib.SB2_GREEN_LINEAR


class precision_t:
    fp64 = _lib.SB2_PRECISION_FP64
    mixed = _lib.SB2_PRECISION_MIXED


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _pu8(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if a is not None else None


class Four_momentum:
    """foundation/four_momentum.{h,cc}: kept as (mass, how, value) so the C
    side rebuilds gamma, beta and p with the reference's own arithmetic."""

    def __init__(self, mass, total_energy=None):
        self.mass = mass
        if total_energy is None:
            self._kind, self._value = _lib.SB2_REF_TOTAL_ENERGY, mass
        else:
            self._kind, self._value = _lib.SB2_REF_TOTAL_ENERGY, total_energy

    def set_momentum(self, p):
        self._kind, self._value = _lib.SB2_REF_MOMENTUM, p

    def set_kinetic_energy(self, k):
        self._kind, self._value = _lib.SB2_REF_KINETIC_ENERGY, k

    def set_total_energy(self, e):
        self._kind, self._value = _lib.SB2_REF_TOTAL_ENERGY, e

    def _gamma(self):
        if self._kind == _lib.SB2_REF_TOTAL_ENERGY:
            return self._value / self.mass
        if self._kind == _lib.SB2_REF_KINETIC_ENERGY:
            return (self.mass + self._value) / self.mass
        r2 = self._value ** 2 / self.mass ** 2
        b = math.sqrt(r2 / (1 + r2))
        return 1.0 / math.sqrt(1.0 - b * b)

    def get_gamma(self):
        return self._gamma()

    def get_beta(self):
        g = self._gamma()
        return math.sqrt(1.0 - 1.0 / (g * g))

    def get_momentum(self):
        g = self._gamma()
        return g * self.get_beta() * self.mass

    def get_total_energy(self):
        return self._gamma() * self.mass


class Reference_particle:
    def __init__(self, charge, four_momentum):
        self.charge = charge
        self.four_momentum = four_momentum

    def get_charge(self):
        return self.charge

    def get_mass(self):
        return self.four_momentum.mass

    def get_beta(self):
        return self.four_momentum.get_beta()

    def get_gamma(self):
        return self.four_momentum.get_gamma()

    def get_momentum(self):
        return self.four_momentum.get_momentum()

    def _spec(self):
        fm = self.four_momentum
        return self.charge, fm.mass, fm._value, fm._kind


class Lattice_element:
    """lattice/lattice_element.h: type name, element name, attributes."""

    def __init__(self, type_name, name):
        self.type = type_name
        self.name = name
        self.double = {}
        self.string = {}
        self.vector = {}

    def set_double_attribute(self, k, v):
        self.double[k] = float(v)

    def set_string_attribute(self, k, v):
        self.string[k] = str(v)

    def set_vector_attribute(self, k, v):
        self.vector[k] = [float(x) for x in v]

    def get_double_attribute(self, k, default=None):
        if k in self.double:
            return self.double[k]
        if default is None:
            raise KeyError(k)
        return default

    def get_length(self):
        return self.double.get("l", 0.0)

    def get_type_name(self):
        return self.type

    def get_name(self):
        return self.name


class Lattice:
    def __init__(self, name="lattice", elements=None, reference_particle=None):
        self.name = name
        self.elements = list(elements or [])
        self.reference_particle = reference_particle

    def append(self, element):
        self.elements.append(element)

    def set_reference_particle(self, ref):
        self.reference_particle = ref

    def get_reference_particle(self):
        return self.reference_particle

    def get_elements(self):
        return self.elements

    def get_length(self):
        L = 0.0
        for e in self.elements:
            L += e.get_length()
        return L

    def _handle(self):
        """Builds the C-side lattice (caller destroys)."""
        h = ctypes.c_void_p()
        check(lib().sb2_lattice_create(self.name.encode(), ctypes.byref(h)))
        if self.reference_particle is not None:
            check(lib().sb2_lattice_set_reference_particle(h, *self.reference_particle._spec()))
        idx = ctypes.c_int32()
        for e in self.elements:
            check(lib().sb2_lattice_append(h, e.type.encode(), e.name.encode(), ctypes.byref(idx)))
            for k, v in e.double.items():
                check(lib().sb2_lattice_set_double(h, idx, k.encode(), v))
            for k, v in e.string.items():
                check(lib().sb2_lattice_set_string(h, idx, k.encode(), v.encode()))
            for k, v in e.vector.items():
                a = np.asarray(v, dtype=np.float64)
                check(lib().sb2_lattice_set_vector(h, idx, k.encode(), _pd(a), len(a)))
        return h


class Bunch:
    """bunch/bunch.h: N x 7 FP64 column-major particles + uint8 masks on the
    GPU.  Columns x, xp, y, yp, cdt, dpop, id."""
    x, xp, y, yp, cdt, dpop, id = range(7)

    def __init__(self, reference_particle, total_num, real_num):
        self.reference_particle = reference_particle
        self.n = int(total_num)
        h = ctypes.c_void_p()
        check(lib().sb2_bunch_create(*reference_particle._spec(), self.n, float(real_num), ctypes.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                lib().sb2_bunch_destroy(h)
            except Exception:
                pass
            self.h = None

    def size(self):
        return self.n

    def set_particles(self, parts, masks=None):
        """checkin: parts is (N, 7) (any order; copied as column-major)."""
        p = np.asfortranarray(parts, dtype=np.float64)
        assert p.shape == (self.n, 7)
        m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint8)
        check(lib().sb2_bunch_set_particles(self.h, _pd(p), _pu8(m)))

    def get_particles(self):
        """checkout: returns (parts (N,7) F-order, masks, discards)."""
        p = np.zeros((self.n, 7), order="F")
        m = np.zeros(self.n, np.uint8)
        d = np.zeros(self.n, np.uint8)
        check(lib().sb2_bunch_get_particles(self.h, _pd(p), _pu8(m), _pu8(d)))
        return p, m, d

    def get_local_particles(self):
        return self.get_particles()[0]

    def counts(self):
        a, v, t, r = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        check(lib().sb2_bunch_counts(self.h, ctypes.byref(a), ctypes.byref(v), ctypes.byref(t), ctypes.byref(r)))
        return dict(size=a.value, local_num=v.value, total_num=t.value, real_num=r.value)

    def get_local_num(self):
        return self.counts()["local_num"]

    def get_total_num(self):
        return self.counts()["total_num"]

    def get_real_num(self):
        return self.counts()["real_num"]

    def design_state(self):
        st = np.zeros(6)
        sn = ctypes.c_double()
        check(lib().sb2_bunch_design_state(self.h, _pd(st), ctypes.byref(sn)))
        return st, sn.value

    def populate_gaussian(self, sigmas, seed):
        s = np.asarray(sigmas, dtype=np.float64)
        check(lib().sb2_bunch_populate_gaussian(self.h, _pd(s), int(seed)))

    def moments(self):
        mean, mom2, emit = np.zeros(6), np.zeros(36), np.zeros(3)
        check(lib().sb2_bunch_moments(self.h, _pd(mean), _pd(mom2), _pd(emit)))
        return mean, mom2.reshape(6, 6), emit

    def get_state(self):
        """Host-side state (reference particles, turns, counts): an
        sb2_bunch_state (include/sb2.h)."""
        st = _lib.sb2_bunch_state()
        check(lib().sb2_bunch_get_state(self.h, ctypes.byref(st)))
        return st

    def set_state(self, st):
        check(lib().sb2_bunch_set_state(self.h, ctypes.byref(st)))

    def set_discards(self, discards):
        d = np.ascontiguousarray(discards, dtype=np.uint8)
        assert d.shape == (self.n,)
        check(lib().sb2_bunch_set_discards(self.h, _pu8(d)))

    def snapshot(self, stream=None, pinned=True):
        """Stream-ordered device -> host copy of the resident particles
        (sb2_bunch_snapshot_async): returns a BunchSnapshot at once; its
        wait() returns (parts, masks, discards, state) when the copy is done.
        Later propagate calls on the same stream may be queued meanwhile."""
        return BunchSnapshot(self, stream, pinned)

    def write_openpmd_file(self, filename, num_part=-1, offset=0):
        """Bunch::write_openpmd_file (bunch.cc:466-600), openPMD JSON series."""
        from . import particle_io
        particle_io.check_extension(filename, (".json",))
        parts, masks, _ = self.get_particles()
        st = self.get_state()
        particle_io.write_openpmd_json(filename, parts, masks, st.ref.mass, st.ref.beta, st.ref.gamma,
                                       num_part=num_part, offset=offset)

    def read_openpmd_file(self, filename, iteration=None):
        """Bunch::read_openpmd_file (bunch.cc:189-320): particles, masks and
        the reference particle's four momentum (from beta_ref / gamma_ref)."""
        from . import particle_io
        particle_io.check_extension(filename, (".json",))
        parts, masks, mass, beta_ref, gamma_ref = particle_io.read_openpmd_json(filename, iteration)
        if parts.shape[0] != self.n:
            raise ValueError("file holds %d particles, the bunch %d" % (parts.shape[0], self.n))
        self.set_particles(parts, masks)
        st = self.get_state()
        st.ref.gamma = gamma_ref  # Four_momentum::set_gamma (four_momentum.cc:8-16)
        st.ref.energy = gamma_ref * st.ref.mass
        st.ref.beta = math.sqrt(1.0 - 1.0 / (gamma_ref * gamma_ref))
        st.ref.momentum = gamma_ref * st.ref.beta * st.ref.mass
        self.set_state(st)

    def write_file(self, filename, num_part=-1, offset=0):
        """Bunch::write_file (bunch_particles.cc:677-702): datasets
        "particles" and "particles_masks" in a .npz archive."""
        from . import particle_io
        particle_io.check_extension(filename, (".npz",))
        parts, masks, _ = self.get_particles()
        particle_io.write_npz(filename, parts, masks, num_part, offset)

    def read_file(self, filename):
        from . import particle_io
        particle_io.check_extension(filename, (".npz",))
        parts, masks = particle_io.read_npz(filename)
        if parts.shape[0] != self.n:
            raise ValueError("file holds %d particles, the bunch %d" % (parts.shape[0], self.n))
        self.set_particles(parts, masks)

    def device_arrays(self):
        p, m, d = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        st = ctypes.c_int64()
        check(lib().sb2_bunch_device_arrays(self.h, ctypes.byref(p), ctypes.byref(st), ctypes.byref(m),
                                            ctypes.byref(d)))
        return p.value, st.value, m.value, d.value


class BunchSnapshot:
    """A pending sb2_bunch_snapshot_async: host buffers (pinned when torch
    with CUDA is available, so the copy does not block) and the bunch's
    host-side state captured when the snapshot was queued."""

    def __init__(self, bunch, stream, pinned):
        n = bunch.n
        self.bunch, self.stream = bunch, stream
        self.state = bunch.get_state()
        self._keep = None
        if pinned:
            try:
                import torch
                if torch.cuda.is_available():
                    t = (torch.empty(7 * n, dtype=torch.float64, pin_memory=True),
                         torch.empty(n, dtype=torch.uint8, pin_memory=True),
                         torch.empty(n, dtype=torch.uint8, pin_memory=True))
                    self._keep = t
                    self.parts = t[0].numpy().reshape((n, 7), order="F")
                    self.masks, self.discards = t[1].numpy(), t[2].numpy()
            except ImportError:
                pass
        if self._keep is None:
            self.parts = np.zeros((n, 7), order="F")
            self.masks = np.zeros(n, np.uint8)
            self.discards = np.zeros(n, np.uint8)
        check(lib().sb2_bunch_snapshot_async(bunch.h, _pd(self.parts), _pu8(self.masks), _pu8(self.discards),
                                             stream))

    def wait(self):
        import torch
        if self.stream is None:
            torch.cuda.synchronize()
        else:
            torch.cuda.ExternalStream(int(self.stream)).synchronize()
        nv, nt, rn = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        check(lib().sb2_bunch_snapshot_counts(self.bunch.h, ctypes.byref(nv), ctypes.byref(nt), ctypes.byref(rn)))
        self.state.n_valid, self.state.n_total, self.state.real_num = nv.value, nt.value, rn.value
        return self.parts, self.masks, self.discards, self.state


class Space_charge_3d_open_hockney_options:
    """simulation/implemented_collective_options.h:67-126."""

    def __init__(self, gridx=32, gridy=32, gridz=64):
        self._o = _lib.sb2_sc3d_options()
        check(lib().sb2_sc3d_options_init(ctypes.byref(self._o), gridx, gridy, gridz))

    def set_fixed_domain(self, offset, size):
        o = np.asarray(offset, dtype=np.float64)
        s = np.asarray(size, dtype=np.float64)
        check(lib().sb2_sc3d_options_set_fixed_domain(ctypes.byref(self._o), _pd(o), _pd(s)))

    def __getattr__(self, k):
        if k == "_o":
            raise AttributeError(k)
        o = self.__dict__["_o"]
        v = getattr(o, k)
        return list(v) if hasattr(v, "__len__") else v

    def __setattr__(self, k, v):
        if k == "_o":
            object.__setattr__(self, k, v)
            return
        o = self.__dict__["_o"]
        cur = getattr(o, k)
        if hasattr(cur, "__len__"):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(o, k, v)


class Space_charge_3d_open_hockney:
    """The collective operator alone (space_charge_3d_open_hockney.cc:400-453)."""

    def __init__(self, options):
        self.options = options
        h = ctypes.c_void_p()
        check(lib().sb2_sc3d_create(ctypes.byref(options._o), ctypes.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                lib().sb2_sc3d_destroy(h)
            except Exception:
                pass
            self.h = None

    def apply(self, bunch, time_step):
        check(lib().sb2_sc3d_apply(self.h, bunch.h, float(time_step), None))

    def last(self):
        gx, gy, gz = self.options.shape
        return _sc_last(lambda *a: lib().sb2_sc3d_last(self.h, *a), gx, gy, gz)


def _sc_last(fn, gx, gy, gz):
    left, h, sc = np.zeros(3), np.zeros(3), np.zeros(8)
    arrs = [np.zeros((gz, gy, gx)) for _ in range(5)]
    check(fn(_pd(left), _pd(h), *[_pd(a) for a in arrs], _pd(sc)))
    return dict(left=left, h=h, rho=arrs[0], phi=arrs[1], ex=arrs[2], ey=arrs[3], ez=arrs[4], fn_norm=sc[0],
                factor=sc[1], mean_std=sc[2:8])


class _Stepper:
    kind = None

    def __init__(self, collective_options, num):
        self.collective_options = collective_options
        self.num = num


class Split_operator_stepper(_Stepper):
    """simulation/split_operator_stepper.cc: num_steps split-operator steps."""
    kind = _lib.SB2_STEPPER_SPLIT_OPERATOR

    def __init__(self, collective_options, num_steps):
        super().__init__(collective_options, num_steps)


class Split_operator_stepper_elements(_Stepper):
    kind = _lib.SB2_STEPPER_SPLIT_OPERATOR_ELEMENTS

    def __init__(self, collective_options, steps_per_element):
        super().__init__(collective_options, steps_per_element)


class Independent_stepper_elements(_Stepper):
    kind = _lib.SB2_STEPPER_INDEPENDENT_ELEMENTS

    def __init__(self, steps_per_element):
        super().__init__(None, steps_per_element)


class LibFF_operation:
    """simulation/independent_operation.h:45-60: the libFF maps of a list of
    lattice slices, rows (element index, left, right), applied in order by
    FF_element::apply (libFF/ff_element.h:25-67); the bunch's design
    reference particle moves with them."""

    def __init__(self, lattice, slices):
        self.lattice = lattice
        self.slices = np.ascontiguousarray(slices, dtype=np.float64).reshape(-1, 3)

    def apply(self, bunch, stream=None):
        lh = self.lattice._handle()
        try:
            check(lib().sb2_libff_apply(lh, _pd(self.slices), self.slices.shape[0], bunch.h, stream))
        finally:
            lib().sb2_lattice_destroy(lh)


class Aperture_operation:
    """simulation/aperture_operation.h:8-115: Bunch::apply_aperture with the
    attributes of lattice element `index`; aperture_type "finite",
    "circular", "elliptical" or "rectangular"."""

    def __init__(self, lattice, index, aperture_type):
        self.lattice = lattice
        self.index = int(index)
        self.aperture_type = aperture_type

    def apply(self, bunch, stream=None):
        """Returns the number of particles discarded."""
        lh = self.lattice._handle()
        nd = ctypes.c_int32()
        try:
            check(lib().sb2_aperture_apply(lh, self.index, self.aperture_type.encode(), bunch.h, ctypes.byref(nd),
                                           stream))
        finally:
            lib().sb2_lattice_destroy(lh)
        return nd.value


class Propagator:
    """simulation/propagator.cc: Propagator(lattice, stepper).propagate."""

    def __init__(self, lattice, stepper):
        self.lattice = lattice
        self.stepper = stepper
        lh = lattice._handle()
        try:
            h = ctypes.c_void_p()
            opts = stepper.collective_options
            check(lib().sb2_propagator_create(lh, stepper.kind, stepper.num,
                                              ctypes.byref(opts._o) if opts is not None else None,
                                              ctypes.byref(h)))
            self.h = h
        finally:
            lib().sb2_lattice_destroy(lh)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                lib().sb2_propagator_destroy(h)
            except Exception:
                pass
            self.h = None

    def num_steps(self):
        n = ctypes.c_int32()
        check(lib().sb2_propagator_num_steps(self.h, ctypes.byref(n)))
        return n.value

    def step_slices(self, step, op):
        out = np.zeros((256, 3))
        n = ctypes.c_int32()
        check(lib().sb2_propagator_step_slices(self.h, step, op, _pd(out), 256, ctypes.byref(n)))
        return None if n.value < 0 else out[: n.value]

    def propagate(self, bunch, turns, stream=None):
        check(lib().sb2_propagator_propagate(self.h, bunch.h, int(turns), stream))

    def propagate_steps(self, bunch, first, count, stream=None):
        check(lib().sb2_propagator_propagate_steps(self.h, bunch.h, int(first), int(count), stream))

    def set_graphs(self, on=True):
        """Replay each turn from a CUDA graph (captured on first use):
        every turn of propagate, every whole turn inside the range of
        propagate_steps."""
        check(lib().sb2_propagator_set_graphs(self.h, 1 if on else 0))

    def prepare_steps(self, bunch, first, count, stream=None):
        """Capture ahead, without running them, the graphs that
        propagate_steps(bunch, first, count) will replay
        (sb2_propagator_prepare_steps); the bunch is left as it was."""
        check(lib().sb2_propagator_prepare_steps(self.h, bunch.h, int(first), int(count), stream))

    def graph_stats(self):
        c, r = ctypes.c_int64(), ctypes.c_int64()
        check(lib().sb2_propagator_graph_stats(self.h, ctypes.byref(c), ctypes.byref(r)))
        return c.value, r.value

    def set_allreduce(self, fn, on_host=True, typed=False):
        """Run this propagator on one shard of a bunch split over ranks
        (sb2_propagator_set_allreduce).  on_host: fn(array) receives a numpy
        view of pinned host memory and sums it in place over the ranks;
        otherwise fn(pointer, count) gets the device pointer.  typed
        (sb2_propagator_set_allreduce_typed): the buffers are float64 or
        float32 -- the array's dtype on the host, fn(pointer, count, dtype)
        on the device, dtype a numpy dtype -- so a mixed-precision
        propagator exchanges its FP32 charge grid as float.  None returns to
        a whole bunch."""
        if fn is None:
            self._allreduce = None
            check(lib().sb2_propagator_set_allreduce(self.h, None, None, 0))
            return
        if typed:
            def tcb(ctx, data, count, dtype, host):
                try:
                    dt = np.dtype(np.float32 if dtype == 1 else np.float64)
                    if host:
                        buf = (ctypes.c_char * (int(count) * dt.itemsize)).from_address(data)
                        fn(np.frombuffer(buf, dtype=dt))
                    else:
                        fn(int(data), int(count), dt)
                    return 0
                except Exception:  # reported as a failed collective
                    return 1

            self._allreduce = _lib.ALLREDUCE_TYPED_FN(tcb)  # kept alive with the propagator
            check(lib().sb2_propagator_set_allreduce_typed(self.h, self._allreduce, None, 1 if on_host else 0))
            return

        def cb(ctx, data, count, host):
            try:
                if host:
                    fn(np.ctypeslib.as_array(data, shape=(int(count),)))
                else:
                    fn(ctypes.cast(data, ctypes.c_void_p).value, int(count))
                return 0
            except Exception:  # reported as a failed collective
                return 1

        self._allreduce = _lib.ALLREDUCE_FN(cb)  # kept alive with the propagator
        check(lib().sb2_propagator_set_allreduce(self.h, self._allreduce, None, 1 if on_host else 0))

    def set_loss_diagnostics(self, capacity):
        """Record every particle an aperture discards (Diagnostics_loss),
        up to `capacity` records; 0 disables."""
        check(lib().sb2_propagator_set_loss_diagnostics(self.h, int(capacity)))
        self._loss_cap = int(capacity)

    def losses(self):
        """Lost-particle records: (k, 10) array of x, xp, y, yp, cdt, dpop,
        id, repetition, s, s_n, ordered by aperture and id."""
        cap = getattr(self, "_loss_cap", 0)
        out = np.zeros((max(cap, 1), 10))
        n = ctypes.c_int32()
        check(lib().sb2_propagator_read_losses(self.h, cap, ctypes.byref(n), _pd(out)))
        return out[: n.value]

    _TUNE_FIELDS = ("light_shape", "full_occ", "full_ppt", "quad_variant", "ctas_per_sm", "sort_interval",
                    "fft_plan", "deposit_chunk")

    def get_tune(self):
        """Launch shape of the particle passes and the re-sort interval
        (sb2_tune) as a dict."""
        t = _lib.sb2_tune()
        check(lib().sb2_propagator_get_tune(self.h, ctypes.byref(t)))
        return {k: getattr(t, k) for k in self._TUNE_FIELDS}

    def set_tune(self, **fields):
        cur = self.get_tune()
        cur.update(fields)
        t = _lib.sb2_tune(*[int(cur[k]) for k in self._TUNE_FIELDS])
        check(lib().sb2_propagator_set_tune(self.h, ctypes.byref(t)))

    def autotune(self, bunch, steps=16):
        """The project's autotuner (sb2_propagator_autotune): coordinate
        descent over get_tune()'s fields, each candidate timed on `steps`
        steps of a scratch copy of `bunch`; applies and returns the best
        configuration and the list of trials (fields + milliseconds)."""
        best = _lib.sb2_tune()
        cap = 64
        nf = len(self._TUNE_FIELDS)
        trials = np.zeros((nf + 1) * cap)
        nt = ctypes.c_int32()
        check(lib().sb2_propagator_autotune(self.h, bunch.h, int(steps), ctypes.byref(best), _pd(trials), cap,
                                            ctypes.byref(nt)))
        rows = trials[: (nf + 1) * min(nt.value, cap)].reshape(-1, nf + 1)
        log = [dict(zip(self._TUNE_FIELDS + ("ms",), [int(v) for v in r[:nf]] + [float(r[nf])])) for r in rows]
        return {k: getattr(best, k) for k in self._TUNE_FIELDS}, log

    def set_step_counts(self, capacity):
        """Per-step count records (sb2_propagator_set_step_counts): the k-th
        step propagated from now on writes (n_valid, n_total, real_num) into
        a host buffer (pinned when torch with CUDA is available)."""
        self._step_buf = None
        if capacity > 0:
            nbytes = ctypes.sizeof(_lib.sb2_step_counts) * capacity
            keep = None
            try:
                import torch
                if torch.cuda.is_available():
                    keep = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            except ImportError:
                pass
            if keep is None:
                keep = np.zeros(nbytes, np.uint8)
                ptr = keep.ctypes.data
            else:
                ptr = keep.data_ptr()
            self._step_buf = (keep, ptr, capacity)
            check(lib().sb2_propagator_set_step_counts(self.h, ctypes.c_void_p(ptr), capacity))
        else:
            check(lib().sb2_propagator_set_step_counts(self.h, None, 0))

    def step_counts(self):
        """Records written so far: a list of (n_valid, n_total, real_num)."""
        if not getattr(self, "_step_buf", None):
            return []
        n = ctypes.c_int32()
        check(lib().sb2_propagator_step_counts_written(self.h, ctypes.byref(n)))
        _, ptr, cap = self._step_buf
        recs = (_lib.sb2_step_counts * cap).from_address(ptr)
        return [(recs[i].n_valid, recs[i].n_total, recs[i].real_num) for i in range(min(n.value, cap))]

    def set_diagnostics(self, capacity):
        """Per-turn Diagnostics_full2 records on the device (initial state of
        the first propagate call, then every turn end); 0 disables."""
        check(lib().sb2_propagator_set_diagnostics(self.h, int(capacity)))
        self._diag_cap = int(capacity)

    def diagnostics(self):
        """The records so far: dict of arrays (one row per record) with the
        Diagnostics_full2 fields."""
        cap = getattr(self, "_diag_cap", 0)
        rs = lib().sb2_diagnostics_record_size()
        rec = np.zeros((max(cap, 1), rs))
        s_path = np.zeros(max(cap, 1))
        turns = np.zeros(max(cap, 1), np.int32)
        n = ctypes.c_int32()
        check(lib().sb2_propagator_read_diagnostics(self.h, cap, ctypes.byref(n), _pd(rec), _pd(s_path),
                                                    turns.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        k = n.value
        r = rec[:k]
        return {"s": s_path[:k], "turns": turns[:k], "num_particles": r[:, 0], "real_num_particles": r[:, 1],
                "mean": r[:, 2:8], "std": r[:, 8:14], "min": r[:, 14:17], "max": r[:, 17:20],
                "mom2": r[:, 20:56].reshape(k, 6, 6), "corr": r[:, 56:92].reshape(k, 6, 6),
                "emitx": r[:, 92], "emity": r[:, 93], "emitz": r[:, 94], "emitxy": r[:, 95], "emitxyz": r[:, 96]}

    def deposited_charge(self, index):
        c = ctypes.c_double()
        check(lib().sb2_propagator_deposited_charge(self.h, index, ctypes.byref(c)))
        return c.value

    def sc_last(self):
        gx, gy, gz = self.stepper.collective_options.shape
        return _sc_last(lambda *a: lib().sb2_propagator_sc_last(self.h, *a), gx, gy, gz)


class Batch:
    """Independent (propagator, bunch) jobs advanced concurrently, one CUDA
    stream per job.  A propagator must not be shared between jobs."""

    def __init__(self):
        h = ctypes.c_void_p()
        check(lib().sb2_batch_create(ctypes.byref(h)))
        self.h = h
        self.jobs = {}

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                lib().sb2_batch_destroy(h)
            except Exception:
                pass
            self.h = None

    def add(self, propagator, bunch):
        slot = ctypes.c_int32()
        check(lib().sb2_batch_add(self.h, propagator.h, bunch.h, ctypes.byref(slot)))
        self.jobs[slot.value] = (propagator, bunch)
        return slot.value

    def remove(self, slot):
        check(lib().sb2_batch_remove(self.h, slot))
        self.jobs.pop(slot, None)

    def run(self, turns_by_slot):
        """Advance each listed slot by its number of turns, concurrently."""
        items = list(turns_by_slot.items())
        if not items:
            return
        slots = (ctypes.c_int32 * len(items))(*[k for k, _ in items])
        turns = (ctypes.c_int32 * len(items))(*[int(v) for _, v in items])
        check(lib().sb2_batch_run(self.h, slots, turns, len(items)))

    def run_lockstep(self, slots, turns):
        """Advance the listed slots by `turns` turns together, one work-list
        launch per kernel kind (and grid shape) per step for all of them
        (sb2_batch_run_lockstep)."""
        slots = list(slots)
        arr = (ctypes.c_int32 * len(slots))(*slots)
        check(lib().sb2_batch_run_lockstep(self.h, arr, len(slots), int(turns)))

    def launch(self, slot, turns):
        """Enqueue `turns` turns of one slot and return at once."""
        check(lib().sb2_batch_launch(self.h, int(slot), int(turns)))

    def query(self, slot):
        """True once the slot's launched turns have finished."""
        d = ctypes.c_int32()
        check(lib().sb2_batch_query(self.h, int(slot), ctypes.byref(d)))
        return bool(d.value)


from .checkpoint import checkpoint_load, checkpoint_save, resume  # noqa: E402
