"""ORACLE — test infrastructure only.

ctypes binding of the CPU FP64 restatement in oracle/sb2_oracle.cc.  Only the
tests, the smoke check and bench.py's cpu_baseline leg import this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

# operation counting (orc_flops_*): categories and operation kinds, in the
# order of the oracle's FlopCat / FlopOp
FLOP_CATEGORIES = ("drift", "quadrupole", "sbend", "thin", "thick_other", "aperture", "sc_domain",
                   "sc_deposit", "sc_kick")
FLOP_OPS = ("add", "mul", "div", "sqrt", "fn")

STEPPER_SPLIT, STEPPER_SPLIT_ELEMENTS, STEPPER_INDEP_ELEMENTS = 0, 1, 2
REF_TOTAL_ENERGY, REF_MOMENTUM, REF_KINETIC_ENERGY = 0, 1, 2
MP = 0.938272046


class SCOptions(ctypes.Structure):
    """Mirror of Space_charge_3d_open_hockney_options
    (simulation/implemented_collective_options.h:67-126)."""
    _fields_ = [("shape", ctypes.c_int * 3), ("doubled_shape", ctypes.c_int * 3),
                ("size", ctypes.c_double * 3), ("offset", ctypes.c_double * 3),
                ("green_fn", ctypes.c_int), ("periodic_z", ctypes.c_int),
                ("z_period", ctypes.c_double), ("grid_entire_period", ctypes.c_int),
                ("n_sigma", ctypes.c_double), ("kick_scale", ctypes.c_double),
                ("domain_fixed", ctypes.c_int)]

    @classmethod
    def make(cls, gx, gy, gz, green_fn=1, n_sigma=8.0, kick_scale=1.0, fixed=None):
        o = cls()
        for i, g in enumerate((gx, gy, gz)):
            o.shape[i] = g
            o.doubled_shape[i] = 2 * g
        o.green_fn = green_fn
        o.n_sigma = n_sigma
        o.kick_scale = kick_scale
        if fixed is not None:
            offset, size = fixed
            for i in range(3):
                o.offset[i] = offset[i]
                o.size[i] = size[i]
            o.domain_fixed = 1
        return o


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-C", _HERE], stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(path)
        vp, d, i, i64 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int64
        pd = ctypes.POINTER(ctypes.c_double)
        pu8 = ctypes.POINTER(ctypes.c_uint8)
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_lattice_new.restype = vp
        L.orc_lattice_new.argtypes = [i, d, d, i]
        L.orc_lattice_free.argtypes = [vp]
        L.orc_lattice_append.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p]
        L.orc_lattice_set_double.argtypes = [vp, i, ctypes.c_char_p, d]
        L.orc_lattice_set_string.argtypes = [vp, i, ctypes.c_char_p, ctypes.c_char_p]
        L.orc_lattice_set_vector.argtypes = [vp, i, ctypes.c_char_p, pd, i]
        L.orc_lattice_length.restype = d
        L.orc_lattice_length.argtypes = [vp]
        L.orc_sim_new.argtypes = [vp, i, i, ctypes.POINTER(SCOptions), i, d, d, i, i64, d,
                                  ctypes.POINTER(vp)]
        L.orc_sim_free.argtypes = [vp]
        L.orc_sim_num_steps.argtypes = [vp]
        L.orc_sim_step_slices.argtypes = [vp, i, i, pd, i]
        L.orc_sim_set_particles.argtypes = [vp, pd, pu8]
        L.orc_sim_get_particles.argtypes = [vp, pd, pu8, pu8]
        L.orc_sim_counts.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i), pd]
        L.orc_sim_design_state.argtypes = [vp, pd, pd]
        L.orc_sim_propagate.argtypes = [vp, i]
        L.orc_sim_propagate_steps.argtypes = [vp, i, i]
        L.orc_sim_libff_apply.argtypes = [vp, pd, i]
        L.orc_sim_aperture_apply.argtypes = [vp, i, ctypes.c_char_p, ctypes.POINTER(i)]
        L.orc_sim_sc_last.argtypes = [vp, pd, pd, pd, pd, pd, pd, pd, pd]
        L.orc_sc_apply.argtypes = [ctypes.POINTER(SCOptions), i, d, d, i, i64, d, i, pd, pu8, d,
                                   pd, pd, pd, pd, pd, pd, pd, pd]
        L.orc_deposit.argtypes = [ctypes.POINTER(ctypes.c_int), pd, pd, i, d, i, i64, pd, pu8, pd]
        L.orc_fft3d.argtypes = [pd, i, i, i, i]
        L.orc_green.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), pd, i, pd]
        L.orc_set_threads.argtypes = [i]
        L.orc_flops_begin.argtypes = [i64]
        L.orc_flops_end.argtypes = [ctypes.POINTER(i)]
        L.orc_flops_record.argtypes = [i, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i64)]
        _LIB = L
    return _LIB


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _pu8(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if a is not None else None


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())


def set_threads(n):
    return lib().orc_set_threads(n)


class Lattice:
    """Element list with attributes; `elements` is a list of dicts
    {type, name, double: {...}, string: {...}, vector: {...}}."""

    def __init__(self, elements, charge=1, mass=MP, value=None, kind=REF_TOTAL_ENERGY):
        self.elements = elements
        self.h = lib().orc_lattice_new(charge, mass, value, kind)
        for e in elements:
            idx = lib().orc_lattice_append(self.h, e["type"].encode(), e.get("name", "e").encode())
            for k, v in e.get("double", {}).items():
                lib().orc_lattice_set_double(self.h, idx, k.encode(), float(v))
            for k, v in e.get("string", {}).items():
                lib().orc_lattice_set_string(self.h, idx, k.encode(), v.encode())
            for k, v in e.get("vector", {}).items():
                a = np.asarray(v, dtype=np.float64)
                lib().orc_lattice_set_vector(self.h, idx, k.encode(), _pd(a), len(a))

    def length(self):
        return lib().orc_lattice_length(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_lattice_free(self.h)
            self.h = None


class Sim:
    """One bunch tracked through a lattice by a stepper, optionally with the
    3D open Hockney space-charge operator."""

    def __init__(self, lattice, n, real_num, stepper=STEPPER_SPLIT, num=1, sc=None, charge=1,
                 mass=MP, value=None, kind=REF_TOTAL_ENERGY):
        self.n = n
        self.lattice = lattice
        h = ctypes.c_void_p()
        _check(lib().orc_sim_new(lattice.h, stepper, num, ctypes.byref(sc) if sc is not None else None,
                                 charge, mass, value, kind, n, real_num, ctypes.byref(h)))
        self.h = h.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_sim_free(self.h)
            self.h = None

    def num_steps(self):
        return lib().orc_sim_num_steps(self.h)

    def step_slices(self, step, op):
        out = np.zeros((256, 3))
        k = lib().orc_sim_step_slices(self.h, step, op, _pd(out), 256)
        return None if k < 0 else out[:k]

    def set_particles(self, parts, masks=None):
        parts = np.asfortranarray(parts, dtype=np.float64)
        assert parts.shape == (self.n, 7)
        m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint8)
        lib().orc_sim_set_particles(self.h, _pd(parts), _pu8(m))

    def get_particles(self):
        parts = np.zeros((self.n, 7), order="F")
        masks = np.zeros(self.n, np.uint8)
        disc = np.zeros(self.n, np.uint8)
        lib().orc_sim_get_particles(self.h, _pd(parts), _pu8(masks), _pu8(disc))
        return parts, masks, disc

    def counts(self):
        nv, nt, rn = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        lib().orc_sim_counts(self.h, ctypes.byref(nv), ctypes.byref(nt), ctypes.byref(rn))
        return nv.value, nt.value, rn.value

    def design_state(self):
        st = np.zeros(6)
        sn = np.zeros(1)
        lib().orc_sim_design_state(self.h, _pd(st), _pd(sn))
        return st, sn[0]

    def propagate(self, turns):
        _check(lib().orc_sim_propagate(self.h, turns))

    def propagate_steps(self, first, count):
        _check(lib().orc_sim_propagate_steps(self.h, first, count))

    def libff_apply(self, slices):
        """LibFF_operation over explicit slices: rows (element index, left,
        right), applied in order."""
        a = np.ascontiguousarray(slices, dtype=np.float64).reshape(-1, 3)
        _check(lib().orc_sim_libff_apply(self.h, _pd(a), a.shape[0]))

    def aperture_apply(self, index, aperture_type):
        """Aperture_operation with the attributes of element `index`;
        returns the number of particles discarded."""
        nd = ctypes.c_int()
        _check(lib().orc_sim_aperture_apply(self.h, index, aperture_type.encode(), ctypes.byref(nd)))
        return nd.value

    def count_flops(self, index, first, count):
        """Runs steps [first, first+count) as propagate_steps does and
        counts the algorithmic FP64 operations of particle `index` in the
        oracle's own particle code.  Returns one record per operator of each
        step: (step, 'I' or 'C', counts) with counts[category][op] (see
        FLOP_CATEGORIES, FLOP_OPS).  Raises if an element kind whose particle
        loop is not instrumented ran."""
        L = lib()
        L.orc_flops_begin(index)
        try:
            rc = L.orc_sim_propagate_steps(self.h, first, count)
        finally:
            unc = ctypes.c_int()
            nrec = L.orc_flops_end(ctypes.byref(unc))
        _check(rc)
        if unc.value:
            raise RuntimeError("operation counting: an element kind without an instrumented particle loop ran")
        out = []
        buf = (ctypes.c_int64 * (len(FLOP_CATEGORIES) * len(FLOP_OPS)))()
        st, kd = ctypes.c_int(), ctypes.c_int()
        for r in range(nrec):
            _check(L.orc_flops_record(r, ctypes.byref(st), ctypes.byref(kd), buf))
            a = np.array(buf[:], dtype=np.int64).reshape(len(FLOP_CATEGORIES), len(FLOP_OPS))
            out.append((st.value, chr(kd.value), {c: dict(zip(FLOP_OPS, map(int, a[i])))
                                                  for i, c in enumerate(FLOP_CATEGORIES)}))
        return out

    def sc_last(self, shape):
        gx, gy, gz = shape
        left, h = np.zeros(3), np.zeros(3)
        arrs = [np.zeros((gz, gy, gx)) for _ in range(5)]
        sc = np.zeros(8)
        _check(lib().orc_sim_sc_last(self.h, _pd(left), _pd(h), *[_pd(a) for a in arrs], _pd(sc)))
        return dict(left=left, h=h, rho=arrs[0], phi=arrs[1], ex=arrs[2], ey=arrs[3], ez=arrs[4],
                    fn_norm=sc[0], factor=sc[1], mean_std=sc[2:8])


def sc_apply(opts, parts, time_step, real_num, masks=None, n_total=0, charge=1, mass=MP,
             value=None, kind=REF_TOTAL_ENERGY):
    """One space-charge kick of the collective operator alone; returns the
    kicked particles and the solve's intermediate grids."""
    parts = np.array(parts, dtype=np.float64, order="F", copy=True)
    n = parts.shape[0]
    gx, gy, gz = opts.shape[0], opts.shape[1], opts.shape[2]
    left, h = np.zeros(3), np.zeros(3)
    arrs = [np.zeros((gz, gy, gx)) for _ in range(5)]
    sc = np.zeros(8)
    m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint8)
    _check(lib().orc_sc_apply(ctypes.byref(opts), charge, mass, value, kind, n, real_num, n_total,
                              _pd(parts), _pu8(m), time_step, _pd(left), _pd(h),
                              *[_pd(a) for a in arrs], _pd(sc)))
    return parts, dict(left=left, h=h, rho=arrs[0], phi=arrs[1], ex=arrs[2], ey=arrs[3],
                       ez=arrs[4], fn_norm=sc[0], factor=sc[1], mean_std=sc[2:8])


def deposit(shape, size, offset, parts, real_num, n_total, charge=1, masks=None):
    parts = np.asfortranarray(parts, dtype=np.float64)
    n = parts.shape[0]
    sh = (ctypes.c_int * 3)(*shape)
    sz = np.asarray(size, dtype=np.float64)
    of = np.asarray(offset, dtype=np.float64)
    out = np.zeros((shape[2], shape[1], shape[0]))
    m = None if masks is None else np.ascontiguousarray(masks, dtype=np.uint8)
    _check(lib().orc_deposit(sh, _pd(sz), _pd(of), charge, real_num, n_total, n, _pd(parts),
                             _pu8(m), _pd(out)))
    return out


def fft3d(a, sign=-1):
    """Oracle FFT of a complex (nz, ny, nx) array; unnormalised."""
    b = np.ascontiguousarray(a, dtype=np.complex128).copy()
    nz, ny, nx = b.shape
    lib().orc_fft3d(b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nx, ny, nz, sign)
    return b


def green(shape, dshape, size, green_fn=1):
    sh = (ctypes.c_int * 3)(*shape)
    dsh = (ctypes.c_int * 3)(*dshape)
    sz = np.asarray(size, dtype=np.float64)
    out = np.zeros((dshape[2], dshape[1], dshape[0]))
    _check(lib().orc_green(sh, dsh, _pd(sz), green_fn, _pd(out)))
    return out
