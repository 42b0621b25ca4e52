"""ctypes binding of libsb2.so (include/sb2.h).

The library must have been built (python -m synergia2_b200.build); loading
fails loudly otherwise — there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsb2.so")
_LIB = None

SB2_OK, SB2_ERR_INVALID, SB2_ERR_CUDA, SB2_ERR_RUNTIME, SB2_ERR_UNSUPPORTED, SB2_ERR_NOMEM = range(6)
SB2_GREEN_POINTLIKE, SB2_GREEN_LINEAR = 0, 1
SB2_PRECISION_FP64, SB2_PRECISION_MIXED = 0, 1
SB2_REF_TOTAL_ENERGY, SB2_REF_MOMENTUM, SB2_REF_KINETIC_ENERGY = 0, 1, 2
SB2_STEPPER_SPLIT_OPERATOR, SB2_STEPPER_SPLIT_OPERATOR_ELEMENTS, SB2_STEPPER_INDEPENDENT_ELEMENTS = 0, 1, 2

# Every function the header declares, with its ctypes signature.
_c = ctypes
_vp, _i32, _i64, _d, _u64, _cp = _c.c_void_p, _c.c_int32, _c.c_int64, _c.c_double, _c.c_uint64, _c.c_char_p
_pd, _pu8, _pi32, _pi64 = _c.POINTER(_c.c_double), _c.POINTER(_c.c_uint8), _c.POINTER(_c.c_int32), _c.POINTER(_c.c_int64)


class sb2_sc3d_options(ctypes.Structure):
    _fields_ = [("shape", _c.c_int32 * 3), ("doubled_shape", _c.c_int32 * 3), ("size", _c.c_double * 3),
                ("offset", _c.c_double * 3), ("green_fn", _c.c_int32), ("periodic_z", _c.c_int32),
                ("z_period", _c.c_double), ("grid_entire_period", _c.c_int32), ("n_sigma", _c.c_double),
                ("kick_scale", _c.c_double), ("domain_fixed", _c.c_int32), ("comm_group_size", _c.c_int32),
                ("precision", _c.c_int32)]


_popts = _c.POINTER(sb2_sc3d_options)


class sb2_refpart_state(ctypes.Structure):
    _fields_ = [("charge", _c.c_int32), ("repetition", _c.c_int32), ("mass", _c.c_double), ("gamma", _c.c_double),
                ("beta", _c.c_double), ("momentum", _c.c_double), ("energy", _c.c_double),
                ("state", _c.c_double * 6), ("s", _c.c_double), ("s_n", _c.c_double)]


class sb2_bunch_state(ctypes.Structure):
    _fields_ = [("ref", sb2_refpart_state), ("design", sb2_refpart_state), ("design_set", _c.c_int32),
                ("turns_done", _c.c_int32), ("n_valid", _c.c_int64), ("n_total", _c.c_int64),
                ("real_num", _c.c_double)]


_pstate = _c.POINTER(sb2_bunch_state)


class sb2_tune(ctypes.Structure):
    _fields_ = [("light_shape", _c.c_int32), ("full_occ", _c.c_int32), ("full_ppt", _c.c_int32),
                ("quad_variant", _c.c_int32), ("ctas_per_sm", _c.c_int32), ("sort_interval", _c.c_int32),
                ("fft_plan", _c.c_int32), ("deposit_chunk", _c.c_int32)]


class sb2_step_counts(ctypes.Structure):
    _fields_ = [("n_valid", _c.c_int32), ("n_total", _c.c_int32), ("real_num", _c.c_double)]
_ppv = _c.POINTER(_c.c_void_p)

SIGNATURES = {
    "sb2_last_error": (_cp, []),
    "sb2_version": (_cp, []),
    "sb2_set_device": (_i32, [_i32]),
    "sb2_profile_enable": (_i32, [_i32]),
    "sb2_profile_read": (_i32, [_i32, _c.POINTER(_cp), _pd, _pi64, _i32]),
    "sb2_fp64_peak_probe": (_i32, [_pd, _vp]),
    "sb2_sc3d_options_init": (_i32, [_popts, _c.c_int, _c.c_int, _c.c_int]),
    "sb2_sc3d_options_set_fixed_domain": (_i32, [_popts, _pd, _pd]),
    "sb2_bunch_create": (_i32, [_i32, _d, _d, _i32, _i64, _d, _ppv]),
    "sb2_bunch_wrap": (_i32, [_i32, _d, _d, _i32, _vp, _i64, _vp, _vp, _i64, _d, _ppv]),
    "sb2_bunch_destroy": (_i32, [_vp]),
    "sb2_bunch_set_particles": (_i32, [_vp, _pd, _pu8]),
    "sb2_bunch_get_particles": (_i32, [_vp, _pd, _pu8, _pu8]),
    "sb2_bunch_device_arrays": (_i32, [_vp, _ppv, _pi64, _ppv, _ppv]),
    "sb2_bunch_counts": (_i32, [_vp, _pi64, _pi64, _pi64, _pd]),
    "sb2_bunch_design_state": (_i32, [_vp, _pd, _pd]),
    "sb2_bunch_get_state": (_i32, [_vp, _pstate]),
    "sb2_bunch_set_state": (_i32, [_vp, _pstate]),
    "sb2_bunch_set_discards": (_i32, [_vp, _pu8]),
    "sb2_bunch_snapshot_async": (_i32, [_vp, _pd, _pu8, _pu8, _vp]),
    "sb2_bunch_snapshot_counts": (_i32, [_vp, _pi64, _pi64, _pd]),
    "sb2_bunch_populate_gaussian": (_i32, [_vp, _pd, _u64]),
    "sb2_bunch_moments": (_i32, [_vp, _pd, _pd, _pd]),
    "sb2_lattice_create": (_i32, [_cp, _ppv]),
    "sb2_lattice_destroy": (_i32, [_vp]),
    "sb2_lattice_set_reference_particle": (_i32, [_vp, _i32, _d, _d, _i32]),
    "sb2_lattice_append": (_i32, [_vp, _cp, _cp, _pi32]),
    "sb2_lattice_set_double": (_i32, [_vp, _i32, _cp, _d]),
    "sb2_lattice_set_string": (_i32, [_vp, _i32, _cp, _cp]),
    "sb2_lattice_set_vector": (_i32, [_vp, _i32, _cp, _pd, _i32]),
    "sb2_lattice_length": (_i32, [_vp, _pd]),
    "sb2_lattice_num_elements": (_i32, [_vp, _pi32]),
    "sb2_propagator_create": (_i32, [_vp, _i32, _i32, _popts, _ppv]),
    "sb2_propagator_destroy": (_i32, [_vp]),
    "sb2_propagator_num_steps": (_i32, [_vp, _pi32]),
    "sb2_propagator_step_slices": (_i32, [_vp, _i32, _i32, _pd, _i32, _pi32]),
    "sb2_propagator_propagate": (_i32, [_vp, _vp, _i32, _vp]),
    "sb2_propagator_propagate_steps": (_i32, [_vp, _vp, _i32, _i32, _vp]),
    "sb2_propagator_deposited_charge": (_i32, [_vp, _i32, _pd]),
    "sb2_propagator_set_graphs": (_i32, [_vp, _i32]),
    "sb2_propagator_graph_stats": (_i32, [_vp, _pi64, _pi64]),
    "sb2_batch_create": (_i32, [_ppv]),
    "sb2_batch_destroy": (_i32, [_vp]),
    "sb2_batch_add": (_i32, [_vp, _vp, _vp, _pi32]),
    "sb2_batch_remove": (_i32, [_vp, _i32]),
    "sb2_batch_run": (_i32, [_vp, _pi32, _pi32, _i32]),
    "sb2_batch_launch": (_i32, [_vp, _i32, _i32]),
    "sb2_propagator_set_diagnostics": (_i32, [_vp, _i32]),
    "sb2_propagator_set_allreduce": (_i32, [_vp, _vp, _vp, _i32]),
    "sb2_propagator_read_diagnostics": (_i32, [_vp, _i32, _pi32, _pd, _pd, _pi32]),
    "sb2_diagnostics_record_size": (_i32, []),
    "sb2_propagator_set_loss_diagnostics": (_i32, [_vp, _i32]),
    "sb2_propagator_read_losses": (_i32, [_vp, _i32, _pi32, _pd]),
    "sb2_propagator_get_tune": (_i32, [_vp, _vp]),
    "sb2_propagator_set_tune": (_i32, [_vp, _vp]),
    "sb2_propagator_autotune": (_i32, [_vp, _vp, _i32, _vp, _pd, _i32, _pi32]),
    "sb2_propagator_set_step_counts": (_i32, [_vp, _vp, _i32]),
    "sb2_propagator_step_counts_written": (_i32, [_vp, _pi32]),
    "sb2_batch_query": (_i32, [_vp, _i32, _pi32]),
    "sb2_propagator_sc_last": (_i32, [_vp, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    "sb2_sc3d_create": (_i32, [_popts, _ppv]),
    "sb2_sc3d_destroy": (_i32, [_vp]),
    "sb2_sc3d_apply": (_i32, [_vp, _vp, _d, _vp]),
    "sb2_sc3d_last": (_i32, [_vp, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    "sb2_sc3d_apply_noalloc": (_i32, [_popts, _vp, _i64, _vp, _i64, _i32, _d, _i32, _d, _d, _i32, _d, _vp]),
    "sb2_allreduce_stream": (_vp, []),
    "sb2_propagator_prepare_steps": (_i32, [_vp, _vp, _i32, _i32, _vp]),
    "sb2_propagator_set_allreduce_typed": (_i32, [_vp, _vp, _vp, _i32]),
    "sb2_batch_run_lockstep": (_i32, [_vp, _pi32, _i32, _i32]),
    "sb2_libff_apply": (_i32, [_vp, _pd, _i32, _vp, _vp]),
    "sb2_aperture_apply": (_i32, [_vp, _i32, _cp, _vp, _pi32, _vp]),
}


class SB2Error(RuntimeError):
    """Raised when a C-ABI call returns a non-zero sb2_status; carries the
    library's message (the text the reference throws, where it throws)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("synergia2_b200: %s is not built (run python -m synergia2_b200.build)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


# sb2_allreduce_fn: int32_t (*)(void* ctx, double* data, int64_t count, int32_t on_host)
ALLREDUCE_FN = _c.CFUNCTYPE(_c.c_int32, _c.c_void_p, _c.POINTER(_c.c_double), _c.c_int64, _c.c_int32)
# sb2_allreduce_typed_fn: int32_t (*)(void* ctx, void* data, int64_t count, int32_t dtype, int32_t on_host)
ALLREDUCE_TYPED_FN = _c.CFUNCTYPE(_c.c_int32, _c.c_void_p, _c.c_void_p, _c.c_int64, _c.c_int32, _c.c_int32)


def check(rc):
    if rc != SB2_OK:
        raise SB2Error(rc, lib().sb2_last_error().decode())
    return rc
