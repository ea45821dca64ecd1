"""ctypes binding of libaq.so (declarations in include/aq.h).

The library is built in-tree by autoquantizer_b200/build.py.  Loading it
never falls back to anything else: if libaq.so is missing or fails to load,
`lib()` raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaq.so")

AQ_MAX_SLOTS = 32
AQ_MAX_GROUPS = 4
AQ_MAX_MATERIALS = 4

AQ_FIXED, AQ_INT, AQ_FLOAT_EXP, AQ_SHARED_EXP, AQ_RAW_F32, AQ_RAW_F64 = range(6)
AQ_MAT_FLUID, AQ_MAT_ELASTIC, AQ_MAT_COROTATED = range(3)
AQ_ST_OUT_OF_DOMAIN, AQ_ST_NAN, AQ_ST_FALLBACK, AQ_ST_POOL_FULL = 0x1, 0x2, 0x4, 0x8

ERRORS = {0: "ok", -1: "bad argument", -2: "layout does not fit the simulator schema", -3: "CUDA error",
          -4: "device allocation failed", -5: "call not valid in the current state",
          -6: "size above the documented maximum"}

# every symbol include/aq.h declares (checked by the CPU test suite)
EXPORTS = [
    "aq_layout_build", "aq_encode", "aq_decode", "aq_sim_create", "aq_sim_destroy", "aq_sim_set_state",
    "aq_sim_get_state", "aq_sim_set_words", "aq_sim_get_words", "aq_sim_substeps", "aq_sim_loss",
    "aq_sim_field_stats", "aq_sim_set_collider", "aq_sim_collider_get", "aq_sim_collider_pose",
    "aq_sim_collider_velocity_mode", "aq_sim_sparse_blocks", "aq_sim_grid_mass", "aq_voxelize", "aq_adjoint_set_collider",
    "aq_sim_ranges_enable", "aq_sim_ranges_get", "aq_sim_status", "aq_sim_step_count", "aq_sim_set_step_count", "aq_sim_launches",
    "aq_state_error", "aq_error_string", "aq_abi_version", "aq_sim_profile_enable", "aq_sim_profile_get",
    "aq_sim_kernel_is_jit", "aq_adjoint_create", "aq_adjoint_destroy", "aq_adjoint_forward", "aq_adjoint_backward",
    "aq_mlp_param_count", "aq_mlp_to_bf16", "aq_mlp_forward", "aq_mlp_backward", "aq_mlp_mse_grad", "aq_mlp_adam",
    "aq_state_error_noalloc", "aq_sim_create_streamed", "aq_sim_stream_set_words", "aq_sim_stream_get_words",
    "aq_sim_stream_chunks", "aq_sim_set_count", "aq_sim_append", "aq_sim_count",
]


class ScalarSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("bits", C.c_int32), ("is_signed", C.c_int32), ("exp_bits", C.c_int32),
                ("group", C.c_int32), ("_pad", C.c_int32), ("range", C.c_double), ("offset", C.c_double)]


class Slot(C.Structure):
    _fields_ = [("kind", C.c_int32), ("bits", C.c_int32), ("is_signed", C.c_int32), ("exp_bits", C.c_int32),
                ("bit_offset", C.c_int32), ("exp_offset", C.c_int32), ("group", C.c_int32),
                ("exp_first", C.c_int32), ("scale_f32", C.c_float), ("inv_scale_f32", C.c_float),
                ("offset_f32", C.c_float), ("_pad2", C.c_float), ("scale_f64", C.c_double),
                ("inv_scale_f64", C.c_double), ("offset_f64", C.c_double), ("_pad3", C.c_double)]


class Layout(C.Structure):
    _fields_ = [("n_slots", C.c_int32), ("n_words", C.c_int32), ("total_bits", C.c_int32),
                ("compute_f64", C.c_int32), ("use_dithering", C.c_int32), ("n_groups", C.c_int32),
                ("_pad", C.c_int32 * 2), ("slot", Slot * AQ_MAX_SLOTS)]


class Material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("_pad", C.c_int32), ("mu", C.c_double), ("lam", C.c_double)]


class Params(C.Structure):
    _fields_ = [("dim", C.c_int32), ("precision", C.c_int32), ("res", C.c_int32 * 3), ("has_F", C.c_int32),
                ("has_mat", C.c_int32), ("n_materials", C.c_int32), ("use_friction", C.c_int32),
                ("use_bound_clip", C.c_int32), ("sort_interval", C.c_int32), ("jit", C.c_int32),
                ("dx", C.c_double), ("dt", C.c_double), ("p_vol", C.c_double), ("p_mass", C.c_double),
                ("gravity", C.c_double), ("lb", C.c_double * 3), ("ub", C.c_double * 3),
                ("mat", Material * AQ_MAX_MATERIALS), ("n_particles", C.c_int64), ("seed", C.c_uint64),
                ("sparse", C.c_int32), ("reserved", C.c_int32)]


class AqError(RuntimeError):
    pass


_lib = None


def lib():
    """Load libaq.so (building it first if this is a source checkout without
    a built library)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build

        _build.build()
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
    sig = {
        "aq_layout_build": ([i32, C.POINTER(ScalarSpec), i32, i32, C.POINTER(Layout)], C.c_int),
        "aq_encode": ([C.POINTER(Layout), vp, i32, vp, i64, vp, u64, i64, vp, vp], C.c_int),
        "aq_decode": ([C.POINTER(Layout), vp, vp, i32, i64, vp], C.c_int),
        "aq_sim_create": ([C.POINTER(Params), C.POINTER(Layout), C.POINTER(vp)], C.c_int),
        "aq_sim_create_streamed": ([C.POINTER(Params), C.POINTER(Layout), i64, C.POINTER(vp)], C.c_int),
        "aq_sim_stream_set_words": ([vp, vp, vp], C.c_int),
        "aq_sim_stream_get_words": ([vp, vp, vp], C.c_int),
        "aq_sim_stream_chunks": ([vp, C.POINTER(i64), C.POINTER(i64)], C.c_int),
        "aq_sim_set_count": ([vp, i64], C.c_int),
        "aq_sim_append": ([vp, vp, i32, i64, vp], C.c_int),
        "aq_sim_count": ([vp, C.POINTER(i64), C.POINTER(i64)], C.c_int),
        "aq_sim_destroy": ([vp], C.c_int),
        "aq_sim_set_state": ([vp, vp, i32, vp], C.c_int),
        "aq_sim_get_state": ([vp, vp, i32, vp], C.c_int),
        "aq_sim_set_words": ([vp, vp, vp], C.c_int),
        "aq_sim_get_words": ([vp, vp, vp], C.c_int),
        "aq_sim_substeps": ([vp, i32, vp], C.c_int),
        "aq_sim_loss": ([vp, i32, C.POINTER(C.c_double), vp], C.c_int),
        "aq_sim_field_stats": ([vp, vp, i32, C.POINTER(C.c_double), vp], C.c_int),
        "aq_sim_grid_mass": ([vp, vp, vp], C.c_int),
        "aq_voxelize": ([vp, C.c_int64, C.POINTER(C.c_int32), C.c_double, i32, C.c_double, vp, vp], C.c_int),
        "aq_adjoint_set_collider": ([vp, vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), i32, C.c_double,
                                     C.c_double, C.c_double, C.c_double], C.c_int),
        "aq_sim_set_collider": ([vp, vp, vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), i32, C.c_double,
                                 C.c_double, C.c_double, C.c_double], C.c_int),
        "aq_sim_collider_get": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
        "aq_sim_collider_pose": ([vp, C.c_double, C.c_double], C.c_int),
        "aq_sim_collider_velocity_mode": ([vp, i32], C.c_int),
        "aq_sim_sparse_blocks": ([vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), vp], C.c_int),
        "aq_sim_ranges_enable": ([vp, i32, vp], C.c_int),
        "aq_sim_ranges_get": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_double), vp], C.c_int),
        "aq_sim_status": ([vp, C.POINTER(C.c_uint32), C.POINTER(C.c_int64), i32, vp], C.c_int),
        "aq_sim_step_count": ([vp, C.POINTER(C.c_int64)], C.c_int),
        "aq_sim_set_step_count": ([vp, i64], C.c_int),
        "aq_sim_launches": ([vp, C.POINTER(C.c_int64)], C.c_int),
        "aq_sim_kernel_is_jit": ([vp, C.POINTER(C.c_int32)], C.c_int),
        "aq_state_error": ([vp, i32, vp, i32, i64, i32, C.POINTER(C.c_double), C.POINTER(C.c_double), vp],
                           C.c_int),
        "aq_sim_profile_enable": ([vp, i32], C.c_int),
        "aq_sim_profile_get": ([vp, i32, C.POINTER(C.c_double), C.POINTER(C.c_int64)], C.c_int),
        "aq_adjoint_create": ([C.POINTER(Params), C.POINTER(vp)], C.c_int),
        "aq_adjoint_destroy": ([vp], C.c_int),
        "aq_adjoint_forward": ([vp, vp, i32, i32, vp, vp], C.c_int),
        "aq_adjoint_backward": ([vp, vp, vp, C.POINTER(C.c_double), vp], C.c_int),
        "aq_mlp_param_count": ([i32, i32, i32], i64),
        "aq_mlp_to_bf16": ([vp, vp, i64, vp], C.c_int),
        "aq_mlp_forward": ([i32, i32, i32, vp, vp, vp, i32, vp, vp, vp], C.c_int),
        "aq_mlp_backward": ([i32, i32, i32, vp, vp, i32, vp, vp, vp, vp], C.c_int),
        "aq_mlp_mse_grad": ([vp, vp, vp, vp, i64, C.c_float, vp, vp], C.c_int),
        "aq_mlp_adam": ([vp, vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, i32, vp], C.c_int),
        "aq_state_error_noalloc": ([vp, i32, vp, i32, i64, i32, C.POINTER(C.c_double), C.POINTER(C.c_double), vp],
                                   C.c_int),
        "aq_error_string": ([i32], C.c_char_p),
        "aq_abi_version": ([], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(rc, what=""):
    if rc != 0:
        msg = lib().aq_error_string(rc).decode()
        raise AqError("%s failed (%d): %s" % (what or "libaq call", rc, msg))
    return rc


def stream_ptr(stream=None):
    """cudaStream_t of a torch stream (or the current one) as an int."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)
