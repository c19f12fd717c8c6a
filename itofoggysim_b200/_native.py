"""ctypes binding of libfoggy_b200.so (the C ABI declared in include/foggy_gpu.h).

The library is the only compute path: if it is missing or cannot be loaded this module raises,
it never falls back to a CPU implementation.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfoggy_b200.so")

FOGGY_OK = 0
FOGGY_ERR_ARGUMENT = -1
FOGGY_ERR_STATE = -2
FOGGY_ERR_CUDA = -3
FOGGY_ERR_NOMEM = -4
FOGGY_ERR_NOT_CONVERGED = -5
FOGGY_ERR_BREAKDOWN = -6
FOGGY_ERR_NAN = -7
FOGGY_ERR_UNSUPPORTED = -8
STATUS_NAMES = {0: "OK", -1: "ARGUMENT", -2: "STATE", -3: "CUDA", -4: "NOMEM", -5: "NOT_CONVERGED",
                -6: "BREAKDOWN", -7: "NAN", -8: "UNSUPPORTED"}

FOGGY_MEM_HOST = 0
FOGGY_MEM_DEVICE = 1
FOGGY_MATVEC_DIRECT = 0
FOGGY_MATVEC_MLFMM = 1

# every symbol include/foggy_gpu.h declares
EXPORTS = [
    "foggy_default_params", "foggy_create", "foggy_destroy", "foggy_last_error", "foggy_set_params",
    "foggy_set_spheres", "foggy_set_plane_waves", "foggy_vector_length", "foggy_get_mie_coefficients",
    "foggy_get_vector_b", "foggy_matvec", "foggy_solve", "foggy_get_backward_error",
    "foggy_cross_sections", "foggy_translation_coefficients", "foggy_wigner_3j", "foggy_build_tree",
    "foggy_universal_index", "foggy_tree_boxes", "foggy_matvec_static", "foggy_tree_domain",
    "foggy_get_field", "foggy_set_gaussian_beams", "foggy_solve_rhs", "foggy_server_start",
    "foggy_server_submit", "foggy_server_poll", "foggy_server_cancel", "foggy_server_release",
    "foggy_server_stop", "foggy_matvec_rhs", "foggy_tree_parent", "foggy_tree_children",
    "foggy_tree_centre_of_box", "foggy_tree_neighbours", "foggy_estimate_solve_bytes", "foggy_solve_block",
    "foggy_matvec_block", "foggy_block_tiles", "foggy_fmm_lists",
]


class FoggyParams(C.Structure):
    _fields_ = [
        ("lambda_0", C.c_double),
        ("n_medium", C.c_double),
        ("n_range", C.c_int32 * 2),
        ("z_coupling", C.c_int32),
        ("reference_row_rule", C.c_int32),
        ("matvec_mode", C.c_int32),
        ("use_initial_guess", C.c_int32),
        ("gmres_restart", C.c_int32),
        ("gmres_max_iterations", C.c_int32),
        ("gmres_tolerance", C.c_double),
        ("tree_l_max", C.c_int32),
        ("tree_s_opt", C.c_int32),
        ("fmm_digits", C.c_double),
        ("device_memory_budget", C.c_int64),
        ("pair_tables", C.c_int32),
        ("fmm_convention", C.c_int32),
        ("z_translation_gt_r", C.c_int32),
        ("precision", C.c_int32),
    ]


class FoggyStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("restarts", C.c_int32),
        ("matvecs", C.c_int32),
        ("status", C.c_int32),
        ("backward_error", C.c_double),
        ("ms_total", C.c_double),
        ("ms_matvec", C.c_double),
        ("ms_setup", C.c_double),
        ("kernel_launches", C.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FoggyRequest(C.Structure):
    _fields_ = [
        ("params", C.POINTER(FoggyParams)),
        ("n_spheres", C.c_int32),
        ("centres", C.c_void_p),
        ("param_index", C.c_void_p),
        ("n_param", C.c_int32),
        ("refractive_index", C.c_void_p),
        ("radius", C.c_void_p),
        ("n_range", C.c_void_p),
        ("nw", C.c_int32),
        ("theta", C.c_void_p),
        ("phi", C.c_void_p),
        ("jones", C.c_void_p),
        ("g", C.c_void_p),
        ("phase", C.c_void_p),
        ("d_0_i", C.c_void_p),
        ("rhs_per_wave", C.c_int32),
    ]


class FoggyRequestInfo(C.Structure):
    _fields_ = [
        ("state", C.c_int32),
        ("status", C.c_int32),
        ("nrhs", C.c_int32),
        ("reserved", C.c_int32),
        ("x_len", C.c_int64),
        ("footprint", C.c_int64),
        ("ms_queued", C.c_double),
        ("ms_solve", C.c_double),
        ("ms_latency", C.c_double),
        ("stats", FoggyStats),
        ("error", C.c_char * 256),
    ]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED, REQ_REFUSED = range(6)


class FoggyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS_NAMES.get(code, "?"), code, msg))
        self.code = code


_lib = None


def load():
    """Load libfoggy_b200.so; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfoggy_b200.so is not built (run python -m itofoggysim_b200.build); "
                          "there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    pd = C.POINTER(C.c_double)
    pi32 = C.POINTER(C.c_int32)
    pi64 = C.POINTER(C.c_int64)
    sig = {
        "foggy_default_params": (None, [C.POINTER(FoggyParams)]),
        "foggy_create": (i32, [C.POINTER(FoggyParams), i32, C.POINTER(vp)]),
        "foggy_destroy": (i32, [vp]),
        "foggy_last_error": (C.c_char_p, [vp]),
        "foggy_set_params": (i32, [vp, C.POINTER(FoggyParams)]),
        "foggy_set_spheres": (i32, [vp, i32, pd, pi32, i32, pd, pd, pi32]),
        "foggy_set_plane_waves": (i32, [vp, i32, pd, pd, pd, pd, pd, pd]),
        "foggy_vector_length": (i64, [vp]),
        "foggy_get_mie_coefficients": (i32, [vp, i32, pd, pd]),
        "foggy_get_vector_b": (i32, [vp, vp, i32]),
        "foggy_matvec": (i32, [vp, vp, vp, i32]),
        "foggy_solve": (i32, [vp, vp, vp, i32, C.POINTER(FoggyStats)]),
        "foggy_get_backward_error": (dbl, [vp]),
        "foggy_cross_sections": (i32, [vp, vp, i32, pd]),
        "foggy_translation_coefficients": (i32, [dbl, dbl, dbl, pi32, pi32, i32, pd, pd]),
        "foggy_wigner_3j": (dbl, [i32] * 6),
        "foggy_build_tree": (i32, [vp, pi64, pi32, pi32, pi32]),
        "foggy_universal_index": (i32, [i32, pd, i32, pi64]),
        "foggy_tree_boxes": (i32, [vp, i32, pi64, pi32]),
        "foggy_matvec_static": (i32, [vp, vp, vp]),
        "foggy_tree_domain": (i32, [vp, i32, i64, i32, pi64, pi32]),
        "foggy_get_field": (i32, [vp, vp, i32, i32, vp, dbl, vp, vp]),
        "foggy_set_gaussian_beams": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "foggy_solve_rhs": (i32, [vp, i32, vp, vp, i32, C.POINTER(FoggyStats), vp]),
        "foggy_server_start": (i32, [i32, i32, i64, C.POINTER(vp)]),
        "foggy_server_submit": (i32, [vp, C.POINTER(FoggyRequest), pi64]),
        "foggy_server_poll": (i32, [vp, i64, i32, C.POINTER(FoggyRequestInfo), vp, i64, vp]),
        "foggy_server_cancel": (i32, [vp, i64]),
        "foggy_server_release": (i32, [vp, i64]),
        "foggy_server_stop": (i32, [vp]),
        "foggy_matvec_rhs": (i32, [vp, i32, vp, vp, i32]),
        "foggy_tree_parent": (i32, [i64, i32, i32, pi64]),
        "foggy_tree_children": (i32, [i64, i32, pi64]),
        "foggy_tree_centre_of_box": (i32, [i64, i32, pd]),
        "foggy_tree_neighbours": (i32, [i64, i32, pi64, pi32]),
        "foggy_estimate_solve_bytes": (i32, [C.POINTER(FoggyParams), i32, pi32, i32, pi32, pi64, pi64]),
        "foggy_solve_block": (i32, [vp, i32, vp, vp, i32, C.POINTER(FoggyStats), vp, vp, vp]),
        "foggy_matvec_block": (i32, [vp, i32, i32, vp, vp, i32]),
        "foggy_block_tiles": (i32, [vp, i32, i32, pi32, pi32]),
        "foggy_fmm_lists": (i32, [vp, i32, pi32, pi32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def ptr(a, ctype=C.c_double):
    """Pointer to the data of a contiguous numpy array (complex arrays as interleaved doubles)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def check(rc, handle=None):
    if rc != FOGGY_OK:
        msg = load().foggy_last_error(handle)
        raise FoggyError(rc, msg.decode() if msg else "")
    return rc


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def as_c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)
