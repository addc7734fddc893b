"""ctypes binding of libkerrsplat_b200.so (the C ABI in include/kerrsplat_b200.h).

The library is loaded from this package directory only (built in-tree by kerrsplat_b200/build.py).
There is no fallback: if the shared library is missing or a GPU is absent, the calls raise.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkerrsplat_b200.so")

KS_OK = 0
KS_ERR_ARGUMENT = 1
KS_ERR_NOT_REGENERATED = 2
KS_ERR_OUT_OF_MEMORY = 3
KS_ERR_NONFINITE = 4
KS_ERR_DEVICE = 5
KS_ERR_TIMEOUT = 6

KS_FP64 = 0
KS_MIXED = 1
KS_MIXED_GEO64 = 2
KS_ORDER_SORTED = 0
KS_ORDER_SCREEN = 1

KS_THIN14 = 0
KS_THERMAL21 = 1
KS_POWERLAW22 = 2
KS_KAPPA22 = 3
KS_KNOT21 = 4

KS_NOALLOC_MAX_SPLATS = 256
KS_RIAF_PARAMS = 10

NROWS = {KS_THIN14: 14, KS_THERMAL21: 21, KS_POWERLAW22: 22, KS_KAPPA22: 22, KS_KNOT21: 21}

_D = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p


class SplatSetC(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("nsplat", ctypes.c_int32), ("params", _VP), ("hyp", _VP),
                ("knots", _VP), ("knot_times", _VP), ("nknots", ctypes.c_int32), ("gamma_max", ctypes.c_double)]


# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("ks_context_create", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP)]),
    ("ks_context_destroy", ctypes.c_int, [_VP]),
    ("ks_last_error", ctypes.c_char_p, [_VP]),
    ("ks_camera_set", ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32]),
    ("ks_regenerate", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32]),
    ("ks_regenerate_uneven", ctypes.c_int, [_VP, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32]),
    ("ks_get_nsamples", ctypes.c_int, [_VP, _VP]),
    ("ks_get_perm", ctypes.c_int, [_VP, _VP]),
    ("ks_get_ranges", ctypes.c_int, [_VP, _VP]),
    ("ks_get_residuals", ctypes.c_int, [_VP, _VP, _VP]),
    ("ks_get_ray_constants", ctypes.c_int, [_VP, _VP]),
    ("ks_march_samples", ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    ("ks_thin_image", ctypes.c_int, [_VP, _VP, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _VP, ctypes.c_int32]),
    ("ks_render", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32,
                                 ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _VP, ctypes.c_int32]),
    ("ks_visibilities", ctypes.c_int, [_VP, _VP, ctypes.c_int32, ctypes.c_int64, _VP, _VP, _VP, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, _VP]),
    ("ks_vis_seed", ctypes.c_int, [_VP, _VP, ctypes.c_int64, _VP, _VP, _VP, ctypes.c_double, ctypes.c_double, ctypes.c_int32, _VP,
                                   ctypes.c_int32]),
    ("ks_frame_chi2_seed", ctypes.c_int, [_VP, _VP, ctypes.c_int32, ctypes.c_int64, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int32, _D, _VP]),
    ("ks_adjoint", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32,
                                  ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _VP, ctypes.c_int32, _VP, ctypes.c_int32]),
    ("ks_jvp", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32,
                              ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _VP, ctypes.c_int32, _VP, ctypes.c_int32, _VP]),
    ("ks_vis_chi2_gradient", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int64, _VP, _VP, _VP,
                                            _VP, _VP, _VP, ctypes.c_double, ctypes.c_double, _VP, _VP, ctypes.c_int32, _VP]),
    ("ks_spacetime_derivatives", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32,
                                                ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _VP, _VP]),
    ("ks_normal_matrix", ctypes.c_int, [_VP, _VP, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, _VP]),
    ("ks_sample_adjoint", ctypes.c_int, [_VP, ctypes.c_int64, _VP, _VP, _VP, _VP, ctypes.c_int32, _VP]),
    ("ks_chi2_gradient", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32,
                                        ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _VP, _VP, ctypes.c_double, _VP,
                                        _VP, _VP, ctypes.c_int32, _VP]),
    ("ks_riaf_image", ctypes.c_int, [_VP, _VP, ctypes.c_int32, _VP, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _VP, ctypes.c_int32]),
]
# library extensions outside include/kerrsplat_b200.h's reference-facing set
EXTRA_SIGNATURES = [
    ("ks_context_stream", ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    ("ks_kernel_stats", ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    ("ks_set_event_counting", ctypes.c_int, [_VP, ctypes.c_int]),
    ("ks_event_counts", ctypes.c_int, [_VP, _VP]),
    ("ks_adjoint_stats", ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    ("ks_consume_stats", ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    ("ks_set_stage_test", ctypes.c_int, [_VP, ctypes.c_int32]),
    ("ks_set_tensor_path", ctypes.c_int, [_VP, ctypes.c_int32]),
    ("ks_gemm_stats", ctypes.c_int, [_VP, _D, ctypes.POINTER(ctypes.c_longlong), _D, ctypes.c_int]),
    ("ks_render_graph_capture", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32,
                                               ctypes.c_double, ctypes.c_int32, ctypes.c_double, _VP, ctypes.c_int32]),
    ("ks_graph_launch", ctypes.c_int, [_VP, ctypes.c_int32]),
    ("ks_chi2_gradient_graph_capture", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP,
                                                      ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_double, _VP, _VP,
                                                      ctypes.c_double, _VP, _VP, _VP, ctypes.c_int32]),
    ("ks_chi2_gradient_graph_launch", ctypes.c_int, [_VP, ctypes.c_int32]),
    ("ks_graph_destroy", ctypes.c_int, [_VP]),
    ("ks_autotune", ctypes.c_int, [_VP, ctypes.POINTER(SplatSetC), ctypes.c_int32, _VP, ctypes.c_int32, _VP, ctypes.c_int32, ctypes.c_double,
                                   ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_int32), _D]),
    ("ks_thin_image_noalloc", ctypes.c_int, [_VP, _VP, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _VP, ctypes.c_int32]),
]

_lib = None


def load():
    """Load the shared library (once) and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m kerrsplat_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES + EXTRA_SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class KsError(RuntimeError):
    """A failed library call; `status` is the C status code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


def check(status, ctx=None):
    """Raise the Python exception that corresponds to a C status code (the reference throws
    ArgumentError / DimensionMismatch at the same places, cache.jl:155-156, 203, 249-250)."""
    if status == KS_OK:
        return
    msg = load().ks_last_error(ctx).decode() if ctx else f"status {status}"
    if status == KS_ERR_ARGUMENT:
        raise ValueError(msg)
    if status == KS_ERR_NONFINITE:
        raise FloatingPointError(msg)
    if status == KS_ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise KsError(status, msg)
