"""ctypes binding of libweno_sb.so (declared in include/weno_sb.h).

The shared library is the product: every compute call goes to its CUDA
kernels.  If the library is missing this module raises instead of falling
back to anything else.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libweno_sb.so")

# status codes (include/weno_sb.h)
OK = 0
ERR_ARG = 1001
ERR_HANDLE = 1002
ERR_UNSUPPORTED = 1003
ERR_INJECTED = 1004
ERR_TIMEOUT = 1005
ERR_ALIGN = 1006
ERR_HOST = 1007

# weight families
JS, MAPPED, Z, TENO, NONE = 0, 1, 2, 3, 4
# storage precision
FP64, FP32 = 0, 1
# flags
F_SPLIT, F_SPECIALIZED, F_MP, F_FOLDED, F_ACCUMULATE = 1, 2, 4, 8, 16

# array ids of the handle API
A_V_VF = 0


def A_RS(d): return 1 + d
def A_VL(d): return 4 + d
def A_VR(d): return 7 + d
def A_POLYL(d): return 10 + d
def A_POLYR(d): return 13 + d
def A_DL(d): return 16 + d
def A_DR(d): return 19 + d
def A_BETA(d): return 22 + d


A_COUNT = 25

# Every symbol include/weno_sb.h declares.
EXPORTED = [
    "weno_sb_version", "weno_sb_last_error_string", "weno_sb_extents",
    "weno_sb_init", "weno_sb_finalize", "weno_sb_upload", "weno_sb_upload_async", "weno_sb_download",
    "weno_sb_array_info", "weno_sb_initialize_weno", "weno_sb_weno",
    "weno_sb_preserve_monotonicity", "weno_sb_vjp", "weno_sb_checksum", "weno_sb_sync",
    "weno_sb_stream", "weno_sb_reshape_dev", "weno_sb_order1_dev",
    "weno_sb_weno_dev", "weno_sb_weno_uniform_dev", "weno_sb_vjp_dev", "weno_sb_preserve_monotonicity_dev",
    "weno_sb_checksum_scratch_bytes", "weno_sb_checksum_dev", "weno_sb_check_device",
    "weno_sb_selftest_rcp", "weno_sb_selftest_timeout", "weno_sb_checksum_noalloc",
    "weno_sb_coefficients", "weno_sb_batch_create", "weno_sb_batch_autotune", "weno_sb_batch_launch", "weno_sb_batch_destroy",
    "weno_sb_batch_configure", "weno_sb_batch_query",
]


class WenoGrid(ctypes.Structure):
    """struct weno_sb_grid (the &grid_params namelist, f90:117-118)."""
    _fields_ = [
        ("m_cells", ctypes.c_int32), ("n_cells", ctypes.c_int32), ("p_cells", ctypes.c_int32),
        ("v_size", ctypes.c_int32), ("buff_size", ctypes.c_int32), ("scheme", ctypes.c_int32),
        ("weno_eps", ctypes.c_double), ("teno_CT", ctypes.c_double),
    ]


class WenoCoefs(ctypes.Structure):
    """struct weno_sb_coefs: device pointers of one direction's coefficients."""
    _fields_ = [("polyL", ctypes.c_void_p), ("polyR", ctypes.c_void_p), ("dL", ctypes.c_void_p),
                ("dR", ctypes.c_void_p), ("beta_coef", ctypes.c_void_p)]


class WenoFaceCoefs(ctypes.Structure):
    """struct weno_sb_face_coefs: one face's coefficients on the host,
    index order [s][r] (polyL(j,r,s) -> polyL[s][r])."""
    _fields_ = [("polyL", (ctypes.c_double * 5) * 3), ("polyR", (ctypes.c_double * 5) * 3),
                ("dL", ctypes.c_double * 5), ("dR", ctypes.c_double * 5),
                ("beta_coef", (ctypes.c_double * 5) * 6)]


class WenoBlock(ctypes.Structure):
    """struct weno_sb_block: one entry of a batch."""
    _fields_ = [("grid", WenoGrid), ("dir", ctypes.c_int32), ("order", ctypes.c_int32),
                ("flags", ctypes.c_uint32), ("dtype", ctypes.c_int32), ("v_in", ctypes.c_void_p),
                ("coefs", WenoCoefs), ("vL", ctypes.c_void_p), ("vR", ctypes.c_void_p)]


class WenoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"weno_sb error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> ctypes.CDLL:
    """Load libweno_sb.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -m wenostandalone_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    i32, u32, vp, dp = ctypes.c_int, ctypes.c_uint, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    gp = ctypes.POINTER(WenoGrid)
    i64p = ctypes.POINTER(ctypes.c_int64)
    sig = {
        "weno_sb_version": ([], i32),
        "weno_sb_last_error_string": ([], ctypes.c_char_p),
        "weno_sb_extents": ([gp, i32, i64p, i64p, i64p], i32),
        "weno_sb_init": ([gp, i32, ctypes.POINTER(ctypes.c_int)], i32),
        "weno_sb_finalize": ([i32], i32),
        "weno_sb_upload": ([i32, i32, vp], i32),
        "weno_sb_upload_async": ([i32, i32, vp], i32),
        "weno_sb_download": ([i32, i32, vp], i32),
        "weno_sb_array_info": ([i32, i32, ctypes.POINTER(ctypes.c_void_p), i64p, ctypes.POINTER(ctypes.c_int)], i32),
        "weno_sb_initialize_weno": ([i32, i32], i32),
        "weno_sb_weno": ([i32, i32, i32, u32], i32),
        "weno_sb_preserve_monotonicity": ([i32, i32], i32),
        "weno_sb_vjp": ([i32, i32, i32, u32, vp, vp, vp], i32),
        "weno_sb_checksum": ([i32, i32, dp], i32),
        "weno_sb_sync": ([i32], i32),
        "weno_sb_stream": ([i32, ctypes.POINTER(ctypes.c_void_p)], i32),
        "weno_sb_reshape_dev": ([gp, i32, i32, vp, vp, vp], i32),
        "weno_sb_order1_dev": ([gp, i32, i32, vp, vp, vp, vp], i32),
        "weno_sb_weno_dev": ([gp, i32, i32, u32, i32, vp, ctypes.POINTER(WenoCoefs), vp, vp, vp], i32),
        "weno_sb_weno_uniform_dev": ([gp, i32, i32, u32, i32, vp, ctypes.POINTER(WenoFaceCoefs), vp, vp, vp], i32),
        "weno_sb_vjp_dev": ([gp, i32, i32, u32, vp, ctypes.POINTER(WenoCoefs), ctypes.POINTER(WenoFaceCoefs),
                             vp, vp, vp, vp], i32),
        "weno_sb_preserve_monotonicity_dev": ([gp, i32, i32, vp, vp, vp, vp], i32),
        "weno_sb_checksum_scratch_bytes": ([ctypes.c_int64], ctypes.c_size_t),
        "weno_sb_checksum_dev": ([i32, vp, ctypes.c_int64, vp, vp, vp], i32),
        "weno_sb_check_device": ([vp], i32),
        "weno_sb_selftest_rcp": ([vp, vp, vp, ctypes.c_int64, vp], i32),
        "weno_sb_selftest_timeout": ([ctypes.c_int64, vp], i32),
        "weno_sb_checksum_noalloc": ([i32, ctypes.POINTER(ctypes.c_void_p), i64p, i32, vp, vp], i32),
        "weno_sb_coefficients": ([i32, ctypes.c_int64, vp, vp, vp, vp, vp, vp], i32),
        "weno_sb_batch_create": ([ctypes.POINTER(WenoBlock), i32, ctypes.POINTER(ctypes.c_int)], i32),
        "weno_sb_batch_autotune": ([i32, vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_double)], i32),
        "weno_sb_batch_launch": ([i32, vp], i32),
        "weno_sb_batch_destroy": ([i32], i32),
        "weno_sb_batch_configure": ([i32, i32, i32, i32, i32], i32),
        "weno_sb_batch_query": ([i32, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def last_error() -> str:
    s = lib().weno_sb_last_error_string()
    return s.decode() if s else ""


def check(rc: int) -> None:
    if rc != OK:
        raise WenoError(rc, last_error())
