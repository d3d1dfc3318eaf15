"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle.

The oracle (``weno_oracle.c``) restates the reference harness
wilfonba/WenoStandalone ``inputs/weno_standalone.f90`` on the CPU.  Only the
test suite, the smoke check and the bench's CPU-baseline / reference arm use
this module; the product library never imports it.

Arrays are numpy float64 in Fortran (column-major) order with the shapes of
the reference's allocations (first index fastest):

* ``v_vf``            (N1+6, N2+6, N3+6, V)              f90:163-165
* sweep input ``rs``  (ns+6, c1, c2, V)                  f90:167-169
* sweep output        (ns, c1, c2, V)                    f90:1779-1784
* ``poly``            (nc, 5, 3), ``d`` (5, nc), ``beta`` (nc, 5, 6)
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libweno_oracle.so")

JS, MAPPED, Z, TENO, NONE = 0, 1, 2, 3, 4

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        i = ctypes.c_int
        L.wo_fill_input_field.argtypes = [i, i, i, i, i, dp]
        L.wo_fill_input_field.restype = None
        L.wo_fill_coefficients.argtypes = [i, ctypes.c_double, dp, dp, dp, dp, dp]
        L.wo_fill_coefficients.restype = None
        L.wo_reshape.argtypes = [i, i, i, i, i, i, dp, dp]
        L.wo_reshape.restype = i
        L.wo_order1_copy.argtypes = [i, i, i, i, i, i, dp, dp, dp]
        L.wo_order1_copy.restype = i
        L.wo_reconstruct.argtypes = [i, i, i, i, i, i, ctypes.c_double, ctypes.c_double,
                                     dp, dp, dp, dp, dp, dp, dp, dp]
        L.wo_reconstruct.restype = i
        L.wo_teno_margin.argtypes = [i, i, i, i, i, ctypes.c_double, ctypes.c_double, dp, dp, dp]
        L.wo_teno_margin.restype = i
        L.wo_preserve_monotonicity.argtypes = [i, i, i, i, dp, dp, dp]
        L.wo_preserve_monotonicity.restype = i
        L.wo_checksum.argtypes = [ctypes.c_longlong, dp]
        L.wo_checksum.restype = ctypes.c_double
        L.wo_harness_run.argtypes = [i, i, i, i, i, ctypes.c_double, i, ctypes.c_double, i, dp]
        L.wo_harness_run.restype = i
        L.wo_vjp.argtypes = [i, i, i, i, i, i, i, ctypes.c_double, ctypes.c_double,
                             dp, dp, dp, dp, dp, dp, dp, dp, dp]
        L.wo_vjp.restype = i
        L.wo_set_threads.argtypes = [i]
        L.wo_set_threads.restype = None
        L.wo_get_threads.argtypes = []
        L.wo_get_threads.restype = i
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.f_contiguous, "need Fortran-ordered float64"
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n: int) -> None:
    lib().wo_set_threads(int(n))


def get_threads() -> int:
    return int(lib().wo_get_threads())


def extents(m, n, p, buff, direction):
    """(ns, c1, c2) of a direction's sweep arrays."""
    N1, N2, N3 = m + 2 * buff + 1, n + 2 * buff + 1, p + 2 * buff + 1
    return {0: (N1, N2, N3), 1: (N2, N1, N3), 2: (N3, N2, N1)}[direction]


def fill_input_field(m, n, p, nv, buff) -> np.ndarray:
    """f90:221-244: the harness's synthetic field."""
    a = np.empty((m + 2 * buff + 7, n + 2 * buff + 7, p + 2 * buff + 7, nv), order="F")
    lib().wo_fill_input_field(m, n, p, nv, buff, _p(a))
    return a


def fill_coefficients(nc, offset):
    """f90:246-279: (polyL, polyR, dL, dR, beta)."""
    pL = np.empty((nc, 5, 3), order="F")
    pR = np.empty((nc, 5, 3), order="F")
    dL = np.empty((5, nc), order="F")
    dR = np.empty((5, nc), order="F")
    bc = np.empty((nc, 5, 6), order="F")
    lib().wo_fill_coefficients(nc, float(offset), _p(pL), _p(pR), _p(dL), _p(dR), _p(bc))
    return pL, pR, dL, dR, bc


def reshape(v_vf, m, n, p, buff, direction) -> np.ndarray:
    """f90:281-330: s_initialize_weno_{x,y,z}."""
    nv = v_vf.shape[3]
    ns, c1, c2 = extents(m, n, p, buff, direction)
    out = np.empty((ns + 6, c1, c2, nv), order="F")
    rc = lib().wo_reshape(m, n, p, nv, buff, direction, _p(v_vf), _p(out))
    assert rc == 0
    return out


def order1_copy(v_vf, m, n, p, buff, direction, vL=None, vR=None):
    """f90:332-390: s_order1_copy_{x,y,z}."""
    nv = v_vf.shape[3]
    ns, c1, c2 = extents(m, n, p, buff, direction)
    if vL is None:
        vL = np.empty((ns, c1, c2, nv), order="F")
    if vR is None:
        vR = np.empty((ns, c1, c2, nv), order="F")
    rc = lib().wo_order1_copy(m, n, p, nv, buff, direction, _p(v_vf), _p(vL), _p(vR))
    assert rc == 0
    return vL, vR


def reconstruct(rs, coefs, order, scheme=JS, eps=1e-16, teno_ct=1e-5, vL=None, vR=None):
    """f90:392-475 (order 3), 477-669 (order 5), 1419-1542 (order 7).

    ``vL``/``vR`` are updated in place on the faces the order writes (all
    faces for WENO3, core faces for WENO5/7) and returned.
    """
    ns6, c1, c2, nv = rs.shape
    ns = ns6 - 6
    if vL is None:
        vL = np.zeros((ns, c1, c2, nv), order="F")
    if vR is None:
        vR = np.zeros((ns, c1, c2, nv), order="F")
    pL, pR, dL, dR, bc = coefs
    rc = lib().wo_reconstruct(ns, c1, c2, nv, order, scheme, float(eps), float(teno_ct),
                              _p(rs), _p(pL), _p(pR), _p(dL), _p(dR), _p(bc), _p(vL), _p(vR))
    assert rc == 0, rc
    return vL, vR


def teno_margin(rs, coefs, order, eps=1e-16, teno_ct=1e-5):
    """Per face of the sweep output layout: min over the TENO cutoff tests of
    |omega_q - CT| / CT (f90:578-590 for WENO5, f90:1491-1506 for WENO7),
    +inf outside the core.  A cutoff decision can only differ between two
    correct implementations where this is at rounding level."""
    ns6, c1, c2, nv = rs.shape
    out = np.empty((ns6 - 6, c1, c2, nv), order="F")
    rc = lib().wo_teno_margin(ns6 - 6, c1, c2, nv, order, float(eps), float(teno_ct), _p(rs),
                              _p(np.asfortranarray(coefs[4])), _p(out))
    assert rc == 0, rc
    return out


def preserve_monotonicity(rs, vL, vR):
    """f90:1544-1615: MP limiter, in place on the core faces."""
    ns6, c1, c2, nv = rs.shape
    rc = lib().wo_preserve_monotonicity(ns6 - 6, c1, c2, nv, _p(rs), _p(vL), _p(vR))
    assert rc == 0
    return vL, vR


def checksum(a: np.ndarray) -> float:
    """f90:1617-1620: sum(abs(arr)) in array order."""
    a = np.asfortranarray(a)
    return float(lib().wo_checksum(a.size, _p(a)))


def harness_run(m=199, n=199, p=199, nv=8, buff=6, eps=1e-16, scheme=JS, teno_ct=1e-5,
                all_mode=False):
    """The driver's golden path (f90:1734-1861 with WENO_KERNEL_MODE=weno5,
    scope=full, warmup 0, bench 1) or its 'all' path; returns (X, Y, Z, T)."""
    out = np.zeros(4)
    rc = lib().wo_harness_run(m, n, p, nv, buff, float(eps), scheme, float(teno_ct),
                              1 if all_mode else 0,
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0, rc
    return tuple(float(x) for x in out)


def vjp(rs, coefs, order, gL, gR, scheme=JS, mp=False, eps=1e-16, teno_ct=1e-5):
    """Adjoint of one sweep by forward-mode dual numbers on the reference
    formulas (weno_oracle_ad.cpp): gv = (dF/dv)^T (gL, gR), layout of rs."""
    ns6, c1, c2, nv = rs.shape
    gv = np.zeros(rs.shape, order="F")
    pL, pR, dL, dR, bc = coefs
    gL = np.asfortranarray(gL)
    gR = np.asfortranarray(gR)
    rc = lib().wo_vjp(ns6 - 6, c1, c2, nv, order, scheme, 1 if mp else 0, float(eps), float(teno_ct),
                      _p(rs), _p(pL), _p(pR), _p(dL), _p(dR), _p(bc), _p(gL), _p(gR), _p(gv))
    assert rc == 0, rc
    return gv
