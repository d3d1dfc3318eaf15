"""B200-native WENO reconstruction (MFC m_weno path of wilfonba/WenoStandalone).

The compute lives in libweno_sb.so (hand-written sm_100a CUDA behind the C
ABI of include/weno_sb.h).  This package is the host-side mirror of the
reference harness's interface plus input generators.
"""
from ._lib import (FP32, FP64, F_ACCUMULATE, F_FOLDED, F_MP, F_SPECIALIZED, F_SPLIT, JS, MAPPED, NONE, TENO, Z,
                   WenoError, lib)
from .api import Grid, Harness

__all__ = ["Grid", "Harness", "WenoError", "lib", "JS", "MAPPED", "Z", "TENO", "NONE", "FP64", "FP32",
           "F_SPLIT", "F_SPECIALIZED", "F_MP", "F_FOLDED", "F_ACCUMULATE"]
