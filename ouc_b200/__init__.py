"""ouc_b200 -- B200-native elastic P/S-decoupled finite-difference modeling
and reverse-time migration (sm_100a CUDA kernels behind the C ABI of
include/ouc.h).  See ``api.Context``.
"""
from .api import (Config, Context, Shot, ricker, stencil_weights, MODEL_INTERIOR, MODEL_PADDED, STRIP_REFERENCE,
                  STRIP_EXACT, IMAGE_REFERENCE, IMAGE_EXACT, PREC_FP32, PREC_FP16, PREC_BF16, SRC_THETA, SRC_FORCE_Z,
                  GATHER_XT, GATHER_TX)
from ._lib import LIB_PATH, OucError, lib

__all__ = ["Config", "Context", "Shot", "ricker", "stencil_weights", "lib", "LIB_PATH", "OucError"]
