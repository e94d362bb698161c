"""ctypes binding of libouc.so (include/ouc.h).

The shared library is built in-tree (``make -C ouc_b200`` or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libouc.so")

OUC_OK, OUC_EINVAL, OUC_ECUDA, OUC_ENOMEM, OUC_EUNSTABLE, OUC_ESTATE, OUC_ETIMEOUT, OUC_ENODEV, OUC_ESCRATCH = range(9)


class ouc_config(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("npml", C.c_int), ("half_order", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float), ("nt", C.c_int), ("pml_r", C.c_double),
                ("model_layout", C.c_int), ("strip_level", C.c_int), ("image_align", C.c_int),
                ("strip_precision", C.c_int), ("compensated_image", C.c_int), ("gather_layout", C.c_int),
                ("device", C.c_int), ("stream", C.c_void_p), ("max_batch", C.c_int), ("snapshot_every", C.c_int),
                ("density", C.c_int), ("gradient", C.c_int), ("use_graphs", C.c_int)]


class ouc_shot(C.Structure):
    _fields_ = [("sx", C.c_int), ("sz", C.c_int), ("rz", C.c_int), ("src_type", C.c_int), ("t0", C.c_int),
                ("mute", C.c_int)]


class ouc_aperture(C.Structure):
    _fields_ = [("x0", C.c_int), ("x1", C.c_int)]


class ouc_timing(C.Structure):
    _fields_ = [("forward_ms", C.c_float), ("backward_ms", C.c_float), ("finalize_ms", C.c_float),
                ("copy_ms", C.c_float), ("kernel_launches", C.c_longlong)]


_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_vp = C.c_void_p

# name -> (restype, argtypes); every symbol include/ouc.h declares
SIGNATURES = {
    "ouc_strerror": (C.c_char_p, [C.c_int]),
    "ouc_last_error": (C.c_char_p, [_vp]),
    "ouc_version": (C.c_int, []),
    "ouc_stencil_weights": (C.c_int, [C.c_int, _fp]),
    "ouc_ricker": (C.c_int, [C.c_float, C.c_float, C.c_int, _fp, C.POINTER(C.c_int)]),
    "ouc_create": (C.c_int, [C.POINTER(ouc_config), _fp, _fp, _fp, C.POINTER(_vp)]),
    "ouc_destroy": (C.c_int, [_vp]),
    "ouc_dims": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ouc_set_step_kernel": (C.c_int, [_vp, C.c_int]),
    "ouc_tune": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "ouc_get_step_kernel": (C.c_int, [_vp, C.POINTER(C.c_int)]),
    "ouc_debug_copy_stall": (C.c_int, [_vp, C.c_int]),
    "ouc_time_step_kernels": (C.c_int, [_vp, C.c_int, C.c_int, _fp]),
    "ouc_stream": (_vp, [_vp]),
    "ouc_last_timing": (C.c_int, [_vp, C.POINTER(ouc_timing)]),
    "ouc_device_bytes": (C.c_size_t, [_vp]),
    "ouc_forward": (C.c_int, [_vp, C.POINTER(ouc_shot), _fp, _fp, _fp, _fp]),
    "ouc_forward_dev": (C.c_int, [_vp, C.POINTER(ouc_shot), _vp, _vp, _vp]),
    "ouc_forward_fo": (C.c_int, [_vp, C.POINTER(ouc_shot), _fp, _fp, _fp, _fp]),
    "ouc_backward_fo": (C.c_int, [_vp, C.POINTER(ouc_shot), _fp, _fp, _fp]),
    "ouc_rtm_shot": (C.c_int, [_vp, C.POINTER(ouc_shot), _fp, _fp, _fp, _fp, _fp]),
    "ouc_rtm_shot_dev": (C.c_int, [_vp, C.POINTER(ouc_shot), _vp, _vp, _vp, _vp, _vp]),
    "ouc_rtm_batch": (C.c_int, [_vp, C.c_int, C.POINTER(ouc_shot), _fp, C.POINTER(_fp), C.POINTER(_fp),
                                C.POINTER(_fp), C.POINTER(_fp)]),
    "ouc_rtm_batch_dev": (C.c_int, [_vp, C.c_int, C.POINTER(ouc_shot), _vp, C.POINTER(_vp), C.POINTER(_vp),
                                    C.POINTER(_vp), C.POINTER(_vp)]),
    "ouc_survey_forward": (C.c_int, [_vp, C.c_int, C.POINTER(ouc_shot), C.POINTER(ouc_aperture), _fp, C.POINTER(_fp),
                                     C.POINTER(_fp)]),
    "ouc_survey_rtm": (C.c_int, [_vp, C.c_int, C.POINTER(ouc_shot), C.POINTER(ouc_aperture), _fp, C.POINTER(_fp),
                                 C.POINTER(_fp), C.POINTER(_fp), C.POINTER(_fp)]),
    "ouc_tune_batch": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "ouc_set_run_batch": (C.c_int, [_vp, C.c_int]),
    "ouc_forward_noalloc": (C.c_int, [C.POINTER(ouc_config), C.POINTER(ouc_shot), _vp, _vp, _vp, _vp, _vp]),
    "ouc_stack": (C.c_int, [_vp, _dp, _dp, _dp, C.c_int]),
    "ouc_gradient": (C.c_int, [_vp, _dp, _dp, _dp, C.c_int]),
    "ouc_stack_dev": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
    "ouc_step_begin": (C.c_int, [_vp, C.POINTER(ouc_shot), _fp, _fp, _fp]),
    "ouc_step_forward": (C.c_int, [_vp, C.c_int]),
    "ouc_step_receiver": (C.c_int, [_vp, C.c_int]),
    "ouc_step_reconstruct": (C.c_int, [_vp, C.c_int]),
    "ouc_image_finalize": (C.c_int, [_vp, _fp, _fp]),
    "ouc_step_fields": (C.c_int, [_vp, C.c_int, _fp]),
    # include/ouc_corrector.h
    "ouc_cnn_nparams": (C.c_int, []),
    "ouc_cnn_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "ouc_cnn_destroy": (C.c_int, [_vp]),
    "ouc_cnn_set_params": (C.c_int, [_vp, _fp]),
    "ouc_cnn_get_params": (C.c_int, [_vp, _fp]),
    "ouc_cnn_forward_dev": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp]),
    "ouc_cnn_backward_dev": (C.c_int, [_vp, _vp, _vp]),
    "ouc_cnn_zero_grad": (C.c_int, [_vp, _vp]),
    "ouc_cnn_get_grads": (C.c_int, [_vp, _fp]),
    "ouc_cnn_adam_step": (C.c_int, [_vp, C.c_float, C.c_float, C.c_float, C.c_float, _vp]),
    "ouc_cnn_error": (C.c_int, [_vp]),
    "ouc_cnn_train": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_float, C.c_uint, _fp, _vp]),
    "ouc_coarse_wavelet": (C.c_int, [_fp, C.c_int, _fp]),
    "ouc_forward_learned": (C.c_int, [_vp, _vp, C.POINTER(ouc_shot), _fp, C.c_int, _fp, _fp]),
    "ouc_forward_restricted": (C.c_int, [_vp, C.POINTER(ouc_shot), _fp, C.c_int, _fp, _fp]),
    "ouc_learned_pairs": (C.c_int, [_vp, _vp, _vp, C.POINTER(ouc_shot), _fp, C.c_int, C.c_float, C.c_uint, C.c_int,
                                    _vp, _vp, C.POINTER(C.c_int)]),
}

_lib = None


def lib() -> C.CDLL:
    """Load libouc.so once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `make -C {HERE}` (needs nvcc for sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class OucError(RuntimeError):
    def __init__(self, code, detail=""):
        self.code = code
        msg = lib().ouc_strerror(code).decode()
        super().__init__(f"ouc error {code} ({msg}){': ' + detail if detail else ''}")


def check(code, ctx=None):
    if code != OUC_OK:
        detail = lib().ouc_last_error(ctx).decode() if ctx else ""
        raise OucError(code, detail)
