"""Python mirror of the learned corrector's C ABI (include/ouc_corrector.h).

``Net`` owns the network on one GPU; images are device arrays given as
integer addresses (e.g. ``torch.Tensor.data_ptr()``), NHWC float32.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import lib

N_IN, WIDTH, N_OUT = 10, 32, 8


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(rc, what):
    if rc != 0:
        raise _lib.OucError(rc, what)


class Net:
    def __init__(self, device=0, params=None):
        h = C.c_void_p()
        _check(lib().ouc_cnn_create(device, C.byref(h)), "ouc_cnn_create")
        self._h = h
        self.n = lib().ouc_cnn_nparams()
        if params is not None:
            self.set_params(params)

    def close(self):
        if getattr(self, "_h", None):
            lib().ouc_cnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.shape == (self.n,)
        _check(lib().ouc_cnn_set_params(self._h, _fp(p)), "ouc_cnn_set_params")

    def params(self):
        p = np.zeros(self.n, np.float32)
        _check(lib().ouc_cnn_get_params(self._h, _fp(p)), "ouc_cnn_get_params")
        return p

    def grads(self):
        g = np.zeros(self.n, np.float32)
        _check(lib().ouc_cnn_get_grads(self._h, _fp(g)), "ouc_cnn_get_grads")
        return g

    def forward_dev(self, n, H, W, d_in, d_out, stream=None):
        _check(lib().ouc_cnn_forward_dev(self._h, n, H, W, d_in, d_out, stream), "ouc_cnn_forward_dev")

    def backward_dev(self, d_gout, stream=None):
        _check(lib().ouc_cnn_backward_dev(self._h, d_gout, stream), "ouc_cnn_backward_dev")

    def zero_grad(self, stream=None):
        _check(lib().ouc_cnn_zero_grad(self._h, stream), "ouc_cnn_zero_grad")

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        _check(lib().ouc_cnn_adam_step(self._h, lr, beta1, beta2, eps, stream), "ouc_cnn_adam_step")

    def error(self):
        return lib().ouc_cnn_error(self._h)
