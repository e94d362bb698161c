"""The learned coarse path (include/ouc_corrector.h): a half-order-2 run at
twice the spacing and time step, corrected every few steps by a small CNN
trained on fine/coarse pairs that the method itself generates; the fine
half-order-5 run is the referee (sparse spot-check traces) and the fallback.

``Twin`` holds a fine context and its coarse twin on one model; ``pairs``
generates training data on the GPU, ``train`` fits the network (tensor-core
kernels, Adam), ``model_shots`` runs a survey of shots on the coarse path with
the spot check and the fine-grid fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import _lib
from ._lib import check, lib
from .api import Config, Context, Shot, GATHER_TX, _f32, _p
from .corrector import Net, N_IN, N_OUT, WIDTH

LAYERS = [(N_IN, WIDTH), (WIDTH, WIDTH), (WIDTH, WIDTH), (WIDTH, N_OUT)]
TAPS = 25


def init_params(seed=0, out_scale=0.1):
    """He-normal weights (the last layer scaled by out_scale so the first
    corrections are small), zero biases: the layout of ouc_cnn_set_params."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, (ci, co) in enumerate(LAYERS):
        w = rng.normal(0.0, np.sqrt(2.0 / (ci * TAPS)), co * ci * TAPS)
        if k == len(LAYERS) - 1:
            w *= out_scale
        parts += [w, np.zeros(co)]
    return np.concatenate(parts).astype(np.float32)


def coarse_config(fine: Config) -> Config:
    """The coarse twin of a fine configuration: half the cells (and absorbing
    width), twice the spacing and time step, half the steps, half-order 2."""
    if fine.nx % 2 or fine.nz % 2 or fine.npml % 2 or fine.nt % 2:
        raise ValueError("fine nx, nz, npml and nt must be even")
    return replace(fine, nx=fine.nx // 2, nz=fine.nz // 2, npml=fine.npml // 2, dx=2 * fine.dx, dz=2 * fine.dz,
                   dt=2 * fine.dt, nt=fine.nt // 2, half_order=2, max_batch=1, snapshot_every=0)


def coarse_wavelet(w_fine, nt_coarse):
    w = _f32(w_fine)
    out = np.zeros(nt_coarse, np.float32)
    check(lib().ouc_coarse_wavelet(_p(w), int(nt_coarse), _p(out)))
    return out


def coarse_shot(s: Shot) -> Shot:
    if (s.sx | s.sz | s.rz) & 1:
        raise ValueError("fine shot coordinates must be even")
    return replace(s, sx=s.sx // 2, sz=s.sz // 2, rz=s.rz // 2)


class Twin:
    """A fine context (half-order 5 by default) and its coarse twin on one
    model (vp, vs interior nx x nz of the fine grid)."""

    def __init__(self, fine_cfg: Config, vp, vs):
        self.fine_cfg = fine_cfg
        self.coarse_cfg = coarse_config(fine_cfg)
        vp, vs = _f32(vp), _f32(vs)
        self.fine = Context(fine_cfg, vp, vs)
        self.coarse = Context(self.coarse_cfg, np.ascontiguousarray(vp[::2, ::2]), np.ascontiguousarray(vs[::2, ::2]))

    def close(self):
        self.fine.close()
        self.coarse.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def H(self):
        return self.coarse.X

    @property
    def W(self):
        return self.coarse.Z

    def interior(self):
        L = self.coarse_cfg.npml
        return L, self.coarse.X - L, L, self.coarse.Z - L

    def pairs(self, shot: Shot, w_fine, every, d_in, d_tgt, max_pairs, net: Net | None = None, noise=0.0, seed=0):
        """Training pairs of one fine shot into device buffers (addresses);
        returns how many were written.  net None: each interval starts from the
        fine solution; otherwise from the coarse state `net` corrected.  noise:
        relative size of the input perturbation (augmentation)."""
        n = C.c_int()
        sc = shot.c()
        w = _f32(w_fine)
        check(lib().ouc_learned_pairs(self.fine.handle, self.coarse.handle, net.handle if net else None, C.byref(sc),
                                      _p(w), int(every), float(noise), int(seed) & 0xFFFFFFFF, int(max_pairs), d_in,
                                      d_tgt, C.byref(n)), self.coarse.handle)
        return n.value

    def _gshape(self, X, nt, cfg):
        return (nt, X) if cfg.gather_layout == GATHER_TX else (X, nt)

    def coarse_forward(self, shot: Shot, w_fine, net: Net | None, every=8):
        """Coarse gathers (X_c x nt_c in the gather layout) of the fine shot,
        corrected by `net` every `every` steps (net None: plain coarse run)."""
        cfg = self.coarse_cfg
        wc = coarse_wavelet(w_fine, cfg.nt)
        gx = np.zeros(self._gshape(self.coarse.X, cfg.nt, cfg), np.float32)
        gz = np.zeros_like(gx)
        sc = coarse_shot(shot).c()
        check(lib().ouc_forward_learned(self.coarse.handle, net.handle if net else None, C.byref(sc), _p(wc),
                                        int(every), _p(gx), _p(gz)), self.coarse.handle)
        return gx, gz

    def fine_forward_restricted(self, shot: Shot, w_fine):
        """The fine run's gathers as the coarse grid sees them (the referee)."""
        cfg = self.coarse_cfg
        gx = np.zeros(self._gshape(self.coarse.X, cfg.nt, self.fine_cfg), np.float32)
        gz = np.zeros_like(gx)
        sc = shot.c()
        w = _f32(w_fine)
        check(lib().ouc_forward_restricted(self.fine.handle, C.byref(sc), _p(w), int(cfg.nt), _p(gx), _p(gz)),
              self.fine.handle)
        return gx, gz


def train(net: Net, d_in, d_tgt, npairs, H, W, rect, batch=4, epochs=10, lr=1e-3, seed=0):
    """Fit the network on device pairs (addresses); returns the per-epoch loss."""
    loss = np.zeros(epochs, np.float32)
    i0, i1, j0, j1 = rect
    rc = lib().ouc_cnn_train(net.handle, d_in, d_tgt, int(npairs), int(H), int(W), int(i0), int(i1), int(j0), int(j1),
                             int(batch), int(epochs), float(lr), int(seed) & 0xFFFFFFFF, _p(loss), None)
    if rc != 0:
        raise _lib.OucError(rc, "ouc_cnn_train")
    if net.error():
        raise _lib.OucError(_lib.OUC_ETIMEOUT, "a corrector kernel wait ran out")
    return loss


def trace_error(g, ref, cols, interior_x, layout_tx=False):
    """Relative L2 misfit over the spot-check receiver columns `cols`
    (interior receiver indices) of two (vx, vz) gather pairs."""
    L0 = interior_x
    num = den = 0.0
    for a, b in zip(g, ref):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        if layout_tx:
            a, b = a.T, b.T
        a = a[[L0 + c for c in cols]]
        b = b[[L0 + c for c in cols]]
        num += float(np.sum((a - b) ** 2))
        den += float(np.sum(b ** 2))
    return float(np.sqrt(num / max(den, 1e-300)))


@dataclass
class ShotResult:
    gathers: tuple          # coarse-grid (vx, vz) gathers delivered for the shot
    checked: bool           # spot-checked against the fine run
    error: float | None     # spot-check trace misfit (checked shots)
    fallback: bool          # the fine run's gathers were delivered instead


def model_shots(twin: Twin, net: Net, shots, w_fine, every=8, check_every=4, ntrace=8, tol=0.01):
    """Forward-model `shots` on the learned coarse path.  Every
    `check_every`-th shot is spot-checked: the fine half-order-5 run is made
    and `ntrace` evenly spaced receiver traces of the two are compared; a
    checked shot whose misfit exceeds `tol` is replaced by the fine run (the
    fallback), and so is every unchecked shot that follows a failed check
    until the next check passes."""
    nxc = twin.coarse_cfg.nx
    cols = list(np.linspace(0, nxc - 1, ntrace).astype(int))
    tx = twin.coarse_cfg.gather_layout == GATHER_TX
    out = []
    failing = False
    for k, s in enumerate(shots):
        g = twin.coarse_forward(s, w_fine, net, every)
        if k % check_every == 0:
            ref = twin.fine_forward_restricted(s, w_fine)
            e = trace_error(g, ref, cols, twin.coarse_cfg.npml, tx)
            failing = e > tol
            out.append(ShotResult(ref if failing else g, True, e, failing))
        elif failing:
            out.append(ShotResult(twin.fine_forward_restricted(s, w_fine), False, None, True))
        else:
            out.append(ShotResult(g, False, None, False))
    return out
