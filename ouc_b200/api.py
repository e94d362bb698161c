"""Python mirror of the modeling / RTM operator surface (include/ouc.h).

The reference exposes no library API; its operator surface is the set of
kernels its main() drives (P-S-seperating.cu:2258-2376).  ``Context`` owns
one model on the device and offers the two operations that main() performs
per shot -- forward modeling with receiver extraction, and one RTM shot --
plus the cross-shot stack.  Arrays are numpy, x-major with z contiguous.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib

MODEL_INTERIOR, MODEL_PADDED = 0, 1
STRIP_REFERENCE, STRIP_EXACT = 0, 1
IMAGE_REFERENCE, IMAGE_EXACT = 0, 1
PREC_FP32, PREC_FP16, PREC_BF16 = 0, 1, 2
SRC_THETA, SRC_FORCE_Z = 0, 1
GATHER_XT, GATHER_TX = 0, 1
STEP_TILE_QUEUE = -1


@dataclass
class Config:
    nx: int
    nz: int
    npml: int
    dx: float
    dz: float
    dt: float
    nt: int
    half_order: int = 5
    pml_r: float = 1e-3
    model_layout: int = MODEL_INTERIOR
    strip_level: int = STRIP_REFERENCE
    image_align: int = IMAGE_REFERENCE
    strip_precision: int = PREC_FP32
    compensated_image: int = 0
    gather_layout: int = GATHER_XT
    device: int = 0
    stream: int = 0
    max_batch: int = 1
    snapshot_every: int = 0     # 0: strips + reconstruction; K: source snapshots every K imaging levels
    density: int = 0            # 1: variable density from rho (0: the reference's density-normalised equations)
    gradient: int = 0           # 1: RTM shots also accumulate the FWI gradient (Context.gradient)
    use_graphs: int = 1         # whole-shot time loops as CUDA graphs (captured once, replayed)

    def c(self):
        c = _lib.ouc_config()
        for name, _ in _lib.ouc_config._fields_:
            v = getattr(self, name)
            setattr(c, name, v if name != "stream" else (v or None))
        return c

    @property
    def X(self):
        return self.nx + 2 * self.npml

    @property
    def Z(self):
        return self.nz + 2 * self.npml


@dataclass
class Shot:
    sx: int
    sz: int
    rz: int
    src_type: int = SRC_THETA
    t0: int = 0
    mute: int = 1

    def c(self):
        return _lib.ouc_shot(self.sx, self.sz, self.rz, self.src_type, self.t0, self.mute)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def stencil_weights(n):
    out = np.zeros(n, np.float32)
    check(lib().ouc_stencil_weights(n, _p(out)))
    return out


def ricker(fm, dt, nt):
    """Ricker wavelet as the reference builds it (P-S-seperating.cu:1954-1958)."""
    out = np.zeros(nt, np.float32)
    t0 = C.c_int()
    check(lib().ouc_ricker(fm, dt, nt, _p(out), C.byref(t0)))
    return out, t0.value


class Context:
    """One model resident on one B200; shots run on the context's stream."""

    def __init__(self, cfg: Config, vp, vs, rho=None):
        self.cfg = cfg
        vp, vs = _f32(vp), _f32(vs)
        rho = None if rho is None else _f32(rho)
        want = (cfg.X, cfg.Z) if cfg.model_layout == MODEL_PADDED else (cfg.nx, cfg.nz)
        if vp.shape != want or vs.shape != want:
            raise ValueError(f"model shape {vp.shape} / {vs.shape}, expected {want}")
        h = C.c_void_p()
        cc = cfg.c()
        rc = lib().ouc_create(C.byref(cc), _p(vp), _p(vs), _p(rho), C.byref(h))
        if rc != 0:
            raise _lib.OucError(rc, "ouc_create")
        self._h = h
        X, Z = C.c_int(), C.c_int()
        check(lib().ouc_dims(h, C.byref(X), C.byref(Z)), h)
        self.X, self.Z = X.value, Z.value

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().ouc_destroy(self._h)
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

    @property
    def stream(self):
        return lib().ouc_stream(self._h)

    def device_bytes(self):
        return int(lib().ouc_device_bytes(self._h))

    def timing(self):
        t = _lib.ouc_timing()
        check(lib().ouc_last_timing(self._h, C.byref(t)), self._h)
        return dict(forward_ms=t.forward_ms, backward_ms=t.backward_ms, finalize_ms=t.finalize_ms,
                    copy_ms=t.copy_ms, kernel_launches=int(t.kernel_launches))

    def _gshape(self):
        nt = self.cfg.nt
        return (self.X, nt) if self.cfg.gather_layout == GATHER_XT else (nt, self.X)

    # ------------------------------------------------------------------
    def forward(self, shot: Shot, wavelet, fields=False):
        """Forward modeling: (gather_vx, gather_vz, fields or None).

        fields: final Ux, Uz, Px, Pz, Sx, Sz on the padded grid, (6, X, Z)."""
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        gx = np.zeros(self._gshape(), np.float32)
        gz = np.zeros(self._gshape(), np.float32)
        f = np.zeros((6, self.X, self.Z), np.float32) if fields else None
        sc = shot.c()
        check(lib().ouc_forward(self._h, C.byref(sc), _p(w), _p(gx), _p(gz), _p(f)), self._h)
        return gx, gz, f

    def forward_first_order(self, shot: Shot, wavelet, fields=False):
        """Forward modeling with the first-order velocity-stress scheme (the
        reference's stress/velocity kernels, P-S-seperating.cu:390-560):
        (gather_vx, gather_vz, fields or None).

        fields: final Vx Vz Vpx Vpz Vsx Vsz theta omega duzdx duzdz duxdx duxdz
        theta_x theta_z omega_x omega_z on the padded grid, (16, X, Z)."""
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        gx = np.zeros(self._gshape(), np.float32)
        gz = np.zeros(self._gshape(), np.float32)
        f = np.zeros((16, self.X, self.Z), np.float32) if fields else None
        sc = shot.c()
        check(lib().ouc_forward_fo(self._h, C.byref(sc), _p(w), _p(gx), _p(gz), _p(f)), self._h)
        return gx, gz, f

    def backward_first_order(self, shot: Shot, rec_vx, rec_vz):
        """Receiver back-propagation with the first-order scheme (the
        reference's *_backward_propagation kernels, P-S-seperating.cu:728-887,
        records written into U at the receiver row before each step, t = nt-1
        .. 0); rec_* in the configured gather layout.  Returns the final
        fields, (16, X, Z), in the order of forward_first_order."""
        rx, rz = _f32(rec_vx), _f32(rec_vz)
        assert rx.shape == self._gshape() and rz.shape == self._gshape()
        f = np.zeros((16, self.X, self.Z), np.float32)
        sc = shot.c()
        check(lib().ouc_backward_fo(self._h, C.byref(sc), _p(rx), _p(rz), _p(f)), self._h)
        return f

    def rtm_shot(self, shot: Shot, wavelet, rec=None):
        """One RTM shot; rec = (rec_vx, rec_vz) in the configured gather layout,
        or None to migrate the records this shot's own forward pass produces."""
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        rx = rz = None
        if rec is not None:
            rx, rz = _f32(rec[0]), _f32(rec[1])
            assert rx.shape == self._gshape() and rz.shape == self._gshape()
        pp = np.zeros((self.cfg.nx, self.cfg.nz), np.float32)
        ps = np.zeros((self.cfg.nx, self.cfg.nz), np.float32)
        sc = shot.c()
        check(lib().ouc_rtm_shot(self._h, C.byref(sc), _p(w), _p(rx), _p(rz), _p(pp), _p(ps)), self._h)
        return pp, ps

    def rtm_shot_dev(self, shot: Shot, d_wavelet, d_rec_vx=None, d_rec_vz=None, d_img_pp=None, d_img_ps=None):
        """Device-pointer variant (integers); no host copies."""
        sc = shot.c()
        check(lib().ouc_rtm_shot_dev(self._h, C.byref(sc), d_wavelet, d_rec_vx, d_rec_vz, d_img_pp, d_img_ps),
              self._h)

    def rtm_batch(self, shots, wavelet, recs=None):
        """RTM of several shots advanced together (up to cfg.max_batch per
        launch); recs = list of (rec_vx, rec_vz) or None.  Returns a list of
        (img_pp, img_ps)."""
        n = len(shots)
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        sh = (_lib.ouc_shot * n)(*[s.c() for s in shots])
        FP = C.POINTER(C.c_float)
        keep = []
        rx = rz = None
        if recs is not None:
            ax_ = [_f32(r[0]) for r in recs]
            az_ = [_f32(r[1]) for r in recs]
            for a_ in ax_ + az_:
                assert a_.shape == self._gshape()
            keep += ax_ + az_
            rx = (FP * n)(*[_p(a_) for a_ in ax_])
            rz = (FP * n)(*[_p(a_) for a_ in az_])
        imgs = [(np.zeros((self.cfg.nx, self.cfg.nz), np.float32), np.zeros((self.cfg.nx, self.cfg.nz), np.float32))
                for _ in range(n)]
        ipp = (FP * n)(*[_p(i[0]) for i in imgs])
        ips = (FP * n)(*[_p(i[1]) for i in imgs])
        check(lib().ouc_rtm_batch(self._h, n, sh, _p(w), rx, rz, ipp, ips), self._h)
        return imgs

    def rtm_batch_dev(self, shots, d_wavelet, d_rx=None, d_rz=None, d_ipp=None, d_ips=None):
        """Device-pointer variant: lists of device addresses (integers)."""
        n = len(shots)
        sh = (_lib.ouc_shot * n)(*[s.c() for s in shots])
        VP = C.c_void_p

        def arr(xs):
            return None if xs is None else (VP * n)(*xs)
        check(lib().ouc_rtm_batch_dev(self._h, n, sh, d_wavelet, arr(d_rx), arr(d_rz), arr(d_ipp), arr(d_ips)),
              self._h)

    # -- survey on per-shot sub-grids (the batching form)
    def _survey_args(self, shots, apertures):
        n = len(shots)
        if len(apertures) != n:
            raise ValueError("one aperture (x0, x1) per shot")
        sh = (_lib.ouc_shot * n)(*[s.c() for s in shots])
        ap = (_lib.ouc_aperture * n)(*[_lib.ouc_aperture(int(a[0]), int(a[1])) for a in apertures])
        return n, sh, ap

    def _sub_gshape(self, ap):
        Xb = ap[1] - ap[0] + 2 * self.cfg.npml
        nt = self.cfg.nt
        return (Xb, nt) if self.cfg.gather_layout == GATHER_XT else (nt, Xb)

    def survey_forward(self, shots, apertures, wavelet):
        """Forward modeling of shots on their sub-grids: apertures are interior
        column ranges (x0, x1) of this model; returns [(gather_vx, gather_vz)],
        each (x1 - x0 + 2 npml) wide."""
        n, sh, ap = self._survey_args(shots, apertures)
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        out = [(np.zeros(self._sub_gshape(a), np.float32), np.zeros(self._sub_gshape(a), np.float32)) for a in apertures]
        FP = C.POINTER(C.c_float)
        gx = (FP * n)(*[_p(o[0]) for o in out])
        gz = (FP * n)(*[_p(o[1]) for o in out])
        check(lib().ouc_survey_forward(self._h, n, sh, ap, _p(w), gx, gz), self._h)
        return out

    def survey_rtm(self, shots, apertures, wavelet, recs=None):
        """RTM of shots on their sub-grids; recs = [(rec_vx, rec_vz)] shaped as
        survey_forward's gathers, or None (self-modelled).  Returns
        [(img_pp, img_ps)], each (x1 - x0) x nz; all enter the FP64 stack."""
        n, sh, ap = self._survey_args(shots, apertures)
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        FP = C.POINTER(C.c_float)
        rx = rz = None
        keep = []
        if recs is not None:
            ax_ = [_f32(r[0]) for r in recs]
            az_ = [_f32(r[1]) for r in recs]
            for a_, b_, apk in zip(ax_, az_, apertures):
                assert a_.shape == self._sub_gshape(apk) and b_.shape == self._sub_gshape(apk)
            keep += ax_ + az_
            rx = (FP * n)(*[_p(a_) for a_ in ax_])
            rz = (FP * n)(*[_p(a_) for a_ in az_])
        imgs = [(np.zeros((a[1] - a[0], self.cfg.nz), np.float32), np.zeros((a[1] - a[0], self.cfg.nz), np.float32))
                for a in apertures]
        ipp = (FP * n)(*[_p(i[0]) for i in imgs])
        ips = (FP * n)(*[_p(i[1]) for i in imgs])
        check(lib().ouc_survey_rtm(self._h, n, sh, ap, _p(w), rx, rz, ipp, ips), self._h)
        return imgs

    def forward_dev(self, shot: Shot, d_wavelet, d_gx=None, d_gz=None):
        sc = shot.c()
        check(lib().ouc_forward_dev(self._h, C.byref(sc), d_wavelet, d_gx, d_gz), self._h)

    # -- step-level interface: one RTM shot, one reference time step per call
    def step_begin(self, shot: Shot, wavelet, recs=None):
        w = _f32(wavelet)
        assert w.shape == (self.cfg.nt,)
        rx = rz = None
        if recs is not None:
            rx, rz = _f32(recs[0]), _f32(recs[1])
            assert rx.shape == self._gshape() and rz.shape == self._gshape()
        sc = shot.c()
        check(lib().ouc_step_begin(self._h, C.byref(sc), _p(w), _p(rx), _p(rz)), self._h)

    def step_forward(self, t):
        check(lib().ouc_step_forward(self._h, int(t)), self._h)

    def step_receiver(self, t):
        check(lib().ouc_step_receiver(self._h, int(t)), self._h)

    def step_reconstruct(self, t):
        check(lib().ouc_step_reconstruct(self._h, int(t)), self._h)

    def image_finalize(self):
        pp = np.zeros((self.cfg.nx, self.cfg.nz), np.float32)
        ps = np.zeros_like(pp)
        check(lib().ouc_image_finalize(self._h, _p(pp), _p(ps)), self._h)
        return pp, ps

    def step_fields(self, side=0):
        """(6, X, Z): Ux, Uz, Px, Pz, Sx, Sz of the source (0) or receiver (1) side."""
        f = np.zeros((6, self.X, self.Z), np.float32)
        check(lib().ouc_step_fields(self._h, int(side), _p(f)), self._h)
        return f

    def stack_dev(self):
        """Device addresses of the context's FP64 stacks (PP, PS, illumination),
        each nx x nz, x-major; valid until the context is closed."""
        p = [C.c_void_p(), C.c_void_p(), C.c_void_p()]
        check(lib().ouc_stack_dev(self._h, C.byref(p[0]), C.byref(p[1]), C.byref(p[2])), self._h)
        return tuple(q.value for q in p)

    def gradient(self, reset=False):
        """FP64 stacks of the FWI gradient w.r.t. Vp and Vs and of the source
        illumination, each nx x nz (cfg.gradient = 1)."""
        n = (self.cfg.nx, self.cfg.nz)
        gp, gs, il = np.zeros(n), np.zeros(n), np.zeros(n)
        dp = C.POINTER(C.c_double)
        check(lib().ouc_gradient(self._h, gp.ctypes.data_as(dp), gs.ctypes.data_as(dp), il.ctypes.data_as(dp),
                                 int(reset)), self._h)
        return gp, gs, il

    def set_step_kernel(self, seg_rows):
        """Step-kernel geometry (ouc_set_step_kernel): 0 the 32 x 64 tile
        kernel, STEP_TILE_QUEUE (-1) the tile kernel as a persistent launch
        with a dynamic tile queue, or x-marching segments of seg_rows rows
        (a multiple of 16)."""
        check(lib().ouc_set_step_kernel(self._h, int(seg_rows)), self._h)

    def time_step_kernels(self, n, reps=10):
        """Device ms per launch of the forward, receiver and reconstruction
        step kernels at batch n, on the state of the last RTM batch."""
        ms = np.zeros(3, np.float32)
        check(lib().ouc_time_step_kernels(self._h, int(n), int(reps), _p(ms)), self._h)
        return [float(x) for x in ms]

    def debug_copy_stall(self, on):
        """Test hook (ouc_debug_copy_stall): make the tile kernels' bounded
        copy waits run out, so that the next call reports OUC_ETIMEOUT."""
        check(lib().ouc_debug_copy_stall(self._h, int(bool(on))), self._h)

    def step_kernel(self):
        v = C.c_int()
        check(lib().ouc_get_step_kernel(self._h, C.byref(v)), self._h)
        return v.value

    def stack(self, reset=False):
        n = (self.cfg.nx, self.cfg.nz)
        pp, ps, il = np.zeros(n), np.zeros(n), np.zeros(n)
        dp = C.POINTER(C.c_double)
        check(lib().ouc_stack(self._h, pp.ctypes.data_as(dp), ps.ctypes.data_as(dp), il.ctypes.data_as(dp),
                              int(reset)), self._h)
        return pp, ps, il
