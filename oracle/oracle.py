"""TEST INFRASTRUCTURE -- ctypes access to the CPU oracle and the reference builds.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, always as a checker or as the timed CPU baseline; the product
(ouc_b200) never does.

* ``Oracle`` wraps oracle/liboracle.so: the plain C++/OpenMP restatement of the
  launched kernels of P-S-seperating.cu, in float (bit-exact against the
  reference's kernels run on the CPU) and double (the FP64 oracle).
* ``RefBuild`` wraps oracle/_ref/libpsref_{emu,cuda}_<cfg>.so: the reference's
  own kernels with its launch sequence (oracle/refemu/ref_harness.inc), either
  emulated on the CPU or compiled for sm_100a.  Their grid sizes are fixed at
  compile time (oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


class OrcCfg(C.Structure):
    _fields_ = [("X", C.c_int), ("Z", C.c_int), ("L", C.c_int), ("N", C.c_int), ("nt", C.c_int),
                ("sx", C.c_int), ("sz", C.c_int), ("rz", C.c_int), ("t0", C.c_int),
                ("strip_level", C.c_int), ("image_align", C.c_int), ("do_mute", C.c_int),
                ("src_in_recon", C.c_int),
                ("dx", C.c_float), ("dz", C.c_float), ("dt", C.c_float), ("dh", C.c_float),
                ("coeff", C.c_float * 8), ("src_type", C.c_int)]


def _ptr(a, kind=np.float32):
    if a is None:
        return None
    assert a.dtype == kind and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_fp if kind == np.float32 else _dp)


def weights(n):
    """float32 staggered weights a_1..a_N (oracle/coeffs.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("orc_coeffs", os.path.join(HERE, "coeffs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return np.array(mod.float32_weights(n), dtype=np.float32)


def weights_first_order(n):
    """float32 weights of the reference's first-order kernels (oracle/coeffs.py)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("orc_coeffs", os.path.join(HERE, "coeffs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return np.array(mod.float32_weights_first_order(n), dtype=np.float32)


@dataclass
class Shot:
    X: int
    Z: int
    L: int
    N: int
    nt: int
    sx: int
    sz: int
    rz: int
    dx: float
    dz: float
    dt: float
    t0: int = 0
    strip_level: int = 0
    image_align: int = 0
    do_mute: int = 1
    src_in_recon: int = 0
    src_type: int = 0      # 0: theta source (the reference's); 1: vertical force on Uz

    def cfg(self) -> OrcCfg:
        c = OrcCfg()
        for k in ("X", "Z", "L", "N", "nt", "sx", "sz", "rz", "t0", "strip_level", "image_align", "do_mute",
                  "src_in_recon", "src_type"):
            setattr(c, k, int(getattr(self, k)))
        c.dx, c.dz, c.dt, c.dh = self.dx, self.dz, self.dt, self.dx
        w = weights(self.N)
        for k in range(8):
            c.coeff[k] = float(w[k]) if k < self.N else 0.0
        return c


class Oracle:
    def __init__(self, path=None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        self.lib = C.CDLL(path)
        for name, t in (("orc_forward_f32", _fp), ("orc_forward_f64", _dp)):
            f = getattr(self.lib, name)
            f.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, t, t, t]
            f.restype = C.c_int
        for name, t in (("orc_rtm_f32", _fp), ("orc_rtm_f64", _dp)):
            f = getattr(self.lib, name)
            f.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, _fp, _fp, t, t, t, t, t, t, t]
            f.restype = C.c_int
        self.lib.orc_forward_rho_f64.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, _fp, _dp, _dp, _dp]
        self.lib.orc_forward_rho_f64.restype = C.c_int
        self.lib.orc_rtm_rho_f64.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _dp, _dp, _dp,
                                             _dp, _dp, _dp, _dp]
        self.lib.orc_rtm_rho_f64.restype = C.c_int
        for name, t in (("orc_forward_fo_f32", _fp), ("orc_forward_fo_f64", _dp)):
            f = getattr(self.lib, name)
            f.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, t, t, t]
            f.restype = C.c_int
        for name, t in (("orc_backward_fo_f32", _fp), ("orc_backward_fo_f64", _dp)):
            f = getattr(self.lib, name)
            f.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, _fp, t]
            f.restype = C.c_int
        for name, t in (("orc_rtm_grad_f32", _fp), ("orc_rtm_grad_f64", _dp)):
            f = getattr(self.lib, name)
            f.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, t, t, t]
            f.restype = C.c_int
        self.lib.orc_pad_model.argtypes = [_fp, C.c_int, C.c_int, C.c_int]
        self.lib.orc_cpml_profile.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_double, _fp, _fp]
        self.lib.orc_num_threads.restype = C.c_int
        self.lib.orc_rtm_stored_f64.argtypes = [C.POINTER(OrcCfg), _fp, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, _dp, _dp,
                                                _dp]
        self.lib.orc_rtm_stored_f64.restype = C.c_int
        self.lib.orc_ricker.argtypes = [C.c_float, C.c_float, C.c_int, _fp, C.POINTER(C.c_int)]
        self.lib.orc_ricker.restype = C.c_int
        self.lib.orc_set_threads.argtypes = [C.c_int]

    def threads(self, n=None):
        if n:
            self.lib.orc_set_threads(int(n))
        return self.lib.orc_num_threads()

    def ricker(self, fm, dt, nt):
        """Ricker wavelet of the reference's main() (PS:1954-1958) and its delay t0."""
        out = np.zeros(nt, np.float32)
        t0 = C.c_int()
        if self.lib.orc_ricker(fm, dt, nt, _ptr(out), C.byref(t0)):
            raise ValueError("bad Ricker parameters")
        return out, t0.value

    def pad(self, a, L):
        a = np.ascontiguousarray(a, dtype=np.float32).copy()
        self.lib.orc_pad_model(_ptr(a), a.shape[0], a.shape[1], L)
        return a

    def profile(self, vp, L, R=1e-3):
        vp = np.ascontiguousarray(vp, dtype=np.float32)
        ax = np.zeros_like(vp)
        az = np.zeros_like(vp)
        self.lib.orc_cpml_profile(_ptr(vp), vp.shape[0], vp.shape[1], L, R, _ptr(ax), _ptr(az))
        return ax, az

    def forward(self, shot: Shot, vp, vs, ax, az, src, fp64=False, rho=None):
        """rho (padded density): the variable-density extension, FP64 only."""
        dt = np.float64 if fp64 or rho is not None else np.float32
        X, Z, nt = shot.X, shot.Z, shot.nt
        rx = np.zeros((X, nt), dt)
        rz = np.zeros((X, nt), dt)
        fields = np.zeros((12, X, Z), dt)
        c = shot.cfg()
        if rho is not None:
            rc = self.lib.orc_forward_rho_f64(C.byref(c), _ptr(vp), _ptr(vs), _ptr(rho), _ptr(ax), _ptr(az), _ptr(src),
                                              _ptr(rx, dt), _ptr(rz, dt), _ptr(fields, dt))
            assert rc == 0
            return rx, rz, fields
        f = self.lib.orc_forward_f64 if fp64 else self.lib.orc_forward_f32
        rc = f(C.byref(c), _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(src), _ptr(rx, dt), _ptr(rz, dt),
               _ptr(fields, dt))
        assert rc == 0
        return rx, rz, fields

    def forward_fo(self, shot: Shot, vp, vs, ax, az, src, fp64=False):
        """First-order velocity-stress forward modeling (the reference's
        stress/velocity kernels): (rec_vx, rec_vz, fields[16])."""
        dt = np.float64 if fp64 else np.float32
        X, Z, nt = shot.X, shot.Z, shot.nt
        rx = np.zeros((X, nt), dt)
        rz = np.zeros((X, nt), dt)
        fields = np.zeros((16, X, Z), dt)
        c = shot.cfg()
        for k, w in enumerate(weights_first_order(shot.N)):
            c.coeff[k] = float(w)
        f = self.lib.orc_forward_fo_f64 if fp64 else self.lib.orc_forward_fo_f32
        rc = f(C.byref(c), _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(src), _ptr(rx, dt), _ptr(rz, dt),
               _ptr(fields, dt))
        assert rc == 0
        return rx, rz, fields

    def backward_fo(self, shot: Shot, vp, vs, ax, az, rec_vx, rec_vz, fp64=False):
        """First-order receiver back-propagation (the reference's
        *_backward_propagation kernels, records injected at the receiver row
        for t = nt-1 .. 0): fields[16] after the step at t = 0.  rec_*: X x nt."""
        dt = np.float64 if fp64 else np.float32
        fields = np.zeros((16, shot.X, shot.Z), dt)
        c = shot.cfg()
        for k, w in enumerate(weights_first_order(shot.N)):
            c.coeff[k] = float(w)
        f = self.lib.orc_backward_fo_f64 if fp64 else self.lib.orc_backward_fo_f32
        rc = f(C.byref(c), _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(np.ascontiguousarray(rec_vx, np.float32)),
               _ptr(np.ascontiguousarray(rec_vz, np.float32)), _ptr(fields, dt))
        assert rc == 0
        return fields

    def rtm_stored(self, shot: Shot, vp, vs, ax, az, src, every=1, rec=None):
        """FP64 RTM from the stored source wavefield of every `every`-th imaging
        level (no reconstruction): the reference of the snapshot form.  Keeps
        nt/every x 2 x nx x nz doubles."""
        X, Z, nt, L = shot.X, shot.Z, shot.nt, shot.L
        nx, nz = X - 2 * L, Z - 2 * L
        out = dict(lap_pp=np.zeros((nx, nz)), lap_ps=np.zeros((nx, nz)), acc=np.zeros((3, X, Z)))
        rx = rz = None
        if rec is not None:
            rx = np.ascontiguousarray(rec[0], dtype=np.float32)
            rz = np.ascontiguousarray(rec[1], dtype=np.float32)
        c = shot.cfg()
        rc = self.lib.orc_rtm_stored_f64(C.byref(c), _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(src), _ptr(rx),
                                         _ptr(rz), int(every), _ptr(out["lap_pp"], np.float64),
                                         _ptr(out["lap_ps"], np.float64), _ptr(out["acc"], np.float64))
        assert rc == 0
        return out

    def rtm(self, shot: Shot, vp, vs, ax, az, src, rec=None, fp64=False, rho=None):
        """rho (padded density): the variable-density extension, FP64 only."""
        dt = np.float64 if fp64 or rho is not None else np.float32
        X, Z, nt, L = shot.X, shot.Z, shot.nt, shot.L
        nx, nz = X - 2 * L, Z - 2 * L
        out = dict(lap_pp=np.zeros((nx, nz), dt), lap_ps=np.zeros((nx, nz), dt), img_pp=np.zeros((X, Z), dt),
                   img_ps=np.zeros((X, Z), dt), acc=np.zeros((3, X, Z), dt), rec=np.zeros((2, X, nt), dt),
                   fields=np.zeros((12, X, Z), dt))
        rx = rz = None
        if rec is not None:
            rx = np.ascontiguousarray(rec[0], dtype=np.float32)
            rz = np.ascontiguousarray(rec[1], dtype=np.float32)
        c = shot.cfg()
        outs = [_ptr(out[k], dt) for k in ("lap_pp", "lap_ps", "img_pp", "img_ps", "acc", "rec", "fields")]
        if rho is not None:
            rc = self.lib.orc_rtm_rho_f64(C.byref(c), _ptr(vp), _ptr(vs), _ptr(rho), _ptr(ax), _ptr(az), _ptr(src),
                                          _ptr(rx), _ptr(rz), *outs)
        else:
            f = self.lib.orc_rtm_f64 if fp64 else self.lib.orc_rtm_f32
            rc = f(C.byref(c), _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(src), _ptr(rx), _ptr(rz), *outs)
        assert rc == 0
        return out


def _none_or(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def rtm_gradient(orc, shot, vp, vs, ax, az, src, rec=None, rho=None, fp64=True):
    """RTM with the FWI gradient: (lap_pp, lap_ps, grad [3][X][Z]) -- gradient
    w.r.t. Vp, w.r.t. Vs and the source illumination of one shot."""
    dt = np.float64 if fp64 else np.float32
    X, Z, L = shot.X, shot.Z, shot.L
    lpp = np.zeros((X - 2 * L, Z - 2 * L), dt)
    lps = np.zeros_like(lpp)
    grad = np.zeros((3, X, Z), dt)
    rx = rz = None
    if rec is not None:
        rx, rz = _none_or(rec[0]), _none_or(rec[1])
    f = orc.lib.orc_rtm_grad_f64 if fp64 else orc.lib.orc_rtm_grad_f32
    c = shot.cfg()
    rc = f(C.byref(c), _ptr(vp), _ptr(vs), _ptr(_none_or(rho)), _ptr(ax), _ptr(az), _ptr(src), _ptr(rx), _ptr(rz),
           _ptr(lpp, dt), _ptr(lps, dt), _ptr(grad, dt))
    assert rc == 0
    return lpp, lps, grad


class RefBuild:
    """The reference's kernels, compiled with fixed sizes (emu: CPU, cuda: sm_100a)."""

    def __init__(self, name, kind="emu"):
        path = os.path.join(REF_DIR, f"libpsref_{kind}_{name}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference is mounted")
        self.lib = C.CDLL(path)
        ip = C.POINTER(C.c_int)
        self.lib.psr_info.argtypes = [ip, ip, ip, ip, ip]
        v = [C.c_int() for _ in range(5)]
        self.lib.psr_info(*[C.byref(x) for x in v])
        self.X, self.Z, self.L, self.N, self.NT = [x.value for x in v]
        self.lib.psr_pad.argtypes = [_fp, _fp, _fp]
        self.lib.psr_forward.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _fp, _fp, _fp,
                                         _fp, _fp, C.c_int, _fp, _fp, _fp, _fp]
        self.lib.psr_forward.restype = C.c_int
        self.lib.psr_forward_fo.argtypes = self.lib.psr_forward.argtypes
        self.lib.psr_forward_fo.restype = C.c_int
        self.lib.psr_backward_fo.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, _fp, _fp, _fp, _fp, _fp, _fp,
                                             C.c_int, _fp, _fp]
        self.lib.psr_backward_fo.restype = C.c_int
        self.lib.psr_rtm_shot.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                          C.c_float, _fp, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, _fp, _fp, _fp,
                                          _fp, _fp, _fp, _fp, _fp]
        self.lib.psr_rtm_shot.restype = C.c_int

    def pad(self, P, vp, vs):
        P, vp, vs = (np.ascontiguousarray(a, dtype=np.float32).copy() for a in (P, vp, vs))
        self.lib.psr_pad(_ptr(P), _ptr(vp), _ptr(vs))
        return P, vp, vs

    def forward(self, sx, sz, rz, dt, dx, dz, vp, vs, ax, az, src, nt_run):
        X, Z, NT = self.X, self.Z, self.NT
        src_full = np.zeros(NT, np.float32)
        src_full[: len(src)] = src[:NT]
        rx = np.zeros((X, NT), np.float32)
        rzr = np.zeros((X, NT), np.float32)
        fields = np.zeros((12, X, Z), np.float32)
        ms = np.zeros(1, np.float32)
        rc = self.lib.psr_forward(sx, sz, rz, dt, dx, dz, _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(src_full),
                                  nt_run, _ptr(rx), _ptr(rzr), _ptr(fields), _ptr(ms))
        assert rc == 0, rc
        return rx[:, :nt_run], rzr[:, :nt_run], fields, float(ms[0])

    def forward_fo(self, sx, sz, rz, dt, dx, dz, vp, vs, ax, az, src, nt_run):
        """The reference's first-order stress + velocity kernels: (rec_vx, rec_vz, fields[16], ms)."""
        X, Z, NT = self.X, self.Z, self.NT
        src_full = np.zeros(NT, np.float32)
        src_full[: len(src)] = src[:NT]
        rx = np.zeros((X, NT), np.float32)
        rzr = np.zeros((X, NT), np.float32)
        fields = np.zeros((16, X, Z), np.float32)
        ms = np.zeros(1, np.float32)
        rc = self.lib.psr_forward_fo(sx, sz, rz, dt, dx, dz, _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(src_full),
                                     nt_run, _ptr(rx), _ptr(rzr), _ptr(fields), _ptr(ms))
        assert rc == 0, rc
        return rx[:, :nt_run], rzr[:, :nt_run], fields, float(ms[0])

    def backward_fo(self, rz, dt, dx, dz, vp, vs, ax, az, rec_vx, rec_vz, nt_run):
        """The reference's first-order backward-propagation kernels with
        load_record injection: (fields[16], ms).  rec_*: X x nt_run."""
        X, Z, NT = self.X, self.Z, self.NT
        rx = np.zeros((X, NT), np.float32)
        rzz = np.zeros((X, NT), np.float32)
        rx[:, :nt_run] = rec_vx
        rzz[:, :nt_run] = rec_vz
        fields = np.zeros((16, X, Z), np.float32)
        ms = np.zeros(1, np.float32)
        rc = self.lib.psr_backward_fo(rz, dt, dx, dz, _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az), _ptr(rx), _ptr(rzz),
                                      nt_run, _ptr(fields), _ptr(ms))
        assert rc == 0, rc
        return fields, float(ms[0])

    def rtm(self, sx, sz, rz, t0, dt, dx, dz, vp, vs, ax, az, src, rec=None, do_mute=1):
        X, Z, NT, L = self.X, self.Z, self.NT, self.L
        out = dict(lap_pp=np.zeros((X, Z), np.float32), lap_ps=np.zeros((X, Z), np.float32),
                   img_pp=np.zeros((X, Z), np.float32), img_ps=np.zeros((X, Z), np.float32),
                   acc=np.zeros((3, X, Z), np.float32), rec=np.zeros((2, X, NT), np.float32),
                   fields=np.zeros((12, X, Z), np.float32))
        ms = np.zeros(2, np.float32)
        rx = rzz = None
        if rec is not None:
            rx = np.ascontiguousarray(rec[0], dtype=np.float32)
            rzz = np.ascontiguousarray(rec[1], dtype=np.float32)
        rc = self.lib.psr_rtm_shot(sx, sz, rz, t0, dt, dx, dz, dx, _ptr(vp), _ptr(vs), _ptr(ax), _ptr(az),
                                   _ptr(np.ascontiguousarray(src, dtype=np.float32)), _ptr(rx), _ptr(rzz), do_mute,
                                   *[_ptr(out[k]) for k in ("lap_pp", "lap_ps", "img_pp", "img_ps", "acc", "rec",
                                                            "fields")], _ptr(ms))
        assert rc == 0, rc
        out["lap_pp"] = out["lap_pp"][L:X - L, L:Z - L].copy()
        out["lap_ps"] = out["lap_ps"][L:X - L, L:Z - L].copy()
        out["ms"] = (float(ms[0]), float(ms[1]))
        return out


def layered_model(X, Z, L, kind="reference"):
    """Small layered test models on the padded grid (interior filled, then padded).

    "reference" is the reference's built-in 3-layer Vp / 2-layer Vs model
    (P-S-seperating.cu:1999-2040) scaled to the interior depth.
    """
    nz = Z - 2 * L
    vp = np.zeros((X, Z), np.float32)
    vs = np.zeros((X, Z), np.float32)
    zi = np.arange(Z)
    d1, d2 = L + nz // 4, L + nz // 2
    vp[:, :] = np.where(zi < d1, 3400.0, np.where(zi < d2, 3800.0, 4500.0))[None, :]
    vs[:, :] = np.where(zi < d2, 2900.0, 3800.0)[None, :]
    return vp, vs
