"""FWI gradient (cfg.gradient = 1; the formula of the reference's unused
gradfun, PS:1518-1633): the device accumulation against the FP64 oracle
(oracle/oracle.cpp Engine::gradient, the same definition), images unchanged
by the gradient, and the FP64 stack of several shots."""
import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import models
from helpers import rel_l2
from oracle.oracle import Shot, rtm_gradient

pytestmark = pytest.mark.gpu

NX, NZ, L, N, NT, DX, DT = 96, 80, 12, 5, 400, 10.0, 1e-3
TOL = 1e-3     # FP32 device (FMA contractions, other summation order) vs FP64, relative L2


def model():
    vp, vs, rho = models.flat_layers(NX, NZ, 3, np.random.default_rng(3))
    return vp, vs, (1000.0 * rho).astype(np.float32)


def cfg(gradient, batch=1):
    return o.Config(nx=NX, nz=NZ, npml=L, dx=DX, dz=DX, dt=DT, nt=NT, half_order=N, device=0, gradient=gradient,
                    max_batch=batch)


def test_gradient_matches_the_fp64_oracle(oracle):
    vp, vs, rho = model()
    w, t0 = o.ricker(20.0, DT, NT)
    shot = o.Shot(sx=48, sz=2, rz=2, t0=t0)
    with o.Context(cfg(1), vp, vs, rho) as ctx:
        pp, ps = ctx.rtm_shot(shot, w)
        gvp, gvs, il = ctx.gradient()
    with o.Context(cfg(0), vp, vs, rho) as c0:
        pp0, ps0 = c0.rtm_shot(shot, w)
    assert np.array_equal(pp, pp0, equal_nan=True) and np.array_equal(ps, ps0, equal_nan=True)
    vpp, vsp, rhop = (oracle.pad(np.pad(a, L), L) for a in (vp, vs, rho))
    ax, az = oracle.profile(vpp, L)
    sh = Shot(X=NX + 2 * L, Z=NZ + 2 * L, L=L, N=N, nt=NT, sx=48 + L, sz=2 + L, rz=2 + L, dx=DX, dz=DX, dt=DT,
              t0=t0)
    _, _, g = rtm_gradient(oracle, sh, vpp, vsp, ax, az, w, rho=rhop)
    ref = [g[k][L:NX + L, L:NZ + L] for k in range(3)]
    e = [rel_l2(x, r) for x, r in zip((gvp, gvs, il), ref)]
    print("gradient vs FP64 oracle (Vp, Vs, illumination)", e)
    assert np.abs(ref[0]).max() > 0 and np.abs(ref[1]).max() > 0
    assert max(e) < TOL


def test_gradient_stack_of_a_batch_is_the_sum_of_its_shots():
    vp, vs, rho = model()
    w, t0 = o.ricker(20.0, DT, NT)
    shots = [o.Shot(sx=s, sz=2, rz=2, t0=t0) for s in (20, 48, 75)]
    with o.Context(cfg(1, batch=3), vp, vs, rho) as ctx:
        ctx.rtm_batch(shots, w)
        batch = ctx.gradient(reset=True)
        single = [np.zeros((NX, NZ)) for _ in range(3)]
        for s in shots:
            ctx.rtm_shot(s, w)
            for acc, part in zip(single, ctx.gradient(reset=True)):
                acc += part
    for a, b in zip(batch, single):
        assert rel_l2(a, b) < 1e-12


def test_gradient_needs_the_strip_form_and_normalised_density():
    vp, vs, rho = model()
    bad = o.Config(nx=NX, nz=NZ, npml=L, dx=DX, dz=DX, dt=DT, nt=NT, half_order=N, device=0, gradient=1, density=1)
    with pytest.raises(o.OucError):
        o.Context(bad, vp, vs, rho)
    with o.Context(cfg(0), vp, vs) as c0, pytest.raises(o.OucError):
        c0.gradient()
