"""Variable density (cfg.density = 1; no counterpart in the reference, whose
equations are density-normalised): moduli rho Vp^2 and rho Vs^2, and each
displacement component's acceleration scaled by the buoyancy averaged onto
its staggered position.  Judged against the FP64 oracle with the same
extension (oracle/oracle.cpp, Model::dens); with rho = 1 every added
operation is exact, so the result equals the density-normalised path bit for
bit."""
import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import models
from helpers import rel_l2
from oracle.oracle import Shot

pytestmark = pytest.mark.gpu

NX, NZ, L, N, NT, DX, DT = 128, 96, 16, 5, 500, 10.0, 1e-3


def model():
    vp, vs, rho = models.flat_layers(NX, NZ, 4, np.random.default_rng(33))
    return vp, vs, (1000.0 * rho).astype(np.float32)    # Gardner, kg/m^3


def cfg(density):
    return o.Config(nx=NX, nz=NZ, npml=L, dx=DX, dz=DX, dt=DT, nt=NT, half_order=N, device=0, density=density)


def test_unit_density_equals_the_density_normalised_path():
    vp, vs, _ = model()
    ones = np.ones_like(vp)
    w, t0 = o.ricker(20.0, DT, NT)
    shot = o.Shot(sx=64, sz=4, rz=4, t0=t0)
    with o.Context(cfg(0), vp, vs) as c0, o.Context(cfg(1), vp, vs, ones) as c1:
        g0 = c0.forward(shot, w, fields=True)
        g1 = c1.forward(shot, w, fields=True)
        i0 = c0.rtm_shot(shot, w)
        i1 = c1.rtm_shot(shot, w)
    for a, b in zip(g0, g1):
        assert np.array_equal(a, b)
    for a, b in zip(i0, i1):
        assert np.array_equal(a, b, equal_nan=True)


def test_density_forward_and_rtm_match_the_fp64_oracle(oracle):
    """Errors of the FP32 density path against the FP64 oracle stay at the
    FP32 round-off floor: within 3x (plus 1e-6) of the density-normalised
    path's own errors on the same grid and shot."""
    vp, vs, rho = model()
    w, t0 = o.ricker(20.0, DT, NT)
    shot = o.Shot(sx=64, sz=4, rz=4, t0=t0)
    vpp, vsp, rhop = (oracle.pad(np.pad(a, L), L) for a in (vp, vs, rho))
    ax, az = oracle.profile(vpp, L)
    X, Z = NX + 2 * L, NZ + 2 * L
    sh = Shot(X=X, Z=Z, L=L, N=N, nt=NT, sx=64 + L, sz=4 + L, rz=4 + L, dx=DX, dz=DX, dt=DT, t0=t0)

    def errors(density, r):
        with o.Context(cfg(density), vp, vs, r) as ctx:
            gx, gz, f = ctx.forward(shot, w, fields=True)
            pp, ps = ctx.rtm_shot(shot, w)
        kw = {"rho": rhop} if density else {"fp64": True}
        ox, oz, of = oracle.forward(sh, vpp, vsp, ax, az, w, **kw)
        rr = oracle.rtm(sh, vpp, vsp, ax, az, w, **kw)
        # oracle fields: Ux, Uz, Px, Pz, Sx, Sz, ... of the final level
        return {"gather_vx": rel_l2(gx, ox), "gather_vz": rel_l2(gz, oz), "Px": rel_l2(f[2], of[2]),
                "Pz": rel_l2(f[3], of[3]), "Sx": rel_l2(f[4], of[4]), "Sz": rel_l2(f[5], of[5]),
                "pp": rel_l2(pp, rr["lap_pp"]), "ps": rel_l2(ps, rr["lap_ps"])}, gx

    e1, g1 = errors(1, rho)
    e0, _ = errors(0, None)
    print("density vs FP64 oracle", e1)
    print("density-normalised vs FP64 oracle", e0)
    for k in e1:
        assert e1[k] <= 3.0 * e0[k] + 1e-6, (k, e1[k], e0[k])
    assert e1["gather_vx"] < 1e-5 and e1["pp"] < 5e-3
    # the density contrasts matter: against a constant density of the same mean
    with o.Context(cfg(1), vp, vs, np.full_like(rho, rho.mean())) as cc:
        gc, _, _ = cc.forward(shot, w)
    assert rel_l2(g1, gc) > 1e-2


def test_density_needs_a_positive_model():
    vp, vs, rho = model()
    with pytest.raises(o.OucError):
        o.Context(cfg(1), vp, vs)                  # no rho
    bad = rho.copy()
    bad[3, 3] = 0.0
    with pytest.raises(o.OucError):
        o.Context(cfg(1), vp, vs, bad)
