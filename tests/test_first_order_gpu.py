"""GPU parity of the first-order velocity-stress scheme (ouc_forward_fo, the
reference's stress/velocity kernels P-S-seperating.cu:390-560).

  * against those kernels compiled for sm_100a (same hardware, same FMA
    contraction): bit-identical gathers and all 16 final fields;
  * against the FP64 oracle: the error of the reference's own kernels run
    in FP32 on the CPU (no contraction) is the floor; ours stays within 2x
    of it plus 1e-7 (the two FP32 evaluations round differently).
Models are seeded random layered media inside the absorbing layer, padded
the reference's way.
"""
import os

import numpy as np
import pytest

import ouc_b200 as o
from helpers import rel_l2
from oracle.oracle import REF_DIR, RefBuild, Shot

pytestmark = pytest.mark.gpu

FIELDS = ("Vx", "Vz", "Vpx", "Vpz", "Vsx", "Vsz", "theta", "omega", "duzdx", "duzdz", "duxdx", "duxdz",
          "theta_x", "theta_z", "omega_x", "omega_z")


def _model(ref, seed):
    X, Z, L = ref.X, ref.Z, ref.L
    rng = np.random.default_rng(seed)
    nx, nz = X - 2 * L, Z - 2 * L
    vp = np.empty((nx, nz), np.float32)
    depth = np.linspace(0, 1, nz, dtype=np.float32)
    vp[:] = 2000 + 1500 * depth + rng.uniform(-150, 150, (nx, nz)).astype(np.float32)
    vs = (vp / rng.uniform(1.7, 1.9)).astype(np.float32)
    return vp, vs


def _wavelet(nt, dt=6e-4, f0=25.0):
    t = np.arange(nt) * dt - 1.2 / f0
    a = (np.pi * f0 * t) ** 2
    return ((1 - 2 * a) * np.exp(-a)).astype(np.float32)


def _padded(ref, vp, vs):
    X, Z, L = ref.X, ref.Z, ref.L
    full_vp = np.zeros((X, Z), np.float32)
    full_vs = np.zeros((X, Z), np.float32)
    full_vp[L:X - L, L:Z - L] = vp
    full_vs[L:X - L, L:Z - L] = vs
    _, pvp, pvs = ref.pad(np.ones_like(full_vp), full_vp, full_vs)
    return pvp, pvs


def _context(ref, vp, vs, **over):
    kw = dict(nx=ref.X - 2 * ref.L, nz=ref.Z - 2 * ref.L, npml=ref.L, dx=8.0, dz=8.0, dt=6e-4, nt=ref.NT,
              half_order=ref.N)
    kw.update(over)
    return o.Context(o.Config(**kw), vp, vs)


# (sx, sz, rz) in interior coordinates: mid-grid, and a source on the first
# interior row and last interior column with receivers on the last row
def _shots(ref):
    nx, nz = ref.X - 2 * ref.L, ref.Z - 2 * ref.L
    return [(nx // 3, 5, 2), (0, nz - 1, nz - 1)]


@pytest.mark.parametrize("name", ["g64n6", "g72x56n5", "c1"])
def test_first_order_bit_exact_vs_reference_sm100(oracle, name):
    if not os.path.exists(os.path.join(REF_DIR, f"libpsref_cuda_{name}.so")):
        pytest.skip("reference sm_100a build not present")
    ref = RefBuild(name, "cuda")
    vp, vs = _model(ref, 3)
    pvp, pvs = _padded(ref, vp, vs)
    ax, az = oracle.profile(pvp, ref.L)   # the context's damping profile (same formula and R)
    w = _wavelet(ref.NT)
    shots = _shots(ref) if name != "c1" else _shots(ref)[:1]
    with _context(ref, vp, vs) as ctx:
        for sx, sz, rz in shots:
            gx, gz, f = ctx.forward_first_order(o.Shot(sx=sx, sz=sz, rz=rz), w, fields=True)
            L = ref.L
            rx, rzz, rf, _ = ref.forward_fo(sx + L, sz + L, rz + L, np.float32(6e-4), np.float32(8.0),
                                            np.float32(8.0), pvp, pvs, ax, az, w, ref.NT)
            assert np.abs(rx).max() > 0
            diff = {n: int(np.count_nonzero(f[k] != rf[k])) for k, n in enumerate(FIELDS)}
            print(name, (sx, sz, rz), "cells differing from the reference:", diff)
            assert np.array_equal(gx, rx) and np.array_equal(gz, rzz)
            assert not any(diff.values()), diff


@pytest.mark.parametrize("name", ["g64n6", "g72x56n5", "g48x40n2"])
def test_first_order_error_vs_fp64_oracle(oracle, name):
    if not os.path.exists(os.path.join(REF_DIR, f"libpsref_emu_{name}.so")):
        pytest.skip("reference CPU build not present")
    ref = RefBuild(name, "emu")
    vp, vs = _model(ref, 5)
    pvp, pvs = _padded(ref, vp, vs)
    w = _wavelet(ref.NT)
    L = ref.L
    sx, sz, rz = _shots(ref)[0]
    with _context(ref, vp, vs) as ctx:
        gx, gz, f = ctx.forward_first_order(o.Shot(sx=sx, sz=sz, rz=rz), w, fields=True)
    ax, az = oracle.profile(pvp, L)
    sh = Shot(X=ref.X, Z=ref.Z, L=L, N=ref.N, nt=ref.NT, sx=sx + L, sz=sz + L, rz=rz + L, dx=8.0, dz=8.0, dt=6e-4)
    d_x, d_z, d_f = oracle.forward_fo(sh, pvp, pvs, ax, az, w, fp64=True)
    e_x, e_z, e_f, _ = ref.forward_fo(sx + L, sz + L, rz + L, np.float32(6e-4), np.float32(8.0), np.float32(8.0),
                                      pvp, pvs, ax, az, w, ref.NT)
    ours = {"gx": rel_l2(gx, d_x), "gz": rel_l2(gz, d_z)}
    ours.update({n: rel_l2(f[k], d_f[k]) for k, n in enumerate(FIELDS)})
    floor = {"gx": rel_l2(e_x, d_x), "gz": rel_l2(e_z, d_z)}
    floor.update({n: rel_l2(e_f[k], d_f[k]) for k, n in enumerate(FIELDS)})
    print(name, "vs FP64 oracle", {k: f"{ours[k]:.2e} (ref {floor[k]:.2e})" for k in ours})
    for k in ours:
        assert ours[k] <= 2 * floor[k] + 1e-7, (k, ours[k], floor[k])
    assert ours["gx"] < 1e-5 and ours["gz"] < 1e-5


@pytest.mark.parametrize("name", ["g64n6", "g72x56n5", "c1"])
@pytest.mark.parametrize("layout", [o.GATHER_XT, o.GATHER_TX])
def test_first_order_backward_bit_exact_vs_reference_sm100(oracle, name, layout):
    """Receiver back-propagation of the reference kernels' own records (the
    *_backward_propagation kernels with load_record injection)."""
    if not os.path.exists(os.path.join(REF_DIR, f"libpsref_cuda_{name}.so")):
        pytest.skip("reference sm_100a build not present")
    if name == "c1" and layout == o.GATHER_TX:
        pytest.skip("one layout suffices at this size")
    ref = RefBuild(name, "cuda")
    vp, vs = _model(ref, 7)
    pvp, pvs = _padded(ref, vp, vs)
    ax, az = oracle.profile(pvp, ref.L)
    w = _wavelet(ref.NT)
    L = ref.L
    sx, sz, rz = _shots(ref)[0]
    args = (np.float32(6e-4), np.float32(8.0), np.float32(8.0), pvp, pvs, ax, az)
    rx, rzz, _, _ = ref.forward_fo(sx + L, sz + L, rz + L, *args, w, ref.NT)
    bf, _ = ref.backward_fo(rz + L, *args, rx, rzz, ref.NT)
    with _context(ref, vp, vs, gather_layout=layout) as ctx:
        recs = (rx, rzz) if layout == o.GATHER_XT else (rx.T, rzz.T)
        f = ctx.backward_first_order(o.Shot(sx=sx, sz=sz, rz=rz), *recs)
        t = ctx.timing()
    assert np.abs(bf[0]).max() > 0
    diff = {n: int(np.count_nonzero(f[k] != bf[k])) for k, n in enumerate(FIELDS)}
    print(name, layout, "cells differing from the reference:", diff, "backward ms", t["backward_ms"])
    assert not any(diff.values()), diff


def test_first_order_throughput_c2(oracle):
    """Cell-updates per second of the first-order forward loop on the
    1000 x 500 interior (L = 30, N = 5, nt = 4000), ours against the
    reference's stress + velocity kernels on the same GPU; the final state
    must agree bit for bit."""
    if not os.path.exists(os.path.join(REF_DIR, "libpsref_cuda_c2.so")):
        pytest.skip("reference sm_100a build not present")
    ref = RefBuild("c2", "cuda")
    vp, vs = _model(ref, 9)
    pvp, pvs = _padded(ref, vp, vs)
    ax, az = oracle.profile(pvp, ref.L)
    w = _wavelet(ref.NT)
    L = ref.L
    sx, sz, rz = (ref.X - 2 * L) // 2, 10, 5
    cells = (ref.X - 2 * ref.N) * (ref.Z - 2 * ref.N) * ref.NT
    with _context(ref, vp, vs) as ctx:
        ctx.forward_first_order(o.Shot(sx=sx, sz=sz, rz=rz), w)   # warm-up
        gx, gz, f = ctx.forward_first_order(o.Shot(sx=sx, sz=sz, rz=rz), w, fields=True)
        ms = ctx.timing()["forward_ms"]
    rx, rzz, rf, rms = ref.forward_fo(sx + L, sz + L, rz + L, np.float32(6e-4), np.float32(8.0), np.float32(8.0),
                                      pvp, pvs, ax, az, w, ref.NT)
    print(f"first-order forward c2: ours {ms:.1f} ms = {cells / ms / 1e6:.2f} Gcell/s; "
          f"reference kernels {rms:.1f} ms = {cells / rms / 1e6:.2f} Gcell/s")
    assert np.array_equal(gx, rx) and np.array_equal(gz, rzz)
    assert all(np.array_equal(f[k], rf[k]) for k in range(16))


def test_first_order_rejects_unsupported_forms():
    ref_like = type("R", (), dict(X=64, Z=64, L=12, N=6, NT=50))
    vp, vs = _model(ref_like, 1)
    w = _wavelet(50)
    with _context(ref_like, vp, vs) as ctx:
        with pytest.raises(o.OucError, match="theta source"):
            ctx.forward_first_order(o.Shot(sx=5, sz=5, rz=2, src_type=o.SRC_FORCE_Z), w)
        with pytest.raises(o.OucError, match="outside"):
            ctx.forward_first_order(o.Shot(sx=40, sz=5, rz=2), w)
        # the context stays usable after a rejected call
        gx, _, _ = ctx.forward_first_order(o.Shot(sx=5, sz=5, rz=2), w)
        assert np.isfinite(gx).all() and np.abs(gx).max() > 0
    rho = np.full_like(vp, 2000.0)
    with o.Context(o.Config(nx=40, nz=40, npml=12, dx=8.0, dz=8.0, dt=6e-4, nt=50, half_order=6, density=1),
                   vp, vs, rho) as ctx:
        with pytest.raises(o.OucError, match="density"):
            ctx.forward_first_order(o.Shot(sx=5, sz=5, rz=2), w)
