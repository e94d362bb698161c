"""CPU tests of the oracle: pinned against the reference's own outputs.

The golden fixtures hold outputs of the reference's kernels (run on the CPU
from the reference sources, tests/golden/make_golden.py).  The oracle's
float instantiation must reproduce them bit for bit; its double
instantiation (the FP64 oracle) must agree to FP32 round-off.
"""
import os

import numpy as np
import pytest

from helpers import CASES, load_golden, rel_l2, shot_cfg
from oracle.oracle import REF_DIR, RefBuild, layered_model, weights


@pytest.mark.parametrize("name", CASES)
def test_oracle_forward_bit_exact_vs_reference_fixture(oracle, name):
    g = load_golden(name)
    sh = shot_cfg(g)
    gx, gz, _ = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    assert np.array_equal(gx, g["fwd_gx"])
    assert np.array_equal(gz, g["fwd_gz"])
    sh.nt = int(g["nt_mid"])
    _, _, f = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    assert np.array_equal(f[:6], g["fwd_fields"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_rtm_bit_exact_vs_reference_fixture(oracle, name):
    g = load_golden(name)
    sh = shot_cfg(g)
    o = oracle.rtm(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    L, X, Z = int(g["L"]), int(g["X"]), int(g["Z"])
    assert np.array_equal(o["acc"], g["rtm_acc"])
    assert np.array_equal(o["rec"], g["rtm_rec"])
    assert np.array_equal(o["fields"][:6], g["rtm_fields"])
    # the reference writes the Laplacian over the interior; the oracle's rim is zero as the zeroed buffer
    assert np.array_equal(o["lap_pp"], g["rtm_lap_pp"])
    assert np.array_equal(o["lap_ps"], g["rtm_lap_ps"])
    assert np.isfinite(o["lap_pp"]).all() and np.abs(o["lap_pp"]).max() > 0


@pytest.mark.parametrize("name", CASES)
def test_fp64_oracle_agrees_to_fp32_roundoff(oracle, name):
    g = load_golden(name)
    sh = shot_cfg(g)
    gx, gz, _ = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], fp64=True)
    assert rel_l2(gx, g["fwd_gx"]) < 1e-5 and rel_l2(gz, g["fwd_gz"]) < 1e-5
    sh.nt = int(g["nt_mid"])
    _, _, f = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], fp64=True)
    # the separated P/S fields carry cancellation between the theta/omega and Q terms:
    # their FP32 round-off floor against FP64 is ~1e-4 (relative L2), the gathers' ~1e-6
    for k in range(6):
        assert rel_l2(f[k], g["fwd_fields"][k]) < 2e-4


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "libpsref_emu_g72x56n5.so")),
                    reason="reference CPU build not present (needs the reference sources)")
def test_oracle_bit_exact_vs_reference_kernels_other_geometry(oracle):
    """Fresh inputs, not the fixture ones: a different model and shot."""
    ref = RefBuild("g72x56n5", "emu")
    X, Z, L, N, NT = ref.X, ref.Z, ref.L, ref.N, ref.NT
    rng = np.random.default_rng(7)
    vp = np.zeros((X, Z), np.float32)
    vs = np.zeros((X, Z), np.float32)
    vp[L:X - L, L:Z - L] = rng.uniform(2000, 3500, (X - 2 * L, Z - 2 * L))
    vs[L:X - L, L:Z - L] = vp[L:X - L, L:Z - L] / 1.8
    _, vp, vs = ref.pad(np.ones_like(vp), vp, vs)
    ax, az = oracle.profile(vp, L, R=1e-4)
    src = np.sin(np.arange(NT) * 0.2).astype(np.float32) * np.exp(-np.arange(NT) / 40.0).astype(np.float32)
    from oracle.oracle import Shot
    sh = Shot(X=X, Z=Z, L=L, N=N, nt=NT, sx=L + 30, sz=L + 4, rz=L + 1, dx=8.0, dz=8.0, dt=8e-4, t0=10)
    r = ref.rtm(sh.sx, sh.sz, sh.rz, sh.t0, np.float32(8e-4), np.float32(8.0), np.float32(8.0), vp, vs, ax, az, src)
    o = oracle.rtm(sh, vp, vs, ax, az, src)
    for k in ("acc", "rec", "fields", "lap_pp", "lap_ps"):
        assert np.array_equal(r[k], o[k]), k


@pytest.mark.parametrize("name", ["g64n6", "g72x56n5", "g48x40n2"])
def test_first_order_oracle_bit_exact_vs_reference_kernels(oracle, name):
    """The first-order velocity-stress scheme (the reference's stress and
    velocity kernels, never called by its main()): the oracle's float build
    against those kernels run on the CPU, gathers and all 16 fields."""
    if not os.path.exists(os.path.join(REF_DIR, f"libpsref_emu_{name}.so")):
        pytest.skip("reference CPU build not present (needs the reference sources)")
    ref = RefBuild(name, "emu")
    X, Z, L, N, NT = ref.X, ref.Z, ref.L, ref.N, ref.NT
    rng = np.random.default_rng(11)
    vp = np.zeros((X, Z), np.float32)
    vs = np.zeros((X, Z), np.float32)
    vp[L:X - L, L:Z - L] = rng.uniform(2000, 3500, (X - 2 * L, Z - 2 * L))
    vs[L:X - L, L:Z - L] = vp[L:X - L, L:Z - L] / 1.8
    _, vp, vs = ref.pad(np.ones_like(vp), vp, vs)
    ax, az = oracle.profile(vp, L)
    src = np.sin(np.arange(NT) * 0.2).astype(np.float32) * np.exp(-np.arange(NT) / 40.0).astype(np.float32)
    from oracle.oracle import Shot
    sh = Shot(X=X, Z=Z, L=L, N=N, nt=NT, sx=L + 17, sz=L + 5, rz=L + 2, dx=8.0, dz=8.0, dt=6e-4)
    rx, rz, rf, _ = ref.forward_fo(sh.sx, sh.sz, sh.rz, np.float32(6e-4), np.float32(8.0), np.float32(8.0), vp, vs,
                                   ax, az, src, NT)
    ox, oz, of = oracle.forward_fo(sh, vp, vs, ax, az, src)
    assert np.abs(rx).max() > 0
    assert np.array_equal(rx, ox) and np.array_equal(rz, oz)
    for k in range(16):
        assert np.array_equal(rf[k], of[k]), k
    dx_, dz_, df = oracle.forward_fo(sh, vp, vs, ax, az, src, fp64=True)
    assert rel_l2(rx, dx_) < 1e-5

    # receiver back-propagation of these records (load_record injection,
    # stress_backward_propagation, velocity_backward_propagation)
    bf, _ = ref.backward_fo(sh.rz, np.float32(6e-4), np.float32(8.0), np.float32(8.0), vp, vs, ax, az, rx, rz, NT)
    of = oracle.backward_fo(sh, vp, vs, ax, az, rx, rz)
    assert np.abs(bf[0]).max() > 0
    for k in range(16):
        assert np.array_equal(bf[k], of[k]), k
    df = oracle.backward_fo(sh, vp, vs, ax, az, rx, rz, fp64=True)
    assert rel_l2(bf[2], df[2]) < 1e-4


FO_STATE = [2, 3, 4, 5, 8, 9, 10, 11, 12, 13, 14, 15]   # Vpx..Vsz, the Q fields, theta_x..omega_z


@pytest.mark.parametrize("name", CASES)
def test_first_order_oracle_matches_golden(oracle, name):
    """The oracle's first-order restatement against the fixtures of the
    reference's stress/velocity kernels (and their backward-propagation twins)
    run on the CPU: bit-exact gathers, mid-run state and back-propagated
    state.  Needs no reference sources."""
    g = load_golden(name)
    sh = shot_cfg(g)
    gx, gz, _ = oracle.forward_fo(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    assert np.abs(g["fo_gx"]).max() > 0
    assert np.array_equal(gx, g["fo_gx"]) and np.array_equal(gz, g["fo_gz"])
    sh_mid = shot_cfg(g)
    sh_mid.nt = int(g["nt_mid"])
    _, _, f = oracle.forward_fo(sh_mid, g["vp"], g["vs"], g["ax"], g["az"], g["src"][: sh_mid.nt])
    for k, i in enumerate(FO_STATE):
        assert np.array_equal(f[i], g["fo_fields"][k]), i
    b = oracle.backward_fo(sh, g["vp"], g["vs"], g["ax"], g["az"], g["fo_gx"], g["fo_gz"])
    for k, i in enumerate(FO_STATE):
        assert np.array_equal(b[i], g["fo_bwd_fields"][k]), i


def test_padding_matches_reference(oracle):
    """orc_pad_model restates xiangbian (PS:37-119); compare with the fixture's padded model."""
    g = load_golden("g72x56n5")
    L, X, Z = int(g["L"]), int(g["X"]), int(g["Z"])
    inner = np.zeros_like(g["vp"])
    inner[L:X - L, L:Z - L] = g["vp"][L:X - L, L:Z - L]
    assert np.array_equal(oracle.pad(inner, L), g["vp"])


def test_damping_profile_formula(oracle):
    """PS:2067-2105: d = log10(1/R)*1.5*Vp/L*(dist/L)^4, L damped cells left/top, L-1 right/bottom."""
    X, Z, L = 40, 30, 8
    vp = np.full((X, Z), 3000.0, np.float32)
    ax, az = oracle.profile(vp, L, R=1e-3)
    d0 = np.log10(1e3) * 1.5 * 3000.0 / L
    assert ax[0, 5] == np.float32(d0 * 1.0)
    assert ax[L, 5] == 0 and ax[X - L, 5] == 0
    assert ax[X - L + 1, 5] == np.float32(d0 * (1.0 / L) ** 4)
    assert (ax[L:X - L + 1] == 0).all()
    assert az[3, 0] == np.float32(d0)
    assert (az[:, L:Z - L + 1] == 0).all()
    assert np.count_nonzero(ax[:, 0]) == 2 * L - 1


def test_stencil_weights_taylor_conditions():
    for n in (2, 4, 5):
        w = weights(n).astype(np.float64)
        odd = 2 * np.arange(1, n + 1) - 1
        assert abs(np.sum(w * odd) - 1.0) < 1e-6
        for p in range(2, n + 1):
            assert abs(np.sum(w * odd ** (2 * p - 1))) < 1e-6 * odd[-1] ** (2 * p - 1)
    # N = 6 uses the reference's literals (PS:221), one ulp from the exact weights at most
    w6 = weights(6)
    from oracle.coeffs import exact
    ex = np.array([float(v) for v in exact(6)], np.float32)
    assert np.max(np.abs(w6.view(np.int32) - ex.view(np.int32))) <= 1


def test_layered_model_shape():
    vp, vs = layered_model(40, 32, 6)
    assert vp.shape == (40, 32) and vs.min() > 0


def test_oracle_force_source_float_and_double_agree(oracle):
    """The vertical-force source (an extension without a reference
    counterpart): the float and double instantiations agree to FP32
    round-off, and the force run differs from the theta-source run."""
    g = load_golden("g72x56n5")
    sh = shot_cfg(g)
    sh.src_type = 1
    fx32, fz32, f32 = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    fx64, fz64, f64 = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], fp64=True)
    assert rel_l2(fx32, fx64) < 1e-5 and rel_l2(fz32, fz64) < 1e-5
    # separated P/S fields carry FP32 cancellation (about 5e-4 here; U is 5e-6)
    assert max(rel_l2(f32[k], f64[k]) for k in range(2)) < 1e-5
    assert max(rel_l2(f32[k], f64[k]) for k in range(2, 6)) < 2e-3
    sh.src_type = 0
    tx, tz, _ = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    assert rel_l2(fz32, tz) > 0.5


def test_oracle_stored_source_rtm_equals_exact_reconstruction(oracle):
    """The FP64 RTM from the stored source wavefield (the reference of the
    snapshot form) equals the FP64 RTM that reconstructs the source field
    from exactly restored strips, on a short run where that reconstruction
    is accurate; imaging only every 4th level gives a different image."""
    g = load_golden("g72x56n5")
    sh = shot_cfg(g)
    sh.strip_level = 1
    r = oracle.rtm(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], fp64=True)
    s1 = oracle.rtm_stored(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], every=1)
    s4 = oracle.rtm_stored(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], every=4)
    fin = np.isfinite(r["lap_pp"])
    assert rel_l2(s1["lap_pp"][fin], r["lap_pp"][fin]) < 1e-8
    assert rel_l2(s1["lap_ps"][fin], r["lap_ps"][fin]) < 1e-8
    assert rel_l2(s1["acc"], r["acc"]) < 1e-8
    assert rel_l2(s4["lap_pp"][fin], s1["lap_pp"][fin]) > 1e-4
