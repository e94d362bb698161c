"""GPU parity of the CUDA path (libouc.so, through the C ABI) with the
reference's outputs (golden fixtures from the reference's own kernels), the
FP64 oracle and, where built, the reference's kernels compiled for sm_100a.

Tolerances (relative L2 per field):
  * against the reference's kernels compiled for sm_100a (same hardware,
    same FMA contraction): 1e-5 after nt steps -- the bar for the FP32 path;
  * against the golden fixtures, which come from the reference's kernels run
    on the CPU without FMA contraction: the FP32 round-off floor, measured
    by the FP64 oracle as ~1e-6 for gathers, ~1e-4 for the separated P/S
    fields and ~1e-3 for the images -> 1e-5, 5e-4 and 3e-3;
  * against the FP64 oracle: asserted at the same floors and printed.
"""
import dataclasses
import os

import numpy as np
import pytest

import ouc_b200 as o
from helpers import CASES, finite_rel_l2, golden_shot, load_golden, make_context, rel_l2, shot_cfg, worst
from oracle.oracle import REF_DIR, RefBuild

pytestmark = pytest.mark.gpu

TOL_REF = 1e-5        # vs the reference's sm_100a kernels
TOL_GATHER = 1e-5     # vs CPU-run reference / FP64 oracle
TOL_FIELD = 5e-4
TOL_IMAGE = 3e-3


@pytest.mark.parametrize("name", CASES)
def test_forward_matches_reference(name):
    g = load_golden(name)
    with make_context(g) as ctx:
        gx, gz, _ = ctx.forward(golden_shot(g), g["src"])
    with make_context(g, nt=int(g["nt_mid"])) as ctx:
        _, _, f = ctx.forward(golden_shot(g), g["src"][: int(g["nt_mid"])], fields=True)
    eg = {"gx": rel_l2(gx, g["fwd_gx"]), "gz": rel_l2(gz, g["fwd_gz"])}
    ef = {n: rel_l2(f[k], g["fwd_fields"][k]) for k, n in enumerate(("Ux", "Uz", "Px", "Pz", "Sx", "Sz"))}
    print(name, eg, ef)
    assert worst(eg) <= TOL_GATHER, eg
    assert worst(ef) <= TOL_FIELD, ef


@pytest.mark.parametrize("name", CASES)
def test_forward_error_vs_fp64_oracle(oracle, name):
    g = load_golden(name)
    sh = shot_cfg(g)
    gx64, _, _ = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], fp64=True)
    sh.nt = int(g["nt_mid"])
    _, _, f64 = oracle.forward(sh, g["vp"], g["vs"], g["ax"], g["az"], g["src"], fp64=True)
    with make_context(g) as ctx:
        gx, _, _ = ctx.forward(golden_shot(g), g["src"])
    with make_context(g, nt=sh.nt) as ctx:
        _, _, f = ctx.forward(golden_shot(g), g["src"][: sh.nt], fields=True)
    e = {"gx": rel_l2(gx, gx64), "Px": rel_l2(f[2], f64[2]), "Sx": rel_l2(f[4], f64[4])}
    print(name, "vs FP64 oracle", e)
    assert e["gx"] < TOL_GATHER and max(e["Px"], e["Sx"]) < TOL_FIELD


@pytest.mark.parametrize("name", CASES)
def test_rtm_matches_reference(name):
    g = load_golden(name)
    with make_context(g) as ctx:
        pp, ps = ctx.rtm_shot(golden_shot(g), g["src"])
        spp, sps, sil = ctx.stack()
    errs = {"lap_pp": finite_rel_l2(pp, g["rtm_lap_pp"]), "lap_ps": finite_rel_l2(ps, g["rtm_lap_ps"])}
    print(name, errs)
    assert worst(errs) <= TOL_IMAGE, errs
    assert np.allclose(spp, pp.astype(np.float64)) and np.allclose(sps, ps.astype(np.float64))
    L, X, Z = int(g["L"]), int(g["X"]), int(g["Z"])
    assert rel_l2(sil, g["rtm_acc"][2][L:X - L, L:Z - L]) < TOL_FIELD


@pytest.mark.parametrize("layout", [o.GATHER_XT, o.GATHER_TX])
def test_rtm_external_records_equal_self_modelled(layout):
    g = load_golden("g72x56n5")
    with make_context(g, gather_layout=layout) as ctx:
        sh = golden_shot(g)
        gx, gz, _ = ctx.forward(sh, g["src"])
        pp1, ps1 = ctx.rtm_shot(sh, g["src"], rec=(gx, gz))
        pp0, ps0 = ctx.rtm_shot(sh, g["src"])
    assert np.array_equal(pp0, pp1) and np.array_equal(ps0, ps1)


def test_forward_deterministic_and_layouts_agree():
    g = load_golden("g64n6")
    with make_context(g) as a, make_context(g, gather_layout=o.GATHER_TX) as b:
        gx1, gz1, _ = a.forward(golden_shot(g), g["src"])
        gx2, gz2, _ = a.forward(golden_shot(g), g["src"])
        tx, tz, _ = b.forward(golden_shot(g), g["src"])
    assert np.array_equal(gx1, gx2) and np.array_equal(gz1, gz2)
    assert np.array_equal(gx1, tx.T) and np.array_equal(gz1, tz.T)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "libpsref_cuda_g72x56n5.so")),
                    reason="reference sm_100a build not present")
@pytest.mark.parametrize("name", ["g64n6", "g72x56n5"])
def test_matches_reference_cuda_kernels_on_b200(name):
    """The reference's own kernels compiled for sm_100a on the same inputs."""
    g = load_golden(name)
    ref = RefBuild(name, "cuda")
    dt, dx = np.float32(g["dt"]), np.float32(g["dx"])
    sx, sz, rz = int(g["sx"]), int(g["sz"]), int(g["rz"])
    rgx, rgz, rf, _ = ref.forward(sx, sz, rz, dt, dx, dx, g["vp"], g["vs"], g["ax"], g["az"], g["src"], ref.NT)
    r = ref.rtm(sx, sz, rz, int(g["t0"]), dt, dx, dx, g["vp"], g["vs"], g["ax"], g["az"], g["src"])
    with make_context(g) as ctx:
        gx, gz, f = ctx.forward(golden_shot(g), g["src"], fields=True)
        pp, ps = ctx.rtm_shot(golden_shot(g), g["src"])
    # fields after the full nt as well as at mid-propagation
    nm = int(g["nt_mid"])
    _, _, rfm, _ = ref.forward(sx, sz, rz, dt, dx, dx, g["vp"], g["vs"], g["ax"], g["az"], g["src"], nm)
    with make_context(g, nt=nm) as ctx:
        _, _, fm = ctx.forward(golden_shot(g), g["src"][:nm], fields=True)
    e = {"gx": rel_l2(gx, rgx), "gz": rel_l2(gz, rgz), "lap_pp": finite_rel_l2(pp, r["lap_pp"]),
         "lap_ps": finite_rel_l2(ps, r["lap_ps"])}
    for k, n in enumerate(("Ux", "Uz", "Px", "Pz", "Sx", "Sz")):
        e[n] = rel_l2(f[k], rf[k])
        e[n + "_mid"] = rel_l2(fm[k], rfm[k])
    bitexact = {k: bool(np.array_equal(a, b)) for k, a, b in
                (("gx", gx, rgx), ("fields", f[2:6], rf[2:6]), ("lap_pp", pp, r["lap_pp"]))}
    print(name, "vs reference CUDA", e, bitexact)
    assert worst(e) <= TOL_REF, e


@pytest.mark.parametrize("name", ["c1", "c2", "c4s"])
def test_workload_grids_match_reference_cuda_kernels(name):
    """Workload-size grids (many tiles in both directions, interior tiles,
    long runs): gathers, the six displacement fields (U, P, S; after nt steps
    and at mid-run) and the RTM images against the reference's sm_100a
    kernels on the same model and shot, at 1e-5 relative L2 per field; the
    gathers and fields are also asserted bit-identical (the kernels reproduce
    every rounding of the reference's compiled expressions).  c4s is the
    largest grid (4000 x 1500 interior, 4060 x 1560 padded) over its first
    2000 steps."""
    from ouc_b200 import models
    lib = os.path.join(REF_DIR, f"libpsref_cuda_{name}.so")
    if not os.path.exists(lib):
        pytest.skip("reference sm_100a build not present")
    from oracle.oracle import Oracle
    w = {"c1": models.c1, "c2": models.c2, "c4s": lambda: models.c4(nt=2000)}[name]()
    cfg = w.cfg
    vp, vs = (w.vp, w.vs) if w.vp_mig is None else (w.vp_mig, w.vs_mig)
    L = cfg.npml
    orc = Oracle()
    vpp = orc.pad(np.pad(vp, L), L)
    vsp = orc.pad(np.pad(vs, L), L)
    ax, az = orc.profile(vpp, L)
    wav, t0 = o.ricker(w.fm, cfg.dt, cfg.nt)
    sh = w.shots[len(w.shots) // 2 if name == "c4s" else 0]
    shot = o.Shot(sh.sx, sh.sz, sh.rz, t0=t0)
    ref = RefBuild(name, "cuda")
    f32 = np.float32
    fargs = (L + sh.sx, L + sh.sz, L + sh.rz, f32(cfg.dt), f32(cfg.dx), f32(cfg.dz), vpp, vsp, ax, az, wav)
    rgx, rgz, rf, _ = ref.forward(*fargs, cfg.nt)
    nm = cfg.nt // 2
    _, _, rfm, _ = ref.forward(*fargs, nm)
    r = ref.rtm(L + sh.sx, L + sh.sz, L + sh.rz, t0, f32(cfg.dt), f32(cfg.dx), f32(cfg.dz), vpp, vsp, ax, az, wav)
    with o.Context(cfg, vp, vs) as ctx:
        gx, gz, f = ctx.forward(shot, wav, fields=True)
        pp, ps = ctx.rtm_shot(shot, wav)
    cm = dataclasses.replace(cfg, nt=nm)
    with o.Context(cm, vp, vs) as ctx:
        _, _, fm = ctx.forward(shot, wav[:nm], fields=True)
    e = {"gx": rel_l2(gx, rgx), "gz": rel_l2(gz, rgz), "lap_pp": finite_rel_l2(pp, r["lap_pp"]),
         "lap_ps": finite_rel_l2(ps, r["lap_ps"])}
    names = ("Ux", "Uz", "Px", "Pz", "Sx", "Sz")
    for k, n in enumerate(names):
        e[n] = rel_l2(f[k], rf[k])
        e[n + "_mid"] = rel_l2(fm[k], rfm[k])
    bitexact = {"gathers": bool(np.array_equal(gx, rgx) and np.array_equal(gz, rgz)),
                "fields": all(np.array_equal(f[k], rf[k]) for k in range(6)),
                "fields_mid": all(np.array_equal(fm[k], rfm[k]) for k in range(6)),
                "images": bool(np.array_equal(pp, r["lap_pp"], equal_nan=True)
                               and np.array_equal(ps, r["lap_ps"], equal_nan=True))}
    finite = float(np.isfinite(pp).mean())
    print(name, "vs reference CUDA", e, "bit-exact:", bitexact, f"finite image cells {finite:.3f}")
    assert finite > (0.05 if name == "c4s" else 0.5)
    assert worst(e) <= TOL_REF, e
    assert bitexact["gathers"] and bitexact["fields"] and bitexact["fields_mid"], bitexact


def test_batched_shots_equal_single_shots():
    """Shots advanced together in one launch per stage give the same images
    as the same shots run one by one, and the FP64 stack is their sum."""
    g = load_golden("g72x56n5")
    L = int(g["L"])
    shots = [golden_shot(g)]
    for sx in (9, 30):
        s = golden_shot(g)
        s.sx = sx
        shots.append(s)
    with make_context(g) as one:
        singles = [one.rtm_shot(s, g["src"]) for s in shots]
        st1 = one.stack()
    with make_context(g, max_batch=2) as many:   # 3 shots -> groups of 2 and 1
        batched = many.rtm_batch(shots, g["src"])
        st2 = many.stack()
    for (a, b), (c, d) in zip(singles, batched):
        assert np.array_equal(a, c) and np.array_equal(b, d)
    assert np.allclose(st1[0], st2[0], rtol=1e-12, atol=0) and np.allclose(st1[1], st2[1], rtol=1e-12, atol=0)
    assert np.allclose(st1[0], sum(s[0].astype(np.float64) for s in singles), rtol=1e-12, atol=1e-30)
