"""TEST INFRASTRUCTURE -- times the reference's own CUDA build on this GPU.

Runs one RTM shot of the reference's kernels (compiled for sm_100a from the
reference sources by oracle/Makefile, launch sequence of its main()) and one
RTM shot of libouc.so on the same model, grid and geometry, and prints one
JSON line per configuration:

  c2      1060 x 560 padded, N = 5, nt = 4000 (the benchmark workload)
  ref600  600 x 600 padded (200 x 200 interior, 200-cell absorbing layer),
          N = 6, nt = 6000, dt = 1 ms, dx = 10 m: the reference's own setting
          (P-S-seperating.cu:14-26, 1685-1688) with its built-in layer model.

Timings are CUDA-event times of the forward and backward loops; the
reference's per-shot zero-fill copies are outside them.
Usage: python oracle/ref_timing.py [c2] [ref600]
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[0] = ROOT   # the script's own directory would shadow the oracle package

import ouc_b200 as o  # noqa: E402
from ouc_b200 import models  # noqa: E402
from oracle.oracle import Oracle, RefBuild  # noqa: E402


def reference_layer_model(nx=200, nz=200):
    """The reference's built-in model (PS:1999-2040): Vp 3400/3800/4500 at
    depth offsets 0/50/100, Vs 2900/3800 at 0/100."""
    z = np.arange(nz)
    vp = np.where(z < 50, 3400.0, np.where(z < 100, 3800.0, 4500.0))[None, :].repeat(nx, 0).astype(np.float32)
    vs = np.where(z < 100, 2900.0, 3800.0)[None, :].repeat(nx, 0).astype(np.float32)
    return vp, vs


def case(name):
    if name == "c2":
        w = models.c2()
        return w.cfg, w.vp_mig, w.vs_mig, w.fm, w.shots[0].sx, 2, 2
    if name == "ref600":
        vp, vs = reference_layer_model()
        cfg = o.Config(nx=200, nz=200, npml=200, dx=10.0, dz=10.0, dt=1e-3, nt=6000, half_order=6)
        return cfg, vp, vs, 30.0, 5, 0, 0
    raise ValueError(name)


def run(name):
    cfg, vp, vs, fm, sx, sz, rz = case(name)
    L = cfg.npml
    orc = Oracle()
    vpp = orc.pad(np.pad(vp, L), L)
    vsp = orc.pad(np.pad(vs, L), L)
    ax, az = orc.profile(vpp, L)
    w, t0 = o.ricker(fm, cfg.dt, cfg.nt)
    ref = RefBuild(name, "cuda")
    assert (ref.X, ref.Z, ref.NT, ref.N) == (cfg.X, cfg.Z, cfg.nt, cfg.half_order)
    t1 = time.perf_counter()
    r = ref.rtm(L + sx, L + sz, L + rz, t0, np.float32(cfg.dt), np.float32(cfg.dx), np.float32(cfg.dz), vpp, vsp, ax,
                az, w)
    ref_wall = time.perf_counter() - t1
    shot = o.Shot(sx=sx, sz=sz, rz=rz, t0=t0)
    with o.Context(cfg, vp, vs) as ctx:
        ctx.rtm_shot(shot, w)    # warm-up
        pp, ps = ctx.rtm_shot(shot, w)
        tm = ctx.timing()
    ours_ms = tm["forward_ms"] + tm["backward_ms"] + tm["finalize_ms"]
    ref_ms = r["ms"][0] + r["ms"][1]
    cells = cfg.nt * (2 * cfg.X * cfg.Z + cfg.nx * cfg.nz)
    rel = float(np.linalg.norm(pp.astype(np.float64) - r["lap_pp"]) / np.linalg.norm(r["lap_pp"].astype(np.float64)))
    out = {"config": name, "grid": [cfg.X, cfg.Z], "nt": cfg.nt, "half_order": cfg.half_order,
           "reference_ms": {"forward": r["ms"][0], "backward": r["ms"][1], "total": ref_ms, "wall_s": ref_wall},
           "ouc_ms": {"forward": tm["forward_ms"], "backward": tm["backward_ms"], "finalize": tm["finalize_ms"],
                      "total": ours_ms},
           "reference_gcells": cells / (ref_ms / 1e3) / 1e9, "ouc_gcells": cells / (ours_ms / 1e3) / 1e9,
           "speedup": ref_ms / ours_ms, "image_pp_rel_l2_vs_reference": rel,
           "image_pp_bit_exact": bool(np.array_equal(pp, r["lap_pp"]))}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    for n in sys.argv[1:] or ["c2", "ref600"]:
        run(n)
