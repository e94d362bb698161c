"""The precision form on the large-model configuration's physics: the 4 m
grid, dt = 0.4 ms, 25 Hz, N = 5 and the full nt = 8000 of that
configuration, on a window of its seeded layered model (200 interior columns
by the top 500 rows, which hold several of its interfaces), migrated with the
true model so that the image holds reflections.

Reference: the FP64 oracle's RTM from the stored source wavefield at the
same imaging levels (every 4th; no reconstruction, so nothing amplifies its
round-off -- it equals the FP64 reconstruction from exactly restored strips
to 1e-11 on this window, tests/test_oracle.py checks the same on a golden
case).  Measured: the precision form (source P snapshots every 4 imaging
levels stored as scaled FP16, compensated FP32 imaging sums) and its FP32
floor (the same levels stored in FP32).  Bounds: PP and PS within the 1 %
bar below the acquisition rows, and the FP16 form within 0.2 percentage
points of the FP32 floor over the whole image.  The oracle keeps
2000 x 2 x 200 x 500 doubles (3.2 GB); the test is skipped when the host has
less than four times that available."""
import dataclasses

import numpy as np
import pytest

import ouc_b200 as o
from helpers import rel_l2, require_host_memory

pytestmark = pytest.mark.gpu

ACQ_ROWS = 16
WINDOW = (1900, 2100)    # interior columns of the model (the window's centre holds the shot)
DEPTH = 500              # interior rows of the window (from the surface)
K = 4


def test_snapshot_form_at_the_large_model_physics_vs_fp64():
    from oracle.oracle import Oracle, Shot
    from ouc_b200 import models
    w = models.c4()
    x0, x1 = WINDOW
    vp = np.ascontiguousarray(w.vp[x0:x1, :DEPTH])
    vs = np.ascontiguousarray(w.vs[x0:x1, :DEPTH])
    cfg = dataclasses.replace(w.cfg, nx=x1 - x0, nz=DEPTH)
    L = cfg.npml
    require_host_memory((cfg.nt // K) * 2 * cfg.nx * cfg.nz * 8)
    wav, t0 = o.ricker(w.fm, cfg.dt, cfg.nt)
    shot = o.Shot((x1 - x0) // 2, 2, 2, t0=t0)
    orc = Oracle()
    vpp = orc.pad(np.pad(vp, L), L)
    vsp = orc.pad(np.pad(vs, L), L)
    ax, az = orc.profile(vpp, L)
    sh = Shot(X=cfg.X, Z=cfg.Z, L=L, N=cfg.half_order, nt=cfg.nt, sx=L + shot.sx, sz=L + 2, rz=L + 2, dx=cfg.dx,
              dz=cfg.dz, dt=cfg.dt, t0=t0)
    r = orc.rtm_stored(sh, vpp, vsp, ax, az, wav, every=K)

    def run(**over):
        with o.Context(dataclasses.replace(cfg, **over), vp, vs) as ctx:
            return ctx.rtm_shot(shot, wav)

    def errs(pp, ps):
        d = slice(ACQ_ROWS, None)
        return ({"pp": rel_l2(pp, r["lap_pp"]), "ps": rel_l2(ps, r["lap_ps"])},
                {"pp": rel_l2(pp[:, d], r["lap_pp"][:, d]), "ps": rel_l2(ps[:, d], r["lap_ps"][:, d])})

    e, ed = errs(*run(snapshot_every=K, strip_precision=o.PREC_FP16, compensated_image=1))
    f, fd = errs(*run(snapshot_every=K, strip_precision=o.PREC_FP32))
    print(f"large-model physics window {cfg.X} x {cfg.Z}, nt = {cfg.nt}: FP16 snapshots every {K} vs FP64 {e}, "
          f"below row {ACQ_ROWS} {ed}; FP32 snapshots (the floor) {f}, below {fd}")
    assert max(ed.values()) <= 1e-2, ed
    assert e["pp"] <= f["pp"] + 2e-3 and e["ps"] <= f["ps"] + 2e-3, (e, f)
