"""Config 1 as a measured workload: single-shot forward modeling on the
two-layer 256^2 model (20-cell CPML, nt = 1000, vertical-force source),
timed with the context's CUDA events (forward time loop as a CUDA graph,
after one warm-up shot).  The padded grid (296^2, 2.8 MB per field) is
L2-resident and a step is ~45 tile CTAs, so the number is bounded by launch
and tile latency, not HBM; it is printed for the results table, and the
test asserts only that the modelling is not pathologically slow."""
import numpy as np
import pytest

import ouc_b200 as o

pytestmark = pytest.mark.gpu


def test_config1_forward_throughput():
    from ouc_b200 import models
    w = models.c1()
    cfg = w.cfg
    wav, t0 = o.ricker(w.fm, cfg.dt, cfg.nt)
    s = w.shots[0]
    shot = o.Shot(s.sx, s.sz, s.rz, src_type=o.SRC_FORCE_Z, t0=t0)
    with o.Context(cfg, w.vp, w.vs) as ctx:
        ctx.forward(shot, wav)                      # warm-up (graph capture)
        ms = []
        for _ in range(5):
            gx, gz, _ = ctx.forward(shot, wav)
            ms.append(ctx.timing()["forward_ms"])
    ms = float(np.median(ms))
    cells = cfg.X * cfg.Z * cfg.nt
    gcells = cells / (ms / 1e3) / 1e9
    print(f"config 1 forward (296 x 296 padded, nt = {cfg.nt}, one shot): {ms:.2f} ms, {gcells:.2f} Gcell-updates/s, "
          f"{cfg.nt / (ms / 1e3):.0f} steps/s")
    assert np.abs(gz).max() > 0
    assert gcells > 1.0
