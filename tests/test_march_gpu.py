"""The x-marching step kernel and the dynamic-queue (persistent) launch of
the tile kernel against the 32 x 64 tile kernel.

Both kernels implement the same fused time step (the reference's forward_s +
forward_u pair, PS:316-384 / PS:205-314, and its receiver and reconstruction
twins) with the same roundings, so every output must agree bit for bit:
gathers, the six displacement fields, PP/PS images and the FP64 stack, for
several segment lengths (one block per segment up to whole-grid segments),
all three stencil orders, every strip precision, the snapshot form,
compensated imaging, variable density, the force source, batches of shots
and the survey's uneven sub-grids.  The tile kernel itself is pinned to the
reference by the parity tests.
"""
import numpy as np
import pytest

import ouc_b200 as o
from helpers import CASES, golden_shot, load_golden, make_context

pytestmark = pytest.mark.gpu

QUEUE = -1          # OUC_STEP_TILE_QUEUE
SEGS = [QUEUE, 16, 48, 128, 4096]


def _run(g, seg, shots=None, **over):
    shots = shots or [golden_shot(g)]
    with make_context(g, max_batch=len(shots), **over) as ctx:
        ctx.set_step_kernel(seg)
        assert ctx.step_kernel() == seg
        gx, gz, f = ctx.forward(shots[0], g["src"], fields=True)
        imgs = ctx.rtm_batch(shots, g["src"])
        st = ctx.stack()
    return gx, gz, f, imgs, st


def _same(a, b):
    gx, gz, f, imgs, st = a
    hx, hz, h, jmgs, su = b
    assert np.array_equal(gx, hx) and np.array_equal(gz, hz)
    assert np.array_equal(f, h)
    for (p, q), (r, s) in zip(imgs, jmgs):
        assert np.array_equal(p, r, equal_nan=True) and np.array_equal(q, s, equal_nan=True)
    for x, y in zip(st, su):
        assert np.array_equal(x, y, equal_nan=True)


@pytest.mark.parametrize("name", CASES)
def test_march_equals_tiles(name):
    g = load_golden(name)
    ref = _run(g, 0)
    for seg in SEGS:
        _same(_run(g, seg), ref)


@pytest.mark.parametrize("over", [dict(strip_precision=o.PREC_FP16), dict(strip_precision=o.PREC_BF16),
                                  dict(snapshot_every=4), dict(compensated_image=1),
                                  dict(strip_level=o.STRIP_EXACT, image_align=o.IMAGE_EXACT)])
def test_march_equals_tiles_in_every_form(over):
    g = load_golden("g72x56n5")
    shots = [golden_shot(g)]
    for sx in (9, 41):
        s = golden_shot(g)
        s.sx = sx
        shots.append(s)
    ref = _run(g, 0, shots, **over)
    _same(_run(g, 48, shots, **over), ref)
    _same(_run(g, QUEUE, shots, **over), ref)


def test_march_equals_tiles_force_source_and_density():
    g = load_golden("g72x56n5")
    L = int(g["L"])
    X, Z = int(g["X"]), int(g["Z"])
    rho = np.linspace(1800, 2600, (X - 2 * L) * (Z - 2 * L)).reshape(X - 2 * L, Z - 2 * L).astype(np.float32)
    res = []
    for seg in (0, 32, QUEUE):
        sh = golden_shot(g)
        sh.src_type = o.SRC_FORCE_Z
        with make_context(g) as ctx:
            ctx.set_step_kernel(seg)
            res.append(ctx.forward(sh, g["src"], fields=True))
        kw = dict(nx=X - 2 * L, nz=Z - 2 * L, npml=L, dx=float(g["dx"]), dz=float(g["dx"]), dt=float(g["dt"]),
                  nt=int(g["NT"]), half_order=int(g["N"]), density=1)
        with o.Context(o.Config(**kw), g["vp"][L:X - L, L:Z - L], g["vs"][L:X - L, L:Z - L], rho) as ctx:
            ctx.set_step_kernel(seg)
            res.append(ctx.forward(golden_shot(g), g["src"], fields=True))
            res.append(ctx.rtm_shot(golden_shot(g), g["src"]))
    for other in (res[3:6], res[6:9]):
        for a, b in zip(res[:3], other):
            for x, y in zip(a, b):
                assert np.array_equal(x, y, equal_nan=True)


def test_march_equals_tiles_on_a_survey():
    from ouc_b200 import models
    vp, vs, _ = models.flat_layers(300, 112, 4, np.random.default_rng(21))
    cfg = o.Config(nx=300, nz=112, npml=20, dx=5.0, dz=5.0, dt=5e-4, nt=300, half_order=5, max_batch=3)
    wav, t0 = o.ricker(30.0, cfg.dt, cfg.nt)
    shots = [o.Shot(40, 2, 2, t0=t0), o.Shot(150, 2, 2, t0=t0), o.Shot(260, 2, 2, t0=t0)]
    aps = [(0, 120), (60, 250), (150, 300)]
    out = []
    for seg in (0, 64, QUEUE):
        with o.Context(cfg, vp, vs) as ctx:
            ctx.set_step_kernel(seg)
            recs = ctx.survey_forward(shots, aps, wav)
            imgs = ctx.survey_rtm(shots, aps, wav, recs)
            out.append((recs, imgs, ctx.stack()))
    r0, i0, s0 = out[0]
    for r1, i1, s1 in out[1:]:
        for a, b in zip(r0, r1):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        for a, b in zip(i0, i1):
            assert np.array_equal(a[0], b[0], equal_nan=True) and np.array_equal(a[1], b[1], equal_nan=True)
        for a, b in zip(s0, s1):
            assert np.array_equal(a, b, equal_nan=True)


def test_step_kernel_rejects_bad_segments():
    g = load_golden("g64n6")
    with make_context(g) as ctx:
        for bad in (-16, -2, 8, 20):
            with pytest.raises(o.OucError):
                ctx.set_step_kernel(bad)
        assert ctx.step_kernel() == 0   # the default is the tile kernel (measured faster); tuning may pick the march
