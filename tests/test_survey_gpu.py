"""The batching form: shots of uneven aperture on their own sub-grids of one
model, advanced together in one launch per stage.  Each shot must equal, bit
for bit, a single-shot run of a context created on its window of the padded
model (model_layout = PADDED), and the FP64 stack must equal the sum of the
per-shot images placed at their rows."""
import numpy as np
import pytest

import ouc_b200 as o
from helpers import golden_shot, load_golden, make_context
from ouc_b200 import models

pytestmark = pytest.mark.gpu

NX, NZ, L, N, NT, DX, DT = 300, 112, 20, 5, 400, 5.0, 5e-4
APERTURES = [(0, 120), (60, 250), (100, 180), (150, 300), (30, 90)]
SOURCES = [40, 150, 140, 260, 60]


def layered():
    vp, vs, _ = models.flat_layers(NX, NZ, 4, np.random.default_rng(21))
    return vp, vs


def cfg(nx, batch, layout=o.MODEL_INTERIOR):
    return o.Config(nx=nx, nz=NZ, npml=L, dx=DX, dz=DX, dt=DT, nt=NT, half_order=N, device=0, max_batch=batch,
                    model_layout=layout)


def window_context(vp_pad, vs_pad, ap):
    x0, x1 = ap
    return o.Context(cfg(x1 - x0, 1, o.MODEL_PADDED), np.ascontiguousarray(vp_pad[x0:x1 + 2 * L]),
                     np.ascontiguousarray(vs_pad[x0:x1 + 2 * L]))


@pytest.fixture(scope="module")
def model_and_wavelet(oracle):
    vp, vs = layered()
    vp_pad = oracle.pad(np.pad(vp, L), L)
    vs_pad = oracle.pad(np.pad(vs, L), L)
    w, t0 = o.ricker(25.0, DT, NT)
    shots = [o.Shot(sx=s, sz=2, rz=2, t0=t0, mute=1) for s in SOURCES]
    return vp, vs, vp_pad, vs_pad, w, shots


def test_subgrid_gathers_equal_window_runs(model_and_wavelet):
    vp, vs, vp_pad, vs_pad, w, shots = model_and_wavelet
    with o.Context(cfg(NX, 4), vp, vs) as ctx:
        got = ctx.survey_forward(shots, APERTURES, w)
    for s, ap, (gx, gz) in zip(shots, APERTURES, got):
        with window_context(vp_pad, vs_pad, ap) as wc:
            rx, rz, _ = wc.forward(o.Shot(sx=s.sx - ap[0], sz=s.sz, rz=s.rz, t0=s.t0, mute=s.mute), w)
        assert np.array_equal(gx, rx) and np.array_equal(gz, rz), ap


def test_subgrid_rtm_equals_window_runs_and_stacks(model_and_wavelet):
    vp, vs, vp_pad, vs_pad, w, shots = model_and_wavelet
    with o.Context(cfg(NX, 4), vp, vs) as ctx:
        recs = ctx.survey_forward(shots, APERTURES, w)
        imgs = ctx.survey_rtm(shots, APERTURES, w, recs)
        spp, sps, _ = ctx.stack()
    ref_pp = np.zeros((NX, NZ))
    ref_ps = np.zeros((NX, NZ))
    for s, ap, (pp, ps), rec in zip(shots, APERTURES, imgs, recs):
        with window_context(vp_pad, vs_pad, ap) as wc:
            wpp, wps = wc.rtm_shot(o.Shot(sx=s.sx - ap[0], sz=s.sz, rz=s.rz, t0=s.t0, mute=s.mute), w, rec)
        assert np.array_equal(pp, wpp) and np.array_equal(ps, wps), ap
        assert np.abs(pp).max() > 0
        ref_pp[ap[0]:ap[1]] += wpp
        ref_ps[ap[0]:ap[1]] += wps
    assert np.array_equal(spp, ref_pp) and np.array_equal(sps, ref_ps)


def test_subgrid_arguments_are_checked(model_and_wavelet):
    vp, vs, _, _, w, shots = model_and_wavelet
    with o.Context(cfg(NX, 2), vp, vs) as ctx:
        with pytest.raises(o.OucError):
            ctx.survey_forward(shots[:1], [(200, 300)], w)      # source outside its aperture
        with pytest.raises(o.OucError):
            ctx.survey_forward(shots[:1], [(0, 400)], w)        # beyond the model


def test_migrate_on_one_rank_equals_rtm_batch_and_stack():
    """survey.migrate at world size 1 (the function a multi-GPU survey calls
    on every rank) gives the stack of rtm_batch over the same shots."""
    from ouc_b200 import survey
    g = load_golden("g72x56n5")
    shots = [golden_shot(g)]
    for sx in (9, 30, 41):
        s = golden_shot(g)
        s.sx = sx
        shots.append(s)
    with make_context(g, max_batch=2) as a:
        a.rtm_batch(shots, g["src"])
        ref = a.stack(reset=True)
    with make_context(g, max_batch=2) as b:
        got = survey.migrate(b, shots, g["src"])
    for x, y in zip(got, ref):
        assert np.array_equal(x, y)
