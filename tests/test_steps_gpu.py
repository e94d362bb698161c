"""The step-level interface (ouc_step_*): one RTM shot driven one reference
time step per call, in the order of the reference's main() (forward steps
t = 0..nt-1, then receiver + reconstruction steps t = nt-1..0, then the image
finalisation).  It must give exactly the whole-shot results, expose the
wavefields between steps, and refuse calls out of order.
"""
import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import _lib
from helpers import golden_shot, load_golden, make_context, rel_l2, worst

pytestmark = pytest.mark.gpu

TOL_FIELD = 5e-4      # vs the golden fields (CPU-run reference kernels): the FP32 round-off floor


def _step_shot(ctx, shot, w, recs=None, probe=None):
    ctx.step_begin(shot, w, recs)
    nt = ctx.cfg.nt
    seen = {}
    for t in range(nt):
        ctx.step_forward(t)
        if probe is not None and t + 1 == probe:
            seen["fwd"] = ctx.step_fields(0)
    for t in range(nt - 1, -1, -1):
        ctx.step_receiver(t)
        ctx.step_reconstruct(t)
    pp, ps = ctx.image_finalize()
    return pp, ps, seen


@pytest.mark.parametrize("name", ["g72x56n5", "g64n6"])
def test_stepped_shot_equals_whole_shot(name):
    g = load_golden(name)
    shot = golden_shot(g)
    with make_context(g) as ctx:
        pp0, ps0 = ctx.rtm_shot(shot, g["src"])
        spp0, sps0, sil0 = ctx.stack(reset=True)
        pp1, ps1, _ = _step_shot(ctx, shot, g["src"])
        spp1, sps1, sil1 = ctx.stack(reset=True)
    assert np.abs(pp0).max() > 0
    assert np.array_equal(pp0, pp1) and np.array_equal(ps0, ps1)
    assert np.array_equal(spp0, spp1) and np.array_equal(sps0, sps1) and np.array_equal(sil0, sil1)


def test_stepped_shot_with_observed_records():
    g = load_golden("g72x56n5")
    shot = golden_shot(g, mute=0)
    recs = (g["rtm_rec"][0], g["rtm_rec"][1])
    with make_context(g) as ctx:
        pp0, ps0 = ctx.rtm_shot(shot, g["src"], rec=recs)
        pp1, ps1, _ = _step_shot(ctx, shot, g["src"], recs=recs)
    assert np.array_equal(pp0, pp1) and np.array_equal(ps0, ps1)


def test_step_fields_match_forward_fields():
    g = load_golden("g72x56n5")
    nm = int(g["nt_mid"])
    shot = golden_shot(g)
    with make_context(g, nt=nm) as ctx:
        _, _, f_whole = ctx.forward(shot, g["src"][:nm], fields=True)
    with make_context(g) as ctx:
        _, _, seen = _step_shot(ctx, shot, g["src"], probe=nm)
    f = seen["fwd"]
    assert np.array_equal(f, f_whole)
    e = {n: rel_l2(f[k], g["fwd_fields"][k]) for k, n in enumerate(("Ux", "Uz", "Px", "Pz", "Sx", "Sz"))}
    print("stepped fields at t =", nm, "vs golden", e)
    assert worst(e) <= TOL_FIELD, e


def test_step_calls_out_of_order_are_refused():
    g = load_golden("g48x40n2")
    shot = golden_shot(g)
    with make_context(g) as ctx:
        with pytest.raises(o.OucError) as ei:
            ctx.step_forward(0)                  # nothing begun
        assert ei.value.code == _lib.OUC_ESTATE
        ctx.step_begin(shot, g["src"])
        ctx.step_forward(0)
        for bad in (lambda: ctx.step_forward(2), lambda: ctx.step_receiver(ctx.cfg.nt - 1),
                    lambda: ctx.image_finalize()):
            with pytest.raises(o.OucError) as ei:
                bad()
            assert ei.value.code == _lib.OUC_ESTATE
        ctx.step_forward(1)                      # the refused calls changed nothing
        ctx.rtm_shot(shot, g["src"])             # a whole-shot call ends the stepped shot
        with pytest.raises(o.OucError) as ei:
            ctx.step_forward(2)
        assert ei.value.code == _lib.OUC_ESTATE
