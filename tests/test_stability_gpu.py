"""Runtime detection of a non-finite wavefield.

The reference checks nothing (its main() writes whatever the kernels
produce).  The library checks, after every forward pass, that the recorded
gathers and the final level are finite, and after every backward pass that
the imaging accumulators are, and returns OUC_EUNSTABLE instead of images
when they are not.  The failure is made with finite-looking inputs the
kernels turn into infinities (a wavelet sample near the float limit): the
arithmetic overflows, nothing faults, and the context stays usable for the
next call.
"""
import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import _lib
from helpers import golden_shot, load_golden, make_context

pytestmark = pytest.mark.gpu


def _bad_wavelet(g):
    w = g["src"].copy()
    w[int(g["t0"])] = 3e38          # theta and the displacement overflow within a few steps
    return w


def test_forward_reports_unstable_and_context_stays_usable():
    g = load_golden("g72x56n5")
    with make_context(g) as ctx:
        with pytest.raises(o.OucError) as e:
            ctx.forward(golden_shot(g), _bad_wavelet(g))
        assert e.value.code == _lib.OUC_EUNSTABLE
        gx, gz, _ = ctx.forward(golden_shot(g), g["src"])     # the next call is clean
    with make_context(g) as fresh:
        hx, hz, _ = fresh.forward(golden_shot(g), g["src"])
    assert np.array_equal(gx, hx) and np.array_equal(gz, hz)


def test_rtm_reports_unstable_and_context_stays_usable():
    g = load_golden("g72x56n5")
    with make_context(g) as ctx:
        with pytest.raises(o.OucError) as e:
            ctx.rtm_shot(golden_shot(g), _bad_wavelet(g))
        assert e.value.code == _lib.OUC_EUNSTABLE
        ctx.stack(reset=True)
        pp, ps = ctx.rtm_shot(golden_shot(g), g["src"])
    with make_context(g) as fresh:
        qp, qs = fresh.rtm_shot(golden_shot(g), g["src"])
    assert np.array_equal(pp, qp, equal_nan=True) and np.array_equal(ps, qs, equal_nan=True)
