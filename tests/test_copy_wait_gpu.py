"""The step kernels' bounded copy wait reports instead of hanging.

With the test hook on, every tile expects 16 bytes more than its tensor
copies deliver, so the CTA's mbarrier wait runs out (about 40 ms), records
the failure in the context's status word and leaves the tile unwritten.  The
call must return OUC_ETIMEOUT, and the same context, with the hook off, must
then reproduce a fresh context's result bit for bit: no GPU fault, no hang,
the context stays usable."""
import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import _lib

pytestmark = pytest.mark.gpu


def _case():
    nx, nz, L = 48, 40, 12
    rng = np.random.default_rng(5)
    vp = (2600.0 + rng.uniform(-100, 100, (nx, nz))).astype(np.float32)
    vs = (vp / 1.8).astype(np.float32)
    cfg = o.Config(nx=nx, nz=nz, npml=L, dx=10.0, dz=10.0, dt=1e-3, nt=6, half_order=5, device=0)
    w = np.zeros(cfg.nt, np.float32)
    w[:3] = [1.0, -0.5, 0.25]
    return cfg, vp, vs, w, o.Shot(sx=20, sz=4, rz=4)


def test_copy_wait_times_out_and_context_recovers():
    cfg, vp, vs, w, shot = _case()
    with o.Context(cfg, vp, vs) as ref:
        gx0, gz0, _ = ref.forward(shot, w)
    assert np.abs(gz0).max() > 0
    with o.Context(cfg, vp, vs) as ctx:
        ctx.debug_copy_stall(True)
        with pytest.raises(o.OucError) as e:
            ctx.forward(shot, w)
        assert e.value.code == _lib.OUC_ETIMEOUT
        ctx.debug_copy_stall(False)
        gx, gz, _ = ctx.forward(shot, w)
    assert np.array_equal(gx, gx0) and np.array_equal(gz, gz0)
