"""The learned coarse path: half-order 2 at twice the spacing and time step,
corrected every 8 steps by the CNN trained on the GPU on fine/coarse pairs
the method generates; the fine half-order-5 run is the referee.

Workload: fine 2 m / 0.2 ms, 256 x 192 interior + 20-cell CPML (coarse 4 m /
0.4 ms, 128 x 96 + 10), 30 Hz Ricker, seeded random flat-layer models with
Vp ~ U[1800, 4500] m/s and Vp/Vs ~ U[1.6, 2.0]; sources at fine depth 96,
receivers at fine depth 48 (away from the absorbing layers).  Misfits are
taken over the first 0.12 s (300 coarse steps: the direct and first
reflected arrivals) at receivers 12 or more coarse cells from the source;
later samples are dominated by the absorbing layers' late-time residue,
which differs between stencil orders even on one grid."""
import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import learned, models
from ouc_b200.corrector import Net, N_IN

pytestmark = pytest.mark.gpu

NX, NZ, L, DX, DT, NT = 256, 192, 20, 2.0, 2e-4, 1200
FM = 30.0
EVERY = 8
EARLY = 300          # coarse samples compared (0.12 s)
SZ, RZ = 96, 48      # fine source and receiver depths (interior cells)


def fine_cfg():
    return o.Config(nx=NX, nz=NZ, npml=L, dx=DX, dz=DX, dt=DT, nt=NT, half_order=5, device=0)


def model(seed):
    rng = np.random.default_rng(seed)
    vp, vs, _ = models.flat_layers(NX, NZ, 5, rng)
    return vp, vs


def shots_for(seed, n):
    rng = np.random.default_rng(seed + 7)
    return [o.Shot(sx=2 * int(rng.integers(20, NX // 2 - 20)), sz=SZ, rz=RZ, mute=0) for _ in range(n)]


def misfit(g, ref, shot):
    cols = [c for c in range(0, NX // 2, 2) if abs(c - shot.sx // 2) >= 12]
    early = lambda pair: tuple(np.asarray(a)[:, :EARLY] for a in pair)
    return learned.trace_error(early(g), early(ref), cols, L // 2)


def test_restricted_gathers_sample_the_fine_state():
    """The referee's gathers equal the 4-point midpoint restriction of the fine
    run's own displacement (numpy, from the final fields of the same run)."""
    vp, vs = model(5)
    w, _ = o.ricker(FM, DT, NT)
    shot = o.Shot(sx=128, sz=4, rz=4, mute=0)
    with learned.Twin(fine_cfg(), vp, vs) as tw:
        gx, gz = tw.fine_forward_restricted(shot, w)
        _, _, f = tw.fine.forward(shot, w, fields=True)
        Xc = tw.coarse.X
    ux, uz = f[0].astype(np.float64), f[1].astype(np.float64)
    j = 2 * ((shot.rz + L) // 2)
    i = 2 * np.arange(Xc)

    def at(a, ii, jj):
        ok = (ii >= 0) & (ii < a.shape[0]) & (jj >= 0) & (jj < a.shape[1])
        return np.where(ok, a[np.clip(ii, 0, a.shape[0] - 1), np.clip(jj, 0, a.shape[1] - 1)], 0.0)
    rx = (9 * (at(ux, i, j) + at(ux, i + 1, j)) - (at(ux, i - 1, j) + at(ux, i + 2, j))) / 16
    rz = (9 * (at(uz, i, j) + at(uz, i, j + 1)) - (at(uz, i, j - 1) + at(uz, i, j + 2))) / 16
    last_x, last_z = gx[:, -1], gz[:, -1]        # coarse level nt_c = fine level nt
    assert np.allclose(last_x, rx, rtol=1e-5, atol=1e-6 * np.abs(rx).max())
    assert np.allclose(last_z, rz, rtol=1e-5, atol=1e-6 * np.abs(rz).max())


def test_plain_coarse_run_tracks_the_fine_run():
    """The coarse method itself: in a homogeneous medium it stays within 2 %
    of the fine run over the direct arrivals (little dispersion at 30 Hz on
    4 m); in layered media within 20 % (the interfaces are resolved at 4 m
    and treated differently by the two stencils)."""
    w, _ = o.ricker(FM, DT, NT)
    shot = o.Shot(sx=128, sz=SZ, rz=RZ, mute=0)
    vh = np.full((NX, NZ), 3000.0, np.float32)
    cases = {"homogeneous": (vh, vh / np.float32(1.8)), "layered": model(6)}
    e = {}
    for name, (vp, vs) in cases.items():
        with learned.Twin(fine_cfg(), vp, vs) as tw:
            e[name] = misfit(tw.coarse_forward(shot, w, None), tw.fine_forward_restricted(shot, w), shot)
    print("plain coarse misfit", e)
    assert e["homogeneous"] < 0.02
    assert e["layered"] < 0.2


@pytest.fixture(scope="module")
def trained():
    """Teacher-forced pairs (3 models x 2 shots) with 2 % input noise, 8
    epochs; then one on-policy round (2 models, the network in the loop) and
    4 more epochs."""
    import torch
    dev = torch.device("cuda", 0)
    w, _ = o.ricker(FM, DT, NT)
    cc = learned.coarse_config(fine_cfg())
    H, W = cc.X, cc.Z
    cap = 640
    d_in = torch.empty((cap, H, W, N_IN), dtype=torch.float32, device=dev)
    d_tgt = torch.empty((cap, H, W, 8), dtype=torch.float32, device=dev)
    net = Net(0, learned.init_params(seed=1))

    def gen(seeds, nshots, n, with_net):
        for m in seeds:
            vp, vs = model(m)
            with learned.Twin(fine_cfg(), vp, vs) as tw:
                for s in shots_for(m, nshots):
                    n += tw.pairs(s, w, EVERY, d_in.data_ptr() + n * H * W * N_IN * 4,
                                  d_tgt.data_ptr() + n * H * W * 8 * 4, cap - n, net if with_net else None,
                                  noise=0.02, seed=m)
                rect = tw.interior()
        return n, rect
    n, rect = gen(range(100, 103), 2, 0, False)
    loss1 = learned.train(net, d_in.data_ptr(), d_tgt.data_ptr(), n, H, W, rect, batch=8, epochs=8, lr=1e-3, seed=2)
    n, _ = gen(range(200, 202), 1, n, True)
    loss2 = learned.train(net, d_in.data_ptr(), d_tgt.data_ptr(), n, H, W, rect, batch=8, epochs=4, lr=5e-4, seed=3)
    torch.cuda.synchronize()
    print("pairs", n, "loss", loss1, loss2)
    yield net, n, loss1
    net.close()


def test_training_lowers_the_loss(trained):
    _, n, loss = trained
    assert n >= 400
    assert np.all(np.isfinite(loss))
    assert loss[-1] < 0.7 * loss[0]


def test_trained_corrector_against_the_plain_coarse_run(trained):
    """What the trained network gains over the coarse method without it, on
    held-out models: measured and printed (the corrected run must stay
    finite).  On this workload the gain is negative -- the corrected run
    misfits 0.1-1.6 against the plain run's 0.04-0.10, varying between runs
    because the weight-gradient sums are accumulated in no fixed order: at
    30 Hz on 4 m the coarse method's own error over one 8-step interval is
    small, and the network's residual on held-out states is larger than what
    it corrects.  The spot check below is what keeps such shots out of
    the delivered results."""
    net, _, _ = trained
    w, _ = o.ricker(FM, DT, NT)
    plain, corr = [], []
    for m in range(2):
        vp, vs = model(900 + m)
        with learned.Twin(fine_cfg(), vp, vs) as tw:
            for s in shots_for(900 + m, 2):
                ref = tw.fine_forward_restricted(s, w)
                plain.append(misfit(tw.coarse_forward(s, w, None), ref, s))
                corr.append(misfit(tw.coarse_forward(s, w, net, EVERY), ref, s))
    gain = 1.0 - np.mean(corr) / np.mean(plain)
    print("misfit plain", np.round(plain, 4), "corrected", np.round(corr, 4), "gain %.3f" % gain)
    assert net.error() == 0
    assert np.all(np.isfinite(corr))


def test_spot_check_and_fallback(trained):
    """Checked shots above the tolerance are replaced by the fine run, and so
    are the unchecked shots after them; below it the coarse result stands."""
    net, _, _ = trained
    w, _ = o.ricker(FM, DT, NT)
    vp, vs = model(950)
    shots = shots_for(950, 4)
    with learned.Twin(fine_cfg(), vp, vs) as tw:
        strict = learned.model_shots(tw, net, shots, w, EVERY, check_every=2, tol=0.0)
        loose = learned.model_shots(tw, net, shots, w, EVERY, check_every=2, tol=1e9)
        ref1 = tw.fine_forward_restricted(shots[1], w)
    assert [r.checked for r in strict] == [True, False, True, False]
    assert all(r.fallback for r in strict)
    assert not any(r.fallback for r in loose)
    assert np.array_equal(strict[1].gathers[0], ref1[0])
    assert all(r.error is not None and r.error > 0 for r in strict if r.checked)
