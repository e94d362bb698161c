"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference's own kernels (P-S-seperating.cu, sizes patched, compiled
for the CPU by oracle/Makefile through oracle/refemu) with the launch
sequence of its main() for one shot, and stores inputs and outputs as .npz.
Needs the reference sources (only where they are mounted):

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures are what the tests compare the oracle and the CUDA path with on
machines that do not have the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Oracle, RefBuild, layered_model  # noqa: E402


def ricker_ref(fm, dt, nt):
    """PS:1954-1958 with the reference's constants and mixed precision."""
    nk = np.float32(3.1415926 * 3.1415926 * fm * fm * float(np.float32(dt)) * float(np.float32(dt)))
    t0 = int(np.ceil(1.0 / (fm * float(np.float32(dt)))))
    t = np.arange(nt)
    d = (t - t0).astype(np.float32)
    e = np.exp((-nk * d * d).astype(np.float32)).astype(np.float32)
    return ((1.0 - 2.0 * float(nk) * (t - t0) ** 2) * e.astype(np.float64)).astype(np.float32), t0


CASES = {
    # name: (fm, dt, dx, source offset along x from L, source z offset, receiver z offset)
    "g64n6": (30.0, 1e-3, 10.0, 5, 0, 0),
    "g72x56n5": (25.0, 1e-3, 10.0, 17, 2, 2),
    "g48x40n2": (30.0, 1e-3, 10.0, 9, 0, 0),
}


def make(name):
    fm, dt, dx, ox, oz, orz = CASES[name]
    ref = RefBuild(name, "emu")
    orc = Oracle()
    X, Z, L, N, NT = ref.X, ref.Z, ref.L, ref.N, ref.NT
    vp, vs = layered_model(X, Z, L)
    _, vp, vs = ref.pad(np.ones_like(vp), vp, vs)          # the reference's own padding
    ax, az = orc.profile(vp, L)
    src, t0 = ricker_ref(fm, dt, NT)
    sx, sz, rz = L + ox, L + oz, L + orz
    gx, gz, _, _ = ref.forward(sx, sz, rz, np.float32(dt), np.float32(dx), np.float32(dx), vp, vs, ax, az, src, NT)
    # fields are compared at mid-propagation: after NT steps these small grids hold only
    # the residual of the absorbed waves, where round-off dominates
    nt_mid = NT // 2
    _, _, f, _ = ref.forward(sx, sz, rz, np.float32(dt), np.float32(dx), np.float32(dx), vp, vs, ax, az, src, nt_mid)
    r = ref.rtm(sx, sz, rz, t0, np.float32(dt), np.float32(dx), np.float32(dx), vp, vs, ax, az, src)
    # first-order velocity-stress kernels (stress/velocity and their
    # backward-propagation twins): gathers, the 12 state fields at mid-run
    # (Vpx Vpz Vsx Vsz, the four Q fields, theta_x theta_z omega_x omega_z)
    # and the state after back-propagating the gathers
    args = (np.float32(dt), np.float32(dx), np.float32(dx), vp, vs, ax, az)
    fo_gx, fo_gz, _, _ = ref.forward_fo(sx, sz, rz, *args, src, NT)
    _, _, fo_f, _ = ref.forward_fo(sx, sz, rz, *args, src, nt_mid)
    fo_b, _ = ref.backward_fo(rz, *args, fo_gx, fo_gz, NT)
    fo_state = [2, 3, 4, 5, 8, 9, 10, 11, 12, 13, 14, 15]
    out = dict(X=X, Z=Z, L=L, N=N, NT=NT, nt_mid=nt_mid, fm=fm, dt=dt, dx=dx, sx=sx, sz=sz, rz=rz, t0=t0,
               vp=vp, vs=vs, ax=ax, az=az, src=src,
               fwd_gx=gx, fwd_gz=gz, fwd_fields=f[:6],
               rtm_lap_pp=r["lap_pp"], rtm_lap_ps=r["lap_ps"], rtm_acc=r["acc"], rtm_rec=r["rec"],
               rtm_fields=r["fields"][:6],
               fo_gx=fo_gx, fo_gz=fo_gz, fo_fields=fo_f[fo_state], fo_bwd_fields=fo_b[fo_state])
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    for n in sys.argv[1:] or CASES:
        make(n)
