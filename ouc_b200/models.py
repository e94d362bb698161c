"""Seeded synthetic models and survey geometries for the modeling / RTM
workloads (the reference ships only a built-in three-layer model,
P-S-seperating.cu:1999-2040; these workloads scale it up).

All randomness uses numpy's PCG64 generator with an explicit seed, so a
workload is reproducible from its name and seed.  Models are interior grids
(nx, nz), x-major with z contiguous; the library pads them into the
absorbing layer itself.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .api import Config, Shot


@dataclass
class Workload:
    name: str
    cfg: Config
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    fm: float
    shots: list = field(default_factory=list)
    vp_mig: np.ndarray | None = None   # migration model (None: the true model)
    vs_mig: np.ndarray | None = None
    apertures: list | None = None      # per-shot sub-grids: interior columns (x0, x1)

    def cell_updates_per_shot(self, rtm=True):
        """Cell-updates of one shot: forward and receiver on the padded grid,
        reconstruction on the interior."""
        C = self.cfg.X * self.cfg.Z
        Ci = self.cfg.nx * self.cfg.nz
        return self.cfg.nt * ((2 * C + Ci) if rtm else C)


def gaussian_smooth(a, sigma):
    """Separable Gaussian smoothing (sigma in cells, edges reflected)."""
    r = int(np.ceil(3 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = np.asarray(a, dtype=np.float64)
    for axis in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[axis] = (r, r)
        p = np.pad(out, pad, mode="reflect")
        acc = np.zeros_like(out)
        n = out.shape[axis]
        for i, w in enumerate(k):
            sl = [slice(None), slice(None)]
            sl[axis] = slice(i, i + n)
            acc += w * p[tuple(sl)]
        out = acc
    return out.astype(np.float32)


def gardner(vp):
    return (0.31 * np.asarray(vp, np.float64) ** 0.25).astype(np.float32)


def two_layer(nx=256, nz=256, zi=128):
    """Homogeneous medium with one flat interface at depth index zi."""
    z = np.arange(nz)
    vp = np.where(z < zi, 3000.0, 3800.0)[None, :].repeat(nx, 0).astype(np.float32)
    vs = np.where(z < zi, 3000.0 / 1.73, 2200.0)[None, :].repeat(nx, 0).astype(np.float32)
    rho = np.where(z < zi, 2000.0, 2300.0)[None, :].repeat(nx, 0).astype(np.float32)
    return vp, vs, rho


def flat_layers(nx, nz, nlayers, rng, vp_lo=1800.0, vp_hi=4500.0, ratio=(1.6, 2.0)):
    """nlayers flat layers with seeded thicknesses and velocities."""
    cuts = np.sort(rng.choice(np.arange(1, nz), size=nlayers - 1, replace=False))
    vps = rng.uniform(vp_lo, vp_hi, nlayers)
    rs = rng.uniform(ratio[0], ratio[1], nlayers)
    idx = np.searchsorted(cuts, np.arange(nz), side="right")
    vp = vps[idx][None, :].repeat(nx, 0).astype(np.float32)
    vs = (vps / rs)[idx][None, :].repeat(nx, 0).astype(np.float32)
    return vp, vs, gardner(vp)


def folded_model(nx, nz, rng, nlayers=10, nfaults=3, nanom=20):
    """Folded layers (sinusoidal interfaces), dipping faults with random
    throw and Gaussian velocity anomalies of +/-10%."""
    x = np.arange(nx)[:, None].astype(np.float64)
    z = np.arange(nz)[None, :].astype(np.float64)
    base = np.sort(rng.uniform(0.05 * nz, 0.95 * nz, nlayers - 1))
    amp = rng.uniform(5, 40, nlayers - 1)
    lam = rng.uniform(0.3 * nx, 1.5 * nx, nlayers - 1)
    ph = rng.uniform(0, 2 * np.pi, nlayers - 1)
    zz = np.broadcast_to(z, (nx, nz)).copy()
    # faults: shift depth on one side of a dipping plane
    for _ in range(nfaults):
        x0 = rng.uniform(0.1 * nx, 0.9 * nx)
        dip = rng.uniform(-1.5, 1.5)
        throw = rng.uniform(-30, 30)
        side = (x - x0 - dip * z) > 0
        zz = zz + np.where(side, throw, 0.0)
    layer = np.zeros((nx, nz), np.int64)
    for k in range(nlayers - 1):
        iface = base[k] + amp[k] * np.sin(2 * np.pi * x / lam[k] + ph[k])
        layer += (zz > iface).astype(np.int64)
    vps = np.sort(rng.uniform(1800, 4500, nlayers))
    rs = rng.uniform(1.6, 2.0, nlayers)
    vp = vps[layer]
    vs = (vps / rs)[layer]
    pert = np.ones((nx, nz))
    for _ in range(nanom):
        cx, cz = rng.uniform(0, nx), rng.uniform(0, nz)
        sg = rng.uniform(5, 30)
        pert += rng.uniform(-0.1, 0.1) * np.exp(-((x - cx) ** 2 + (z - cz) ** 2) / (2 * sg * sg))
    vp = (vp * pert).astype(np.float32)
    vs = (vs * pert).astype(np.float32)
    return vp, vs, gardner(vp)


def c1(nt=1000):
    """Plain single-shot forward modeling: 256^2 interior + 20-cell CPML,
    dx = 10 m, dt = 1 ms, 20 Hz Ricker at (128, 2), receivers on z = 2."""
    vp, vs, rho = two_layer()
    cfg = Config(nx=256, nz=256, npml=20, dx=10.0, dz=10.0, dt=1e-3, nt=nt, half_order=5)
    return Workload("c1_forward_256x256_nt1000", cfg, vp, vs, rho, 20.0, [Shot(128, 2, 2)])


def c2(nt=4000, seed=1236, nshots=40):
    """Plain elastic P/S RTM: 1000 x 500 interior, dx = 5 m, 30-cell CPML,
    8 seeded flat layers, migration model Gaussian-smoothed (sigma = 10),
    40 shots evenly spaced on z = 2, full-spread receivers, 25 Hz,
    dt = 0.5 ms, nt = 4000."""
    rng = np.random.default_rng(seed)
    vp, vs, rho = flat_layers(1000, 500, 8, rng)
    cfg = Config(nx=1000, nz=500, npml=30, dx=5.0, dz=5.0, dt=5e-4, nt=nt, half_order=5)
    xs = np.linspace(0, 999, nshots).round().astype(int)
    shots = [Shot(int(x), 2, 2) for x in xs]
    return Workload("c2_rtm_1000x500_nt4000", cfg, vp, vs, rho, 25.0, shots,
                    gaussian_smooth(vp, 10.0), gaussian_smooth(vs, 10.0))


def c3(nt=6000, seed=1237, nshots=256):
    """Batched uneven-shot RTM: 2000 x 800 interior, dx = 5 m, 30-cell CPML;
    folded layers with 3 faults and 20 velocity anomalies (+/-10 %); 256
    shots on z = 2, each on its own sub-grid: a receiver aperture of U[400,
    1600] cells centred on the source (shifted inside the model); 30 Hz,
    dt = 0.4 ms, nt = 6000; migration model Gaussian-smoothed (sigma = 10)."""
    rng = np.random.default_rng(seed)
    vp, vs, rho = folded_model(2000, 800, rng)
    cfg = Config(nx=2000, nz=800, npml=30, dx=5.0, dz=5.0, dt=4e-4, nt=nt, half_order=5)
    xs = np.linspace(0, 1999, nshots).round().astype(int)
    widths = rng.uniform(400, 1600, nshots).round().astype(int)
    shots, aps = [], []
    for x, a in zip(xs, widths):
        x0 = int(max(0, min(x - a // 2, 2000 - a)))
        shots.append(Shot(int(x), 2, 2))
        aps.append((x0, x0 + int(a)))
    return Workload("c3_survey_2000x800_nt6000", cfg, vp, vs, rho, 30.0, shots, gaussian_smooth(vp, 10.0),
                    gaussian_smooth(vs, 10.0), aps)


def c4(nt=8000, seed=1238, nshots=128):
    """Mixed-precision RTM family at scale: 4000 x 1500, dx = 4 m, nt = 8000.
    dt = 0.4 ms: the 0.5 ms of the smaller workload would exceed the
    10th-order CFL limit at 4500 m/s and 4 m spacing."""
    rng = np.random.default_rng(seed)
    vp, vs, rho = flat_layers(4000, 1500, 8, rng)
    cfg = Config(nx=4000, nz=1500, npml=30, dx=4.0, dz=4.0, dt=4e-4, nt=nt, half_order=5)
    xs = np.linspace(0, 3999, nshots).round().astype(int)
    return Workload("c4_rtm_4000x1500_nt8000", cfg, vp, vs, rho, 25.0, [Shot(int(x), 2, 2) for x in xs],
                    gaussian_smooth(vp, 10.0), gaussian_smooth(vs, 10.0))
