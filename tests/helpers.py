"""Shared test helpers: fixtures, error norms, context construction."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("g64n6", "g72x56n5", "g48x40n2")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def worst(errors):
    """Largest error of a dict of errors; a NaN error counts as infinite (a
    plain max() would skip it depending on the order)."""
    v = [float(x) for x in errors.values()]
    return float("inf") if any(np.isnan(x) for x in v) else max(v)


def finite_rel_l2(a, b):
    """rel_l2 over the cells finite in both; the NaN/Inf cells must coincide
    (0/0 image cells where the illumination is zero, as the reference gives)."""
    fa, fb = np.isfinite(a), np.isfinite(b)
    assert np.array_equal(fa, fb), "non-finite cells differ"
    return rel_l2(np.asarray(a)[fa], np.asarray(b)[fb])


def shot_cfg(g):
    from oracle.oracle import Shot
    return Shot(X=int(g["X"]), Z=int(g["Z"]), L=int(g["L"]), N=int(g["N"]), nt=int(g["NT"]), sx=int(g["sx"]),
                sz=int(g["sz"]), rz=int(g["rz"]), dx=float(g["dx"]), dz=float(g["dx"]), dt=float(g["dt"]),
                t0=int(g["t0"]))


def make_context(g, **over):
    """Library context on the golden case's model (interior part; the library pads)."""
    import ouc_b200 as o
    L = int(g["L"])
    X, Z = int(g["X"]), int(g["Z"])
    kw = dict(nx=X - 2 * L, nz=Z - 2 * L, npml=L, dx=float(g["dx"]), dz=float(g["dx"]), dt=float(g["dt"]),
              nt=int(g["NT"]), half_order=int(g["N"]))
    kw.update(over)
    cfg = o.Config(**kw)
    vp = g["vp"][L:X - L, L:Z - L]
    vs = g["vs"][L:X - L, L:Z - L]
    return o.Context(cfg, vp, vs)


def golden_shot(g, mute=1):
    import ouc_b200 as o
    L = int(g["L"])
    return o.Shot(sx=int(g["sx"]) - L, sz=int(g["sz"]) - L, rz=int(g["rz"]) - L, t0=int(g["t0"]), mute=mute)


def strip_bytes_fp64(cfg):
    """Host bytes of the FP64 oracle's boundary strips for one RTM shot of
    `cfg` (8 fields of the 2N-wide bands around the interior, every step)."""
    N, X, Z = cfg.half_order, cfg.nx + 2 * cfg.npml, cfg.nz + 2 * cfg.npml
    return 8 * 8 * (cfg.nt - 1) * 2 * 2 * N * (X + Z)


def require_host_memory(nbytes, factor=4):
    """Skip the test unless the host has `factor` x nbytes of memory available
    (the FP64 oracle of a long shot keeps large strip arrays)."""
    import psutil
    import pytest
    avail = psutil.virtual_memory().available
    if avail < factor * nbytes:
        pytest.skip(f"needs {factor * nbytes / 2**30:.0f} GiB of host memory, {avail / 2**30:.0f} GiB available")
