"""CPU tests of the product's host side: the C ABI library loads and exports
every symbol include/ouc.h declares, and the host logic that runs before any
device work (weights, wavelet, configuration checks)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import ouc_b200 as o
from helpers import load_golden
from oracle.oracle import weights

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(ouc_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(o.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    from ouc_b200._lib import SIGNATURES
    assert set(declared_symbols()) <= set(SIGNATURES)


def test_version_and_strerror():
    lib = o.lib()
    assert lib.ouc_version() >= 1
    assert lib.ouc_strerror(0) == b"ok"
    assert b"CFL" in lib.ouc_strerror(4)


@pytest.mark.parametrize("n", [2, 4, 5, 6])
def test_stencil_weights_match_oracle(n):
    assert np.array_equal(o.stencil_weights(n), weights(n))


def test_ricker_matches_reference_construction():
    g = load_golden("g64n6")
    w, t0 = o.ricker(float(g["fm"]), float(g["dt"]), int(g["NT"]))
    assert t0 == int(g["t0"])
    assert np.max(np.abs(w - g["src"])) <= 2e-7 * np.max(np.abs(g["src"]))
    assert w[t0] == 1.0


@pytest.mark.parametrize("fm,dt,nt", [(30.0, 1e-3, 240), (25.0, 5e-4, 4000), (20.0, 1e-3, 1000), (30.0, 4e-4, 600)])
def test_oracle_ricker_equals_the_library_bit_for_bit(oracle, fm, dt, nt):
    # the CPU baseline builds its wavelet with the oracle's restatement
    w, t0 = o.ricker(fm, dt, nt)
    wo, t0o = oracle.ricker(fm, dt, nt)
    assert t0 == t0o
    assert np.array_equal(w, wo)


def test_create_rejects_bad_configs_without_touching_the_device():
    vp = np.full((64, 64), 3000, np.float32)
    vs = np.full((64, 64), 1700, np.float32)
    base = dict(nx=64, nz=64, npml=12, dx=10.0, dz=10.0, dt=1e-3, nt=10)
    with pytest.raises(o.OucError) as e:
        o.Context(o.Config(**base, half_order=3), vp, vs)
    assert e.value.code == 1
    with pytest.raises(o.OucError) as e:
        o.Context(o.Config(**{**base, "npml": 3}), vp, vs)
    assert e.value.code == 1
    with pytest.raises(o.OucError) as e:   # CFL: 3000*2e-3/10*1.3167*sqrt(2) = 1.12 > 1
        o.Context(o.Config(**{**base, "dt": 2e-3}), vp, vs)
    assert e.value.code == 4
    bad = vp.copy()
    bad[3, 3] = np.nan
    with pytest.raises(o.OucError) as e:
        o.Context(o.Config(**base), bad, vs)
    assert e.value.code == 1
    with pytest.raises(ValueError):
        o.Context(o.Config(**base), vp[:10], vs)
    for bad_cfg in ({"strip_precision": 3}, {"compensated_image": 2}):
        with pytest.raises(o.OucError) as e:
            o.Context(o.Config(**base, **bad_cfg), vp, vs)
        assert e.value.code == 1


def test_create_rejects_grids_beyond_32bit_field_offsets():
    """The kernels address within one field with 32-bit offsets, so a grid
    whose padded field would exceed 2^31 cells is refused before the model is
    read or the device touched.  Called through the C ABI with a dummy model
    (the Python wrapper would first want a model of that size), in a child
    process, so that a missing check fails this test instead of the run."""
    import subprocess
    import sys

    def field_cells(nx, nz, L):   # rows and pitch of one padded field
        X, Z = nx + 2 * L, nz + 2 * L
        rows = -(-X // 32) * 32 + 32
        pitch = -(-(-(-Z // 64) * 64 + 32) // 32) * 32
        return rows * pitch

    for nx, nz in ((50000, 50000), (200000, 12000)):
        assert field_cells(nx, nz, 20) > 2**31 - 1
        code = f"""
import ctypes as C, numpy as np, ouc_b200 as o
small = np.full(16, 3000, np.float32)
p = small.ctypes.data_as(C.POINTER(C.c_float))
h = C.c_void_p()
cfg = o.Config(nx={nx}, nz={nz}, npml=20, dx=10.0, dz=10.0, dt=1e-3, nt=10, half_order=5)
print(o.lib().ouc_create(C.byref(cfg.c()), p, p, None, C.byref(h)), bool(h.value))
"""
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120,
                           cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        assert r.returncode == 0, r.stderr[-2000:]
        assert r.stdout.split() == ["1", "False"], r.stdout
