"""ouc_run, the command-line driver that reproduces the reference's main()
workflow (per-shot Laplacian images and stacks as raw float32 files under
the reference's names, plus a manifest for resuming).

CPU tests: argument handling and the resume guard, which run before any
device work.  GPU tests: the files equal the library's own results, and a
run stopped part-way and resumed writes exactly what an uninterrupted run
writes.
"""
import os
import subprocess

import numpy as np
import pytest

import ouc_b200 as o
from helpers import load_golden

BIN = os.path.join(os.path.dirname(o.LIB_PATH), "..", "bin", "ouc_run")


def _run(*args, check_rc=None):
    assert os.path.exists(BIN), f"{BIN} is not built; run `make -C ouc_b200`"
    p = subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=600)
    if check_rc is not None:
        assert p.returncode == check_rc, (p.returncode, p.stdout, p.stderr)
    return p


def _case(tmp_path):
    """Small survey on the layered golden model: interior 52 x 36, N = 5, 5 shots."""
    g = load_golden("g72x56n5")
    L = int(g["L"])
    vp = np.ascontiguousarray(g["vp"][L:-L, L:-L])
    vs = np.ascontiguousarray(g["vs"][L:-L, L:-L])
    vp.tofile(tmp_path / "vp.bin")
    vs.tofile(tmp_path / "vs.bin")
    nx, nz = vp.shape
    args = ["--nx", nx, "--nz", nz, "--npml", L, "--order", 5, "--nt", 300, "--dx", 10, "--dz", 10, "--dt", 1e-3,
            "--fm", 25, "--shots", 5, "--sx0", 4, "--dsx", 10, "--sz", 2, "--rz", 2, "--batch", 2,
            "--vp", tmp_path / "vp.bin", "--vs", tmp_path / "vs.bin"]
    return args, vp, vs


def test_cli_usage_and_bad_arguments(tmp_path):
    assert "usage" in _run("--help", check_rc=0).stdout
    _run("--no-such-option", check_rc=1)
    _run("--vp", tmp_path / "x.bin", check_rc=1)          # --vp without --vs
    _run("--nx", "abc", check_rc=1)


def test_cli_resume_refuses_a_manifest_of_other_parameters(tmp_path):
    out = tmp_path / "img"
    out.mkdir()
    (out / "manifest.txt").write_text("ouc_run nx=1 something else\ndone illum_0_0.f64 0\n")
    p = _run("--out", out, "--resume", check_rc=1)
    assert "other parameters" in p.stderr
    assert (out / "manifest.txt").read_text().startswith("ouc_run nx=1")   # left as it was


@pytest.mark.gpu
def test_cli_files_equal_library_results(tmp_path):
    args, vp, vs = _case(tmp_path)
    out = tmp_path / "a"
    _run(*args, "--out", out, check_rc=0)
    nx, nz = vp.shape
    cfg = o.Config(nx=nx, nz=nz, npml=10, dx=10.0, dz=10.0, dt=1e-3, nt=300, half_order=5, max_batch=2)
    w, t0 = o.ricker(25.0, cfg.dt, cfg.nt)
    shots = [o.Shot(sx=4 + 10 * l, sz=2, rz=2, t0=t0) for l in range(5)]
    with o.Context(cfg, vp, vs) as ctx:
        imgs = ctx.rtm_batch(shots, w)
        spp, sps, sil = ctx.stack()
    acc_pp = np.zeros((nx, nz), np.float32)
    for l, (pp, ps) in enumerate(imgs):
        fpp = np.fromfile(out / f"image_PP_lap_{nx}_{nz}_{l}.dat", np.float32).reshape(nx, nz)
        fps = np.fromfile(out / f"image_PS_lap_{nx}_{nz}_{l}.dat", np.float32).reshape(nx, nz)
        assert np.array_equal(fpp, pp) and np.array_equal(fps, ps), l
        acc_pp += fpp                                      # the reference's float32 sum in shot order
    assert np.array_equal(np.fromfile(out / "All_image_PP_lap.dat", np.float32).reshape(nx, nz), acc_pp)
    np.testing.assert_allclose(np.fromfile(out / "All_image_PP_lap_f64.dat").reshape(nx, nz), spp, rtol=1e-12,
                               atol=1e-12 * np.abs(spp).max())
    np.testing.assert_allclose(np.fromfile(out / "All_illum_f64.dat").reshape(nx, nz), sil, rtol=1e-12,
                               atol=1e-12 * np.abs(sil).max())


@pytest.mark.gpu
def test_cli_stopped_and_resumed_equals_uninterrupted(tmp_path):
    args, _, _ = _case(tmp_path)
    a, b = tmp_path / "a", tmp_path / "b"
    _run(*args, "--out", a, check_rc=0)
    p = _run(*args, "--out", b, "--stop-after", 2, check_rc=3)
    assert "resume" in p.stdout
    assert not (b / "All_image_PP_lap.dat").exists()
    p = _run(*args, "--out", b, "--resume", check_rc=0)
    assert "2 done before, 3 to migrate" in p.stdout
    for f in sorted(os.listdir(a)):
        if f.endswith(".dat") or f.startswith("All_"):
            assert (a / f).read_bytes() == (b / f).read_bytes(), f
    p = _run(*args, "--out", b, "--resume", check_rc=0)    # all done: nothing migrated, same stacks
    assert "0 to migrate" in p.stdout
    assert (a / "All_illum_f64.dat").read_bytes() == (b / "All_illum_f64.dat").read_bytes()
