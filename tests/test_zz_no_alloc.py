"""The no-allocation forward-modeling entry point (ouc_forward_noalloc).

It exists for callers that cannot allocate device memory when they need a
modeling run -- an application whose own pool owns the GPU's memory and
forbids other allocations, or a pipeline that reserved everything up front
and must not enter the allocator (which synchronises the device and can fail
under memory pressure).  Its wavefield state lives in a fixed device array
inside the library.  This test calls it through the C ABI with the caller's
own device buffers, twice in a row (the array keeps the previous call's
contents, which the second call must not see), and checks both results
against the regular entry point ouc_forward at the gather tolerance of the
parity tests.  It sits in its own file so that it is collected last.
"""
import ctypes as C

import numpy as np
import pytest

import ouc_b200 as o
from ouc_b200 import _lib
from helpers import golden_shot, load_golden, make_context, rel_l2

pytestmark = pytest.mark.gpu

TOL_GATHER = 1e-5   # the parity tests' gather tolerance


def _noalloc(cfg, shot, d_vp, d_vs, d_w, d_gx, d_gz):
    c = cfg.c()
    s = shot.c()
    return o.lib().ouc_forward_noalloc(C.byref(c), C.byref(s), d_vp.data_ptr(), d_vs.data_ptr(), d_w.data_ptr(),
                                       d_gx.data_ptr(), d_gz.data_ptr())


def _compare_calls(name, calls, gather_layout):
    """`calls` no-allocation runs of golden case `name` against ouc_forward."""
    import dataclasses

    import torch
    g = load_golden(name)
    shot = golden_shot(g)
    with make_context(g, gather_layout=gather_layout) as ctx:
        gx_ref, gz_ref, _ = ctx.forward(shot, g["src"])
        cfg = dataclasses.replace(ctx.cfg, model_layout=o.MODEL_PADDED)
    dev = torch.device("cuda", 0)
    d_vp = torch.from_numpy(g["vp"]).to(dev)           # padded X x Z, as the reference keeps it
    d_vs = torch.from_numpy(g["vs"]).to(dev)
    d_w = torch.from_numpy(g["src"]).to(dev)
    for call in range(calls):
        d_gx = torch.full(gx_ref.shape, float("nan"), dtype=torch.float32, device=dev)
        d_gz = torch.full(gz_ref.shape, float("nan"), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        rc = _noalloc(cfg, shot, d_vp, d_vs, d_w, d_gx, d_gz)
        assert rc == 0, _lib.OucError(rc)
        torch.cuda.synchronize()
        gx, gz = d_gx.cpu().numpy(), d_gz.cpu().numpy()
        e = (rel_l2(gx, gx_ref), rel_l2(gz, gz_ref))
        print(name, "call", call, "relative L2 vs ouc_forward", e)
        assert np.isfinite(gx).all() and np.isfinite(gz).all()
        assert max(e) <= TOL_GATHER, e


def test_noalloc_forward_matches_ouc_forward_on_two_calls():
    _compare_calls("g72x56n5", 2, o.GATHER_XT)
    # then a smaller grid of another stencil order in the other gather
    # layout: nothing left in the array by the larger calls may show
    _compare_calls("g48x40n2", 1, o.GATHER_TX)


def test_noalloc_refuses_unsupported_arguments_before_any_work():
    import torch
    dev = torch.device("cuda", 0)
    small = torch.zeros(16, dtype=torch.float32, device=dev)
    base = o.Config(nx=40, nz=40, npml=10, dx=10.0, dz=10.0, dt=1e-3, nt=10, half_order=5,
                    model_layout=o.MODEL_PADDED)
    import dataclasses
    bad = [dataclasses.replace(base, model_layout=o.MODEL_INTERIOR),   # it reads padded models only
           dataclasses.replace(base, density=1),                      # density-normalised only
           dataclasses.replace(base, gather_layout=7),
           dataclasses.replace(base, half_order=4)]
    for cfg in bad:
        assert _noalloc(cfg, o.Shot(10, 2, 2), small, small, small, small, small) == _lib.OUC_EINVAL, cfg
    # extents whose padded sizes would overflow 32-bit arithmetic
    huge = dataclasses.replace(base, nx=2 ** 31 - 8, npml=10)
    assert _noalloc(huge, o.Shot(10, 2, 2), small, small, small, small, small) == _lib.OUC_ESCRATCH


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    dev = torch.device("cuda", 0)
    small = torch.zeros(16, dtype=torch.float32, device=dev)
    cfg = o.Config(nx=4000, nz=1500, npml=30, dx=4.0, dz=4.0, dt=4e-4, nt=100, half_order=5,
                   model_layout=o.MODEL_PADDED)
    rc = _noalloc(cfg, o.Shot(10, 2, 2), small, small, small, small, small)
    assert rc == _lib.OUC_ESCRATCH
    assert b"scratch" in o.lib().ouc_strerror(rc)
