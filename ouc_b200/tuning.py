"""Autotuned launch batch and step-kernel geometry, persisted across runs.

``tune(ctx)`` returns the number of shots per launch for this context's grid
and applies it together with the step-kernel geometry (32 x 64 tiles, or the
x-marching kernel with its segment length): from the JSON cache when an
entry for (padded grid, stencil half-order, max batch, GPU name, library
version) exists, otherwise measured by ``ouc_tune`` (timed forward steps at
1, 2, 4, ... up to cfg.max_batch shots per launch, each with the tile kernel
and with segments of 64 .. 512 rows) and stored.  The cache file is
``$OUC_TUNE_CACHE`` or ``~/.cache/ouc_b200/tune.json``.
"""
from __future__ import annotations

import ctypes as C
import json
import os

from ._lib import check, lib


def cache_path():
    return os.environ.get("OUC_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "ouc_b200", "tune.json")


def _key(ctx, device_name):
    c = ctx.cfg
    return f"X{ctx.X}_Z{ctx.Z}_N{c.half_order}_max{c.max_batch}_{device_name}_v{lib().ouc_version()}"


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def tune(ctx, steps=20, path=None, device_name=None, force=False):
    """Shots per launch for `ctx` (applied to it, with the tuned step-kernel
    geometry); returns (batch, ns per cell-update or None when taken from the
    cache, from_cache).  ``ctx.step_kernel()`` reads the geometry chosen."""
    path = path or cache_path()
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(ctx.cfg.device).replace(" ", "_")
    key = _key(ctx, device_name)
    cache = _load(path)
    ent = cache.get(key)
    if not force and ent and 1 <= int(ent.get("batch", 0)) <= max(1, ctx.cfg.max_batch) and "seg_rows" in ent:
        check(lib().ouc_set_run_batch(ctx.handle, int(ent["batch"])), ctx.handle)
        check(lib().ouc_set_step_kernel(ctx.handle, int(ent["seg_rows"])), ctx.handle)
        return int(ent["batch"]), None, True
    best = C.c_int()
    seg = C.c_int()
    ns = C.c_float()
    check(lib().ouc_tune(ctx.handle, int(steps), C.byref(best), C.byref(seg), C.byref(ns)), ctx.handle)
    cache[key] = {"batch": best.value, "seg_rows": seg.value, "ns_per_cell_update": ns.value, "steps": steps}
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    return best.value, ns.value, False
