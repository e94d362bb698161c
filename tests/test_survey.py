"""Shot sharding and the FP64 stack exchange (ouc_b200.survey) on the host.

The multi-GPU path splits a survey's shots across ranks and sums the ranks'
FP64 stacks once at the end.  These tests run that logic as gloo ranks on
the CPU (world size 2): the partition covers every shot exactly once, the
reduced stack equals the serial sum over all shots, and a rank that dies
before the exchange makes the surviving rank fail within the process
group's timeout instead of waiting forever.  Per-shot images come from the
oracle on a small grid, so the sums are of real migrated images.
"""
import os
import socket

import numpy as np
import pytest

from ouc_b200 import survey

SHOTS = [4, 10, 17, 23, 30]      # interior x of the sources on the small grid


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shot_stack(oracle, sx):
    """FP64 contributions of one shot: Laplacian PP, PS, illumination."""
    from oracle.oracle import Shot, layered_model
    X, Z, L, N, nt = 48, 40, 8, 2, 160
    vp, vs = layered_model(X, Z, L)
    ax, az = oracle.profile(vp, L)
    sh = Shot(X=X, Z=Z, L=L, N=N, nt=nt, sx=sx + L, sz=L + 2, rz=L + 2, dx=10.0, dz=10.0, dt=1e-3)
    src = np.zeros(nt, np.float32)
    src[:40] = np.sin(np.linspace(0, 2 * np.pi, 40)).astype(np.float32)
    out = oracle.rtm(sh, vp, vs, ax, az, src)
    il = out["acc"][2][L:X - L, L:Z - L]
    return [out["lap_pp"].astype(np.float64), out["lap_ps"].astype(np.float64), il.astype(np.float64)]


def _rank_main(rank, world, port, outdir, die_rank):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
    oracle = Oracle()
    oracle.threads(1)
    mine = survey.partition(len(SHOTS), world, rank)
    acc = None
    for k in mine:
        c = _shot_stack(oracle, SHOTS[k])
        acc = c if acc is None else [a + b for a, b in zip(acc, c)]
    if rank == die_rank:
        os._exit(3)                      # leaves between steps, nothing in flight
    t = [torch.from_numpy(a) for a in acc]
    try:
        survey.reduce_stack(*t)
        np.save(os.path.join(outdir, f"stack{rank}.npy"), np.stack([x.numpy() for x in t]))
    except Exception as e:               # noqa: BLE001 -- the failure path under test
        with open(os.path.join(outdir, f"error{rank}.txt"), "w") as f:
            f.write(repr(e))
    dist.destroy_process_group()


def _spawn(world, tmp_path, die_rank=-1):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), die_rank)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    codes = [p.exitcode for p in ps]
    for p in ps:
        if p.is_alive():
            p.kill()
    return codes


def test_partition_round_robin_covers_every_shot_once():
    for n in (0, 1, 5, 40, 41):
        for world in (1, 2, 3, 8):
            parts = [survey.partition(n, world, r) for r in range(world)]
            allk = sorted(k for p in parts for k in p)
            assert allk == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_partition_by_cost_balances_and_is_deterministic():
    rng = np.random.default_rng(7)
    cost = rng.uniform(400, 1600, size=256)      # sub-grid apertures of a survey
    for world in (2, 3, 8):
        parts = [survey.partition(len(cost), world, r, cost) for r in range(world)]
        assert sorted(k for p in parts for k in p) == list(range(len(cost)))
        loads = [cost[p].sum() for p in parts]
        assert max(loads) - min(loads) <= cost.max()
        assert parts == [survey.partition(len(cost), world, r, cost) for r in range(world)]


def test_partition_rejects_bad_requests():
    with pytest.raises(ValueError):
        survey.partition(4, 2, 2)
    with pytest.raises(ValueError):
        survey.partition(3, 2, 0, cost=[1.0, -1.0, 2.0])
    with pytest.raises(ValueError):
        survey.partition(3, 2, 0, cost=[1.0, 2.0])


def test_stack_exchange_two_gloo_ranks_equals_serial_sum(tmp_path, oracle):
    codes = _spawn(2, tmp_path)
    assert codes == [0, 0], codes
    serial = None
    for sx in SHOTS:
        c = _shot_stack(oracle, sx)
        serial = c if serial is None else [a + b for a, b in zip(serial, c)]
    serial = np.stack(serial)
    for r in range(2):
        got = np.load(tmp_path / f"stack{r}.npy")
        assert got.dtype == np.float64
        assert np.abs(serial).max() > 0
        np.testing.assert_allclose(got, serial, rtol=1e-12, atol=1e-12 * np.abs(serial).max())


def test_rank_lost_before_the_exchange_fails_the_survivor(tmp_path):
    codes = _spawn(2, tmp_path, die_rank=1)
    assert codes[1] == 3
    assert codes[0] == 0, codes                  # ended by itself, with an error recorded
    assert (tmp_path / "error0.txt").exists()
    assert not (tmp_path / "stack0.npy").exists()
