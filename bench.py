"""Benchmark: plain elastic P/S RTM shots on B200 (one JSON line on rank 0).

Workload (the headline metric's configuration): 1000 x 500 interior,
dx = 5 m, 30-cell CPML (1060 x 560 padded), 10th-order (N = 5) staggered
stencil, dt = 0.5 ms, nt = 4000, 25 Hz Ricker; 8 seeded flat layers,
migration model Gaussian-smoothed (sigma = 10 cells); 40 shot positions on
z = 2 with full-spread receivers.  Observed records are modelled once with
the true model before timing (acquisition, not migration).

One step = one RTM shot: forward with boundary-strip save, receiver
back-propagation with record injection, source-wavefield reconstruction,
PP/PS imaging, image normalisation + Laplacian and the FP64 stack.

  value : Gcell-updates/s with records resident in HBM (device API)
  e2e   : the same through ouc_rtm_shot with pinned host buffers (records
          in, images out, copies inside the timed region)
  N > 1 : one process per GPU, shots sharded round-robin, FP64 stacks
          all-reduced once at the end (weak scaling)

--impl reference times the CPU transcription of the reference kernels
(OpenMP, float) on the same grid for a bounded number of time steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s & RTM shots/hr on 1 B200, learned vs plain at <=1% L2 vs FP64"
UNIT = "Gcell-updates/s"


def algorithmic_bytes_forward(cfg, n_rcv, ring_cells, strip_bytes_per_value=4):
    """Algorithmic HBM bytes of one forward step (each byte moved once):
    56 B per cell (read P/S at levels n and n-1, Vp^2 and Vs^2, write level
    n+1), 48 B per damped cell per axis (six CPML memories read + written),
    8 B per receiver, and the boundary ring of 8 fields written."""
    X, Z, L = cfg.X, cfg.Z, cfg.npml
    C = X * Z
    c_xpml = (2 * L - 1) * Z
    c_zpml = (2 * L - 1) * X
    return 56 * C + 48 * (c_xpml + c_zpml) + 8 * n_rcv + 8 * ring_cells * strip_bytes_per_value


def ring_cells(cfg):
    N = cfg.half_order
    return 4 * N * (cfg.nx + cfg.nz)


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while alive."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per launch of the step kernels from the committed ncu
    capture (profiles/k_step_traffic_c2_b16.json: a list of entries with
    kernel, workload, batch, dram_bytes_per_launch), or []."""
    p = os.path.join(ROOT, "profiles", "k_step_traffic_c2_b16.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return d if isinstance(d, list) else [d]
    except Exception:
        return []


def cpu_sample(steps_hint=None, threads=None, budget_s=12.0):
    """FP32 OpenMP transcription of the reference kernels (oracle) on the
    benchmark grid: one RTM shot truncated to a bounded number of time steps.
    Returns (Gcell-updates/s, cores, sample description)."""
    from oracle.oracle import Oracle, Shot
    from ouc_b200 import models
    orc = Oracle()
    cores = orc.threads(threads or os.cpu_count())
    w = models.c2()
    cfg = w.cfg
    X, Z, L = cfg.X, cfg.Z, cfg.npml
    vp = orc.pad(np.pad(w.vp_mig, L), L)
    vs = orc.pad(np.pad(w.vs_mig, L), L)
    ax, az = orc.profile(vp, L)
    nts = steps_hint or 8
    while True:
        src, t0 = orc.ricker(w.fm, cfg.dt, nts)   # the oracle's restatement: this arm never maps libouc.so
        sh = Shot(X=X, Z=Z, L=L, N=cfg.half_order, nt=nts, sx=L + w.shots[0].sx, sz=L + 2, rz=L + 2, dx=cfg.dx,
                  dz=cfg.dz, dt=cfg.dt, t0=t0)
        t1 = time.perf_counter()
        orc.rtm(sh, vp, vs, ax, az, src)
        el = time.perf_counter() - t1
        if steps_hint or el > budget_s / 4 or nts >= 4000:
            break
        nts = min(4000, int(nts * max(2.0, budget_s / max(el, 1e-3) * 0.9)))
    cells = nts * (2 * X * Z + cfg.nx * cfg.nz)
    return cells / el / 1e9, cores, f"one RTM shot of the benchmark grid truncated to nt={nts} steps ({el:.1f} s)"


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    vals = []
    desc = None
    cores = None
    for _ in range(args.warmup):
        cpu_sample(steps_hint=8)
    for _ in range(args.steps):
        v, cores, desc = cpu_sample(steps_hint=args.ref_steps)
        vals.append(v)
    value = statistics.median(vals)
    from ouc_b200 import models
    w = models.c2()
    ref_cuda = reference_cuda_shot(w)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "grid": [w.cfg.X, w.cfg.Z], "nt": w.cfg.nt, "half_order": w.cfg.half_order},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_cuda": ref_cuda}
    print(json.dumps(line), flush=True)
    return 0


def reference_cuda_shot(w):
    """The reference's own kernels compiled for sm_100a (oracle/_ref, built
    from its sources by oracle/Makefile with its main()'s launch sequence):
    one RTM shot of the benchmark grid on this GPU, CUDA events around its
    forward and backward loops.  None when the build or a GPU is absent."""
    from oracle.oracle import REF_DIR, Oracle, RefBuild
    if not os.path.exists(os.path.join(REF_DIR, "libpsref_cuda_c2.so")):
        return None
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except ImportError:
        return None
    cfg = w.cfg
    L = cfg.npml
    orc = Oracle()
    vp = orc.pad(np.pad(w.vp_mig, L), L)
    vs = orc.pad(np.pad(w.vs_mig, L), L)
    ax, az = orc.profile(vp, L)
    src, t0 = orc.ricker(w.fm, cfg.dt, cfg.nt)
    ref = RefBuild("c2", "cuda")
    sx = L + w.shots[0].sx
    f32 = np.float32
    r = ref.rtm(sx, L + 2, L + 2, t0, f32(cfg.dt), f32(cfg.dx), f32(cfg.dz), vp, vs, ax, az, src)
    ms = r["ms"][0] + r["ms"][1]
    cells = cfg.nt * (2 * cfg.X * cfg.Z + cfg.nx * cfg.nz)
    return {"value": cells / (ms / 1e3) / 1e9, "unit": UNIT, "ms_per_shot": ms,
            "shots_per_hour": 3600.0 / (ms / 1e3),
            "what": "the reference's kernels (forward_s/forward_u, rt_*, reshot_*, corr_v...) built for sm_100a, "
                    "one RTM shot of the same grid at a time, CUDA events around its time loops"}


def run_survey(args, rank, world):
    """Batched uneven-shot RTM (the c3 survey): each step migrates one batch of
    shots on their own sub-grids through ouc_survey_rtm (host records in,
    per-shot images out, copies inside the timed region).  One GPU."""
    import torch
    import ouc_b200 as o
    from ouc_b200 import models, tuning
    if world > 1:
        raise SystemExit("the survey workload runs on one GPU")
    torch.cuda.set_device(0)
    w = models.c3(nt=args.nt) if args.nt else models.c3()
    cfg = w.cfg
    B = max(1, args.batch)
    cfg.max_batch = B
    cfg.strip_precision = {"fp32": o.PREC_FP32, "fp16": o.PREC_FP16, "bf16": o.PREC_BF16}[args.strips]
    wavelet, t0 = o.ricker(w.fm, cfg.dt, cfg.nt)
    shots = [o.Shot(s.sx, s.sz, s.rz, t0=t0) for s in w.shots]
    # one batch of shots spread over the survey (every len/B-th shot)
    pick = list(range(0, len(shots), max(1, len(shots) // B)))[:B]
    sh = [shots[k] for k in pick]
    aps = [w.apertures[k] for k in pick]
    true_ctx = o.Context(cfg, w.vp, w.vs, w.rho)
    recs = true_ctx.survey_forward(sh, aps, wavelet)          # acquisition, not timed
    true_ctx.close()
    pin = [(torch.from_numpy(r[0]).pin_memory().numpy(), torch.from_numpy(r[1]).pin_memory().numpy()) for r in recs]
    mig = o.Context(cfg, w.vp_mig, w.vs_mig, w.rho)
    tuned, ns_cell, cached = tuning.tune(mig, steps=10)
    for _ in range(args.warmup):
        mig.survey_rtm(sh, aps, wavelet, pin)
    clocks = Clocks(0)
    times, fwd, bwd = [], [], []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        mig.survey_rtm(sh, aps, wavelet, pin)
        times.append(time.perf_counter() - t1)
        t = mig.timing()
        fwd.append(t["forward_ms"])
        bwd.append(t["backward_ms"])
    clk = clocks.stop()
    launches = mig.timing()["kernel_launches"]
    mig.close()
    s_step = statistics.median(times)
    L = cfg.npml
    cells = sum(cfg.nt * (2 * (x1 - x0 + 2 * L) * cfg.Z + (x1 - x0) * cfg.nz) for x0, x1 in aps)
    value = cells / s_step / 1e9
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * s_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded folded model, modelled records)",
                "config": {"workload": w.name, "model": [cfg.nx, cfg.nz], "nt": cfg.nt, "dx_m": cfg.dx,
                           "dt_s": cfg.dt, "shots_per_step": len(sh), "apertures": aps, "strips": args.strips,
                           "step": "one batch of uneven sub-grid RTM shots, host records in, images out",
                           "launch_batch": tuned, "tuned_ns_per_cell_update": ns_cell, "tuning_cached": cached,
                           "graphs": True, "l2": "per-step working set of the batch exceeds L2"},
                "shots_per_hour": 3600.0 * len(sh) / s_step,
                "phase_ms": {"forward": statistics.median(fwd), "backward": statistics.median(bwd)},
                "e2e": {"value": value, "unit": UNIT,
                        "h2d_bytes_per_step": sum(2 * r[0].size * 4 for r in recs) + cfg.nt * 4,
                        "d2h_bytes_per_step": sum(2 * (x1 - x0) * cfg.nz * 4 for x0, x1 in aps)},
                "gpu_launches": int(launches), "clocks": clk}
        print(json.dumps(line), flush=True)
    return 0


def relaunch(n):
    """--gpus N > 1 without a launcher: run this script as N ranks (one
    process per GPU) under torch.distributed.run on 127.0.0.1; rank 0 prints
    the line.  An outer timeout bounds ranks that wait for one another."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = ["timeout", "-k", "60", "1800", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ouc", choices=["ouc", "reference"])
    ap.add_argument("--nt", type=int, default=None, help="time steps per shot (default: the workload's)")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4"],
                    help="c2: the headline 1000x500 RTM workload; c4: the 4000x1500 grid (HBM-bound profiling)")
    ap.add_argument("--ref-steps", type=int, default=None, help="CPU sample length (time steps)")
    ap.add_argument("--batch", type=int, default=16, help="shots advanced together per step (c3: shots per step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--strips", default="fp32", choices=["fp32", "fp16", "bf16"],
                    help="boundary-strip storage (fp16: scaled per slot and field)")
    ap.add_argument("--compensated", action="store_true", help="compensated FP32 imaging sums")
    ap.add_argument("--seg-rows", type=int, default=None,
                    help="step kernel: x-marching segment rows (multiple of 16), 0 for the 32 x 64 tile kernel, "
                         "-1 for the tile kernel with a dynamic tile queue (default: the library's choice)")
    ap.add_argument("--snapshot-every", type=int, default=0,
                    help="0: reconstruct the source wavefield from boundary strips (the reference's method); "
                         "K: store source snapshots every K imaging levels instead (--strips sets their storage)")
    args = ap.parse_args()

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch(args.gpus)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world != args.gpus and "WORLD_SIZE" in os.environ and args.gpus > 1:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "c3":
        return run_survey(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    import ouc_b200 as o
    from ouc_b200 import models
    make = models.c2 if args.workload == "c2" else models.c4
    w = make(nt=args.nt) if args.nt else make()
    cfg = w.cfg
    cfg.device = local
    wavelet, t0 = o.ricker(w.fm, cfg.dt, cfg.nt)
    X, nt = cfg.X, cfg.nt

    # observed records with the true model (not timed): one record set per
    # shot of a batch, shot positions spread over the survey
    B = max(1, args.batch)
    my_shots = [w.shots[(rank + k * world * max(1, len(w.shots) // (B * world))) % len(w.shots)] for k in range(B)]
    my_shots = [o.Shot(s.sx, s.sz, s.rz, t0=t0) for s in my_shots]
    true_ctx = o.Context(cfg, w.vp, w.vs, w.rho)
    records = [true_ctx.forward(s, wavelet)[:2] for s in my_shots]
    true_ctx.close()
    cfg.max_batch = B
    cfg.strip_precision = {"fp32": o.PREC_FP32, "fp16": o.PREC_FP16, "bf16": o.PREC_BF16}[args.strips]
    cfg.compensated_image = int(args.compensated)
    cfg.snapshot_every = args.snapshot_every
    mig = o.Context(cfg, w.vp_mig, w.vs_mig, w.rho)
    if args.seg_rows is not None:
        mig.set_step_kernel(args.seg_rows)
    stream = torch.cuda.ExternalStream(mig.stream, device=torch.device("cuda", local))

    # device-resident inputs
    d_w = torch.from_numpy(wavelet).cuda()
    d_rec = [(torch.from_numpy(r[0]).cuda(), torch.from_numpy(r[1]).cuda()) for r in records]
    d_img = torch.empty((B, 2, cfg.nx, cfg.nz), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # 256 MiB > L2
    torch.cuda.synchronize()

    def step_dev():
        mig.rtm_batch_dev(my_shots, d_w.data_ptr(), [r[0].data_ptr() for r in d_rec], [r[1].data_ptr() for r in d_rec],
                          [d_img[b, 0].data_ptr() for b in range(B)], [d_img[b, 1].data_ptr() for b in range(B)])

    for k in range(args.warmup):
        step_dev()
    launches_per_step = mig.timing()["kernel_launches"]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    fwd_ms = []
    bwd_ms = []
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))          # between timed steps: evict L2
            ev[k][0].record(stream)
        step_dev()                         # synchronous on the context stream
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
        t = mig.timing()
        fwd_ms.append(t["forward_ms"])
        bwd_ms.append(t["backward_ms"])
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    # the cross-shot exchange after the timed shots: sum of the ranks' FP64
    # stacks (PP, PS, illumination); it also leaves the stack empty for e2e
    from ouc_b200 import survey
    stk = [torch.from_numpy(a).cuda() for a in mig.stack(reset=True)]
    if world > 1:
        tt = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        survey.reduce_stack(*stk)
        dist.barrier()
    clk = clocks.stop()
    # cell-updates actually performed: forward + receiver on the padded grid,
    # plus the reconstruction on the interior when the strips form runs it
    cells = (w.cell_updates_per_shot() if not args.snapshot_every else 2 * cfg.nt * cfg.X * cfg.Z) * B
    value = cells * args.steps * world / (ms / 1e3) / 1e9
    shots_per_hour = 3600.0 * B * args.steps * world / (ms / 1e3)

    # e2e through the survey call a user makes (ouc_b200.survey.migrate):
    # this rank's shots through the host API with pinned records in and
    # images out, its FP64 stacks read back and summed over the ranks
    pin = [(torch.from_numpy(r[0]).pin_memory().numpy(), torch.from_numpy(r[1]).pin_memory().numpy()) for r in records]
    all_shots = [None] * (B * world)
    all_recs = [None] * (B * world)
    for k in range(B):                       # round-robin: rank r migrates shots r, r + world, ...
        all_shots[rank + k * world] = my_shots[k]
        all_recs[rank + k * world] = pin[k]
    for k in range(len(all_shots)):          # other ranks' slots: placeholders this rank never runs
        if all_shots[k] is None:
            all_shots[k] = my_shots[0]
    e2e_steps = max(2, args.steps // 2)
    survey.migrate(mig, all_shots, wavelet, recs=all_recs, rank=rank, world=world)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t1 = time.perf_counter()
    for k in range(e2e_steps):
        survey.migrate(mig, all_shots, wavelet, recs=all_recs, rank=rank, world=world)
    e2e_s = time.perf_counter() - t1
    if world > 1:
        tt = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = cells * e2e_steps * world / e2e_s / 1e9

    # rooflines of the three step kernels.  Algorithmic bytes per launch
    # (each byte moved once, the batch's B shots): forward and receiver 56 B
    # per padded cell + 48 B per damped cell per axis (+ the strip write of
    # the ring, resp. the record row read); reconstruction + imaging 56 B +
    # 24 B (three accumulators read and written) per interior cell + the
    # strip read.  The forward launch is timed over the timed region (its
    # phase holds nothing else); all three are also timed one launch kind at
    # a time on the state the last batch left (ouc_time_step_kernels).
    peak, peak_kind = measured_peak()
    sb = 4 if args.strips == "fp32" else 2
    C, Ci, L = X * cfg.Z, cfg.nx * cfg.nz, cfg.npml
    damp = 48 * ((2 * L - 1) * cfg.Z + (2 * L - 1) * X)
    alg = {"forward": (56 * C + damp + 8 * ring_cells(cfg) * sb) * B,
           "receiver": (56 * C + damp + 8 * X) * B,
           "reconstruction": (80 * Ci + 8 * ring_cells(cfg) * sb) * B}
    seg = mig.step_kernel()
    kname = (lambda m: f"k_march<{cfg.half_order}, {m}> ({seg}-row segments, 16-row blocks)" if seg > 0 else
             f"k_step_q<{cfg.half_order}, {m}> (32 x 64 tiles, persistent launch with a dynamic tile queue)" if seg < 0
             else f"k_step<{cfg.half_order}, {m}> (32 x 64 tiles)")
    kern = {}
    if not args.snapshot_every:
        iso = mig.time_step_kernels(B, reps=20)
        for k, name in enumerate(("forward", "receiver", "reconstruction")):
            a_gbs = alg[name] / (iso[k] / 1e3) / 1e9
            kern[name] = {"kernel": kname(name), "launch_ms": iso[k], "algorithmic_bytes_per_launch": alg[name],
                          "achieved": a_gbs, "frac": a_gbs / peak,
                          "traffic": next((t.get("dram_bytes_per_launch") for t in committed_traffic()
                                           if t.get("workload") == w.name and t.get("batch") == B and
                                           t.get("kernel") == kname(name)), None)}
    per_launch_ms = statistics.median(fwd_ms) / nt        # forward launch, over the timed region
    dom = max(kern, key=lambda k: kern[k]["launch_ms"]) if kern else "forward"
    if dom == "forward":
        r_ms, r_bytes, r_src = per_launch_ms, alg["forward"], "forward phase of the timed region / nt"
    else:
        r_ms, r_bytes, r_src = kern[dom]["launch_ms"], alg[dom], "isolated launches (ouc_time_step_kernels)"
    achieved = r_bytes / (r_ms / 1e3) / 1e9
    traffic = next((t.get("dram_bytes_per_launch") for t in committed_traffic()
                    if t.get("workload") == w.name and t.get("batch") == B and t.get("kernel") == kname(dom)), None)

    # saved source wavefield per shot: 8 ring fields per step (strip form) or
    # the two P components of every K-th imaging level (snapshot form)
    elem = 4 if args.strips == "fp32" else 2
    if args.snapshot_every:
        saved, saved_what = -(-nt // args.snapshot_every) * 2 * cfg.nx * cfg.nz * elem, "source snapshots"
    else:
        saved, saved_what = (nt - 1) * 8 * ring_cells(cfg) * elem, "boundary strips"

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline:
            v, cores, desc = cpu_sample()
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered model, modelled records)",
            "config": {"workload": w.name, "grid": [cfg.X, cfg.Z], "interior": [cfg.nx, cfg.nz], "nt": nt,
                       "half_order": cfg.half_order, "dx_m": cfg.dx, "dt_s": cfg.dt, "step": f"one batch of {B} RTM shots advanced together", "batch": B,
                       "strips": args.strips, "compensated_image": bool(args.compensated),
                       "source_wavefield": (f"snapshots every {args.snapshot_every} imaging levels" if args.snapshot_every
                                            else "reconstructed from boundary strips"),
                       "l2": f"256 MiB buffer written between timed shots; {saved / 1e9:.1f} GB of {saved_what} per shot",
                       "parallelism": f"shots sharded over {world} GPU(s)"},
            "shots_per_hour": shots_per_hour,
            "phase_ms": {"forward": statistics.median(fwd_ms), "backward": statistics.median(bwd_ms)},
            "e2e": {"value": e2e, "unit": UNIT, "call": "ouc_b200.survey.migrate (ouc_rtm_batch + ouc_stack + FP64 "
                                                           "stack all-reduce)",
                    "h2d_bytes_per_step": B * 2 * nt * X * 4 + nt * 4,
                    "d2h_bytes_per_step": B * 2 * cfg.nx * cfg.nz * 4 + 3 * cfg.nx * cfg.nz * 8,
                    "shots_per_hour": 3600.0 * B * e2e_steps * world / e2e_s},
            "roofline": {"kernel": f"{kname(dom)}, {B} shots per launch (the slowest of the three step kernels)",
                         "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": r_bytes,
                         "launch_ms": r_ms, "launch_ms_from": r_src, "traffic": traffic,
                         "forward_launch_ms_timed_region": per_launch_ms,
                         "backward_step_ms_timed_region": statistics.median(bwd_ms) / nt},
            "step_kernels": kern,
            "cpu_baseline": cpu,
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    mig.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
