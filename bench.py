#!/usr/bin/env python3
"""Benchmark of the DG elastic-wave time loop on B200.

One bench step = one time step of the whole workload: sponge, source, velocity half-step,
stress half-step and receiver record for every element, shot and mesh.  The default workload is
the multi-shot batch: a layered elastic mesh of 200,000 triangles advanced for 64 shots at once
in FP32 (shots innermost).  Beside it the line reports the plain FP64 path on one shot of the same
mesh (timed exactly as the batch, and again with L2 flushed before every step), the FP32-vs-FP64
trace error, the roofline of the dominant kernel, an end-to-end figure through the public API
with host buffers, and the reference's own CPU code timed on this host.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]
                    [--precision fp32|fp32_kahan|fp64]

Under torchrun (N > 1) the ranks share one job: the multi-shot job has 64 shots per GPU, cut into
contiguous shot ranges (sharding.shard_shots); the uneven batch's meshes go to ranks by cost
(sharding.shard_meshes).  Nothing is exchanged while the ranks step; the end-to-end figure ends
with every rank's traces gathered on rank 0 (sharding.gather_traces).  Times are the maximum over
ranks.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-updates/s batched FP32 vs plain FP64 at ≤1e-4 trace L2; HBM % of peak"
UNIT = "DOF-updates/s"
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def pkg():
    return importlib.import_module("discontinuous-galerkin-method_b200")


def _multishot(steps, rank, world):
    """This rank's share of the multi-shot job: the layered 200,000-triangle mesh with 64 shots per
    rank (64 * world sources evenly spaced along the surface), cut into contiguous shot ranges by
    sharding.shard_shots, so every rank advances 64 shots on the wavefront step."""
    import dataclasses
    job = pkg().workloads.layered_multishot(steps=steps, shots=64 * world)
    r = pkg().sharding.shard_shots(job.shots, world)[rank]
    return [dataclasses.replace(job, src=job.src[r.start:r.stop].copy())]


def _uneven(steps, rank, world, n_meshes=48):
    """This rank's share of the uneven batch: the meshes sharding.shard_meshes gives it by cost
    (elements x shots x steps)."""
    ws, _ = pkg().workloads.uneven_batch(n_meshes=n_meshes, seed=5)
    for w in ws:
        w.steps = steps
    sh = pkg().sharding
    mine = sh.shard_meshes([sh.mesh_cost(w.K, w.shots, steps) for w in ws], world)[rank]
    return [ws[i] for i in mine]


def _replica(make):
    """A one-mesh, one-shot workload that does not split: every rank runs the same one."""
    return lambda steps, rank, world: [make(steps)]


WORKLOADS = {
    # name: (constructor(steps, rank, world) -> this rank's workloads, description, how N GPUs
    # share the job: "weak" = a fixed share per GPU, "strong" = a fixed job split, "replicas")
    "multishot": (_multishot, "multi-shot layered elastic batch: 200,000 triangles x 64 shots per GPU", "weak"),
    # one shot of that mesh: the plain FP64 path's workload, for profiling it on its own
    "layered1": (_replica(lambda steps: one_shot(pkg().workloads.layered_multishot(steps=steps))),
                 "layered elastic mesh of the multi-shot batch, 200,000 triangles, 1 shot", "replicas"),
    "slope": (_replica(lambda steps: pkg().workloads.coupled_slope(steps=steps)),
              "coupled acoustic-elastic slope: ~400,000 triangles, 1 shot", "replicas"),
    "random": (_replica(lambda steps: pkg().workloads.random_medium(steps=steps)),
               "heterogeneous random medium: 2,000,000 triangles, 1 shot", "replicas"),
    "square": (_replica(lambda steps: pkg().workloads.homogeneous_square(steps=steps)),
               "homogeneous square: 20,000 triangles, 1 shot", "replicas"),
    "uneven": (_uneven, "uneven batch: 48 meshes, 5,000-500,000 triangles (log-uniform), 1-8 shots each, "
                        "split over the GPUs by cost", "strong"),
    # the first 12 meshes of that batch: a smaller case of the same kernels, for profiling
    "uneven12": (lambda steps, rank, world: _uneven(steps, rank, world, 12),
                 "uneven batch: 12 meshes, 5,000-500,000 triangles (log-uniform), 1-8 shots each", "strong"),
}


def job_traces(engine, ws, t0, n):
    """This rank's traces of steps [t0, t0 + n): (shots of all its meshes, 2, n, n_rec) for one
    mesh, or a flat array of every mesh's block for several (meshes differ in receivers)."""
    import numpy as np
    blocks = []
    for k, _ in enumerate(ws):
        tx, tz = engine.fetch_traces(t0, n, mesh=k)
        blocks.append(np.stack([tx, tz], 1))
    return blocks[0] if len(blocks) == 1 else np.concatenate([b.ravel() for b in blocks])


def gather_job(dist, local, device):
    """Every rank's traces on rank 0 (sharding.gather_traces; the job's one collective), None on
    the other ranks; a one-rank job returns its own."""
    if dist is None:
        return [local]
    return pkg().sharding.gather_traces(dist, local, root=0, device=device)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the GPU works."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args, join: bool = True):
    """Rank, world size and local rank from the launcher's environment; with `join` and more than
    one rank, also the process group.  Under NCCL each rank binds its own GPU (LOCAL_RANK) before
    the group exists, so that NCCL's communicator and the barrier's synchronize both use it."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1 and join:
        import datetime

        import torch
        import torch.distributed as dist
        backend = os.environ.get("DG_BENCH_BACKEND", "nccl")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120), **kw)
    return rank, world, local, dist


def max_over_ranks(x: float, dist, device) -> float:
    """Maximum of a per-rank time over all ranks (device: a CUDA ordinal, or "cpu" for gloo)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(dof_per_step_per_rank: float, steps: int, local_ms: float, world: int, dist, device):
    """Whole-job DOF-updates/s when every rank does the same work: every rank's work over the
    slowest rank's device time."""
    t_max = max_over_ranks(local_ms, dist, device)
    return world * dof_per_step_per_rank * steps / (t_max * 1e-3), t_max


def sum_over_ranks(x: float, dist, device) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_value(dof_per_step_local: float, steps: int, local_ms: float, dist, device):
    """Whole-job DOF-updates/s for ranks with different shares: all ranks' work over the slowest
    rank's device time."""
    t_max = max_over_ranks(local_ms, dist, device)
    return sum_over_ranks(dof_per_step_local, dist, device) * steps / (t_max * 1e-3), t_max


def barrier(dist, device):
    if dist is not None:
        import torch
        dist.barrier()
        if device != "cpu":
            torch.cuda.synchronize(device)


def as_list(w):
    return w if isinstance(w, list) else [w]


def one_shot(w):
    return pkg().workloads.Workload(w.name, w.mesh, w.vp, w.vs, w.rho, w.fp, w.sponge, w.src[:1], w.rec, w.steps)


REF_BUILDS = {True: "throughput build -O3 -march=x86-64-v3 (no FP contraction: the parity build's bits)",
              False: "parity build -O2"}


def cpu_reference(w, steps_hint: float = 6.0):
    """Time the reference's own OpenMP code (oracle/_ref, its throughput build where this host
    runs it) on this host: one shot, all cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun  # CPU-baseline leg only

    cores = os.cpu_count() or 1
    w1 = one_shot(w)
    fast = refrun.available(w1, fast=True)
    build = ""
    if fast or refrun.available(w1):
        with tempfile.TemporaryDirectory() as d:
            probe = refrun.run(w1, os.path.join(d, "p"), steps=5, threads=cores, dump_setup=0,
                               work_dir=os.path.join(d, "w"), fast=fast)
            per = probe["timing"]["loop_seconds"] / 5
            # steps from the early-step probe; later steps run up to 3x slower (subnormal values
            # spread ahead of the wave front), so the sample ends near 10-30 s; at most 1,000
            n = int(max(10, min(1000, steps_hint / max(per, 1e-6))))
            r = refrun.run(w1, os.path.join(d, "r"), steps=n, threads=cores, dump_setup=0,
                           work_dir=os.path.join(d, "w"), fast=fast)
            sec = r["timing"]["loop_seconds"]
            th = int(r["timing"]["threads"])
        kind = "reference"
        build = ", " + REF_BUILDS[fast]
    else:
        import oracle
        s = pkg().host.build_setup(w1, full=True, n_steps=4000)
        o = oracle.Oracle.from_setup(s)
        t = time.perf_counter()
        o.run(0, 3, threads=cores, record=True)
        per = (time.perf_counter() - t) / 3
        n = int(max(10, min(1000, s.n_steps - 3, steps_hint / max(per, 1e-6))))
        t = time.perf_counter()
        o.run(0, n, threads=cores, record=True)
        sec = time.perf_counter() - t
        th = cores
        kind = "port"
    dof = 30.0 * w1.K * n
    return {"value": dof / sec, "unit": UNIT, "cores": th, "kind": kind,
            "sample": "1 of %d shots of a %d-triangle mesh, first %d time steps, OpenMP %d threads, loop time only "
                      "(%.1f s)%s" % (w.shots, w1.K, n, th, sec, build)}


def run_reference_arm(args):
    # rank 0 alone times the CPU code; no collective, so no process group is joined
    rank, world, local, dist = dist_setup(args, join=False)
    if rank != 0:
        return 0
    ctor, desc, _ = WORKLOADS[args.workload]
    w = ctor(max(args.steps, args.warmup) + 10, 0, 1)[0]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    cores = os.cpu_count() or 1
    w1 = one_shot(w)
    fast = refrun.available(w1, fast=True)
    build = "the oracle port (C restatement)"
    with tempfile.TemporaryDirectory() as d:
        if fast or refrun.available(w1):
            if args.warmup:
                refrun.run(w1, os.path.join(d, "w"), steps=args.warmup, threads=cores, dump_setup=0,
                           work_dir=os.path.join(d, "in"), fast=fast)
            r = refrun.run(w1, os.path.join(d, "t"), steps=args.steps, threads=cores, dump_setup=0,
                           work_dir=os.path.join(d, "in"), fast=fast)
            sec = r["timing"]["loop_seconds"]
            kind, th = "reference", int(r["timing"]["threads"])
            build = "the reference's code, " + REF_BUILDS[fast]
        else:
            import oracle
            s = pkg().host.build_setup(w1, full=True)
            o = oracle.Oracle.from_setup(s)
            o.run(0, args.warmup, threads=cores)
            t = time.perf_counter()
            o.run(0, args.steps, threads=cores)
            sec = time.perf_counter() - t
            kind, th = "port", cores
    value = 30.0 * w1.K * args.steps / sec
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "shots_timed": 1, "K": w1.K, "threads": th},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": th, "kind": kind,
                             "sample": "1 shot of the first mesh, %d time steps after %d warm-up steps, %s"
                                       % (args.steps, args.warmup, build)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def read_traffic(workload: str, kernel: str, precision: str = "fp32"):
    """DRAM bytes per launch from the committed ncu summary (profiles/), if one exists: the file
    for this arithmetic (traffic_<kernel>_<workload>_<precision>.txt), or for FP32 the one
    without the suffix."""
    names = ["traffic_%s_%s_%s.txt" % (kernel, workload, precision)]
    if precision == "fp32":
        names.append("traffic_%s_%s.txt" % (kernel, workload))
    for name in names:
        try:
            with open(os.path.join(ROOT, "profiles", name)) as f:
                for line in f:
                    if line.startswith("traffic_bytes_per_launch:"):
                        return float(line.split(":", 1)[1])
        except OSError:
            continue
    return None


def kernel_bytes(ws, precision):
    """Algorithmic bytes of one velocity and one stress launch over the batch."""
    w = 8 if precision.startswith("fp64") else 4
    comp = precision == "fp32_kahan"
    bv = sum(x.K * (42 * x.shots * w + (24 * x.shots * 4 if comp else 0) + 5 * w + 16) for x in ws)
    bs = sum(x.K * (48 * x.shots * w + (36 * x.shots * 4 if comp else 0) + 8 * w + 16) for x in ws)
    return bv, bs


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local, dist = dist_setup(args)
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the engine has no CPU fallback)")
    device = local
    torch.cuda.set_device(device)
    P = pkg()
    eng = P.engine
    ctor, desc, share = WORKLOADS[args.workload]
    K_steps, W_steps = args.steps, args.warmup
    # the host gets the traces every 100 steps: the cadence at which the reference's own loop
    # hands its state to the host (Save_Data every 100 steps, DG_leap_Frog_OpenMP.c:433-444)
    e2e_chunk = 100
    e2e_steps = max(e2e_chunk, (K_steps // e2e_chunk) * e2e_chunk)
    acc_steps = 1000   # FP32 against FP64: long enough for arrivals at the receivers of every workload
    table = max(W_steps + 2 * K_steps, W_steps + e2e_steps, acc_steps) + 8
    ws = ctor(table, rank, world)
    setups = [P.host.build_setup(w, full=False, n_steps=table) for w in ws]
    meshes = [eng.mesh_from_setup(s, with_ref_ops=False) for s in setups]
    peak, peak_src = peaks()
    sampler = ClockSampler(device)
    sampler.start()

    # ---- headline: the batch in the requested arithmetic, inputs resident in HBM ------------
    e = eng.Engine(meshes, args.precision, device=device, variant=args.variant)
    st = e.stats()
    bytes_step, dof_step = st["bytes_per_step"], st["dof_per_step"]
    e.step(W_steps)
    # K steps through the call a user makes (CUDA graphs, or one persistent launch), timed with
    # CUDA events on the context's stream around the whole run
    stream = e.stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist, device)
    torch.cuda.synchronize(device)
    ev0.record(stream)
    e.step(K_steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize(device)
    barrier(dist, device)
    total_ms = ev0.elapsed_time(ev1)
    launches = e.stats()["launches"]
    value, t_max = job_value(dof_step, K_steps, total_ms, dist, device)
    dof_job = sum_over_ranks(dof_step, dist, device)
    names = eng.KERNEL_NAMES[st["kernel_family"]]
    if names[1] is None:
        # the whole step in one launch (or the whole run in one persistent launch): the kernel's
        # time per step is the timed region's, on the stream it runs on
        t_one = total_ms / K_steps
        dom = (names[0], bytes_step, t_one)
        kernels = {names[0]: {"ms": t_one, "GBs": bytes_step / (t_one * 1e-3) / 1e9}}
        time_source = ("the timed region: CUDA events on the context's stream around the %d-step call, "
                       "%d launches of %s" % (K_steps, launches, names[0]))
    else:
        # two launches a step: K more steps with events around every launch give each kernel's time
        mv, ms, _ = e.step_profiled(K_steps)
        t_vel, t_str = float(np.mean(mv)), float(np.mean(ms))
        b_vel, b_str = kernel_bytes(ws, args.precision)
        dom = (names[1], b_str, t_str) if t_str >= t_vel else (names[0], b_vel, t_vel)
        kernels = {names[0]: {"ms": t_vel, "GBs": b_vel / (t_vel * 1e-3) / 1e9},
                   names[1]: {"ms": t_str, "GBs": b_str / (t_str * 1e-3) / 1e9}}
        time_source = ("a separate run of %d steps after the timed region, CUDA events around every launch"
                       % K_steps)
    achieved = dom[1] / (dom[2] * 1e-3) / 1e9
    traffic = read_traffic(args.workload, dom[0], args.precision)
    S_tot = sum(x.shots for x in ws)
    K_tot = sum(x.K for x in ws)
    R_tot = sum(x.shots * x.rec.shape[0] for x in ws)
    wbytes = 8 if args.precision == "fp64" else 4
    state_bytes = sum(30 * x.K * x.shots for x in ws) * (wbytes + (4 if args.precision == "fp32_kahan" else 0))

    # ---- end to end through the public API with pinned host buffers ------------------------
    e.reset()
    e.step(W_steps)
    e.fetch_traces(0, W_steps, mesh=eng.ALL_MESHES)   # the warm-up steps' traces: the fetch path warm too
    # every mesh's wavelet chunk in one pinned buffer and one call, every mesh's traces in one call
    wav = torch.empty(len(ws) * e2e_chunk, dtype=torch.float64).pin_memory()
    n_tr = sum(x.shots * x.rec.shape[0] for x in ws) * e2e_chunk
    n_chunks = e2e_steps // e2e_chunk
    # the run's traces, as a user keeps them: each chunk's fetch lands in its own slice of one
    # pinned buffer
    kept = torch.empty((2, n_chunks, n_tr), dtype=torch.float64).pin_memory()
    wav_np = wav.numpy()
    barrier(dist, device)
    t0 = time.perf_counter()
    for c in range(n_chunks):
        t_at = W_steps + c * e2e_chunk
        for k, s in enumerate(setups):
            wav_np[k * e2e_chunk:(k + 1) * e2e_chunk] = s.arrays["wavelet"][t_at:t_at + e2e_chunk]
        # samples no enqueued step reads: the upload does not wait for the chunk in flight
        e.set_wavelet(t_at, wav, mesh=eng.ALL_MESHES)
        e.step_async(e2e_chunk)
        if c > 0:  # the previous chunk's traces, copied while this chunk steps
            t_prev = t_at - e2e_chunk
            e.fetch_traces(t_prev, e2e_chunk, mesh=eng.ALL_MESHES, out_x=kept[0, c - 1], out_z=kept[1, c - 1])
    t_last = W_steps + (n_chunks - 1) * e2e_chunk
    e.fetch_traces(t_last, e2e_chunk, mesh=eng.ALL_MESHES, out_x=kept[0, n_chunks - 1], out_z=kept[1, n_chunks - 1])
    e.synchronize()
    # the job's one collective: every rank's traces to rank 0
    gathered = gather_job(dist, kept.numpy(), device)
    t_e2e = time.perf_counter() - t0
    barrier(dist, device)
    t_e2e = max_over_ranks(t_e2e, dist, device)
    e2e_value = dof_job * e2e_steps / t_e2e
    if rank == 0:
        assert len(gathered) == world and all(np.isfinite(g).all() for g in gathered)
    h2d = 8.0 * len(ws)
    d2h = 2.0 * 8.0 * R_tot

    # ---- accuracy: the batch against FP64 over the first steps -----------------------------
    def traces(engine):
        """All traces, and each mesh's slice of them."""
        out, cuts = [], [0]
        for k, x in enumerate(ws):
            for m in range(x.shots):
                out += [engine.fetch("trace_x", k, m).ravel(), engine.fetch("trace_z", k, m).ravel()]
            cuts.append(sum(a.size for a in out))
        return np.concatenate(out), cuts

    # energy (FP64 sums on the device) of up to 8 (mesh, shot) pairs, every quarter of the run
    pairs = [(k, m) for k, x in enumerate(ws) for m in range(x.shots)]
    pairs = pairs[:: max(1, len(pairs) // 8)][:8]
    quarters = 4

    def run_accuracy(engine):
        energy = []
        for _ in range(quarters):
            engine.step(acc_steps // quarters)
            energy.append([engine.fetch("energy", k, m) for k, m in pairs])
        return np.array(energy)

    e.reset()
    en = run_accuracy(e)
    tr, cuts = traces(e)
    e.close()
    accuracy = None
    if args.precision != "fp64":
        with eng.Engine(meshes, "fp64", device=device) as e64:
            en64 = run_accuracy(e64)
            tr64, _ = traces(e64)
            field_max = max(float(np.abs(e64.fetch(f, k, 0)).max()) for k in range(len(ws)) for f in ("Vx", "Vz"))
        drift = [float(np.abs(en[:, j] - en64[:, j]).max() / en64[:, j].max())
                 for j in range(len(pairs)) if en64[:, j].max() > 0]
        energy_acc = {"energy_rel_vs_fp64": max(drift) if drift else None,
                      "energy_what": "max over t of |E(t) - E_fp64(t)| / max E_fp64, %d (mesh, shot) pairs, "
                                     "every %d steps" % (len(pairs), acc_steps // quarters)}
        trace_max = float(np.abs(tr64).max())
        energy_acc.update({"trace_max_fp64": trace_max, "field_max_fp64": field_max})
        # traces below 1e-10 of the largest field value hold only the numerical precursor ahead of
        # the wave front (FP32 rounds it away): no arrival yet, nothing to compare
        if trace_max > 1e-10 * field_max:
            accuracy = {"trace_rel_l2_vs_fp64": float(np.linalg.norm(tr - tr64) / np.linalg.norm(tr64)),
                        "steps": acc_steps, "shots": S_tot, **energy_acc}
            if len(ws) > 1:
                # each mesh on its own; None where the wave has not reached a receiver yet (its FP64
                # traces hold only the numerical precursor, below 1e-10 of the batch's largest
                # amplitude, which FP32 rounds to zero)
                top = np.abs(tr64).max()
                per = []
                for a, b in zip(cuts[:-1], cuts[1:]):
                    if np.abs(tr64[a:b]).max() < 1e-10 * top:
                        per.append(None)
                        continue
                    per.append(float(np.linalg.norm(tr[a:b] - tr64[a:b]) / np.linalg.norm(tr64[a:b])))
                accuracy["per_mesh"] = per
                accuracy["per_mesh_max"] = max((v for v in per if v is not None), default=None)
                accuracy["per_mesh_note"] = ("None: no arrival at a receiver in these steps (FP64 traces "
                                             "below 1e-10 of the batch maximum)")
        else:  # the wave has not reached a receiver yet: nothing to compare
            accuracy = {"trace_rel_l2_vs_fp64": None, "steps": acc_steps, "shots": S_tot, **energy_acc,
                        "note": "no arrival at a receiver in %d steps (FP64 traces below 1e-10 of the largest "
                                "field value); the long-run accuracy of this workload is checked in "
                                "tests/test_gpu_fullsize.py" % acc_steps}

    # ---- plain FP64 path on the first mesh, one shot, timed two ways ------------------------
    # (1) exactly as `value`: one dg_gpu_step(K) call (CUDA graphs), events on the context's stream
    #     around it, no flush (a one-shot FP64 state of this mesh may sit in L2 between steps);
    # (2) events around every launch with a 256 MB write before every step, so each step starts
    #     from a cold L2 (the state streams from HBM, as it does for the batch, whose 1.5 GB
    #     cannot stay in L2)
    s1 = P.host.build_setup(one_shot(ws[0]), full=False, n_steps=table)
    with eng.Engine(eng.mesh_from_setup(s1, with_ref_ops=False), "fp64", device=device) as e1:
        e1.step(W_steps)
        st1 = e1.stats()
        s64 = e1.stream()
        torch.cuda.synchronize(device)
        ev0.record(s64)
        e1.step(K_steps)
        ev1.record(s64)
        ev1.synchronize()
        same1 = ev0.elapsed_time(ev1)
        _, _, tot1 = e1.step_profiled(K_steps, flush_l2=True)
    fp64_same = st1["dof_per_step"] * K_steps / (same1 * 1e-3)
    fp64_value = st1["dof_per_step"] * K_steps / (tot1 * 1e-3)
    fp64_state = 30 * ws[0].K * 8
    clocks = sampler.stop()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K_steps, "warmup": W_steps,
            "ms_per_step": t_max / K_steps, "higher_is_better": True,
            "scaling": {"weak": "weak", "strong": "strong", "replicas": "weak"}[share], "vs_baseline": None,
            "dtype": {"fp32": "f32", "fp32_kahan": "f32 (Kahan-compensated)", "fp64": "f64"}[args.precision],
            "data": "synthetic (seeded meshes and media)",
            "config": {"workload": desc, "meshes": len(ws), "K": K_tot, "shots": S_tot, "precision": args.precision,
                       "kernels": eng.KERNEL_FAMILIES[st["kernel_family"]], "variant": args.variant,
                       "parallelism": ("single GPU" if world == 1 else
                                       {"weak": "one job of %d shots, 64 contiguous shots per GPU (shard_shots)"
                                                % (64 * world),
                                        "strong": "one job of meshes split over %d GPUs by cost (shard_meshes)"
                                                  % world,
                                        "replicas": "the same one-shot mesh on every GPU (no split)"}[share]),
                       "l2": ("inputs larger than L2: state %.2f GB per GPU" % (state_bytes / 1e9))
                       if state_bytes > 126e6 * 1.5 else "state smaller than L2 (not flushed)",
                       "block_threads": st["block_threads"]},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "bytes_per_launch": dom[1], "ms_per_launch": dom[2], "time_source": time_source,
                         "step_GBs": bytes_step / (t_max / K_steps * 1e-3) / 1e9,
                         "kernels": kernels},
            "fp64_plain": {"value": fp64_value, "unit": UNIT, "shots": 1, "K": ws[0].K,
                           "kernels": eng.KERNEL_FAMILIES[st1["kernel_family"]],
                           "l2": "flushed before every step (256 MB write), events around every launch",
                           "ms_per_step": tot1 / K_steps,
                           "GBs": st1["bytes_per_step"] / (tot1 / K_steps * 1e-3) / 1e9,
                           "ratio_batched_over_fp64_plain": value / world / fp64_value,
                           "value_same_timing": fp64_same,
                           "same_timing": "one dg_gpu_step(%d) call, CUDA graphs, events around the call, no "
                                          "flush: the timing of `value`; FP64 state %.0f MB (L2 126 MB)"
                                          % (K_steps, fp64_state / 1e6),
                           "ms_per_step_same_timing": same1 / K_steps,
                           "GBs_same_timing": st1["bytes_per_step"] / (same1 / K_steps * 1e-3) / 1e9,
                           "ratio_same_timing": value / world / fp64_same},
            "accuracy": accuracy,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "chunk_steps": e2e_chunk,
                    "what": "dg_gpu_set_wavelet (every mesh, pinned host wavelets) + dg_gpu_step_async per "
                            "%d-step chunk, and dg_gpu_fetch_traces (every mesh and shot, pinned host buffers) "
                            "of each chunk while the next one steps, then every rank's traces gathered on rank 0 "
                            "(sharding.gather_traces), wall clock, slowest rank" % e2e_chunk},
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(ws[0])
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="multishot")
    ap.add_argument("--precision", choices=["fp32", "fp32_kahan", "fp64"], default="fp32")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=0,
                    help="dg_gpu_opts.variant of the headline run (0 automatic; see include/dg_gpu.h)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
