#!/usr/bin/env python
"""Benchmark: particle-substeps/s of the PBF solver step on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--legs all|main|...]

Workload (one step = one PBF substep): the 262,144-particle dam break (64^3
lattice at spacing 0.5h with +-0.01h seeded jitter, h = 0.1, box 80h x 40h x
40h, rest density 6378, eps 600, s_corr k 0.1 n 4 dq 0.2h, XSPH 0.01,
vorticity 0.0005, dt = 1/120, 4 Jacobi iterations), synthetic data.

Timing: W untimed substeps, then K substeps, each bracketed by CUDA events on
the launching stream after an L2 flush (a 256 MiB write); value = particles x K
/ sum of substep times, whole job (max over ranks). Under torchrun every rank
runs its own replica of the scene (no data-path collective).

e2e: the same K substeps through the public host-buffer call (pbf_step_host):
step k copies the state the timed step k started from up from pinned host
memory, uploads it, runs one substep and copies the positions back; beside it
the same chain from device-resident inputs and the host link's rates.

--impl reference times the reference's own CPU solver (src/solver.cpp built
from its sources into oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "particle-substeps/s at ≤1% max density error: plain vs learned+batched, 1×B200"
UNIT = "particle-substeps/s"
L2_FLUSH_BYTES = 256 << 20
# algorithmic bytes per particle and launch (12-byte vectors, each array read or written once)
ALG_BYTES = {"hash": 16, "reorder": 80, "lambda": 16, "dp": 28, "curl": 36, "vort": 48, "neighbors": 12}
# algorithmic bytes of the HBM-bound kernels of this design, per particle (scan: per cell key):
# hash reads x, v and writes cell, ticket; scatter reads cell, ticket, the cell start and writes
# one slot; reorder reads x, v, cell, perm, the cell start, the cell's slot and writes x, v,
# x_old, perm and the sorted cell; scan reads a count and writes a start and a cleared count
MEM_BYTES = {"hash": 32, "scatter": 16, "reorder": 84, "scan_per_key": 12}
# algorithmic flops per neighbour pair (FMA = 2)
ALG_FLOPS_PER_PAIR = {"lambda": 30, "dp": 40, "curl": 25, "vort": 30}


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured", p
    return 6650.0, "fallback", {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self) -> dict:
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def measure_fp32_peaks() -> dict:
    """Measured FP32 FMA throughput (TFLOP/s) of this GPU, scalar and packed f32x2."""
    import ctypes as C

    from pbf_b200._lib import check, lib
    sc, pk = C.c_double(), C.c_double()
    check(lib().pbf_measure_fp32_peak(C.byref(sc), C.byref(pk)))
    return {"scalar_tflops": round(sc.value, 2), "f32x2_tflops": round(pk.value, 2),
            "best": max(sc.value, pk.value)}


def link_rates(pin_pos, pin_vel, d_pos, d_vel, out_h, d_out, stream, reps: int = 10) -> dict:
    """Host link rates of one step's copies on `stream`: positions and velocities
    up (24 B per particle), positions down (12 B), and both directions at once
    (the down copy on a second stream)."""
    import torch
    nb_in = pin_pos.numel() * 4 + pin_vel.numel() * 4
    nb_out = out_h.numel() * 4
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    a, b = ev(), ev()
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        d_pos.copy_(pin_pos, non_blocking=True)
        d_vel.copy_(pin_vel, non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize()
    h2d = nb_in * reps / (a.elapsed_time(b) * 1e-3) / 1e9
    a.record(stream)
    for _ in range(reps):
        out_h.copy_(d_out, non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize()
    d2h = nb_out * reps / (a.elapsed_time(b) * 1e-3) / 1e9
    side = torch.cuda.Stream()
    a.record(stream)
    side.wait_event(a)
    for _ in range(reps):
        d_pos.copy_(pin_pos, non_blocking=True)
        d_vel.copy_(pin_vel, non_blocking=True)
    with torch.cuda.stream(side):
        for _ in range(reps):
            out_h.copy_(d_out, non_blocking=True)
    stream.wait_stream(side)
    b.record(stream)
    torch.cuda.synchronize()
    both = (nb_in + nb_out) * reps / (a.elapsed_time(b) * 1e-3) / 1e9
    return {"h2d_gbs": round(h2d, 1), "d2h_gbs": round(d2h, 1), "both_directions_gbs": round(both, 1),
            "copy_ms_per_step": round(1e3 * (nb_in / (h2d * 1e9) + nb_out / (d2h * 1e9)), 4)}


REF_SAMPLE = ("reference PBFSolver::solve (src/solver.cpp built from its sources, -O3 -fopenmp, stdout to "
              "/dev/null) on the 262,144-particle dam break itself (64^3 lattice, box 80h x 40h x 40h, grid "
              "80x40x40, 4 iterations), with the reference's own formulas: it has no stable mode")


def host_threads() -> int:
    """Host threads this process may run on (its affinity mask; the machine's
    count where the platform has no mask)."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_baseline(seconds: float = 12.0) -> dict:
    """The reference CPU solver (kind "reference"), or the oracle port when the
    reference could not be built, on a bounded sample of the same workload: the
    262,144-particle dam break from its initial state, whole substeps until
    `seconds` have passed (at least two)."""
    from oracle import oracle as O
    from pbf_b200 import scenes
    sc = scenes.config1(stable=False)
    if O.refcpu_available():
        ref = O.RefCpu(sc.para, sc.grid_space, dims=(80, 40, 40))
        threads = host_threads()
        ref.set_threads(threads)
        pos, vel = sc.pos, sc.vel
        steps, t0 = 0, time.perf_counter()
        while True:
            pos, vel = ref.solve(pos, vel, substeps=1, quiet=True)
            steps += 1
            el = time.perf_counter() - t0
            if (el >= seconds and steps >= 2) or steps >= 200:
                break
        return {"value": sc.n * steps / el, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{REF_SAMPLE}; the first {steps} substeps, {el:.1f} s"}
    orc = O.Oracle(O.params_for_scene(sc, arith=1), sc.pos, sc.vel)
    steps, t0 = 0, time.perf_counter()
    while True:
        orc.substep()
        steps += 1
        el = time.perf_counter() - t0
        if (el >= seconds and steps >= 2) or steps >= 200:
            break
    return {"value": sc.n * steps / el, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle port on the 262,144-particle dam break, the first {steps} substeps, {el:.1f} s"}


def run_reference(args) -> int:
    """The reference's CPU solver on the same workload as the GPU arm: the
    262,144-particle dam break, W untimed substeps, then K timed ones (each a
    whole PBFSolver::solve), on all host cores."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from oracle import oracle as O
    from pbf_b200 import scenes
    sc = scenes.config1(stable=False)
    line = {"metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "impl": "reference", "scaling": "weak", "dtype": "f32",
            "data": "synthetic", "config": workload_config(args)}
    line["config"]["workload"] = line["config"]["workload"].replace("stable mode", "the reference CPU solver's own "
                                                                    "formulas (src/solver.cpp)")
    line["config"]["formulas"] = "the reference's own (src/solver.cpp); the GPU arm runs the stable mode"
    if not O.refcpu_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU solver not built (oracle/_ref missing)"}))
        return 0
    ref = O.RefCpu(sc.para, sc.grid_space, dims=(80, 40, 40))
    threads = host_threads()
    ref.set_threads(threads)
    pos, vel = sc.pos, sc.vel
    for _ in range(args.warmup):
        pos, vel = ref.solve(pos, vel, substeps=1, quiet=True)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        pos, vel = ref.solve(pos, vel, substeps=1, quiet=True)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    v = sc.n * args.steps / tot
    line.update({"value": v, "ms_per_step": 1e3 * tot / args.steps, "vs_baseline": None,
                 "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                                  "sample": f"{REF_SAMPLE}; each step one substep, after {args.warmup} untimed"},
                 "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line))
    return 0


def workload_config(args, sc=None) -> dict:
    if args.main_scene == "large":
        return {"workload": f"double dam break {sc.n}: two 128^3 lattices, sphere r=20h, box 320h x 160h x 160h, "
                            "rho0 6378, eps 600, 4 Jacobi iterations, dt 1/120, stable mode",
                "particles": sc.n, "iterations": 4, "grid": [320, 160, 160],
                "l2": "inputs larger than L2, and flushed before every timed step (256 MiB write)",
                "parallelism": f"{args.gpus} independent replicas" if args.gpus > 1 else "single scene"}
    return {"workload": "dam_break_262144: 64^3 lattice, spacing 0.5h, jitter 0.01h, h=0.1, box 80h x 40h x 40h, "
                        "rho0 6378, eps 600, 4 Jacobi iterations, dt 1/120, stable mode",
            "particles": 262144, "iterations": 4, "grid": [80, 40, 40],
            "l2": "flushed before every timed step (256 MiB write)",
            "parallelism": f"{args.gpus} independent replicas" if args.gpus > 1 else "single scene"}


def run_b200(args) -> int:
    import numpy as np
    import torch
    import torch.distributed as dist

    import pbf_b200
    from pbf_b200 import Solver, scenes

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from pbf_b200 import autotune
    if args.main_scene == "large":
        sc = scenes.config4(seed=rank, iterations=4, n_small=0)[0]
    else:
        sc = scenes.config1(seed=rank, iterations=4)
    n = sc.n
    stream = torch.cuda.current_stream()
    if args.pair_lanes and args.cell_scale and args.block_size:
        tuned = {"cell_scale": args.cell_scale, "block_size": args.block_size, "pair_lanes": args.pair_lanes,
                 "table": "fixed on the command line"}
    else:
        # timed over the substeps the benchmark times (after its warm-up)
        tuned = autotune.tune([sc], iterations=4, warm=max(args.warmup, 3), substeps=min(max(args.steps, 4), 10))
    ext_kw = dict(grid_dims=autotune.dims_for_scale(sc.ext_overrides["grid_dims"], tuned["cell_scale"]),
                  **autotune.ext_for(tuned))
    solver = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(**ext_kw))
    solver.upload(sc.pos, sc.vel)
    kernels = solver.kernel_count()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    fp32_peaks = measure_fp32_peaks()

    for _ in range(max(args.warmup, 3)):
        solver.step(1, stream)
    torch.cuda.synchronize()
    state_pos, state_vel = solver.download()  # start of the timed region, reused by the profiled pass

    errs = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        time.sleep(0.3)  # let the sampler start before the timed steps
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            solver.step(1, stream)
            ev[k][1].record(stream)
            errs.append(solver.measure_density_error(stream))  # after the step's end event
        torch.cuda.synchronize()
        time.sleep(0.3)
    barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    tot_s = max_over_ranks(sum(step_ms) / 1e3)
    value = n * world * args.steps / tot_s
    ncnt = solver.fetch("ncnt")
    pairs = float(ncnt.sum())

    # Per-kernel durations: the same K substeps from the same state on a handle
    # whose graph records a CUDA event pair around every launch (the event nodes
    # slow the graph down, so the headline timing above runs without them).
    prof = Solver(sc.para, sc.grid_space, sc.boundary, sc.ext(profile=1, **ext_kw))
    prof.upload(state_pos, state_vel)
    stage_acc = {}
    # the state each timed substep starts from (host, particle order), for the
    # end-to-end legs; at most 2 GB of them (step k then takes frame k mod count)
    frames = []
    max_frames = max(1, int(2e9 // (24 * n)))
    for k in range(args.steps):
        if len(frames) < max_frames:
            fp, fv = prof.download()
            frames.append((torch.from_numpy(fp).pin_memory(), torch.from_numpy(fv).pin_memory()))
        flush.zero_()
        prof.step(1, stream)
        for name, ms in prof.stage_times().items():
            stage_acc[name] = stage_acc.get(name, 0.0) + ms
    stages = {k: v / args.steps for k, v in stage_acc.items() if v > 0}
    prof.close()

    # L2-warm throughput: the same substeps back to back without flushing
    warm = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    warm[0].record(stream)
    solver.step(args.steps, stream)
    warm[1].record(stream)
    torch.cuda.synchronize()
    warm_s = max_over_ranks(warm[0].elapsed_time(warm[1]) / 1e3)

    # end to end through the public API: pinned host state in, step, positions
    # out; step k uploads the state the timed step k started from, so these legs
    # run the same substeps as `value`
    out_h = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    d_pos = torch.empty((n, 3), dtype=torch.float32, device=dev)
    d_vel = torch.empty((n, 3), dtype=torch.float32, device=dev)
    d_out = torch.empty((n, 3), dtype=torch.float32, device=dev)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        e2e_ev[k][0].record(stream)
        d_pos.copy_(frames[k % len(frames)][0], non_blocking=True)
        d_vel.copy_(frames[k % len(frames)][1], non_blocking=True)
        solver.upload_device(d_pos, d_vel, stream)
        solver.step(1, stream)
        solver.download_device(d_out, None, stream)
        out_h.copy_(d_out, non_blocking=True)
        e2e_ev[k][1].record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_serial_s = max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev) / 1e3)

    # the same frames through pbf_step_host, pipelined across calls: each call
    # copies its own pinned host inputs up, uploads them, runs one substep and
    # copies the positions down; the library double-buffers the device staging
    # and runs the copies on its own streams, so a call's copies overlap the
    # substeps of its neighbours. The L2 flush stays in the timed region, and the
    # last call's copy-out ends it (host_fence).
    oh2 = [torch.empty((n, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
    solver.step_host(frames[0][0], frames[0][1], oh2[0], 1, stream)  # creates the staging
    solver.host_fence(stream)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    t0.record(stream)
    for k in range(args.steps):
        flush.zero_()
        solver.step_host(frames[k % len(frames)][0], frames[k % len(frames)][1], oh2[k % 2], 1, stream)
    solver.host_fence(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_s = max_over_ranks(t0.elapsed_time(t1) / 1e3)
    e2e_value = n * world * args.steps / e2e_s

    # What bounds the pipelined figure. (a) The same chain with the inputs
    # already on the device: flush, upload (the hash of the upload order),
    # one substep from the uploaded state, download into device memory.
    # (b) The host link's rates for this step's own copies.
    d_frames = [(fp.to(dev), fv.to(dev)) for fp, fv in frames]
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    c0.record(stream)
    for k in range(args.steps):
        flush.zero_()
        solver.upload_device(d_frames[k % len(frames)][0], d_frames[k % len(frames)][1], stream)
        solver.step(1, stream)
        solver.download_device(d_out, None, stream)
    c1.record(stream)
    torch.cuda.synchronize()
    barrier()
    chain_ms = 1e3 * max_over_ranks(c0.elapsed_time(c1) / 1e3) / args.steps
    link = link_rates(frames[0][0], frames[0][1], d_pos, d_vel, out_h, d_out, stream)
    del d_frames
    assert np.isfinite(oh2[(args.steps - 1) % 2].numpy()).all()

    hbm_peak, peak_kind, mp = peaks()
    nkeys_main = solver.ncells + 1
    dom = max(("lambda", "dp", "neighbors", "curl", "vort"), key=lambda s: stages.get(s, 0.0))
    per_launch = {"lambda": 4, "dp": 4}.get(dom, 1)
    launch_ms = stages[dom] / per_launch
    alg_bytes = ALG_BYTES[dom] * n
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    traffic = load_traffic(dom)
    fp32_peak, fp32_kind = fp32_peaks["best"], "measured (FMA probe: pbf_measure_fp32_peak, best of scalar and f32x2)"
    flops = ALG_FLOPS_PER_PAIR.get(dom, 0) * pairs
    step_bytes = (283.8 + 44 * 4) * n
    clocks = clk.summary()
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded jittered lattice)",
        "config": workload_config(args, sc),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 12 * n,
                "note": "every step one pbf_step_host call: pinned host positions+velocities in (step k: the "
                        "state the timed step k started from, in particle order), upload, one substep, positions "
                        "out to pinned host memory; the library overlaps the copies of neighbouring calls with "
                        "the substeps (own copy streams, double-buffered staging); serial_value: the same steps "
                        "as separate upload/step/download calls, not overlapped; device_chain_ms_per_step: the "
                        "same steps from device-resident inputs (no host copies); link: this step's copies alone",
                "serial_value": n * world * args.steps / e2e_serial_s,
                "ms_per_step": 1e3 * e2e_s / args.steps, "device_chain_ms_per_step": chain_ms, "link": link},
        "gpu_launches": kernels * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg_bytes, "launch_ms": launch_ms},
        "roofline_fp32": {"kernel": dom, "achieved": flops / (launch_ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                          "peak": fp32_peak, "frac": flops / (launch_ms * 1e-3) / 1e12 / fp32_peak,
                          "peak_kind": fp32_kind, "probe": fp32_peaks, "pairs": pairs},
        "roofline_step": {"alg_bytes_per_step": step_bytes, "achieved_gbs": step_bytes / (tot_s / args.steps) / 1e9,
                          "frac_hbm": step_bytes / (tot_s / args.steps) / 1e9 / hbm_peak},
        "stages_ms": {k: round(v, 5) for k, v in stages.items()},
        "stages_note": "per-kernel CUDA-event times from a profiled pass over the same K substeps and state",
        "membound": membound_table(stages, n, nkeys_main, hbm_peak),
        "autotune": dict(autotune.ext_for(tuned), table=tuned["table"]),
        "value_l2_warm": n * world * args.steps / warm_s,
        "density_error": dict(error_summary(errs), note="one-sided rho/rho0 - 1 in FP64 after every timed "
                              "substep; max = over all particles and timed substeps"),
        "clocks": clocks,
    }
    legs = set(args.legs.split(","))
    if legs & {"all", "sweep"}:
        out["sweep"] = measure_sweep(args, flush, stream)
    if legs & {"all", "render"}:
        out["render"] = measure_render(args, solver, sc, stream)
    if legs & {"all", "batched", "learned", "large"}:
        out["batched"] = measure_batched(args, rank, world, dev, flush, stream, barrier, max_over_ranks)
    if legs & {"all", "learned", "large"}:
        plain_ref = {"value": value, "ext_kw": ext_kw, "state": (state_pos, state_vel),
                     "density_error_max": max(e[0] for e in errs),
                     "batched_tune": autotune.ext_for(out["batched"]["autotune"])}
        out["learned"] = measure_learned(args, rank, world, flush, stream, barrier, max_over_ranks, plain_ref,
                                         out["batched"])
        weights = out["learned"].pop("_weights")
        if legs & {"all", "large"}:
            out["large"] = measure_large(args, rank, world, flush, stream, barrier, max_over_ranks, weights)
    if rank == 0 and world == 1 and legs & {"all", "cpu"}:
        out["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(out))
    solver.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def measure_batched(args, rank, world, dev, flush, stream, barrier, max_over_ranks) -> dict:
    """64 independent scenes (particle counts log-uniform in [4,096, 65,536],
    seeded), one launch per phase over all scenes of this rank, block size and
    cell size chosen by the autotuner; scenes are sharded over ranks."""
    import torch

    from pbf_b200 import BatchSolver, autotune, multigpu, scenes
    scs = scenes.config2(seed=0)
    parts = multigpu.assign_scenes([s.n for s in scs], world)
    mine = [scs[i] for i in parts[rank]]
    tuned = autotune.tune(mine, iterations=4, warm=max(args.warmup, 3), substeps=min(max(args.steps, 4), 10))
    para, descs, ov, pos, vel = scenes.batch_inputs(mine, iterations=4)
    for d in descs:
        d["grid_dims"] = autotune.dims_for_scale(d["grid_dims"], tuned["cell_scale"])
    ov.update(autotune.ext_for(tuned))
    b = BatchSolver(para, descs, scenes.default_ext(**ov))
    b.upload(pos, vel)
    b.step(max(args.warmup, 3), stream)
    t, err = _timed_errors(b, args.steps, flush, stream, barrier, max_over_ranks)
    total = sum(s.n for s in scs)
    out = {"workload": "64 scenes, counts log-uniform in [4096, 65536] (seed 0), box aspect U[1,3], 4 iterations",
           "scenes": len(scs), "particles": total, "value": total * args.steps / t, "unit": UNIT,
           "ms_per_step": 1e3 * t / args.steps, "kernels_per_step": b.kernel_count(),
           "autotune": dict(autotune.ext_for(tuned), table=tuned["table"]), "density_error": err}
    b.close()
    return out


def error_summary(errs) -> dict:
    """Density error over the timed substeps, each measured after its substep in
    FP64: max = the largest one-sided error of any particle after any timed
    substep (the metric's max); mean_of_substep_max = the per-substep max
    averaged over the substeps; mean = over particles and substeps."""
    worst = max(e[0] for e in errs)
    return {"max": worst, "mean_of_substep_max": statistics.mean(e[0] for e in errs),
            "mean": statistics.mean(e[1] for e in errs), "target_max": 0.01, "meets_target": worst <= 0.01}


def _timed_errors(solver, steps, flush, stream, barrier, max_over_ranks):
    """K flushed, event-timed substeps; density error measured after each (untimed)."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    errs = []
    barrier()
    torch.cuda.synchronize()
    for k in range(steps):
        flush.zero_()
        ev[k][0].record(stream)
        solver.step(1, stream)
        ev[k][1].record(stream)
        errs.append(solver.measure_density_error(stream))
    torch.cuda.synchronize()
    barrier()
    t = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1e3)
    return t, error_summary(errs)


# Training recipe of the warm-start network: trajectories of the plain solver
# with LEARN_COLLECT_ITERS Jacobi iterations per substep (the target is the total
# lambda those iterations apply), and the trust region factor (0: none).
LEARN_COLLECT_ITERS = 4
LEARN_TRAIN_SEED = 1000  # scene seed of the training run (evaluation runs use the rank)
LEARN_CLAMP = 32.0
LEARN_FLOOR = 1
LEARN_CORRECTIONS = 2
# common max-error tolerances at which both solvers run adaptively (each
# substep iterates until its max one-sided error is within the tolerance)
LEARN_TOLERANCES = (0.1, 0.05, 0.03)
WARM_BLOCK = 256


def measure_learned(args, rank, world, flush, stream, barrier, max_over_ranks, plain, plain_batched) -> dict:
    """Learned lambda warm start. The MLP is trained here, on the GPU with the
    library's tensor-core kernels, from 2,000 substeps of the 262,144-particle dam
    break run by the plain solver from another lattice jitter than the runs it is
    evaluated on (2,048 random particles per substep), then used
    with LEARN_CORRECTIONS corrections (lambda0 + plain iterations) on config 3
    (the same dam break) and on the 64-scene batch. Every speed-up is taken at
    the same max density error (the largest one-sided error of any particle after
    any timed substep): the other solver runs adaptively (a device-side loop of
    corrections, at most 64) with that error as its per-substep tolerance, so its
    own max error is at most the one it is compared with."""
    import time as _t

    from pbf_b200 import BatchSolver, Solver, autotune, learned, multigpu, scenes
    t0 = _t.perf_counter()
    ext_kw = plain["ext_kw"]
    # trained on the same dam break with another lattice jitter (seed), so the
    # trajectories it is evaluated on below were not seen in training
    scc = scenes.config1(seed=LEARN_TRAIN_SEED + rank, iterations=LEARN_COLLECT_ITERS)
    feat, target = learned.collect(scc, substeps=2000, rows_per_substep=2048, seed=rank, ext=ext_kw)
    t1 = _t.perf_counter()
    tr, losses = learned.train(feat, target, epochs=3, batch=4096, lr=2e-3, log_every=500)
    w32, b32, w16 = tr.params()
    tr.close()
    t2 = _t.perf_counter()
    del feat, target
    out = {"training": {"substeps": 2000, "collect_iterations": LEARN_COLLECT_ITERS, "rows": 2000 * 2048,
                        "epochs": 3, "batch": 4096, "loss_first": losses[0][1], "loss_last": losses[-1][1],
                        "collect_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2)},
           "corrections": LEARN_CORRECTIONS, "warm_clamp": LEARN_CLAMP, "warm_floor": LEARN_FLOOR,
           "train_scene_seed": LEARN_TRAIN_SEED + rank}

    # The fused warm pass stages the network's weights once per block and runs
    # 128-row MMA tiles: warm-started solvers take 256-thread blocks, one block
    # per tile of slots; plain ones keep the autotuner's choice.
    def launch(kw, warm):
        return dict(kw, block_size=WARM_BLOCK, persistent=0) if warm else dict(kw)

    def single(iters, warm, **kw):
        sc = scenes.config1(seed=rank, iterations=iters)
        s = Solver(sc.para, sc.grid_space, sc.boundary,
                   sc.ext(warm_start=1 if warm else 0, warm_clamp=LEARN_CLAMP, warm_floor=LEARN_FLOOR,
                          **launch(ext_kw, warm), **kw))
        if warm:
            learned.install(s, w16, b32)
        s.upload(sc.pos, sc.vel)
        s.step(max(args.warmup, 3), stream)
        before = s.stats()["total_iterations"]
        t, err = _timed_errors(s, args.steps, flush, stream, barrier, max_over_ranks)
        corr = (s.stats()["total_iterations"] - before) / args.steps
        s.close()
        r = {"value": sc.n * world * args.steps / t, "unit": UNIT, "ms_per_step": 1e3 * t / args.steps,
             "density_error": err, "corrections_per_substep": corr}
        if kw.get("adaptive"):
            r["density_tol"] = kw["density_tol"]
        return r

    scs = scenes.config2(seed=0)
    parts = multigpu.assign_scenes([x.n for x in scs], world)
    mine = [scs[i] for i in parts[rank]]
    total = sum(x.n for x in scs)
    bt = plain["batched_tune"]

    def batch(iters, warm, **kw):
        para, descs, ov, pos, vel = scenes.batch_inputs(mine, iterations=iters)
        for d in descs:
            d["grid_dims"] = autotune.dims_for_scale(d["grid_dims"], bt["cell_scale"])
        ov.update(launch(bt, warm), warm_start=1 if warm else 0, warm_clamp=LEARN_CLAMP, warm_floor=LEARN_FLOOR,
                  **kw)
        b = BatchSolver(para, descs, scenes.default_ext(**ov))
        if warm:
            learned.install(b, w16, b32)
        b.upload(pos, vel)
        b.step(max(args.warmup, 3), stream)
        before = b.stats()["total_iterations"]
        t, err = _timed_errors(b, args.steps, flush, stream, barrier, max_over_ranks)
        corr = (b.stats()["total_iterations"] - before) / args.steps
        b.close()
        r = {"scenes": len(scs), "particles": total, "value": total * args.steps / t, "unit": UNIT,
             "ms_per_step": 1e3 * t / args.steps, "density_error": err, "corrections_per_substep": corr}
        if kw.get("adaptive"):
            r["density_tol"] = kw["density_tol"]
        return r

    adapt = lambda tol: {"adaptive": 1, "density_tol": float(tol), "max_iterations": 64}  # noqa: E731
    # config 3: the learned single scene, and plain at its error / learned at plain's
    out["single"] = single(LEARN_CORRECTIONS, True)
    e_l = out["single"]["density_error"]["max"]
    e_p = plain["density_error_max"]
    out["plain_at_learned_error"] = single(1, False, **adapt(e_l))
    out["learned_at_plain_error"] = single(1, True, **adapt(e_p))
    # the 64-scene batch, the same both ways
    out["batched"] = batch(LEARN_CORRECTIONS, True)
    e_lb = out["batched"]["density_error"]["max"]
    e_pb = plain_batched["density_error"]["max"]
    out["plain_batched_at_learned_error"] = batch(1, False, **adapt(e_lb))
    out["learned_batched_at_plain_error"] = batch(1, True, **adapt(e_pb))
    # learned + batched against the plain single scene at the learned batch's error
    out["plain_single_at_learned_batch_error"] = single(1, False, **adapt(e_lb))
    # both solvers adaptive to the same tight tolerances, on config 3 and on the batch
    out["at_tolerance"] = {}
    for tol in LEARN_TOLERANCES:
        r = {"single_learned": single(1, True, **adapt(tol)), "single_plain": single(1, False, **adapt(tol)),
             "batch_learned": batch(1, True, **adapt(tol)), "batch_plain": batch(1, False, **adapt(tol))}
        r["speedup_single"] = r["single_learned"]["value"] / r["single_plain"]["value"]
        r["speedup_batch"] = r["batch_learned"]["value"] / r["batch_plain"]["value"]
        r["speedup_learned_batched_vs_plain_single"] = r["batch_learned"]["value"] / r["single_plain"]["value"]
        out["at_tolerance"][str(tol)] = r
    out["speedup"] = {
        "config3_at_learned_error": out["single"]["value"] / out["plain_at_learned_error"]["value"],
        "config3_at_plain4_error": out["learned_at_plain_error"]["value"] / plain["value"],
        "batch_at_learned_error": out["batched"]["value"] / out["plain_batched_at_learned_error"]["value"],
        "batch_at_plain4_error": out["learned_batched_at_plain_error"]["value"] / plain_batched["value"],
        "learned_batched_vs_plain_single_at_learned_batch_error":
            out["batched"]["value"] / out["plain_single_at_learned_batch_error"]["value"],
        "note": "value / value of the other solver run adaptively to the same max density error (tolerance = "
                "the max error the first one reached; corrections capped at 64)"}
    out["_weights"] = (w16, b32)
    return out


def measure_large(args, rank, world, flush, stream, barrier, max_over_ranks, weights) -> dict:
    """The 4,194,304-particle double dam break (two 128^3 blocks, sphere of radius
    20h at the centre of a 320h x 160h x 160h box) batched with 8 scenes of
    65,536 particles: plain with 4 iterations; then, at the max density error the
    plain run reached (mean over its substeps) as the tolerance, the adaptive
    plain loop and the learned warm start + adaptive plain loop (at least 2
    corrections, at most 16)."""
    from pbf_b200 import BatchSolver, learned, multigpu, scenes
    out = {"workload": "double dam break 2 x 128^3 + sphere r=20h, box 320h x 160h x 160h, + 8 x 65,536"}
    w16, b32 = weights
    legs = [("plain", 4, {})]
    for label, iters, kw in legs + [("plain_adaptive", 2, {"adaptive": 1, "max_iterations": 16}),
                                    ("learned_adaptive", 2, {"warm_start": 1, "warm_floor": LEARN_FLOOR,
                                                             "warm_clamp": LEARN_CLAMP,
                                                             "adaptive": 1, "max_iterations": 16})]:
        if kw.get("adaptive"):
            kw = dict(kw, density_tol=out["plain"]["density_error"]["max"])
        scs = scenes.config4(seed=0, iterations=iters)
        parts = multigpu.assign_scenes([x.n for x in scs], world)
        mine = [scs[i] for i in parts[rank]]
        para, descs, ov, pos, vel = scenes.batch_inputs(mine, iterations=iters)
        ov.update(kw)
        b = BatchSolver(para, descs, scenes.default_ext(**ov))
        if kw.get("warm_start"):
            learned.install(b, w16, b32)
        b.upload(pos, vel)
        b.step(max(args.warmup, 3), stream)
        before = b.stats()
        t, err = _timed_errors(b, args.steps, flush, stream, barrier, max_over_ranks)
        total = sum(x.n for x in scs)
        st = b.stats()
        out[label] = {"min_iterations": iters, "particles": total, "value": total * args.steps / t, "unit": UNIT,
                      "ms_per_step": 1e3 * t / args.steps, "density_error": err,
                      "mean_iterations": (st["total_iterations"] - before["total_iterations"]) / args.steps}
        if label == "plain":
            # per-kernel times of the same substeps on a profiled handle
            pos_s, vel_s = b.download()
            prof = BatchSolver(para, descs, scenes.default_ext(profile=1, **ov))
            prof.upload(pos_s, vel_s)
            acc = {}
            for _ in range(args.steps):
                flush.zero_()
                prof.step(1, stream)
                for name, ms in prof.stage_times().items():
                    acc[name] = acc.get(name, 0.0) + ms
            nkeys = sum(prof.scene_layout(i)["ncells"] + 1 for i in range(prof.nscenes))
            prof.close()
            stages = {k: v / args.steps for k, v in acc.items() if v > 0}
            out[label]["stages_ms"] = {k: round(v, 5) for k, v in stages.items()}
            out[label]["membound"] = membound_table(stages, sum(x.n for x in mine), nkeys, peaks()[0])
        if kw.get("adaptive"):
            out[label]["density_tol"] = kw["density_tol"]
        b.close()
    return out


def measure_sweep(args, flush, stream) -> dict:
    """Max density error against Jacobi iterations: for the 32,768- and
    262,144-particle dam breaks and the 64-scene batch, each iteration count
    (and the adaptive loop at 1 % with a cap of 64) runs its own trajectory from
    the initial state: W untimed substeps, then K timed ones with the one-sided
    error measured in FP64 after each. Rows: [iterations, ms per substep,
    max error over the timed substeps, mean error, corrections per substep]."""
    import torch

    from pbf_b200 import BatchSolver, Solver, autotune, scenes
    out = {"launch": {"cell_scale": 0.5, "block_size": 256, "pair_lanes": 2},
           "columns": ["iterations", "ms_per_substep", "max_error", "mean_error", "corrections_per_substep"]}
    counts = (2, 4, 8, 16, 32, 64)

    def make(kind, iters, **kw):
        lk = dict(cell_scale=0.5, block_size=256, pair_lanes=2, **kw)
        if kind == "batch":
            scs = scenes.config2(seed=0, iterations=iters)
            para, descs, ov, pos, vel = scenes.batch_inputs(scs, iterations=iters)
            for d in descs:
                d["grid_dims"] = autotune.dims_for_scale(d["grid_dims"], 0.5)
            ov.update(lk)
            s = BatchSolver(para, descs, scenes.default_ext(**ov))
        else:
            sc = scenes.config0(iterations=iters) if kind == "config0" else scenes.config1(iterations=iters)
            s = Solver(sc.para, sc.grid_space, sc.boundary,
                       sc.ext(grid_dims=autotune.dims_for_scale(sc.ext_overrides["grid_dims"], 0.5), **lk))
            pos, vel = sc.pos, sc.vel
        s.upload(pos, vel)
        return s

    def run(s):
        s.step(max(args.warmup, 3), stream)
        before = s.stats()["total_iterations"]
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        errs = []
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            s.step(1, stream)
            ev[k][1].record(stream)
            errs.append(s.measure_density_error(stream))
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
        corr = (s.stats()["total_iterations"] - before) / args.steps
        return [round(ms, 4), round(max(e[0] for e in errs), 5), round(statistics.mean(e[1] for e in errs), 6),
                round(corr, 2)]

    for kind in ("config0", "config1", "batch"):
        rows = []
        for it in counts:
            s = make(kind, it)
            rows.append([it] + run(s))
            s.close()
        s = make(kind, 1, adaptive=1, density_tol=0.01, max_iterations=64, measure_error=1)
        rows.append(["adaptive 1% (cap 64)"] + run(s))
        s.close()
        out[kind] = rows
    reached = [(k, r[0], r[1]) for k in ("config0", "config1", "batch") for r in out[k] if r[2] <= 0.01]
    out["reaches_1pct"] = [{"workload": k, "iterations": it, "ms_per_substep": ms} for k, it, ms in reached]
    return out


def membound_table(stages: dict, n: int, nkeys: int, peak: float) -> dict:
    """Achieved bandwidth of the HBM-bound kernels from per-launch stage times (ms)."""
    out = {}
    for name in ("hash", "scan", "scatter", "reorder"):
        ms = stages.get(name)
        if not ms:
            continue
        b = MEM_BYTES["scan_per_key"] * nkeys if name == "scan" else MEM_BYTES[name] * n
        gbs = b / (ms * 1e-3) / 1e9
        out[name] = {"ms": round(ms, 5), "alg_bytes": b, "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    return out


def measure_render(args, solver, sc, stream) -> dict:
    """Headless screen-space rendering of the single-scene state (the reference
    app's passes: sprite depth, 60 smoothing passes, thickness, normals, room,
    shading) at 800 x 800, timed with CUDA events per frame."""
    import torch

    from pbf_b200 import render
    w = h = 800
    cam = render.box_camera(sc.grid_space, w, h, float(sc.para.radius), smooth_iterations=60)
    r = render.Renderer(w, h)
    for _ in range(3):
        r.frame(cam, solver=solver, stream=stream)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for a, b in ev:
        a.record(stream)
        r.frame(cam, solver=solver, stream=stream)
        b.record(stream)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
    covered = int((r.read("depth_raw") > 0).sum())
    r.close()
    return {"width": w, "height": h, "smooth_iterations": 60, "particles": sc.n, "ms_per_frame": ms,
            "frames_per_s": 1e3 / ms, "covered_pixels": covered}


def load_traffic(kernel: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    return t.get(kernel, {}).get("dram_bytes_per_launch")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--legs", default="all",
                    help="comma list of legs after the single-scene one: all, sweep, batched, learned, large, cpu, "
                         "render (main = the single-scene leg alone)")
    ap.add_argument("--pair-lanes", type=int, default=0, help="with --cell-scale and --block-size: skip the "
                    "autotuner of the single-scene leg and use these launch settings")
    ap.add_argument("--cell-scale", type=float, default=0.0)
    ap.add_argument("--main-scene", choices=["config1", "large"], default="config1",
                    help="scene of the single-scene leg: the 262,144-particle dam break (the headline) or the "
                         "4,194,304-particle double dam break with the sphere (for profiling at scale)")
    ap.add_argument("--block-size", type=int, default=0)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
