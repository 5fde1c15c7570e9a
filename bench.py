#!/usr/bin/env python
"""Throughput of the 3D Flow Lenia step on B200.

Workload (the headline configuration): one world of 128^3 cells x 4 channels,
16 kernels of radius 13 (one per channel pair, parameters drawn from the
seeded sampler), Sobel gradients, RT reintegration (sigma 0.65, dt 0.2), zero
borders.  A "step" is one full simulation step (spectral growth, flow,
transport).  Metric: cell-updates/s = cells x channels x steps / s.  The
world is tuned by the library's autotuner before the timed region
(`config.tuning`: convolution mode, FFT row tile, fused or split growth).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 every rank (one process per GPU) advances its own world (the
single-world step does not shard: replicas, weak scaling); `value` is the sum
over ranks divided by the slowest rank's time.  Started as one process with
`--gpus N`, the script launches its N ranks itself under torch.distributed.run
(lenia_b200/launch.py); started by torchrun, it is one of them.
`--impl reference` times the reference's CPU step (rank 0 only) on the host
cores: every asked step if the run fits its time budget, else the steps that
fit, and the line reports the steps it timed.

Beside the headline: `config1_schedule` (500 steps with every channel
meshed every 10 steps, each mesh with its host synchronisation); and, with
N = 1 only, `batched` (config 3 mix as one batch) and `conv_modes`: the growth stage of the 256^3, radius-20 precision workload in
each convolution mode (FP32 FFT, direct BF16 and BF16x3 on the tensor cores,
with the direct kernel's tensor roofline) and the autotuner's choice.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s at 128^3x4ch"
UNIT = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=128)
    ap.add_argument("--mode", default="rt", choices=["rt", "adv"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--jsonl", default=None, help="also append the result line to this JSONL file")
    ap.add_argument("--batch-worlds", type=int, default=4096,
                    help="worlds of the batched measurement (config 3 mix; 0 = skip)")
    ap.add_argument("--conv-width", type=int, default=256,
                    help="side of the convolution-mode measurement (config 2 workload; 0 = skip)")
    ap.add_argument("--growth", default="auto", choices=["auto", "split", "fused"],
                    help="growth form of the headline world: chosen by the autotuner (default), or fixed "
                         "(FFT convolution, the size's default row tile), e.g. for a profiler run in which "
                         "the autotuner's timings would not be the real ones")
    return ap.parse_args()


def workload(args, rank=0):
    from lenia_b200 import params as P
    mode = P.MODE_RT if args.mode == "rt" else P.MODE_ADV
    return P.config1(seed=1 + rank, width=args.width, mode=mode)


def config_dict(args, wl, n):
    return {
        "workload": f"single world {wl.desc.width}^3 x {wl.desc.channels}ch, {len(wl.kernels)} kernels "
                    f"R={wl.kernels[0].radius}, Sobel, {'RT' if args.mode == 'rt' else 'advection'}, zero borders",
        "grid": [wl.desc.width, wl.desc.height, wl.desc.width],
        "channels": wl.desc.channels,
        "kernels": len(wl.kernels),
        "kernel_radius": wl.kernels[0].radius,
        "parallelism": f"replicas x{n}" if n > 1 else "single GPU",
        "l2": "state ~0.7 GB per world, larger than the 126 MB L2 (no flush needed)",
    }


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", self.gpu_id], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # wait for the first sample so that nvidia-smi's start-up does not
            # overlap the timed region
            t0 = time.time()
            while time.time() - t0 < 20 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_uuid(dev: int) -> str:
    import torch
    try:
        u = torch.cuda.get_device_properties(dev).uuid
        s = str(u)
        return s if s.startswith("GPU-") else "GPU-" + s
    except Exception:
        return str(dev)


# ----------------------------------------------------- algorithmic bytes
def kernel_bytes(wl) -> dict:
    """Algorithmic HBM bytes per step of each kernel (one launch per step;
    the inverse rows of the split growth run as ceil(K / 16) launches that
    together move these bytes): each input read once,
    each output written once (half spectra of KX x D x H complex values,
    octant kernel spectra of KX x (D/2+1) x (H/2+1) floats, 4-byte fields)."""
    d = wl.desc
    W, H, C = d.width, d.height, d.channels
    D = W
    N = W * H * D
    K = len(wl.kernels)
    KX = W // 2 + 1
    HS = KX * D * H  # complex entries of a half spectrum
    KH = KX * (D // 2 + 1) * (H // 2 + 1)
    crt = C if d.rt_all_channels else min(C, 3)
    back = 1 if d.growth_type == 1 else 0
    return {
        "fwd_rows": C * N * 4 + C * HS * 8,
        "planes_fwd": 2 * C * HS * 8,
        "planes_inv": K * HS * 8 * 2 + K * KH * 4,
        "growth_rows": K * HS * 8 + back * C * N * 4 + (2 + back) * C * N * 4,
        # the split growth: inverse rows store u_k, the growth reads them back
        "inverse_rows": K * HS * 8 + K * N * 4,
        "growth_u": K * N * 4 + back * C * N * 4 + (2 + back) * C * N * 4,
        "flow": N * 4 + C * N * (4 + 4 + 12 + 12 + 12),
        "transport": crt * N * 16 + C * N * (4 + 4 + 4) + N * 4,
    }


def step_bytes_per_cell(wl) -> int:
    """Algorithmic HBM bytes per cell of one whole step: every field crosses
    HBM once per producer-consumer edge (forward spectra C*8P with P = 2 passes
    above 36 cells per side, inverse spectra K*(14 + 8(P-1)), stencil C*48 + 4,
    reintegration C*20 + 4)."""
    d = wl.desc
    C, K = d.channels, len(wl.kernels)
    P = 1 if max(d.width, d.height) <= 36 else 2
    return C * 8 * P + K * (14 + 8 * (P - 1)) + C * 48 + 4 + C * 20 + 4


def ncu_traffic(kernel: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    a kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#") and parts[0] == kernel:
                return float(parts[1])
    except OSError:
        pass
    return None


def measured_tensor_peak():
    """Dense BF16 tensor peak in TFLOP/s: the sustained figure (the direct
    convolution runs for tens of milliseconds per launch)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        j = json.load(open(p))
        return float(j["bf16_tflops_sustained"]), "measured sustained"
    except Exception:
        return 1400.0, "fallback sustained"


def conv_measure(args):
    """The growth stage (convolution and growth table) of the precision
    workload (width^3, 3 channels, 9 kernels of radius 20) in every
    convolution mode, per-kernel device times from the library's profiler;
    the direct modes against the tensor-core peak (issued and useful
    multiply-adds); and the autotuner's choice for that world."""
    from lenia_b200 import params as P
    from lenia_b200.world import World
    wl = P.config2(width=args.conv_width, radius=20)
    peak, peak_kind = measured_tensor_peak()
    out = {"workload": f"{args.conv_width}^3 x 3 channels, 9 kernels R=20, growth stage (config 2)", "modes": {}}
    reps = 3
    for mode in ("FFT", "DIRECT_BF16", "DIRECT_BF16X3"):
        w = World(wl.desc, wl.kernels)
        w.set_conv_mode(mode)
        w.set_state(wl.A0.ravel())
        w.stage("GROWTH")
        w.sync()
        w.set_profiling(True)
        for _ in range(reps):
            w.stage("GROWTH")
        w.sync()
        prof = w.profile_read()
        r = {"growth_stage_ms": sum(v[0] for v in prof.values()) / reps,
             "kernels_ms": {k: v[0] / v[1] for k, v in prof.items()}}
        if mode != "FFT":
            issued, useful = w.conv_macs()
            conv_s = prof["direct_conv"][0] / prof["direct_conv"][1] / 1000.0
            r["tensor_roofline"] = {"bound": "tensor", "kernel": "direct_conv", "unit": "TFLOP/s",
                                    "achieved": 2 * issued / conv_s / 1e12, "peak": peak, "peak_kind": peak_kind,
                                    "frac": 2 * issued / conv_s / 1e12 / peak,
                                    "useful_tflops": 2 * useful / conv_s / 1e12,
                                    "issued_over_useful": issued / useful}
        out["modes"][mode] = r
        w.close()
    w = World(wl.desc, wl.kernels)
    w.set_state(wl.A0.ravel())
    out["autotune"] = w.autotune()
    w.close()
    return out


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        j = json.load(open(p))
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------- CPU legs
def cpu_port_rate(wl, steps: int, warmup: int):
    """The oracle's restatement of the reference step (complex-to-complex
    spectral path like the reference's FFTW calls), timed on the host."""
    from oracle.oracle import RestateOracle
    p, ks = wl.desc.as_dict(), [k.as_dict() for k in wl.kernels]
    o = RestateOracle(p, ks, fft_mode="c2c")
    o.set_state(A=wl.A0.ravel())
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    cells = wl.desc.cells * wl.desc.channels
    return cells * steps / dt, dt


def reference_lib(wl):
    """The reference build whose compile-time grid fits this workload (its own
    lenia.cpp / reintegration.cpp / transposition.cpp / mesh.cpp, unmodified),
    or None."""
    from oracle import oracle as O
    w, h, k = wl.desc.width, wl.desc.height, len(wl.kernels)
    for path, side, kmax in ((O.REF_LIB, 32, 12), (O.REF_LIB_128, 128, 16)):
        if w == side and h == side and k <= kmax and os.path.exists(path):
            return path
    return None


def cpu_reference_rate(wl, path: str, steps: int, warmup: int, budget_s: float):
    """The reference's own step (the build at `path`) on the host, each event's
    two slabs on two threads at once as its two sim threads run them.  Up to
    `steps` timed steps, fewer when the next would pass `budget_s` seconds;
    returns (cell-updates/s, seconds timed, steps timed)."""
    from oracle.oracle import RefOracle
    p, ks = wl.desc.as_dict(), [k.as_dict() for k in wl.kernels]
    o = RefOracle(p, ks, lib=path)
    o.set_state(A=wl.A0.ravel())
    if warmup:
        o.step(warmup, slab_threads=True)
    t_start = time.perf_counter()
    timed, dt = 0, 0.0
    while timed < steps:
        t0 = time.perf_counter()
        o.step(1, slab_threads=True)
        dt += time.perf_counter() - t0
        timed += 1
        if timed < steps and (time.perf_counter() - t_start) + dt / timed > budget_s:
            break
    cells = wl.desc.cells * wl.desc.channels
    return cells * timed / dt, dt, timed


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# The reference arm's whole run (warm-up and timed steps) is kept to about
# this many seconds of host time: a step that would take it past the budget
# is not started, and the line reports the steps actually timed.
REF_BUDGET_S = 180.0


def run_reference(args):
    """The reference's CPU step on the host cores, on this arm's workload:
    rank 0 alone runs (the other ranks of a multi-rank launch exit at once).
    Warm-up steps (at most `--warmup`, within a quarter of the budget), then
    up to `--steps` timed steps, each one full step of the world; the steps
    actually timed are the line's `steps`."""
    rank = int(os.environ.get("RANK", "0"))
    n = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    from oracle.oracle import RestateOracle
    wl = workload(args)
    path = reference_lib(wl)
    if path is not None:
        return run_reference_build(args, wl, path, n)
    p, ks = wl.desc.as_dict(), [k.as_dict() for k in wl.kernels]
    o = RestateOracle(p, ks, fft_mode="c2c")
    o.set_state(A=wl.A0.ravel())
    t_start = time.perf_counter()
    warm = 0
    for _ in range(args.warmup):
        t0 = time.perf_counter()
        o.step(1)
        warm += 1
        if (time.perf_counter() - t_start) + (time.perf_counter() - t0) > REF_BUDGET_S / 4:
            break
    timed, dt = 0, 0.0
    while timed < args.steps:
        t0 = time.perf_counter()
        o.step(1)
        dt += time.perf_counter() - t0
        timed += 1
        if timed < args.steps and (time.perf_counter() - t_start) + dt / timed > REF_BUDGET_S:
            break
    cells = wl.desc.cells * wl.desc.channels
    rate = cells * timed / dt
    cores = cpu_threads()
    sample = (f"{timed} timed steps (+{warm} warm-up) of the whole world on the host"
              + ("" if timed == args.steps else f" (of {args.steps} asked: the run is kept within "
                 f"{REF_BUDGET_S:.0f} s)")
              + f"; C restatement of the reference step with its complex-to-complex FFT structure, "
                f"OpenMP over {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": n,
        "steps": timed, "warmup": warm, "ms_per_step": dt * 1000.0 / timed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": config_dict(args, wl, 1),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line, args)
    return 0


def run_reference_build(args, wl, path: str, n: int):
    """The reference arm on the reference's own code: its lenia.cpp,
    reintegration.cpp, transposition.cpp and mesh.cpp built at this
    workload's size (oracle/_ref), stepped with its two sim threads (each
    event's two slabs at once, as render.cpp:357-604 runs them).  The
    reference uses two host threads by design (SIM_THREADS, render.h:14); the
    project's FFT stands in for FFTW, which is absent."""
    warm = min(args.warmup, 1)
    rate, dt, timed = cpu_reference_rate(wl, path, args.steps, warm, REF_BUDGET_S)
    sample = (f"{timed} timed steps (+{warm} warm-up) of the whole world on the host"
              + ("" if timed == args.steps else f" (of {args.steps} asked: the run is kept within "
                 f"{REF_BUDGET_S:.0f} s)")
              + "; the reference's own step code built at this size, two sim threads (slab 0 and "
                "slab 1 of every event at once); a project FFT stands in for FFTW")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": n,
        "steps": timed, "warmup": warm, "ms_per_step": dt * 1000.0 / timed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": config_dict(args, wl, 1),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 2, "kind": "reference", "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line, args)
    return 0


# ------------------------------------------------------------ batches
def batch_measure(args, rank, n, stream, barrier, max_over_ranks):
    """World-steps/s of a batch of independent worlds (the config 3 mix:
    sides 24-96, 3 channels, 9 kernels, RT or advection per world), sharded
    across the ranks by cost with no exchange while stepping; beside it the
    plain loop (each world its own World, stepped one after another) over a
    subset of this rank's worlds.  The batch is tuned first
    (lenia_batch_autotune: per grid shape the convolution mode, row tile and
    fused or split growth that time fastest), outside the timed region."""
    import torch
    from lenia_b200 import params as P
    from lenia_b200.batch import Batch, shard_worlds, world_cost
    from lenia_b200.world import World
    wls = P.config3(args.batch_worlds, seed=3)
    mine = shard_worlds([world_cost(wl.desc, len(wl.kernels)) for wl in wls], n)[rank]
    sub = [wls[i] for i in mine]
    b = Batch([wl.desc for wl in sub], [wl.kernels for wl in sub], lanes=64)
    for i, wl in enumerate(sub):
        b.set_state(i, wl.A0)
    tune = b.autotune()
    choices = {}
    for wl, r in zip(sub, tune):
        choices.setdefault(str(wl.desc.width), {"conv_mode": r["conv_mode"], "growth_split": r["growth_split"],
                                                "row_tile": r["row_tile"]})
    b.set_stream(stream.cuda_stream)
    b.step(3)
    steps = 10
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1)) / steps
    b.sync()
    launches = b.launches_per_step()
    grouped = b.grouped_worlds()
    # the same batch with every world on its own launches (the lanes), for
    # comparison; the fields are the same either way
    b.set_batched_launches(False)
    b.set_stream(stream.cuda_stream)
    b.step(2)
    barrier()
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    barrier()
    lanes_ms = max_over_ranks(e0.elapsed_time(e1)) / steps
    lanes_launches = b.launches_per_step()
    b.sync()
    b.close()
    plain = sub[:min(64, len(sub))]
    ws = []
    for wl in plain:
        w = World(wl.desc, wl.kernels)
        w.set_stream(stream.cuda_stream)
        w.set_state(wl.A0.ravel())
        w.step(2)
        ws.append(w)
    barrier()
    e0.record(stream)
    for _ in range(3):
        for w in ws:
            w.step(1)
    e1.record(stream)
    barrier()
    plain_ms = e0.elapsed_time(e1) / 3
    for w in ws:
        w.close()
    cells = sum(wl.desc.width ** 3 * wl.desc.channels for wl in wls)
    # the whole-step byte model summed over the batch's worlds, against the
    # measured copy bandwidth
    peak, peak_kind = measured_peaks()
    step_bytes = sum(step_bytes_per_cell(wl) * wl.desc.width ** 2 * wl.desc.height for wl in wls)
    return {
            "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_bytes / (ms / 1000.0) / 1e9 / n,
                              "peak": peak, "peak_kind": peak_kind, "unit": "GB/s per GPU",
                              "frac": step_bytes / (ms / 1000.0) / 1e9 / n / peak},"workload": f"{args.batch_worlds} worlds, sides 24-96 (config 3 mix), 3 channels, 9 kernels, "
                        f"RT or advection per world, sharded over {n} GPU(s)",
            "world_steps_per_s": args.batch_worlds / (ms / 1000.0), "ms_per_step": ms,
            "cell_updates_per_s": cells / (ms / 1000.0), "graph_launches_per_step": 1,
            "gpu_launches_per_step": launches, "worlds_in_batched_launches": grouped * n,
            "per_world_launches": {"world_steps_per_s": args.batch_worlds / (lanes_ms / 1000.0),
                                   "ms_per_step": lanes_ms, "gpu_launches_per_step": lanes_launches},
            "plain_world_steps_per_s_per_gpu": len(ws) / (plain_ms / 1000.0),
            "plain_sample_worlds": len(ws), "autotune_by_side": choices}


# ------------------------------------------------------------ GPU arm
def run_ours(args):
    import numpy as np
    import torch

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    n = int(os.environ.get("WORLD_SIZE", "1"))
    if local >= torch.cuda.device_count():
        raise SystemExit(f"rank {rank}: local rank {local} but {torch.cuda.device_count()} visible GPU(s)")
    torch.cuda.set_device(local)
    dist = None
    if n > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    from lenia_b200.world import World
    wl = workload(args, rank)
    w = World(wl.desc, wl.kernels)
    stream = torch.cuda.current_stream()
    w.set_stream(stream.cuda_stream)
    w.set_state(wl.A0.ravel())
    C, N = wl.desc.channels, wl.desc.cells
    # the world as its user runs it: tuned by the library's autotuner
    # (convolution mode, row tile, fused or split growth), outside the timing
    if args.growth == "auto":
        tuning = w.autotune()
    else:
        w.set_tuning(0, args.growth == "split")
        tuning = {"conv_mode": "FFT", "row_tile": 0, "growth_split": args.growth == "split", "ms": None}

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(gpu_uuid(local)) as clk:
        w.step(args.warmup)
        barrier()
        e0.record(stream)
        w.step(args.steps)
        e1.record(stream)
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    w.sync()
    launches = w.launches_per_step * args.steps
    value = n * N * C * args.steps / (ms / 1000.0)

    # per-kernel device time over a second timed pass (CUDA events around
    # every launch, on the launching stream)
    w.set_profiling(True)
    prof_steps = max(10, min(args.steps, 200))
    w.step(prof_steps)
    prof = w.profile_read()
    w.set_profiling(False)
    total = sum(v[0] for v in prof.values()) or 1.0
    kb = kernel_bytes(wl)
    top = max(prof.items(), key=lambda kv: kv[1][0])
    top_name, (top_ms, top_n) = top
    per_step_ms = top_ms / prof_steps
    peak, peak_kind = measured_peaks()
    achieved = kb.get(top_name, 0) / (per_step_ms / 1000.0) / 1e9
    kernels_table = {k: {"ms_per_launch": v[0] / v[1], "launches_per_step": v[1] / prof_steps,
                         "share": v[0] / total,
                         "gbs": kb.get(k, 0) / (v[0] / prof_steps / 1000.0) / 1e9 if k in kb else None}
                     for k, v in prof.items()}

    # end to end through the public API with host buffers: each step uploads
    # the world state (A, V, GA, SUM) from pinned host memory, steps, and reads
    # the new state back
    host = {name: torch.empty(w.field_size(name), dtype=torch.float32).pin_memory()
            for name in ("A", "V", "GA", "SUM")}
    for name, t in host.items():
        w.get(name, out=t.numpy())
    e2e_steps = max(3, min(args.steps // 10, 50))
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        for name, t in host.items():
            w.set(name, t.numpy())
        w.step(1)
        for name, t in host.items():
            w.get(name, out=t.numpy())
    f1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    h2d = sum(t.numel() * 4 for t in host.values())
    e2e = {"value": n * N * C * e2e_steps / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": h2d}

    # marching cubes of the final grid, every channel at the reference's iso
    # value, two slabs with a shared vertex map as the reference meshes; each
    # mesh includes the one host synchronisation that sizes its output
    from lenia_b200.mesh import Mesher
    A_dev = torch.empty(C * N, dtype=torch.float32, device="cuda")
    w.get("A", out=A_dev)
    mesher = Mesher(wl.desc.width, wl.desc.height, C, iso_value=wl.desc.iso_value, slabs=2, share_channels=True)
    for _ in range(3):
        mesher.run(A_dev, stream=stream.cuda_stream)
    mesh_runs = 10
    barrier()
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0.record(stream)
    for _ in range(mesh_runs):
        mesher.run(A_dev, stream=stream.cuda_stream)
    m1.record(stream)
    barrier()
    mesh_ms = m0.elapsed_time(m1) / mesh_runs
    mesh = {"ms_per_mesh": mesh_ms, "cubes_per_s": C * N / (mesh_ms / 1000.0),
            "vertices": mesher.n_vertices, "triangles": mesher.n_triangles, "gpu_launches_per_mesh": 6}
    mesher.close()

    # config 1's schedule: 500 steps with mesh snapshots, the grid of every
    # channel meshed at the reference's iso value every 10 steps (view
    # NORMAL, as the reference meshes its snapshot)
    sched_steps, sched_every = (500, 10) if args.steps >= 500 else (50, 10)
    ws = World(wl.desc, wl.kernels)
    ws.set_conv_mode(tuning["conv_mode"])
    ws.set_tuning(tuning["row_tile"], tuning["growth_split"])
    ws.set_stream(stream.cuda_stream)
    ws.set_snapshots(True)
    ws.set_state(wl.A0.ravel())
    smesh = Mesher.for_view("NORMAL", wl.desc.width, wl.desc.height, C, iso_value=wl.desc.iso_value)
    barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    tri = 0
    for i in range(sched_steps // sched_every):
        ws.step(sched_every)
        tri += smesh.run_world(ws, "NORMAL")[1]
    s1.record(stream)
    barrier()
    sched_ms = max_over_ranks(s0.elapsed_time(s1))
    schedule = {"steps": sched_steps, "mesh_every": sched_every, "ms": sched_ms,
                "ms_per_step_with_meshing": sched_ms / sched_steps, "triangles_total": int(tri)}
    smesh.close()
    ws.close()

    # config 1's other reintegration: the same world with advection (semi-
    # Lagrangian pull of every channel, reintegration.cpp:1112-1260), tuned
    # and timed the same way
    adv = None
    if args.mode == "rt":
        from lenia_b200 import params as P
        wa = P.config1(seed=1 + rank, width=args.width, mode=P.MODE_ADV)
        wv = World(wa.desc, wa.kernels)
        wv.set_stream(stream.cuda_stream)
        wv.set_state(wa.A0.ravel())
        atune = wv.autotune() if args.growth == "auto" else None
        wv.step(args.warmup)
        adv_steps = max(10, min(args.steps, 200))
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        wv.step(adv_steps)
        a1.record(stream)
        barrier()
        adv_ms = max_over_ranks(a0.elapsed_time(a1))
        wv.close()
        adv = {"workload": config_dict(argparse.Namespace(mode="adv"), wa, n)["workload"],
               "value": n * N * C * adv_steps / (adv_ms / 1000.0), "unit": UNIT, "steps": adv_steps,
               "ms_per_step": adv_ms / adv_steps, "tuning": atune}

    batched = batch_measure(args, rank, n, stream, barrier, max_over_ranks) if args.batch_worlds > 0 else None
    conv = conv_measure(args) if (args.conv_width > 0 and n == 1) else None

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": dict(config_dict(args, wl, n), tuning=tuning),
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "roofline": {"bound": "hbm", "kernel": top_name, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": ncu_traffic(top_name),
                         "algorithmic_bytes_per_launch": (kb[top_name] * prof_steps / top_n
                                                          if top_name in kb else None),
                         "launches_per_step": top_n / prof_steps},
            "step_roofline": {"bytes_per_cell": step_bytes_per_cell(wl),
                              "achieved": step_bytes_per_cell(wl) * N * args.steps / (ms / 1000.0) / 1e9,
                              "peak": peak, "unit": "GB/s",
                              "frac": step_bytes_per_cell(wl) * N * args.steps / (ms / 1000.0) / 1e9 / peak},
            "kernels": kernels_table,
            "mesh": mesh,
            "config1_schedule": schedule,
        }
        if adv is not None:
            line["advection"] = adv
        if batched is not None:
            line["batched"] = batched
        if conv is not None:
            line["conv_modes"] = conv
        if n == 1 and not args.no_cpu_baseline:
            rate, dt = cpu_port_rate(wl, 2, 1)
            port = {"value": rate, "unit": UNIT, "cores": cpu_threads(), "kind": "port",
                    "sample": "2 timed steps (+1 warm-up) of the same world, C restatement of the reference "
                              "step (complex-to-complex FFT structure), OpenMP over all host threads"}
            path = reference_lib(wl)
            if path is not None:
                rrate, rdt, rsteps = cpu_reference_rate(wl, path, 3, 1, 30.0)
                line["cpu_baseline"] = {
                    "value": rrate, "unit": UNIT, "cores": 2, "kind": "reference",
                    "sample": f"{rsteps} timed steps (+1 warm-up) of the same world: the reference's own step "
                              "code built at this size, its two sim threads (slabs of every event at once); a "
                              "project FFT stands in for FFTW"}
                line["cpu_port"] = port
            else:
                line["cpu_baseline"] = port
    w.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        emit(line, args)
    return 0


def emit(line: dict, args) -> None:
    """Prints the result line; with --jsonl also appends it, time-stamped, to
    that file (one JSON object per run)."""
    print(json.dumps(line), flush=True)
    if args.jsonl:
        import datetime
        rec = dict(line, time=datetime.datetime.now(datetime.timezone.utc).isoformat(timespec="seconds"))
        with open(args.jsonl, "a") as f:
            f.write(json.dumps(rec) + "\n")


def main():
    args = parse()
    # `--gpus N` started as one process: launch N ranks (one per GPU) of this
    # script under torch.distributed.run and return their exit code
    from lenia_b200.launch import maybe_spawn
    rc = maybe_spawn(os.path.abspath(__file__), sys.argv[1:], args.gpus)
    if rc is not None:
        return rc
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
