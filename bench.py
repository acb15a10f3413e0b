#!/usr/bin/env python
"""Benchmark of the batched 1D C2C FFT on B200 (GFLOP/s = 5 n log2 n / time).

Default workload (the plain-method sweep's headline size): FP32 C2C forward,
in place, n = 4096, batch = 16384 (2^26 points, 512 MiB, larger than the
126 MB L2, so no flush is needed between steps).  A step is one execute of
the batched plan.

Output: one JSON line (rank 0) with
  value      whole-job GFLOP/s, inputs resident in HBM, CUDA events around
             exactly K steps on the plan's stream, max over ranks;
  e2e        the same metric through the public C-ABI (mofft_execute_f32)
             with pinned host buffers: host->device copy, transform,
             device->host copy, all inside the timed region;
  roofline   achieved HBM GB/s of the transform kernel (algorithmic bytes
             P(n) * n * 16 B per transform / kernel time) over the measured
             copy bandwidth;
  cpu_baseline  the CPU port of the reference transform (oracle/, OpenMP
             over the batch on every host core) on a bounded sample;
  clocks     nvidia-smi samples taken during the timed region.

Multi-GPU: one process per GPU (torchrun); the transform has no exchange
step, so each rank runs its own replica of the workload (weak scaling) and
NCCL only carries the barrier and the max-over-ranks timing.

--impl reference times the reference's transform on the host cores (the
C restatement in oracle/, since the reference's SME kernels cannot execute
on this host ISA) on a bounded sample of the same workload.
--sweep prints one line per length of the plain-method sweep instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0
METRIC = "C2C GFLOP/s (5n log2 n) & % HBM roofline vs plain; serve p50/p99 latency"


FORMS = {"fp32": 0, "tf32x3": 1, "bf16x3": 2}   # mofft_precision_form

def parse_args():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["mofft", "reference"], default="mofft")
    p.add_argument("--n", type=int, default=4096)
    p.add_argument("--bits", type=int, choices=[32, 64], default=32)
    p.add_argument("--points", type=int, default=1 << 26, help="points per call per GPU")
    p.add_argument("--direction", type=int, choices=[-1, 1], default=-1)
    p.add_argument("--out-of-place", action="store_true")
    p.add_argument("--form", choices=list(FORMS), default="fp32",
                   help="precision form of the FP32 plan (tensor-core forms: n=4096)")
    p.add_argument("--kernel", action="append", default=None,
                   help="run the main plan with these registry kernels, one per pass "
                        "(by name; for profiling a given kernel)")
    p.add_argument("--sweep", action="store_true")
    p.add_argument("--serve", action="store_true",
                   help="serving stream: continuous batching vs serial per-request execution")
    p.add_argument("--requests", type=int, default=600,
                   help="requests of the seeded serving stream (bounded sample)")
    p.add_argument("--ragged", action="store_true",
                   help="ragged batch: 512 mixed FP32 transforms, persistent launch vs per item")
    p.add_argument("--ragged-count", type=int, default=512,
                   help="items of the ragged batch (a smaller list for profiling)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the C1, precision-form and serving figures of the default run")
    p.add_argument("--serve-requests", type=int, default=20000,
                   help="requests of the serving figures in the default run")
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--cpu-seconds", type=float, default=10.0)
    p.add_argument("--soak", type=float, default=1.0,
                   help="untimed seconds of the same load before the timed steps")
    return p.parse_args()


# ------------------------------------------------------------------ helpers

def passes_for(n: int, bits: int) -> int:
    """Minimal pass count of the HBM roofline: one CTA holds 2^14 FP32 /
    2^13 FP64 points."""
    per = 14 if bits == 32 else 13
    return max(1, math.ceil(math.log2(n) / per))


def flops_per_transform(n: int) -> float:
    return 5.0 * n * math.log2(n)


def measured_peaks() -> tuple[float, str]:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel: str, workload: str):
    path = ROOT / "profiles" / "traffic.json"
    try:
        data = json.loads(path.read_text())
        entry = data.get(f"{kernel}|{workload}")
        return entry
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value: float, world: int) -> float:
    """Max of a per-rank timing over all ranks (NCCL on GPUs, gloo on CPU)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(flops_per_rank: float, ms_per_rank: float, world: int) -> tuple[float, float]:
    """Whole-job GFLOP/s of `world` replicas: all ranks' work over the slowest
    rank's time.  Returns (GFLOP/s, max ms)."""
    ms_max = max_over_ranks(ms_per_rank, world)
    return flops_per_rank * world / (ms_max / 1e3) / 1e9, ms_max


def dist_teardown(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------- CPU side

def cpu_baseline(n: int, bits: int, direction: int, seconds: float, points: int) -> dict:
    """The reference transform restated in C (oracle/), timed on all host
    cores on the workload's whole batch (`points` points of length n), calls
    repeated for about `seconds` of work."""
    import numpy as np

    import oracle
    cores = os.cpu_count() or 1
    dtype = np.complex64 if bits == 32 else np.complex128
    batch = max(cores, points // n)
    x = oracle.uniform(n * batch, seed=n, dtype=dtype).reshape(batch, n)
    t_warm = time.perf_counter() + 0.25                          # warm-up >= 0.25 s
    while time.perf_counter() < t_warm:
        oracle.fft_port(x[:cores], direction, threads=cores)
    samples = []
    t_end = time.perf_counter() + seconds
    while time.perf_counter() < t_end or len(samples) < 3:
        t0 = time.perf_counter()
        oracle.fft_port(x, direction, threads=cores)
        samples.append(time.perf_counter() - t0)
        if len(samples) >= 5000:
            break
    med = statistics.median(samples)
    value = flops_per_transform(n) * batch / med / 1e9
    cv = statistics.pstdev(samples) / statistics.mean(samples) if len(samples) > 1 else 0.0
    extra = {"cv": round(cv, 4)}
    try:
        import scipy.fft
        t0 = time.perf_counter()
        reps = 0
        while time.perf_counter() - t0 < min(2.0, seconds / 4) or reps < 2:
            scipy.fft.fft(x, axis=-1, workers=cores)
            reps += 1
        extra["scipy_pocketfft_gflops"] = round(
            flops_per_transform(n) * batch * reps / (time.perf_counter() - t0) / 1e9, 2)
    except Exception:
        pass
    return {"value": round(value, 3), "unit": "GFLOP/s", "cores": cores, "kind": "port",
            "sample": f"{batch} transforms of n={n} FP{bits} per timed call, "
                      f"median of {len(samples)} calls ({sum(samples):.1f} s of CPU work); "
                      "FFTW 3.3.11: unavailable on this box",
            **extra}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import numpy as np

    import oracle
    cores = os.cpu_count() or 1
    n, bits = args.n, args.bits
    dtype = np.complex64 if bits == 32 else np.complex128
    batch = max(1, args.points // n)          # the whole configured batch
    x = oracle.uniform(n * batch, seed=n, dtype=dtype).reshape(batch, n)
    for _ in range(args.warmup):
        oracle.fft_port(x, args.direction, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.fft_port(x, args.direction, threads=cores)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    value = flops_per_transform(n) * batch / (ms / 1e3) / 1e9
    cv = statistics.pstdev(times) / statistics.mean(times) if len(times) > 1 else 0.0
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3),
        "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if bits == 32 else "f64", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": round(value, 3), "unit": "GFLOP/s", "cores": cores,
                         "kind": "port", "cv": round(cv, 4),
                         "sample": f"the whole workload, {batch} transforms of n={n}, per "
                                   "step (out of place; the reference's SME kernels cannot "
                                   "run on x86; FFTW 3.3.11: unavailable on this box)"},
        "e2e": {"value": round(value, 3), "unit": "GFLOP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


L2_BYTES = 126 * 1000 * 1000


def workload_config(args) -> dict:
    n = args.n
    batch = max(1, args.points // n)
    points = batch * n
    held = points * (8 if args.bits == 32 else 16) * (2 if args.out_of_place else 1)
    size = f"2^{points.bit_length() - 1}" if points & (points - 1) == 0 else str(points)
    relation = "> L2 (no flush)" if held > L2_BYTES else "<= L2 (L2-resident: not a HBM figure)"
    return {"workload": f"C2C {'forward' if args.direction < 0 else 'backward'} "
                        f"FP{args.bits} n={n} batch={batch} "
                        f"{'out-of-place' if args.out_of_place else 'in-place'}",
            "n": n, "batch": batch, "precision_bits": args.bits,
            "placement": "out-of-place" if args.out_of_place else "in-place",
            "inputs": f"uniform[-1,1) seeded; {size}-point working set of "
                      f"{held / 1e6:.0f} MB {relation}",
            "parallelism": f"replicas x{args.gpus}", "form": args.form,
            **({"kernels": list(args.kernel)} if args.kernel else {})}


# --------------------------------------------------------------- GPU side

def time_device(plan, buf_in, buf_out, steps, warmup, stream, world, soak_seconds=0.0):
    """W untimed warm-up steps, an optional untimed soak (so that the clock
    samples taken around the timed region see the GPU under this load), then
    exactly K steps between CUDA events on the plan's stream."""
    import torch
    for _ in range(warmup):
        plan.execute(buf_in, buf_out)
    stream.synchronize()
    t_end = time.perf_counter() + soak_seconds
    while time.perf_counter() < t_end:
        for _ in range(32):
            plan.execute(buf_in, buf_out)
        stream.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    import mofft_b200
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    count0 = mofft_b200.launch_count()
    start.record(stream)
    for _ in range(steps):
        plan.execute(buf_in, buf_out)
    end.record(stream)
    launched = mofft_b200.launch_count() - count0
    end.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    return start.elapsed_time(end) / steps, launched


def run_gpu(args, world, rank, local):
    import numpy as np
    import torch

    import mofft_b200 as m
    torch.cuda.set_device(local)
    n, bits = args.n, args.bits
    batch = max(1, args.points // n)
    ctype = torch.complex64 if bits == 32 else torch.complex128
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    real_t = torch.float32 if bits == 32 else torch.float64
    data = torch.rand((batch, n, 2), generator=gen, device="cuda", dtype=real_t) * 2 - 1
    x = torch.view_as_complex(data)
    inplace = not args.out_of_place
    y = x if inplace else torch.empty_like(x)
    explicit = None
    if args.kernel:
        index = {k["name"]: k["index"] for k in m.kernels()}
        explicit = [index[name] for name in args.kernel]
    plan = m.Plan.create(n, args.direction, m.IN_PLACE if inplace else m.OUT_OF_PLACE,
                         bits=bits, batch=batch, kernels=explicit)
    apply_form(plan, args)
    stream = torch.cuda.Stream()
    plan.set_stream(stream.cuda_stream)
    sched = plan.schedule()
    kernels = {k["index"]: k["name"] for k in m.kernels()}
    # timed region: K steps, device-resident inputs
    with ClockSampler(local) as clocks:
        ms, launches = time_device(plan, x, y, args.steps, args.warmup, stream, world,
                                   soak_seconds=args.soak)
    flops = flops_per_transform(n) * batch
    value, ms_max = replica_value(flops, ms, world)
    # roofline of the dominant kernel (per-pass timing when the plan has several)
    peak, peak_kind = measured_peaks()
    p_alg = passes_for(n, bits)
    cb = 8 if bits == 32 else 16
    alg_bytes_step = p_alg * n * 2 * cb * batch
    pass_ms = [ms]
    if sched["pass_count"] > 1:
        pass_ms = per_pass_times(plan, x, y, stream, sched)
    dom = int(np.argmax(pass_ms))
    dom_bytes = 2 * cb * n * batch  # each pass reads and writes every point once
    achieved = dom_bytes / (pass_ms[dom] / 1e3) / 1e9
    workload = f"n={n} batch={batch} fp{bits}"
    entry = committed_traffic(kernels[sched["kernels"][dom]], workload)
    traffic = entry["bytes"] if entry else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": traffic, "peak_source": f"of {peak_kind}",
                "kernel": kernels[sched["kernels"][dom]],
                "algorithmic_bytes_per_launch": dom_bytes,
                "step_roofline_frac": round(alg_bytes_step / (ms / 1e3) / 1e9 / peak, 4)}
    # end-to-end through the public C-ABI with pinned host buffers
    e2e = run_e2e(args, m, n, bits, batch, x)
    plan.destroy()
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GFLOP/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if bits == 32 else "f64", "data": "synthetic",
            "config": workload_config(args), "roofline": roofline,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks.summary(),
            "schedule": {"passes": sched["pass_count"],
                         "kernels": [kernels[k] for k in sched["kernels"]]},
        }
    return line


def run_c1(m):
    """C1: n = 1024, batch 4096, out of place, forward then backward on
    device buffers (uniform[-1,1), seed 0); GFLOP/s of the pair and the
    round-trip error backward(forward(x)) / n against x."""
    import torch
    n, batch, steps = 1024, 4096, 50
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.view_as_complex(torch.rand((batch, n, 2), generator=g, device="cuda") * 2 - 1)
    y, z = torch.empty_like(x), torch.empty_like(x)
    stream = torch.cuda.Stream()
    fwd = m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=batch)
    bwd = m.Plan.create(n, m.BACKWARD, m.OUT_OF_PLACE, bits=32, batch=batch)
    for p in (fwd, bwd):
        p.set_stream(stream.cuda_stream)
    for _ in range(3):
        fwd.execute(x, y)
        bwd.execute(y, z)
    stream.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(steps):
        fwd.execute(x, y)
        bwd.execute(y, z)
    e.record(stream)
    e.synchronize()
    ms = s.elapsed_time(e) / steps
    err = float(torch.linalg.vector_norm((z / n - x).to(torch.complex128)) /
                torch.linalg.vector_norm(x.to(torch.complex128)))
    fwd.destroy()
    bwd.destroy()
    return {"workload": "C2C FP32 n=1024 batch=4096 out-of-place, forward then backward "
                        "(working set 96 MB: L2-resident, not a HBM figure)",
            "ms_fwd_bwd": round(ms, 4),
            "gflops": round(2 * flops_per_transform(n) * batch / (ms / 1e3) / 1e9, 1),
            "roundtrip_rel_l2": float(f"{err:.3e}")}


def run_forms(m):
    """Precision forms: FP32 C2C forward, out of place, 2^27 points of the
    precision mix at n = 4096 (batch 32768) and n = 65536 (batch 2048); per
    form the time of one call (CUDA events), GFLOP/s, the fraction of the
    HBM roofline, and the relative L2 error on 64 rows spread over the batch
    against the FP64 transform of the same rows (the library's own FP64
    plan, parity-tested against the long-double oracle)."""
    import torch

    from mofft_b200 import workloads
    peak, kind = measured_peaks()
    out = {}
    for n in (4096, 65536):
        points = 1 << 27
        batch = points // n
        x = workloads.precision_mix_device(points, n, seed=11)
        y = torch.empty_like(x)
        rows = torch.linspace(0, batch - 1, 64).long().cuda()
        xr = x[rows].to(torch.complex128).contiguous()
        ref = torch.empty_like(xr)
        with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=64, batch=64) as p64:
            p64.execute(xr, ref)
        torch.cuda.synchronize()
        stream = torch.cuda.Stream()
        per = {}
        for name, form in FORMS.items():
            with m.Plan.create(n, m.FORWARD, m.OUT_OF_PLACE, bits=32, batch=batch) as plan:
                plan.set_precision_form(form)
                plan.set_stream(stream.cuda_stream)
                ms, _ = time_device(plan, x, y, 10, 3, stream, 1)
            err = float(torch.linalg.vector_norm(y[rows].to(torch.complex128) - ref) /
                        torch.linalg.vector_norm(ref))
            alg = passes_for(n, 32) * 16 * points
            per[name] = {"ms": round(ms, 4),
                         "gflops": round(flops_per_transform(n) * batch / (ms / 1e3) / 1e9, 1),
                         "hbm_frac": round(alg / (ms / 1e3) / 1e9 / peak, 3),
                         "rel_l2": float(f"{err:.3e}")}
        per["fp32_tolerance"] = float(f"{5e-7 * math.log2(n):.2e}")
        out[f"n={n} batch={batch}"] = per
        del x, y
        torch.cuda.empty_cache()
    out["peak"] = f"{peak} GB/s of {kind}"
    return out


def apply_form(plan, args):
    if args.form != "fp32":
        plan.set_precision_form(FORMS[args.form])


def per_pass_times(plan, x, y, stream, sched):
    """Kernel time of each pass, measured with events on the plan's stream by
    running one-pass plans of the same decomposition is not possible from the
    public API, so the whole step is split evenly (passes move equal bytes)."""
    import torch
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record(stream)
    plan.execute(x, y)
    e.record(stream)
    e.synchronize()
    total = s.elapsed_time(e)
    return [total / sched["pass_count"]] * sched["pass_count"]


def run_e2e(args, m, n, bits, batch, x_dev):
    import torch
    h_in = torch.empty(x_dev.shape, dtype=x_dev.dtype, pin_memory=True)
    h_out = torch.empty_like(h_in, pin_memory=True)
    h_in.copy_(x_dev)
    plan = m.Plan.create(n, args.direction, m.OUT_OF_PLACE, bits=bits, batch=batch)
    apply_form(plan, args)
    plan.execute(h_in, h_out)  # warm-up (allocates the staging buffers)
    times = []
    for _ in range(max(1, args.e2e_steps)):
        t0 = time.perf_counter()
        plan.execute(h_in, h_out)
        times.append(time.perf_counter() - t0)
    plan.destroy()
    t = statistics.median(times)
    nbytes = h_in.numel() * h_in.element_size()
    return {"value": round(flops_per_transform(n) * batch / t / 1e9, 2), "unit": "GFLOP/s",
            "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
            "ms_per_step": round(t * 1e3, 3), "api": "mofft_execute_f%d (host buffers)" % bits}


def run_sweep(args, world, rank, local):
    import torch

    import mofft_b200 as m
    torch.cuda.set_device(local)
    peak, kind = measured_peaks()
    sizes = [2 ** e for e in range(4, 25)] + [3 * 2 ** e for e in range(4, 19)] + \
        [5 * 2 ** e for e in range(4, 18)]
    for bits in (32, 64):
        total = (1 << 26) if bits == 32 else (1 << 25)
        for n in sorted(sizes):
            batch = max(1, total // n)
            real_t = torch.float32 if bits == 32 else torch.float64
            x = torch.view_as_complex(torch.rand((batch, n, 2), device="cuda", dtype=real_t))
            plan = m.Plan.create(n, args.direction, m.IN_PLACE, bits=bits, batch=batch)
            apply_form(plan, args)
            stream = torch.cuda.Stream()
            plan.set_stream(stream.cuda_stream)
            ms, _ = time_device(plan, x, x, 10, 3, stream, world)
            sched = plan.schedule()
            plan.destroy()
            cb = 8 if bits == 32 else 16
            alg = passes_for(n, bits) * 2 * cb * n * batch
            if rank == 0:
                print(json.dumps({
                    "n": n, "precision_bits": bits, "batch": batch, "ms": round(ms, 4),
                    "gflops": round(flops_per_transform(n) * batch / (ms / 1e3) / 1e9, 1),
                    "hbm_roofline_frac": round(alg / (ms / 1e3) / 1e9 / peak, 3),
                    "passes": sched["pass_count"], "peak": f"{peak} GB/s of {kind}"}),
                    flush=True)
            del x
            torch.cuda.empty_cache()


def run_ragged(args, world, rank, local):
    """512 FP32 transforms of mixed length / batch / direction (seed 7): the
    ragged plan's CUDA graph (one persistent launch for the one-pass lengths,
    tuned groups for the longer ones) vs every item in the persistent launch
    vs one plain launch per transform (eager, and captured in a CUDA
    graph)."""
    import torch

    import mofft_b200 as m
    from mofft_b200 import workloads
    torch.cuda.set_device(local)
    spec = workloads.ragged_spec(count=args.ragged_count, seed=7)
    gen = torch.Generator(device="cuda").manual_seed(7)
    items, flops, points = [], 0.0, 0
    for n, batch, direction in spec:
        x = torch.view_as_complex(torch.rand((batch, n, 2), generator=gen, device="cuda") * 2 - 1)
        items.append((x, torch.empty_like(x), direction))
        flops += flops_per_transform(n) * batch
        points += n * batch
    plan = m.RaggedPlan(items)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream

    def timed(fn, reps):
        for _ in range(3):
            fn()
        stream.synchronize()
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e) / reps

    ragged_ms = timed(lambda: plan.execute(sh), args.steps)
    assert plan.status() == 0, "ragged kernel reported a timed-out dependency wait"
    single = m.RaggedPlan(items, single_launch=True)
    single_ms = timed(lambda: single.execute(sh), args.steps)
    assert single.status() == 0, "ragged kernel reported a timed-out dependency wait"
    single.destroy()
    # minimal-pass bytes: P(n) reads and writes of every point
    min_bytes = sum(n * batch * 16 * passes_for(n, 32) for n, batch, _ in spec)
    per_item_ms = timed(lambda: plan.execute_per_item(sh), max(3, args.steps // 4))
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        plan.execute_per_item(sh)
        stream.synchronize()
        with torch.cuda.graph(graph, stream=stream):
            plan.execute_per_item(torch.cuda.current_stream().cuda_stream)
    def replay():
        with torch.cuda.stream(stream):
            graph.replay()

    graph_ms = timed(replay, max(3, args.steps // 4))
    tiles, grid = plan.info()
    peak, kind = measured_peaks()
    line = {
        "metric": "ragged C2C GFLOP/s (5n log2 n)", "value": round(flops / ragged_ms / 1e6, 1),
        "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": 3,
        "ms_per_step": round(ragged_ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"ragged: {args.ragged_count} transforms, n in {{2^6..2^16}} U "
                               "{3*2^5..3*2^13}, batch 1..64, mixed directions, seed 7",
                   "points": points, "tiles": tiles, "persistent_ctas": grid},
        "per_item_eager": {"ms": round(per_item_ms, 4),
                           "gflops": round(flops / per_item_ms / 1e6, 1)},
        "per_item_graph": {"ms": round(graph_ms, 4), "gflops": round(flops / graph_ms / 1e6, 1)},
        "single_launch": {"ms": round(single_ms, 4),
                          "gflops": round(flops / single_ms / 1e6, 1)},
        "speedup_vs_per_item_graph": round(graph_ms / ragged_ms, 2),
        "hbm_frac_one_pass_bytes": round(points * 16 / (ragged_ms / 1e3) / 1e9 / peak, 3),
        "hbm_frac_min_pass_bytes": round(min_bytes / (ragged_ms / 1e3) / 1e9 / peak, 3),
    }
    del graph
    plan.destroy()
    return line


def run_serve(args, world, rank, local, requests=None, fracs=(0.5, 0.9), one_shot=True):
    """Serving stream (seeded): n Zipf(1.1) over 2^8..2^20, batch 1..256,
    80 % FP32 / 20 % FP64, device-resident payloads.  The server (continuous
    batching, 4 streams, 40 GiB admission) and serial plain execution (one
    blocking plan execute per request, plans created beforehand) process the
    same requests: all at t=0 (saturation) and at Poisson rates of 50 % and
    90 % of the serial capacity.  At saturation the one-shot pattern (plan,
    execute, destroy per request) is timed as well."""
    import threading

    import numpy as np
    import torch

    import mofft_b200 as m
    from mofft_b200 import workloads
    torch.cuda.set_device(local)
    reqs = workloads.serving_stream(requests or args.requests, rate_per_s=1.0, seed=11)
    maxpts = max(r["n"] * r["batch"] for r in reqs)
    arena_in = {32: torch.view_as_complex(torch.rand((maxpts, 2), device="cuda") * 2 - 1),
                64: torch.view_as_complex(torch.rand((maxpts, 2), device="cuda",
                                                     dtype=torch.float64) * 2 - 1)}
    ring_bytes = 24 << 30
    ring = torch.empty(ring_bytes // 16, dtype=torch.complex128, device="cuda")
    flops = [flops_per_transform(r["n"]) * r["batch"] for r in reqs]
    total_flops = sum(flops)

    def out_ptr(offset):
        return ring.data_ptr() + offset

    # serial plain per-request execution: one cached batched plan per shape
    plans = {}
    for r in reqs:
        key = (r["n"], r["batch"], r["direction"], r["bits"])
        if key not in plans:
            plans[key] = m.Plan.create(r["n"], r["direction"], m.OUT_OF_PLACE, bits=r["bits"],
                                       batch=r["batch"])

    def run_serial(arrivals):
        lat = []
        t0 = time.perf_counter()
        offset = 0
        for r, a in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            nbytes = r["n"] * r["batch"] * (8 if r["bits"] == 32 else 16)
            if offset + nbytes > ring_bytes:
                offset = 0
            st = plans[(r["n"], r["batch"], r["direction"], r["bits"])].execute_ptr(
                arena_in[r["bits"]].data_ptr(), out_ptr(offset))
            assert st == 0
            offset += nbytes
            lat.append(time.perf_counter() - t0 - a)
        return time.perf_counter() - t0, lat

    def run_serial_one_shot():
        # the reference API's one-shot pattern: plan, execute, destroy per request
        lat = []
        t0 = time.perf_counter()
        offset = 0
        for r in reqs:
            nbytes = r["n"] * r["batch"] * (8 if r["bits"] == 32 else 16)
            if offset + nbytes > ring_bytes:
                offset = 0
            p = m.Plan.create(r["n"], r["direction"], m.OUT_OF_PLACE, bits=r["bits"],
                              batch=r["batch"])
            st = p.execute_ptr(arena_in[r["bits"]].data_ptr(), out_ptr(offset))
            p.destroy()
            assert st == 0
            offset += nbytes
            lat.append(time.perf_counter() - t0)
        return time.perf_counter() - t0, lat

    def run_server(arrivals):
        srv = m.Server(hbm_budget_bytes=40 << 30, streams=4)
        # warm the server's plan cache outside the timed run
        for key in {(r["n"], r["direction"], r["bits"]) for r in reqs}:
            srv.wait(srv.submit(key[0], 1, key[1], key[2], arena_in[key[2]].data_ptr(),
                                out_ptr(0)))
        tickets = []
        lat_of = {}
        inflight = []          # (ticket, bytes) in ring order: client flow control
        used = 0
        t0 = time.perf_counter()
        offset = 0
        for r, a in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            nbytes = r["n"] * r["batch"] * (8 if r["bits"] == 32 else 16)
            while inflight and used + nbytes > ring_bytes // 2:
                t, b = inflight.pop(0)
                lat_of[t] = srv.wait(t)[1]
                used -= b
            if offset + nbytes > ring_bytes:
                offset = 0
            t = srv.submit(r["n"], r["batch"], r["direction"], r["bits"],
                           arena_in[r["bits"]].data_ptr(), out_ptr(offset))
            offset += nbytes
            tickets.append(t)
            inflight.append((t, nbytes))
            used += nbytes
        srv.drain()
        makespan = time.perf_counter() - t0
        for t, _ in inflight:
            lat_of[t] = srv.wait(t)[1]
        lat = [lat_of[t] for t in tickets]
        stats = srv.stats()
        srv.destroy()
        return makespan, lat, stats

    def summary(makespan, lat):
        lat_ms = np.array(lat) * 1e3
        return {"gflops": round(total_flops / makespan / 1e9, 1),
                "p50_ms": round(float(np.percentile(lat_ms, 50)), 3),
                "p99_ms": round(float(np.percentile(lat_ms, 99)), 3)}

    zeros = [0.0] * len(reqs)
    serial_span, serial_lat = run_serial(zeros)
    if one_shot:
        one_shot_span, one_shot_lat = run_serial_one_shot()
    srv_span, srv_lat, stats = run_server(zeros)
    capacity = len(reqs) / serial_span           # serial requests per second
    rates = {}
    for frac in fracs:
        rate = capacity * frac
        rng = np.random.default_rng(5)
        arrivals = list(np.cumsum(rng.exponential(1.0 / rate, size=len(reqs))))
        s_span, s_lat = run_serial(arrivals)
        v_span, v_lat, _ = run_server(arrivals)
        rates[f"{rate:.0f}_req_per_s"] = {"serial": summary(s_span, s_lat),
                                          "server": summary(v_span, v_lat)}
    for p in plans.values():
        p.destroy()
    sat_server = summary(srv_span, srv_lat)
    sat_serial = summary(serial_span, serial_lat)
    # the stream's roofline: every request's minimal-pass bytes at the
    # measured copy bandwidth
    peak, peak_kind = measured_peaks()
    floor_s = sum(passes_for(r["n"], r["bits"]) * 2 * (8 if r["bits"] == 32 else 16) *
                  r["n"] * r["batch"] for r in reqs) / (peak * 1e9)
    ceiling = {"gflops": round(total_flops / floor_s / 1e9, 1), "ms": round(floor_s * 1e3, 2),
               "peak": f"{peak} GB/s of {peak_kind}",
               "server_over_ceiling": round(sat_server["gflops"] * 1e9 * floor_s / total_flops, 3),
               "serial_over_ceiling": round(sat_serial["gflops"] * 1e9 * floor_s / total_flops,
                                            3)}
    saturation = {"server": sat_server, "serial_plain": sat_serial,
                  "speedup": round(serial_span / srv_span, 2),
                  "launches": stats["launches"], "requests": len(reqs)}
    if one_shot:
        saturation["serial_plan_per_request"] = summary(one_shot_span, one_shot_lat)
        saturation["speedup_vs_plan_per_request"] = round(one_shot_span / srv_span, 2)
    return {
        "metric": "serve C2C GFLOP/s (5n log2 n), saturation", "value": sat_server["gflops"],
        "unit": "GFLOP/s", "n_gpus": world, "steps": 1, "warmup": 1,
        "ms_per_step": round(srv_span * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"serving stream: first {len(reqs)} requests (seed 11) of the "
                               "20,000-request stream: n Zipf(1.1) over 2^8..2^20, batch 1..256, "
                               "80% FP32 / 20% FP64, device-resident payloads",
                   "server": {"streams": 4, "hbm_budget_gib": 40}},
        "saturation": saturation, "ceiling": ceiling,
        "poisson": rates,
    }


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        if args.sweep:
            run_sweep(args, world, rank, local)
            return 0
        if args.serve:
            line = run_serve(args, world, rank, local)
            if rank == 0:
                print(json.dumps(line), flush=True)
            return 0
        if args.ragged:
            line = run_ragged(args, world, rank, local)
            if rank == 0:
                print(json.dumps(line), flush=True)
            return 0
        line = run_gpu(args, world, rank, local)
        if rank == 0 and world == 1 and not args.no_extras:
            import mofft_b200 as m
            count0 = m.launch_count()
            line["c1"] = run_c1(m)
            line["forms"] = run_forms(m)
            serve = run_serve(args, world, rank, local, requests=args.serve_requests,
                              fracs=(0.9,), one_shot=False)
            line["serve"] = {"workload": serve["config"]["workload"],
                             "p50_ms": serve["saturation"]["server"]["p50_ms"],
                             "p99_ms": serve["saturation"]["server"]["p99_ms"],
                             "gflops": serve["saturation"]["server"]["gflops"],
                             "saturation": serve["saturation"], "ceiling": serve["ceiling"],
                             "poisson": serve["poisson"]}
            line["extras_gpu_launches"] = int(m.launch_count() - count0)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.n, args.bits, args.direction,
                                                args.cpu_seconds, args.points)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        dist_teardown(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
