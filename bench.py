#!/usr/bin/env python
"""Benchmark: batched FP32 complex-to-complex forward FFT throughput on one B200 (or N replicas).

Workload ("large and mixed-radix 1D FP32"): forward C2C at N in {4096, 65536, 2^20, 107520 = 3*5*7*2^10}, each with
the batch that fills 2 GiB of complex64 input (65536 / 4096 / 256 / 2496 transforms), inputs uniform[-1, 1) from a
seed, out of place. One step = one forward execute of each of the four batches (8 GiB read, 8 GiB written).
Metric: GFLOP/s by the 5 N log2 N convention, whole job (all ranks); inputs are 2 GiB per size, far above the
126 MB L2, so no flush is needed between iterations.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). ``--impl reference`` times the reference's own CPU crd-hesap-fft (compiled from its
sources into oracle/_ref/libcrdref.so) on this host's cores over a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SIZES = [(4096, 65536), (65536, 4096), (1 << 20, 256), (107520, 2496)]
WORKLOAD = "c2c_fwd_fp32_2GiB_each_N4096_65536_1048576_107520"
METRIC = "batched C2C GFLOP/s & %HBM roofline: TC split-BF16 vs plain FP32 @ rel-L2<=1e-6"
SEED = 0x5EED0002


def flops(n: int, batch: int) -> float:
    return 5.0 * n * math.log2(n) * batch


def algorithmic_bytes(n: int, batch: int) -> int:
    return 16 * n * batch  # 8 B read + 8 B written per complex64 point


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic() -> dict:
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd[1:1] = ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ---- the reference's CPU implementation (reference arm and cpu_baseline) -------------------------------------------


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_cpu(steps: int, warmup: int, budget_bytes: int) -> dict:
    """Time the reference's crd-hesap-fft (FftPlan<float> for powers of two, BluesteinPlan<float> for 107520; one
    plan per thread over contiguous ranges, batch_arms.hpp:59-77) on this host, in place, over a sample of each
    size's batch of at most budget_bytes. Returns GFLOP/s over all sizes."""
    import numpy as np

    import oracle  # the CPU checkers: only this leg of the benchmark uses them

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libcrdref.so not built")
    R = oracle.ref()
    threads = host_threads()
    total_flops = 0.0
    total_time = 0.0
    sample = []
    per_size = {}
    for n, batch in SIZES:
        count = max(1, min(batch, budget_bytes // (8 * n)))
        count = max(count, min(batch, threads))
        buf = oracle.lcg_complex64(SEED ^ n, n * count)
        ptr = buf.view(np.float32).ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        rescale = np.float32(1.0 / math.sqrt(n))
        times = []
        for it in range(warmup + steps):
            t0 = time.perf_counter()
            rc = R.crdref_c2c_f32(n, count, ptr, 0, threads)
            dt = time.perf_counter() - t0
            if rc != 0:
                raise RuntimeError(f"crdref_c2c_f32 failed for n={n}")
            buf *= rescale  # untimed: keeps repeated in-place transforms in range
            if it >= warmup:
                times.append(dt)
        t = sum(times)
        total_flops += flops(n, count) * len(times)
        total_time += t
        per_size[str(n)] = round(flops(n, count) * len(times) / t / 1e9, 2)
        sample.append(f"N={n} x{count} transforms x{len(times)} passes")
    return {
        "value": total_flops / total_time / 1e9,
        "cores": threads,
        "level": int(R.crdref_level()),
        "algorithms": {str(n): R.crdref_plan_algorithm_f32(n).decode() for n, _ in SIZES},
        "sample": "; ".join(sample) + f"; {threads} threads, one plan each, in place",
        "per_size_gflops": per_size,
        "seconds": total_time,
    }


def run_reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    res = reference_cpu(args.steps, args.warmup, budget_bytes=1 << 30)
    value = res["value"]
    ms_per_step = res["seconds"] / args.steps * 1e3
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "GFLOP/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sizes": [[n, b] for n, b in SIZES], "direction": "forward",
                   "l2": "per-size batches of 2 GiB (sampled to <= 1 GiB here)", "parallelism": "host threads"},
        "cpu_baseline": {"value": round(value, 2), "unit": "GFLOP/s", "cores": res["cores"], "kind": "reference",
                         "sample": res["sample"], "level": res["level"], "algorithms": res["algorithms"],
                         "per_size_gflops": res["per_size_gflops"]},
        "e2e": {"value": round(value, 2), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm ---------------------------------------------------------------------------------------------------


def run_ours(args) -> None:
    import numpy as np
    import torch
    import torch.distributed as dist

    import crd_b200 as cf

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    import crd_b200.hesap as F

    if args.wisdom and os.path.exists(args.wisdom):
        with open(args.wisdom) as f:
            F.wisdom_import(f.read())
    F.set_planner(args.planner)

    # One 2 GiB input (uniform[-1,1) from the seed, every size views it as its own batch) and one 2 GiB output.
    max_pts = max(n * b for n, b in SIZES)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + rank)
    xin = (torch.rand(2 * max_pts, generator=gen, device=dev, dtype=torch.float32) * 2 - 1).view(torch.complex64)
    xout = torch.empty(max_pts, dtype=torch.complex64, device=dev)
    plans = []
    for n, b in SIZES:
        p = cf.Plan([n], batch=b)
        plans.append(p)
    launches_per_step = sum(p.info()["passes"] for p in plans)
    if args.planner_log and rank == 0:
        with open(args.planner_log, "w") as f:
            f.write(F.planner_log())
        with open(args.planner_log + ".wisdom", "w") as f:
            f.write(F.wisdom_export())
    stream = torch.cuda.current_stream()

    def step(events=None):
        for i, ((n, b), p) in enumerate(zip(SIZES, plans)):
            if events is not None:
                events[i][0].record(stream)
            p.execute(xin[: n * b], xout[: n * b], cf.FORWARD)
            if events is not None:
                events[i][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    gpu_id = None
    try:
        props = torch.cuda.get_device_properties(dev)
        gpu_id = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
    except Exception:
        gpu_id = None
    sampler = ClockSampler(gpu_id)
    sampler.start()
    time.sleep(0.3)

    ev = [[[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] for _ in SIZES]
          for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    t_start.record(stream)
    for k in range(args.steps):
        step(ev[k])
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()

    total_ms = max_over_ranks(t_start.elapsed_time(t_end))
    per_size_ms = [sum(ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(args.steps)) / args.steps
                   for i in range(len(SIZES))]
    step_flops = sum(flops(n, b) for n, b in SIZES)
    value = step_flops * args.steps * world / (total_ms / 1e3) / 1e9
    ms_per_step = total_ms / args.steps

    # Accuracy of the measured outputs: transform 0 and the last of each size against numpy's float64 FFT.
    rel = {}
    for (n, b), p in zip(SIZES, plans):
        p.execute(xin[: n * b], xout[: n * b], cf.FORWARD)
        torch.cuda.synchronize()
        worst = 0.0
        for t in (0, b - 1):
            x = xin[t * n:(t + 1) * n].cpu().numpy().astype(np.complex128)
            y = xout[t * n:(t + 1) * n].cpu().numpy().astype(np.complex128)
            want = np.fft.fft(x)
            worst = max(worst, float(np.linalg.norm(y - want) / np.linalg.norm(want)))
        rel[str(n)] = worst

    peaks = measured_peaks()
    # Dominant kernel: the N=4096 single-pass line FFT (one launch moves its whole 2 GiB batch in and out).
    i4096 = 0
    dom_bytes = algorithmic_bytes(*SIZES[i4096])
    dom_ms = per_size_ms[i4096] / max(1, plans[i4096].info()["passes"])
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = profiled_traffic().get("line_fft_4096_bytes_per_launch")
    per_size = {}
    for (n, b), p, ms in zip(SIZES, plans, per_size_ms):
        gbs = algorithmic_bytes(n, b) / (ms / 1e3) / 1e9
        per_size[str(n)] = {
            "batch": b,
            "algorithm": p.info()["algorithm"],
            "launches": p.info()["passes"],
            "ms": round(ms, 4),
            "gflops": round(flops(n, b) / (ms / 1e3) / 1e9, 1),
            "hbm_gbs": round(gbs, 1),
            "hbm_frac": round(gbs / peaks["hbm_gbs"], 4),
            "rel_l2_vs_fp64": rel[str(n)],
        }

    # End to end through the public API with host buffers: every step copies each size's 2 GiB input from pinned
    # host memory, transforms it, and copies the 2 GiB spectrum back.
    e2e = None
    if not args.no_e2e:
        hin = torch.empty(max_pts, dtype=torch.complex64, pin_memory=True)
        hin.copy_(xin)
        hout = torch.empty(max_pts, dtype=torch.complex64, pin_memory=True)
        e_steps = max(1, min(args.steps, 3))

        def e2e_step():
            for (n, b), p in zip(SIZES, plans):
                xin[: n * b].copy_(hin[: n * b], non_blocking=True)
                p.execute(xin[: n * b], xout[: n * b], cf.FORWARD)
                hout[: n * b].copy_(xout[: n * b], non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e_steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(e0.elapsed_time(e1))
        bytes_moved = sum(8 * n * b for n, b in SIZES)
        e2e = {"value": round(step_flops * e_steps * world / (e_ms / 1e3) / 1e9, 2), "unit": "GFLOP/s",
               "h2d_bytes_per_step": bytes_moved, "d2h_bytes_per_step": bytes_moved, "steps": e_steps,
               "ms_per_step": round(e_ms / e_steps, 3)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            res = reference_cpu(steps=2, warmup=1, budget_bytes=256 << 20)
            cpu = {"value": round(res["value"], 2), "unit": "GFLOP/s", "cores": res["cores"], "kind": "reference",
                   "sample": res["sample"], "level": res["level"], "per_size_gflops": res["per_size_gflops"]}
        except Exception as exc:  # the GPU number stands; say why the baseline is missing
            cpu = {"value": None, "unit": "GFLOP/s", "cores": host_threads(), "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(value, 2),
            "unit": "GFLOP/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "sizes": [[n, b] for n, b in SIZES], "direction": "forward",
                       "precision": "fp32", "placement": "out-of-place", "planner": args.planner,
                       "l2": "inputs 2 GiB per size (> 126 MB L2), no flush needed",
                       "parallelism": f"replicas{world}"},
            "roofline": {"bound": "hbm", "kernel": "line_fft_kernel N=4096 single pass",
                         "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peaks["source"],
                         "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes},
            "hbm_frac_step": round(sum(algorithmic_bytes(n, b) for n, b in SIZES) / (ms_per_step / 1e3) / 1e9
                                   / peaks["hbm_gbs"], 4),
            "per_size": per_size,
            "rel_l2_vs_fp64_max": max(rel.values()),
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clocks,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--planner", choices=["estimate", "measure"], default="measure",
                    help="measure: time each pass's candidate launch shapes at plan creation (outside the timed "
                         "region) and keep the fastest")
    ap.add_argument("--wisdom", default=os.path.join(ROOT, "profiles", "wisdom_b200.txt"),
                    help="planner wisdom to load first (if the file exists)")
    ap.add_argument("--planner-log", default=None, help="write the planner's timing log here")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
