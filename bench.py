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


# ---- workloads -------------------------------------------------------------------------------------------------
#
# A workload is a list of ops; one step runs every op once. Each op has a device input and output, a run(in, out)
# that enqueues it on the current stream, its FLOP count (5 N log2 N per complex transform, 2.5 N log2 N per real
# one), its algorithmic HBM bytes, the number of kernel launches it issues, and a check that returns the rel-L2 of
# its output against numpy's float64 FFT on a sample.

WORKLOADS = ("mixed", "n1024", "r2c", "uneven", "nd", "precision", "conv", "welch", "cwt")


WORKLOAD_CONFIGS = {
    "mixed": {"workload": WORKLOAD, "sizes": [[n, b] for n, b in SIZES], "direction": "forward",
              "l2": "inputs 2 GiB per size (> 126 MB L2), no flush needed"},
    "n1024": {"workload": "c2c_fwd_fp32_N1024_batch4096", "sizes": [[1024, 4096]], "direction": "forward",
              "l2": "8 input + 8 output buffers in turn (512 MiB)", "step": "8 executes, one CUDA graph"},
    "r2c": {"workload": "r2c_c2r_fp32_N1048576_batch512", "sizes": [[1 << 20, 512]],
            "l2": "2 GiB real input, no flush needed", "flops": "2.5 N log2 N per real transform"},
    "uneven": {"workload": "uneven_20000_7smooth_16_65536", "transforms": 20000,
               "l2": "about 2.5 GB moved per step (> 126 MB L2)"},
    "nd": {"workload": "nd_c2c_fp32_4096x4096_512x512x512", "inputs": "uniform[-1,1) + 1% x 1e4",
           "l2": "2-D input rotates over 4 buffers (512 MiB); 3-D input 1 GiB"},
    "conv": {"workload": "fused_conv_1d_N256_1024_4096_2^25_points_real_N1024_4096_2^26_points_real2d_4096x4096x4",
             "filter": "one spectrum shared by the batch",
             "l2": "256 MiB input per size (> 126 MB L2)",
             "flops": "complex: 10 N log2 N + 6 N per signal; real: 5 N log2 N + 3 N per signal"},
    "welch": {"workload": "welch_spectrogram_64_signals_2^22_samples_nperseg1024_noverlap512_hann",
              "l2": "1 GiB of float input (> 126 MB L2)", "flops": "2.5 N log2 N per segment (its real FFT)"},
    "cwt": {"workload": "cwt_morl_64_signals_4096_samples_64_scales_1_to_128",
            "l2": "128 MiB of coefficients written per step (> 126 MB L2)",
            "flops": "the work of this path: per signal 5 L log2 L (forward FFT) + nscales (5 L log2 L + 6 L) (spectrum "
                     "product and inverse FFT), L = 8192 (FFT length); the kernel spectra the reference recomputes "
                     "every call are made once at plan time and counted in neither arm",
            "bytes": "algorithmic: the signals read (4 B a sample) and the coefficients written (8 B a scale and sample)"},
    "precision": {"workload": "nd_c2c_4096x4096_512x512x512_fp32_splitbf16_fp16", "inputs": "uniform[-1,1) + 1% x 1e4",
                  "l2": "2-D input rotates over 4 buffers (512 MiB); 3-D input 1 GiB"},
}


class Op:
    def __init__(self, name, inp, out, run, flops_, bytes_, launches, check, info=None, host=None):
        self.name, self.inp, self.out, self.run = name, inp, out, run
        self.flops, self.bytes, self.launches, self.check = flops_, bytes_, launches, check
        self.info = info or {}
        # host(hin, hout): the same op on host buffers through the library's host-memory execute, or None (the
        # end-to-end leg then copies in, runs and copies out itself)
        self.host = host
        # peer: (name, callable) running the vendor library's route for the same op on the same data, timed beside it
        self.peer = None


def _rel(a, b):
    import numpy as np

    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def build_mixed(dev, rank, cf):
    """Large and mixed-radix C2C: forward C2C at N in {4096, 65536, 2^20, 107520}, batch filling 2 GiB."""
    import numpy as np
    import torch

    max_pts = max(n * b for n, b in SIZES)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + rank)
    xin = (torch.rand(2 * max_pts, generator=gen, device=dev, dtype=torch.float32) * 2 - 1).view(torch.complex64)
    xout = torch.empty(max_pts, dtype=torch.complex64, device=dev)
    ops = []
    for n, b in SIZES:
        plan = cf.Plan([n], batch=b)
        info = {"batch": b, "algorithm": plan.info()["algorithm"]}

        def check(n=n, b=b, plan=plan, info=info):
            plan.execute(xin[: n * b], xout[: n * b], cf.FORWARD)  # the output buffer is shared: redo this op
            torch.cuda.synchronize()
            # round trip of the first and last transforms: forward, then inverse scaled by 1/N
            inv = cf.Plan([n], batch=1, norm=cf.NORM_INVERSE)
            back = torch.empty(n, dtype=torch.complex64, device=dev)
            worst, trip = 0.0, 0.0
            for t in (0, b - 1):
                inv.execute(xout[t * n:(t + 1) * n], back, cf.INVERSE)
                torch.cuda.synchronize()
                x = xin[t * n:(t + 1) * n].cpu().numpy()
                y = xout[t * n:(t + 1) * n].cpu().numpy()
                worst = max(worst, _rel(y, np.fft.fft(x.astype(np.complex128))))
                trip = max(trip, _rel(back.cpu().numpy(), x))
            info["round_trip_rel_l2"] = trip
            return worst

        ops.append(Op(str(n), xin[: n * b], xout[: n * b],
                      lambda i, o, plan=plan: plan.execute(i, o, cf.FORWARD), flops(n, b), algorithmic_bytes(n, b),
                      plan.info()["passes"], check, info,
                      host=lambda hi, ho, plan=plan: plan.execute_host(hi, ho, cf.FORWARD)))
    return ops, dict(WORKLOAD_CONFIGS["mixed"])


def build_n1024(dev, rank, cf):
    """Plain batched C2C: forward N = 1024, batch 4096, contiguous (32 MiB in, 32 MiB out per execute). One step runs
    the execute on each of eight input/output buffer pairs in turn (512 MiB, four times the 126 MB L2, so no execute
    finds its input in L2), the eight executes captured once in a CUDA graph: a 20-microsecond transform is
    otherwise paced by the host's launch rate, not the GPU."""
    import numpy as np
    import torch

    n, b, ring = 1024, 4096, 8
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED - 1 + rank)
    xin = (torch.rand(2 * n * b * ring, generator=gen, device=dev, dtype=torch.float32) * 2 - 1).view(torch.complex64)
    xout = torch.empty(n * b * ring, dtype=torch.complex64, device=dev)
    ins = [xin[k * n * b:(k + 1) * n * b] for k in range(ring)]
    outs = [xout[k * n * b:(k + 1) * n * b] for k in range(ring)]
    plan = cf.Plan([n], batch=b)
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for k in range(ring):
            plan.execute(ins[k], outs[k], cf.FORWARD)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for k in range(ring):
            plan.execute(ins[k], outs[k], cf.FORWARD)

    def check():
        plan.execute(ins[0], outs[0], cf.FORWARD)
        torch.cuda.synchronize()
        x = ins[0].view(b, n)[:: b // 8].cpu().numpy().astype(np.complex128)
        return _rel(outs[0].view(b, n)[:: b // 8].cpu().numpy(), np.fft.fft(x, axis=1))

    # host buffers: the eight batches in one call (a plan of 8 x 4096 transforms), so that the chunked copies in
    # both directions stay overlapped from the first batch to the last
    host_plan = cf.Plan([n], batch=b * ring)

    def host(hi, ho):
        host_plan.execute_host(hi, ho, cf.FORWARD)

    op = Op("1024", xin, xout, lambda i, o: graph.replay(), ring * flops(n, b), ring * algorithmic_bytes(n, b),
            ring * plan.info()["passes"], check, {"batch": b, "executes_per_step": ring,
                                                   "algorithm": plan.info()["algorithm"]}, host=host)
    op.keep = graph  # the graph lives as long as the op
    return [op], dict(WORKLOAD_CONFIGS["n1024"])


def build_r2c(dev, rank, cf):
    """Real transforms: R2C and C2R at N = 2^20, batch 512 (2 GiB of real input)."""
    import numpy as np
    import torch

    n, b = 1 << 20, 512
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 7 + rank)
    real = torch.rand(n * b, generator=gen, device=dev, dtype=torch.float32) * 2 - 1
    spec = torch.empty(b * (n // 2 + 1), dtype=torch.complex64, device=dev)
    back = torch.empty(n * b, dtype=torch.float32, device=dev)
    r2c = cf.Plan([n], batch=b, kind=cf.R2C)
    c2r = cf.Plan([n], batch=b, kind=cf.C2R)
    fl = 2.5 * n * math.log2(n) * b
    by = (4 * n + 8 * (n // 2 + 1)) * b

    def check_r2c():
        r2c.execute(real, spec, cf.FORWARD)
        torch.cuda.synchronize()
        x = real[:n].cpu().numpy().astype(np.float64)
        return _rel(spec[: n // 2 + 1].cpu().numpy(), np.fft.rfft(x))

    def check_c2r():
        c2r.execute(spec, back, cf.INVERSE)
        torch.cuda.synchronize()
        s0 = spec[: n // 2 + 1].cpu().numpy().astype(np.complex128)
        return _rel(back[:n].cpu().numpy(), np.fft.irfft(s0, n) * n)

    ops = [Op("r2c", real, spec, lambda i, o: r2c.execute(i, o, cf.FORWARD), fl, by, r2c.info()["passes"],
              check_r2c, {"batch": b, "algorithm": r2c.info()["algorithm"]},
              host=lambda hi, ho: r2c.execute_host(hi, ho, cf.FORWARD)),
           Op("c2r", spec, back, lambda i, o: c2r.execute(i, o, cf.INVERSE), fl, by, c2r.info()["passes"],
              check_c2r, {"batch": b, "algorithm": c2r.info()["algorithm"]},
              host=lambda hi, ho: c2r.execute_host(hi, ho, cf.INVERSE))]
    return ops, dict(WORKLOAD_CONFIGS["r2c"])


def build_uneven(dev, rank, cf):
    """Uneven batch: 20,000 transforms, sizes log-uniform over the 7-smooth integers in [16, 65536], each at
    its own offset of a packed buffer, Gaussian inputs, one persistent graph-captured launch."""
    import numpy as np
    import torch

    from crd_b200.workloads import uneven_sizes

    sizes = uneven_sizes(20000, seed=0x5EED0003)
    plan = cf.UnevenPlan(sizes)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 3 + rank)
    xin = torch.randn(2 * plan.total, generator=gen, device=dev, dtype=torch.float32).view(torch.complex64)
    xout = torch.empty(plan.total, dtype=torch.complex64, device=dev)
    fl = sum(5.0 * s * math.log2(s) for s in sizes)
    by = sum(16 * s for s in sizes)

    def check():
        plan.execute(xin, xout, cf.FORWARD)
        torch.cuda.synchronize()
        worst = 0.0
        x = xin.cpu().numpy()
        y = xout.cpu().numpy()
        for t in range(0, len(sizes), 997):
            n, o = sizes[t], plan.offsets[t]
            worst = max(worst, _rel(y[o:o + n], np.fft.fft(x[o:o + n].astype(np.complex128))))
        return worst

    return [Op("uneven", xin, xout, lambda i, o: plan.execute(i, o, cf.FORWARD), fl, by, 1, check,
               {"transforms": len(sizes), "items": plan.info()["factors"][1], "algorithm": "uneven-batch"})], \
        dict(WORKLOAD_CONFIGS["uneven"], size_classes=len(set(sizes)))


PRECISIONS = {"fp32": 0, "split-bf16": 1, "fp16-scaled": 2, "split-bf16-hilo": 3, "split-fp16-hilo": 4}


def _build_nd_forms(dev, rank, cf, forms, shapes=((4096, 4096), (512, 512, 512))):
    """2-D C2C 4096 x 4096 and 3-D C2C 512^3, uniform[-1,1) plus 1% of entries scaled by 1e4, at each precision form
    in `forms`. Four input buffers of the 2-D shape rotate across steps so its 128 MiB input is not L2-resident."""
    import numpy as np
    import torch

    ops = []
    for dims in shapes:
        nbuf = 4 if len(dims) == 2 else 1
        total = int(np.prod(dims))
        gen = torch.Generator(device=dev)
        gen.manual_seed(SEED + 4 + rank + total)
        bufs = []
        for _ in range(nbuf):
            x = (torch.rand(2 * total, generator=gen, device=dev, dtype=torch.float32) * 2 - 1).view(torch.complex64)
            idx = torch.randperm(total, generator=gen, device=dev)[: total // 100]
            x[idx] *= 1e4
            bufs.append(x)
        out = torch.empty(total, dtype=torch.complex64, device=dev)
        want = {}
        for form in forms:
            plan = cf.Plan(list(dims), batch=1, precision=PRECISIONS[form])
            state = {"k": 0}

            def run(i, o, plan=plan, bufs=bufs, state=state):
                plan.execute(bufs[state["k"] % len(bufs)], o, cf.FORWARD)
                state["k"] += 1

            def check(plan=plan, bufs=bufs, out=out, dims=dims, want=want):
                plan.execute(bufs[0], out, cf.FORWARD)
                torch.cuda.synchronize()
                if "y" not in want:  # the FP64 answer, once per shape
                    want["y"] = np.fft.fftn(bufs[0].cpu().numpy().reshape(dims).astype(np.complex128))
                return _rel(out.cpu().numpy().reshape(dims), want["y"])

            name = "x".join(str(d) for d in dims) + ("" if forms == ("fp32",) else f"/{form}")
            ops.append(Op(name, bufs[0], out, run, 5.0 * total * math.log2(total), 16 * total,
                          plan.info()["passes"], check, {"algorithm": plan.info()["algorithm"], "precision": form}))
    return ops


def build_nd(dev, rank, cf):
    """Multi-dimensional C2C at FP32: 2-D 4096 x 4096 and 3-D 512^3."""
    return _build_nd_forms(dev, rank, cf, ("fp32",)), \
        dict(WORKLOAD_CONFIGS["nd"])


CONV_SIZES = (256, 1024, 4096)
CONV_POINTS = 1 << 25  # per size: 256 MiB of complex64 input (> 126 MB L2)
REAL_CONV_DIMS = ((1024,), (4096,), (4096, 4096))  # real signals, 2^26 points (256 MiB of float32) each


def build_conv(dev, rank, cf):
    """Fused FFT convolution, y = IFFT(FFT(x) * H) / N, batched 1-D at N in {256, 1024, 4096} over 2^25 points each,
    one spectrum shared by the batch; beside it the vendor route (cuFFT through torch.fft: forward FFT, elementwise
    product, inverse FFT: three global passes) on the same buffers."""
    import numpy as np
    import torch

    ops = []
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 11 + rank)
    xin = (torch.rand(2 * CONV_POINTS, generator=gen, device=dev, dtype=torch.float32) * 2 - 1).view(torch.complex64)
    xout = torch.empty(CONV_POINTS, dtype=torch.complex64, device=dev)
    for n in CONV_SIZES:
        b = CONV_POINTS // n
        plan = cf.ConvPlan([n], batch=b)
        H = (torch.rand(2 * n, generator=gen, device=dev, dtype=torch.float32) * 2 - 1).view(torch.complex64)

        def check(n=n, b=b, plan=plan, H=H):
            plan.execute(xin, H, xout)
            torch.cuda.synchronize()
            x = xin.view(b, n)[:: b // 4].cpu().numpy().astype(np.complex128)
            want = np.fft.ifft(np.fft.fft(x, axis=1) * H.cpu().numpy().astype(np.complex128), axis=1)
            return _rel(xout.view(b, n)[:: b // 4].cpu().numpy(), want)

        op = Op(f"conv{n}", xin, xout, lambda i, o, plan=plan, H=H: plan.execute(i, H, o),
                b * (10.0 * n * math.log2(n) + 6.0 * n), 16 * n * b, 1, check,
                {"batch": b, "algorithm": plan.info()["algorithm"]})
        op.peer = ("cufft_3pass", lambda n=n, b=b, H=H: torch.fft.ifft(torch.fft.fft(xin.view(b, n)) * H))
        ops.append(op)
    # real signals: the half spectrum, one launch a batch (1-D) or R2C rows, half-width column convolution, C2R rows
    # (2-D); the same 256 MiB buffers read as float32
    rin, rout = xin.view(torch.float32), xout.view(torch.float32)
    for dims in REAL_CONV_DIMS:
        pts = int(np.prod(dims))
        b = (2 * CONV_POINTS) // pts
        hw = dims[-1] // 2 + 1
        hshape = tuple(dims[:-1]) + (hw,)
        plan = cf.ConvPlan(list(dims), batch=b, real=True)
        H = (torch.rand(2 * int(np.prod(hshape)), generator=gen, device=dev, dtype=torch.float32) * 2 - 1)
        H = H.view(torch.complex64).view(hshape)
        name = "rconv" + "x".join(str(v) for v in dims)
        axes = tuple(range(1, len(dims) + 1))

        def rcheck(dims=dims, b=b, plan=plan, H=H, axes=axes):
            plan.execute(rin, H, rout)
            torch.cuda.synchronize()
            x = rin.view((b,) + tuple(dims))[:: max(1, b // 4)].cpu().numpy().astype(np.float64)
            spec = np.fft.rfftn(x, axes=axes) * H.cpu().numpy().astype(np.complex128)
            for ax in axes[:-1]:
                spec = np.fft.ifft(spec, axis=ax)
            want = _irfft_ref(spec, dims[-1])
            return _rel(rout.view((b,) + tuple(dims))[:: max(1, b // 4)].cpu().numpy(), want)

        op = Op(name, rin, rout, lambda i, o, plan=plan, H=H: plan.execute(i, H, o),
                b * (5.0 * pts * math.log2(pts) + 3.0 * pts), 8 * pts * b, plan.info()["passes"], rcheck,
                {"batch": b, "algorithm": plan.info()["algorithm"]})
        if len(dims) == 1:
            op.peer = ("cufft_3pass", lambda n=dims[0], b=b, H=H: torch.fft.irfft(
                torch.fft.rfft(rin.view(b, n)) * H, n))
        else:
            op.peer = ("cufft_3pass", lambda dims=dims, b=b, H=H: torch.fft.irfft2(
                torch.fft.rfft2(rin.view((b,) + tuple(dims))) * H, s=dims))
        ops.append(op)
    return ops, dict(WORKLOAD_CONFIGS["conv"])


def precision_contrast(dev, rank, cf, steps: int, warmup: int) -> dict:
    """The metric's contrast on the 2-D 4096 x 4096 input of the precision configuration (uniform[-1,1) plus 1 % of
    entries x 1e4): each precision form's ms per execute (CUDA events, four input buffers in turn so none is
    L2-resident) and its rel-L2 against numpy's FP64 FFT. Timed outside the job's clock."""
    import numpy as np
    import torch

    ops = [op for op in _build_nd_forms(dev, rank, cf, tuple(PRECISIONS), shapes=((4096, 4096),))]
    out = {"shape": "4096x4096", "inputs": "uniform[-1,1) + 1% x 1e4", "bar": "rel-L2 <= 1e-6 vs FP64"}
    stream = torch.cuda.current_stream()
    for op in ops:
        for _ in range(warmup):
            op.run(op.inp, op.out)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            op.run(op.inp, op.out)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[op.info["precision"]] = {"ms": round(ms, 4), "rel_l2_vs_fp64": op.check(),
                                     "algorithm": op.info["algorithm"],
                                     "hbm_frac": round(op.bytes / (ms / 1e3) / 1e9 / measured_peaks()["hbm_gbs"], 4)}
    f32, bf = out["fp32"]["ms"], out["split-bf16"]["ms"]
    out["split_bf16_speedup_vs_fp32"] = round(f32 / bf, 3)
    ok = [k for k in PRECISIONS if k != "fp32" and out[k]["rel_l2_vs_fp64"] <= 1e-6]
    best = min(ok, key=lambda k: out[k]["ms"]) if ok else None
    out["fastest_tensor_core_form_at_1e-6"] = best
    out["its_speedup_vs_fp32"] = round(f32 / out[best]["ms"], 3) if best else None
    return out


def build_precision(dev, rank, cf):
    """The same 2-D and 3-D transforms with the first radix-16 stage of each unit-stride pass on the tensor cores
    (split-BF16: rel-L2 <= 1e-6 against FP64; FP16 with a per-line scale: reported), beside plain FP32."""
    return _build_nd_forms(dev, rank, cf, tuple(PRECISIONS)), \
        dict(WORKLOAD_CONFIGS["precision"])


def _irfft_ref(y, n):
    """The reference's normalised irfft over the last axis (real_fft.hpp:65-92), which the library's C2R follows:
    numpy's irfft drops the imaginary parts of Y[0] and Y[n/2]; the reference's pair formula keeps them, which adds a
    constant to the even and to the odd samples."""
    import numpy as np

    out = np.fft.irfft(y, n, axis=-1)
    h = n // 2
    im0, imh = y[..., 0].imag, y[..., h].imag
    out[..., 0::2] += (-(im0 + imh) / 2 / h)[..., None]
    out[..., 1::2] += ((im0 - imh) / 2 / h)[..., None]
    return out


WELCH = (64, 1 << 22, 1024, 512)  # signals, samples a signal, nperseg, noverlap


def _periodograms64(x, nper, nov):
    """FP64 segment periodograms of the rows of x (fs 1, periodic Hann, mean removed): the result check."""
    import numpy as np

    hop = nper - nov
    nseg = (x.shape[-1] - nov) // hop
    w = 0.5 - 0.5 * np.cos(2 * np.pi * np.arange(nper) / nper)
    idx = np.arange(nseg)[:, None] * hop + np.arange(nper)[None, :]
    seg = x[..., idx]
    seg = seg - seg.mean(axis=-1, keepdims=True)
    p = np.abs(np.fft.rfft(seg * w, axis=-1)) ** 2 / np.sum(w * w)
    p[..., 1:-1] *= 2
    return p


def build_welch(dev, rank, cf):
    """hesap-dsp's spectral estimators on the device: Welch's PSD and the spectrogram of 64 signals of 2^22 samples
    (1 GiB of float input), periodic Hann window, nperseg 1024, noverlap 512, fs 1; segment mean removed. One launch
    over all 524,224 segments (plus the fixed-order average for Welch)."""
    import numpy as np
    import torch

    count, ns, nper, nov = WELCH
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 21 + rank)
    x = torch.randn(count * ns, generator=gen, device=dev, dtype=torch.float32) + 0.5
    welch = cf.SpectralPlan(cf.SPECTRAL_WELCH, ns, count, 1.0, nper, nov)
    spec = cf.SpectralPlan(cf.SPECTRAL_SPECTROGRAM, ns, count, 1.0, nper, nov)
    pw = torch.empty(welch.out_shape(), dtype=torch.float32, device=dev)
    ps = torch.empty(spec.out_shape(), dtype=torch.float32, device=dev)
    nseg = welch.nseg
    fl = count * nseg * 2.5 * nper * math.log2(nper)

    def check_w():
        welch.execute(x, pw)
        torch.cuda.synchronize()
        xs = x.view(count, ns)[:2, : 64 * nper].cpu().numpy().astype(np.float64)
        want = _periodograms64(xs, nper, nov).mean(axis=-2)
        got = cf.SpectralPlan(cf.SPECTRAL_WELCH, 64 * nper, 2, 1.0, nper, nov).execute(
            x.view(count, ns)[:2, : 64 * nper].contiguous()).cpu().numpy()
        return _rel(got, want)

    def check_s():
        spec.execute(x, ps)
        torch.cuda.synchronize()
        xs = x.view(count, ns)[0, : 33 * (nper - nov) + nov].cpu().numpy().astype(np.float64)
        want = _periodograms64(xs, nper, nov)
        return _rel(ps[0, :want.shape[0]].cpu().numpy(), want)

    ops = [Op("welch", x, pw, lambda i, o: welch.execute(i, o), fl, 4 * count * ns + 4 * pw.numel(),
              welch.info()["passes"], check_w, {"segments": count * nseg, "algorithm": welch.info()["algorithm"]}),
           Op("spectrogram", x, ps, lambda i, o: spec.execute(i, o), fl, 4 * count * ns + 4 * ps.numel(),
              spec.info()["passes"], check_s, {"segments": count * nseg, "algorithm": spec.info()["algorithm"]})]
    return ops, dict(WORKLOAD_CONFIGS["welch"])


CWT = (64, 4096, 64, 128.0)  # signals, samples a signal, scales, largest scale (geometric from 1)


def _cwt64_morl(x, scales):
    """FP64 CWT of the rows of x with the real Morlet wavelet on 2^12 grid points over [-8, 8]: the integrated
    wavelet sampled at floor(m / (a step)) and reversed, convolved with the signal through a zero-padded FFT,
    -sqrt(a) (w[t+1] - w[t]) at t = (taps - 2) / 2 + i. The result check."""
    import numpy as np

    grid = 1 << 12
    step = 16.0 / (grid - 1)
    t = -8.0 + np.arange(grid) * step
    ipsi = np.cumsum(np.exp(-t * t / 2) * np.cos(5 * t)) * step
    n = x.shape[-1]
    taps = []
    for a in scales:
        kk = 0
        for m in range(int(math.ceil(a * 16.0 + 1.0))):
            if int(m / (a * step)) >= grid:
                break
            kk += 1
        taps.append(kk)
    L = 1
    while L < n + max(taps):
        L <<= 1
    X = np.fft.fft(x, L, axis=-1)
    out = np.zeros(x.shape[:-1] + (len(scales), n), dtype=np.complex128)
    for s, (a, kk) in enumerate(zip(scales, taps)):
        m = kk - 1 - np.arange(kk)
        kb = np.zeros(L)
        kb[:kk] = ipsi[(m / (a * step)).astype(np.int64)]
        w = np.fft.ifft(X * np.fft.fft(kb), axis=-1)
        i = (kk - 2) // 2 + np.arange(n)
        out[..., s, :] = -math.sqrt(a) * (w[..., i + 1] - w[..., i])
    return out


def build_cwt(dev, rank, cf):
    """hesap-wavelet's cwt on the device: 64 signals of 4096 samples, 64 scales from 1 to 128, real Morlet (FFT
    length 8192): one batched forward FFT of the signals, then one kernel over all 4096 (signal, scale) lines: the
    product with the kernel spectra (made at plan time), the inverse FFT in shared memory and the difference
    epilogue."""
    import numpy as np
    import torch

    count, n, ns, top = CWT
    scales = np.geomspace(1.0, top, ns)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED + 31 + rank)
    x = torch.randn(count * n, generator=gen, device=dev, dtype=torch.float32)
    plan = cf.CwtPlan(n, scales, "morl", count)
    out = torch.empty((count, ns, n), dtype=torch.complex64, device=dev)
    L = plan.fft_length
    fl = count * (5.0 * L * math.log2(L) + ns * (5.0 * L * math.log2(L) + 6.0 * L))
    rounds = -(-count // plan.signals_per_round)
    launches = 1 + cf.Plan([L], batch=count).info()["passes"] + (1 if plan.fused else rounds * (
        2 + cf.Plan([L], batch=plan.signals_per_round * ns).info()["passes"]))

    def check():
        plan.execute(x, out)
        torch.cuda.synchronize()
        xs = x.view(count, n)[:2].cpu().numpy().astype(np.float64)
        return _rel(out[:2].cpu().numpy(), _cwt64_morl(xs, scales))

    op = Op("cwt", x, out, lambda i, o: plan.execute(i, o), fl, 4 * count * n + 8 * count * ns * n, launches, check,
            {"signals": count, "scales": ns, "fft_length": L, "fused": plan.fused,
             "signals_per_round": plan.signals_per_round})
    return [op], dict(WORKLOAD_CONFIGS["cwt"])


BUILDERS = {"mixed": build_mixed, "n1024": build_n1024, "r2c": build_r2c, "uneven": build_uneven, "nd": build_nd,
            "precision": build_precision, "conv": build_conv, "welch": build_welch, "cwt": build_cwt}


# ---- the reference's CPU implementation (reference arm and cpu_baseline) -------------------------------------------


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model() -> dict:
    """The host CPU's model name and physical core count, from lscpu."""
    info = {"model": None, "physical_cores": None, "threads": host_threads()}
    try:
        txt = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
    except (OSError, subprocess.TimeoutExpired):
        return info
    kv = {}
    for ln in txt.splitlines():
        if ":" in ln:
            k, v = ln.split(":", 1)
            kv[k.strip()] = v.strip()
    info["model"] = kv.get("Model name")
    try:
        info["physical_cores"] = int(kv["Core(s) per socket"]) * int(kv.get("Socket(s)", "1"))
    except (KeyError, ValueError):
        pass
    return info


def cpu_rows(workload: str) -> list:
    """Two more rows of the reference's CPU path, each in a child process (its kernel level is fixed at first use):
    one host thread at the best level, and all threads with CRD_CPU_LEVEL=avx2."""
    rows = []
    for threads, level in ((1, None), (host_threads(), "avx2")):
        env = dict(os.environ)
        if level is not None:
            env["CRD_CPU_LEVEL"] = level
        try:
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--impl", "reference", "--workload",
                                workload, "--cpu-row", str(threads)], capture_output=True, text=True, env=env,
                               timeout=300)
            row = json.loads(r.stdout.strip().splitlines()[-1])
        except Exception as exc:  # the main row stands; say why this one is missing
            row = {"threads": threads, "value": None, "error": str(exc)[:200]}
        row["level_request"] = level or "auto"
        rows.append(row)
    return rows


def reference_cpu(workload: str, steps: int, warmup: int, budget_bytes: int, threads: int | None = None) -> dict:
    """Time the reference's crd-hesap-fft (oracle/_ref/libcrdref.so: FftPlan<float> for powers of two,
    BluesteinPlan<float> otherwise, RealFftPlan<float>, NdFftPlan<float>; one plan per thread over contiguous
    ranges, detail/batch_arms.hpp:59-77) on this host, in place, over a bounded sample of the workload."""
    import numpy as np

    import oracle  # the CPU checkers: only this leg of the benchmark uses them

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libcrdref.so not built")
    R = oracle.ref()
    threads = threads or host_threads()
    total_flops = 0.0
    total_time = 0.0
    sample = []
    per = {}

    def timed(fn, fl, label, rescale=None):
        nonlocal total_flops, total_time
        times = []
        for it in range(warmup + steps):
            t0 = time.perf_counter()
            fn()
            dt = time.perf_counter() - t0
            if rescale is not None:
                rescale()  # untimed: keeps repeated in-place transforms in range
            if it >= warmup:
                times.append(dt)
        t = sum(times)
        total_flops += fl * len(times)
        total_time += t
        per[label] = round(fl * len(times) / t / 1e9, 2)

    fp = ctypes.POINTER(ctypes.c_float)
    if workload == "mixed":
        for n, batch in SIZES:
            count = max(1, min(batch, budget_bytes // (8 * n)))
            count = max(count, min(batch, threads))
            buf = oracle.lcg_complex64(SEED ^ n, n * count)
            ptr = buf.view(np.float32).ctypes.data_as(fp)
            sc = np.float32(1.0 / math.sqrt(n))

            def run(n=n, count=count, ptr=ptr):
                if R.crdref_c2c_f32(n, count, ptr, 0, threads) != 0:
                    raise RuntimeError(f"crdref_c2c_f32 failed for n={n}")

            def rs(buf=buf, sc=sc):
                buf *= sc

            timed(run, flops(n, count), str(n), rs)
            sample.append(f"N={n} x{count} transforms")
    elif workload == "n1024":
        n, batch = 1024, 4096
        buf = oracle.lcg_complex64(SEED - 1, n * batch)
        ptr = buf.view(np.float32).ctypes.data_as(fp)
        sc = np.float32(1.0 / math.sqrt(n))

        def run():
            if R.crdref_c2c_f32(n, batch, ptr, 0, threads) != 0:
                raise RuntimeError("crdref_c2c_f32 failed for n=1024")

        def rs():
            buf[:] *= sc

        timed(run, flops(n, batch), "1024", rs)
        sample.append(f"N=1024 x{batch} transforms (the whole batch)")
    elif workload == "conv":
        # the reference's CPU route to the same result: FftPlan forward, the product, FftPlan inverse and 1/N
        for n in CONV_SIZES:
            count = max(threads, min(CONV_POINTS // n, budget_bytes // (8 * n)))
            buf = oracle.lcg_complex64(SEED ^ (n + 11), n * count)
            H = oracle.lcg_complex64(SEED ^ (n + 12), n)
            ptr = buf.view(np.float32).ctypes.data_as(fp)

            def run(n=n, count=count, buf=buf, ptr=ptr, H=H):
                R.crdref_c2c_f32(n, count, ptr, 0, threads)
                v = buf.reshape(count, n)
                v *= H
                R.crdref_c2c_f32(n, count, ptr, 1, threads)
                v *= np.float32(1.0 / n)

            timed(run, count * (10.0 * n * math.log2(n) + 6.0 * n), f"conv{n}")
            sample.append(f"conv N={n} x{count}")
        # real signals: RealFftPlan rfft, the product with the half spectrum, irfft (normalised: the 1/N)
        for dims in REAL_CONV_DIMS:
            if len(dims) != 1:
                continue  # the reference's real plans are 1-D (real_fft.hpp)
            n = dims[0]
            count = max(threads, min((2 * CONV_POINTS) // n, budget_bytes // (4 * n)))
            x = oracle.lcg_float32(SEED ^ (n + 13), n * count)
            H = oracle.lcg_complex64(SEED ^ (n + 14), n // 2 + 1)
            spec = np.empty(count * (n // 2 + 1), dtype=np.complex64)
            back = np.empty(n * count, dtype=np.float32)

            def rrun(n=n, count=count, x=x, H=H, spec=spec, back=back):
                R.crdref_rfft_f32(n, count, x.ctypes.data_as(fp), spec.view(np.float32).ctypes.data_as(fp), threads)
                spec.reshape(count, n // 2 + 1)[:] *= H
                R.crdref_irfft_f32(n, count, spec.view(np.float32).ctypes.data_as(fp), back.ctypes.data_as(fp),
                                   threads)

            timed(rrun, count * (5.0 * n * math.log2(n) + 3.0 * n), f"rconv{n}")
            sample.append(f"real conv N={n} x{count}")
    elif workload == "welch":
        # the reference's dsp::welch_psd<float> over the signals, one signal at a time per thread
        count, ns, nper, nov = WELCH
        cnt = max(1, min(count, budget_bytes // (4 * ns)))
        x = oracle.lcg_float32(SEED ^ 0x3E1C, cnt * ns)
        out = np.empty(cnt * (nper // 2 + 1), dtype=np.float32)
        nseg = (ns - nov) // (nper - nov)

        def wrun():
            if R.crdref_welch_f32(ns, cnt, x.ctypes.data_as(fp), 1.0, nper, nov, out.ctypes.data_as(fp),
                                  threads) != 0:
                raise RuntimeError("crdref_welch_f32 failed")

        timed(wrun, cnt * nseg * 2.5 * nper * math.log2(nper), "welch")
        sample.append(f"welch {cnt} signals x {ns} samples, nperseg {nper}, noverlap {nov}")
    elif workload == "cwt":
        # the reference's wavelet::cwt<float> over the signals, one signal at a time per thread
        count, n, ns, top = CWT
        scales = np.geomspace(1.0, top, ns).astype(np.float32)
        cnt = max(threads, 1) if count > threads else count
        x = oracle.lcg_float32(SEED ^ 0xC3, cnt * n)
        out = np.empty(cnt * ns * n * 2, dtype=np.float32)
        freqs = np.empty(ns)
        L = 8192
        fl = cnt * (5.0 * L * math.log2(L) + ns * (5.0 * L * math.log2(L) + 6.0 * L))

        def crun():
            if R.crdref_cwt_f32(n, cnt, x.ctypes.data_as(fp), scales.ctypes.data_as(fp), ns, b"morl",
                                out.ctypes.data_as(fp), freqs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                threads) != 0:
                raise RuntimeError("crdref_cwt_f32 failed")

        timed(crun, fl, "cwt")
        sample.append(f"cwt<float> morl {cnt} signals x {n} samples, {ns} scales")
    elif workload == "r2c":
        n = 1 << 20
        count = max(threads, min(512, budget_bytes // (4 * n)))
        x = oracle.lcg_float32(SEED, n * count)
        spec = np.empty(count * (n // 2 + 1), dtype=np.complex64)
        back = np.empty(n * count, dtype=np.float32)
        fl = 2.5 * n * math.log2(n) * count
        timed(lambda: R.crdref_rfft_f32(n, count, x.ctypes.data_as(fp), spec.view(np.float32).ctypes.data_as(fp),
                                        threads), fl, "r2c")
        timed(lambda: R.crdref_irfft_f32(n, count, spec.view(np.float32).ctypes.data_as(fp), back.ctypes.data_as(fp),
                                         threads), fl, "c2r")
        sample.append(f"RealFftPlan<float>(2^20) rfft+irfft x{count}")
    elif workload == "uneven":
        from crd_b200.workloads import uneven_sizes

        all_sizes = uneven_sizes(20000, seed=0x5EED0003)
        sizes, used = [], 0
        for s in all_sizes:  # a bounded prefix of the batch
            if used + 8 * s > budget_bytes:
                break
            sizes.append(s)
            used += 8 * s
        offs, total = [], 0
        for s in sizes:
            offs.append(total)
            total += s
        buf = oracle.gauss_complex64(0x5EED0003, total)
        i64 = ctypes.c_int64 * len(sizes)
        cs, co = i64(*sizes), i64(*offs)

        def run():
            R.crdref_uneven_f32(len(sizes), cs, co, buf.view(np.float32).ctypes.data_as(fp), 0, threads)

        def rs():
            buf[:] *= np.float32(1.0 / 256.0)

        fl = sum(5.0 * s * math.log2(s) for s in sizes)
        timed(run, fl, "uneven", rs)
        sample.append(f"first {len(sizes)} of 20000 transforms ({len(set(sizes))} sizes), per-thread plan cache "
                      "built in the warm-up pass")
    elif workload in ("nd", "precision"):  # the reference has FP32 only
        for dims in ((4096, 4096), (512, 512, 512)):
            total = int(np.prod(dims))
            x = oracle.lcg_complex64(SEED + total, total)
            d = (ctypes.c_size_t * len(dims))(*dims)
            sc = np.float32(1.0 / math.sqrt(total))

            def run(x=x, d=d, dims=dims):
                R.crdref_nd_f32(len(dims), d, x.view(np.float32).ctypes.data_as(fp), 0)

            def rs(x=x, sc=sc):
                x *= sc

            timed(run, 5.0 * total * math.log2(total), "x".join(map(str, dims)), rs)
            sample.append(f"NdFftPlan<float>({'x'.join(map(str, dims))}) on 1 thread")
        threads = 1
    return {
        "value": total_flops / total_time / 1e9,
        "cores": threads,
        "level": int(R.crdref_level()),
        "sample": "; ".join(sample) + f"; {threads} threads, in place",
        "per_op_gflops": per,
        "seconds": total_time,
    }


def run_cpu_row(args) -> None:
    """One bounded CPU row (child of cpu_rows): 64 MiB per size at one thread, 256 MiB otherwise."""
    budget = (64 << 20) if args.cpu_row == 1 else (256 << 20)
    res = reference_cpu(args.workload, steps=2, warmup=1, budget_bytes=budget, threads=args.cpu_row)
    print(json.dumps({"threads": res["cores"], "value": round(res["value"], 2), "unit": "GFLOP/s",
                      "level": res["level"], "sample": res["sample"]}), flush=True)


def run_reference_arm(args) -> None:
    if getattr(args, "cpu_row", None) is not None:
        run_cpu_row(args)
        return
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    res = reference_cpu(args.workload, args.steps, args.warmup, budget_bytes=1 << 30)
    value = res["value"]
    ms_per_step = res["seconds"] / args.steps * 1e3
    config = dict(WORKLOAD_CONFIGS[args.workload])
    config["parallelism"] = "host threads"
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
        "config": config,
        "cpu_baseline": {"value": round(value, 2), "unit": "GFLOP/s", "cores": res["cores"], "kind": "reference",
                         "sample": res["sample"], "level": res["level"], "per_op_gflops": res["per_op_gflops"],
                         "host": cpu_model()},
        "e2e": {"value": round(value, 2), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm ---------------------------------------------------------------------------------------------------


def max_over_ranks_of(v: float, world: int, device) -> float:
    """The largest of a per-rank value over the job's ranks (the slowest rank's time is the job's time)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank_step: float, steps: int, world: int, total_ms: float) -> float:
    """Whole-job rate per second: every rank runs its own replica of the per-GPU workload (weak scaling), so the job
    processes world times one rank's units in the slowest rank's time."""
    return units_per_rank_step * steps * world / (total_ms / 1e3)


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    import crd_b200 as cf
    import crd_b200.hesap as F

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
        return max_over_ranks_of(v, world, dev)

    if args.wisdom and os.path.exists(args.wisdom):
        with open(args.wisdom) as f:
            F.wisdom_import(f.read())
    F.set_planner(args.planner)

    ops, config = BUILDERS[args.workload](dev, rank, cf)
    launches_per_step = sum(op.launches for op in ops)
    if args.planner_log and rank == 0:
        with open(args.planner_log, "w") as f:
            f.write(F.planner_log())
        with open(args.planner_log + ".wisdom", "w") as f:
            f.write(F.wisdom_export())
    stream = torch.cuda.current_stream()

    def step(events=None):
        for i, op in enumerate(ops):
            if events is not None:
                events[i][0].record(stream)
            op.run(op.inp, op.out)
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

    ev = [[[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] for _ in ops]
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
    per_ms = [sum(ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(args.steps)) / args.steps
              for i in range(len(ops))]
    step_flops = sum(op.flops for op in ops)
    step_bytes = sum(op.bytes for op in ops)
    value = job_rate(step_flops, args.steps, world, total_ms) / 1e9
    ms_per_step = total_ms / args.steps

    rel = {op.name: op.check() for op in ops}
    F.device_status(cf.Plan([16]))  # the library's status word path works (a fresh plan: OK)

    peaks = measured_peaks()
    # Dominant op: the op with the largest share of the step's device time. Its achieved rate is its algorithmic
    # bytes over its event-timed duration (for a multi-launch op, the four-step's passes and waves, that is the same
    # as algorithmic bytes per launch over the average launch). Beside it, the longest single-launch kernel.
    dom = max(range(len(ops)), key=lambda i: per_ms[i])
    dom_bytes = ops[dom].bytes / max(1, ops[dom].launches)
    dom_ms = per_ms[dom] / max(1, ops[dom].launches)
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    single = [i for i, op in enumerate(ops) if op.launches == 1]
    one = max(single, key=lambda i: per_ms[i]) if single else None
    traffic_doc = profiled_traffic()
    traffic = traffic_doc.get(f"{args.workload}:{ops[dom].name}")
    if traffic is not None:
        traffic = round(traffic / max(1, ops[dom].launches))
    single_roof = None
    if one is not None and one != dom:
        ach1 = ops[one].bytes / (per_ms[one] / 1e3) / 1e9
        single_roof = {"kernel": f"{ops[one].name} ({ops[one].info.get('algorithm', '')})",
                       "achieved": round(ach1, 1), "frac": round(ach1 / peaks["hbm_gbs"], 4),
                       "traffic": traffic_doc.get(f"{args.workload}:{ops[one].name}"),
                       "algorithmic_bytes_per_launch": ops[one].bytes}
    per = {}
    for op, ms in zip(ops, per_ms):
        gbs = op.bytes / (ms / 1e3) / 1e9
        per[op.name] = dict(op.info, launches=op.launches, ms=round(ms, 4),
                            gflops=round(op.flops / (ms / 1e3) / 1e9, 1), hbm_gbs=round(gbs, 1),
                            hbm_frac=round(gbs / peaks["hbm_gbs"], 4), rel_l2_vs_fp64=rel[op.name])
        if op.peer is not None:
            # the vendor route for the same op, same data, same event timing (untimed by the job's clock)
            name, fn = op.peer
            for _ in range(max(3, args.warmup)):
                fn()
            p0 = torch.cuda.Event(enable_timing=True)
            p1 = torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            for _ in range(args.steps):
                fn()
            p1.record(stream)
            torch.cuda.synchronize()
            pms = p0.elapsed_time(p1) / args.steps
            per[op.name].update({"peer": name, "peer_ms": round(pms, 4), "speedup_vs_peer": round(pms / ms, 2)})

    precision = None
    if args.workload == "mixed" and not args.no_precision:
        precision = precision_contrast(dev, rank, cf, max(3, args.steps), max(3, args.warmup))

    # End to end through the public API with host buffers: every step copies each op's input from pinned host
    # memory, runs it, and copies its whole output back (crdfft_execute_host where the op has it: the batch in chunks,
    # copies in both directions overlapping the transforms).
    e2e = None
    if not args.no_e2e:
        hins = [torch.empty(op.inp.shape, dtype=op.inp.dtype, pin_memory=True) for op in ops]
        houts = [torch.empty(op.out.shape, dtype=op.out.dtype, pin_memory=True) for op in ops]
        for h, op in zip(hins, ops):
            h.copy_(op.inp)
        e_steps = max(1, min(args.steps, 3))

        def e2e_step():
            for h, ho, op in zip(hins, houts, ops):
                if op.host is not None:
                    op.host(h, ho)  # chunked: copies in both directions overlap the transforms
                else:
                    op.inp.copy_(h, non_blocking=True)
                    op.run(op.inp, op.out)
                    ho.copy_(op.out, non_blocking=True)

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
        h2d = sum(op.inp.numel() * op.inp.element_size() for op in ops)
        d2h = sum(op.out.numel() * op.out.element_size() for op in ops)
        e2e = {"value": round(job_rate(step_flops, e_steps, world, e_ms) / 1e9, 2), "unit": "GFLOP/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e_steps,
               "ms_per_step": round(e_ms / e_steps, 3)}
        # The end-to-end bound: PCIe with copies running both ways at once. Measured here on the same pinned buffers
        # (the first op's input host->device on one stream while its output goes device->host on another).
        big = max(range(len(ops)), key=lambda i: ops[i].inp.numel() * ops[i].inp.element_size())
        hi, ho, op = hins[big], houts[big], ops[big]
        nbytes = min(hi.numel() * hi.element_size(), ho.numel() * ho.element_size())
        s_a, s_b = torch.cuda.Stream(), torch.cuda.Stream()

        hin_b, hout_b = hi.view(-1).view(torch.uint8), ho.view(-1).view(torch.uint8)
        din_b, dout_b = op.inp.view(-1).view(torch.uint8), op.out.view(-1).view(torch.uint8)

        def both_ways(chunk):
            # whole buffers, or 64 MiB chunks (the host pipeline's copy size); each direction on its own stream
            step = chunk or nbytes
            for o in range(0, nbytes, step):
                m = min(step, nbytes - o)
                with torch.cuda.stream(s_a):
                    din_b[o:o + m].copy_(hin_b[o:o + m], non_blocking=True)
                with torch.cuda.stream(s_b):
                    hout_b[o:o + m].copy_(dout_b[o:o + m], non_blocking=True)

        c_ms = []
        for chunk in (0, 64 << 20):
            both_ways(chunk)
            torch.cuda.synchronize()
            for _ in range(3):
                c0 = torch.cuda.Event(enable_timing=True)
                c1 = torch.cuda.Event(enable_timing=True)
                c0.record(stream)
                s_a.wait_event(c0)
                s_b.wait_event(c0)
                both_ways(chunk)
                stream.wait_stream(s_a)
                stream.wait_stream(s_b)
                c1.record(stream)
                torch.cuda.synchronize()
                c_ms.append(c0.elapsed_time(c1))
        peak_dir = nbytes / (min(c_ms) / 1e3) / 1e9
        ach_dir = max(h2d, d2h) / (e_ms / e_steps / 1e3) / 1e9
        e2e["roofline"] = {"bound": "pcie", "unit": "GB/s per direction", "achieved": round(ach_dir, 1),
                           "peak": round(peak_dir, 1), "frac": round(ach_dir / peak_dir, 3),
                           "peak_source": "measured here: pinned copies both ways at once (whole buffers and 64 MiB chunks, "
                                          "the best of six)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            # the reference arm's sample (1 GiB per size) with a few steps
            res = reference_cpu(args.workload, steps=5, warmup=2, budget_bytes=1 << 30)
            cpu = {"value": round(res["value"], 2), "unit": "GFLOP/s", "cores": res["cores"], "kind": "reference",
                   "sample": res["sample"], "level": res["level"], "per_op_gflops": res["per_op_gflops"],
                   "host": cpu_model(), "rows": cpu_rows(args.workload)}
        except Exception as exc:  # the GPU number stands; say why the baseline is missing
            cpu = {"value": None, "unit": "GFLOP/s", "cores": host_threads(), "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        config.update({"precision": "per op" if args.workload == "precision" else "fp32",
                       "placement": "out-of-place", "planner": args.planner, "parallelism": f"replicas{world}"})
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
            "config": config,
            "roofline": {"bound": "hbm", "kernel": f"{ops[dom].name} ({ops[dom].info.get('algorithm', '')})",
                         "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peaks["source"],
                         "traffic": traffic, "algorithmic_bytes_per_launch": round(dom_bytes),
                         "launches_per_execute": ops[dom].launches,
                         "share_of_step": round(per_ms[dom] / sum(per_ms), 4),
                         "single_launch_kernel": single_roof},
            "hbm_frac_step": round(step_bytes / (ms_per_step / 1e3) / 1e9 / peaks["hbm_gbs"], 4),
            "per_op": per,
            "rel_l2_vs_fp64_max": max(rel.values()),
            "gpu_launches": launches_per_step * args.steps,
            "precision": precision,
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
    ap.add_argument("--workload", choices=WORKLOADS, default="mixed",
                    help="mixed (default): C2C at N 4096/65536/2^20/107520; n1024: N 1024 x 4096; r2c: R2C/C2R 2^20; uneven: 20,000 "
                         "7-smooth sizes; nd: FP32 2-D 4096^2 / 3-D 512^3; precision: the same 2-D/3-D at FP32, "
                         "split-BF16 and FP16-scaled; conv: fused FFT convolution beside cuFFT's three passes")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the split-BF16 vs FP32 contrast the default workload reports beside its line")
    ap.add_argument("--cpu-row", type=int, default=None, help=argparse.SUPPRESS)  # one CPU row, in a child
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
