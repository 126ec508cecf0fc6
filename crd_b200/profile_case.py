"""One plan, executed a few times: the small, self-contained case that profilers capture.

    python -m crd_b200.profile_case N BATCH REPS [estimate|measure|learned] [WISDOM_FILE]
    python -m crd_b200.profile_case r2c N BATCH REPS
    python -m crd_b200.profile_case welch|spectrogram NPERSEG NOVERLAP COUNT NSAMPLES REPS
    python -m crd_b200.profile_case uneven COUNT REPS
    python -m crd_b200.profile_case nd PREC REPS DIM0 DIM1 [DIM2]

The first form creates a forward C2C plan of BATCH transforms of length N (planner mode and optional wisdom as
given), fills the input with uniform[-1, 1) values and runs REPS out-of-place executes on the current CUDA device.
The second runs a real-to-complex plan the same way; the third a spectral estimator over COUNT signals of NSAMPLES
Gaussian samples (periodic Hann window, fs 1); the fourth an uneven batch of COUNT transforms with the benchmark's size
distribution (log-uniform over the 7-smooth lengths in [16, 65536]); the fifth a 2-D or 3-D C2C transform at precision
form PREC (0 FP32, 1 split-BF16, 2 FP16 scaled) with uniform[-1, 1) inputs plus 1 % of entries scaled by 1e4.
"""

from __future__ import annotations

import os
import sys


def main(argv=None) -> None:
    # the library's one-time known-answer check runs small plans at the first plan creation; a profiler capture of
    # the case should not count their launches
    os.environ.setdefault("CRDFFT_SELF_CHECK", "0")
    import torch

    import crd_b200 as cf
    import crd_b200.hesap as F

    argv = sys.argv[1:] if argv is None else argv
    if argv[0] == "r2c":
        n, batch, reps = int(argv[1]), int(argv[2]), int(argv[3])
        x = torch.rand(n * batch, device="cuda") * 2 - 1
        y = torch.empty(batch * (n // 2 + 1), dtype=torch.complex64, device="cuda")
        plan = cf.Plan([n], batch=batch, kind=cf.R2C)
        print(plan.info())
        for _ in range(reps):
            plan.execute(x, y, cf.FORWARD)
        torch.cuda.synchronize()
        print("ok")
        return
    if argv[0] == "uneven":
        from crd_b200.workloads import uneven_sizes

        count, reps = int(argv[1]), int(argv[2])
        plan = cf.UnevenPlan(uneven_sizes(count))
        x = torch.randn(2 * plan.total, device="cuda").view(torch.complex64)
        y = torch.empty_like(x)
        print(plan.info())
        for _ in range(reps):
            plan.execute(x, y)
        torch.cuda.synchronize()
        print("ok")
        return
    if argv[0] == "nd":
        prec, reps = int(argv[1]), int(argv[2])
        dims = [int(v) for v in argv[3:]]
        total = 1
        for v in dims:
            total *= v
        x = (torch.rand(2 * total, device="cuda") * 2 - 1).view(torch.complex64)
        idx = torch.randperm(total, device="cuda")[: total // 100]
        x[idx] *= 1e4
        y = torch.empty_like(x)
        plan = cf.Plan(dims, batch=1, precision=prec)
        print(plan.info())
        for _ in range(reps):
            plan.execute(x, y)
        torch.cuda.synchronize()
        print("ok")
        return
    if argv[0] in ("welch", "spectrogram"):
        nper, nov, count, ns, reps = (int(v) for v in argv[1:6])
        mode = cf.SPECTRAL_WELCH if argv[0] == "welch" else cf.SPECTRAL_SPECTROGRAM
        x = torch.randn(count * ns, device="cuda")
        plan = cf.SpectralPlan(mode, ns, count, 1.0, nper, nov)
        print(plan.info())
        out = torch.empty(plan.out_shape(), dtype=torch.float32, device="cuda")
        for _ in range(reps):
            plan.execute(x, out)
        torch.cuda.synchronize()
        print("ok")
        return
    n, batch, reps = int(argv[0]), int(argv[1]), int(argv[2])
    if len(argv) > 4 and os.path.exists(argv[4]):
        with open(argv[4]) as f:
            F.wisdom_import(f.read())
    F.set_planner(argv[3] if len(argv) > 3 else "estimate")
    x = (torch.rand(2 * n * batch, device="cuda") * 2 - 1).view(torch.complex64)
    y = torch.empty_like(x)
    plan = cf.Plan([n], batch=batch)
    print(plan.info())
    for _ in range(reps):
        plan.execute(x, y)
    torch.cuda.synchronize()
    print("ok")


if __name__ == "__main__":
    main()
