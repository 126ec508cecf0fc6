"""One plan, executed a few times: the small, self-contained case that profilers capture.

    python -m crd_b200.profile_case N BATCH REPS [estimate|measure|learned] [WISDOM_FILE]

Creates a forward C2C plan of BATCH transforms of length N (planner mode and optional wisdom as given), fills the
input with uniform[-1, 1) values and runs REPS out-of-place executes on the current CUDA device.
"""

from __future__ import annotations

import os
import sys


def main(argv=None) -> None:
    import torch

    import crd_b200 as cf
    import crd_b200.hesap as F

    argv = sys.argv[1:] if argv is None else argv
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
