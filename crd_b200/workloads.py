"""Synthetic workloads of the benchmark configurations (seeded; no datasets exist for this path).

* ``smooth_sizes(lo, hi)``: every 7-smooth integer in [lo, hi] (601 of them in [16, 65536]).
* ``uneven_sizes(count, seed)``: the uneven-batch configuration: sizes log-uniform over the 7-smooth integers in
  [16, 65536]: x = exp(U[ln 16, ln 65536]) from the seed, rounded up to the next 7-smooth integer.
"""

from __future__ import annotations

import bisect
import math

import numpy as np


def smooth_sizes(lo: int = 16, hi: int = 65536) -> list:
    out = []
    p2 = 1
    while p2 <= hi:
        p3 = p2
        while p3 <= hi:
            p5 = p3
            while p5 <= hi:
                p7 = p5
                while p7 <= hi:
                    if p7 >= lo:
                        out.append(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


def uneven_sizes(count: int = 20000, seed: int = 0x5EED0003, lo: int = 16, hi: int = 65536) -> list:
    table = smooth_sizes(lo, hi)
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))
    return [table[min(bisect.bisect_left(table, float(v)), len(table) - 1)] for v in x]
