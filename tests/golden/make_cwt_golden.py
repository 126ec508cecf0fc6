"""Extract the reference tests' CWT golden vectors into ``cwt_refs.npz`` (this directory).

The reference's hesap-wavelet tests check its continuous wavelet transform against pywt.cwt outputs kept in
``tests/numerics/hesap-wavelet/cwt_refs.inc`` (used by test_cwt.cpp:31-98): a 96-sample signal, four scales, and
for mexh, morl, gaus2, gaus4 (real coefficients) and cmor1.5-1.0, cgau2, shan1.0-0.5, fbsp2-1.0-0.5 (interleaved
complex coefficients) the coefficients [scale][sample] and the scales' frequencies. This script reads that file as
text, where the reference sources lie, and stores the arrays unchanged:

    python tests/golden/make_cwt_golden.py [REFERENCE_ROOT]
"""

from __future__ import annotations

import os
import re
import sys

import numpy as np

if len(sys.argv) < 2:
    sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout>")
REF = sys.argv[1]
SRC = os.path.join(REF, "tests", "numerics", "hesap-wavelet", "cwt_refs.inc")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cwt_refs.npz")


def main() -> None:
    text = open(SRC).read()
    arrays = {}
    for m in re.finditer(r"inline const double (\w+)\[\]\s*=\s*\{([^}]*)\}", text):
        arrays[m.group(1).removeprefix("ref_cwt_")] = np.array([float(v) for v in m.group(2).split(",") if v.strip()])
    np.savez_compressed(OUT, **arrays)
    print(OUT, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
