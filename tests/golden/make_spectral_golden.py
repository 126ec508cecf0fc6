"""Extract the reference tests' spectral golden vectors into ``spectral_refs.npz`` (this directory).

The reference's hesap-dsp tests check its spectral estimators against scipy.signal outputs kept in
``tests/numerics/hesap-dsp/spectral_refs.inc`` (used by test_spectral.cpp:18-253): a 512-sample test signal x and a
second signal y, Welch's PSD (fs = 100, nperseg = 64, default overlap), the spectrogram (nperseg = 64, noverlap =
32), the periodogram, the cross-spectral density and the coherence. This script reads that file as text, where the
reference sources lie, and stores the arrays unchanged:

    python tests/golden/make_spectral_golden.py [REFERENCE_ROOT]
"""

from __future__ import annotations

import os
import re
import sys

import numpy as np

if len(sys.argv) < 2:
    sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout>")
REF = sys.argv[1]
SRC = os.path.join(REF, "tests", "numerics", "hesap-dsp", "spectral_refs.inc")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "spectral_refs.npz")


def main() -> None:
    text = open(SRC).read()
    arrays = {}
    for m in re.finditer(r"inline const double (\w+)\[\]\s*=\s*\{([^}]*)\}", text):
        arrays[m.group(1).removeprefix("ref_")] = np.array([float(v) for v in m.group(2).split(",") if v.strip()])
    for m in re.finditer(r"inline const int (\w+)\s*=\s*(-?\d+)", text):
        arrays[m.group(1).removeprefix("ref_")] = np.array(int(m.group(2)))
    np.savez_compressed(OUT, **arrays)
    print(OUT, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
