"""Generate the golden vectors in this directory from the reference implementation itself.

Run in a container that has the reference sources, after ``make -C oracle ref`` built ``oracle/_ref/libcrdref.so``
from them:

    python tests/golden/make_golden.py

Writes ``reference_f32.npz``: inputs and the reference's outputs, all produced by calling the reference's own plans
(yatiyr/CRD engine/numerics/hesap-fft) through oracle/ref_shim.cpp:

* ``selfcheck_*``: the cases of the reference's known-answer self-check (src/fft_self_check.cpp:67-77: sizes 2..128,
  small-integer inputs from its value() rule, :45-50) run on the FftAlgorithm::Stockham plans the check uses. The
  reference verified its own digests over these outputs (crdref_self_check_level), so these bits are its golden
  answers, and it checked them once against a 200-bit DFT (:4-6).
* ``c2c_<n>``: FftPlan<float>(n) forward/inverse (power-of-two n) or BluesteinPlan<float>(n) (other n) on the
  reference tests' LCG inputs (test_fft.cpp:31-44, seed 0x9E3779B97F4A7C15 ^ n as at :71).
* ``rfft_<n>`` / ``irfft_<n>``: RealFftPlan<float>(n).
* ``nd_<dims>``: NdFftPlan<float>(dims).
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_f32.npz")

K_VALUES = [1, -2, 2, -1, -2, 1, 2]


def value(k: int, salt: int) -> int:
    """src/fft_self_check.cpp:45-50."""
    return K_VALUES[(k * (salt % 5 + 2) + salt * 3 + k // 7) % 7]


# src/fft_self_check.cpp:67-77, in its order: (n, batch, inverse, tiny); batch 0 = execute, -1 = the f32 tail
# batch of 19 transforms; tiny scales the inputs by 2^-140 so the results are subnormal (:111-121).
SELFCHECK_CASES = [
    (2, 0, 0, 0), (2, 0, 1, 0), (4, 0, 0, 0), (4, 0, 1, 0), (8, 0, 0, 0), (8, 0, 1, 0), (16, 0, 0, 0),
    (16, 0, 1, 0), (16, 0, 0, 1), (32, 0, 0, 0), (32, 0, 1, 0), (64, 0, 0, 0), (64, 0, 1, 0), (128, 0, 0, 0),
    (128, 0, 1, 0), (8, 8, 0, 0), (8, -1, 0, 0), (8, -1, 1, 0), (16, 8, 0, 0), (16, -1, 0, 0), (16, -1, 1, 0),
    (32, 8, 0, 0), (32, -1, 0, 0), (32, -1, 1, 0), (64, 8, 0, 0), (64, 3, 1, 0),
]
TINY = np.array([0x00000200], dtype=np.uint32).view(np.float32)[0]


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libcrdref.so is missing: run `make -C oracle ref` first")
    R = oracle.ref()
    data = {}
    for idx, (n, batch, inv, tiny) in enumerate(SELFCHECK_CASES):
        transforms = 19 if batch == -1 else (1 if batch == 0 else batch)
        pts = n * transforms
        scale = TINY if tiny else np.float32(1.0)
        re = np.array([value(i, 2 * idx) for i in range(pts)], dtype=np.float32) * scale
        im = np.array([value(i, 2 * idx + 1) for i in range(pts)], dtype=np.float32) * scale
        x = (re + 1j * im).astype(np.complex64)
        y = x.copy()
        rc = R.crdref_stockham_f32(n, 0 if batch == 0 else transforms, oracle._ptr_f(y.view(np.float32)), inv)
        assert rc == 0
        key = f"selfcheck_{idx}"
        data[key + "_in"] = x
        data[key + "_out"] = y
        data[key + "_meta"] = np.array([n, 0 if batch == 0 else transforms, inv, tiny], dtype=np.int64)

    for n in (16, 105, 240, 1024, 4096):
        x = oracle.lcg_complex64(0x9E3779B97F4A7C15 ^ n, n)
        data[f"c2c_{n}_in"] = x
        data[f"c2c_{n}_fwd"] = oracle.ref_c2c_f32(x, inverse=False)
        data[f"c2c_{n}_inv"] = oracle.ref_c2c_f32(x, inverse=True)

    for n in (64, 1024):
        x = oracle.lcg_float32(31337 + n, n)
        data[f"rfft_{n}_in"] = x
        data[f"rfft_{n}_out"] = oracle.ref_rfft_f32(x)
        spec = oracle.lcg_complex64(0x5EED + n, n // 2 + 1)
        spec[0] = spec[0].real  # a Hermitian half spectrum has real end points
        spec[-1] = spec[-1].real
        data[f"irfft_{n}_in"] = spec
        data[f"irfft_{n}_out"] = oracle.ref_irfft_f32(spec, n)

    for dims in ((8, 16), (4, 6, 5), (16, 12)):
        tag = "x".join(str(d) for d in dims)
        total = int(np.prod(dims))
        x = oracle.lcg_complex64(0x9E3779B97F4A7C15 ^ total, total).reshape(dims)
        data[f"nd_{tag}_in"] = x
        data[f"nd_{tag}_fwd"] = oracle.ref_nd_f32(x, inverse=False)
        data[f"nd_{tag}_inv"] = oracle.ref_nd_f32(x, inverse=True)

    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT}: {len(data)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
