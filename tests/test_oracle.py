"""CPU tests: pin the oracle before trusting it.

The oracle (oracle/oracle.c) is checked against (1) the brute-force FP64 DFT, the reference's correctness gate
(tests/numerics/hesap-fft/test_fft.cpp:1-4, 47-65), (2) numpy's float64 FFT as an independent implementation, and
(3) the golden vectors in tests/golden/reference_f32.npz, which are the reference's own outputs; the test first
re-derives the reference's published known-answer digests from them (src/fft_self_check.cpp:96-97).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import oracle

K_ANSWERS32 = (0xCC3A7A3D345F533F, 0x9F5EABF56E31535E)  # src/fft_self_check.cpp:97


def _fnv_fold(h: int, word: int) -> int:
    for i in range(4):
        h = ((h ^ ((word >> (8 * i)) & 0xFF)) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def test_golden_reproduces_reference_digests(golden):
    """The committed self-check outputs hash to the reference's own kAnswers32 digests, bit for bit."""
    h = [0xCBF29CE484222325, 0xCBF29CE484222325]
    for idx in range(26):
        meta = golden[f"selfcheck_{idx}_meta"]
        routine = 0 if meta[1] == 0 else 1
        for w in golden[f"selfcheck_{idx}_out"].view(np.float32).view(np.uint32):
            h[routine] = _fnv_fold(h[routine], int(w))
    assert tuple(h) == K_ANSWERS32


def test_oracle_matches_reference_known_answers(golden):
    """FP64 oracle vs the reference's self-check outputs, at the bound the reference states for them (within 1e-7
    of the transform's largest output; 9.2e-5 relative for the subnormal case, src/fft_self_check.cpp:4-6)."""
    for idx in range(26):
        n, batch, inv, tiny = (int(v) for v in golden[f"selfcheck_{idx}_meta"])
        x = golden[f"selfcheck_{idx}_in"].astype(np.complex128)
        ref = golden[f"selfcheck_{idx}_out"].astype(np.complex128)
        if batch == 0:
            want = oracle.fft64(x, inverse=bool(inv))
        else:
            want = oracle.fft64(x.reshape(n, batch).T, inverse=bool(inv)).T.reshape(-1)
        scale = np.max(np.abs(want))
        err = np.max(np.abs(ref - want))
        bound = (9.2e-5 if tiny else 1.0e-7) * scale * 1.5
        assert err <= bound, (idx, n, batch, inv, err, scale)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 9, 12, 15, 16, 17, 30, 32, 49, 64, 100, 105, 128, 243, 256, 360,
                               1000, 1009, 1024])
def test_fft64_matches_naive_dft(n):
    x = oracle.lcg_complex64(0x9E3779B97F4A7C15 ^ n, n)
    for inv in (False, True):
        d = oracle.naive_dft(x, inverse=inv)
        f = oracle.fft64(x, inverse=inv)
        assert np.max(np.abs(d - f)) <= 1e-12 * (1 + np.max(np.abs(d)))


@pytest.mark.parametrize("n", [4096, 65536, 107520, 3 * 5 * 7 * 64])
def test_fft64_matches_numpy(n):
    x = oracle.lcg_complex64(n, n).astype(np.complex128)
    assert oracle.max_rel(oracle.fft64(x), np.fft.fft(x)) < 1e-13
    assert oracle.max_rel(oracle.fft64(x, inverse=True), np.fft.ifft(x) * n) < 1e-13


def test_execute_reference_restatement(golden):
    """The radix-2 restatement of FftPlan::execute_reference (fft.hpp:417-460) against the DFT gate the reference
    applies to it (test_fft.cpp:215-219) and against the reference's FftPlan<float> outputs."""
    for n in (2, 16, 64, 1024):
        x = oracle.lcg_complex64(31337 + n, n)
        d = oracle.naive_dft(x)
        assert oracle.max_rel(oracle.execute_reference_f32(x), d) < 2e-4
        assert oracle.max_rel(oracle.execute_reference_f32(x, inverse=True), oracle.naive_dft(x, True)) < 2e-4
    for n in (16, 1024, 4096):
        x = golden[f"c2c_{n}_in"]
        assert oracle.max_rel(oracle.execute_reference_f32(x), golden[f"c2c_{n}_fwd"].astype(np.complex128)) < 2e-6


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 17, 100, 360, 1009, 1031, 4000])
def test_bluestein_restatement(n):
    """The reference's Bluestein sizes and gate (test_fft.cpp:582-658: f64 vs DFT at 1e-12); inverse normalised."""
    x = oracle.lcg_complex64(0x9E3779B97F4A7C15 ^ n, n)
    d = oracle.naive_dft(x)
    assert oracle.max_rel(oracle.bluestein64(x), d) < 1e-12
    assert oracle.max_rel(oracle.bluestein64(x, inverse=True), oracle.naive_dft(x, True) / n) < 1e-12


def test_golden_c2c_within_reference_class(golden):
    """The reference's f32 outputs agree with the FP64 oracle at its own f32 tolerance class."""
    for n in (16, 105, 240, 1024, 4096):
        x = golden[f"c2c_{n}_in"]
        want = oracle.fft64(x)
        assert oracle.max_rel(golden[f"c2c_{n}_fwd"], want) < oracle.f32_class(n)
        scale = 1.0 if (n & (n - 1)) == 0 else 1.0 / n  # FftPlan inverse unnormalised, Bluestein's normalised
        want_inv = oracle.fft64(x, inverse=True) * scale
        assert oracle.max_rel(golden[f"c2c_{n}_inv"], want_inv) < oracle.f32_class(n)


def test_real_restatement(golden):
    for n in (64, 1024):
        x = golden[f"rfft_{n}_in"].astype(np.float64)
        want = oracle.rfft64(x)
        np.testing.assert_allclose(want, np.fft.rfft(x), atol=1e-12 * n)
        assert oracle.max_rel(golden[f"rfft_{n}_out"], want) < 2e-4
        spec = golden[f"irfft_{n}_in"]
        back = oracle.irfft64(spec, n)
        np.testing.assert_allclose(back, np.fft.irfft(spec.astype(np.complex128), n), atol=1e-12)
        assert np.max(np.abs(golden[f"irfft_{n}_out"] - back)) < 2e-4 * (1 + np.max(np.abs(back)))


def test_nd_restatement(golden):
    for dims in ((8, 16), (4, 6, 5), (16, 12)):
        tag = "x".join(str(d) for d in dims)
        x = golden[f"nd_{tag}_in"]
        f = oracle.nd64(x)
        np.testing.assert_allclose(f, np.fft.fftn(x.astype(np.complex128)), atol=1e-10)
        i = oracle.nd64(x, inverse=True)
        np.testing.assert_allclose(i, np.fft.ifftn(x.astype(np.complex128)), atol=1e-12)
        assert oracle.max_rel(golden[f"nd_{tag}_fwd"], f) < 2e-4
        assert oracle.max_rel(golden[f"nd_{tag}_inv"], i) < 2e-4


def test_nd_axes_matches_strided_oracle():
    """The axis-by-axis N-D oracle used at the benchmark shapes agrees with the strided restatement (nd64)."""
    for dims in ((8, 16), (4, 6, 5), (16, 12), (32, 8, 64)):
        x = oracle.lcg_complex64(0xA0 + len(dims), int(np.prod(dims))).reshape(dims)
        np.testing.assert_allclose(oracle.nd64_axes(x), oracle.nd64(x), rtol=0, atol=1e-10)


def test_lcg_matches_reference_rule():
    """test_fft.cpp:31-44: first draws of the seed-0 stream, computed by hand."""
    s = 0
    vals = []
    for _ in range(4):
        s = (s * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        vals.append(np.float32((s >> 11) / float(1 << 53) * 2.0 - 1.0))
    np.testing.assert_array_equal(oracle.lcg_float32(0, 4), np.array(vals, dtype=np.float32))


def test_reference_library_when_built():
    """When the reference was compiled here, its self-check passes at every built level."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    R = oracle.ref()
    assert R.crdref_level() in (0, 3, 4)
    for level in (0, 3, 4):
        assert R.crdref_self_check_level(level) == 0


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_reference_shim_exits_cleanly_after_cached_plans():
    """The shim keeps per-thread plan caches across uneven-batch calls; a process that used them (the bench's CPU
    baseline) must exit without crashing in static destructors."""
    import subprocess
    import sys

    code = (
        "import sys, ctypes, numpy as np\n"
        f"sys.path.insert(0, {os.path.dirname(os.path.dirname(os.path.abspath(__file__)))!r})\n"
        "import oracle\n"
        "R = oracle.ref()\n"
        "s = np.array([16, 48, 1024, 1000, 4096, 105], dtype=np.int64)\n"
        "o = np.concatenate([[0], np.cumsum(s)[:-1]]).astype(np.int64)\n"
        "d = oracle.lcg_complex64(1, int(s.sum()))\n"
        "P = ctypes.POINTER(ctypes.c_int64)\n"
        "for _ in range(2):\n"
        "    R.crdref_uneven_f32(len(s), s.ctypes.data_as(P), o.ctypes.data_as(P),\n"
        "                        d.view(np.float32).ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 0, 4)\n"
        "print('done')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "done" in r.stdout, (r.returncode, r.stderr[-500:])
