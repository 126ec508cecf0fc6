"""CPU tests of the continuous wavelet transform: the FP64 oracle pinned to the pywt vectors of the reference's
tests (tests/numerics/hesap-wavelet/test_cwt.cpp:31-98 with cwt_refs.inc, stored in tests/golden/cwt_refs.npz),
its tone-localisation gate (test_cwt.cpp:100-145), and the library's host-only parts (frequencies, FFT length,
descriptor validation), which need no device."""

from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import pytest

import oracle
from crd_b200 import _lib
from oracle import wavelet as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cwt_refs.npz")

# (name, golden key, complex coefficients, frequency tolerance) as test_cwt.cpp:45-46, 78-81 lists them
CASES = [
    ("mexh", "mexh", False, 1e-9),
    ("morl", "morl", False, 1e-9),
    ("gaus2", "gaus2", False, 1e-9),
    ("gaus4", "gaus4", False, 1e-9),
    ("cmor1.5-1.0", "cmor1_5_1_0", True, 1e-7),
    ("cgau2", "cgau2", True, 1e-7),
    ("shan1.0-0.5", "shan1_0_0_5", True, 1e-7),
    ("fbsp2-1.0-0.5", "fbsp2_1_0_0_5", True, 1e-7),
]


def golden_coeffs(g, key, cplx, ns, n):
    v = g[key]
    c = v[0::2] + 1j * v[1::2] if cplx else v + 0j
    return c.reshape(ns, n)


@pytest.mark.parametrize("name,key,cplx,ftol", CASES)
def test_oracle_matches_pywt_vectors(name, key, cplx, ftol):
    g = np.load(GOLDEN)
    x, scales = g["input"], g["scales"]
    coeffs, freqs = W.cwt(x, scales, name)
    want = golden_coeffs(g, key, cplx, len(scales), len(x))
    # the reference's own gate: 1e-8 absolute on every coefficient (test_cwt.cpp:57-58, 93-94)
    assert np.abs(coeffs.real - want.real).max() <= 1e-8
    assert np.abs(coeffs.imag - want.imag).max() <= 1e-8
    assert np.abs(freqs - g[key + "_freqs"]).max() <= ftol


@pytest.mark.parametrize("name", ["morl", "paul4"])
def test_oracle_tone_localises_to_its_scale(name):
    """A tone of frequency f0 peaks near scale fc / f0 (test_cwt.cpp:100-145)."""
    n, f0, ns = 512, 0.05, 48
    x = np.cos(2.0 * math.pi * f0 * np.arange(n))
    scales = 64.0 ** (np.arange(ns) / (ns - 1))
    coeffs, _ = W.cwt(x, scales, name)
    power = (np.abs(coeffs[:, n // 4: 3 * n // 4]) ** 2).sum(axis=1)
    expected = W.central_frequency(W.continuous_wavelet(name)) / f0
    peak = scales[int(np.argmax(power))]
    assert expected * 0.7 < peak < expected * 1.43


def _desc(name, scales, n=96, count=1, precision=0, period=0.0):
    d = _lib.CwtDesc()
    d.wavelet = name.encode()
    d.scales = scales.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.nsamples, d.count, d.nscales = n, count, len(scales)
    d.precision, d.sampling_period = precision, period
    return d


def test_cwt_descriptor_layout():
    # two pointers + 3 int64 + double + 2 int32 = 56 bytes
    assert ctypes.sizeof(_lib.CwtDesc) == 56


@pytest.mark.parametrize("name,key,cplx,ftol", CASES + [("paul4", None, True, 0.0)])
def test_library_frequencies_and_fft_length_without_device(name, key, cplx, ftol):
    L = _lib.lib()
    g = np.load(GOLDEN)
    scales = np.ascontiguousarray(g["scales"], dtype=np.float64)
    d = _desc(name, scales, period=0.5)
    out = np.zeros(len(scales))
    assert L.crdfft_cwt_frequencies(ctypes.byref(d), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == _lib.OK
    _, want = W.cwt(g["input"], scales, name, sampling_period=0.5)
    np.testing.assert_allclose(out, want, rtol=1e-14, atol=0)
    if key is not None:
        np.testing.assert_allclose(out * 0.5, g[key + "_freqs"], rtol=0, atol=ftol)
    for n in (96, 1000, 5000):
        d.nsamples = n
        assert L.crdfft_cwt_fft_length(ctypes.byref(d)) == W.geometry(n, scales, name)[0]


def test_library_tap_counts_follow_the_reference_rule():
    """The FFT length depends on the longest kernel's tap count; a scale too small for two taps (kk < 2) is allowed
    and gives zero coefficients (cwt.hpp:561-567)."""
    L = _lib.lib()
    for name in ("mexh", "shan1.0-0.5", "paul4"):
        for top in (0.01, 1.0, 3.7, 100.0, 1000.0):
            scales = np.array([0.01, top], dtype=np.float64)
            d = _desc(name, scales, n=777)
            assert L.crdfft_cwt_fft_length(ctypes.byref(d)) == W.geometry(777, scales, name)[0]
    assert W.geometry(10, [0.01], "mexh")[1] == [1]


def test_cwt_invalid_descriptors_rejected_without_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    ok = np.array([1.0, 2.0])
    assert L.crdfft_cwt_plan_create(None, ctypes.byref(h)) == _lib.INVALID_ARG
    for bad in (_desc("morl", ok, n=0), _desc("morl", ok, count=0), _desc("morl", ok, precision=25),
                _desc("morl", ok, period=-1.0), _desc("gaus16", ok), _desc("morl", np.array([1.0, -2.0])),
                _desc("morl", np.array([1.0, float("nan")]))):
        assert L.crdfft_cwt_plan_create(ctypes.byref(bad), ctypes.byref(h)) == _lib.INVALID_DESC
        assert L.crdfft_cwt_fft_length(ctypes.byref(bad)) == -1
    huge = _desc("morl", np.array([1e8]))
    assert L.crdfft_cwt_plan_create(ctypes.byref(huge), ctypes.byref(h)) == _lib.UNSUPPORTED_SIZE
    assert L.crdfft_cwt_execute(None, None, None, None) == _lib.INVALID_ARG
    assert L.crdfft_cwt_plan_destroy(None) == _lib.OK


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("name", ["mexh", "morl", "gaus4", "cmor1.5-1.0", "cgau2", "shan1.0-0.5", "fbsp2-1.0-0.5",
                                  "paul4"])
def test_reference_cwt_f32_agrees_with_the_oracle(name):
    """The reference's own cwt<float>, compiled from its sources (oracle/_ref), against the FP64 restatement: the
    same steps, so only FP32 rounding separates them (measured 3e-7 to 2e-6)."""
    rng = np.random.default_rng(11)
    x = rng.standard_normal((2, 700)).astype(np.float32)
    scales = np.geomspace(1.0, 40.0, 12).astype(np.float32)
    got, freqs = oracle.ref_cwt(x, scales, name, threads=2)
    for c in range(2):
        want, wf = W.cwt(x[c].astype(np.float64), scales.astype(np.float64), name)
        assert np.linalg.norm(got[c] - want) / np.linalg.norm(want) <= 2e-5
    np.testing.assert_allclose(freqs, wf, rtol=1e-6)
