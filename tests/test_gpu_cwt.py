"""Device continuous wavelet transform (crdfft_cwt_*: cwt_plan.cpp; the fused line kernel in conv.cu, or cwt.cu's
product and epilogue around a batched inverse FFT plan) against
the FP64 oracle (oracle/wavelet.py, pinned to the reference tests' pywt vectors) and against those vectors
directly. FP32 kernels and FFTs against FP64: rel-L2 <= 2e-5 over each signal's coefficients and <= 1e-4 over each
scale (the epilogue differences neighbouring filtered samples, which costs up to about 30x the FFT's relative error
at the largest scales; an FP32 emulation of the same steps in numpy measures 0.4e-6 to 2.6e-6 overall and up to
8.5e-6 per scale on these cases)."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import crd_b200 as cf
from oracle import wavelet as W

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "cwt_refs.npz"))
REL_L2 = 2e-5
REL_L2_SCALE = 1e-4


def _check(got, want):
    assert got.shape == want.shape
    rel = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert rel <= REL_L2, rel
    for s in range(want.shape[0]):
        nrm = np.linalg.norm(want[s])
        if nrm == 0.0:
            assert not np.any(got[s]), f"scale {s} should be all zeros"
        else:
            assert np.linalg.norm(got[s] - want[s]) / nrm <= REL_L2_SCALE, s


@pytest.mark.parametrize("name,key,cplx", [
    ("mexh", "mexh", False), ("morl", "morl", False), ("gaus2", "gaus2", False), ("gaus4", "gaus4", False),
    ("cmor1.5-1.0", "cmor1_5_1_0", True), ("cgau2", "cgau2", True), ("shan1.0-0.5", "shan1_0_0_5", True),
    ("fbsp2-1.0-0.5", "fbsp2_1_0_0_5", True)])
def test_reference_vectors(name, key, cplx):
    x, scales = GOLD["input"], GOLD["scales"]
    v = GOLD[key]
    want = (v[0::2] + 1j * v[1::2] if cplx else v + 0j).reshape(len(scales), len(x))
    coeffs, freqs = cf.cwt(torch.from_numpy(x.astype(np.float32)).cuda(), scales, name)
    _check(coeffs.cpu().numpy().astype(np.complex128), want)
    np.testing.assert_allclose(freqs, GOLD[key + "_freqs"], rtol=0, atol=1e-7)


# (wavelet, n, scales, signals, fused): FFT lengths 512 .. 32768, real and complex wavelets, a scale too small for two
# taps; 4096 and 8192 run the fused line kernel, 16384 and 32768 the product / inverse FFT / epilogue rounds
CASES = [
    ("morl", 1000, np.geomspace(1.0, 128.0, 32), 3, True),
    ("cmor1.5-1.0", 4096, np.geomspace(0.5, 64.0, 48), 2, True),
    ("mexh", 3000, np.array([0.01, 0.3, 1.0, 2.0, 5.0, 20.0, 90.0]), 1, True),
    ("gaus4", 5000, np.geomspace(1.0, 256.0, 24), 2, True),
    ("paul4", 2048, np.geomspace(1.0, 100.0, 16), 1, True),
    ("fbsp2-1.0-0.5", 100, np.array([1.0, 2.0, 4.0]), 5, None),
    ("cgau2", 12000, np.geomspace(1.0, 64.0, 10), 1, False),
    ("shan1.0-0.5", 20000, np.geomspace(1.0, 64.0, 20), 2, False),
]


@pytest.mark.parametrize("name,n,scales,count,fused", CASES)
def test_against_oracle(name, n, scales, count, fused):
    rng = np.random.default_rng(n + count)
    x = rng.standard_normal((count, n)).astype(np.float32)
    plan = cf.CwtPlan(n, scales, name, count)
    assert plan.fft_length == W.geometry(n, scales, name)[0]
    assert plan.signals_per_round == count
    if fused is not None:
        assert plan.fused == fused
    got = plan.execute(torch.from_numpy(x).cuda()).cpu().numpy().astype(np.complex128)
    for c in range(count):
        want, freqs = W.cwt(x[c].astype(np.float64), scales, name)
        _check(got[c], want)
    np.testing.assert_allclose(plan.frequencies, freqs, rtol=1e-14, atol=0)


def test_signals_in_several_rounds():
    """More signals than 512 MiB of filtered sequences hold: full rounds and a shorter last one (its own inverse
    plan); signals at both ends of each round against the oracle."""
    n, scales = 6000, np.geomspace(1.0, 200.0, 96)  # FFT length 16384: 12 MiB a signal, 42 signals a round
    count = 45
    x = np.random.default_rng(5).standard_normal((count, n)).astype(np.float32)
    plan = cf.CwtPlan(n, scales, "morl", count)
    assert plan.fft_length == 16384 and plan.signals_per_round == 42 and not plan.fused
    got = plan.execute(torch.from_numpy(x).cuda()).cpu().numpy().astype(np.complex128)
    for c in (0, 41, 42, 44):
        want, _ = W.cwt(x[c].astype(np.float64), scales, "morl")
        _check(got[c], want)


def test_run_twice_bit_identical_and_stream_ordered():
    """The reference's run-twice gate (test_cwt.cpp:147-182): fixed schedules, no atomics."""
    n, scales = 3000, np.geomspace(1.0, 96.0, 40)
    x = torch.from_numpy(np.random.default_rng(7).standard_normal((2, n)).astype(np.float32)).cuda()
    plan = cf.CwtPlan(n, scales, "cmor1.5-1.0", 2)
    a = plan.execute(x).clone()
    side = torch.cuda.Stream()
    out = torch.empty_like(a)
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        plan.execute(x, out=out, stream=side)
    side.synchronize()
    assert torch.equal(a, out)
