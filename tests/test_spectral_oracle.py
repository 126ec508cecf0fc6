"""The spectral oracle (oracle/spectral.py) pinned: against the reference tests' scipy vectors
(tests/golden/spectral_refs.npz, made by tests/golden/make_spectral_golden.py) and, where oracle/_ref was built,
against the reference's own welch_psd / spectrogram / periodogram run here. CPU only."""

from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from oracle import spectral as S

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "spectral_refs.npz"))


def _close(a, b, rel, abs_):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= np.maximum(rel * np.abs(b), abs_))


def test_welch_matches_reference_vectors():
    # the reference test's case: fs = 100, nperseg = 64, default overlap (test_spectral.cpp:33-41, rel 1e-11)
    got = S.welch(GOLD["welch_x"], 100.0, 64)
    assert _close(got, GOLD["welch_pxx"], 1e-11, 0.0)


def test_spectrogram_matches_reference_vectors():
    got = S.spectrogram(GOLD["welch_x"], 100.0, 64, 32)
    assert got.shape == (int(GOLD["spec_nseg"]), int(GOLD["spec_nfreq"]))
    assert _close(got.ravel(), GOLD["spec"], 1e-9, 1e-11)  # test_spectral.cpp:79-92


def test_periodogram_matches_reference_vectors():
    got = S.periodogram(GOLD["welch_x"], 100.0)
    assert _close(got, GOLD["periodogram"], 1e-9, 1e-12)  # test_spectral.cpp:226-232


def test_window_and_segments():
    w = S.hann_periodic(8)
    assert np.allclose(w, 0.5 - 0.5 * np.cos(2 * np.pi * np.arange(8) / 8))
    assert S.segment_count(512, 64, 32) == 15 and S.segment_count(63, 64, 32) == 0
    assert np.all(S.welch(np.ones(10), 1.0, 64) == 0)  # no segment: zeros


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
# the reference's RealFftPlan takes powers of two: segment lengths, and the periodogram's whole length, are powers
@pytest.mark.parametrize("n,nperseg,noverlap", [(4096, 256, 128), (2048, 1024, 250), (1024, 64, 63), (512, 128, 0)])
def test_oracle_matches_reference_functions(n, nperseg, noverlap):
    rng = np.random.default_rng(n + nperseg)
    x = rng.normal(size=(3, n)) + 0.3
    assert _close(S.spectrogram(x, 8.0, nperseg, noverlap), oracle.ref_spectrogram(x, 8.0, nperseg, noverlap),
                  1e-9, 1e-15)
    ov = noverlap if noverlap else nperseg // 2  # welch_psd reads 0 as nperseg / 2
    assert _close(S.welch(x, 8.0, nperseg, ov), oracle.ref_welch(x, 8.0, nperseg, noverlap), 1e-9, 1e-15)
    assert _close(S.periodogram(x, 8.0), oracle.ref_periodogram(x, 8.0), 1e-9, 1e-15)


@needs_ref
def test_reference_welch_f32_close_to_oracle():
    rng = np.random.default_rng(5)
    x = rng.normal(size=(2, 8192)).astype(np.float32)
    got = oracle.ref_welch(x, 1.0, 1024, 512, f32=True)
    want = S.welch(x.astype(np.float64), 1.0, 1024, 512)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-5
