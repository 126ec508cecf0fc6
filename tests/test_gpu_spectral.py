"""Device spectral estimators (crd_b200/csrc/spectral.cu, crdfft_spectral_*) against the FP64 oracle
(oracle/spectral.py, itself pinned to the reference's scipy vectors and its own functions) and against those vectors
directly. FP32 on the device: rel-L2 <= 1e-6 over each PSD row set against FP64 (the periodograms are squared
magnitudes, so about twice the FFT's relative error)."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle
from oracle import spectral as S

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "spectral_refs.npz"))
REL_L2 = 1e-6


def _rl2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_reference_vectors():
    x = torch.from_numpy(GOLD["welch_x"].astype(np.float32)).cuda()
    w = cf.welch_psd(x, 100.0, 64).cpu().numpy()
    s = cf.spectrogram(x, 100.0, 64, 32).cpu().numpy()
    p = cf.periodogram(x, 100.0).cpu().numpy()
    assert s.shape == (int(GOLD["spec_nseg"]), int(GOLD["spec_nfreq"]))
    # FP32 input and arithmetic against scipy's FP64 results
    assert _rl2(w, GOLD["welch_pxx"]) <= 2e-6
    assert _rl2(s.ravel(), GOLD["spec"]) <= 2e-6
    assert _rl2(p, GOLD["periodogram"]) <= 2e-6


@pytest.mark.parametrize("nsamples,nperseg,noverlap", [(100000, 1024, 512), (50000, 256, 0), (33333, 2048, 1500),
                                                        (20000, 2000, 1000), (9000, 64, 48), (4096, 16384, 0),
                                                        (70000, 4096, 1024), (12345, 126, 63)])
def test_welch_and_spectrogram_against_oracle(nsamples, nperseg, noverlap):
    count = 5
    rng = np.random.default_rng(nsamples ^ nperseg)
    x = (rng.normal(size=(count, nsamples)) + 0.7).astype(np.float32)
    t = torch.from_numpy(x).cuda()
    w = cf.welch_psd(t, 250.0, nperseg, noverlap).cpu().numpy()
    want = S.welch(x.astype(np.float64), 250.0, nperseg, noverlap)
    assert w.shape == want.shape
    if want.size and np.any(want):
        assert _rl2(w, want) <= REL_L2
    else:
        assert np.all(w == 0)
    ov = noverlap if noverlap else nperseg // 2
    if ov < nperseg:
        s = cf.spectrogram(t, 250.0, nperseg, ov).cpu().numpy()
        ws = S.spectrogram(x.astype(np.float64), 250.0, nperseg, ov)
        assert s.shape == ws.shape
        if ws.size:
            assert _rl2(s, ws) <= REL_L2


@pytest.mark.parametrize("n", [64, 1000, 4096, 16384])
def test_periodogram_against_oracle(n):
    rng = np.random.default_rng(n)
    x = (rng.normal(size=(7, n)) - 0.2).astype(np.float32)
    p = cf.periodogram(torch.from_numpy(x).cuda(), 3.0).cpu().numpy()
    assert _rl2(p, S.periodogram(x.astype(np.float64), 3.0)) <= REL_L2


def test_custom_window_no_detrend_and_odd_offsets():
    """A caller's window, no detrend, and signals whose segments start on odd float offsets (nsamples odd)."""
    count, nsamples, nperseg, noverlap = 3, 10001, 512, 301
    rng = np.random.default_rng(1)
    x = (rng.normal(size=(count, nsamples)) + 2.0).astype(np.float32)
    win = np.blackman(nperseg).astype(np.float32)
    plan = cf.SpectralPlan(cf.SPECTRAL_SPECTROGRAM, nsamples, count, 10.0, nperseg, noverlap, window=win,
                           detrend=False)
    got = plan.execute(torch.from_numpy(x).cuda()).cpu().numpy()
    want = S.spectrogram(x.astype(np.float64), 10.0, nperseg, noverlap, window=win.astype(np.float64),
                         detrend=False)
    assert _rl2(got, want) <= REL_L2


def test_welch_is_deterministic_and_matches_reference_f32():
    count, nsamples = 4, 1 << 16
    rng = np.random.default_rng(2)
    x = rng.normal(size=(count, nsamples)).astype(np.float32)
    t = torch.from_numpy(x).cuda()
    plan = cf.SpectralPlan(cf.SPECTRAL_WELCH, nsamples, count, 1.0, 1024, 512)
    a = plan.execute(t).cpu().numpy()
    b = plan.execute(t).cpu().numpy()
    assert np.array_equal(a, b)
    if oracle.ref_available():
        r = oracle.ref_welch(x, 1.0, 1024, 512, f32=True)
        assert _rl2(a, r.astype(np.float64)) <= 2e-6


def test_short_signal_gives_zeros_and_errors():
    t = torch.ones(3, 100, device="cuda")
    assert torch.all(cf.welch_psd(t, 1.0, 256) == 0)
    assert cf.spectrogram(t, 1.0, 256, 128).shape == (3, 0, 129)
    with pytest.raises(cf.CrdFftError):
        cf.SpectralPlan(cf.SPECTRAL_WELCH, 1000, 1, 1.0, 255)       # odd segment length
    with pytest.raises(cf.CrdFftError):
        cf.SpectralPlan(cf.SPECTRAL_WELCH, 1000, 1, 1.0, 256, 256)  # no hop
    with pytest.raises(cf.CrdFftError):
        cf.SpectralPlan(cf.SPECTRAL_WELCH, 1000, 1, 0.0, 256)       # fs
    plan = cf.SpectralPlan(cf.SPECTRAL_WELCH, 1000, 1, 1.0, 256)
    x = torch.zeros(1000, device="cuda")
    assert cf.hesap.lib().crdfft_execute(plan._h, x.data_ptr(), x.data_ptr(), 0, None) == 7  # CRDFFT_INVALID_ARG
