"""TEST INFRASTRUCTURE ONLY: an FP64 numpy restatement of the reference's spectral estimators (yatiyr/CRD
engine/numerics/hesap-dsp/include/crd/hesap/dsp/spectral.hpp), the checker of crd_b200's device spectral kernels.

The FFT inside is numpy's FP64 real FFT; what is restated here is everything around it: segmenting, the
'constant' detrend, the periodic Hann window, the density scale and the one-sided doubling, and the fixed-order
average. Pinned against the reference tests' scipy vectors (tests/golden/spectral_refs.npz) and, where
oracle/_ref was built, against the reference's own functions.
"""

from __future__ import annotations

import numpy as np


def general_cosine(m: int, a, sym: bool = True) -> np.ndarray:
    """w[i] = sum_k a[k] cos(k fac[i]), fac = -pi + 2 pi i / (N - 1); a periodic window (sym=False) takes N = m + 1
    and drops the last sample (windows.hpp:56-115)."""
    n = m if sym else m + 1
    if n == 1:
        return np.ones(m)
    i = np.arange(m, dtype=np.float64)
    fac = -np.pi + 2.0 * np.pi * i / (n - 1)
    w = np.zeros(m)
    for k, ak in enumerate(a):
        w += ak * np.cos(k * fac)
    return w


def hann_periodic(m: int) -> np.ndarray:
    """hann(m, sym=false) (windows.hpp:120-124)."""
    return general_cosine(m, (0.5, 0.5), sym=False)


def segment_count(nsamples: int, nperseg: int, noverlap: int) -> int:
    """nseg = (n - noverlap) / hop, 0 when n < nperseg (spectral.hpp:52-54)."""
    hop = nperseg - noverlap
    return 0 if nsamples < nperseg else (nsamples - noverlap) // hop


def segment_periodograms(x, fs: float, nperseg: int, noverlap: int, window=None, detrend: bool = True):
    """The per-segment one-sided density periodograms, nseg x (nperseg/2 + 1) (spectral.hpp:44-120): each segment
    minus its mean, times the window, rfft, scale / (fs sum w^2) times |X|^2, doubled except at DC and Nyquist."""
    x = np.asarray(x, dtype=np.float64)
    hop = nperseg - noverlap
    nfreq = nperseg // 2 + 1
    nseg = segment_count(x.shape[-1], nperseg, noverlap)
    win = hann_periodic(nperseg) if window is None else np.asarray(window, dtype=np.float64)
    scale = 1.0 / (fs * np.sum(win * win))
    lead = x.shape[:-1]
    out = np.zeros(lead + (nseg, nfreq))
    for s in range(nseg):
        seg = x[..., s * hop:s * hop + nperseg]
        if detrend:
            seg = seg - seg.mean(axis=-1, keepdims=True)
        X = np.fft.rfft(seg * win, axis=-1)
        p = scale * (X.real ** 2 + X.imag ** 2)
        p[..., 1:nfreq - 1] *= 2.0  # every bin but k = 0 and k = nfreq - 1 (spectral.hpp:107-111)
        out[..., s, :] = p
    return out


def spectrogram(x, fs: float, nperseg: int, noverlap: int, window=None, detrend: bool = True):
    """spectrogram (spectral.hpp:177-183): the matrix of segment_periodograms."""
    return segment_periodograms(x, fs, nperseg, noverlap, window, detrend)


def welch(x, fs: float, nperseg: int, noverlap: int = 0, window=None, detrend: bool = True):
    """welch_psd (spectral.hpp:141-172): noverlap 0 means nperseg/2; the periodograms summed in segment order, then
    divided by nseg (zeros when there is no segment)."""
    if noverlap == 0:
        noverlap = nperseg // 2
    pg = segment_periodograms(x, fs, nperseg, noverlap, window, detrend)
    nseg = pg.shape[-2]
    if nseg == 0:
        return np.zeros(pg.shape[:-2] + (nperseg // 2 + 1,))
    acc = np.zeros(pg.shape[:-2] + (pg.shape[-1],))
    for s in range(nseg):
        acc += pg[..., s, :]
    return acc / nseg


def periodogram(x, fs: float):
    """periodogram (spectral.hpp:188-220): one segment of the whole signal, boxcar window, mean removed,
    |rfft|^2 / (fs n), doubled except at DC and Nyquist."""
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[-1]
    return segment_periodograms(x, fs, n, 0, np.ones(n), True)[..., 0, :]
