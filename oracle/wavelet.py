"""FP64 restatement of crd-hesap-wavelet's continuous wavelet transform, for tests only.

TEST INFRASTRUCTURE: the checker for the device CWT (crdfft_cwt_*). Nothing in the product imports it.

Follows engine/numerics/hesap-wavelet/include/crd/hesap/wavelet/cwt.hpp:
- continuous_wavelet (cwt.hpp:300-407): pywt-style names "mexh", "morl", "cmorB-C", "gausP", "cgauP", "shanB-C",
  "fbspM-B-C", "paulM" with their sampling intervals;
- sample_psi (cwt.hpp:149-280): the wavelet on linspace(lower, upper, 2^precision), L2-normalised for gaus/cgau;
- central_frequency (cwt.hpp:410-438): the peak bin of |FFT(psi)|^2 over k >= 1, folded, / (upper - lower);
- cwt_arm (cwt.hpp:461-614): the integrated wavelet (cumulative sum x step, conjugated for complex wavelets), per
  scale a kernel of kk taps sampled at floor(m / (a step)) and reversed, the product of its FFT with the data's
  FFT (length lfft = the power of two >= n + max kk), the inverse, and -sqrt(a) (w[t+1] - w[t]) / lfft at
  t = (kk - 2) / 2 + i; scales with kk < 2 give zeros.
Pinned to the pywt vectors of the reference's tests (tests/numerics/hesap-wavelet/cwt_refs.inc, through
tests/golden/cwt_refs.npz).
"""

from __future__ import annotations

import math

import numpy as np


def _number(name: str, pos: int) -> tuple[float, int]:
    """The decimal at name[pos:] (cwt.hpp:282-306: optional '-', digits, optional '.digits')."""
    sign = 1.0
    if pos < len(name) and name[pos] == "-":
        sign, pos = -1.0, pos + 1
    v = 0.0
    while pos < len(name) and name[pos].isdigit():
        v, pos = v * 10.0 + float(ord(name[pos]) - 48), pos + 1
    if pos < len(name) and name[pos] == ".":
        pos += 1
        frac = 0.1
        while pos < len(name) and name[pos].isdigit():
            v += float(ord(name[pos]) - 48) * frac
            frac *= 0.1
            pos += 1
    return sign * v, pos


def _numbers(name: str, pos: int, k: int) -> list[float]:
    out = []
    for i in range(k):
        v, pos = _number(name, pos)
        out.append(v)
        if pos < len(name) and name[pos] == "-":
            pos += 1
    return out


def continuous_wavelet(name: str) -> dict:
    """The wavelet descriptor of a pywt-style name (cwt.hpp:300-407)."""
    w = dict(kind="mexh", lower=-8.0, upper=8.0, bandwidth=1.0, center=1.0, order=0, complex=False, l2=False)
    if name in ("mexh", "morl"):
        w["kind"] = name
    elif name.startswith("cmor"):
        b, c = _numbers(name, 4, 2)
        w.update(kind="cmor", bandwidth=b, center=c, complex=True)
    elif name.startswith("cgau"):
        w.update(kind="cgau", lower=-5.0, upper=5.0, order=int(_number(name, 4)[0]), complex=True, l2=True)
    elif name.startswith("gaus"):
        w.update(kind="gaus", lower=-5.0, upper=5.0, order=int(_number(name, 4)[0]), l2=True)
    elif name.startswith("shan"):
        b, c = _numbers(name, 4, 2)
        w.update(kind="shan", lower=-20.0, upper=20.0, bandwidth=b, center=c, complex=True)
    elif name.startswith("fbsp"):
        m, b, c = _numbers(name, 4, 3)
        w.update(kind="fbsp", lower=-20.0, upper=20.0, order=int(m), bandwidth=b, center=c, complex=True)
    elif name.startswith("paul"):
        order = int(_number(name, 4)[0]) if len(name) > 4 else 4
        w.update(kind="paul", lower=-12.0, upper=12.0, order=order, complex=True)
    return w


def _gauss_poly(p: int, complex_phase: bool) -> np.ndarray:
    """Ascending coefficients of the p-th derivative of exp(-x^2) (or exp(-x^2 - i x)) over that exponential:
    D_{k+1} = D_k' + (-2x [- i]) D_k, D_0 = 1 (cwt.hpp:86-147)."""
    c = np.zeros(1, dtype=np.complex128)
    c[0] = 1.0
    for _ in range(p):
        nxt = np.zeros(len(c) + 1, dtype=np.complex128)
        nxt[:-2] += np.arange(1, len(c)) * c[1:]
        nxt[1:] += -2.0 * c
        if complex_phase:
            nxt[:-1] += -1j * c
        c = nxt
    return c


def _sinc(x: np.ndarray) -> np.ndarray:
    return np.sinc(x)  # sin(pi x) / (pi x), 1 at 0: the reference's np_sinc (cwt.hpp:76-84)


def sample_psi(w: dict, grid_n: int) -> np.ndarray:
    """psi on linspace(lower, upper, grid_n) (cwt.hpp:149-280)."""
    step = (w["upper"] - w["lower"]) / (grid_n - 1)
    t = w["lower"] + np.arange(grid_n, dtype=np.float64) * step
    pi = math.pi
    k = w["kind"]
    if k == "mexh":
        c = 2.0 / (math.sqrt(3.0) * pi ** 0.25)
        v = c * (1.0 - t * t) * np.exp(-t * t / 2.0) + 0j
    elif k == "morl":
        v = np.exp(-t * t / 2.0) * np.cos(5.0 * t) + 0j
    elif k == "cmor":
        amp = (pi * w["bandwidth"]) ** -0.5 * np.exp(-t * t / w["bandwidth"])
        v = amp * np.exp(1j * 2.0 * pi * w["center"] * t)
    elif k == "gaus":
        poly = np.polynomial.polynomial.polyval(t, _gauss_poly(w["order"], False).real)
        sign = -1.0 if (w["order"] // 2) & 1 else 1.0
        v = sign * poly * np.exp(-t * t) + 0j
    elif k == "cgau":
        poly = np.polynomial.polynomial.polyval(t, _gauss_poly(w["order"], True))
        v = poly * np.exp(-t * t) * np.exp(-1j * t)
    elif k == "shan":
        amp = math.sqrt(w["bandwidth"]) * _sinc(w["bandwidth"] * t)
        v = amp * np.exp(1j * 2.0 * pi * w["center"] * t)
    elif k == "fbsp":
        m = w["order"]
        amp = math.sqrt(w["bandwidth"]) * _sinc(w["bandwidth"] * t / m) ** m
        v = amp * np.exp(1j * 2.0 * pi * w["center"] * t)
    else:  # paul: 2^m i^m m! / sqrt(pi (2m)!) (1 - i t)^-(m+1)
        m = w["order"]
        norm = 2.0 ** m * math.factorial(m) / math.sqrt(pi * math.factorial(2 * m))
        v = norm * (1j ** m) * (1.0 - 1j * t) ** (-(m + 1.0))
    v = np.asarray(v, dtype=np.complex128)
    if w["l2"]:
        v = v / math.sqrt(float(np.sum(np.abs(v) ** 2) * step))
    return v


def central_frequency(w: dict, precision: int = 12) -> float:
    """Peak of |FFT(psi)|^2 over k >= 1 (first maximum), folded into the lower half (cwt.hpp:410-438)."""
    n = 1 << precision
    spec = np.fft.fft(sample_psi(w, n))
    mag = spec.real ** 2 + spec.imag ** 2
    bin_ = 1 + int(np.argmax(mag[1:]))
    index = bin_ + 1
    if index > n / 2.0:
        index = n - index + 2
    return (index - 1) / (w["upper"] - w["lower"])


def kernel_taps(a: float, step: float, xrange_: float, grid_n: int) -> int:
    """kk: the taps of the scale-a kernel, m < ceil(a xrange + 1) with floor(m / (a step)) < grid_n (cwt.hpp:488-501)."""
    count_raw = int(math.ceil(a * xrange_ + 1.0))
    kk = 0
    for m in range(count_raw):
        if int(float(m) / (a * step)) >= grid_n:
            break
        kk += 1
    return kk


def geometry(n: int, scales, name: str, precision: int = 12) -> tuple[int, list[int]]:
    """(lfft, kk per scale)."""
    w = continuous_wavelet(name)
    grid_n = 1 << precision
    step = (w["upper"] - w["lower"]) / (grid_n - 1)
    kks = [kernel_taps(float(a), step, w["upper"] - w["lower"], grid_n) for a in scales]
    kmax = max([1] + kks)
    lfft = 1
    while lfft < n + kmax:
        lfft <<= 1
    return lfft, kks


def cwt(x, scales, name: str, sampling_period: float = 1.0, precision: int = 12):
    """(coeffs [nscales, n] complex128, frequencies [nscales]) of one real signal, in FP64 (cwt.hpp:461-614)."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    w = continuous_wavelet(name)
    grid_n = 1 << precision
    step = (w["upper"] - w["lower"]) / (grid_n - 1)
    psi = sample_psi(w, grid_n)
    int_psi = np.cumsum(psi) * step
    if w["complex"]:
        int_psi = np.conj(int_psi)
    lfft, kks = geometry(n, scales, name, precision)
    data = np.zeros(lfft, dtype=np.complex128)
    data[:n] = x
    data_f = np.fft.fft(data)
    fc = central_frequency(w, precision)
    out = np.zeros((len(scales), n), dtype=np.complex128)
    for s, a in enumerate(scales):
        a = float(a)
        kk = kks[s]
        if kk < 2:
            continue
        m = kk - 1 - np.arange(kk)
        j = (m.astype(np.float64) / (a * step)).astype(np.int64)
        kb = np.zeros(lfft, dtype=np.complex128)
        kb[:kk] = int_psi[j]
        wb = np.fft.ifft(np.fft.fft(kb) * data_f) * lfft  # the reference's inverse is unnormalised
        off = (kk - 2) // 2
        t = off + np.arange(n)
        out[s] = -math.sqrt(a) * (wb[t + 1] - wb[t]) / lfft
    freqs = np.array([fc / (float(a) * sampling_period) for a in scales])
    return out, freqs
