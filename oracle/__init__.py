"""TEST INFRASTRUCTURE ONLY: the CPU checkers of the GPU FFT path.

Two checkers, loaded with ctypes:

* ``liboracle.so`` (oracle.c): plain-C restatements of the reference's algorithms (yatiyr/CRD,
  engine/numerics/hesap-fft): an FP64 brute-force DFT (tests/numerics/hesap-fft/test_fft.cpp:47-65), an FP64
  mixed-radix self-sorting FFT, the radix-2 ``execute_reference`` (include/crd/hesap/fft/fft.hpp:417-460),
  Bluestein (bluestein.hpp:29-136), the real FFT (real_fft.hpp:41-92) and the N-D plan (nd_fft.hpp:105-182), and
  the reference tests' LCG inputs (test_fft.cpp:31-44).
* ``_ref/libcrdref.so`` (ref_shim.cpp + the reference's own sources, built by ``make ref``): the reference
  implementation itself, run on the host CPU. Present where it was built; it travels with the repository copy.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` import this package. The
product (``crd_b200``) never does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcrdref.so")

_lib = None
_ref = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_sz = ctypes.c_size_t


def build() -> str:
    """Compile liboracle.so (seconds) if it is missing or stale."""
    src = os.path.join(HERE, "oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_lcg_fill_f64.argtypes = [ctypes.c_uint64, _sz, _dp]
        L.orc_lcg_fill_f32.argtypes = [ctypes.c_uint64, _sz, _fp]
        L.orc_gauss_fill_f32.argtypes = [ctypes.c_uint64, _sz, _fp]
        L.orc_naive_dft.argtypes = [_sz, _dp, _dp, ctypes.c_int]
        L.orc_fft_f64.argtypes = [_sz, _dp, _dp, ctypes.c_int]
        L.orc_fft_f64.restype = ctypes.c_int
        L.orc_fft_batch_f64.argtypes = [_sz, _sz, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.orc_fft_batch_f64.restype = ctypes.c_int
        L.orc_execute_reference_f32.argtypes = [_sz, _fp, ctypes.c_int]
        L.orc_execute_reference_f32.restype = ctypes.c_int
        L.orc_execute_reference_f64.argtypes = [_sz, _dp, ctypes.c_int]
        L.orc_execute_reference_f64.restype = ctypes.c_int
        L.orc_bluestein_f64.argtypes = [_sz, _dp, ctypes.c_int]
        L.orc_bluestein_f64.restype = ctypes.c_int
        L.orc_rfft_f64.argtypes = [_sz, _dp, _dp]
        L.orc_rfft_f64.restype = ctypes.c_int
        L.orc_irfft_f64.argtypes = [_sz, _dp, _dp]
        L.orc_irfft_f64.restype = ctypes.c_int
        L.orc_nd_f64.argtypes = [_sz, ctypes.POINTER(ctypes.c_size_t), _dp, ctypes.c_int]
        L.orc_nd_f64.restype = ctypes.c_int
        L.orc_rel_l2_f32.argtypes = [_sz, _fp, _dp]
        L.orc_rel_l2_f32.restype = ctypes.c_double
        L.orc_max_rel_f32.argtypes = [_sz, _fp, _dp]
        L.orc_max_rel_f32.restype = ctypes.c_double
        _lib = L
    return _lib


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


def _ptr_d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _ptr_f(a: np.ndarray):
    return a.ctypes.data_as(_fp)


# ---- inputs ---------------------------------------------------------------------------------------------------------


def lcg_complex64(seed: int, count: int) -> np.ndarray:
    """count complex64 values, re/im interleaved draws of the reference tests' LCG (test_fft.cpp:31-44)."""
    out = np.empty(2 * count, dtype=np.float32)
    lib().orc_lcg_fill_f32(seed & 0xFFFFFFFFFFFFFFFF, 2 * count, _ptr_f(out))
    return out.view(np.complex64)


def lcg_float32(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float32)
    lib().orc_lcg_fill_f32(seed & 0xFFFFFFFFFFFFFFFF, count, _ptr_f(out))
    return out


def gauss_complex64(seed: int, count: int) -> np.ndarray:
    out = np.empty(2 * count, dtype=np.float32)
    lib().orc_gauss_fill_f32(seed & 0xFFFFFFFFFFFFFFFF, 2 * count, _ptr_f(out))
    return out.view(np.complex64)


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def config_seed(config: int, transform: int = 0) -> int:
    """Seed of transform t of a benchmark configuration: 0x5EED0000 + c mixed with t by splitmix64."""
    return splitmix64((0x5EED0000 + config) ^ (transform * 0x9E3779B97F4A7C15 & 0xFFFFFFFFFFFFFFFF))


# ---- FP64 transforms ---------------------------------------------------------------------------------------------


def naive_dft(x, inverse: bool = False) -> np.ndarray:
    x = _c128(x)
    y = np.empty_like(x)
    lib().orc_naive_dft(x.size, _ptr_d(x), _ptr_d(y), int(inverse))
    return y


def fft64(x, inverse: bool = False) -> np.ndarray:
    """FP64 mixed-radix FFT along the last axis (unnormalised both ways)."""
    x = _c128(x)
    n = x.shape[-1]
    batch = x.size // n if n else 0
    y = np.empty_like(x)
    threads = min(8, max(1, batch))
    rc = lib().orc_fft_batch_f64(n, batch, _ptr_d(x), _ptr_d(y), int(inverse), threads)
    if rc != 0:
        raise RuntimeError(f"orc_fft_batch_f64 failed ({rc})")
    return y


def execute_reference_f32(x, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex64).copy()
    if lib().orc_execute_reference_f32(a.size, _ptr_f(a.view(np.float32)), int(inverse)) != 0:
        raise ValueError("power of two only")
    return a


def bluestein64(x, inverse: bool = False) -> np.ndarray:
    a = _c128(x).copy()
    lib().orc_bluestein_f64(a.size, _ptr_d(a), int(inverse))
    return a


def rfft64(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    rows = x.reshape(-1, n)
    out = np.empty((rows.shape[0], n // 2 + 1), dtype=np.complex128)
    for i in range(rows.shape[0]):
        r = np.ascontiguousarray(rows[i])
        o = out[i]
        lib().orc_rfft_f64(n, r.ctypes.data_as(_dp), o.ctypes.data_as(_dp))
    return out.reshape(x.shape[:-1] + (n // 2 + 1,))


def irfft64(x, n: int) -> np.ndarray:
    x = _c128(x)
    rows = x.reshape(-1, n // 2 + 1)
    out = np.empty((rows.shape[0], n), dtype=np.float64)
    for i in range(rows.shape[0]):
        r = np.ascontiguousarray(rows[i])
        o = out[i]
        lib().orc_irfft_f64(n, r.ctypes.data_as(_dp), o.ctypes.data_as(_dp))
    return out.reshape(x.shape[:-1] + (n,))


def nd64(x, inverse: bool = False) -> np.ndarray:
    a = _c128(x).copy()
    dims = (ctypes.c_size_t * a.ndim)(*a.shape)
    lib().orc_nd_f64(a.ndim, dims, _ptr_d(a), int(inverse))
    return a


def nd64_axes(x) -> np.ndarray:
    """Forward FP64 N-D FFT of a large array, axis by axis with the oracle's threaded batch FFT (fft64): the
    row-column order of NdFftPlan::execute (nd_fft.hpp:105-182, one batch of lines per axis, last axis first),
    for shapes whose strided single-threaded walk (nd64) would take minutes. Forward only, unnormalised."""
    a = _c128(x)
    for ax in range(a.ndim - 1, -1, -1):
        if a.shape[ax] < 2:
            continue
        moved = np.ascontiguousarray(np.moveaxis(a, ax, -1))
        a = np.moveaxis(fft64(moved), -1, ax)
    return np.ascontiguousarray(a)


# ---- metrics -----------------------------------------------------------------------------------------------------


def rel_l2(a, truth) -> float:
    a = np.asarray(a)
    truth = np.asarray(truth)
    num = np.linalg.norm((a.astype(np.complex128) - truth).ravel())
    den = np.linalg.norm(truth.ravel())
    return float(num / den) if den > 0 else float(num)


def max_rel(a, truth) -> float:
    """The reference tests' metric: max|a - b| / (1 + max|b|) (test_fft.cpp:68-96)."""
    a = np.asarray(a).astype(np.complex128)
    truth = np.asarray(truth)
    return float(np.max(np.abs(a - truth)) / (1.0 + np.max(np.abs(truth))))


def f32_class(n: int) -> float:
    """The reference's f32 tolerance class for the max_rel metric: 2e-4 below 2^19, 1e-3 from 2^19
    (tests/numerics/hesap-fft/test_fft_kernels.cpp:138-163)."""
    return 1e-3 if n >= (1 << 19) else 2e-4


# ---- the reference implementation itself ---------------------------------------------------------------------------


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """ctypes handle of the reference's own crd-hesap-fft (oracle/_ref/libcrdref.so)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        R = ctypes.CDLL(REF_SO)
        R.crdref_level.restype = ctypes.c_int
        R.crdref_self_check_level.argtypes = [ctypes.c_int]
        R.crdref_self_check_level.restype = ctypes.c_int
        R.crdref_plan_algorithm_f32.argtypes = [_sz]
        R.crdref_plan_algorithm_f32.restype = ctypes.c_char_p
        R.crdref_c2c_f32.argtypes = [_sz, _sz, _fp, ctypes.c_int, ctypes.c_int]
        R.crdref_c2c_f64.argtypes = [_sz, _sz, _dp, ctypes.c_int, ctypes.c_int]
        R.crdref_execute_reference_f32.argtypes = [_sz, _fp, ctypes.c_int]
        R.crdref_execute_reference_f64.argtypes = [_sz, _dp, ctypes.c_int]
        R.crdref_execute_batched_f32.argtypes = [_sz, _sz, _fp, ctypes.c_int]
        R.crdref_stockham_f32.argtypes = [_sz, _sz, _fp, ctypes.c_int]
        R.crdref_rfft_f32.argtypes = [_sz, _sz, _fp, _fp, ctypes.c_int]
        R.crdref_irfft_f32.argtypes = [_sz, _sz, _fp, _fp, ctypes.c_int]
        R.crdref_nd_f32.argtypes = [_sz, ctypes.POINTER(ctypes.c_size_t), _fp, ctypes.c_int]
        R.crdref_nd_f64.argtypes = [_sz, ctypes.POINTER(ctypes.c_size_t), _dp, ctypes.c_int]
        R.crdref_uneven_f32.argtypes = [_sz, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), _fp,
                                        ctypes.c_int, ctypes.c_int]
        R.crdref_welch_f32.argtypes = [_sz, _sz, _fp, ctypes.c_double, _sz, _sz, _fp, ctypes.c_int]
        R.crdref_welch_f64.argtypes = [_sz, _sz, _dp, ctypes.c_double, _sz, _sz, _dp, ctypes.c_int]
        R.crdref_spectrogram_f64.argtypes = [_sz, _sz, _dp, ctypes.c_double, _sz, _sz, _dp, ctypes.c_int]
        R.crdref_periodogram_f64.argtypes = [_sz, _sz, _dp, ctypes.c_double, _dp, ctypes.c_int]
        R.crdref_cwt_f32.argtypes = [_sz, _sz, _fp, _fp, _sz, ctypes.c_char_p, _fp, _dp, ctypes.c_int]
        for f in ("crdref_c2c_f32", "crdref_c2c_f64", "crdref_execute_reference_f32", "crdref_execute_reference_f64",
                  "crdref_execute_batched_f32", "crdref_stockham_f32", "crdref_rfft_f32", "crdref_irfft_f32",
                  "crdref_nd_f32", "crdref_nd_f64", "crdref_uneven_f32", "crdref_welch_f32", "crdref_welch_f64",
                  "crdref_spectrogram_f64", "crdref_periodogram_f64", "crdref_cwt_f32"):
            getattr(R, f).restype = ctypes.c_int
        _ref = R
    return _ref


def ref_welch(x, fs: float, nperseg: int, noverlap: int, f32: bool = False, threads: int = 1) -> np.ndarray:
    """The reference's dsp::welch_psd over the rows of x (spectral.hpp:141-172), in float or double."""
    dt, fn = (np.float32, "crdref_welch_f32") if f32 else (np.float64, "crdref_welch_f64")
    a = np.ascontiguousarray(x, dtype=dt)
    n = a.shape[-1]
    out = np.zeros(a.shape[:-1] + (nperseg // 2 + 1,), dtype=dt)
    ptr = _ptr_f if f32 else _ptr_d
    if getattr(ref(), fn)(n, a.size // n, ptr(a), fs, nperseg, noverlap, ptr(out), threads) != 0:
        raise RuntimeError(f"{fn} failed")
    return out


def ref_cwt(x, scales, wavelet: str, threads: int = 1):
    """The reference's wavelet::cwt<float> over the rows of x (cwt.hpp:616-621): (coefficients rows x nscales x n
    complex64, frequencies)."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    sc = np.ascontiguousarray(scales, dtype=np.float32).reshape(-1)
    n = a.shape[-1]
    out = np.zeros(a.shape[:-1] + (len(sc), n), dtype=np.complex64)
    freqs = np.zeros(len(sc))
    if ref().crdref_cwt_f32(n, a.size // n, _ptr_f(a), _ptr_f(sc), len(sc), wavelet.encode(),
                            out.ctypes.data_as(_fp), _ptr_d(freqs), threads) != 0:
        raise RuntimeError("crdref_cwt_f32 failed")
    return out, freqs


def ref_spectrogram(x, fs: float, nperseg: int, noverlap: int, threads: int = 1) -> np.ndarray:
    """The reference's dsp::spectrogram<double> over the rows of x (spectral.hpp:177-183): rows x nseg x nfreq."""
    a = np.ascontiguousarray(x, dtype=np.float64)
    n = a.shape[-1]
    hop = nperseg - noverlap
    nseg = 0 if n < nperseg else (n - noverlap) // hop
    out = np.zeros(a.shape[:-1] + (nseg, nperseg // 2 + 1))
    if ref().crdref_spectrogram_f64(n, a.size // n, _ptr_d(a), fs, nperseg, noverlap, _ptr_d(out), threads) != 0:
        raise RuntimeError("crdref_spectrogram_f64 failed")
    return out


def ref_periodogram(x, fs: float, threads: int = 1) -> np.ndarray:
    """The reference's dsp::periodogram<double> over the rows of x (spectral.hpp:188-220)."""
    a = np.ascontiguousarray(x, dtype=np.float64)
    n = a.shape[-1]
    out = np.zeros(a.shape[:-1] + (n // 2 + 1,))
    if ref().crdref_periodogram_f64(n, a.size // n, _ptr_d(a), fs, _ptr_d(out), threads) != 0:
        raise RuntimeError("crdref_periodogram_f64 failed")
    return out


def ref_c2c_f32(x, inverse: bool = False, threads: int = 1) -> np.ndarray:
    """The reference's FftPlan<float> (power-of-two n) or BluesteinPlan<float> (other n) over the rows of x."""
    a = np.ascontiguousarray(x, dtype=np.complex64).copy()
    n = a.shape[-1]
    rc = ref().crdref_c2c_f32(n, a.size // n, _ptr_f(a.view(np.float32)), int(inverse), threads)
    if rc != 0:
        raise RuntimeError(f"crdref_c2c_f32 failed ({rc})")
    return a


def ref_rfft_f32(x, threads: int = 1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    n = x.shape[-1]
    batch = x.size // n
    out = np.empty(x.shape[:-1] + (n // 2 + 1,), dtype=np.complex64)
    rc = ref().crdref_rfft_f32(n, batch, _ptr_f(x), _ptr_f(out.view(np.float32)), threads)
    if rc != 0:
        raise RuntimeError(f"crdref_rfft_f32 failed ({rc})")
    return out


def ref_irfft_f32(x, n: int, threads: int = 1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex64)
    batch = x.size // (n // 2 + 1)
    out = np.empty(x.shape[:-1] + (n,), dtype=np.float32)
    rc = ref().crdref_irfft_f32(n, batch, _ptr_f(x.view(np.float32)), _ptr_f(out), threads)
    if rc != 0:
        raise RuntimeError(f"crdref_irfft_f32 failed ({rc})")
    return out


def ref_nd_f32(x, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex64).copy()
    dims = (ctypes.c_size_t * a.ndim)(*a.shape)
    rc = ref().crdref_nd_f32(a.ndim, dims, _ptr_f(a.view(np.float32)), int(inverse))
    if rc != 0:
        raise RuntimeError(f"crdref_nd_f32 failed ({rc})")
    return a
