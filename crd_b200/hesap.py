"""Python mirror of crd-hesap-fft's plan classes over the C ABI (include/crdfft.h), on CUDA tensors.

Each class keeps the reference's name, constructor meaning, verbs and normalisation
(engine/numerics/hesap-fft/include/crd/hesap/fft/):

* ``FftPlan(n)`` - fft.hpp:220-470: ``execute(data, direction)`` in place, unnormalised both ways;
  ``execute_batched(data, batch, direction)`` element-major (element i of transform t at data[i*batch + t]).
* ``RealFftPlan(n)`` - real_fft.hpp:18-101: ``rfft(real_in, out)`` (n reals -> n/2+1 complex, unnormalised) and
  ``irfft(in, real_out)`` (normalised by 1/n).
* ``BluesteinPlan(n)`` - bluestein.hpp:29-149: any n; ``execute`` forward unnormalised, inverse normalised by 1/n.
* ``NdFftPlan(dims)`` - nd_fft.hpp:28-194: row-major 1-3 dims; inverse normalised by 1/prod(dims).
* ``fft(data, direction)`` / ``ifft_normalized(data)`` - fft.hpp:1006-1029.

``Plan(desc)`` exposes the general descriptor (batch, strides, R2C/C2R, precision) the benchmarks use.

Tensors must be CUDA tensors on the plan's device: complex64 (or float32 on the real side of R2C/C2R), contiguous
in the layout the plan describes. Work is enqueued on torch's current CUDA stream, so it orders with the caller's
torch work. The reference's preconditions (sizes, power-of-two-ness where it asserts them) become ``ValueError``;
library status codes become ``CrdFftError``.
"""

from __future__ import annotations

import ctypes
from typing import Iterable, Optional, Sequence

import torch

from . import _lib
from ._lib import (C2C, C2R, CEIR_REJECT, FORWARD, INVERSE, NORM_INVERSE, NORM_NONE, PREC_FP32, R2C,
                   SPECTRAL_PERIODOGRAM, SPECTRAL_SPECTROGRAM, SPECTRAL_WELCH, CeirFftOp, CrdFftError, CwtDesc, Desc,
                   SpectralDesc, PlanInfo, check, lib)

Forward = FORWARD
Inverse = INVERSE


def _dir(direction) -> int:
    if isinstance(direction, str):
        direction = {"forward": FORWARD, "inverse": INVERSE}[direction.lower()]
    d = int(direction)
    if d not in (FORWARD, INVERSE):
        raise ValueError(f"direction must be 0 (forward) or 1 (inverse), not {direction!r}")
    return d


def _stream(stream) -> ctypes.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    if isinstance(stream, torch.cuda.Stream):
        return ctypes.c_void_p(stream.cuda_stream)
    return ctypes.c_void_p(int(stream))


def _ptr(t: torch.Tensor, dtype: torch.dtype, what: str) -> ctypes.c_void_p:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{what} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{what} must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


class _Handle:
    def __init__(self):
        self._h = ctypes.c_void_p()

    def _release(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().crdfft_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def info(self) -> dict:
        inf = PlanInfo()
        check(lib().crdfft_plan_info_get(self._h, ctypes.byref(inf)), "plan_info")
        return {
            "algorithm": inf.algorithm.decode(),
            "passes": inf.passes,
            "device": inf.device,
            "workspace_bytes": inf.workspace_bytes,
            "table_bytes": inf.table_bytes,
            "factors": [int(f) for f in inf.factors if f],
        }

    def workspace_size(self) -> int:
        return int(lib().crdfft_workspace_size(self._h))

    def set_workspace(self, ws: Optional[torch.Tensor]) -> None:
        if ws is None:
            check(lib().crdfft_set_workspace(self._h, None, 0), "set_workspace")
            self._ws = None
            return
        nbytes = ws.numel() * ws.element_size()
        check(lib().crdfft_set_workspace(self._h, ctypes.c_void_p(ws.data_ptr()), nbytes), "set_workspace")
        self._ws = ws  # keep it alive


class Plan(_Handle):
    """The general descriptor plan (crdfft_plan_create)."""

    def __init__(self, dims: Sequence[int], batch: int = 1, kind: int = C2C, precision: int = PREC_FP32,
                 norm: int = NORM_NONE, istride: int = 0, idist: int = 0, ostride: int = 0, odist: int = 0):
        super().__init__()
        dims = [int(d) for d in dims]
        if not 1 <= len(dims) <= 3:
            raise ValueError("rank must be 1, 2 or 3")
        d = Desc()
        d.rank = len(dims)
        d.kind = kind
        d.precision = precision
        d.norm = norm
        for i, v in enumerate(dims):
            d.dims[i] = v
        d.batch = batch
        d.istride, d.idist, d.ostride, d.odist = istride, idist, ostride, odist
        self.dims = tuple(dims)
        self.batch = batch
        self.kind = kind
        check(lib().crdfft_plan_create(ctypes.byref(d), ctypes.byref(self._h)), "plan_create")

    def execute(self, inp: torch.Tensor, out: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
        in_dtype = torch.float32 if self.kind == R2C else torch.complex64
        out_dtype = torch.float32 if self.kind == C2R else torch.complex64
        pi = _ptr(inp, in_dtype, "input")
        po = _ptr(out, out_dtype, "output")
        check(lib().crdfft_execute(self._h, pi, po, _dir(direction), _stream(stream)), "execute")
        return out

    def execute_planar(self, re_in: torch.Tensor, im_in: torch.Tensor, re_out: torch.Tensor, im_out: torch.Tensor,
                       direction=FORWARD, stream=None):
        """Run a C2C plan on split-complex planes (crdfft_execute_planar): float32 device tensors, one per part."""
        if self.kind != C2C:
            raise ValueError("planar operands are for complex-to-complex plans")
        ptrs = [_ptr(t, torch.float32, what) for t, what in
                ((re_in, "re_in"), (im_in, "im_in"), (re_out, "re_out"), (im_out, "im_out"))]
        check(lib().crdfft_execute_planar(self._h, *ptrs, _dir(direction), _stream(stream)), "execute_planar")
        return re_out, im_out

    def execute_host(self, inp: torch.Tensor, out: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
        """Run on HOST tensors (pinned for overlap; crdfft_execute_host): chunked copies in and out overlap the
        transforms on the GPU. Synchronise `stream` (default: the current stream) before reading `out`."""
        in_dtype = torch.float32 if self.kind == R2C else torch.complex64
        out_dtype = torch.float32 if self.kind == C2R else torch.complex64
        for t, dt, what in ((inp, in_dtype, "input"), (out, out_dtype, "output")):
            if t.is_cuda or t.dtype != dt or not t.is_contiguous():
                raise ValueError(f"{what} must be a contiguous host tensor of {dt}")
        check(lib().crdfft_execute_host(self._h, inp.data_ptr(), out.data_ptr(), _dir(direction), _stream(stream)),
              "execute_host")
        return out


def lower_tensor_fft(shape, direction, axis: int = -1, element_f32: bool = True, operand_is_tensor: bool = True,
                     num_operands: int = 2, num_results: int = 2) -> dict:
    """The CEIR tensor.fft lowering (crdfft_ceir_fft_desc): the plan descriptor fields and the direction for an op
    on split-complex tensors of `shape` (a dynamic extent as -1). Raises CrdFftError with the reject reason in its
    message when the op is outside the envelope; host only."""
    op = CeirFftOp()
    op.num_operands, op.num_results = num_operands, num_results
    op.operand_is_tensor, op.element_is_f32 = int(operand_is_tensor), int(element_f32)
    op.rank = len(shape)
    op.axis = axis
    for i, v in enumerate(list(shape)[:8]):
        op.shape[i] = int(v)
    op.direction = direction.encode() if isinstance(direction, str) else None
    d = Desc()
    dr = ctypes.c_int32()
    why = ctypes.c_int32()
    st = lib().crdfft_ceir_fft_desc(ctypes.byref(op), ctypes.byref(d), ctypes.byref(dr), ctypes.byref(why))
    if st != 0:
        raise CrdFftError(st, f"tensor.fft not lowered: {CEIR_REJECT.get(why.value, why.value)}")
    return {"dims": [int(d.dims[0])], "batch": int(d.batch), "istride": int(d.istride), "idist": int(d.idist),
            "ostride": int(d.ostride), "odist": int(d.odist), "norm": int(d.norm), "direction": int(dr.value)}


class ConvPlan(_Handle):
    """Fused FFT convolution (crdfft_conv_plan_create): y = IFFT(FFT(x) * H) * scale over a batch of 1-D signals
    (dims = [n]) or 2-D signals (dims = [rows, cols]); one spectrum H shared by the batch, or one per signal.
    real=True: real signals (float32) and the half spectrum H (complex64, cols/2 + 1 values a row)."""

    def __init__(self, dims: Sequence[int], batch: int = 1, per_signal_filter: bool = False, scale: float = -1.0,
                 real: bool = False):
        super().__init__()
        dims = [int(v) for v in dims]
        d = Desc()
        d.rank = len(dims)
        d.kind = R2C if real else C2C
        self.real = bool(real)
        d.precision = PREC_FP32
        d.norm = NORM_NONE
        for i, v in enumerate(dims):
            d.dims[i] = v
        d.batch = batch
        self.dims = tuple(dims)
        self.batch = batch
        check(lib().crdfft_conv_plan_create(ctypes.byref(d), 1 if per_signal_filter else 0, float(scale),
                                            ctypes.byref(self._h)), "conv_plan_create")

    def execute(self, inp: torch.Tensor, spectrum: torch.Tensor, out: torch.Tensor, stream=None) -> torch.Tensor:
        dt = torch.float32 if self.real else torch.complex64
        pi = _ptr(inp, dt, "input")
        ps = _ptr(spectrum, torch.complex64, "spectrum")
        po = _ptr(out, dt, "output")
        check(lib().crdfft_conv_execute(self._h, pi, ps, po, _stream(stream)), "conv_execute")
        return out


class SpectralPlan(_Handle):
    """hesap-dsp's spectral estimators on the device (crdfft_spectral_plan_create) over `count` real signals of
    `nsamples` samples: mode SPECTRAL_WELCH (welch_psd, spectral.hpp:141-172), SPECTRAL_SPECTROGRAM (spectrogram,
    :177-183) or SPECTRAL_PERIODOGRAM (periodogram, :188-220). window: None for the periodic Hann window."""

    def __init__(self, mode: int, nsamples: int, count: int = 1, fs: float = 1.0, nperseg: int = 256,
                 noverlap: int = 0, window=None, detrend: bool = True):
        super().__init__()
        d = SpectralDesc()
        d.mode, d.detrend = int(mode), 1 if detrend else 0
        d.nsamples, d.count, d.nperseg, d.noverlap, d.fs = int(nsamples), int(count), int(nperseg), int(noverlap), fs
        self._win = None
        if window is not None:
            import numpy as np

            self._win = np.ascontiguousarray(window, dtype=np.float32)
            d.window = self._win.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        self.mode, self.nsamples, self.count = int(mode), int(nsamples), int(count)
        self.nperseg = int(nsamples) if mode == SPECTRAL_PERIODOGRAM else int(nperseg)
        self.nfreq = self.nperseg // 2 + 1
        self.nseg = int(lib().crdfft_spectral_segments(ctypes.byref(d)))
        check(lib().crdfft_spectral_plan_create(ctypes.byref(d), ctypes.byref(self._h)), "spectral_plan_create")

    def out_shape(self):
        if self.mode == SPECTRAL_SPECTROGRAM:
            return (self.count, self.nseg, self.nfreq)
        return (self.count, self.nfreq)

    def execute(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        if x.numel() != self.count * self.nsamples:
            raise ValueError(f"x holds {x.numel()} samples, the plan {self.count} x {self.nsamples}")
        if out is None:
            out = torch.empty(self.out_shape(), dtype=torch.float32, device=x.device)
        if out.numel() == 0:
            return out  # a spectrogram of no segment
        check(lib().crdfft_spectral_execute(self._h, _ptr(x, torch.float32, "x"), _ptr(out, torch.float32, "out"),
                                            _stream(stream)), "spectral_execute")
        return out


def welch_psd(x: torch.Tensor, fs: float, nperseg: int, noverlap: int = 0) -> torch.Tensor:
    """dsp::welch_psd over the rows of x (a 1-D tensor is one signal): the periodic Hann window, noverlap 0 means
    nperseg / 2 (spectral.hpp:141-172)."""
    plan = SpectralPlan(SPECTRAL_WELCH, x.shape[-1], x.numel() // x.shape[-1], fs, nperseg, noverlap)
    return plan.execute(x).reshape(tuple(x.shape[:-1]) + (plan.nfreq,))


def spectrogram(x: torch.Tensor, fs: float, nperseg: int, noverlap: int) -> torch.Tensor:
    """dsp::spectrogram over the rows of x: (..., nseg, nfreq) (spectral.hpp:177-183)."""
    plan = SpectralPlan(SPECTRAL_SPECTROGRAM, x.shape[-1], x.numel() // x.shape[-1], fs, nperseg, noverlap)
    return plan.execute(x).reshape(tuple(x.shape[:-1]) + (plan.nseg, plan.nfreq))


def periodogram(x: torch.Tensor, fs: float) -> torch.Tensor:
    """dsp::periodogram over the rows of x (spectral.hpp:188-220)."""
    plan = SpectralPlan(SPECTRAL_PERIODOGRAM, x.shape[-1], x.numel() // x.shape[-1], fs)
    return plan.execute(x).reshape(tuple(x.shape[:-1]) + (plan.nfreq,))


class CwtPlan:
    """crd-hesap-wavelet's cwt (cwt.hpp:461-621) on the device over `count` real signals of `nsamples` samples:
    coefficients (count, nscales, nsamples) complex64, row s of signal c = CwtResult::coeffs[s * n ...] of that
    signal. wavelet: a pywt-style name ("mexh", "morl", "cmorB-C", "gausP", "cgauP", "shanB-C", "fbspM-B-C",
    "paulM"; continuous_wavelet, cwt.hpp:300-407). The scales' kernels and their spectra are built once, at plan
    time."""

    def __init__(self, nsamples: int, scales, wavelet: str, count: int = 1, sampling_period: float = 1.0,
                 precision: int = 12):
        import numpy as np

        self._h = ctypes.c_void_p()
        self._scales = np.ascontiguousarray(scales, dtype=np.float64).reshape(-1)
        self._name = str(wavelet).encode()
        self.nsamples, self.count, self.nscales = int(nsamples), int(count), len(self._scales)
        self._desc = self._make_desc(sampling_period, precision)
        freqs = np.empty(self.nscales, dtype=np.float64)
        check(lib().crdfft_cwt_frequencies(ctypes.byref(self._desc),
                                           freqs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "cwt_frequencies")
        self.frequencies = freqs
        check(lib().crdfft_cwt_plan_create(ctypes.byref(self._desc), ctypes.byref(self._h)), "cwt_plan_create")
        lfft, rnd, fused = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        check(lib().crdfft_cwt_plan_info(self._h, ctypes.byref(lfft), ctypes.byref(rnd), ctypes.byref(fused)),
              "cwt_plan_info")
        self.fft_length, self.signals_per_round, self.fused = int(lfft.value), int(rnd.value), bool(fused.value)

    def _make_desc(self, sampling_period: float, precision: int) -> CwtDesc:
        d = CwtDesc()
        d.wavelet = self._name
        d.scales = self._scales.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.nsamples, d.count, d.nscales = self.nsamples, self.count, self.nscales
        d.sampling_period, d.precision = float(sampling_period), int(precision)
        return d

    def execute(self, x: torch.Tensor, out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        if x.numel() != self.count * self.nsamples:
            raise ValueError(f"x holds {x.numel()} samples, the plan {self.count} x {self.nsamples}")
        if out is None:
            out = torch.empty((self.count, self.nscales, self.nsamples), dtype=torch.complex64, device=x.device)
        if out.numel() != self.count * self.nscales * self.nsamples:
            raise ValueError("out must hold count x nscales x nsamples values")
        check(lib().crdfft_cwt_execute(self._h, _ptr(x, torch.float32, "x"), _ptr(out, torch.complex64, "out"),
                                       _stream(stream)), "cwt_execute")
        return out

    def __del__(self):
        try:
            if self._h.value:
                lib().crdfft_cwt_plan_destroy(self._h)
                self._h = ctypes.c_void_p()
        except Exception:
            pass


def cwt(x: torch.Tensor, scales, wavelet: str, sampling_period: float = 1.0, precision: int = 12):
    """wavelet::cwt over the rows of x (a 1-D tensor is one signal): (coefficients (..., nscales, n) complex64 on
    x's device, frequencies (nscales,) float64), the reference's CwtResult (cwt.hpp:446-456, 616-621)."""
    n = x.shape[-1]
    plan = CwtPlan(n, scales, wavelet, x.numel() // n, sampling_period, precision)
    out = plan.execute(x.contiguous())
    return out.reshape(tuple(x.shape[:-1]) + (plan.nscales, n)), plan.frequencies


def cwt_fft_length(nsamples: int, scales, wavelet: str, precision: int = 12) -> int:
    """The FFT length a CWT plan uses (no device needed): the power of two >= n + the longest kernel."""
    import numpy as np

    sc = np.ascontiguousarray(scales, dtype=np.float64).reshape(-1)
    d = CwtDesc()
    d.wavelet = str(wavelet).encode()
    d.scales = sc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.nsamples, d.count, d.nscales, d.precision = int(nsamples), 1, len(sc), int(precision)
    return int(lib().crdfft_cwt_fft_length(ctypes.byref(d)))


def cwt_frequencies(scales, wavelet: str, sampling_period: float = 1.0, precision: int = 12):
    """CwtResult::frequencies without a device: central_frequency / (scale * sampling_period) (cwt.hpp:410-444)."""
    import numpy as np

    sc = np.ascontiguousarray(scales, dtype=np.float64).reshape(-1)
    d = CwtDesc()
    d.wavelet = str(wavelet).encode()
    d.scales = sc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.nsamples, d.count, d.nscales = 1, 1, len(sc)
    d.sampling_period, d.precision = float(sampling_period), int(precision)
    out = np.empty(len(sc), dtype=np.float64)
    check(lib().crdfft_cwt_frequencies(ctypes.byref(d), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
          "cwt_frequencies")
    return out


class FftPlan(_Handle):
    """FftPlan<float>(alloc, n) - one size-n complex transform (fft.hpp:224)."""

    def __init__(self, n: int):
        super().__init__()
        if n < 1:
            raise ValueError("n must be >= 1")
        self.n = int(n)
        check(lib().crdfft_fft_plan_create(self.n, ctypes.byref(self._h)), "FftPlan")

    def size(self) -> int:
        return self.n

    def execute(self, data: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
        """In place, unnormalised (fft.hpp:409-413)."""
        if data.numel() != self.n:
            raise ValueError(f"data holds {data.numel()} values, the plan {self.n}")
        check(lib().crdfft_fft_execute(self._h, _ptr(data, torch.complex64, "data"), _dir(direction),
                                       _stream(stream)), "execute")
        return data

    def execute_batched(self, data: torch.Tensor, batch: int, direction=FORWARD, stream=None) -> torch.Tensor:
        """Element-major batch in place (fft.hpp:462-470): element i of transform t at data[i*batch + t]."""
        if data.numel() != self.n * batch:
            raise ValueError(f"data holds {data.numel()} values, expected n*batch = {self.n * batch}")
        check(lib().crdfft_fft_execute_batched(self._h, _ptr(data, torch.complex64, "data"), int(batch),
                                               _dir(direction), _stream(stream)), "execute_batched")
        return data


class RealFftPlan(_Handle):
    """RealFftPlan<float>(alloc, n): real[n] <-> complex[n/2+1] (real_fft.hpp:18-101)."""

    def __init__(self, n: int):
        super().__init__()
        if n < 2 or n % 2:
            raise ValueError("n must be even and >= 2")
        self.n = int(n)
        check(lib().crdfft_real_plan_create(self.n, ctypes.byref(self._h)), "RealFftPlan")

    def size(self) -> int:
        return self.n

    def rfft(self, real_in: torch.Tensor, out: torch.Tensor, stream=None) -> torch.Tensor:
        if real_in.numel() != self.n or out.numel() != self.n // 2 + 1:
            raise ValueError("rfft wants real_in[n] and out[n/2+1]")
        check(lib().crdfft_rfft(self._h, _ptr(real_in, torch.float32, "real_in"), _ptr(out, torch.complex64, "out"),
                                _stream(stream)), "rfft")
        return out

    def irfft(self, inp: torch.Tensor, real_out: torch.Tensor, stream=None) -> torch.Tensor:
        if inp.numel() != self.n // 2 + 1 or real_out.numel() != self.n:
            raise ValueError("irfft wants in[n/2+1] and real_out[n]")
        check(lib().crdfft_irfft(self._h, _ptr(inp, torch.complex64, "in"), _ptr(real_out, torch.float32, "real_out"),
                                 _stream(stream)), "irfft")
        return real_out


class BluesteinPlan(_Handle):
    """BluesteinPlan<float>(alloc, n): any n >= 1; inverse normalised by 1/n (bluestein.hpp:29-149)."""

    def __init__(self, n: int):
        super().__init__()
        if n < 1:
            raise ValueError("n must be >= 1")
        self.n = int(n)
        check(lib().crdfft_bluestein_plan_create(self.n, ctypes.byref(self._h)), "BluesteinPlan")

    def size(self) -> int:
        return self.n

    def execute(self, data: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
        if data.numel() != self.n:
            raise ValueError(f"data holds {data.numel()} values, the plan {self.n}")
        check(lib().crdfft_bluestein_execute(self._h, _ptr(data, torch.complex64, "data"), _dir(direction),
                                             _stream(stream)), "execute")
        return data


class NdFftPlan(_Handle):
    """NdFftPlan<float>(alloc, dims): row-major N-D transform; inverse normalised by 1/prod(dims)
    (nd_fft.hpp:28-194)."""

    def __init__(self, dims: Iterable[int]):
        super().__init__()
        dims = [int(d) for d in dims]
        if not 1 <= len(dims) <= 3 or any(d < 1 for d in dims):
            raise ValueError("1 to 3 dims, each >= 1")
        self.dims = tuple(dims)
        arr = (ctypes.c_int64 * len(dims))(*dims)
        check(lib().crdfft_nd_plan_create(len(dims), arr, ctypes.byref(self._h)), "NdFftPlan")

    def execute(self, data: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
        total = 1
        for d in self.dims:
            total *= d
        if data.numel() != total:
            raise ValueError(f"data holds {data.numel()} values, the plan {total}")
        check(lib().crdfft_nd_execute(self._h, _ptr(data, torch.complex64, "data"), _dir(direction),
                                      _stream(stream)), "execute")
        return data


def uneven_offsets(sizes) -> tuple:
    """Packed offsets (each transform on a 16-byte boundary) and the total complex elements for an uneven batch."""
    n = len(sizes)
    arr = (ctypes.c_int64 * n)(*[int(v) for v in sizes])
    off = (ctypes.c_int64 * n)()
    total = lib().crdfft_uneven_offsets(arr, n, off)
    if total < 0:
        raise ValueError("bad sizes")
    return [int(v) for v in off], int(total)


class UnevenPlan(_Handle):
    """Independent complex transforms of different 7-smooth lengths in one persistent, graph-captured launch
    (crdfft_plan_create_uneven). Transform t occupies elements offsets[t] .. offsets[t]+sizes[t]-1 of the input
    and of the output buffer; both directions unnormalised."""

    def __init__(self, sizes, offsets=None):
        super().__init__()
        self.sizes = [int(v) for v in sizes]
        n = len(self.sizes)
        arr = (ctypes.c_int64 * n)(*self.sizes)
        if offsets is None:
            self.offsets, self.total = uneven_offsets(self.sizes)
        else:
            self.offsets = [int(v) for v in offsets]
            self.total = max(o + s for o, s in zip(self.offsets, self.sizes))
        off = (ctypes.c_int64 * n)(*self.offsets)
        check(lib().crdfft_plan_create_uneven(arr, n, off, ctypes.byref(self._h)), "UnevenPlan")

    def execute(self, inp: torch.Tensor, out: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
        if inp.numel() < self.total or out.numel() < self.total:
            raise ValueError(f"buffers must hold {self.total} complex values")
        check(lib().crdfft_execute(self._h, _ptr(inp, torch.complex64, "input"), _ptr(out, torch.complex64, "output"),
                                   _dir(direction), _stream(stream)), "execute")
        return out


def fft(data: torch.Tensor, direction=FORWARD, stream=None) -> torch.Tensor:
    """One-shot in-place transform, unnormalised (fft.hpp:1006-1012)."""
    check(lib().crdfft_fft(_ptr(data, torch.complex64, "data"), data.numel(), _dir(direction), _stream(stream)), "fft")
    return data


def ifft_normalized(data: torch.Tensor, stream=None) -> torch.Tensor:
    """One-shot in-place inverse scaled by 1/n (fft.hpp:1015-1029)."""
    check(lib().crdfft_ifft_normalized(_ptr(data, torch.complex64, "data"), data.numel(), _stream(stream)),
          "ifft_normalized")
    return data


def self_check() -> None:
    """The device known-answer check (the role of src/fft_self_check.cpp); raises CrdFftError on a mismatch."""
    check(lib().crdfft_self_check(), "self_check")


PLANNER_ESTIMATE = 0
PLANNER_MEASURE = 1
PLANNER_LEARNED = 2


def set_planner(mode) -> None:
    """CRDFFT_PLANNER_ESTIMATE (0, default), CRDFFT_PLANNER_MEASURE (1) or CRDFFT_PLANNER_LEARNED (2);
    "estimate"/"measure"/"learned" also accepted."""
    if isinstance(mode, str):
        mode = {"estimate": PLANNER_ESTIMATE, "measure": PLANNER_MEASURE, "learned": PLANNER_LEARNED}[mode]
    lib().crdfft_set_planner_mode(int(mode))


def _text(fn) -> str:
    need = ctypes.c_size_t(0)
    check(fn(None, 0, ctypes.byref(need)), "size")
    buf = ctypes.create_string_buffer(need.value)
    check(fn(buf, need.value, ctypes.byref(need)), "export")
    return buf.value.decode()


def wisdom_export() -> str:
    return _text(lib().crdfft_wisdom_export)


def wisdom_import(text: str) -> None:
    check(lib().crdfft_wisdom_import(text.encode()), "wisdom_import")


def wisdom_forget() -> None:
    lib().crdfft_wisdom_forget()


def planner_log() -> str:
    return _text(lib().crdfft_planner_log)


def learned_model_import(text: str) -> None:
    """Load the learned cost model (crdfft_learned_model_import); CRDFFT_PLANNER_LEARNED plans rank with it."""
    check(lib().crdfft_learned_model_import(text.encode()), "learned_model_import")


def learned_model_export() -> str:
    return _text(lib().crdfft_learned_model_export)


def learned_model_forget() -> None:
    lib().crdfft_learned_model_forget()


def learned_predict(features) -> float:
    """The imported model's predicted log(ms) for one feature vector (host evaluation)."""
    n = lib().crdfft_pass_feature_count()
    if len(features) != n:
        raise ValueError(f"expected {n} features")
    arr = (ctypes.c_float * n)(*[float(v) for v in features])
    out = ctypes.c_float(0.0)
    check(lib().crdfft_learned_predict(arr, ctypes.byref(out)), "learned_predict")
    return float(out.value)


def device_status(plan: _Handle, stream=None) -> None:
    """Raise CrdFftError(DEVICE_TIMEOUT) if a kernel of `plan` gave up a bounded wait since the last call
    (crdfft_device_status; synchronises the stream)."""
    check(lib().crdfft_device_status(plan._h, _stream(stream)), "device_status")


def stall_waits(on: bool) -> None:
    """Test hook: plans created while on make their pipelined kernels' first barrier wait run out."""
    lib().crdfft_debug_stall_waits(1 if on else 0)


def fail_alloc_after(k: int) -> None:
    """Test hook: the k-th device allocation from now fails (0 = off)."""
    lib().crdfft_debug_fail_alloc_after(int(k))
