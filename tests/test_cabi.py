"""CPU tests of the boundary: libcrdfft.so loads (no GPU needed) and exports every entry point include/crdfft.h
declares; the Python mirror's tables agree with the header; descriptor validation and error strings need no device.
"""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from crd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include")))
           if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(crdfft_[a-z0-9_]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_reference_verbs():
    names = declared_functions()
    for verb in ("crdfft_fft_plan_create", "crdfft_fft_execute", "crdfft_fft_execute_batched",
                 "crdfft_real_plan_create", "crdfft_rfft", "crdfft_irfft", "crdfft_bluestein_plan_create",
                 "crdfft_bluestein_execute", "crdfft_nd_plan_create", "crdfft_nd_execute", "crdfft_fft",
                 "crdfft_ifft_normalized", "crdfft_plan_create", "crdfft_execute", "crdfft_plan_destroy"):
        assert verb in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert sorted(_lib.EXPORTS) == declared_functions()
    _lib.lib()  # loads and sets every signature


def test_status_strings():
    L = _lib.lib()
    for code in range(9):
        assert L.crdfft_status_string(code)
    assert L.crdfft_status_string(3) == b"device out of memory"


def test_descriptor_sizes_match_header():
    # crdfft_desc: 4 int32 + 3 int64 dims + 5 int64 = 80 bytes; crdfft_plan_info: 64 + 2*4 + 2*8 + 8*8 = 152
    assert ctypes.sizeof(_lib.Desc) == 80
    assert ctypes.sizeof(_lib.PlanInfo) == 152


def test_invalid_descriptor_rejected_without_device():
    L = _lib.lib()
    d = _lib.Desc()
    d.rank = 0
    d.batch = 1
    h = ctypes.c_void_p()
    assert L.crdfft_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.INVALID_DESC
    d.rank = 1
    d.dims[0] = 16
    d.batch = 0
    assert L.crdfft_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.INVALID_DESC
    assert L.crdfft_plan_create(None, ctypes.byref(h)) == _lib.INVALID_ARG
    assert L.crdfft_execute(None, None, None, 0, None) == _lib.INVALID_ARG
    assert L.crdfft_plan_destroy(None) == _lib.OK


def test_spectral_descriptor_and_segment_count_without_device():
    """crdfft_spectral_desc layout (2 int32 + 4 int64 + double + pointer = 56 bytes) and the segment count rule of
    the reference's spectral.hpp:50-54 (Welch reads noverlap 0 as nperseg / 2), evaluated on the host."""
    from oracle import spectral as S

    assert ctypes.sizeof(_lib.SpectralDesc) == 56
    L = _lib.lib()

    def segs(mode, ns, nper, nov, fs=1.0):
        d = _lib.SpectralDesc()
        d.mode, d.detrend, d.nsamples, d.count, d.nperseg, d.noverlap, d.fs = mode, 1, ns, 3, nper, nov, fs
        return L.crdfft_spectral_segments(ctypes.byref(d))

    for ns, nper, nov in ((512, 64, 32), (100000, 1024, 512), (63, 64, 0), (5000, 256, 255), (70000, 4096, 1024)):
        want = S.segment_count(ns, nper, nov if nov else nper // 2)
        assert segs(_lib.SPECTRAL_WELCH, ns, nper, nov) == want
    assert segs(_lib.SPECTRAL_SPECTROGRAM, 512, 64, 0) == 8          # no overlap: 512 / 64
    assert segs(_lib.SPECTRAL_PERIODOGRAM, 4096, 0, 0) == 1
    assert segs(_lib.SPECTRAL_WELCH, 1000, 255, 0) == -1               # odd segment length
    assert segs(_lib.SPECTRAL_WELCH, 1000, 256, 256) == -1             # no hop
    assert segs(_lib.SPECTRAL_WELCH, 1000, 256, 0, fs=0.0) == -1       # fs
    assert segs(_lib.SPECTRAL_WELCH, 10 ** 6, 2 * 30000, 0) == -1      # half length beyond one pass
    h = ctypes.c_void_p()
    assert L.crdfft_spectral_plan_create(None, ctypes.byref(h)) == _lib.INVALID_ARG
    assert L.crdfft_spectral_execute(None, None, None, None) == _lib.INVALID_ARG


def test_wisdom_text_round_trip_without_device():
    """Wisdom is host state: the committed file imports, exports the same entries, and malformed text is refused
    without changing what is held."""
    import crd_b200.hesap as H

    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles", "wisdom_b200.txt")
    with open(path) as f:
        text = f.read()
    H.wisdom_forget()
    try:
        H.wisdom_import(text)
        back = H.wisdom_export()
        assert back.splitlines()[0] == "crdfft-wisdom 1"
        entries = lambda t: sorted(ln.split()[0] for ln in t.splitlines()[1:] if ln.strip())  # noqa: E731
        assert entries(back) == entries(text)
        with pytest.raises(_lib.CrdFftError):
            H.wisdom_import("not wisdom")
        assert entries(H.wisdom_export()) == entries(text)
    finally:
        H.wisdom_forget()

def test_wisdom_register_budget_flag_round_trips():
    """A shape measured on the wide register build is remembered with a trailing `w`; any other trailing token is
    refused."""
    import crd_b200.hesap as H

    H.wisdom_forget()
    try:
        text = "crdfft-wisdom 1\nDEV|n4096:r16.16.16:x 0 16 1 0.5 w\nDEV|n1024:r16.16.4:x 0 16 4 0.25\n"
        H.wisdom_import(text)
        lines = sorted(H.wisdom_export().splitlines()[1:])
        assert lines == ["DEV|n1024:r16.16.4:x 0 16 4 0.25", "DEV|n4096:r16.16.16:x 0 16 1 0.5 w"]
        with pytest.raises(_lib.CrdFftError):
            H.wisdom_import("crdfft-wisdom 1\nDEV|n4096:r16.16.16:x 0 16 1 0.5 wide\n")
    finally:
        H.wisdom_forget()


def test_wisdom_tensor_store_flag_round_trips():
    """A row pass measured with its tile stored by the Tensor Memory Accelerator is remembered with a trailing `t`,
    alone or after `w`; another spelling of the flag is refused."""
    import crd_b200.hesap as H

    H.wisdom_forget()
    try:
        text = ("crdfft-wisdom 1\nDEV|n1024:r16.16.4:x 0 16 4 0.25 t\nDEV|n512:r16.8.4:x 0 16 4 0.125 w t\n"
                "DEV|n4096:r16.16.16:x 0 16 1 0.5\n")
        H.wisdom_import(text)
        lines = sorted(H.wisdom_export().splitlines()[1:])
        assert lines == ["DEV|n1024:r16.16.4:x 0 16 4 0.25 t", "DEV|n4096:r16.16.16:x 0 16 1 0.5",
                         "DEV|n512:r16.8.4:x 0 16 4 0.125 w t"]
        with pytest.raises(_lib.CrdFftError):
            H.wisdom_import("crdfft-wisdom 1\nDEV|n1024:r16.16.4:x 0 16 4 0.25 tstore\n")
    finally:
        H.wisdom_forget()
