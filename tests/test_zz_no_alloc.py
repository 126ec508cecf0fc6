"""The entry point that allocates no device memory (crdfft_execute_static_scratch), through the C ABI.

Callers that cannot call cudaMalloc (work enqueued during stream capture, real-time callbacks that must not enter an
allocator, processes whose device memory is owned by a pool) use this entry point: the plan's tables and the
four-step intermediate come from a 64 MiB array the library holds on each GPU. Here its output must match the
ordinary plan's (crdfft_plan_create + crdfft_execute) within the parity tolerance, on consecutive calls, and a
call after the first must not change the device's free memory. This file sorts last so that a run stopping at its
first failure has run every other test already; it also passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import oracle
from crd_b200 import _lib

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6  # the FP32 parity bar of tests/test_gpu_parity.py


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ordinary(x: torch.Tensor, n: int, batch: int, direction: int) -> torch.Tensor:
    L = _lib.lib()
    d = _lib.Desc()
    d.rank = 1
    d.kind = _lib.C2C
    d.dims[0] = n
    d.batch = batch
    h = ctypes.c_void_p()
    _lib.check(L.crdfft_plan_create(ctypes.byref(d), ctypes.byref(h)), "plan_create")
    out = torch.empty_like(x)
    try:
        _lib.check(L.crdfft_execute(h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), direction,
                                    _stream()), "execute")
        torch.cuda.synchronize()
    finally:
        L.crdfft_plan_destroy(h)
    return out


def _static(x: torch.Tensor, n: int, batch: int, direction: int) -> torch.Tensor:
    out = torch.empty_like(x)
    st = _lib.lib().crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                  n, batch, direction, _stream())
    _lib.check(st, "execute_static_scratch")
    torch.cuda.synchronize()
    return out


def _rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a64 = a.cpu().numpy().astype(np.complex128)
    b64 = b.cpu().numpy().astype(np.complex128)
    return float(np.linalg.norm(a64 - b64) / np.linalg.norm(b64))


def test_static_scratch_matches_ordinary_plan_on_consecutive_calls():
    torch.cuda.init()
    cases = [
        (1 << 20, 5, 0, 11),   # four-step with the intermediate in the static array, two waves
        (1 << 20, 5, 1, 12),   # same plan reused, new data, inverse
        (107520, 3, 0, 13),    # a new size rebuilds the plan in the array
        (4096, 64, 0, 14),     # single pass: only tables in the array
    ]
    free_before = None
    for i, (n, batch, direction, seed) in enumerate(cases):
        x = torch.from_numpy(oracle.lcg_complex64(seed, n * batch)).cuda()
        if i == 1:
            free_before = torch.cuda.mem_get_info()[0]
        got = _static(x, n, batch, direction)
        if i == 1:
            assert torch.cuda.mem_get_info()[0] == free_before, "a call on a cached plan allocated device memory"
        want = _ordinary(x, n, batch, direction)
        assert _rel_l2(got, want) <= REL_L2, (n, batch, direction)
        # the same kernels and tables as the ordinary plan: in practice the same bits
        assert torch.equal(got.view(torch.float32), want.view(torch.float32)), (n, batch, direction)
    # and against the FP64 oracle for one transform of the last case
    n, batch = cases[-1][0], cases[-1][1]
    x = oracle.lcg_complex64(cases[-1][3], n * batch).reshape(batch, n)
    got = _static(torch.from_numpy(x).cuda().reshape(-1), n, batch, 0).cpu().numpy().reshape(batch, n)
    assert oracle.rel_l2(got, oracle.fft64(x)) <= REL_L2


def test_static_scratch_rejects_sizes_beyond_its_array():
    L = _lib.lib()
    x = torch.empty(16, dtype=torch.complex64, device="cuda")
    st = L.crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                         (1 << 22) + 1, 1, 0, _stream())
    assert st == _lib.UNSUPPORTED_SIZE
    assert L.crdfft_execute_static_scratch(None, None, 16, 1, 0, _stream()) == _lib.INVALID_ARG
