"""The entry point that allocates no device memory (crdfft_execute_static_scratch), through the C ABI.

Callers that cannot call cudaMalloc (work enqueued during stream capture, real-time callbacks that must not enter an
allocator, processes whose device memory is owned by a pool) use this entry point: the plan's tables and the
four-step intermediate come from a 64 MiB array the library holds on each GPU. Here its output must match the
ordinary plan's (crdfft_plan_create + crdfft_execute) within the parity tolerance, on consecutive calls, and a
call after the first must not change the device's free memory. This file sorts last so that a run stopping at its
first failure has run every other test already; it also passes alone in a fresh process.

A call with a new (n, batch) rebuilds the plan inside the shared array. These tests also check that a rebuild waits
for the previous call's kernels when all calls are queued on one non-blocking stream with no host synchronisation in
between, that the rebuild itself allocates nothing, that the documented limit n = 2^22 works, that a Bluestein length
whose padded sequences fit is accepted (and one that does not fit is refused), and that a rebuild during a stream
capture is refused without breaking the capture.
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


def _static(x: torch.Tensor, n: int, batch: int, direction: int, sync: bool = True) -> torch.Tensor:
    out = torch.empty_like(x)
    st = _lib.lib().crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                  n, batch, direction, _stream())
    _lib.check(st, "execute_static_scratch")
    if sync:
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


def test_static_scratch_rebuilds_in_order_on_a_non_blocking_stream():
    """Three sizes queued back to back on one non-blocking stream, no host synchronisation between the calls: each
    rebuild must wait for the previous call's kernels before it rewrites the shared array."""
    torch.cuda.init()
    cases = [(1 << 20, 5, 0, 21), (107520, 3, 0, 22), (4096, 64, 1, 23)]
    xs = [torch.from_numpy(oracle.lcg_complex64(seed, n * b)).cuda() for n, b, _, seed in cases]
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    outs = []
    with torch.cuda.stream(side):
        for (n, b, d, _), x in zip(cases, xs):
            x.record_stream(side)
            outs.append(_static(x, n, b, d, sync=False))
    side.synchronize()
    for (n, b, d, _), x, got in zip(cases, xs, outs):
        want = _ordinary(x, n, b, d)
        assert torch.equal(got.view(torch.float32), want.view(torch.float32)), (n, b, d)


def test_static_scratch_rebuild_allocates_nothing():
    """The rebuild path (a new size) takes every table and the intermediate from the array: with every device
    allocation made to fail, rebuilds still succeed, and the device's free memory does not change."""
    torch.cuda.init()
    L = _lib.lib()
    cases = [(1 << 19, 3, 31), (3 * 5 * 7 * 2 ** 9, 2, 32), (1000, 40, 33)]
    xs = [torch.from_numpy(oracle.lcg_complex64(seed, n * b)).cuda() for n, b, seed in cases]
    outs = [torch.empty_like(x) for x in xs]
    # the ordinary plans first: their launches load every kernel these sizes use (module loading is lazy and takes
    # device memory the first time a kernel runs), and one static call loads the array itself
    wants = [_ordinary(x, n, b, 0) for (n, b, _), x in zip(cases, xs)]
    _static(torch.zeros(64, dtype=torch.complex64, device="cuda"), 64, 1, 0)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    L.crdfft_debug_fail_alloc_after(1)  # the next cudaMalloc the library makes fails
    try:
        for (n, b, _), x, o in zip(cases, xs, outs):
            st = L.crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(o.data_ptr()), n, b,
                                                 0, _stream())
            _lib.check(st, "execute_static_scratch")
        torch.cuda.synchronize()
    finally:
        L.crdfft_debug_fail_alloc_after(0)
    assert torch.cuda.mem_get_info()[0] == free0, "a rebuild allocated device memory"
    for (n, b, _), o, want in zip(cases, outs, wants):
        assert torch.equal(o.view(torch.float32), want.view(torch.float32)), (n, b)


def test_static_scratch_at_its_limits():
    """n = 2^22, the documented maximum, and a large prime (Bluestein) whose padded sequences fit; a prime whose
    padded length is 2^22 does not fit and is refused."""
    torch.cuda.init()
    for n, b, seed in ((1 << 22, 1, 41), (1048573, 1, 42)):
        x = torch.from_numpy(oracle.lcg_complex64(seed, n * b)).cuda()
        got = _static(x, n, b, 0)
        want = _ordinary(x, n, b, 0)
        assert torch.equal(got.view(torch.float32), want.view(torch.float32)), n
        del x, got, want
    x = torch.empty(2097143, dtype=torch.complex64, device="cuda")
    st = _lib.lib().crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                                  2097143, 1, 0, _stream())
    assert st == _lib.UNSUPPORTED_SIZE
    # after a refusal the next call rebuilds and works
    y = torch.from_numpy(oracle.lcg_complex64(43, 4096)).cuda()
    got = _static(y, 4096, 1, 0)
    assert oracle.rel_l2(got.cpu().numpy(), oracle.fft64(y.cpu().numpy())) <= REL_L2


def test_static_scratch_refuses_a_rebuild_during_capture():
    """A cached (n, batch) can be captured into a graph; a new (n, batch) during the capture is refused with
    CRDFFT_INVALID_ARG and queues nothing, so the capture stays valid, and the graph replays correctly while no
    rebuild has happened since."""
    torch.cuda.init()
    n, b = 4096, 16
    x = torch.from_numpy(oracle.lcg_complex64(51, n * b)).cuda()
    out = torch.empty_like(x)
    _static(x, n, b, 0)  # outside the capture: this (n, batch) is now the array's plan
    L = _lib.lib()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    refused = None
    with torch.cuda.graph(g, stream=side):
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                   n, b, 0, s), "captured call")
        refused = L.crdfft_execute_static_scratch(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                  2048, b, 0, s)
    assert refused == _lib.INVALID_ARG
    out.zero_()
    g.replay()
    torch.cuda.synchronize()
    want = _ordinary(x, n, b, 0)
    assert torch.equal(out.view(torch.float32), want.view(torch.float32))
