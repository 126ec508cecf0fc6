"""The reference's own GPU FFT kernels (its CKIR compiler's CUDA output for N = 1024, built from the reference tree by
`make -C oracle ckir`) on the same B200, beside this library and cuFFT: their results agree with the FP64 oracle,
and the timings of the three on the N = 1024 x 4096 batch are reported (set CRDFFT_COMPARE_OUT to a path to keep
them as JSON)."""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libckir.so")
N = 1024


def _ckir():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libckir.so not built (make -C oracle ckir, needs the reference sources)")
    L = ctypes.CDLL(LIB)
    for f in (L.ckref_fft1024_r16, L.ckref_fft1024_r4):
        f.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int, ctypes.c_void_p]
        f.restype = ctypes.c_int
    return L


def _twiddles():
    k = np.arange(N)
    w = np.exp(-2j * np.pi * k / N)
    return (torch.from_numpy(w.real.astype(np.float32)).cuda(), torch.from_numpy(w.imag.astype(np.float32)).cuda())


@pytest.mark.parametrize("kernel", ["ckref_fft1024_r16", "ckref_fft1024_r4"])
def test_reference_kernels_compute_the_forward_fft(kernel):
    L = _ckir()
    batch = 64
    x = oracle.lcg_complex64(0xCC1, batch * N).reshape(batch, N)
    re = torch.from_numpy(np.ascontiguousarray(x.real)).cuda()
    im = torch.from_numpy(np.ascontiguousarray(x.imag)).cuda()
    ore, oim = torch.empty_like(re), torch.empty_like(im)
    twr, twi = _twiddles()
    assert getattr(L, kernel)(re.data_ptr(), im.data_ptr(), twr.data_ptr(), twi.data_ptr(), ore.data_ptr(),
                              oim.data_ptr(), batch, None) == 0
    torch.cuda.synchronize()
    got = ore.cpu().numpy() + 1j * oim.cpu().numpy()
    assert oracle.rel_l2(got, oracle.fft64(x)) <= 1e-6


def _graph(fn):
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        fn()
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g


def _time(g, reps=20):
    for _ in range(3):
        g.replay()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def test_n1024_beside_reference_kernels_and_cufft():
    """N = 1024, batch 4096 (64 MiB in and out per transform batch), eight buffer sets in turn (512 MiB, beyond L2),
    each arm as one CUDA graph of eight launches."""
    L = _ckir()
    batch, ring = 4096, 8
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5)
    xs = [(torch.rand(batch, N, 2, generator=gen, device="cuda") * 2 - 1).view(torch.complex64).view(batch, N)
          for _ in range(ring)]
    ys = [torch.empty_like(x) for x in xs]
    planes = [(x.real.contiguous(), x.imag.contiguous()) for x in xs]
    outs = [(torch.empty_like(p[0]), torch.empty_like(p[1])) for p in planes]
    twr, twi = _twiddles()
    import crd_b200.hesap as F

    wisdom = os.path.join(os.path.dirname(os.path.dirname(oracle.__file__)), "profiles", "wisdom_b200.txt")
    if os.path.exists(wisdom):
        with open(wisdom) as f:
            F.wisdom_import(f.read())
    F.set_planner("measure")  # the launch shape the bench uses
    try:
        plan = cf.Plan([N], batch=batch)
    finally:
        F.set_planner("estimate")

    def ours():
        for x, y in zip(xs, ys):
            plan.execute(x, y)

    def ref_r16():
        s = torch.cuda.current_stream().cuda_stream
        for (re, im), (ore, oim) in zip(planes, outs):
            L.ckref_fft1024_r16(re.data_ptr(), im.data_ptr(), twr.data_ptr(), twi.data_ptr(), ore.data_ptr(),
                                oim.data_ptr(), batch, s)

    def cufft():
        for x, y in zip(xs, ys):
            torch.fft.fft(x, out=y)

    res = {}
    for name, fn in (("crd_b200", ours), ("reference_ckir_r16", ref_r16), ("cufft", cufft)):
        ms = _time(_graph(fn)) / ring
        res[name] = {"ms_per_batch": round(ms, 5), "gflops": round(5 * N * 10 * batch / (ms / 1e3) / 1e9, 1),
                     "hbm_fraction_16B_per_point": round(16 * N * batch / (ms / 1e3) / 6470e9, 3)}
    print(json.dumps(res))
    out = os.environ.get("CRDFFT_COMPARE_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    # results of every arm agree (ours checked against the oracle elsewhere)
    ref_r16()
    torch.cuda.synchronize()
    ours()
    torch.cuda.synchronize()
    got = outs[0][0].cpu().numpy() + 1j * outs[0][1].cpu().numpy()
    assert oracle.rel_l2(got, ys[0].cpu().numpy().astype(np.complex128)) <= 1e-6
