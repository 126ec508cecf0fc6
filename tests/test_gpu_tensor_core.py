"""Tensor-core precision forms (crd_b200/csrc/tc_fft.cu) against the FP64 oracle, through the C ABI.

* split-BF16 (CRDFFT_PREC_SPLIT_BF16): rel-L2 against FP64 <= 1e-6, the same bar as the FP32 path.
* FP16 with a per-line power-of-two scale (CRDFFT_PREC_FP16_SCALED): about 11 significant bits in the first stage;
  rel-L2 against FP64 <= 2e-3 here, and it is reported as a low-precision form, not held to 1e-6.

* split-FP16 hi+lo with a per-line scale, three products (CRDFFT_PREC_SPLIT_FP16_2): about 22 significant bits;
  rel-L2 against FP64 <= 1e-6, also on lines of very different magnitude and with 1 % of entries scaled by 1e4.
* split-BF16 hi+lo, three products (CRDFFT_PREC_SPLIT_BF16_2, the two-term form): about 16 significant bits of the
  data; reported, held to 2e-5 here (it cannot reach 1e-6).

Passes the tensor-core kernel cannot take (strided loads, other radix schedules) run on the FP32 kernels within the
same plan; the plan's algorithm string says when a tensor-core pass is present.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu

SPLIT_REL_L2 = 1e-6
FP16_REL_L2 = 2e-3


def _run(dims, batch, precision, inverse, seed):
    total = int(np.prod(dims)) * batch
    x = oracle.lcg_complex64(seed, total).reshape((batch,) + tuple(dims))
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    plan = cf.Plan(list(dims), batch=batch, precision=precision)
    plan.execute(t, o, cf.INVERSE if inverse else cf.FORWARD)
    torch.cuda.synchronize()
    axes = tuple(range(1, len(dims) + 1))
    xd = x.astype(np.complex128)
    want = np.fft.ifftn(xd, axes=axes) * np.prod(dims) if inverse else np.fft.fftn(xd, axes=axes)
    return o.cpu().numpy(), want, plan


@pytest.mark.parametrize("n", [512, 1024, 4096])
@pytest.mark.parametrize("inverse", [False, True])
def test_split_bf16_1d(n, inverse):
    got, want, plan = _run([n], 37, cf.PREC_SPLIT_BF16, inverse, 0x7C0 ^ n)
    assert plan.info()["algorithm"].endswith("+tc-bf16x3")
    rl2 = oracle.rel_l2(got, want)
    assert rl2 <= SPLIT_REL_L2, f"n={n}: rel-L2 {rl2:.3e}"
    assert oracle.max_rel(got, want) <= oracle.f32_class(n)


@pytest.mark.parametrize("n", [512, 1024, 4096])
@pytest.mark.parametrize("inverse", [False, True])
def test_fp16_scaled_1d(n, inverse):
    got, want, plan = _run([n], 37, cf.PREC_FP16_SCALED, inverse, 0x7C1 ^ n)
    assert plan.info()["algorithm"].endswith("+tc-fp16")
    rl2 = oracle.rel_l2(got, want)
    assert rl2 <= FP16_REL_L2, f"n={n}: rel-L2 {rl2:.3e}"


def test_fp16_scale_follows_each_line():
    """Lines of very different magnitude in one CTA each keep their own relative accuracy."""
    n, batch = 512, 16
    x = oracle.lcg_complex64(0x7C2, n * batch).reshape(batch, n)
    mags = (2.0 ** np.arange(-24, 24, 3)).astype(np.float32)
    x = (x * mags[:, None]).astype(np.complex64)
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    cf.Plan([n], batch=batch, precision=cf.PREC_FP16_SCALED).execute(t, o)
    torch.cuda.synchronize()
    got = o.cpu().numpy()
    want = np.fft.fft(x.astype(np.complex128), axis=1)
    for b in range(batch):
        assert oracle.rel_l2(got[b], want[b]) <= FP16_REL_L2, f"line {b} (scale {mags[b]:.1e})"


@pytest.mark.parametrize("dims", [(64, 1024), (16, 4096), (8, 16, 512)])
def test_split_bf16_nd(dims):
    for inverse in (False, True):
        got, want, plan = _run(dims, 2, cf.PREC_SPLIT_BF16, inverse, 0x7C3 ^ int(np.prod(dims)))
        assert "+tc" in plan.info()["algorithm"]
        rl2 = oracle.rel_l2(got, want)
        assert rl2 <= SPLIT_REL_L2, f"{dims}: rel-L2 {rl2:.3e}"


def test_partial_last_cta_and_in_place():
    """A line count that leaves the last CTA partly empty, run in place: the other lines are untouched."""
    n, batch = 1024, 7  # 4 lines a CTA
    x = oracle.lcg_complex64(0x7C4, n * (batch + 1)).reshape(batch + 1, n)
    t = torch.from_numpy(x).cuda()
    cf.Plan([n], batch=batch, precision=cf.PREC_SPLIT_BF16).execute(t[:batch], t[:batch])
    torch.cuda.synchronize()
    got = t.cpu().numpy()
    want = np.fft.fft(x[:batch].astype(np.complex128), axis=1)
    assert oracle.rel_l2(got[:batch], want) <= SPLIT_REL_L2
    assert np.array_equal(got[batch], x[batch])


def test_sizes_without_tensor_core_pass_run_fp32():
    """Sizes whose passes the tensor-core kernel does not take still plan and run at FP32 accuracy."""
    for n in (105, 2048, 65536):
        got, want, plan = _run([n], 2, cf.PREC_SPLIT_BF16, False, 0x7C5 ^ n)
        assert "+tc" not in plan.info()["algorithm"]
        assert oracle.rel_l2(got, want) <= SPLIT_REL_L2


def test_split_bf16_matches_fp32_closely():
    n, batch = 4096, 64
    x = oracle.lcg_complex64(0x7C6, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    o32 = torch.empty_like(t)
    otc = torch.empty_like(t)
    cf.Plan([n], batch=batch).execute(t, o32)
    cf.Plan([n], batch=batch, precision=cf.PREC_SPLIT_BF16).execute(t, otc)
    torch.cuda.synchronize()
    assert oracle.rel_l2(otc.cpu().numpy(), o32.cpu().numpy().astype(np.complex128)) <= 1e-6


HILO_BF16_REL_L2 = 2e-5


@pytest.mark.parametrize("n", [512, 1024, 4096])
@pytest.mark.parametrize("inverse", [False, True])
def test_split_fp16_hilo_1d(n, inverse):
    got, want, plan = _run([n], 37, cf.PREC_SPLIT_FP16_2, inverse, 0x7C7 ^ n)
    assert plan.info()["algorithm"].endswith("+tc-fp16x2")
    rl2 = oracle.rel_l2(got, want)
    assert rl2 <= SPLIT_REL_L2, f"n={n}: rel-L2 {rl2:.3e}"


@pytest.mark.parametrize("n", [512, 4096])
def test_split_bf16_hilo_1d_reported(n):
    got, want, plan = _run([n], 37, cf.PREC_SPLIT_BF16_2, False, 0x7C8 ^ n)
    assert plan.info()["algorithm"].endswith("+tc-bf16x2")
    rl2 = oracle.rel_l2(got, want)
    print(f"split-BF16 hi+lo n={n}: rel-L2 {rl2:.3e}")
    assert rl2 <= HILO_BF16_REL_L2, f"n={n}: rel-L2 {rl2:.3e}"


def test_split_fp16_hilo_scale_and_outliers():
    """Lines of very different magnitude, and 1 % of entries scaled by 1e4: each line keeps rel-L2 <= 1e-6."""
    n, batch = 4096, 16
    x = oracle.lcg_complex64(0x7C9, n * batch).reshape(batch, n)
    mags = (2.0 ** np.arange(-24, 24, 3)).astype(np.float32)
    x = (x * mags[:, None]).astype(np.complex64)
    idx = np.random.default_rng(7).choice(x.size, size=x.size // 100, replace=False)
    x.reshape(-1)[idx] *= np.float32(1e4)
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    cf.Plan([n], batch=batch, precision=cf.PREC_SPLIT_FP16_2).execute(t, o)
    torch.cuda.synchronize()
    got = o.cpu().numpy()
    want = np.fft.fft(x.astype(np.complex128), axis=1)
    for b in range(batch):
        assert oracle.rel_l2(got[b], want[b]) <= SPLIT_REL_L2, f"line {b} (scale {mags[b]:.1e})"
