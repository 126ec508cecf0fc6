"""Fused FFT convolution (crdfft_conv_plan_create / crdfft_conv_execute) against the FP64 oracle:
y = IFFT(FFT(x) * H) * scale, rel-L2 <= 1e-6 (the FP32 bar of this project)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6


def _want(x, h, axes, scale):
    X = np.fft.fftn(x.astype(np.complex128), axes=axes)
    return np.fft.ifftn(X * h, axes=axes) * np.prod([x.shape[a] for a in axes]) * scale


@pytest.mark.parametrize("n", [16, 105, 256, 512, 1000, 1024, 4096, 8192])
@pytest.mark.parametrize("per_signal", [False, True])
def test_conv_1d(n, per_signal):
    batch = 37
    x = oracle.lcg_complex64(0xC0 ^ n, batch * n).reshape(batch, n)
    hs = oracle.lcg_complex64(0xC1 ^ n, (batch if per_signal else 1) * n).reshape(-1, n)
    plan = cf.ConvPlan([n], batch=batch, per_signal_filter=per_signal)
    assert plan.info()["algorithm"] == "fused-conv"
    out = torch.empty(batch, n, dtype=torch.complex64, device="cuda")
    plan.execute(torch.from_numpy(x).cuda(), torch.from_numpy(hs).cuda(), out)
    torch.cuda.synchronize()
    want = _want(x, hs.astype(np.complex128), (1,), 1.0 / n)
    rl2 = oracle.rel_l2(out.cpu().numpy(), want)
    assert rl2 <= REL_L2, f"n={n}: rel-L2 {rl2:.2e}"


def test_conv_is_circular_convolution_and_in_place():
    """With H = FFT(h) and the default 1/N scale the result is the circular convolution of x with h."""
    n, batch = 1024, 8
    x = oracle.lcg_complex64(0xC2, batch * n).reshape(batch, n)
    h = np.zeros(n, dtype=np.complex64)
    h[:5] = [0.5, 0.25, -0.125, 0.0625, 1.0]
    H = np.fft.fft(h.astype(np.complex128)).astype(np.complex64)
    t = torch.from_numpy(x.copy()).cuda()
    cf.ConvPlan([n], batch=batch).execute(t, torch.from_numpy(H).cuda(), t)
    torch.cuda.synchronize()
    want = np.stack([sum(h[k] * np.roll(x[b].astype(np.complex128), k) for k in range(5)) for b in range(batch)])
    assert oracle.rel_l2(t.cpu().numpy(), want) <= REL_L2


@pytest.mark.parametrize("dims", [(64, 64), (256, 1024), (105, 96), (1024, 256)])
@pytest.mark.parametrize("per_signal", [False, True])
def test_conv_2d(dims, per_signal):
    batch = 3
    x = oracle.lcg_complex64(0xC3 ^ dims[0], batch * dims[0] * dims[1]).reshape(batch, *dims)
    hs = oracle.lcg_complex64(0xC4 ^ dims[1], (batch if per_signal else 1) * dims[0] * dims[1]).reshape(-1, *dims)
    plan = cf.ConvPlan(list(dims), batch=batch, per_signal_filter=per_signal, scale=0.5)
    assert plan.info()["algorithm"] == "fused-conv-2d"
    out = torch.empty(batch, *dims, dtype=torch.complex64, device="cuda")
    plan.execute(torch.from_numpy(x).cuda(), torch.from_numpy(hs).cuda(), out)
    torch.cuda.synchronize()
    want = _want(x, hs.astype(np.complex128), (1, 2), 0.5)
    rl2 = oracle.rel_l2(out.cpu().numpy(), want)
    assert rl2 <= REL_L2, f"{dims}: rel-L2 {rl2:.2e}"


def test_conv_plan_errors():
    with pytest.raises(cf.CrdFftError):
        cf.ConvPlan([16384])          # longer than one CTA's lines
    with pytest.raises(cf.CrdFftError):
        cf.ConvPlan([8, 8, 8])        # rank 3
    p = cf.ConvPlan([256], batch=2)
    x = torch.zeros(512, dtype=torch.complex64, device="cuda")
    assert cf.hesap.lib().crdfft_execute(p._h, x.data_ptr(), x.data_ptr(), 0, None) == 7  # CRDFFT_INVALID_ARG
