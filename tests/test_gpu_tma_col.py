"""The four-step column pass on the tensor-copy kernel (crd_b200/csrc/tma_col.cu): 2-D bulk tensor copies of
1024- and 512-point column tiles into shared memory, several tiles in flight a CTA. Against the FP64 oracle, and
against the line kernel's column pass (CRDFFT_TMA_COL=0), which runs the same stages."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,batch", [(1 << 20, 3), (1 << 19, 5), (1 << 18, 9), (3 * 1024 * 512, 2)])
@pytest.mark.parametrize("inverse", [False, True])
def test_tma_column_pass_matches_line_kernel_and_oracle(n, batch, inverse, monkeypatch):
    x = oracle.lcg_complex64(0x7A ^ n, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    a = torch.empty_like(t)
    b = torch.empty_like(t)
    d = cf.INVERSE if inverse else cf.FORWARD
    cf.Plan([n], batch=batch, norm=cf.NORM_INVERSE).execute(t, a, d)
    monkeypatch.setenv("CRDFFT_TMA_COL", "0")
    cf.Plan([n], batch=batch, norm=cf.NORM_INVERSE).execute(t, b, d)
    torch.cuda.synchronize()
    got = a.cpu().numpy()
    want = (np.fft.ifft if inverse else np.fft.fft)(x[:2].astype(np.complex128), axis=1)
    assert oracle.rel_l2(got[:2], want) <= 1e-6
    assert np.array_equal(got, b.cpu().numpy())  # the same stages in the same order: the same bits


def test_tma_column_pass_in_l2_waves_and_padded_distance():
    """Transforms of 2 MiB and less run in L2-sized waves on two streams; a padded distance keeps the line kernel."""
    n, batch = 1 << 18, 40
    x = oracle.lcg_complex64(0x7B, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    cf.Plan([n], batch=batch).execute(t, o)
    torch.cuda.synchronize()
    want = np.fft.fft(x[-3:].astype(np.complex128), axis=1)
    assert oracle.rel_l2(o.cpu().numpy()[-3:], want) <= 1e-6
    idist = n + 8
    xp = torch.from_numpy(oracle.lcg_complex64(0x7C, idist * 3)).cuda()
    op = torch.empty(n * 3, dtype=torch.complex64, device="cuda")
    cf.Plan([n], batch=3, idist=idist, odist=n).execute(xp, op)
    torch.cuda.synchronize()
    xs = xp.cpu().numpy().reshape(3, idist)[:, :n].astype(np.complex128)
    assert oracle.rel_l2(op.cpu().numpy().reshape(3, n), np.fft.fft(xs, axis=1)) <= 1e-6
