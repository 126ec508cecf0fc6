"""Host-memory execute (crdfft_execute_host): the plan runs on pinned host buffers in overlapped chunks and gives the
same result as the device execute."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,batch", [(4096, 20000), (65536, 300), (1000, 9), (1 << 20, 3)])
def test_host_execute_matches_device_execute(n, batch):
    x = oracle.lcg_complex64(0x4057 ^ n, n * batch)
    plan = cf.Plan([n], batch=batch)
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.empty_like(d_in)
    plan.execute(d_in, d_out)
    h_in = torch.from_numpy(x).pin_memory()
    h_out = torch.empty(n * batch, dtype=torch.complex64).pin_memory()
    for _ in range(2):  # the second call reuses the staging buffers and chunk plans
        h_out.zero_()
        plan.execute_host(h_in, h_out)
        torch.cuda.synchronize()
        assert np.array_equal(h_out.numpy(), d_out.cpu().numpy())
    t = 0 if batch < 3 else batch // 2
    assert oracle.rel_l2(h_out.numpy()[t * n:(t + 1) * n], oracle.fft64(x[t * n:(t + 1) * n])) <= 1e-6


def test_host_execute_real_padded_and_in_place():
    n, batch = 1 << 16, 700
    idist, odist = n + 8, n // 2 + 1 + 4
    x = oracle.lcg_float32(0x4058, batch * idist)
    r2c = cf.Plan([n], batch=batch, kind=cf.R2C, idist=idist, odist=odist)
    h_spec = torch.zeros(batch * odist, dtype=torch.complex64).pin_memory()
    r2c.execute_host(torch.from_numpy(x).pin_memory(), h_spec)
    torch.cuda.synchronize()
    d_spec = torch.zeros(batch * odist, dtype=torch.complex64, device="cuda")
    r2c.execute(torch.from_numpy(x).cuda(), d_spec)
    assert np.array_equal(h_spec.numpy(), d_spec.cpu().numpy())
    c = oracle.lcg_complex64(0x4059, 4096 * 50)
    h = torch.from_numpy(c.copy()).pin_memory()
    cf.Plan([4096], batch=50).execute_host(h, h, cf.INVERSE)
    torch.cuda.synchronize()
    assert oracle.rel_l2(h.numpy(), oracle.fft64(c.reshape(50, 4096), True).ravel()) <= 1e-6


def test_host_execute_rejects_device_tensors_and_uneven_plans():
    plan = cf.Plan([64], batch=2)
    with pytest.raises(ValueError):
        plan.execute_host(torch.zeros(128, dtype=torch.complex64, device="cuda"), torch.zeros(128, dtype=torch.complex64))
