"""The two-pass four-step as one launch over L2-sized waves (crd_b200/csrc/chain_fft.cu, CRDFFT_CHAIN=1): every
wave's column tiles and row tiles run as one CTA a tile in list order, a row tile waiting on its wave's column tiles
and a column tile on the row tiles that last used its intermediate slot. Its output must be the same bits as the
wave-by-wave form's (the same line code and tables, other launches) and match the FP64 oracle, forward and inverse,
out of place and in place, over batches of several waves and slot reuses with a partial last wave; a wait that can
never be satisfied (test hook) must give up, report CRDFFT_DEVICE_TIMEOUT and leave the context usable."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu


def _plan(n, batch, chain, monkeypatch, slots="4", wave=None):
    monkeypatch.setenv("CRDFFT_CHAIN", "1" if chain else "0")
    monkeypatch.setenv("CRDFFT_CHAIN_SLOTS", slots)
    if wave is not None:
        monkeypatch.setenv("CRDFFT_CHAIN_WAVE_BYTES", str(wave))
    plan = cf.Plan([n], batch=batch)
    info = plan.info()
    assert info["algorithm"] == "four-step", info
    if chain:  # the counter reset and the one launch
        assert info["passes"] == 2, info
    return plan


# (n, batch, wave bytes, slots): 107520 = 105 x 1024 over 4 waves of 19 (the last partial), 2^20 = 1024 x 1024 over
# 5 waves of two (slots reused), 2^19 over 5 waves on 3 slots, a short 107520 wave that leaves 10 waves on 5 slots
CASES = [(107520, 64, None, "4"), (1 << 20, 9, None, "3"), (1 << 19, 20, None, "3"), (107520, 40, 4 << 20, "5")]


@pytest.mark.parametrize("n,batch,wave,slots", CASES)
@pytest.mark.parametrize("inverse", [False, True])
def test_chain_matches_waves_and_oracle(n, batch, wave, slots, inverse, monkeypatch):
    from crd_b200.hesap import device_status

    x = oracle.lcg_complex64(0xC4A1 ^ n, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    d = cf.INVERSE if inverse else cf.FORWARD
    ref_plan = _plan(n, batch, False, monkeypatch)
    ref = torch.empty_like(t)
    ref_plan.execute(t, ref, d)
    plan = _plan(n, batch, True, monkeypatch, slots, wave)
    o = torch.empty_like(t)
    plan.execute(t, o, d)
    plan.execute(t, o, d)  # a second execute: the counters start from zero again
    torch.cuda.synchronize()
    device_status(plan)
    got = o.cpu().numpy()
    rows = np.array([0, 1, batch // 2, batch - 2, batch - 1])
    want = oracle.fft64(x[rows], inverse)
    assert oracle.rel_l2(got[rows], want) <= 1e-6
    if n == 107520:  # the wave form runs the same line kernels (for 2^20 its column pass is the tensor-copy kernel)
        assert np.array_equal(got, ref.cpu().numpy())
    else:
        assert oracle.rel_l2(got, ref.cpu().numpy()) <= 1e-6


def test_chain_in_place_and_round_trip(monkeypatch):
    n, batch = 107520, 48
    x = oracle.lcg_complex64(0xC4A2, n * batch).reshape(batch, n)
    plan = _plan(n, batch, True, monkeypatch)
    t = torch.from_numpy(x).cuda()
    out = torch.empty_like(t)
    plan.execute(t, out, cf.FORWARD)
    t2 = t.clone()
    plan.execute(t2, t2, cf.FORWARD)  # in place: a wave's row tiles overwrite only input its column tiles have read
    torch.cuda.synchronize()
    assert np.array_equal(t2.cpu().numpy(), out.cpu().numpy())
    plan.execute(t2, t2, cf.INVERSE)
    torch.cuda.synchronize()
    back = t2.cpu().numpy() / n
    assert np.max(np.abs(back - x)) <= 1e-5


def test_chain_wait_runs_out_without_fault(monkeypatch):
    from crd_b200.hesap import device_status, stall_waits

    n, batch = 107520, 48
    x = torch.from_numpy(oracle.lcg_complex64(0xC4A3, n * batch)).cuda()
    y = torch.empty_like(x)
    stall_waits(True)
    try:
        bad = _plan(n, batch, True, monkeypatch)
    finally:
        stall_waits(False)
    bad.execute(x, y)
    with pytest.raises(cf.CrdFftError) as e:
        device_status(bad)
    assert e.value.status == 5
    good = _plan(n, batch, True, monkeypatch)
    good.execute(x, y)
    device_status(good)
    rows = np.array([0, batch - 1])
    want = oracle.fft64(x.cpu().numpy().reshape(batch, n)[rows])
    assert oracle.rel_l2(y.cpu().numpy().reshape(batch, n)[rows], want) <= 1e-6
