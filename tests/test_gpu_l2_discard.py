"""Four-step transforms in L2-sized waves (transforms of 2 MiB and less, two internal streams): the row pass drops
the intermediate's L2 lines once it has read them (`discard.global.L2`, crd_b200/csrc/line_fft.cuh), so that L2 does
not write the dead intermediate back to HBM. The output must be the same bits as with the lines kept
(CRDFFT_L2_DISCARD=0) and with the waves on three internal streams instead of two (CRDFFT_L2_LANES=3), and match the
FP64 oracle, over batches of several waves (the workspace slots are reused after a discard), forward and inverse."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,batch", [(107520, 75), (1 << 18, 30), (3 * 5 * 7 * 512, 140), (1 << 17, 60)])
@pytest.mark.parametrize("inverse", [False, True])
def test_l2_wave_discard_keeps_results(n, batch, inverse, monkeypatch):
    x = oracle.lcg_complex64(0xD15C ^ n, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    d = cf.INVERSE if inverse else cf.FORWARD
    outs = {}
    for lanes in ("2", "3"):
        for flag in ("1", "0"):
            monkeypatch.setenv("CRDFFT_L2_LANES", lanes)
            monkeypatch.setenv("CRDFFT_L2_DISCARD", flag)
            plan = cf.Plan([n], batch=batch)
            assert plan.info()["algorithm"] == "four-step", plan.info()
            o = torch.empty_like(t)
            plan.execute(t, o, d)
            plan.execute(t, o, d)  # a second execute over the same slots
            torch.cuda.synchronize()
            outs[lanes, flag] = o.cpu().numpy()
    for key, got in outs.items():
        assert np.array_equal(got, outs["2", "1"]), (n, inverse, key)
    rows = np.array([0, batch // 2, batch - 1])
    want = oracle.fft64(x[rows], inverse)
    assert oracle.rel_l2(outs["2", "1"][rows], want) <= 1e-6
