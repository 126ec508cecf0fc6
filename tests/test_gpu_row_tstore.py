"""The four-step row pass with its transposed tile stored by the Tensor Memory Accelerator (`row_tstore_kernel`,
crd_b200/csrc/tma_col.cu): the measuring planner offers it as a launch shape of the 2^20 and 2^19 row passes; forced
through wisdom it must give the same output as the thread-stored form, bit for bit (same stages, same arithmetic),
and match the FP64 oracle, forward and inverse (the inverse's conjugation rides in the tile). An output off a
16-byte boundary runs the same shape thread-stored."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import crd_b200.hesap as F
import oracle

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6


def _row_pass_keys(n: int, batch: int) -> dict:
    """Plan n x batch in measure mode from empty wisdom; return {key: [log lines]} of the passes for which a
    tensor-store candidate was timed."""
    F.wisdom_forget()
    F.set_planner("measure")
    try:
        cf.Plan([n], batch=batch)
        log = F.planner_log()
    finally:
        F.set_planner("estimate")
    keys = {}
    for line in log.splitlines():
        if " tstore=1 " in line:
            keys.setdefault(line.split()[0], []).append(line)
    return keys


def _run(n, batch, x, direction):
    t = torch.from_numpy(x).cuda()
    out = torch.empty_like(t)
    plan = cf.Plan([n], batch=batch)
    plan.execute(t, out, direction)
    torch.cuda.synchronize()
    return out.cpu().numpy(), plan.info()


@pytest.mark.parametrize("n", [1 << 20, 1 << 19])
def test_tensor_store_row_pass_matches_thread_store_and_oracle(n):
    batch = 3
    keys = _row_pass_keys(n, batch)
    assert keys, "the planner offered no tensor-store row pass"
    for line in next(iter(keys.values())):
        ms = float(line.split(" ms=")[1].split()[0])
        assert ms > 0, line  # every timed candidate ran
    x = oracle.lcg_complex64(0x7570 ^ n, n * batch).reshape(batch, n)
    for inverse in (False, True):
        direction = cf.INVERSE if inverse else cf.FORWARD
        want = oracle.fft64(x, inverse)
        outs = {}
        for tstore in (False, True):
            lpc = 4
            text = "crdfft-wisdom 1\n" + "".join(
                f"{k} 0 16 {lpc} 0.1{' t' if tstore else ''}\n" for k in keys)
            F.wisdom_forget()
            F.wisdom_import(text)
            got, info = _run(n, batch, x, direction)
            assert info["algorithm"] == "four-step"
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            assert err <= REL_L2, (n, inverse, tstore, err)
            outs[tstore] = got
        assert np.array_equal(outs[False], outs[True]), (n, inverse)
        # an output 8 bytes off a 16-byte boundary cannot take the tensor map: the same shape runs thread-stored
        t = torch.from_numpy(x).cuda()
        big = torch.empty(n * batch + 1, dtype=torch.complex64, device="cuda")
        off = big[1:].view(batch, n)
        assert off.data_ptr() % 16 == 8
        cf.Plan([n], batch=batch).execute(t, off, direction)
        torch.cuda.synchronize()
        assert np.array_equal(off.cpu().numpy(), outs[True]), (n, inverse, "offset output")
    F.wisdom_forget()
