"""Decompositions of a 1-D transform: every decomposition the planner may pick (one pass, the cluster four-step,
the two-pass four-step for each split n1 x n2 whose halves fit one CTA), forced through crdfft_set_decomposition,
against the FP64 oracle at rel-L2 <= 1e-6; and the measuring and learned planners choose among them and remember
the choice as wisdom."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import crd_b200.hesap as F
import oracle
from crd_b200 import _lib

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6


def _smooth(v: int) -> bool:
    for p in (2, 3, 5, 7):
        while v % p == 0:
            v //= p
    return v == 1


def _single_ok(v: int) -> bool:
    return _smooth(v) and (v <= 8192 or v == 16384)


# line lengths with a compile-time schedule (crd_b200/csrc/sched_*.cu)
STATIC = {16, 32, 64, 105, 128, 256, 512, 1024, 2048, 4096, 8192, 16384}


def _splits(n: int):
    """The splits the planner times (both halves with compile-time schedules), plus the two admissible splits
    closest to square, which run the run-time schedule when a half has none."""
    ok = [a for a in range(16, n // 16 + 1) if n % a == 0 and _single_ok(a) and _single_ok(n // a)]
    stat = [a for a in ok if a in STATIC and n // a in STATIC]
    rest = sorted((a for a in ok if a not in stat), key=lambda a: abs(np.log(a * a / n)))[:2]
    return stat + rest


@pytest.fixture(autouse=True)
def _clear_overrides():
    yield
    for n in (4096, 8192, 65536, 107520, 1 << 20, 53760):
        _lib.lib().crdfft_set_decomposition(n, 0, 0)


@pytest.mark.parametrize("n", [4096, 65536, 107520, 53760, 1 << 20])
def test_every_four_step_split_matches_oracle(n):
    L = _lib.lib()
    batch = 2
    x = oracle.lcg_complex64(0xDEC ^ n, n * batch).reshape(batch, n)
    want = oracle.fft64(x)
    t = torch.from_numpy(x).cuda()
    for a in _splits(n):
        assert L.crdfft_set_decomposition(n, 3, a) == _lib.OK
        plan = cf.Plan([n], batch=batch)
        assert plan.info()["algorithm"] == "four-step"
        assert plan.info()["factors"][:2] == [a, n // a], (n, a)
        o = torch.empty_like(t)
        plan.execute(t, o, cf.FORWARD)
        back = torch.empty_like(t)
        cf.Plan([n], batch=batch, norm=cf.NORM_INVERSE).execute(o, back, cf.INVERSE)
        torch.cuda.synchronize()
        got = o.cpu().numpy()
        assert oracle.rel_l2(got, want) <= REL_L2, (n, a)
        assert oracle.rel_l2(back.cpu().numpy(), x) <= 2 * REL_L2, (n, a)


def test_override_kinds():
    L = _lib.lib()
    assert L.crdfft_set_decomposition(65536, 2, 0) == _lib.OK
    assert cf.Plan([65536], batch=2).info()["algorithm"] == "cluster-four-step"
    assert L.crdfft_set_decomposition(4096, 1, 0) == _lib.OK
    assert cf.Plan([4096], batch=2).info()["algorithm"] == "single-pass"
    assert L.crdfft_set_decomposition(1 << 20, 1, 0) == _lib.OK  # not admissible: the planner decides
    assert cf.Plan([1 << 20], batch=1).info()["algorithm"] == "four-step"
    assert L.crdfft_set_decomposition(100, 3, 7) == _lib.INVALID_ARG
    assert L.crdfft_set_decomposition(100, 4, 0) == _lib.INVALID_ARG


@pytest.mark.parametrize("mode", ["measure", "learned"])
def test_planner_picks_and_remembers_a_decomposition(mode):
    """The measuring planner times every decomposition of 2^20 (the learned one only the model's top proposals, or
    all of them without a decomposition model) and remembers the fastest as wisdom; a later plan reads it back."""
    n, batch = 1 << 20, 4
    F.wisdom_forget()
    F.set_planner(mode)
    try:
        plan = cf.Plan([n], batch=batch)
        log = F.planner_log()
        wis = F.wisdom_export()
    finally:
        F.set_planner("estimate")
    lines = [ln for ln in log.splitlines() if " decomp " in ln]
    assert lines, "no decomposition was timed"
    assert sum(" best" in ln for ln in lines) == 1
    assert any(ln.startswith("D|") for ln in wis.splitlines())
    best = next(ln for ln in lines if " best" in ln)
    n1 = int(best.split("n1=")[1].split()[0])
    kind = int(best.split("kind=")[1].split()[0])
    if kind == 3:
        assert plan.info()["factors"][:2] == [n1, n // n1]
    # estimate mode now reads the decomposition from wisdom
    again = cf.Plan([n], batch=batch)
    assert again.info()["factors"] == plan.info()["factors"]
    x = oracle.lcg_complex64(0xDED, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    again.execute(t, o)
    torch.cuda.synchronize()
    assert oracle.rel_l2(o.cpu().numpy(), oracle.fft64(x)) <= REL_L2
    F.wisdom_forget()
