"""GPU parity: the CUDA path (through the C ABI in include/crdfft.h) against the FP64 oracle and the reference's own
FP32 outputs, on the reference tests' seeded inputs.

Tolerances, written per test:
* rel-L2 against the FP64 oracle <= 1e-6 (the FP32 accuracy bar of this project), and
* max|gpu - oracle| / (1 + max|oracle|) within the reference's own f32 class: 2e-4 below 2^19, 1e-3 from 2^19
  (tests/numerics/hesap-fft/test_fft_kernels.cpp:138-163), and against the reference's FP32 output too.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6


def _check(got, want, n, what=""):
    rl2 = oracle.rel_l2(got, want)
    mr = oracle.max_rel(got, want)
    assert rl2 <= REL_L2, f"{what} n={n}: rel-L2 {rl2:.3e} > {REL_L2}"
    assert mr <= oracle.f32_class(n), f"{what} n={n}: max-rel {mr:.3e}"
    return rl2


def _c2c(n, batch, inverse, seed=None, norm=cf.NORM_NONE):
    seed = (0x9E3779B97F4A7C15 ^ n) if seed is None else seed
    x = oracle.lcg_complex64(seed, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    plan = cf.Plan([n], batch=batch, norm=norm)
    plan.execute(t, o, cf.INVERSE if inverse else cf.FORWARD)
    torch.cuda.synchronize()
    return x, o.cpu().numpy(), plan


SINGLE = [1, 2, 3, 4, 5, 7, 8, 9, 16, 32, 64, 105, 128, 240, 256, 512, 1000, 1024, 2048, 3000, 4096, 6144, 8192,
          16384]


@pytest.mark.parametrize("n", SINGLE)
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_single_pass(n, inverse):
    batch = 5 if n <= 4096 else 2
    x, got, plan = _c2c(n, batch, inverse)
    assert plan.info()["algorithm"] == "single-pass"
    _check(got, oracle.fft64(x, inverse), n)


@pytest.mark.parametrize("n", [27, 81, 243, 729, 2187, 6561, 5103, 3 * 3 * 5 * 5 * 7 * 16, 25, 125, 625, 3125, 1000,
                               3000, 5625, 7875])
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_radix9_lengths(n, inverse):
    """Lengths with 3^2 or 5^2 as a factor run radix-9 and radix-25 stages (two radix-3 or radix-5 stages in one):
    single passes and a four-step."""
    x, got, plan = _c2c(n, 3, inverse)
    _check(got, oracle.fft64(x, inverse), n)


def test_c2c_radix9_four_step():
    n = 3 ** 10  # 243 x 243, each half 9 x 9 x 3
    x, got, plan = _c2c(n, 2, False)
    assert plan.info()["algorithm"] == "four-step"
    _check(got, oracle.fft64(x), n)


@pytest.mark.parametrize("n", [32768, 65536, 107520, 3 * 5 * 7 * 2 ** 9, 2 ** 20])
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_four_step(n, inverse):
    batch = 3 if n < 2 ** 20 else 2
    x, got, plan = _c2c(n, batch, inverse)
    assert plan.info()["algorithm"] in ("four-step", "cluster-four-step")
    _check(got, oracle.fft64(x, inverse), n)


@pytest.mark.parametrize("inverse", [False, True])
def test_cluster_four_step_matches_two_pass(inverse, monkeypatch):
    """The cluster-fused four-step (DSMEM transpose) and the two-pass four-step agree with the oracle and with each
    other, in place too."""
    n, batch = 65536, 5
    x, got, plan = _c2c(n, batch, inverse)
    assert plan.info()["algorithm"] == "cluster-four-step"
    want = oracle.fft64(x, inverse)
    _check(got, want, n)
    monkeypatch.setenv("CRDFFT_NO_CLUSTER", "1")
    x2, got2, plan2 = _c2c(n, batch, inverse)
    assert plan2.info()["algorithm"] == "four-step"
    _check(got2, want, n)
    monkeypatch.delenv("CRDFFT_NO_CLUSTER")
    t = torch.from_numpy(x.copy()).cuda()
    cf.Plan([n], batch=batch).execute(t, t, cf.INVERSE if inverse else cf.FORWARD)
    _check(t.cpu().numpy(), want, n, "in place")


def test_four_step_waves(monkeypatch):
    """A batch larger than one L2 wave runs as several waves; each transform must come out the same."""
    n = 1 << 17
    monkeypatch.setenv("CRDFFT_WAVE_BYTES", str(n * 8 * 2))  # two transforms a wave
    x, got, plan = _c2c(n, 5, False, seed=77)
    assert plan.info()["algorithm"] == "four-step"
    _check(got, oracle.fft64(x), n)


@pytest.mark.parametrize("n", [11, 17, 143, 1009, 1031])
def test_bluestein_sizes(n):
    """Sizes with a prime factor above 7 run the chirp-z path; inverse normalised as BluesteinPlan's."""
    for inverse in (False, True):
        x, got, plan = _c2c(n, 3, inverse, norm=cf.NORM_INVERSE)
        assert plan.info()["algorithm"] == "bluestein"
        want = oracle.fft64(x, inverse) / (n if inverse else 1)
        _check(got, want, n)


@pytest.mark.parametrize("n", [17, 100, 360, 1009, 4000])
def test_bluestein_plan_class(n):
    """BluesteinPlan<float>(n).execute in place vs the FP64 restatement of the reference's Bluestein."""
    x = oracle.lcg_complex64(0x9E3779B97F4A7C15 ^ n, n)
    for inverse in (False, True):
        t = torch.from_numpy(x.copy()).cuda()
        cf.BluesteinPlan(n).execute(t, cf.INVERSE if inverse else cf.FORWARD)
        _check(t.cpu().numpy(), oracle.bluestein64(x, inverse), n)


@pytest.mark.parametrize("n,batch", [(64, 7), (64, 8), (1024, 3), (105, 4), (65536, 2)])
def test_execute_batched_element_major(n, batch):
    """FftPlan::execute_batched: element i of transform t at data[i*batch + t] (fft.hpp:462-470)."""
    x = oracle.lcg_complex64(n * 31 + batch, n * batch)
    t = torch.from_numpy(x.copy()).cuda()
    cf.FftPlan(n).execute_batched(t, batch, cf.FORWARD)
    got = t.cpu().numpy().reshape(n, batch).T
    _check(got, oracle.fft64(x.reshape(n, batch).T), n)


@pytest.mark.parametrize("n", [2, 4, 64, 1024, 8192, 2 ** 15, 2 ** 20])
def test_real_plan(n):
    """RealFftPlan: rfft unnormalised, irfft normalised (real_fft.hpp:41-92)."""
    x = oracle.lcg_float32(31337 + n, n)
    plan = cf.RealFftPlan(n)
    tin = torch.from_numpy(x).cuda()
    spec = torch.empty(n // 2 + 1, dtype=torch.complex64, device="cuda")
    plan.rfft(tin, spec)
    back = torch.empty(n, dtype=torch.float32, device="cuda")
    plan.irfft(spec, back)
    torch.cuda.synchronize()
    want = oracle.rfft64(x.astype(np.float64))
    _check(spec.cpu().numpy(), want, n, "rfft")
    got_back = back.cpu().numpy()
    assert np.max(np.abs(got_back - x)) <= 1e-5 * (1 + np.max(np.abs(x)))


@pytest.mark.parametrize("n,batch", [(1024, 4), (2 ** 20, 2)])
def test_r2c_c2r_batched(n, batch):
    x = oracle.lcg_float32(n + batch, n * batch).reshape(batch, n)
    r2c = cf.Plan([n], batch=batch, kind=cf.R2C)
    c2r = cf.Plan([n], batch=batch, kind=cf.C2R)
    tin = torch.from_numpy(x).cuda()
    spec = torch.empty(batch, n // 2 + 1, dtype=torch.complex64, device="cuda")
    r2c.execute(tin, spec, cf.FORWARD)
    back = torch.empty(batch, n, dtype=torch.float32, device="cuda")
    c2r.execute(spec, back, cf.INVERSE)  # unnormalised C2R: n * x
    torch.cuda.synchronize()
    _check(spec.cpu().numpy(), oracle.rfft64(x.astype(np.float64)), n, "r2c")
    assert np.max(np.abs(back.cpu().numpy() / n - x)) <= 1e-5 * (1 + np.max(np.abs(x)))


@pytest.mark.parametrize("dims", [(8, 16), (4, 6, 5), (16, 12), (64, 128), (32, 64, 16), (105, 48), (256, 256)])
def test_nd_plan(dims):
    total = int(np.prod(dims))
    x = oracle.lcg_complex64(0x9E3779B97F4A7C15 ^ total, total).reshape(dims)
    for inverse in (False, True):
        t = torch.from_numpy(x.copy()).cuda()
        cf.NdFftPlan(dims).execute(t, cf.INVERSE if inverse else cf.FORWARD)
        _check(t.cpu().numpy(), oracle.nd64(x, inverse), max(dims))


def test_against_reference_f32_outputs(golden):
    """The GPU agrees with the reference's own FP32 outputs at the reference's f32 class."""
    for n in (16, 105, 240, 1024, 4096):
        x = golden[f"c2c_{n}_in"]
        pow2 = (n & (n - 1)) == 0
        for inverse, key in ((False, "fwd"), (True, "inv")):
            t = torch.from_numpy(x.copy()).cuda()
            if pow2:
                cf.FftPlan(n).execute(t, cf.INVERSE if inverse else cf.FORWARD)
            else:
                cf.BluesteinPlan(n).execute(t, cf.INVERSE if inverse else cf.FORWARD)
            ref = golden[f"c2c_{n}_{key}"].astype(np.complex128)
            assert oracle.max_rel(t.cpu().numpy(), ref) < oracle.f32_class(n)
    for n in (64, 1024):
        plan = cf.RealFftPlan(n)
        spec = torch.empty(n // 2 + 1, dtype=torch.complex64, device="cuda")
        plan.rfft(torch.from_numpy(golden[f"rfft_{n}_in"]).cuda(), spec)
        assert oracle.max_rel(spec.cpu().numpy(), golden[f"rfft_{n}_out"].astype(np.complex128)) < 2e-4
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        plan.irfft(torch.from_numpy(golden[f"irfft_{n}_in"]).cuda(), out)
        want = golden[f"irfft_{n}_out"]
        assert np.max(np.abs(out.cpu().numpy() - want)) < 2e-4 * (1 + np.max(np.abs(want)))
    for dims in ((8, 16), (4, 6, 5), (16, 12)):
        tag = "x".join(str(d) for d in dims)
        for inverse, key in ((False, "fwd"), (True, "inv")):
            t = torch.from_numpy(golden[f"nd_{tag}_in"].copy()).cuda()
            cf.NdFftPlan(dims).execute(t, cf.INVERSE if inverse else cf.FORWARD)
            assert oracle.max_rel(t.cpu().numpy(), golden[f"nd_{tag}_{key}"].astype(np.complex128)) < 2e-4


def test_selfcheck_known_answers(golden):
    """The reference's own known-answer cases (src/fft_self_check.cpp:67-77) on the GPU, vs its outputs."""
    for idx in range(26):
        n, batch, inv, tiny = (int(v) for v in golden[f"selfcheck_{idx}_meta"])
        if tiny:
            continue  # subnormal results: the GPU flushes nothing here, but FP32 FMA contraction differs in ulps
        x = golden[f"selfcheck_{idx}_in"]
        t = torch.from_numpy(x.copy()).cuda()
        plan = cf.FftPlan(n)
        if batch == 0:
            plan.execute(t, inv)
        else:
            plan.execute_batched(t, batch, inv)
        ref = golden[f"selfcheck_{idx}_out"].astype(np.complex128)
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(t.cpu().numpy() - ref)) <= 2e-7 * scale + 1e-30


def test_device_self_check():
    cf.self_check()


def test_self_check_gates_first_plan_creation():
    """The known-answer check runs at the first plan creation on a device (the reference checks its kernel table
    before first use, src/fft_kernel_dispatch.cpp:48-52). With a mistake planted in the check's host answers (on the
    CPU), that creation and every later one on the device return CRDFFT_NUMERIC_SELFCHECK; once the device is
    re-checked with correct answers, plans are created again."""
    from crd_b200 import _lib

    L = _lib.lib()
    try:
        L.crdfft_debug_self_check_reset()
        L.crdfft_debug_self_check_mismatch(1)
        with pytest.raises(_lib.CrdFftError) as e:
            cf.Plan([1024], batch=2)
        assert e.value.status == _lib.NUMERIC_SELFCHECK
        L.crdfft_debug_self_check_mismatch(0)
        with pytest.raises(_lib.CrdFftError) as e:  # the verdict sticks for the device
            cf.Plan([64], batch=2)
        assert e.value.status == _lib.NUMERIC_SELFCHECK
    finally:
        L.crdfft_debug_self_check_mismatch(0)
        L.crdfft_debug_self_check_reset()
    x, got, plan = _c2c(1024, 2, False)
    _check(got, oracle.fft64(x), 1024)


def test_run_twice_bit_identical_and_in_place():
    """Fixed schedules, no atomics: two runs give the same bits; in-place equals out-of-place."""
    for n, batch in ((1024, 64), (65536, 3), (107520, 2)):
        x = oracle.lcg_complex64(n, n * batch).reshape(batch, n)
        t = torch.from_numpy(x).cuda()
        plan = cf.Plan([n], batch=batch)
        a = torch.empty_like(t)
        b = torch.empty_like(t)
        plan.execute(t, a)
        plan.execute(t, b)
        c = t.clone()
        plan.execute(c, c)
        torch.cuda.synchronize()
        assert torch.equal(a.view(torch.float32), b.view(torch.float32))
        assert torch.equal(a.view(torch.float32), c.view(torch.float32))


def test_guard_words_kept():
    """NaN canaries just before and after the output survive (test_fft_kernels.cpp:65-135 guard words)."""
    for n, batch in ((1024, 7), (65536, 2), (1000, 3)):
        x = oracle.lcg_complex64(n ^ 5, n * batch)
        buf = torch.full((n * batch + 64,), complex(float("nan"), float("nan")), dtype=torch.complex64,
                         device="cuda")
        out = buf[32:32 + n * batch]
        plan = cf.Plan([n], batch=batch)
        plan.execute(torch.from_numpy(x).cuda(), out)
        torch.cuda.synchronize()
        host = buf.cpu().numpy()
        assert np.all(np.isnan(host[:32])) and np.all(np.isnan(host[32 + n * batch:]))
        assert np.all(np.isfinite(host[32:32 + n * batch]))


def test_special_values_propagate():
    """Inf/NaN inputs propagate into the outputs that depend on them instead of vanishing (the reference's
    special-value cases, test_fft_kernels.cpp:345-420)."""
    n = 1024
    x = np.zeros(n, dtype=np.complex64)
    x[3] = np.inf
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    cf.Plan([n]).execute(t, o)
    got = o.cpu().numpy()
    assert not np.all(np.isfinite(got))


def test_errors_are_status_codes():
    with pytest.raises(cf.CrdFftError) as e:
        cf.Plan([0])
    assert e.value.status == 1
    with pytest.raises(cf.CrdFftError) as e:
        cf.Plan([16], batch=0)
    assert e.value.status == 1
    from crd_b200.hesap import fail_alloc_after

    fail_alloc_after(1)
    try:
        with pytest.raises(cf.CrdFftError) as e:
            cf.Plan([1024])
        assert e.value.status == 3
    finally:
        fail_alloc_after(0)
    p = cf.Plan([1024])  # allocation works again
    assert p.info()["algorithm"] == "single-pass"


def test_bounded_wait_reports_timeout(monkeypatch):
    """A pipelined kernel whose barrier wait can never complete (the test hook points it at a barrier that nothing
    completes) gives up after its iteration limit, reports CRDFFT_DEVICE_TIMEOUT, and leaves the context usable."""
    from crd_b200.hesap import device_status, stall_waits

    n, batch = 256, 256  # a length with a pipelined instance
    x = torch.from_numpy(oracle.lcg_complex64(3, n * batch)).cuda()
    y = torch.empty_like(x)
    monkeypatch.setenv("CRDFFT_PIPELINE", "1")
    stall_waits(True)
    try:
        bad = cf.Plan([n], batch=batch)
    finally:
        stall_waits(False)
        monkeypatch.delenv("CRDFFT_PIPELINE")
    bad.execute(x, y)
    with pytest.raises(cf.CrdFftError) as e:
        device_status(bad)
    assert e.value.status == 5
    device_status(bad)  # the word was cleared
    good = cf.Plan([n], batch=batch)
    good.execute(x, y)
    device_status(good)
    want = oracle.fft64(x.cpu().numpy().reshape(batch, n))
    assert oracle.rel_l2(y.cpu().numpy().reshape(batch, n), want) <= REL_L2


def test_pipelined_and_classic_agree_bitwise(monkeypatch):
    """The pipelined kernel and the classic kernel run the same butterflies in the same order: same bits."""
    for n, batch in ((256, 33), (4096, 9), (65536, 2)):
        x = torch.from_numpy(oracle.lcg_complex64(n + 1, n * batch)).cuda()
        a = torch.empty_like(x)
        b = torch.empty_like(x)
        cf.Plan([n], batch=batch).execute(x, a)
        monkeypatch.setenv("CRDFFT_PIPELINE", "1")
        cf.Plan([n], batch=batch).execute(x, b)
        monkeypatch.delenv("CRDFFT_PIPELINE")
        torch.cuda.synchronize()
        assert torch.equal(a.view(torch.float32), b.view(torch.float32)), n


def test_measuring_planner_and_wisdom():
    """The measuring planner times each pass's candidates, remembers the fastest as wisdom, and a plan built from
    exported-then-imported wisdom makes the same choice and the same bits."""
    from crd_b200 import hesap as H

    n, batch = 4096, 256
    x = torch.from_numpy(oracle.lcg_complex64(9, n * batch)).cuda()
    a = torch.empty_like(x)
    b = torch.empty_like(x)
    H.wisdom_forget()
    H.set_planner("measure")
    try:
        cf.Plan([n], batch=batch).execute(x, a)
    finally:
        H.set_planner("estimate")
    log = H.planner_log()
    assert "best" in log and "n4096" in log
    text = H.wisdom_export()
    assert text.startswith("crdfft-wisdom 1") and "n4096" in text
    H.wisdom_forget()
    H.wisdom_import(text)
    cf.Plan([n], batch=batch).execute(x, b)
    torch.cuda.synchronize()
    assert torch.equal(a.view(torch.float32), b.view(torch.float32))
    with pytest.raises(cf.CrdFftError):
        H.wisdom_import("not wisdom")
    H.wisdom_forget()
    want = oracle.fft64(x.cpu().numpy().reshape(batch, n))
    assert oracle.rel_l2(a.cpu().numpy().reshape(batch, n), want) <= REL_L2


def _uneven_case(count, seed):
    from crd_b200.workloads import uneven_sizes

    sizes = uneven_sizes(count, seed=seed)
    plan = cf.UnevenPlan(sizes)
    x = oracle.gauss_complex64(seed, plan.total)
    return sizes, plan, x


@pytest.mark.parametrize("inverse", [False, True])
def test_uneven_batch(inverse):
    """Config-3 style batch: 7-smooth sizes log-uniform in [16, 65536], Gaussian inputs, one persistent launch;
    every transform against the FP64 oracle."""
    sizes, plan, x = _uneven_case(240, 0x5EED0003 + int(inverse))
    assert any(s > 8192 for s in sizes) and any(s <= 8192 for s in sizes)
    tin = torch.from_numpy(x).cuda()
    tout = torch.full_like(tin, complex(float("nan"), float("nan")))
    plan.execute(tin, tout, cf.INVERSE if inverse else cf.FORWARD)
    plan.execute(tin, tout, cf.INVERSE if inverse else cf.FORWARD)  # the cached graph, again
    torch.cuda.synchronize()
    from crd_b200.hesap import device_status

    device_status(plan)
    got = tout.cpu().numpy()
    by_size = {}
    for t, (n, off) in enumerate(zip(sizes, plan.offsets)):
        by_size.setdefault(n, []).append(off)
    for n, offs in by_size.items():
        xs = np.stack([x[o:o + n] for o in offs])
        gs = np.stack([got[o:o + n] for o in offs])
        _check(gs, oracle.fft64(xs, inverse), n, f"uneven n={n}")


@pytest.mark.parametrize("variant", [0, 1])
def test_uneven_stage_variants(variant):
    """The uneven kernel runs power-of-two line lengths (the small transforms and the halves of long ones) on their
    compile-time stages or on the run-time stages; both against the FP64 oracle, with every power of two from 16 to
    65536 in the batch."""
    from crd_b200 import _lib

    sizes = [1 << k for k in range(4, 17)] * 3 + [105, 3000, 45927]
    L = _lib.lib()
    L.crdfft_debug_uneven_variant(variant)
    try:
        plan = cf.UnevenPlan(sizes)
    finally:
        L.crdfft_debug_uneven_variant(-1)
    x = oracle.gauss_complex64(0x5EED0033 + variant, plan.total)
    tin = torch.from_numpy(x).cuda()
    tout = torch.empty_like(tin)
    plan.execute(tin, tout, cf.FORWARD)
    torch.cuda.synchronize()
    got = tout.cpu().numpy()
    for n, o in zip(sizes, plan.offsets):
        _check(got[o:o + n], oracle.fft64(x[o:o + n]), n, f"uneven variant {variant} n={n}")


def test_uneven_dependency_wait_times_out():
    """A ROW item waiting for a COL item that never comes (the test hook adds one to its count) gives up after its
    bounded wait, the plan reports CRDFFT_DEVICE_TIMEOUT, and the context stays usable."""
    from crd_b200.hesap import device_status, stall_waits

    sizes = [65536, 1024, 105]
    stall_waits(True)
    try:
        bad = cf.UnevenPlan(sizes)
    finally:
        stall_waits(False)
    x = torch.from_numpy(oracle.gauss_complex64(5, bad.total)).cuda()
    y = torch.empty_like(x)
    bad.execute(x, y)
    with pytest.raises(cf.CrdFftError) as e:
        device_status(bad)
    assert e.value.status == 5
    good = cf.UnevenPlan(sizes)
    good.execute(x, y)
    device_status(good)
    xs = x.cpu().numpy()
    ys = y.cpu().numpy()
    for n, o in zip(sizes, good.offsets):
        _check(ys[o:o + n], oracle.fft64(xs[o:o + n]), n)


@pytest.mark.parametrize("dims", [(24, 40), (375, 280), (64, 4096)])
def test_nd_padded_batch_distances(dims):
    """2-D batches whose members sit a padded distance apart (idist, odist above the transform size): each member
    transforms on its own, and the padding of the output is left as it was."""
    total = int(np.prod(dims))
    batch, idist, odist = 3, total + 8, total + 12
    x = oracle.lcg_complex64(0xADD ^ total, batch * idist)
    for inverse in (False, True):
        t = torch.from_numpy(x.copy()).cuda()
        o = torch.full((batch * odist,), 7 + 7j, dtype=torch.complex64, device="cuda")
        plan = cf.Plan(list(dims), batch=batch, idist=idist, odist=odist, norm=cf.NORM_INVERSE)
        plan.execute(t, o, cf.INVERSE if inverse else cf.FORWARD)
        torch.cuda.synchronize()
        got = o.cpu().numpy()
        for b in range(batch):
            xb = x[b * idist:b * idist + total].reshape(dims)
            _check(got[b * odist:b * odist + total].reshape(dims), oracle.nd64(xb, inverse), max(dims))
            assert np.all(got[b * odist + total:(b + 1) * odist] == 7 + 7j)


@pytest.mark.parametrize("inverse", [False, True])
def test_l2_sized_waves_on_two_streams(inverse):
    """Batches larger than two L2-sized waves run the four-step waves alternately on the plan's two internal streams
    (two workspace slots); every transform comes out right and the caller's stream sees all of it."""
    n, batch = 1 << 17, 64
    x, got, plan = _c2c(n, batch, inverse, seed=0x12AB)
    assert plan.info()["algorithm"] == "four-step"
    for t in (0, 23, 24, 47, 48, 63):  # across wave and slot boundaries
        _check(got[t], oracle.fft64(x[t], inverse), n)


def test_l2_waves_then_recombine_real():
    """R2C: the half-length four-step waves on the internal streams, then the recombination on the caller's stream
    (which must wait for both)."""
    n, batch = 1 << 18, 100
    x = oracle.lcg_float32(0x12AC, n * batch).reshape(batch, n)
    t = torch.from_numpy(x).cuda()
    spec = torch.empty(batch, n // 2 + 1, dtype=torch.complex64, device="cuda")
    cf.Plan([n], batch=batch, kind=cf.R2C).execute(t, spec, cf.FORWARD)
    back = torch.empty(batch, n, dtype=torch.float32, device="cuda")
    cf.Plan([n], batch=batch, kind=cf.C2R, norm=cf.NORM_INVERSE).execute(spec, back, cf.INVERSE)
    torch.cuda.synchronize()
    s = spec.cpu().numpy()
    for r in (0, 49, 99):
        assert oracle.rel_l2(s[r], np.fft.rfft(x[r].astype(np.float64))) <= 1e-6
    assert oracle.rel_l2(back.cpu().numpy(), x.astype(np.float64)) <= 1e-6


@pytest.mark.parametrize("dims,batch", [((4096, 256), 2), ((2048, 96), 3), ((6144, 64), 1)])
def test_nd_long_columns_split(dims, batch):
    """2-D batches with long columns: the column FFT runs as two strided passes of short lines (four-step twiddle
    by column index), the rows pass writing the workspace; forward and normalised inverse."""
    total = int(np.prod(dims))
    x = oracle.lcg_complex64(0x5C01 ^ total, batch * total).reshape((batch,) + dims)
    plan = cf.Plan(list(dims), batch=batch, norm=cf.NORM_INVERSE)
    assert plan.info()["algorithm"] == "nd-axes-split-columns"
    for inverse in (False, True):
        t = torch.from_numpy(x.copy()).cuda()
        o = torch.empty_like(t)
        plan.execute(t, o, cf.INVERSE if inverse else cf.FORWARD)
        torch.cuda.synchronize()
        got = o.cpu().numpy()
        for b in range(batch):
            _check(got[b], oracle.nd64(x[b], inverse), max(dims))
