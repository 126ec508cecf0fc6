"""GPU parity at the benchmark configurations' full shapes, through the C ABI, against the FP64 oracle.

The small-shape parity tests (test_gpu_parity.py) pin every plan class; these run the exact shapes the benchmark
measures, so that every throughput figure rests on a checked result at that shape:

* config 1: C2C forward N = 1024, batch 4096, contiguous: every transform against the oracle.
* config 2: C2C forward at N = 4096, 65536, 2^20 and 107520, each batch filling 2 GiB of input, and R2C then C2R at
  N = 2^20, batch 512 (the reference's irfft convention): a seeded sample of 64 transforms per op (plus the first and
  the last) against the oracle, and the whole batch through a size-independent property, the round trip forward then
  normalised inverse.
* config 3: the 20,000-transform uneven batch (7-smooth sizes log-uniform in [16, 65536], Gaussian inputs): a seeded
  sample of 512 transforms plus the first and the last against the oracle.
* config 4: 2-D 4096 x 4096 and 3-D 512^3, uniform[-1,1) with exactly 1 % of the entries (a seeded sample without
  replacement) scaled by 1e4, in the precision forms: FP32, split-BF16 (three terms) and split-FP16 hi+lo (per-line
  scale) at rel-L2 <= 1e-6 against the FP64 N-D oracle; FP16 with a per-line scale (one term, 11 bits) is reported
  and held to 1e-3, split-BF16 hi+lo (two terms, about 16 bits) reported and held to 2e-5.

Inputs are the reference tests' LCG (uniform[-1,1), test_fft.cpp:31-44) or its Box-Muller Gaussian, one stream per
op seeded from the configuration number. Tolerances: rel-L2 <= 1e-6 against FP64, and the reference's f32 class for
max|a - b| / (1 + max|b|) (2e-4 below 2^19, 1e-3 from 2^19; tests/numerics/hesap-fft/test_fft_kernels.cpp:138-163).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle
from crd_b200.workloads import uneven_sizes

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6
FP16_REPORT_BOUND = 1e-3
HILO_REPORT_BOUND = 2e-5  # bf16 hi+lo carries about 16 bits of the data: reported, not a 1e-6 form
SAMPLE = 64
TWO_GIB = 2 << 30


def _sample(batch: int, seed: int, count: int = SAMPLE) -> np.ndarray:
    """A seeded sample of transform indices, the first and the last included."""
    rng = np.random.default_rng(seed)
    pick = rng.choice(batch, size=min(batch, count), replace=False)
    return np.unique(np.concatenate([pick, [0, batch - 1]]))


def _check(got, want, n, what):
    rl2 = oracle.rel_l2(got, want)
    mr = oracle.max_rel(got, want)
    assert rl2 <= REL_L2, f"{what}: rel-L2 {rl2:.3e} > {REL_L2}"
    assert mr <= oracle.f32_class(n), f"{what}: max-rel {mr:.3e}"
    return rl2


def _round_trip_rel_l2(x: torch.Tensor, back: torch.Tensor) -> float:
    """rel-L2 of back against x over the whole batch, in FP64 on the device."""
    d = (back.view(torch.float32).double() - x.view(torch.float32).double()).norm()
    return float(d / x.view(torch.float32).double().norm())


def test_config1_n1024_batch4096_every_transform():
    n, b = 1024, 4096
    x = oracle.lcg_complex64(oracle.config_seed(1), n * b).reshape(b, n)
    t = torch.from_numpy(x).cuda()
    out = torch.empty_like(t)
    plan = cf.Plan([n], batch=b)
    assert plan.info()["algorithm"] == "single-pass"
    plan.execute(t, out, cf.FORWARD)
    torch.cuda.synchronize()
    _check(out.cpu().numpy(), oracle.fft64(x), n, "config 1, all 4096 transforms")


@pytest.mark.parametrize("n", [4096, 65536, 1 << 20, 107520])
def test_config2_c2c_two_gib(n):
    b = TWO_GIB // (8 * n)
    x = torch.from_numpy(oracle.lcg_complex64(oracle.config_seed(2, n), n * b)).cuda()
    out = torch.empty_like(x)
    plan = cf.Plan([n], batch=b)
    plan.execute(x, out, cf.FORWARD)
    torch.cuda.synchronize()
    idx = _sample(b, n)
    xs = x.view(b, n)[idx].cpu().numpy()
    got = out.view(b, n)[idx].cpu().numpy()
    _check(got, oracle.fft64(xs), n, f"config 2, n={n} batch={b} ({plan.info()['algorithm']}), {len(idx)} sampled")
    # the whole batch: forward then inverse scaled by 1/n returns the input
    inv = cf.Plan([n], batch=b, norm=cf.NORM_INVERSE)
    back = torch.empty_like(x)
    inv.execute(out, back, cf.INVERSE)
    torch.cuda.synchronize()
    rt = _round_trip_rel_l2(x, back)
    assert rt <= 2 * REL_L2, f"config 2, n={n}: round trip rel-L2 {rt:.3e}"


def test_config2_r2c_c2r_two_gib():
    n, b = 1 << 20, 512
    h = n // 2 + 1
    x = torch.from_numpy(oracle.lcg_float32(oracle.config_seed(2, 7), n * b)).cuda()
    spec = torch.empty(b * h, dtype=torch.complex64, device="cuda")
    r2c = cf.Plan([n], batch=b, kind=cf.R2C)
    r2c.execute(x, spec, cf.FORWARD)
    torch.cuda.synchronize()
    idx = _sample(b, 0x2C)
    xs = x.view(b, n)[idx].cpu().numpy()
    got = spec.view(b, h)[idx].cpu().numpy()
    _check(got, oracle.rfft64(xs), n, f"config 2 R2C ({r2c.info()['algorithm']}), {len(idx)} sampled")
    # C2R of the computed spectrum, normalised (RealFftPlan::irfft), against the reference's irfft restated in FP64
    back = torch.empty_like(x)
    c2r = cf.Plan([n], batch=b, kind=cf.C2R, norm=cf.NORM_INVERSE)
    c2r.execute(spec, back, cf.INVERSE)
    torch.cuda.synchronize()
    want = oracle.irfft64(spec.view(b, h)[idx].cpu().numpy(), n)
    _check(back.view(b, n)[idx].cpu().numpy(), want, n, f"config 2 C2R ({c2r.info()['algorithm']})")
    # the whole batch: R2C then normalised C2R returns the input
    d = (back.double() - x.double()).norm() / x.double().norm()
    assert float(d) <= 2 * REL_L2, f"config 2 R2C/C2R round trip rel-L2 {float(d):.3e}"


def test_config3_uneven_20000():
    sizes = uneven_sizes(20000, seed=0x5EED0003)
    plan = cf.UnevenPlan(sizes)
    x = oracle.gauss_complex64(oracle.config_seed(3), plan.total)
    t = torch.from_numpy(x).cuda()
    out = torch.empty_like(t)
    plan.execute(t, out, cf.FORWARD)
    torch.cuda.synchronize()
    y = out.cpu().numpy()
    worst = 0.0
    for i in _sample(len(sizes), 0x3C, 512):
        n, o = sizes[i], plan.offsets[i]
        worst = max(worst, _check(y[o:o + n], oracle.fft64(x[o:o + n]), n, f"config 3, transform {i} (n={n})"))
    assert worst <= REL_L2


_ND_CACHE: dict = {}


def _nd_input(dims):
    """uniform[-1,1) with exactly 1 % of the entries, a seeded sample without replacement, scaled by 1e4; the FP64
    answer is computed once per shape."""
    key = tuple(dims)
    if key not in _ND_CACHE:
        total = int(np.prod(dims))
        x = oracle.lcg_complex64(oracle.config_seed(4, total), total)
        idx = np.random.default_rng(0x5EED0004).choice(total, size=total // 100, replace=False)
        x[idx] *= np.float32(1e4)
        x = x.reshape(dims)
        _ND_CACHE.clear()
        _ND_CACHE[key] = (x, oracle.nd64_axes(x))
    return _ND_CACHE[key]


@pytest.mark.parametrize("form,prec", [("fp32", 0), ("split-bf16", 1), ("fp16-scaled", 2), ("split-bf16-hilo", 3),
                                       ("split-fp16-hilo", 4)])
@pytest.mark.parametrize("dims", [(4096, 4096), (512, 512, 512)])
def test_config4_nd_outliers(dims, form, prec):
    x, want = _nd_input(dims)
    t = torch.from_numpy(x.reshape(-1)).cuda()
    out = torch.empty_like(t)
    plan = cf.Plan(list(dims), batch=1, precision=prec)
    plan.execute(t, out, cf.FORWARD)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(dims)
    rl2 = oracle.rel_l2(got, want)
    print(f"config 4 {dims} {form} ({plan.info()['algorithm']}): rel-L2 vs FP64 {rl2:.3e}")
    if form == "fp16-scaled":
        assert rl2 <= FP16_REPORT_BOUND, f"{dims} {form}: rel-L2 {rl2:.3e}"
    elif form == "split-bf16-hilo":
        assert rl2 <= HILO_REPORT_BOUND, f"{dims} {form}: rel-L2 {rl2:.3e}"
    else:
        _check(got, want, max(dims), f"config 4 {dims} {form}")
