"""The fused real-data line kernels (crd_b200/csrc/real_line.cu) through the C ABI, against the FP64 oracle:

* R2C and C2R plans whose half length runs as one pass take one launch ("real-fused"): every schedule class
  (compile-time and run-time, odd half lengths), padded distances, in place, both normalisations.
* The real fused convolution (ConvPlan(real=True)): y = IRFFT(RFFT(x) * H) * scale, 1-D in one launch and 2-D as
  R2C rows, a half-width column convolution and C2R rows; rel-L2 <= 1e-6.

C2R follows the reference's irfft (real_fft.hpp:65-92), restated by the oracle (oracle.irfft64): Y[0] and Y[n/2] enter
the pair recombination with their imaginary parts, where numpy's irfft drops them; the test spectra are not Hermitian
at 0 and n/2, so they check that convention too."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6

# half lengths: compile-time schedules (16x4, 16x8, 16x16, 16x8x4, 32x32, 16x16x8, 16x16x16, 32x16x16) and
# run-time ones (1, 2, 3, 5, 105, 1000, 3000, 6144)
FUSED_N = [4, 6, 10, 128, 210, 256, 512, 1024, 2000, 2048, 4096, 6000, 8192, 12288, 16384]


def _spec64(x):
    return np.fft.rfft(np.asarray(x, dtype=np.float64), axis=-1)


@pytest.mark.parametrize("n", FUSED_N)
def test_r2c_c2r_fused(n):
    batch = 7
    x = oracle.lcg_float32(0xF00 ^ n, batch * n).reshape(batch, n)
    r2c = cf.Plan([n], batch=batch, kind=cf.R2C)
    c2r = cf.Plan([n], batch=batch, kind=cf.C2R)
    assert r2c.info()["algorithm"] == "real-fused" and c2r.info()["algorithm"] == "real-fused"
    spec = torch.empty(batch, n // 2 + 1, dtype=torch.complex64, device="cuda")
    r2c.execute(torch.from_numpy(x).cuda(), spec, cf.FORWARD)
    # a spectrum that is not Hermitian at 0 and n/2
    y = oracle.lcg_complex64(0xF01 ^ n, batch * (n // 2 + 1)).reshape(batch, n // 2 + 1)
    back = torch.empty(batch, n, dtype=torch.float32, device="cuda")
    c2r.execute(torch.from_numpy(y).cuda(), back, cf.INVERSE)
    torch.cuda.synchronize()
    got = spec.cpu().numpy()
    want = _spec64(x)
    assert oracle.rel_l2(got, want) <= REL_L2
    assert oracle.max_rel(got, want) <= oracle.f32_class(n)
    want_back = oracle.irfft64(y, n) * n  # unnormalised C2R, the reference's convention
    assert oracle.rel_l2(back.cpu().numpy(), want_back) <= REL_L2


@pytest.mark.parametrize("n", [6, 1024, 2000])
def test_normalised_irfft_round_trip(n):
    batch = 5
    x = oracle.lcg_float32(0xF02 ^ n, batch * n).reshape(batch, n)
    r2c = cf.Plan([n], batch=batch, kind=cf.R2C)
    c2r = cf.Plan([n], batch=batch, kind=cf.C2R, norm=cf.NORM_INVERSE)
    spec = torch.empty(batch, n // 2 + 1, dtype=torch.complex64, device="cuda")
    back = torch.empty(batch, n, dtype=torch.float32, device="cuda")
    r2c.execute(torch.from_numpy(x).cuda(), spec, cf.FORWARD)
    c2r.execute(spec, back, cf.INVERSE)
    torch.cuda.synchronize()
    assert oracle.rel_l2(back.cpu().numpy(), x.astype(np.float64)) <= REL_L2


@pytest.mark.parametrize("n", [256, 1000])
def test_fused_padded_distances_leave_gaps_alone(n):
    batch, h = 4, n // 2 + 1
    idist, odist = n + 6, h + 3
    x = oracle.lcg_float32(0xF03 ^ n, batch * idist)
    out = torch.full((batch * odist,), 5 + 5j, dtype=torch.complex64, device="cuda")
    plan = cf.Plan([n], batch=batch, kind=cf.R2C, idist=idist, odist=odist)
    assert plan.info()["algorithm"] == "real-fused"
    plan.execute(torch.from_numpy(x).cuda(), out, cf.FORWARD)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(batch, odist)
    want = _spec64(x.reshape(batch, idist)[:, :n])
    assert oracle.rel_l2(got[:, :h], want) <= REL_L2
    assert np.all(got[:, h:] == 5 + 5j)
    # C2R with padded distances on both sides
    y = oracle.lcg_complex64(0xF04 ^ n, batch * odist)
    back = torch.full((batch * idist,), 9.0, dtype=torch.float32, device="cuda")
    cf.Plan([n], batch=batch, kind=cf.C2R, idist=odist, odist=idist).execute(torch.from_numpy(y).cuda(), back,
                                                                              cf.INVERSE)
    torch.cuda.synchronize()
    gb = back.cpu().numpy().reshape(batch, idist)
    want_b = oracle.irfft64(y.reshape(batch, odist)[:, :h], n) * n
    assert oracle.rel_l2(gb[:, :n], want_b) <= REL_L2
    assert np.all(gb[:, n:] == 9.0)


def test_fused_r2c_in_place():
    """In place with the padded layout (each real row 2 (n/2 + 1) floats): a CTA reads its rows before writing."""
    n, batch = 4096, 9
    h = n // 2 + 1
    x = oracle.lcg_float32(0xF05, batch * n).reshape(batch, n)
    buf = torch.zeros(batch, 2 * h, dtype=torch.float32, device="cuda")
    buf[:, :n] = torch.from_numpy(x).cuda()
    plan = cf.Plan([n], batch=batch, kind=cf.R2C, idist=2 * h, odist=h)
    plan.execute(buf, buf.view(torch.complex64), cf.FORWARD)
    torch.cuda.synchronize()
    got = buf.view(torch.complex64).cpu().numpy()
    assert oracle.rel_l2(got, _spec64(x)) <= REL_L2


def test_fused_matches_two_launch_path(monkeypatch):
    """The fused kernel and the half FFT followed by the recombination kernel agree to FP32 rounding."""
    n, batch = 2048, 33
    x = torch.from_numpy(oracle.lcg_float32(0xF06, batch * n).reshape(batch, n)).cuda()
    a = torch.empty(batch, n // 2 + 1, dtype=torch.complex64, device="cuda")
    b = torch.empty_like(a)
    cf.Plan([n], batch=batch, kind=cf.R2C).execute(x, a, cf.FORWARD)
    monkeypatch.setenv("CRDFFT_NO_FUSED_REAL", "1")
    p2 = cf.Plan([n], batch=batch, kind=cf.R2C)
    assert p2.info()["algorithm"] == "real+single-pass"
    p2.execute(x, b, cf.FORWARD)
    torch.cuda.synchronize()
    assert oracle.rel_l2(a.cpu().numpy(), b.cpu().numpy().astype(np.complex128)) <= 5e-7


# ---- real fused convolution ------------------------------------------------------------------------------------


def _irfft_ref(yh, n):
    """The reference's normalised irfft over the last axis (oracle restatement), any leading shape."""
    return oracle.irfft64(np.ascontiguousarray(yh), n)


def _rconv_want(x, hs, axes_shape, scale):
    if len(axes_shape) == 1:
        y = _irfft_ref(np.fft.rfft(x.astype(np.float64), axis=-1) * hs, axes_shape[0])
    else:
        spec = np.fft.rfft2(x.astype(np.float64), axes=(-2, -1)) * hs
        y = _irfft_ref(np.fft.ifft(spec, axis=-2), axes_shape[1])
    return y * np.prod(axes_shape) * scale


@pytest.mark.parametrize("n", [4, 16, 64, 210, 512, 1000, 2048, 4096, 8192, 16384])
@pytest.mark.parametrize("per_signal", [False, True])
def test_real_conv_1d(n, per_signal):
    batch = 11
    h = n // 2 + 1
    x = oracle.lcg_float32(0xF10 ^ n, batch * n).reshape(batch, n)
    hs = oracle.lcg_complex64(0xF11 ^ n, (batch if per_signal else 1) * h).reshape(-1, h)
    plan = cf.ConvPlan([n], batch=batch, per_signal_filter=per_signal, real=True)
    assert plan.info()["algorithm"] == "fused-real-conv"
    out = torch.empty(batch, n, dtype=torch.float32, device="cuda")
    plan.execute(torch.from_numpy(x).cuda(), torch.from_numpy(hs).cuda(), out)
    torch.cuda.synchronize()
    want = _rconv_want(x, hs.astype(np.complex128), (n,), 1.0 / n)
    rl2 = oracle.rel_l2(out.cpu().numpy(), want)
    assert rl2 <= REL_L2, f"n={n}: rel-L2 {rl2:.2e}"


def test_real_conv_is_circular_convolution_in_place():
    n, batch = 1024, 6
    x = oracle.lcg_float32(0xF12, batch * n).reshape(batch, n)
    taps = np.array([0.5, 0.25, -0.125, 0.0625, 1.0])
    k = np.zeros(n)
    k[:5] = taps
    H = np.fft.rfft(k).astype(np.complex64)
    t = torch.from_numpy(x.copy()).cuda()
    cf.ConvPlan([n], batch=batch, real=True).execute(t, torch.from_numpy(H).cuda(), t)
    torch.cuda.synchronize()
    want = np.stack([sum(taps[j] * np.roll(x[b].astype(np.float64), j) for j in range(5)) for b in range(batch)])
    assert oracle.rel_l2(t.cpu().numpy(), want) <= REL_L2


@pytest.mark.parametrize("dims", [(64, 64), (256, 1024), (105, 96), (1024, 256), (512, 2000)])
@pytest.mark.parametrize("per_signal", [False, True])
def test_real_conv_2d(dims, per_signal):
    batch = 3
    rows, cols = dims
    hw = cols // 2 + 1
    x = oracle.lcg_float32(0xF13 ^ rows, batch * rows * cols).reshape(batch, rows, cols)
    hs = oracle.lcg_complex64(0xF14 ^ cols, (batch if per_signal else 1) * rows * hw).reshape(-1, rows, hw)
    plan = cf.ConvPlan(list(dims), batch=batch, per_signal_filter=per_signal, scale=0.25, real=True)
    assert plan.info()["algorithm"] == "fused-real-conv-2d"
    out = torch.empty(batch, rows, cols, dtype=torch.float32, device="cuda")
    plan.execute(torch.from_numpy(x).cuda(), torch.from_numpy(hs).cuda(), out)
    torch.cuda.synchronize()
    want = _rconv_want(x, hs.astype(np.complex128), dims, 0.25)
    rl2 = oracle.rel_l2(out.cpu().numpy(), want)
    assert rl2 <= REL_L2, f"{dims}: rel-L2 {rl2:.2e}"


def test_real_conv_plan_errors():
    with pytest.raises(cf.CrdFftError):
        cf.ConvPlan([1001], real=True)        # odd length
    with pytest.raises(cf.CrdFftError):
        cf.ConvPlan([32768 * 2], real=True)   # half length beyond one CTA's lines
    with pytest.raises(cf.CrdFftError):
        cf.ConvPlan([8, 8, 8], real=True)     # rank 3
    with pytest.raises(cf.CrdFftError):
        cf.Plan([64, 63], kind=cf.R2C)       # odd real axis


# ---- 2-D and 3-D real transforms -------------------------------------------------------------------------------


@pytest.mark.parametrize("dims", [(64, 64), (16, 1024), (105, 96), (256, 2000), (8, 12, 16), (32, 16, 256), (4, 1, 6)])
def test_nd_real_plans(dims):
    batch = 3
    total = int(np.prod(dims))
    half = tuple(dims[:-1]) + (dims[-1] // 2 + 1,)
    x = oracle.lcg_float32(0xF20 ^ total, batch * total).reshape((batch,) + tuple(dims))
    r2c = cf.Plan(list(dims), batch=batch, kind=cf.R2C)
    c2r = cf.Plan(list(dims), batch=batch, kind=cf.C2R, norm=cf.NORM_INVERSE)
    assert r2c.info()["algorithm"] == "nd-real"
    spec = torch.empty((batch,) + half, dtype=torch.complex64, device="cuda")
    r2c.execute(torch.from_numpy(x).cuda(), spec, cf.FORWARD)
    axes = tuple(range(1, len(dims) + 1))
    y = oracle.lcg_complex64(0xF21 ^ total, batch * int(np.prod(half))).reshape((batch,) + half)
    ty = torch.from_numpy(y).cuda()
    back = torch.empty((batch,) + tuple(dims), dtype=torch.float32, device="cuda")
    c2r.execute(ty, back, cf.INVERSE)
    torch.cuda.synchronize()
    want = np.fft.rfftn(x.astype(np.float64), axes=axes)
    assert oracle.rel_l2(spec.cpu().numpy(), want) <= REL_L2
    # normalised: the complex axes inverted (FP64), then the reference's irfft along the last axis
    yc = y.astype(np.complex128)
    for ax in range(1, len(dims)):
        yc = np.fft.ifft(yc, axis=ax)
    want_back = _irfft_ref(yc, dims[-1])
    assert oracle.rel_l2(back.cpu().numpy(), want_back) <= REL_L2
    assert np.array_equal(ty.cpu().numpy(), y)  # C2R leaves its input alone


def test_nd_real_round_trip_unnormalised():
    dims, batch = (128, 256), 2
    x = oracle.lcg_float32(0xF22, batch * dims[0] * dims[1]).reshape(batch, *dims)
    spec = torch.empty(batch, dims[0], dims[1] // 2 + 1, dtype=torch.complex64, device="cuda")
    back = torch.empty(batch, *dims, dtype=torch.float32, device="cuda")
    cf.Plan(list(dims), batch=batch, kind=cf.R2C).execute(torch.from_numpy(x).cuda(), spec, cf.FORWARD)
    cf.Plan(list(dims), batch=batch, kind=cf.C2R).execute(spec, back, cf.INVERSE)
    torch.cuda.synchronize()
    assert oracle.rel_l2(back.cpu().numpy() / (dims[0] * dims[1]), x.astype(np.float64)) <= REL_L2


def test_nd_real_host_execute_matches_device():
    dims, batch = (64, 128), 16
    x = oracle.lcg_float32(0xF23, batch * dims[0] * dims[1]).reshape(batch, *dims)
    plan = cf.Plan(list(dims), batch=batch, kind=cf.R2C)
    dev = torch.empty(batch, dims[0], dims[1] // 2 + 1, dtype=torch.complex64, device="cuda")
    plan.execute(torch.from_numpy(x).cuda(), dev, cf.FORWARD)
    hin = torch.from_numpy(x.copy()).pin_memory()
    hout = torch.empty(dev.shape, dtype=torch.complex64).pin_memory()
    plan.execute_host(hin, hout, cf.FORWARD)
    torch.cuda.synchronize()
    assert np.array_equal(hout.numpy(), dev.cpu().numpy())


# ---- R2C of long transforms: the half-length four-step's row pass fused with the recombination -----------------


@pytest.mark.parametrize("n,batch,pad", [(1 << 20, 3, 0), (1 << 21, 2, 4), (1 << 20, 5, 3)])
def test_long_r2c_fused_row_pass(n, batch, pad, monkeypatch):
    h = n // 2 + 1
    odist = h + pad
    x = torch.from_numpy(oracle.lcg_float32(0xF30 ^ n ^ pad, batch * n)).cuda()
    a = torch.full((batch * odist,), 3 + 3j, dtype=torch.complex64, device="cuda")
    b = torch.full_like(a, 3 + 3j)
    plan = cf.Plan([n], batch=batch, kind=cf.R2C, odist=odist)
    assert plan.info()["algorithm"] == "real+four-step-fused"
    plan.execute(x, a, cf.FORWARD)
    monkeypatch.setenv("CRDFFT_NO_FUSED_REAL", "1")
    ref = cf.Plan([n], batch=batch, kind=cf.R2C, odist=odist)
    assert ref.info()["algorithm"] == "real+four-step"
    ref.execute(x, b, cf.FORWARD)
    torch.cuda.synchronize()
    got = a.cpu().numpy().reshape(batch, odist)
    assert np.array_equal(got, b.cpu().numpy().reshape(batch, odist))  # same arithmetic, fused or not
    want = _spec64(x.cpu().numpy().reshape(batch, n)[[0, -1]])
    assert oracle.rel_l2(got[[0, -1], :h], want) <= REL_L2
    assert np.all(got[:, h:] == 3 + 3j)



@pytest.mark.parametrize("n,batch,pad,norm", [(1 << 20, 3, 0, 0), (1 << 21, 2, 5, 1)])
def test_long_c2r_follows_reference_irfft(n, batch, pad, norm):
    """C2R of long transforms (recombination kernel, then the half-length four-step) against the reference's irfft
    restated by the oracle, on spectra that are not Hermitian at 0 and n/2; the input is only read."""
    h = n // 2 + 1
    idist = h + pad
    nm = cf.NORM_INVERSE if norm else cf.NORM_NONE
    y = oracle.lcg_complex64(0xF31 ^ n ^ pad, batch * idist)
    ty = torch.from_numpy(y).cuda()
    out = torch.empty(batch * n, dtype=torch.float32, device="cuda")
    cf.Plan([n], batch=batch, kind=cf.C2R, idist=idist, norm=nm).execute(ty, out, cf.INVERSE)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(batch, n)
    want = oracle.irfft64(y.reshape(batch, idist)[[0, -1], :h], n) * (1 if norm else n)
    assert oracle.rel_l2(got[[0, -1]], want) <= REL_L2
    assert np.array_equal(ty.cpu().numpy(), y)


@pytest.mark.parametrize("n,batch", [(107520, 3), (2 * 105 * 512, 2)])
def test_r2c_c2r_with_odd_column_count(n, batch):
    """R2C/C2R whose half-length four-step has an odd number of columns (53760 = 105 x 512): the row pass cannot
    pair rows p and n1 - p in one CTA, so the recombination runs as its own step; both directions against the
    oracle."""
    h = n // 2 + 1
    x = torch.from_numpy(oracle.lcg_float32(0xF32 ^ n, batch * n)).cuda()
    spec = torch.empty(batch * h, dtype=torch.complex64, device="cuda")
    r2c = cf.Plan([n], batch=batch, kind=cf.R2C)
    r2c.execute(x, spec, cf.FORWARD)
    back = torch.empty_like(x)
    cf.Plan([n], batch=batch, kind=cf.C2R, norm=cf.NORM_INVERSE).execute(spec, back, cf.INVERSE)
    torch.cuda.synchronize()
    got = spec.cpu().numpy().reshape(batch, h)
    assert oracle.rel_l2(got, oracle.rfft64(x.cpu().numpy().reshape(batch, n))) <= REL_L2
    assert oracle.rel_l2(back.cpu().numpy(), x.cpu().numpy()) <= 2 * REL_L2
