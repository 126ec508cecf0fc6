"""Split-complex (planar) operands through the C ABI (crdfft_execute_planar), and the CEIR tensor.fft lowering run
end to end: op attributes -> crdfft_ceir_fft_desc -> plan -> the op's four planes, against the FP64 oracle.
Tolerance: rel-L2 <= 1e-6 against FP64 (the FP32 parity bar of test_gpu_parity.py)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import crd_b200 as cf
import oracle

pytestmark = pytest.mark.gpu

REL_L2 = 1e-6


def _planes(x: np.ndarray):
    re = torch.from_numpy(np.ascontiguousarray(x.real.astype(np.float32))).cuda()
    im = torch.from_numpy(np.ascontiguousarray(x.imag.astype(np.float32))).cuda()
    return re, im


def _join(re: torch.Tensor, im: torch.Tensor) -> np.ndarray:
    return re.cpu().numpy().astype(np.float64) + 1j * im.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("n,batch", [(2, 9), (64, 33), (1024, 16), (4096, 8), (65536, 3), (1 << 20, 2), (105, 7),
                                     (1000, 5), (17, 6)])
@pytest.mark.parametrize("inverse", [False, True])
def test_planar_matches_oracle(n, batch, inverse):
    x = oracle.lcg_complex64(0x91A ^ n, n * batch).reshape(batch, n)
    re, im = _planes(x)
    ro, io = torch.empty_like(re), torch.empty_like(im)
    plan = cf.Plan([n], batch=batch)
    plan.execute_planar(re, im, ro, io, cf.INVERSE if inverse else cf.FORWARD)
    torch.cuda.synchronize()
    got = _join(ro, io).reshape(batch, n)
    assert oracle.rel_l2(got, oracle.fft64(x, inverse)) <= REL_L2
    # the input planes are only read
    assert np.array_equal(re.cpu().numpy(), x.real.astype(np.float32))


def test_planar_in_place_equals_interleaved_bits():
    """In place on the planes, and bit for bit the interleaved execute of the same plan."""
    n, batch = 4096, 12
    x = oracle.lcg_complex64(0x91B, n * batch)
    re, im = _planes(x)
    plan = cf.Plan([n], batch=batch)
    plan.execute_planar(re, im, re, im, cf.FORWARD)
    t = torch.from_numpy(x).cuda()
    o = torch.empty_like(t)
    plan.execute(t, o, cf.FORWARD)
    torch.cuda.synchronize()
    assert torch.equal(re, o.real.contiguous()) and torch.equal(im, o.imag.contiguous())


def test_planar_2d():
    dims, batch = (64, 128), 3
    x = oracle.lcg_complex64(0x91C, int(np.prod(dims)) * batch).reshape((batch,) + dims)
    re, im = _planes(x)
    ro, io = torch.empty_like(re), torch.empty_like(im)
    cf.Plan(list(dims), batch=batch).execute_planar(re, im, ro, io, cf.FORWARD)
    torch.cuda.synchronize()
    got = _join(ro, io).reshape((batch,) + dims)
    want = np.stack([oracle.nd64(x[b]) for b in range(batch)])
    assert oracle.rel_l2(got, want) <= REL_L2


@pytest.mark.parametrize("shape,axis,direction", [([1024], -1, "forward"), ([4, 6, 256], -1, "inverse"),
                                                  ([512, 8], 0, "forward"), ([3, 107520], -1, "forward"),
                                                  ([40, 1000], -1, "inverse")])
def test_tensor_fft_lowered_end_to_end(shape, axis, direction):
    """A tensor.fft op lowered by crdfft_ceir_fft_desc and run on its four planes: re_out + i im_out equals the FFT
    of re_in + i im_in along the op's axis, unnormalised both ways like the op."""
    d = cf.lower_tensor_fft(shape, direction, axis=axis)
    total = int(np.prod(shape))
    x = oracle.lcg_complex64(0x91D ^ total, total).reshape(shape)
    re, im = _planes(x.reshape(-1))
    ro, io = torch.empty_like(re), torch.empty_like(im)
    plan = cf.Plan(d["dims"], batch=d["batch"], norm=d["norm"], istride=d["istride"], idist=d["idist"],
                   ostride=d["ostride"], odist=d["odist"])
    plan.execute_planar(re, im, ro, io, d["direction"])
    torch.cuda.synchronize()
    got = _join(ro, io).reshape(shape)
    ax = axis % len(shape)
    moved = np.moveaxis(x, ax, -1)
    want = np.moveaxis(oracle.fft64(np.ascontiguousarray(moved), direction == "inverse"), -1, ax)
    assert oracle.rel_l2(got, want) <= REL_L2


def test_planar_rejects_layouts_that_do_not_tile_the_planes():
    x = torch.zeros(4096, device="cuda")
    plan = cf.Plan([1024], batch=2, idist=2048, odist=2048)  # padded distances: gaps between transforms
    with pytest.raises(cf.CrdFftError):
        plan.execute_planar(x, x, x, x, cf.FORWARD)
