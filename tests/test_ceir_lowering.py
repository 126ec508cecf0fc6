"""The CEIR tensor.fft lowering (crdfft_ceir_fft_desc), host only: the op's attributes and operand shape mapped to a
plan descriptor, and each of the reference's rejections (engine/execution/ceir-gpu/src/ckir_synth.cpp:318-366) in
its order, with the envelope widened from powers of two to every static length and to a batch."""

from __future__ import annotations

import pytest

import crd_b200 as cf
from crd_b200 import _lib


def test_rank1_power_of_two_as_the_reference():
    d = cf.lower_tensor_fft([1024], "forward")
    assert d == {"dims": [1024], "batch": 1, "istride": 1, "idist": 1024, "ostride": 1, "odist": 1024,
                 "norm": cf.NORM_NONE, "direction": cf.FORWARD}
    assert cf.lower_tensor_fft([2], "inverse")["direction"] == cf.INVERSE  # unnormalised: the 1/N is the caller's


@pytest.mark.parametrize("n", [3, 105, 1000, 17, 107520, 1])
def test_lengths_beyond_the_power_of_two_envelope(n):
    """The reference names a non-power-of-two length forward (FftLengthNotPow2); here it is planned."""
    d = cf.lower_tensor_fft([n], "forward")
    assert d["dims"] == [n] and d["batch"] == 1


def test_innermost_axis_of_higher_rank_is_a_packed_batch():
    d = cf.lower_tensor_fft([4, 6, 256], "forward")
    assert (d["dims"], d["batch"], d["istride"], d["idist"]) == ([256], 24, 1, 256)
    assert cf.lower_tensor_fft([4, 6, 256], "forward", axis=2) == d


def test_axis0_of_rank2_is_the_element_major_batch():
    d = cf.lower_tensor_fft([512, 8], "inverse", axis=0)
    assert (d["dims"], d["batch"], d["istride"], d["idist"], d["ostride"], d["odist"]) == ([512], 8, 8, 1, 8, 1)
    assert d["direction"] == cf.INVERSE


@pytest.mark.parametrize("kw,reason", [
    (dict(num_operands=1), "op-not-supported"),
    (dict(num_results=1), "op-not-supported"),
    (dict(operand_is_tensor=False), "operand-not-tensor"),
    (dict(element_f32=False), "element-not-f32"),
    (dict(shape=[8, -1]), "shape-not-static"),
    (dict(direction="sideways"), "direction-unknown"),
    (dict(direction=None), "direction-unknown"),
    (dict(shape=[4, 8, 16], axis=1), "axis-unsupported"),
    (dict(shape=[4, 8], axis=2), "axis-unsupported"),
    (dict(shape=[2] * 9), "rank-unsupported"),
])
def test_rejections(kw, reason):
    args = dict(shape=[64], direction="forward")
    args.update(kw)
    shape, direction = args.pop("shape"), args.pop("direction")
    with pytest.raises(_lib.CrdFftError, match=reason):
        cf.lower_tensor_fft(shape, direction, **args)


def test_arity_is_checked_before_the_operand():
    """As in the reference, a malformed arity is reported before anything about re_in is read."""
    with pytest.raises(_lib.CrdFftError, match="op-not-supported"):
        cf.lower_tensor_fft([64], "forward", num_operands=1, operand_is_tensor=False, element_f32=False)
