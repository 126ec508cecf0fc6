// The lowering of CEIR's `tensor.fft` op onto this library: the decision the reference's GPU provider makes in
// synth_fft (engine/execution/ceir-gpu/src/ckir_synth.cpp:318-366) before it authors a radix-2 CKIR kernel, restated
// so that the provider can call crdfft_plan_create / crdfft_execute_planar instead.
//
// The op (engine/execution/ceir/src/tensor.cpp:174-192, 344): operands re_in, im_in, results re_out, im_out, all f32
// tensors of one shape (split-complex planes), attributes `direction` ("forward" or "inverse") and `axis`; the
// inverse is unnormalised (the 1/N is the caller's, engine/gpu/kir/include/crd/kir/ckir_fft.hpp:21). The reference
// accepts rank 1, a static power-of-two n >= 2 (ckir_synth.cpp:343-366) and names everything else forward. Here the
// same checks come first, in the same order; the envelope then widens to every length this library plans (7-smooth
// lengths natively, others through Bluestein) and to a leading batch: the transformed axis is the innermost one of
// a rank-r tensor (batch = the product of the other extents, packed), or axis 0 of a rank-2 tensor (the
// element-major batch, stride = the second extent). Anything else is rejected with a reason.

#include "../../include/crdfft.h"

#include <cstring>

extern "C" crdfft_status crdfft_ceir_fft_desc(const crdfft_ceir_fft_op* op, crdfft_desc* desc, int32_t* direction,
                                              int32_t* reject)
{
    if (op == nullptr || desc == nullptr || direction == nullptr || reject == nullptr)
        return CRDFFT_INVALID_ARG;
    auto fail = [&](crdfft_ceir_reject why, crdfft_status st) {
        *reject = why;
        return st;
    };
    // arity before any operand is looked at (ckir_synth.cpp:325-329)
    if (op->num_operands < 2 || op->num_results < 2)
        return fail(CRDFFT_CEIR_OP_NOT_SUPPORTED, CRDFFT_INVALID_DESC);
    if (!op->operand_is_tensor) // re_in (ckir_synth.cpp:331-336)
        return fail(CRDFFT_CEIR_OPERAND_NOT_TENSOR, CRDFFT_INVALID_DESC);
    if (!op->element_is_f32) // :337-341
        return fail(CRDFFT_CEIR_ELEMENT_NOT_F32, CRDFFT_INVALID_DESC);
    if (op->rank < 1 || op->rank > CRDFFT_CEIR_MAX_RANK) // the reference: rank 1 only (:344-349)
        return fail(CRDFFT_CEIR_RANK_UNSUPPORTED, CRDFFT_UNSUPPORTED_SIZE);
    long long total = 1;
    for (int i = 0; i < op->rank; ++i)
    {
        if (op->shape[i] < 1) // a dynamic (or empty) extent (:350-355)
            return fail(CRDFFT_CEIR_SHAPE_NOT_STATIC, CRDFFT_UNSUPPORTED_SIZE);
        total *= op->shape[i];
    }
    const int axis = op->axis < 0 ? op->rank - 1 : op->axis;
    if (axis >= op->rank)
        return fail(CRDFFT_CEIR_AXIS_UNSUPPORTED, CRDFFT_INVALID_DESC);
    // the direction attribute (:362-381)
    if (op->direction == nullptr)
        return fail(CRDFFT_CEIR_DIRECTION_UNKNOWN, CRDFFT_INVALID_DESC);
    int dir;
    if (std::strcmp(op->direction, "forward") == 0)
        dir = CRDFFT_FORWARD;
    else if (std::strcmp(op->direction, "inverse") == 0)
        dir = CRDFFT_INVERSE;
    else
        return fail(CRDFFT_CEIR_DIRECTION_UNKNOWN, CRDFFT_INVALID_DESC);

    const long long n = op->shape[axis];
    crdfft_desc d{};
    d.rank = 1;
    d.kind = CRDFFT_C2C;
    d.precision = CRDFFT_PREC_FP32;
    d.norm = CRDFFT_NORM_NONE; // the op's inverse is unnormalised
    d.dims[0] = n;
    d.batch = total / n;
    if (axis == op->rank - 1)
    {
        d.istride = d.ostride = 1; // packed: transform t at t * n
        d.idist = d.odist = n;
    }
    else if (op->rank == 2 && axis == 0)
    {
        d.istride = d.ostride = op->shape[1]; // element-major: element i of transform t at i * batch + t
        d.idist = d.odist = 1;
    }
    else
        return fail(CRDFFT_CEIR_AXIS_UNSUPPORTED, CRDFFT_UNSUPPORTED_SIZE);
    *desc = d;
    *direction = dir;
    *reject = CRDFFT_CEIR_NONE;
    return CRDFFT_OK;
}
