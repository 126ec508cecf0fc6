"""ctypes binding of libcrdfft.so (the C ABI declared in include/crdfft.h).

The library is built in-tree (``make -C crd_b200``, or ``__graft_entry__.build()``). There is no fallback: if the
shared object is missing or fails to load, every entry point raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcrdfft.so")

OK = 0
INVALID_DESC = 1
UNSUPPORTED_SIZE = 2
OOM = 3
LAUNCH = 4
DEVICE_TIMEOUT = 5
NUMERIC_SELFCHECK = 6
INVALID_ARG = 7
NO_DEVICE = 8

FORWARD = 0
INVERSE = 1

C2C = 0
R2C = 1
C2R = 2

PREC_FP32 = 0
PREC_SPLIT_BF16 = 1
PREC_FP16_SCALED = 2
PREC_SPLIT_BF16_2 = 3
PREC_SPLIT_FP16_2 = 4
PLANNER_ESTIMATE = 0
PLANNER_MEASURE = 1
PLANNER_LEARNED = 2

NORM_NONE = 0
NORM_INVERSE = 1

SPECTRAL_WELCH = 0
SPECTRAL_SPECTROGRAM = 1
SPECTRAL_PERIODOGRAM = 2

# Every function include/crdfft.h declares; the CPU tests check the library exports each of them.
EXPORTS = (
    "crdfft_plan_create",
    "crdfft_plan_destroy",
    "crdfft_execute",
    "crdfft_execute_host",
    "crdfft_conv_plan_create",
    "crdfft_conv_execute",
    "crdfft_spectral_plan_create",
    "crdfft_spectral_segments",
    "crdfft_spectral_execute",
    "crdfft_cwt_plan_create",
    "crdfft_cwt_plan_destroy",
    "crdfft_cwt_execute",
    "crdfft_cwt_frequencies",
    "crdfft_cwt_fft_length",
    "crdfft_cwt_plan_info",
    "crdfft_plan_info_get",
    "crdfft_workspace_size",
    "crdfft_set_workspace",
    "crdfft_status_string",
    "crdfft_fft_plan_create",
    "crdfft_fft_execute",
    "crdfft_fft_execute_batched",
    "crdfft_real_plan_create",
    "crdfft_rfft",
    "crdfft_irfft",
    "crdfft_bluestein_plan_create",
    "crdfft_bluestein_execute",
    "crdfft_nd_plan_create",
    "crdfft_nd_execute",
    "crdfft_fft",
    "crdfft_ifft_normalized",
    "crdfft_self_check",
    "crdfft_debug_self_check_mismatch",
    "crdfft_debug_self_check_reset",
    "crdfft_debug_uneven_variant",
    "crdfft_debug_fail_alloc_after",
    "crdfft_device_status",
    "crdfft_debug_stall_waits",
    "crdfft_set_planner_mode",
    "crdfft_set_decomposition",
    "crdfft_wisdom_export",
    "crdfft_wisdom_import",
    "crdfft_wisdom_forget",
    "crdfft_planner_log",
    "crdfft_execute_static_scratch",
    "crdfft_execute_planar",
    "crdfft_ceir_fft_desc",
    "crdfft_plan_create_uneven",
    "crdfft_uneven_offsets",
    "crdfft_pass_feature_count",
    "crdfft_learned_model_import",
    "crdfft_learned_model_export",
    "crdfft_learned_model_forget",
    "crdfft_learned_predict",
    "crdfft_mlp_param_count",
    "crdfft_mlp_workspace_floats",
    "crdfft_mlp_forward",
    "crdfft_mlp_gradients",
    "crdfft_mlp_adam",
)


class CrdFftError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().crdfft_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


class Desc(ctypes.Structure):
    _fields_ = [
        ("rank", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("norm", ctypes.c_int32),
        ("dims", ctypes.c_int64 * 3),
        ("batch", ctypes.c_int64),
        ("istride", ctypes.c_int64),
        ("idist", ctypes.c_int64),
        ("ostride", ctypes.c_int64),
        ("odist", ctypes.c_int64),
    ]


class CeirFftOp(ctypes.Structure):
    """crdfft_ceir_fft_op: what the reference's GPU provider knows about a CEIR tensor.fft op."""

    _fields_ = [
        ("num_operands", ctypes.c_int32),
        ("num_results", ctypes.c_int32),
        ("operand_is_tensor", ctypes.c_int32),
        ("element_is_f32", ctypes.c_int32),
        ("rank", ctypes.c_int32),
        ("axis", ctypes.c_int32),
        ("shape", ctypes.c_int64 * 8),
        ("direction", ctypes.c_char_p),
    ]


CEIR_REJECT = {0: "none", 1: "op-not-supported", 2: "operand-not-tensor", 3: "element-not-f32",
               4: "rank-unsupported", 5: "shape-not-static", 6: "direction-unknown", 7: "axis-unsupported"}


class SpectralDesc(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("detrend", ctypes.c_int32),
        ("nsamples", ctypes.c_int64),
        ("count", ctypes.c_int64),
        ("nperseg", ctypes.c_int64),
        ("noverlap", ctypes.c_int64),
        ("fs", ctypes.c_double),
        ("window", ctypes.POINTER(ctypes.c_float)),
    ]


class CwtDesc(ctypes.Structure):
    _fields_ = [
        ("wavelet", ctypes.c_char_p),
        ("scales", ctypes.POINTER(ctypes.c_double)),
        ("nsamples", ctypes.c_int64),
        ("count", ctypes.c_int64),
        ("nscales", ctypes.c_int64),
        ("sampling_period", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("algorithm", ctypes.c_char * 64),
        ("passes", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("workspace_bytes", ctypes.c_int64),
        ("table_bytes", ctypes.c_int64),
        ("factors", ctypes.c_int64 * 8),
    ]


_lib = None


def lib():
    """Load libcrdfft.so once. Raises if it is absent: the CUDA path has no substitute."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C crd_b200` (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    pp = ctypes.POINTER(ctypes.c_void_p)
    i32, i64 = ctypes.c_int32, ctypes.c_int64
    sig = {
        "crdfft_plan_create": ([ctypes.POINTER(Desc), pp], i32),
        "crdfft_plan_destroy": ([vp], i32),
        "crdfft_execute": ([vp, vp, vp, i32, vp], i32),
        "crdfft_execute_host": ([vp, vp, vp, i32, vp], i32),
        "crdfft_conv_plan_create": ([ctypes.POINTER(Desc), i32, ctypes.c_double, pp], i32),
        "crdfft_conv_execute": ([vp, vp, vp, vp, vp], i32),
        "crdfft_spectral_plan_create": ([ctypes.POINTER(SpectralDesc), pp], i32),
        "crdfft_spectral_segments": ([ctypes.POINTER(SpectralDesc)], i64),
        "crdfft_spectral_execute": ([vp, vp, vp, vp], i32),
        "crdfft_cwt_plan_create": ([ctypes.POINTER(CwtDesc), pp], i32),
        "crdfft_cwt_plan_destroy": ([vp], i32),
        "crdfft_cwt_execute": ([vp, vp, vp, vp], i32),
        "crdfft_cwt_frequencies": ([ctypes.POINTER(CwtDesc), ctypes.POINTER(ctypes.c_double)], i32),
        "crdfft_cwt_fft_length": ([ctypes.POINTER(CwtDesc)], i64),
        "crdfft_cwt_plan_info": ([vp, ctypes.POINTER(i64), ctypes.POINTER(i64), ctypes.POINTER(i32)], i32),
        "crdfft_plan_info_get": ([vp, ctypes.POINTER(PlanInfo)], i32),
        "crdfft_workspace_size": ([vp], ctypes.c_size_t),
        "crdfft_set_workspace": ([vp, vp, ctypes.c_size_t], i32),
        "crdfft_status_string": ([i32], ctypes.c_char_p),
        "crdfft_fft_plan_create": ([i64, pp], i32),
        "crdfft_fft_execute": ([vp, vp, i32, vp], i32),
        "crdfft_fft_execute_batched": ([vp, vp, i64, i32, vp], i32),
        "crdfft_real_plan_create": ([i64, pp], i32),
        "crdfft_rfft": ([vp, vp, vp, vp], i32),
        "crdfft_irfft": ([vp, vp, vp, vp], i32),
        "crdfft_bluestein_plan_create": ([i64, pp], i32),
        "crdfft_bluestein_execute": ([vp, vp, i32, vp], i32),
        "crdfft_nd_plan_create": ([i32, ctypes.POINTER(i64), pp], i32),
        "crdfft_nd_execute": ([vp, vp, i32, vp], i32),
        "crdfft_fft": ([vp, i64, i32, vp], i32),
        "crdfft_ifft_normalized": ([vp, i64, vp], i32),
        "crdfft_self_check": ([], i32),
        "crdfft_debug_self_check_mismatch": ([i32], None),
        "crdfft_debug_self_check_reset": ([], None),
        "crdfft_debug_uneven_variant": ([i32], None),
        "crdfft_debug_fail_alloc_after": ([i32], None),
        "crdfft_device_status": ([vp, vp], i32),
        "crdfft_debug_stall_waits": ([i32], None),
        "crdfft_set_planner_mode": ([i32], None),
        "crdfft_set_decomposition": ([i64, i32, i64], i32),
        "crdfft_wisdom_export": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], i32),
        "crdfft_wisdom_import": ([ctypes.c_char_p], i32),
        "crdfft_wisdom_forget": ([], None),
        "crdfft_planner_log": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], i32),
        "crdfft_execute_static_scratch": ([vp, vp, i64, i64, i32, vp], i32),
        "crdfft_execute_planar": ([vp, vp, vp, vp, vp, i32, vp], i32),
        "crdfft_ceir_fft_desc": ([ctypes.POINTER(CeirFftOp), ctypes.POINTER(Desc), ctypes.POINTER(i32),
                                  ctypes.POINTER(i32)], i32),
        "crdfft_plan_create_uneven": ([ctypes.POINTER(i64), i64, ctypes.POINTER(i64), pp], i32),
        "crdfft_uneven_offsets": ([ctypes.POINTER(i64), i64, ctypes.POINTER(i64)], i64),
        "crdfft_pass_feature_count": ([], i32),
        "crdfft_learned_model_import": ([ctypes.c_char_p], i32),
        "crdfft_learned_model_export": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], i32),
        "crdfft_learned_model_forget": ([], None),
        "crdfft_learned_predict": ([ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)], i32),
        "crdfft_mlp_param_count": ([i32, i32], ctypes.c_size_t),
        "crdfft_mlp_workspace_floats": ([i32, i32, i64], ctypes.c_size_t),
        "crdfft_mlp_forward": ([i32, i32, vp, vp, i64, vp, vp, vp], i32),
        "crdfft_mlp_gradients": ([i32, i32, vp, vp, vp, i64, vp, vp, vp, vp], i32),
        "crdfft_mlp_adam": ([vp, vp, vp, vp, i64, i32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                             ctypes.c_float, vp], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise CrdFftError(status, what)
