"""crd_b200: a B200-native (sm_100a) replacement for crd-hesap-fft's plan + execute path.

The compute runs in ``libcrdfft.so`` (hand-written CUDA kernels behind the C ABI in ``include/crdfft.h``); this
package is the Python mirror of the reference's plan classes over that ABI (``crd_b200.hesap``).
"""

from .hesap import (BluesteinPlan, ConvPlan, CwtPlan, FftPlan, Forward, Inverse, NdFftPlan, Plan, RealFftPlan,
                    SpectralPlan, UnevenPlan, cwt, cwt_fft_length, cwt_frequencies, fft, ifft_normalized,
                    lower_tensor_fft, periodogram, self_check, spectrogram, uneven_offsets, welch_psd)
from ._lib import (C2C, C2R, FORWARD, INVERSE, NORM_INVERSE, NORM_NONE, PREC_FP16_SCALED, PREC_FP32,
                   PREC_SPLIT_BF16, PREC_SPLIT_BF16_2, PREC_SPLIT_FP16_2, R2C, SPECTRAL_PERIODOGRAM, SPECTRAL_SPECTROGRAM, SPECTRAL_WELCH, CrdFftError)

__all__ = [
    "BluesteinPlan", "ConvPlan", "FftPlan", "NdFftPlan", "Plan", "RealFftPlan", "SpectralPlan", "UnevenPlan", "fft",
    "ifft_normalized", "self_check", "uneven_offsets", "welch_psd", "spectrogram", "periodogram", "CwtPlan", "cwt",
    "cwt_fft_length", "cwt_frequencies", "lower_tensor_fft",
    "SPECTRAL_WELCH", "SPECTRAL_SPECTROGRAM", "SPECTRAL_PERIODOGRAM",
    "Forward", "Inverse", "C2C", "R2C", "C2R", "FORWARD", "INVERSE", "NORM_NONE", "NORM_INVERSE", "PREC_FP32",
    "PREC_SPLIT_BF16", "PREC_FP16_SCALED", "PREC_SPLIT_BF16_2", "PREC_SPLIT_FP16_2", "CrdFftError",
]
