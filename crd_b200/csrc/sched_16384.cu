// Compile-time schedule 16 x 16 x 16 x 4 (n = 16384), 32 points a thread: classic kernels.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_16384, 32, 16,16,16,4)

} // namespace lfft
} // namespace crdfft
