// Compile-time schedule 16 x 16 x 16 (n = 4096), 32 points a thread: classic kernels.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_4096c, 32, 16,16,16)

} // namespace lfft
} // namespace crdfft
