// Compile-time schedule 16 x 4 (n = 64), 16 points a thread: the classic kernel.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_64, 16, 16,4)
} // namespace lfft
} // namespace crdfft
