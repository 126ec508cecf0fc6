// Compile-time schedule 8 x 4 (n = 32), 16 points a thread: the classic kernel.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_32, 16, 8,4)
} // namespace lfft
} // namespace crdfft
