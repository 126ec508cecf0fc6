// Compile-time schedule 16 x 16 x 8 (n = 2048), 16 points a thread: the classic kernel.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_2048, 16, 16,16,8)
} // namespace lfft
} // namespace crdfft
