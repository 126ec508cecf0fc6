// Compile-time schedule 16 (n = 16), 16 points a thread: the classic kernel.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_16, 16, 16)
} // namespace lfft
} // namespace crdfft
