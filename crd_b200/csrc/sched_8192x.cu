// Compile-time schedule 32 x 16 x 16 (n = 8192), 32 points a thread: the classic kernel (radix-32 stages, one
// exchange through shared memory fewer than the radix-16 schedule of the same length).

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_8192x, 32, 32,16,16)
} // namespace lfft
} // namespace crdfft
