// Compile-time schedule 7 x 5 x 3 (n = 105), 16 points a thread: classic and pipelined kernels.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_105, 16, 7,5,3)
CRDFFT_DEFINE_PIPE(s_105, 16, 7,5,3)
} // namespace lfft
} // namespace crdfft
