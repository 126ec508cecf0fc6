// Compile-time schedule 16 x 8 x 4 (n = 512), 16 points a thread: classic and pipelined kernels.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_512, 16, 16,8,4)
CRDFFT_DEFINE_PIPE(s_512, 16, 16,8,4)
} // namespace lfft
} // namespace crdfft
