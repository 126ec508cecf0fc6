// Compile-time schedule 16 x 16 x 4 (n = 1024), 16 points a thread: classic and pipelined kernels.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_1024, 16, 16,16,4)
CRDFFT_DEFINE_PIPE(s_1024, 16, 16,16,4)
} // namespace lfft
} // namespace crdfft
