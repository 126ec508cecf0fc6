// Compile-time schedule 16 x 16 (n = 256), 16 points a thread: classic and pipelined kernels.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_256, 16, 16,16)
CRDFFT_DEFINE_PIPE(s_256, 16, 16,16)
} // namespace lfft
} // namespace crdfft
