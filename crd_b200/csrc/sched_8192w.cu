// Compile-time schedule 16 x 16 x 8 x 4 (n = 8192), 32 points a thread: the classic kernel.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_8192w, 32, 16,16,8,4)
} // namespace lfft
} // namespace crdfft
