// Compile-time schedule 16 x 16 x 4 (n = 1024), 32 points a thread: the classic kernel only. With 32 threads a line,
// a 512-thread CTA holds 16 column lines, so column passes read and write 128-byte runs.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
CRDFFT_DEFINE_SCHEDULE(s_1024w, 32, 16,16,4)
} // namespace lfft
} // namespace crdfft
