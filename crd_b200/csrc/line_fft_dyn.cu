// The line-FFT kernel with its radix schedule read from the descriptor at run time: every 7-smooth line length up to
// 8192 that has no compile-time schedule (the uneven-size batches, Bluestein's inner lengths, odd N-D axes).

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{

KernelFn select_dynamic(const PassDesc& d, const PassShape& sh)
{
    if (sh.points_per_thread != 16)
        return nullptr;
    return pick<DynSched, 16>(sh.map, sh.direct_load, sh.direct_store, pass_epi(d));
}

} // namespace lfft
} // namespace crdfft
