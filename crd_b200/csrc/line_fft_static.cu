// Compile-time radix schedules of the line-FFT kernels: the line lengths the benchmarks and the four-step halves run
// (1024 and 4096 single-pass; 256 and 1024 as four-step halves of 65536 and 2^20; 105 = 7*5*3 for 107520 = 105*1024;
// 512 and 4096 for the 3-D and 2-D axes). Every division by n, L and R folds to a constant here.

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{
namespace
{
bool same_radices(const PassDesc& d, std::initializer_list<int> rs)
{
    if (static_cast<int>(rs.size()) != d.nstages)
        return false;
    int i = 0;
    for (int r : rs)
        if (d.radix[i++] != r)
            return false;
    return true;
}
} // namespace

KernelFn select_static(const PassDesc& d, const PassShape& sh)
{
#define CRDFFT_STATIC(P_, ...)                                                                                         \
    if (sh.points_per_thread == P_ && same_radices(d, {__VA_ARGS__}))                                                  \
        return pick<Sched<__VA_ARGS__>, P_>(sh.map, sh.direct_load, sh.direct_store);
    CRDFFT_STATIC(16, 16, 16, 4)     // 1024
    CRDFFT_STATIC(16, 16, 16)        // 256
    CRDFFT_STATIC(16, 16, 8, 4)      // 512
    CRDFFT_STATIC(16, 16, 16, 16)    // 4096 (rows)
    CRDFFT_STATIC(32, 16, 16, 16)    // 4096 (columns)
    CRDFFT_STATIC(32, 16, 16, 16, 4) // 16384
    CRDFFT_STATIC(16, 7, 5, 3)       // 105
#undef CRDFFT_STATIC
    return nullptr;
}

PipeFn select_pipe(const PassDesc& d, const PassShape& sh)
{
#define CRDFFT_PIPE(P_, ...)                                                                                           \
    if (sh.points_per_thread == P_ && same_radices(d, {__VA_ARGS__}))                                                  \
        return pick_pipe<Sched<__VA_ARGS__>, P_>(sh.map, sh.direct_store);
    CRDFFT_PIPE(16, 16, 16, 4)  // 1024
    CRDFFT_PIPE(16, 16, 16)     // 256
    CRDFFT_PIPE(16, 16, 8, 4)   // 512
    CRDFFT_PIPE(16, 16, 16, 16) // 4096
    CRDFFT_PIPE(16, 7, 5, 3)    // 105
#undef CRDFFT_PIPE
    return nullptr;
}

} // namespace lfft
} // namespace crdfft
