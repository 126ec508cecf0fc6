// crdfft_execute_static_scratch: a batched 1-D complex FFT that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that enqueues work while a CUDA stream is being captured into a graph
// (an allocation there is an error), real-time audio or signal-processing callbacks that must never enter an
// allocator, and processes whose device memory is handed in full to a pool they do not own. They can still pass
// their own input and output buffers. This entry point gives them the library's normal plan and kernels, with every
// piece of device memory a plan needs (twiddle tables, the status word, the two-pass four-step's intermediate)
// carved from one file-scope device array instead of cudaMalloc.
//
// The array is kStaticScratchBytes (64 MiB) and lives on every GPU that loads the library until the process exits.
// Half of it is available for the four-step intermediate, so a transform may hold at most 2^22 complex points
// (32 MiB); larger n are rejected with CRDFFT_UNSUPPORTED_SIZE. A length with a prime factor above 7 runs Bluestein
// over a padded power-of-two length m >= 2n - 1, whose tables and padded sequences take about 8 m (batch + 3) bytes:
// such n are accepted while that fits in the array (for one transform, n up to about 2^20) and are otherwise also
// rejected with CRDFFT_UNSUPPORTED_SIZE.
//
// Every call on a device shares the one array: the most recent call's plan (its tables) stays in it, and two calls
// whose work overlaps on the GPU (different streams, no ordering between them) race on it and may produce wrong
// results; order such calls on one stream. A call with a new size or batch rebuilds the plan into the array: it first
// waits until the device has finished all work queued so far (the previous call's kernels may still be reading the
// old tables, on whatever stream they were queued), writes the new tables and waits for them to land, then queues the
// transform. A call that would rebuild while its stream is being captured returns CRDFFT_INVALID_ARG and queues
// nothing (the wait and the table uploads cannot be part of a capture); make the first call with each (n, batch)
// outside the capture. Work captured from this entry point reads the array as it was when captured, so a graph
// captured with one (n, batch) is valid only until a call with a different (n, batch) rebuilds the array. The first
// call on a device also looks up the array's device address, so make it before any stream capture.

#include "../../include/crdfft.h"
#include "kernels.hpp"

#include <cuda_runtime.h>

#include <map>
#include <mutex>

namespace
{

constexpr size_t kStaticScratchBytes = size_t{64} << 20;
constexpr long long kMaxStaticScratchPoints = 1LL << 22;

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct DeviceScratch
{
    bool ready = false;
    char* base = nullptr; // the array's device address (cudaGetSymbolAddress); never the host-side name
    crdfft_plan* plan = nullptr;
    long long n = 0;
    long long batch = 0;
    crdfft::Arena arena{};
};

std::mutex g_mu;
std::map<int, DeviceScratch> g_devices;

} // namespace

extern "C" crdfft_status crdfft_execute_static_scratch(const void* in, void* out, int64_t n, int64_t batch,
                                                       int32_t direction, void* stream)
{
    if (in == nullptr || out == nullptr || n < 1 || batch < 1)
        return CRDFFT_INVALID_ARG;
    if (direction != CRDFFT_FORWARD && direction != CRDFFT_INVERSE)
        return CRDFFT_INVALID_ARG;
    if (n > kMaxStaticScratchPoints)
        return CRDFFT_UNSUPPORTED_SIZE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return CRDFFT_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceScratch& s = g_devices[dev];
    if (!s.ready)
    {
        void* addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_static_scratch) != cudaSuccess || addr == nullptr)
            return CRDFFT_LAUNCH;
        s.base = static_cast<char*>(addr);
        s.ready = true;
    }
    if (s.plan == nullptr || s.n != n || s.batch != batch)
    {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap) != cudaSuccess)
            return CRDFFT_LAUNCH;
        if (cap != cudaStreamCaptureStatusNone)
            return CRDFFT_INVALID_ARG; // a rebuild cannot be captured; the array is left as it was
        // The previous call's kernels may still read the array (its tables, its intermediate) on any stream: let
        // every queued kernel finish before the array is rewritten.
        if (cudaDeviceSynchronize() != cudaSuccess)
            return CRDFFT_LAUNCH;
        if (s.plan != nullptr)
        {
            crdfft_plan_destroy(s.plan); // arena-backed: releases host state only
            s.plan = nullptr;
        }
        s.arena = crdfft::Arena{s.base, kStaticScratchBytes, 0};
        crdfft_desc d{};
        d.rank = 1;
        d.kind = CRDFFT_C2C;
        d.precision = CRDFFT_PREC_FP32;
        d.norm = CRDFFT_NORM_NONE;
        d.dims[0] = n;
        d.batch = batch;
        crdfft::arena_bind(&s.arena);
        crdfft_plan* p = nullptr;
        crdfft_status st = crdfft_plan_create(&d, &p);
        crdfft::arena_bind(nullptr);
        if (st != CRDFFT_OK)
        {
            if (p != nullptr)
                crdfft_plan_destroy(p);
            return st == CRDFFT_OOM ? CRDFFT_UNSUPPORTED_SIZE : st;
        }
        s.plan = p;
        s.n = n;
        s.batch = batch;
    }
    return crdfft_execute(s.plan, in, out, direction, stream);
}
