// The recombination of a real transform's pairs (k, M - k) around its half-length complex FFT (n = 2M points):
// the math of the reference's RealFftPlan (include/crd/hesap/fft/real_fft.hpp:41-92), with W = exp(-2 pi i / n),
// E = (Z[k] + conj Z[M-k]) / 2 and O = (Z[k] - conj Z[M-k]) / 2i:
//   X[k] = E + W^k O,   X[M-k] = conj(E - W^k O);
// and for the inverse, with a = Y[k] + conj Y[M-k], b = Y[k] - conj Y[M-k]:
//   Q[k] = a + i b W^-k,   Q[M-k] = conj(a) + i conj(b W^-k).

#pragma once

#include "line_fft.cuh"

namespace crdfft
{
namespace lfft
{

__device__ __forceinline__ float2 conjf2(float2 v) { return make_float2(v.x, -v.y); }

// X[k], X[M-k] from Z[k], Z[M-k] (0 < k <= M/2); w = W^k.
__device__ __forceinline__ void r2c_pair(float2 zk, float2 zm, float2 w, float2& xk, float2& xm)
{
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    // (Z[k] - conj Z[M-k]) / 2i: (u + iv) / 2i = (v - iu) / 2
    const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    const float2 t = cmul(w, o);
    xk = make_float2(e.x + t.x, e.y + t.y);
    xm = make_float2(e.x - t.x, t.y - e.y);
}

// Q[k], Q[M-k] from Y[k], Y[M-k] (0 < k <= M/2); w = W^k.
__device__ __forceinline__ void c2r_pair(float2 yk, float2 ym, float2 w, float2& qk, float2& qm)
{
    const float2 a = make_float2(yk.x + ym.x, yk.y - ym.y);
    const float2 b = make_float2(yk.x - ym.x, yk.y + ym.y);
    const float2 bw = cmul(b, conjf2(w));
    qk = make_float2(a.x - bw.y, a.y + bw.x);
    qm = make_float2(a.x + bw.y, bw.x - a.y);
}

} // namespace lfft
} // namespace crdfft
