// Register-resident DFT codelets for radix 2, 3, 4, 5, 7, 8, 9, 16 and 25, and the complex helpers the pass kernels use.
//
// These replace the reference's machine-generated straight-line SIMD codelets (engine/numerics/hesap-fft/kernels/
// fft_*_codelets_*.cpp, emitted by scripts/gen_fft_batched.py and scripts/gen_fft_codelets.py) and add the odd radices
// 3, 5 and 7, which the reference does not have (its non-power-of-two sizes go through Bluestein,
// include/crd/hesap/fft/bluestein.hpp:29-139). Every codelet computes the forward DFT y_k = sum_j x_j W_R^{jk},
// W_R = exp(-2πi/R), in place on R complex values in registers; the inverse is obtained by conjugating the pass's
// input and output (IDFT(x) = conj(DFT(conj x))). The constants are cos/sin of 2πj/R written out to 20 digits.

#pragma once

#include <cuda_runtime.h>

namespace crdfft
{

// ---- complex values -------------------------------------------------------------------------------------------
//
// The codelets are templates over the value type they transform (float2: x real, y imaginary), written against the
// small set of operations below, so a kernel could instantiate them for another representation of complex values.

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cneg(float2 a) { return make_float2(-a.x, -a.y); }
// -i * a
__device__ __forceinline__ float2 cmul_mi(float2 a) { return make_float2(a.y, -a.x); }
// +i * a
__device__ __forceinline__ float2 cmul_pi(float2 a) { return make_float2(-a.y, a.x); }
// a + (-i) b and a - (-i) b
__device__ __forceinline__ float2 add_mi(float2 a, float2 b) { return make_float2(a.x + b.y, a.y - b.x); }
__device__ __forceinline__ float2 sub_mi(float2 a, float2 b) { return make_float2(a.x - b.y, a.y + b.x); }
// a (c - i s): multiplication by the forward root of angle θ with c = cos θ, s = sin θ
__device__ __forceinline__ float2 crot(float2 a, float c, float s) { return make_float2(a.x * c + a.y * s, a.y * c - a.x * s); }
// H (1 - i) a, H (-1 - i) a, H (-1 + i) a, H (1 + i) a
__device__ __forceinline__ float2 crot_h1(float2 a, float h) { return make_float2(h * (a.x + a.y), h * (a.y - a.x)); }
__device__ __forceinline__ float2 crot_h3(float2 a, float h) { return make_float2(h * (a.y - a.x), -h * (a.x + a.y)); }
__device__ __forceinline__ float2 crot_h5(float2 a, float h) { return make_float2(-h * (a.x + a.y), h * (a.x - a.y)); }
__device__ __forceinline__ float2 crot_h7(float2 a, float h) { return make_float2(h * (a.x - a.y), h * (a.x + a.y)); }
// acc + c a (real c)
__device__ __forceinline__ float2 cmadd(float2 acc, float2 a, float c)
{
    return make_float2(fmaf(c, a.x, acc.x), fmaf(c, a.y, acc.y));
}
template <class C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }

// Multiply by the compile-time root W_16^J (forward sign), specialised so the trivial roots cost no multiplies.
template <int J, class C> __device__ __forceinline__ C w16mul(C a)
{
    constexpr float CS = 0.92387953251128675613f; // cos(π/8)
    constexpr float SN = 0.38268343236508977173f; // sin(π/8)
    constexpr float H = 0.70710678118654752440f;  // cos(π/4)
    constexpr int j = J & 15;
    if constexpr (j == 0)
        return a;
    else if constexpr (j == 4)
        return cmul_mi(a);
    else if constexpr (j == 8)
        return cneg(a);
    else if constexpr (j == 12)
        return cmul_pi(a);
    else if constexpr (j == 2)
        return crot_h1(a, H);
    else if constexpr (j == 6)
        return crot_h3(a, H);
    else if constexpr (j == 10)
        return crot_h5(a, H);
    else if constexpr (j == 14)
        return crot_h7(a, H);
    else
    {
        // W_16^j = cos(2πj/16) - i sin(2πj/16); the remaining j are odd.
        constexpr float c = (j == 1 || j == 15) ? CS : (j == 3 || j == 13) ? SN : (j == 5 || j == 11) ? -SN : -CS;
        constexpr float s = (j == 1 || j == 7) ? SN : (j == 3 || j == 5) ? CS : (j == 9 || j == 15) ? -SN : -CS;
        return crot(a, c, s);
    }
}

template <int R> struct Dft;

template <> struct Dft<2>
{
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <> struct Dft<4>
{
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        const C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const C s13 = cadd(v[1], v[3]), t13 = csub(v[1], v[3]);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = add_mi(d02, t13);
        v[3] = sub_mi(d02, t13);
    }
};

template <> struct Dft<8>
{
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        C e[4] = {v[0], v[2], v[4], v[6]};
        C o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4>::run(e);
        Dft<4>::run(o);
        o[1] = w16mul<2>(o[1]);
        o[2] = w16mul<4>(o[2]);
        o[3] = w16mul<6>(o[3]);
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            v[k] = cadd(e[k], o[k]);
            v[k + 4] = csub(e[k], o[k]);
        }
    }
};

template <> struct Dft<16>
{
    // 16 = 4 x 4: DFT4 over n1 for each n2 (x[4 n1 + n2]), twiddle W_16^{n2 k1}, DFT4 over n2 -> y[k1 + 4 k2].
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        C a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2)
        {
#pragma unroll
            for (int n1 = 0; n1 < 4; ++n1)
                a[n2][n1] = v[4 * n1 + n2];
            Dft<4>::run(a[n2]);
        }
        a[1][1] = w16mul<1>(a[1][1]);
        a[1][2] = w16mul<2>(a[1][2]);
        a[1][3] = w16mul<3>(a[1][3]);
        a[2][1] = w16mul<2>(a[2][1]);
        a[2][2] = w16mul<4>(a[2][2]);
        a[2][3] = w16mul<6>(a[2][3]);
        a[3][1] = w16mul<3>(a[3][1]);
        a[3][2] = w16mul<6>(a[3][2]);
        a[3][3] = w16mul<9>(a[3][3]);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1)
        {
            C b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            Dft<4>::run(b);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2)
                v[k1 + 4 * k2] = b[k2];
        }
    }
};

// Multiply by the compile-time root W_32^J = cos(πJ/16) - i sin(πJ/16): the even J through W_16, the odd J from the
// two first-octant pairs (cos, sin)(π/16) and (cos, sin)(3π/16) by the symmetries of the circle.
template <int J, class C> __device__ __forceinline__ C w32mul(C a)
{
    constexpr int j = J & 31;
    if constexpr ((j & 1) == 0)
        return w16mul<j / 2>(a);
    else
    {
        constexpr float C1 = 0.98078528040323044913f; // cos(π/16)
        constexpr float S1 = 0.19509032201612826785f; // sin(π/16)
        constexpr float C3 = 0.83146961230254523708f; // cos(3π/16)
        constexpr float S3 = 0.55557023301960222474f; // sin(3π/16)
        // cos(πj/16), sin(πj/16) for odd j in [1, 31]
        constexpr float c = j == 1 ? C1 : j == 3 ? C3 : j == 5 ? S3 : j == 7 ? S1 : j == 9 ? -S1 : j == 11 ? -S3
                          : j == 13 ? -C3 : j == 15 ? -C1 : j == 17 ? -C1 : j == 19 ? -C3 : j == 21 ? -S3
                          : j == 23 ? -S1 : j == 25 ? S1 : j == 27 ? S3 : j == 29 ? C3 : C1;
        constexpr float s = j == 1 ? S1 : j == 3 ? S3 : j == 5 ? C3 : j == 7 ? C1 : j == 9 ? C1 : j == 11 ? C3
                          : j == 13 ? S3 : j == 15 ? S1 : j == 17 ? -S1 : j == 19 ? -S3 : j == 21 ? -C3
                          : j == 23 ? -C1 : j == 25 ? -C1 : j == 27 ? -C3 : j == 29 ? -S3 : -S1;
        return crot(a, c, s);
    }
}

template <> struct Dft<32>
{
    // 32 = 2 x 16: E = DFT16 of the even points, O = DFT16 of the odd points, y[k] = E[k] + W_32^k O[k] and
    // y[k + 16] = E[k] - W_32^k O[k] (k < 16).
    template <int K, class C> __device__ __forceinline__ static void combine(C* v, const C* e, const C* o)
    {
        if constexpr (K < 16)
        {
            const C t = w32mul<K>(o[K]);
            v[K] = cadd(e[K], t);
            v[K + 16] = csub(e[K], t);
            combine<K + 1>(v, e, o);
        }
    }
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        C e[16], o[16];
#pragma unroll
        for (int m = 0; m < 16; ++m)
        {
            e[m] = v[2 * m];
            o[m] = v[2 * m + 1];
        }
        Dft<16>::run(e);
        Dft<16>::run(o);
        combine<0>(v, e, o);
    }
};

// Odd prime radix p in {3, 5, 7}: with a_k = x_k + x_{p-k}, b_k = x_k - x_{p-k} (k = 1 .. h, h = (p-1)/2),
//   y_m     = x_0 + sum_k cos(2πkm/p) a_k - i sum_k sin(2πkm/p) b_k
//   y_{p-m} = x_0 + sum_k cos(2πkm/p) a_k + i sum_k sin(2πkm/p) b_k.
template <int P> struct OddRoots;
template <> struct OddRoots<3>
{
    __device__ __forceinline__ static float c(int j) { return -0.5f; }
    __device__ __forceinline__ static float s(int j) { return j == 1 ? 0.86602540378443864676f : -0.86602540378443864676f; }
};
template <> struct OddRoots<5>
{
    __device__ __forceinline__ static float c(int j)
    {
        return (j == 1 || j == 4) ? 0.30901699437494742410f : -0.80901699437494742410f;
    }
    __device__ __forceinline__ static float s(int j)
    {
        return j == 1 ? 0.95105651629515357212f
             : j == 2 ? 0.58778525229247312917f
             : j == 3 ? -0.58778525229247312917f
                      : -0.95105651629515357212f;
    }
};
template <> struct OddRoots<7>
{
    __device__ __forceinline__ static float c(int j)
    {
        return (j == 1 || j == 6) ? 0.62348980185873353053f
             : (j == 2 || j == 5) ? -0.22252093395631440429f
                                  : -0.90096886790241912624f;
    }
    __device__ __forceinline__ static float s(int j)
    {
        return j == 1 ? 0.78183148246802980871f
             : j == 2 ? 0.97492791218182360702f
             : j == 3 ? 0.43388373911755812048f
             : j == 4 ? -0.43388373911755812048f
             : j == 5 ? -0.97492791218182360702f
                      : -0.78183148246802980871f;
    }
};

template <int P> struct OddDft
{
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        constexpr int h = (P - 1) / 2;
        C a[h + 1], b[h + 1];
        C y0 = v[0];
#pragma unroll
        for (int k = 1; k <= h; ++k)
        {
            a[k] = cadd(v[k], v[P - k]);
            b[k] = csub(v[k], v[P - k]);
            y0 = cadd(y0, a[k]);
        }
        C out[P];
        out[0] = y0;
#pragma unroll
        for (int m = 1; m <= h; ++m)
        {
            C re = v[0];
            C im = czero<C>();
#pragma unroll
            for (int k = 1; k <= h; ++k)
            {
                re = cmadd(re, a[k], OddRoots<P>::c((k * m) % P));
                im = cmadd(im, b[k], OddRoots<P>::s((k * m) % P));
            }
            out[m] = add_mi(re, im);
            out[P - m] = sub_mi(re, im);
        }
#pragma unroll
        for (int k = 0; k < P; ++k)
            v[k] = out[k];
    }
};

template <> struct Dft<3> : OddDft<3>
{
};
template <> struct Dft<5> : OddDft<5>
{
};
template <> struct Dft<7> : OddDft<7>
{
};

// Multiply by the compile-time root W_25^J (forward sign), J = n2 k1 for n2, k1 in 1..4: cos/sin of 2πJ/25.
template <int J, class C> __device__ __forceinline__ C w25mul(C a)
{
    static_assert(J == 1 || J == 2 || J == 3 || J == 4 || J == 6 || J == 8 || J == 9 || J == 12 || J == 16,
                  "the products n2 k1 of the 5 x 5 split");
    constexpr float c = J == 1 ? 0.9685831611286311f
                          : J == 2 ? 0.8763066800438636f
                          : J == 3 ? 0.7289686274214116f
                          : J == 4 ? 0.5358267949789965f
                          : J == 6 ? 0.06279051952931353f
                          : J == 8 ? -0.4257792915650727f
                          : J == 9 ? -0.6374239897486897f
                          : J == 12 ? -0.9921147013144778f
                                   : -0.6374239897486895f; // J == 16
    constexpr float s = J == 1 ? 0.2486898871648548f
                          : J == 2 ? 0.4817536741017153f
                          : J == 3 ? 0.6845471059286886f
                          : J == 4 ? 0.8443279255020151f
                          : J == 6 ? 0.9980267284282716f
                          : J == 8 ? 0.9048270524660195f
                          : J == 9 ? 0.7705132427757893f
                          : J == 12 ? 0.12533323356430454f
                                   : -0.7705132427757894f; // J == 16
    return crot(a, c, s);
}

// 25 = 5 x 5: DFT5 over n1 for each n2 (x[5 n1 + n2]), twiddle W_25^{n2 k1}, DFT5 over n2 -> y[k1 + 5 k2].
template <int N2, class C> __device__ __forceinline__ void w25row(C* a)
{
    if constexpr (N2 > 0)
    {
        a[1] = w25mul<N2 * 1>(a[1]);
        a[2] = w25mul<N2 * 2>(a[2]);
        a[3] = w25mul<N2 * 3>(a[3]);
        a[4] = w25mul<N2 * 4>(a[4]);
    }
}

// Multiply by the compile-time root W_9^J (forward sign) for J in {1, 2, 4}: cos/sin of 2πJ/9.
template <int J, class C> __device__ __forceinline__ C w9mul(C a)
{
    constexpr float c = J == 1 ? 0.76604444311897804f : J == 2 ? 0.17364817766693041f : -0.93969262078590832f;
    constexpr float s = J == 1 ? 0.64278760968653933f : J == 2 ? 0.98480775301220802f : 0.34202014332566888f;
    return crot(a, c, s);
}

template <> struct Dft<25>
{
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        C a[5][5];
#pragma unroll
        for (int n2 = 0; n2 < 5; ++n2)
        {
#pragma unroll
            for (int n1 = 0; n1 < 5; ++n1)
                a[n2][n1] = v[5 * n1 + n2];
            Dft<5>::run(a[n2]);
        }
        w25row<1>(a[1]);
        w25row<2>(a[2]);
        w25row<3>(a[3]);
        w25row<4>(a[4]);
#pragma unroll
        for (int k1 = 0; k1 < 5; ++k1)
        {
            C b[5] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1], a[4][k1]};
            Dft<5>::run(b);
#pragma unroll
            for (int k2 = 0; k2 < 5; ++k2)
                v[k1 + 5 * k2] = b[k2];
        }
    }
};

// 9 = 3 x 3: DFT3 over n1 for each n2 (x[3 n1 + n2]), twiddle W_9^{n2 k1}, DFT3 over n2 -> y[k1 + 3 k2]. One stage of
// radix 9 replaces two stages of radix 3 (one exchange through shared memory fewer) for lengths with 3^2 as a factor.
template <> struct Dft<9>
{
    template <class C> __device__ __forceinline__ static void run(C* v)
    {
        C a[3][3];
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2)
        {
#pragma unroll
            for (int n1 = 0; n1 < 3; ++n1)
                a[n2][n1] = v[3 * n1 + n2];
            Dft<3>::run(a[n2]);
        }
        a[1][1] = w9mul<1>(a[1][1]);
        a[1][2] = w9mul<2>(a[1][2]);
        a[2][1] = w9mul<2>(a[2][1]);
        a[2][2] = w9mul<4>(a[2][2]);
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1)
        {
            C b[3] = {a[0][k1], a[1][k1], a[2][k1]};
            Dft<3>::run(b);
#pragma unroll
            for (int k2 = 0; k2 < 3; ++k2)
                v[k1 + 3 * k2] = b[k2];
        }
    }
};

} // namespace crdfft
