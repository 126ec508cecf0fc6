/*
 * TEST INFRASTRUCTURE ONLY - the CPU oracle of the GPU FFT path (see oracle.h). Never linked into the product.
 *
 * Restatements, in plain C, of the reference's FFT algorithms (yatiyr/CRD engine/numerics/hesap-fft). Each function
 * names the reference file:line it follows. Compiled with -ffp-contract=off, as the reference's kernel units are
 * (cmake/CrdSimd.cmake:496-498), so the f32 radix-2 restatement rounds like the reference's.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static const long double kQuarterPi = 0.78539816339744830961566084581987572L;

/* exp(-2πi k/n) in extended precision, the angle reduced exactly to at most π/4 (k mod n, octant of 8k/n) so that
 * quarter points are exact. */
static void root(uint64_t k, uint64_t n, double* re, double* im)
{
    k %= n;
    const unsigned __int128 num = (unsigned __int128)k * 8u;
    const uint64_t oct = (uint64_t)(num / n);
    const uint64_t rem = (uint64_t)(num - (unsigned __int128)oct * n);
    long double c, s;
    uint64_t quarters;
    if ((oct & 1u) == 0)
    {
        const long double th = kQuarterPi * (long double)rem / (long double)n;
        c = cosl(th);
        s = sinl(th);
        quarters = oct / 2;
    }
    else
    {
        const long double th = kQuarterPi * (long double)(n - rem) / (long double)n;
        c = cosl(th);
        s = -sinl(th);
        quarters = (oct + 1) / 2;
    }
    long double cr, sr;
    switch (quarters & 3u)
    {
        case 0: cr = c; sr = s; break;
        case 1: cr = -s; sr = c; break;
        case 2: cr = -c; sr = -s; break;
        default: cr = s; sr = -c; break;
    }
    *re = (double)cr;
    *im = (double)(-sr);
}

/* ---- inputs (tests/numerics/hesap-fft/test_fft.cpp:31-44) ---------------------------------------------------- */

static double lcg_next(uint64_t* s)
{
    *s = *s * 6364136223846793005ULL + 1442695040888963407ULL;
    return ((double)(*s >> 11) / (double)(1ULL << 53)) * 2.0 - 1.0;
}

void orc_lcg_fill_f64(uint64_t seed, size_t count, double* out)
{
    uint64_t s = seed;
    for (size_t i = 0; i < count; ++i)
        out[i] = lcg_next(&s);
}

void orc_lcg_fill_f32(uint64_t seed, size_t count, float* out)
{
    uint64_t s = seed;
    for (size_t i = 0; i < count; ++i)
        out[i] = (float)lcg_next(&s);
}

void orc_gauss_fill_f32(uint64_t seed, size_t count, float* out)
{
    uint64_t s = seed;
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t i = 0; i < count; i += 2)
    {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        const double u1 = ((double)(s >> 11) + 1.0) / (double)(1ULL << 53); /* (0, 1] */
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        const double u2 = (double)(s >> 11) / (double)(1ULL << 53);
        const double r = sqrt(-2.0 * log(u1));
        out[i] = (float)(r * cos(two_pi * u2));
        if (i + 1 < count)
            out[i + 1] = (float)(r * sin(two_pi * u2));
    }
}

/* ---- brute-force DFT (test_fft.cpp:47-65) --------------------------------------------------------------------- */

void orc_naive_dft(size_t n, const double* x, double* y, int dir)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double sgn = dir ? 1.0 : -1.0;
    for (size_t k = 0; k < n; ++k)
    {
        double re = 0.0, im = 0.0;
        for (size_t j = 0; j < n; ++j)
        {
            const double ang = sgn * two_pi * (double)((j * k) % n) / (double)n;
            const double c = cos(ang), sn = sin(ang);
            re += x[2 * j] * c - x[2 * j + 1] * sn;
            im += x[2 * j] * sn + x[2 * j + 1] * c;
        }
        y[2 * k] = re;
        y[2 * k + 1] = im;
    }
}

/* ---- FP64 mixed-radix self-sorting FFT ------------------------------------------------------------------------ */
/* The reference's production engine is a Stockham autosort (fft.hpp:9-11; kernels/fft_kernels.cpp:266-353); this is
 * the same self-sorting DIT schedule with a generic radix p per stage:
 *   y[(j - k) p + k + s L] = sum_r (x[j + r n/p] W_{Lp}^{r k}) W_p^{r s},  k = j mod L. */

static int factorize(size_t n, size_t* f)
{
    int c = 0;
    static const size_t pref[] = {4, 2, 3, 5, 7};
    size_t m = n;
    for (int i = 0; i < 5; ++i)
        while (m % pref[i] == 0 && !(pref[i] == 4 && m == 2))
        {
            f[c++] = pref[i];
            m /= pref[i];
        }
    for (size_t p = 11; p * p <= m; p += 2)
        while (m % p == 0)
        {
            f[c++] = p;
            m /= p;
        }
    if (m > 1)
        f[c++] = m;
    return c;
}

int orc_fft_f64(size_t n, const double* x, double* y, int dir)
{
    if (n == 0)
        return -1;
    if (n == 1)
    {
        y[0] = x[0];
        y[1] = x[1];
        return 0;
    }
    size_t fac[64];
    const int nf = factorize(n, fac);
    double* tw = (double*)malloc(sizeof(double) * 2 * n);
    double* a = (double*)malloc(sizeof(double) * 2 * n);
    double* b = (double*)malloc(sizeof(double) * 2 * n);
    size_t maxp = 0;
    for (int i = 0; i < nf; ++i)
        maxp = fac[i] > maxp ? fac[i] : maxp;
    double* v = (double*)malloc(sizeof(double) * 2 * maxp);
    if (!tw || !a || !b || !v)
    {
        free(tw);
        free(a);
        free(b);
        free(v);
        return -2;
    }
    const double sg = dir ? -1.0 : 1.0; /* inverse: conjugate roots */
    for (size_t k = 0; k < n; ++k)
    {
        root(k, n, &tw[2 * k], &tw[2 * k + 1]);
        tw[2 * k + 1] *= sg;
    }
    memcpy(a, x, sizeof(double) * 2 * n);
    size_t L = 1;
    for (int s = 0; s < nf; ++s)
    {
        const size_t p = fac[s];
        const size_t nb = n / p;
        const size_t m = n / (L * p);
        for (size_t j = 0; j < nb; ++j)
        {
            const size_t k = j % L;
            for (size_t r = 0; r < p; ++r)
            {
                const double xr = a[2 * (j + r * nb)], xi = a[2 * (j + r * nb) + 1];
                const size_t t = (r * k * m) % n;
                const double wr = tw[2 * t], wi = tw[2 * t + 1];
                v[2 * r] = xr * wr - xi * wi;
                v[2 * r + 1] = xr * wi + xi * wr;
            }
            const size_t base = (j - k) * p + k;
            for (size_t q = 0; q < p; ++q)
            {
                double sr = 0.0, si = 0.0;
                for (size_t r = 0; r < p; ++r)
                {
                    const size_t t = ((r * q) % p) * nb;
                    const double wr = tw[2 * t], wi = tw[2 * t + 1];
                    sr += v[2 * r] * wr - v[2 * r + 1] * wi;
                    si += v[2 * r] * wi + v[2 * r + 1] * wr;
                }
                b[2 * (base + q * L)] = sr;
                b[2 * (base + q * L) + 1] = si;
            }
        }
        double* t = a;
        a = b;
        b = t;
        L *= p;
    }
    memcpy(y, a, sizeof(double) * 2 * n);
    free(tw);
    free(a);
    free(b);
    free(v);
    return 0;
}

struct batch_job
{
    size_t n, first, last;
    const double* x;
    double* y;
    int dir;
    int rc;
};

static void* batch_worker(void* arg)
{
    struct batch_job* j = (struct batch_job*)arg;
    j->rc = 0;
    for (size_t t = j->first; t < j->last; ++t)
    {
        const int rc = orc_fft_f64(j->n, j->x + 2 * t * j->n, j->y + 2 * t * j->n, j->dir);
        if (rc != 0)
            j->rc = rc;
    }
    return NULL;
}

int orc_fft_batch_f64(size_t n, size_t batch, const double* x, double* y, int dir, int threads)
{
    if (threads < 1)
        threads = 1;
    if ((size_t)threads > batch)
        threads = (int)(batch ? batch : 1);
    pthread_t th[256];
    struct batch_job jobs[256];
    if (threads > 256)
        threads = 256;
    for (int i = 0; i < threads; ++i)
    {
        jobs[i].n = n;
        jobs[i].first = batch * (size_t)i / (size_t)threads;
        jobs[i].last = batch * (size_t)(i + 1) / (size_t)threads;
        jobs[i].x = x;
        jobs[i].y = y;
        jobs[i].dir = dir;
        pthread_create(&th[i], NULL, batch_worker, &jobs[i]);
    }
    int rc = 0;
    for (int i = 0; i < threads; ++i)
    {
        pthread_join(th[i], NULL);
        if (jobs[i].rc != 0)
            rc = jobs[i].rc;
    }
    return rc;
}

/* ---- FftPlan<T>::execute_reference (fft.hpp:251-260 table, 417-460 transform) ---------------------------------- */

static int is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; }

static size_t bitrev(size_t i, unsigned lg)
{
    size_t r = 0;
    for (unsigned b = 0; b < lg; ++b)
        if (i & ((size_t)1 << b))
            r |= (size_t)1 << (lg - 1 - b);
    return r;
}

#define DEFINE_EXECUTE_REFERENCE(NAME, T)                                                                              \
    int NAME(size_t n, T* data, int dir)                                                                               \
    {                                                                                                                  \
        if (!is_pow2(n))                                                                                               \
            return -1;                                                                                                 \
        if (n <= 1)                                                                                                    \
            return 0;                                                                                                  \
        unsigned lg = 0;                                                                                               \
        while (((size_t)1 << lg) < n)                                                                                  \
            ++lg;                                                                                                      \
        T* twr = (T*)malloc(sizeof(T) * n);                                                                            \
        T* twi = (T*)malloc(sizeof(T) * n);                                                                            \
        if (!twr || !twi)                                                                                              \
        {                                                                                                              \
            free(twr);                                                                                                 \
            free(twi);                                                                                                 \
            return -2;                                                                                                 \
        }                                                                                                              \
        const double two_pi = 6.283185307179586476925286766559;                                                        \
        for (size_t k = 0; k < n; ++k)                                                                                 \
        {                                                                                                              \
            const double ang = -two_pi * (double)k / (double)n;                                                        \
            twr[k] = (T)cos(ang);                                                                                      \
            twi[k] = (T)sin(ang);                                                                                      \
        }                                                                                                              \
        for (size_t i = 0; i < n; ++i)                                                                                 \
        {                                                                                                              \
            const size_t j = bitrev(i, lg);                                                                            \
            if (i < j)                                                                                                 \
            {                                                                                                          \
                T tr = data[2 * i], ti = data[2 * i + 1];                                                              \
                data[2 * i] = data[2 * j];                                                                             \
                data[2 * i + 1] = data[2 * j + 1];                                                                     \
                data[2 * j] = tr;                                                                                      \
                data[2 * j + 1] = ti;                                                                                  \
            }                                                                                                          \
        }                                                                                                              \
        const T isign = dir ? (T)-1 : (T)1;                                                                            \
        for (size_t len = 2; len <= n; len <<= 1)                                                                      \
        {                                                                                                              \
            const size_t half = len >> 1, step = n / len;                                                              \
            for (size_t base = 0; base < n; base += len)                                                               \
            {                                                                                                          \
                size_t tw = 0;                                                                                         \
                for (size_t k = 0; k < half; ++k)                                                                      \
                {                                                                                                      \
                    const T wr = twr[tw];                                                                              \
                    const T wi = isign * twi[tw];                                                                      \
                    T* a = data + 2 * (base + k);                                                                      \
                    T* b = data + 2 * (base + k + half);                                                               \
                    const T vr = wr * b[0] - wi * b[1];                                                                \
                    const T vi = wr * b[1] + wi * b[0];                                                                \
                    const T ar = a[0], ai = a[1];                                                                      \
                    a[0] = ar + vr;                                                                                    \
                    a[1] = ai + vi;                                                                                    \
                    b[0] = ar - vr;                                                                                    \
                    b[1] = ai - vi;                                                                                    \
                    tw += step;                                                                                        \
                }                                                                                                      \
            }                                                                                                          \
        }                                                                                                              \
        free(twr);                                                                                                     \
        free(twi);                                                                                                     \
        return 0;                                                                                                      \
    }

DEFINE_EXECUTE_REFERENCE(orc_execute_reference_f32, float)
DEFINE_EXECUTE_REFERENCE(orc_execute_reference_f64, double)

/* ---- BluesteinPlan<double>::execute (bluestein.hpp:29-136) ------------------------------------------------------ */

int orc_bluestein_f64(size_t n, double* x, int dir)
{
    if (n < 1)
        return -1;
    size_t m = 1;
    while (m < 2 * n - 1)
        m <<= 1;
    double* chirp = (double*)malloc(sizeof(double) * 2 * n);
    double* bf = (double*)calloc(2 * m, sizeof(double));
    double* w = (double*)calloc(2 * m, sizeof(double));
    if (!chirp || !bf || !w)
    {
        free(chirp);
        free(bf);
        free(w);
        return -2;
    }
    /* chirp[k] = exp(+iπ k²/n) with k² reduced mod 2n (bluestein.hpp:47-53); exp(+iπ q/n) = conj(W_{2n}^q). */
    for (size_t k = 0; k < n; ++k)
    {
        const uint64_t kk = (uint64_t)(((unsigned __int128)k * k) % (2 * (uint64_t)n));
        double re, im;
        root(kk, 2 * (uint64_t)n, &re, &im);
        chirp[2 * k] = re;
        chirp[2 * k + 1] = -im;
    }
    /* b_circ: b[0] = chirp[0], b[k] = b[m-k] = chirp[k]; FFT_m(b) (bluestein.hpp:57-71). */
    bf[0] = chirp[0];
    bf[1] = chirp[1];
    for (size_t k = 1; k < n; ++k)
    {
        bf[2 * k] = chirp[2 * k];
        bf[2 * k + 1] = chirp[2 * k + 1];
        bf[2 * (m - k)] = chirp[2 * k];
        bf[2 * (m - k) + 1] = chirp[2 * k + 1];
    }
    orc_fft_f64(m, bf, bf, 0);
    const int inv = dir != 0;
    for (size_t k = 0; k < n; ++k) /* a = x conj(chirp), x conjugated first for the inverse (:95-103) */
    {
        const double xr = x[2 * k], xi = inv ? -x[2 * k + 1] : x[2 * k + 1];
        const double cr = chirp[2 * k], ci = chirp[2 * k + 1];
        w[2 * k] = xr * cr + xi * ci;
        w[2 * k + 1] = xi * cr - xr * ci;
    }
    orc_fft_f64(m, w, w, 0);
    for (size_t k = 0; k < m; ++k) /* C = A FFT_m(b) (:109-116) */
    {
        const double ar = w[2 * k], ai = w[2 * k + 1], br = bf[2 * k], bi = bf[2 * k + 1];
        w[2 * k] = ar * br - ai * bi;
        w[2 * k + 1] = ar * bi + ai * br;
    }
    orc_fft_f64(m, w, w, 1);
    const double cm = 1.0 / (double)m;
    for (size_t k = 0; k < n; ++k) /* X = conj(chirp) c / m; inverse: conj and 1/n (:121-134) */
    {
        const double cr = chirp[2 * k], ci = chirp[2 * k + 1];
        double yr = (w[2 * k] * cr + w[2 * k + 1] * ci) * cm;
        double yi = (w[2 * k + 1] * cr - w[2 * k] * ci) * cm;
        if (inv)
        {
            const double s = 1.0 / (double)n;
            yr *= s;
            yi = -yi * s;
        }
        x[2 * k] = yr;
        x[2 * k + 1] = yi;
    }
    free(chirp);
    free(bf);
    free(w);
    return 0;
}

/* ---- RealFftPlan<double> (real_fft.hpp:21-92) ------------------------------------------------------------------ */

int orc_rfft_f64(size_t n, const double* x, double* y)
{
    if (n < 2 || (n & 1u))
        return -1;
    const size_t h = n / 2;
    double* z = (double*)malloc(sizeof(double) * 2 * h);
    if (!z)
        return -2;
    memcpy(z, x, sizeof(double) * n); /* z[j] = x[2j] + i x[2j+1] (:47-50) */
    orc_fft_f64(h, z, z, 0);
    for (size_t k = 0; k <= h; ++k) /* recombine (:52-63) */
    {
        const double zkr = z[2 * (k % h)], zki = z[2 * (k % h) + 1];
        const double znr = z[2 * ((h - k) % h)], zni = z[2 * ((h - k) % h) + 1];
        const double er = (zkr + znr) * 0.5, ei = (zki - zni) * 0.5;
        const double orr = (zki + zni) * 0.5, oii = (znr - zkr) * 0.5;
        double wr, wi;
        root(k, n, &wr, &wi);
        y[2 * k] = er + (wr * orr - wi * oii);
        y[2 * k + 1] = ei + (wr * oii + wi * orr);
    }
    free(z);
    return 0;
}

int orc_irfft_f64(size_t n, const double* x, double* y)
{
    if (n < 2 || (n & 1u))
        return -1;
    const size_t h = n / 2;
    double* z = (double*)malloc(sizeof(double) * 2 * h);
    if (!z)
        return -2;
    for (size_t k = 0; k < h; ++k) /* inverse recombine (:72-84) */
    {
        const double xkr = x[2 * k], xki = x[2 * k + 1];
        const double xhr = x[2 * (h - k)], xhi = x[2 * (h - k) + 1];
        const double er = (xkr + xhr) * 0.5, ei = (xki - xhi) * 0.5;
        const double dr = (xkr - xhr) * 0.5, di = (xki + xhi) * 0.5;
        double wr, wi;
        root(k, n, &wr, &wi);
        const double orr = wr * dr + wi * di, oii = wr * di - wi * dr;
        z[2 * k] = er - oii;
        z[2 * k + 1] = ei + orr;
    }
    orc_fft_f64(h, z, z, 1);
    const double inv = 1.0 / (double)h; /* (:86-91) */
    for (size_t j = 0; j < h; ++j)
    {
        y[2 * j] = z[2 * j] * inv;
        y[2 * j + 1] = z[2 * j + 1] * inv;
    }
    free(z);
    return 0;
}

/* ---- NdFftPlan<double>::execute (nd_fft.hpp:105-182) ---------------------------------------------------------- */

int orc_nd_f64(size_t ndim, const size_t* dims, double* x, int dir)
{
    if (ndim < 1)
        return -1;
    size_t total = 1, maxd = 1;
    for (size_t i = 0; i < ndim; ++i)
    {
        total *= dims[i];
        maxd = dims[i] > maxd ? dims[i] : maxd;
    }
    const int inv = dir != 0;
    if (inv)
        for (size_t i = 0; i < total; ++i)
            x[2 * i + 1] = -x[2 * i + 1];
    double* line = (double*)malloc(sizeof(double) * 2 * maxd);
    if (!line)
        return -2;
    size_t stride = 1;
    for (size_t ax = ndim; ax-- > 0;)
    {
        const size_t d = dims[ax];
        if (d >= 2)
        {
            const size_t lines = total / d;
            for (size_t l = 0; l < lines; ++l) /* transform_lines (:156-182) */
            {
                const size_t base = (l / stride) * d * stride + l % stride;
                for (size_t i = 0; i < d; ++i)
                {
                    line[2 * i] = x[2 * (base + i * stride)];
                    line[2 * i + 1] = x[2 * (base + i * stride) + 1];
                }
                orc_fft_f64(d, line, line, 0);
                for (size_t i = 0; i < d; ++i)
                {
                    x[2 * (base + i * stride)] = line[2 * i];
                    x[2 * (base + i * stride) + 1] = line[2 * i + 1];
                }
            }
        }
        stride *= d;
    }
    if (inv) /* conj and 1/prod(dims) (:138-146) */
    {
        const double s = 1.0 / (double)total;
        for (size_t i = 0; i < total; ++i)
        {
            x[2 * i] *= s;
            x[2 * i + 1] = -x[2 * i + 1] * s;
        }
    }
    free(line);
    return 0;
}

/* ---- metrics ---------------------------------------------------------------------------------------------------- */

double orc_rel_l2_f32(size_t count, const float* a, const double* b)
{
    long double num = 0.0L, den = 0.0L;
    for (size_t i = 0; i < 2 * count; ++i)
    {
        const long double d = (long double)a[i] - (long double)b[i];
        num += d * d;
        den += (long double)b[i] * (long double)b[i];
    }
    return den > 0.0L ? (double)sqrtl(num / den) : (double)sqrtl(num);
}

double orc_max_rel_f32(size_t count, const float* a, const double* b)
{
    double maxref = 0.0, maxerr = 0.0;
    for (size_t i = 0; i < count; ++i)
    {
        const double r = hypot(b[2 * i], b[2 * i + 1]);
        maxref = r > maxref ? r : maxref;
        const double e = hypot((double)a[2 * i] - b[2 * i], (double)a[2 * i + 1] - b[2 * i + 1]);
        maxerr = e > maxerr ? e : maxerr;
    }
    return maxerr / (1.0 + maxref);
}
