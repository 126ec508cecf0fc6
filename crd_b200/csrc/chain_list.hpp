// The work list of the one-launch four-step (chain_fft.cu), shared by the kernel and the host-side checks: which
// tile a list position names, and which earlier tiles it waits for. Plain integer arithmetic, no CUDA types.
//
// For W waves of C column tiles and R row tiles each, with row tiles trailing by `lag` waves:
//     col(0) .. col(lag-1) | col(lag) row(0) | col(lag+1) row(1) | ... | col(W-1+lag) row(W-1)
// where the column tiles of waves >= W are no-ops. A row tile of wave w waits for the C column tiles of wave w; a
// column tile of wave w >= slots waits for the R row tiles of wave w - slots (its intermediate slot).

#pragma once

#ifdef __CUDACC__
#define CRDFFT_HD __host__ __device__ __forceinline__
#else
#define CRDFFT_HD inline
#endif

namespace crdfft
{

struct ChainTile
{
    bool col;  // a column tile (else a row tile)
    int wave;  // its wave (>= W: a no-op column tile)
    int idx;   // the tile within its wave's pass
};

// The tile at list position t (0 <= t < chain_list_length).
CRDFFT_HD ChainTile chain_tile_at(int t, int C, int R, int lag)
{
    const int head = lag * C;
    if (t < head)
    {
        const int w = t / C;
        return ChainTile{true, w, t - w * C};
    }
    const int u = t - head;
    const int sg = u / (C + R);
    const int r = u - sg * (C + R);
    return r < C ? ChainTile{true, sg + lag, r} : ChainTile{false, sg, r - C};
}

CRDFFT_HD long long chain_list_length(long long W, long long C, long long R, int lag)
{
    return lag * C + W * (C + R);
}

// Threads of a chained CTA, and the lines of an n-point pass one tile holds (16 points a thread).
inline constexpr int kChainThreads = 256;
CRDFFT_HD int chain_lines_per_tile(int n) { return kChainThreads / ((n + 15) / 16); }

// How far a wave's row tiles trail its column tiles, for `slots` intermediate slots (3 or more): half of them, so
// that both waits point at least two list segments back. (With slots - 1, a column tile that refills a slot waited
// on row tiles claimed just before it: a stall every wave.)
CRDFFT_HD int chain_lag(int slots) { return slots / 2; }

} // namespace crdfft
