// Host check of the one-launch four-step's work list (crd_b200/csrc/chain_list.hpp): over the list, every column
// and row tile of every wave appears exactly once, only column tiles past the last wave are no-ops, and every tile a
// tile waits for sits earlier in the list (the condition that lets the list drain whatever CTAs are resident). With
// the planner's lag rule and four or more slots, each wait also points at least one whole list segment back.
// Prints "chain list ok" and exits 0, or names the first broken case and exits 1.

#include "chain_list.hpp"

#include <cstdio>
#include <vector>

using crdfft::chain_lag;
using crdfft::chain_lines_per_tile;
using crdfft::chain_list_length;
using crdfft::chain_tile_at;
using crdfft::ChainTile;

namespace
{

struct Case
{
    long long n1, n2, batch, wave_t;
    int slots;
};

bool check(const Case& k)
{
    const long long C = (k.wave_t * k.n2 + chain_lines_per_tile(k.n1) - 1) / chain_lines_per_tile(k.n1);
    const long long R = (k.wave_t * k.n1 + chain_lines_per_tile(k.n2) - 1) / chain_lines_per_tile(k.n2);
    const long long W = (k.batch + k.wave_t - 1) / k.wave_t;
    const int lag = chain_lag(k.slots);
    const long long len = chain_list_length(W, C, R, lag);
    std::vector<long long> col_pos(W * C, -1), row_pos(W * R, -1);
    for (long long t = 0; t < len; ++t)
    {
        const ChainTile c = chain_tile_at(static_cast<int>(t), static_cast<int>(C), static_cast<int>(R), lag);
        if (c.wave >= W)
        {
            if (!c.col)
                return false; // only column tiles may fall past the last wave
            continue;
        }
        std::vector<long long>& pos = c.col ? col_pos : row_pos;
        const long long slot = c.wave * (c.col ? C : R) + c.idx;
        if (c.idx < 0 || c.idx >= (c.col ? C : R) || pos[slot] != -1)
            return false;
        pos[slot] = t;
    }
    for (long long v : col_pos)
        if (v < 0)
            return false;
    for (long long v : row_pos)
        if (v < 0)
            return false;
    const long long need = k.slots >= 4 ? C + R : 1; // at least one whole segment between, or just earlier
    for (long long w = 0; w < W; ++w)
    {
        long long last_col = -1, first_row = len, first_col = len, last_prev_row = -1;
        for (long long i = 0; i < C; ++i)
        {
            last_col = col_pos[w * C + i] > last_col ? col_pos[w * C + i] : last_col;
            first_col = col_pos[w * C + i] < first_col ? col_pos[w * C + i] : first_col;
        }
        for (long long i = 0; i < R; ++i)
            first_row = row_pos[w * R + i] < first_row ? row_pos[w * R + i] : first_row;
        if (first_row - last_col < need) // a row tile waits for all of its wave's column tiles
            return false;
        if (w >= k.slots)
        {
            for (long long i = 0; i < R; ++i)
            {
                const long long p = row_pos[(w - k.slots) * R + i];
                last_prev_row = p > last_prev_row ? p : last_prev_row;
            }
            if (first_col - last_prev_row < need) // a column tile waits for the row tiles that used its slot
                return false;
        }
    }
    return true;
}

} // namespace

int main()
{
    // (n1, n2, batch, transforms a wave, slots): the bench's 107520 and 2^20 batches at 16 MiB waves, the parity
    // tests' shapes, a single wave, and partial last waves
    const Case cases[] = {
        {105, 1024, 2496, 19, 4}, {1024, 1024, 256, 2, 4}, {64, 1024, 4096, 32, 4}, {105, 1024, 64, 19, 4},
        {1024, 1024, 9, 2, 3},    {1024, 512, 20, 4, 3},   {105, 1024, 40, 4, 5},   {512, 1024, 7, 7, 3},
        {105, 1024, 2496, 9, 6},  {64, 1024, 100, 3, 8},
    };
    for (const Case& k : cases)
        if (!check(k))
        {
            std::printf("chain list broken: n1 %lld n2 %lld batch %lld wave %lld slots %d\n", k.n1, k.n2, k.batch,
                        k.wave_t, k.slots);
            return 1;
        }
    std::printf("chain list ok\n");
    return 0;
}
