// fold.cuh -- the reference's sequential double-precision left fold
// s_i = fl(s_{i-1} + x_i), x_i >= 0, reproduced bit for bit in parallel.
//
// The reference accumulates normalising constants and cumulative weights
// with plain `accw += w[i]` loops (core/weight.hpp:221 via std::accumulate,
// algorithm/resample.hpp:395-403, :348-356).  Their results feed the
// resampling search, so an ordinary parallel (tree) sum -- which rounds
// differently -- would move cumulative weights by a few ULPs and flip
// ancestors whose uniform lies in between.  This fold does not.
//
// Why it parallelises: while s stays inside one binade [2^e, 2^(e+1)) every
// partial sum is a multiple of u = ulp(2^e), so
//     s_i = s_{i-1} + u * RN(x_i / u)
// where RN rounds to nearest, ties to the even multiple of u.  Inside a binade
// the fold is therefore an integer prefix sum of per-element increments
// q_i = RN(x_i / u), which every thread computes independently.  Only three
// events break that: the sum leaving the binade, a tie (its direction depends
// on the parity of the running sum), and an increment too large for the grid.
// At an event the single step is done with a real double add, which is the
// reference's own operation.
//
// Parallel structure over tiles of kFoldTile elements:
//   1. k_fold_tilesum / k_fold_scan_tiles: approximate tile sums and their
//      prefix predict each tile's binade, with an error margin;
//   2. k_fold_describe: tiles whose whole range is certainly inside one
//      binade and holds no event get A_t = sum of q_i (a transfer function
//      s -> s + u A_t);
//   3. k_fold_walk (one CTA): chains the exact tile-entry values; certain
//      tiles cost O(1), the others are folded by the CTA with the event loop;
//   4. k_fold_expand: every element of the certain tiles gets
//      s_i = s_entry + u * (prefix of q within the tile).
#pragma once

#include <cstdint>

namespace mckl_b200 {

constexpr int kFoldTile = 4096;

struct FoldDesc {
    int eb;         // biased exponent of the tile's binade (0: subnormal range)
    int flags;      // 1: needs the exact event loop
    long long A;    // sum of rounded increments at that binade
};

__device__ __forceinline__ int biased_exp(double s)
{
    return static_cast<int>((__double_as_longlong(s) >> 52) & 0x7ff);
}

// s / ulp for s's own binade (an integer below 2^53)
__device__ __forceinline__ long long grid_count(double s)
{
    const long long b = __double_as_longlong(s);
    const long long m = b & ((1ll << 52) - 1);
    return ((b >> 52) & 0x7ff) ? (m | (1ll << 52)) : m;
}

__device__ __forceinline__ long long grid_top(int eb)
{
    return eb ? (1ll << 53) : (1ll << 52);
}

__device__ __forceinline__ double grid_unit(int eb)
{
    const int e = (eb ? eb : 1) - 1075;  // u = 2^e, e in [-1074, 972]
    return e >= -1022 ? __longlong_as_double(static_cast<long long>(e + 1023) << 52)
                      : __longlong_as_double(1ll << (e + 1074));
}

__device__ __forceinline__ double from_grid(long long K, int eb)
{
    return __dmul_rn(__ll2double_rn(K), grid_unit(eb));  // exact: K < 2^53, u a power of two
}

// q = RN(x / u) for x >= 0 at the grid of binade eb; `event` when x / u is a
// tie (direction depends on the running sum) or when q would leave the grid.
__device__ __forceinline__ long long grid_increment(double x, int eb, bool &event)
{
    const long long b = __double_as_longlong(x);
    const int ex = static_cast<int>((b >> 52) & 0x7ff);
    long long m = b & ((1ll << 52) - 1);
    if (ex) m |= (1ll << 52);
    event = false;
    if (m == 0) return 0;
    if (ex == 0x7ff) {  // inf / nan: let the real add decide
        event = true;
        return 0;
    }
    const int d = (eb ? eb : 1) - (ex ? ex : 1);  // x / u = m * 2^-d
    if (d <= 0) {
        if (-d >= 10) {
            event = true;
            return 0;
        }
        const long long q = m << (-d);
        if (q >= (1ll << 53)) event = true;
        return q;
    }
    if (d >= 60) return 0;
    long long q = m >> d;
    const long long rem = m & ((1ll << d) - 1);
    const long long half = 1ll << (d - 1);
    if (rem > half) {
        q += 1;
    } else if (rem == half) {
        event = true;
    }
    return q;
}

struct FoldScratch {
    double *tsum;     // [T] approximate tile sums
    double *tpre;     // [T] approximate exclusive prefix of tile sums
    FoldDesc *desc;   // [T]
    double *tstart;   // [T] exact fold value entering each tile
    int *tmode;       // [T] 0: expand from tstart, 1: values already written
    double *final_v;  // [1] the fold's last value
};

// Host driver (fold.cu): folds x[0..n) starting from s0.  `prefix` (device,
// nullable) receives every partial sum; the last one is also left in
// scratch.final_v.  Returns an MCKL_B200_* status.
int fold_exact(const double *x, uint64_t n, double s0, double *prefix, FoldScratch &fs, cudaStream_t s);
size_t fold_scratch_bytes(uint64_t n);
FoldScratch fold_scratch_carve(void *base, uint64_t n);

}  // namespace mckl_b200
