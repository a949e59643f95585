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
// Parallel structure (tiles of kFoldTile elements):
//   1. approximate partial sums A_j (a tree sum) carry a rigorous error bound,
//      so for most elements the binade of the exact partial sum S_j is
//      certain; an element whose S_{j-1} and S_j are certainly in the same
//      binade, with an event-free increment, is a RUN element
//      (S_j = S_{j-1} + u q_j); every other element -- a binade crossing, a
//      tie, an uncertain binade -- is a WINDOW (typically a few dozen per
//      fold: one per doubling of the sum);
//   2. per tile, the run increments are summed and the windows counted; an
//      exclusive scan over tiles places every window in an ordered list with
//      the run-increment prefix before it;
//   3. one thread walks the windows in order: the run before a window is a
//      single integer step on its grid, the window the reference's own
//      double add;
//   4. every partial sum, when asked for, is the value after the window
//      before it plus its run's increments.
// When the windows do not fit their list (inputs with ties everywhere, long
// zero or subnormal stretches) the walk falls back to the event loop: tiles
// certain for their whole length cost O(1) (a transfer function s -> s +
// u A_t), the others are folded by one CTA that handles one event per scan
// round.
#pragma once

#include <cstdint>

namespace mckl_b200 {

constexpr int kFoldTile = 4096;
constexpr unsigned kFoldLocalCap = 32;

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

// The windows of one fold, in order: element index, value, the sum of the run
// increments of the elements before it, the binade of the run before it
// (-1: none), and, after the walk, the fold's value after it.
struct FoldWindows {
    unsigned long long *idx;
    double *x;
    long long *P;
    double *S;
    int *e;
    uint64_t cap;
};

// Per-tile window lists written by the counting pass (capacity `cap` per
// tile, 0: none): the window's offset in its tile, value, the run-increment
// sum before it within the tile, and the binade of the run before it.  A tile
// with at most `cap` windows is placed by copying its list; a fuller one is
// classified again.
struct FoldLocal {
    unsigned *off;
    double *x;
    long long *P;
    int *e;
    unsigned cap;
};

struct FoldScratch {
    double *tsum;     // [T] approximate tile sums
    double *tpre;     // [T] approximate exclusive prefix of tile sums
    double *tpmax;    // [T] tile maxima, then their exclusive prefix maximum
    FoldDesc *desc;   // [T] tile descriptors of the event-loop walk
    double *tstart;   // [T] event-loop walk: exact value entering each tile
    int *tmode;       // [T] event-loop walk: 0 expand from tstart, 1 values already written
    long long *tq;    // [T] sum of the run increments of each tile
    unsigned *tw;     // [T] windows in each tile
    long long *pq;    // [T] exclusive prefix of tq
    unsigned long long *pw;  // [T] exclusive prefix of tw
    long long *tot;   // [2] all run increments, all windows
    int *elast;       // binade of the run holding the last element (-1: it is a window)
    int *mode;        // 0 window walk, 1 event-loop walk
    double *final_v;  // [1] the fold's last value
    FoldWindows win;
    FoldLocal loc;
};

// Host driver (fold.cu): folds x[0..n) starting from s0.  `prefix` (device,
// nullable) receives every partial sum; the last one is also left in
// scratch.final_v.  Returns an MCKL_B200_* status.  `wcap`: capacity of the
// window list (0: fold_window_cap(n)); a fold with more windows than that
// takes the event-loop walk.  The default sizing (wcap 0) also holds per-tile
// window lists of kFoldLocalCap entries; an explicit wcap sizes the scratch
// without them (the tiles with windows are then classified twice).
int fold_exact(const double *x, uint64_t n, double s0, double *prefix, FoldScratch &fs, cudaStream_t s);
uint64_t fold_window_cap(uint64_t n);
size_t fold_scratch_bytes(uint64_t n, uint64_t wcap = 0);
FoldScratch fold_scratch_carve(void *base, uint64_t n, uint64_t wcap = 0);

}  // namespace mckl_b200
