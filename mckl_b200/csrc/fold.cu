// fold.cu -- exact emulation of the sequential double left fold (see fold.cuh).
#include <algorithm>

#include "block_scan.cuh"
#include "common.cuh"
#include "fold.cuh"

namespace mckl_b200 {

namespace {

constexpr int kDescThreads = 512;
constexpr int kPer = kFoldTile / kDescThreads;  // 8 consecutive elements per thread
constexpr int kWalkThreads = 1024;
constexpr int kWalkPer = kFoldTile / kWalkThreads;  // 4
constexpr unsigned kSeqStretch = 256;  // elements folded one at a time after two scan rounds of a tile

__device__ __forceinline__ double ulp_of(double v)
{
    const int eb = biased_exp(v);
    return grid_unit(eb);
}

// Maximum of nonnegative doubles over the CTA (0 for none): the total, and
// the maximum over the threads before this one.  `sh` needs 33 elements.
__device__ __forceinline__ double block_exclusive_max(double v, double *sh, double *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc = fmax(inc, u);
    }
    double prev = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) prev = 0.0;
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        double w = lane < nw ? sh[lane] : 0.0;
        double wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi = fmax(wi, u);
        }
        double we = __shfl_up_sync(0xffffffffu, wi, 1);
        if (lane == 0) we = 0.0;
        if (lane < nw) sh[lane] = we;
        if (lane == nw - 1) sh[32] = wi;
    }
    __syncthreads();
    const double r = warp > 0 ? fmax(sh[warp], prev) : prev;
    *total = sh[32];
    __syncthreads();
    return r;
}


// ---------------------------------------------------------------------------
// Approximate partial sums and the classification of every element.
//
// A_j is a parallel (tree) sum of s0 + x_0 + ... + x_j; S_j the sequential
// fold.  Both are sums of nonnegative terms, so |A_j - S_j| <= (j + 1 + D)
// 2^-53 A_j (first order) with D the depth of A's summation tree (below
// 100 + T / 1024 here: 8 sequential adds per thread, two CTA scans, the
// tile scan with its carries).  ulp(A) > 2^-53 A, so a margin of
// 2 (j + 1) + 2 T + 160 ulps of A_j holds S_j with room to spare: when
// [A_j - margin, A_j + margin] lies inside one binade, S_j certainly does.
// ---------------------------------------------------------------------------
//
// Below 2^-1021 (biased exponent 0 or 1) every sum is exact: all partial
// sums of nonnegative terms are at most the total, and any sum of multiples
// of 2^-1074 below 2^-1021 is representable.  A tree sum below 2^-1021 is
// therefore the exact sum, which the sequential fold also reaches, and its
// binade is certain (this includes zero sums).
//
// The sequential fold never decreases and rounds monotonically, so S_j is at
// least the largest term so far, M_j: the lower end is max(A - margin, M_j).
// Where one term dominates -- degenerate weights, whose largest term is
// exactly 1 = 2^0 with a tiny remainder -- the sum sits just above a binade
// boundary that the margin alone would straddle.
__device__ __forceinline__ int certain_binade(double A, uint64_t j, uint64_t T, double M)
{
    if (biased_exp(A) <= 1 && A >= 0.0) return biased_exp(A);
    const double m = (2.0 * static_cast<double>(j + 1) + 2.0 * static_cast<double>(T) + 160.0) * ulp_of(A);
    const double lo = fmax(__dsub_rn(A, m), M), hi = __dadd_rn(A, m);
    if (!(lo > 0.0)) return -1;
    const int e = biased_exp(lo);
    if (e == 0x7ff || biased_exp(hi) != e) return -1;
    return e;
}

// One CTA scan of (sum, maximum) pairs: the exclusive sum (formed without a
// subtraction, as block_exclusive_sum) and the exclusive maximum (0 for
// none).  `shs`, `shm` need 33 elements each.
__device__ __forceinline__ void block_exclusive_sum_max(double v, double m, double *shs, double *shm,
    double *ex_s, double *ex_m)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double is = v, im = m;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double us = __shfl_up_sync(0xffffffffu, is, o);
        const double um = __shfl_up_sync(0xffffffffu, im, o);
        if (lane >= o) {
            is += us;
            im = fmax(im, um);
        }
    }
    double ps = __shfl_up_sync(0xffffffffu, is, 1), pm = __shfl_up_sync(0xffffffffu, im, 1);
    if (lane == 0) ps = pm = 0.0;
    if (lane == 31) {
        shs[warp] = is;
        shm[warp] = im;
    }
    __syncthreads();
    if (warp == 0) {
        double ws = lane < nw ? shs[lane] : 0.0, wm = lane < nw ? shm[lane] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double us = __shfl_up_sync(0xffffffffu, ws, o);
            const double um = __shfl_up_sync(0xffffffffu, wm, o);
            if (lane >= o) {
                ws += us;
                wm = fmax(wm, um);
            }
        }
        double es = __shfl_up_sync(0xffffffffu, ws, 1), em = __shfl_up_sync(0xffffffffu, wm, 1);
        if (lane == 0) es = em = 0.0;
        if (lane < nw) {
            shs[lane] = es;
            shm[lane] = em;
        }
    }
    __syncthreads();
    *ex_s = warp > 0 ? shs[warp] + ps : ps;
    *ex_m = warp > 0 ? fmax(shm[warp], pm) : pm;
    __syncthreads();
}

// The tile's kPer elements of this thread (zeros past n), the approximate
// partial sum before the first of them, their own sum, and the largest term
// before them (s0 included).
__device__ __forceinline__ void tile_load(const double *x, uint64_t n, double s0, const double *tpre,
    const double *tpmax, uint64_t t, double (&xv)[kPer], double *sh, double *Abefore, double *own_sum,
    double *Mbefore)
{
    const uint64_t i0 = t * kFoldTile + static_cast<uint64_t>(threadIdx.x) * kPer;
    double own = 0.0, mx = 0.0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        xv[k] = i0 + k < n ? x[i0 + k] : 0.0;
        own = __dadd_rn(own, xv[k]);
        mx = fmax(mx, xv[k]);
    }
    __shared__ double shm[33];
    double ex, exm;
    block_exclusive_sum_max(own, mx, sh, shm, &ex, &exm);
    *Abefore = __dadd_rn(__dadd_rn(s0, tpre[t]), ex);
    *own_sum = own;
    *Mbefore = fmax(fmax(s0, tpmax[t]), exm);
}

// Element j = i0 + k is a RUN element when the binades of S_{j-1} and S_j
// are certain and equal and x_j's grid increment at that binade has no event
// (tie, too large): then S_j = S_{j-1} + u q_j exactly.  Every other element
// is a WINDOW: the walk folds it with a real double add.  Returns, per
// element, q (0 for windows), the window bit and the certain binade of
// S_{j-1} (-1: uncertain).
//
// Fast case: S_{i0-1} .. S_{i0+kPer-1} all lie in [A_before - m, A_end + m]
// (the partial sums grow, and A_end = A_before + the thread's own sum is a
// summation tree of the same depth as the per-element A_j), with m the margin
// of the last element, the largest.  When that interval lies in one binade,
// every element's binade is certain and the same, and only its increment
// remains to be checked.
__device__ __forceinline__ void classify(const double (&xv)[kPer], uint64_t i0, uint64_t n, uint64_t T, double s0,
    double Abefore, double own, double Mbefore, long long (&q)[kPer], unsigned &win, int (&eprev)[kPer],
    int *fast_e = nullptr)
{
    if (fast_e) *fast_e = -1;
    {
        const double Aend = __dadd_rn(Abefore, own);
        const double c = 2.0 * static_cast<double>(i0 + kPer) + 2.0 * static_cast<double>(T) + 160.0;
        const double lo = fmax(__dsub_rn(Abefore, c * ulp_of(Abefore)), Mbefore);
        const double hi = __dadd_rn(Aend, c * ulp_of(Aend));
        const int e = biased_exp(lo);
        if (lo > 0.0 && e != 0x7ff && biased_exp(hi) == e) {
            win = 0;
#pragma unroll
            for (int k = 0; k < kPer; ++k) {
                bool ev;
                q[k] = grid_increment(xv[k], e, ev);  // xv is 0 past n: q = 0, no event
                eprev[k] = e;
                if (ev) {
                    q[k] = 0;
                    win |= 1u << k;
                }
            }
            if (fast_e) *fast_e = e;
            return;
        }
    }
    // A zero sum lies on the grid of binade 0 (the subnormals'), so a stretch
    // of leading zeros is a run, not a window per element.
    int ep;
    if (i0 == 0) {
        ep = (s0 >= 0.0 && biased_exp(s0) != 0x7ff) ? biased_exp(s0) : -1;  // s0 itself is exact
    } else {
        ep = certain_binade(Abefore, i0 - 1, T, Mbefore);
    }
    double A = Abefore, M = Mbefore;
    win = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const uint64_t j = i0 + k;
        q[k] = 0;
        eprev[k] = ep;
        if (j < n) {
            A = __dadd_rn(A, xv[k]);
            M = fmax(M, xv[k]);
            // a zero term leaves the sum unchanged (S_j = S_{j-1}): it keeps
            // the previous binade, certain or not, and is never a window; a
            // run of zeros alone adds nothing, so the walk needs no binade
            // for it
            if (xv[k] == 0.0) continue;
            const int ej = certain_binade(A, j, T, M);
            bool ev = true;
            if (ej >= 0 && ej == ep) q[k] = grid_increment(xv[k], ej, ev);
            if (ev) {
                q[k] = 0;
                win |= 1u << k;
            }
            ep = ej;
        }
    }
}

// 1. approximate tile sums
__global__ void __launch_bounds__(kDescThreads) k_fold_tilesum(const double *x, uint64_t n, double *tsum,
    double *tmax)
{
    pdl_wait();
    __shared__ double sh[33];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFoldTile;
    double acc = 0, mx = 0;
    for (int k = 0; k < kPer; ++k) {
        const uint64_t i = base + k * kDescThreads + threadIdx.x;
        if (i < n) {
            acc += x[i];
            mx = fmax(mx, x[i]);
        }
    }
    acc = block_sum(acc, sh);
    double mt;
    block_exclusive_max(mx, sh, &mt);
    if (threadIdx.x == 0) {
        tsum[blockIdx.x] = acc;
        tmax[blockIdx.x] = mt;
    }
}

// 2. exclusive prefix of the tile sums (one CTA), formed without subtraction
// (and, in place, the exclusive prefix maximum of the tile maxima)
__global__ void __launch_bounds__(1024) k_fold_scan_tiles(const double *tsum, uint64_t T, double *tpre,
    double *tpmax)
{
    pdl_wait();
    __shared__ double sh[33];
    double carry = 0, mcarry = 0;
    for (uint64_t b = 0; b < T; b += blockDim.x) {
        const uint64_t t = b + threadIdx.x;
        const double v = t < T ? tsum[t] : 0.0;
        const double mv = t < T ? tpmax[t] : 0.0;
        double tot, mtot;
        const double ex = block_exclusive_sum(v, sh, &tot);
        const double exm = block_exclusive_max(mv, sh, &mtot);
        if (t < T) {
            tpre[t] = b == 0 ? ex : carry + ex;
            tpmax[t] = fmax(mcarry, exm);
        }
        carry += tot;
        mcarry = fmax(mcarry, mtot);
    }
}

// 3. per tile: the sum of the run increments and the number of windows, the
// tile's window list (when it fits), and the tile descriptor of the
// event-loop walk (the fallback)
__global__ void __launch_bounds__(kDescThreads) k_fold_count(const double *x, uint64_t n, double s0,
    const double *tsum, const double *tpre, const double *tpmax, uint64_t T, long long *tq, unsigned *tw, FoldDesc *desc, int *elast,
    FoldLocal loc)
{
    pdl_wait();
    __shared__ double shd[33];
    __shared__ long long shl[33];
    __shared__ unsigned shu[33];
    const uint64_t t = blockIdx.x;
    const uint64_t base = t * kFoldTile;
    const uint64_t i0 = base + static_cast<uint64_t>(threadIdx.x) * kPer;
    double xv[kPer], Ab, own, Mb;
    tile_load(x, n, s0, tpre, tpmax, t, xv, shd, &Ab, &own, &Mb);
    long long q[kPer];
    unsigned win;
    int ep[kPer];
    int fe;
    classify(xv, i0, n, T, s0, Ab, own, Mb, q, win, ep, &fe);
    long long qs = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        qs += q[k];
        // the binade of the last element's run (the walk's tail check)
        if (i0 + k == n - 1) *elast = (win >> k) & 1u ? -1 : ep[k];
    }
    // descriptor of the event-loop walk: the tile's binade, certain for the
    // whole tile, and its increments at that binade
    const double S = __dadd_rn(s0, tpre[t]);
    const double hi_est = __dadd_rn(S, tsum[t]);
    const double margin = static_cast<double>(2 * (base + kFoldTile) + 2 * T + 160) * ulp_of(hi_est);
    const double lo = S - margin, hi = hi_est + margin;
    int slow = !(lo > 0.0);
    const int eb = biased_exp(lo);
    if (biased_exp(hi) != eb) slow = 1;
    long long qtot;
    unsigned wtot;
    long long P = block_exclusive_sum(qs, shl, &qtot);
    unsigned r = block_exclusive_sum(static_cast<unsigned>(__popc(win)), shu, &wtot);
    // When every thread classified its range in the tile's binade, the
    // descriptor's increments are the run increments just summed (the
    // windows are then exactly the elements with an event); otherwise they
    // are formed at the tile's binade.  `slow` is the same for the whole CTA.
    long long A = qtot;
    int ev = wtot > 0;
    if (!slow && !__syncthreads_and(fe == eb)) {
        A = 0;
        ev = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if (i0 + k < n) {
                bool e;
                A += grid_increment(xv[k], eb, e);
                ev |= e;
            }
        }
        ev = __syncthreads_or(ev);
        A = block_sum(A, shl);
    }
    if (wtot <= loc.cap) {
        const uint64_t slot0 = t * loc.cap;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if ((win >> k) & 1u) {
                const uint64_t sl = slot0 + r;
                loc.off[sl] = threadIdx.x * kPer + k;
                loc.x[sl] = xv[k];
                loc.P[sl] = P;
                loc.e[sl] = ep[k];
                ++r;
            }
            P += q[k];
        }
    }
    if (threadIdx.x == 0) {
        desc[t].eb = eb;
        desc[t].flags = (slow || ev) ? 1 : 0;
        desc[t].A = A;
        tq[t] = qtot;
        tw[t] = wtot;
    }
}

// 4. exclusive prefixes of the per-tile counts (one CTA); tot[0] = the sum of
// all run increments, tot[1] = the number of windows
__global__ void __launch_bounds__(1024) k_fold_scan_counts(const long long *tq, const unsigned *tw, uint64_t T,
    long long *pq, unsigned long long *pw, long long *tot)
{
    pdl_wait();
    __shared__ long long shl[33];
    __shared__ unsigned long long shu[33];
    long long cq = 0;
    unsigned long long cw = 0;
    for (uint64_t b = 0; b < T; b += blockDim.x) {
        const uint64_t t = b + threadIdx.x;
        const long long vq = t < T ? tq[t] : 0;
        const unsigned long long vw = t < T ? tw[t] : 0;
        long long totq;
        unsigned long long totw;
        const long long eq = block_exclusive_sum(vq, shl, &totq);
        const unsigned long long ew = block_exclusive_sum(vw, shu, &totw);
        if (t < T) {
            pq[t] = cq + eq;
            pw[t] = cw + ew;
        }
        cq += totq;
        cw += totw;
    }
    if (threadIdx.x == 0) {
        tot[0] = cq;
        tot[1] = static_cast<long long>(cw);
    }
}

// 5. the windows in order: index, value, run-increment prefix before it and
// the binade of the run before it
__global__ void __launch_bounds__(kDescThreads) k_fold_emit(const double *x, uint64_t n, double s0,
    const double *tpre, const double *tpmax, uint64_t T, const long long *pq, const unsigned long long *pw, const unsigned *tw,
    const long long *tot, FoldWindows w, FoldLocal loc)
{
    pdl_wait();
    __shared__ double shd[33];
    __shared__ long long shl[33];
    __shared__ unsigned shu[33];
    if (static_cast<unsigned long long>(tot[1]) > w.cap) return;  // the walk takes the event loop
    const uint64_t t = blockIdx.x;
    const unsigned nw = tw[t];
    if (nw == 0) return;
    if (nw <= loc.cap) {  // the counting pass listed them
        for (unsigned k = threadIdx.x; k < nw; k += kDescThreads) {
            const uint64_t sl = t * loc.cap + k, g = pw[t] + k;
            w.idx[g] = t * kFoldTile + loc.off[sl];
            w.x[g] = loc.x[sl];
            w.P[g] = pq[t] + loc.P[sl];
            w.e[g] = loc.e[sl];
        }
        return;
    }
    const uint64_t i0 = t * kFoldTile + static_cast<uint64_t>(threadIdx.x) * kPer;
    double xv[kPer], Ab, own, Mb;
    tile_load(x, n, s0, tpre, tpmax, t, xv, shd, &Ab, &own, &Mb);
    long long q[kPer];
    unsigned win;
    int ep[kPer];
    classify(xv, i0, n, T, s0, Ab, own, Mb, q, win, ep);
    long long qs = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) qs += q[k];
    long long qtot;
    unsigned wtot;
    long long P = pq[t] + block_exclusive_sum(qs, shl, &qtot);
    uint64_t r = pw[t] + block_exclusive_sum(static_cast<unsigned>(__popc(win)), shu, &wtot);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if ((win >> k) & 1u) {
            w.idx[r] = i0 + k;
            w.x[r] = xv[k];
            w.P[r] = P;
            w.e[r] = ep[k];
            ++r;
        }
        P += q[k];
    }
}

// CTA-wide exact fold of one tile with the event loop.  All kWalkThreads
// threads call it; returns the value after the tile's last element.
__device__ double fold_tile_exact(const double *x, uint64_t len, double s, double *prefix)
{
    __shared__ long long shl[33];
    __shared__ unsigned shu[33];
    __shared__ double sh_next;
    double xr[kWalkPer];
    const int j0 = threadIdx.x * kWalkPer;
#pragma unroll
    for (int k = 0; k < kWalkPer; ++k) xr[k] = (static_cast<uint64_t>(j0 + k) < len) ? x[j0 + k] : 0.0;
    unsigned cur = 0;
    int rounds = 0;  // scan rounds since the last sequential stretch
    while (cur < len) {
        if (rounds >= 2) {
            // events are dense here (the first tiles cross a binade every few
            // elements): the next kSeqStretch elements one at a time, by one
            // thread, cost less than a CTA scan per event
            const unsigned end = static_cast<unsigned>(std::min<uint64_t>(len, cur + kSeqStretch));
            if (threadIdx.x == 0) {
                double v = s;
                for (unsigned j = cur; j < end; ++j) {
                    v = __dadd_rn(v, x[j]);
                    if (prefix) prefix[j] = v;
                }
                sh_next = v;
            }
            __syncthreads();
            s = sh_next;
            __syncthreads();
            cur = end;
            rounds = 0;
            continue;
        }
        ++rounds;
        if (s == 0.0) {
            // nothing accumulated yet: the next sum is exact, 0 + x = x
            if (static_cast<unsigned>(j0) <= cur && cur < static_cast<unsigned>(j0 + kWalkPer)) {
                const double v = __dadd_rn(s, xr[cur - j0]);
                if (prefix) prefix[cur] = v;
                sh_next = v;
            }
            __syncthreads();
            s = sh_next;
            __syncthreads();
            ++cur;
            continue;
        }
        const int eb = biased_exp(s);
        const long long K = grid_count(s), top = grid_top(eb);
        long long q[kWalkPer];
        bool evk[kWalkPer];
        long long own = 0;
#pragma unroll
        for (int k = 0; k < kWalkPer; ++k) {
            const unsigned j = j0 + k;
            evk[k] = false;
            q[k] = 0;
            if (j >= cur && j < len) {
                bool e;
                q[k] = grid_increment(xr[k], eb, e);
                evk[k] = e;
            }
            own += q[k];
        }
        long long tot;
        const long long incl = block_inclusive_sum(own, shl, &tot);
        long long run = incl - own;  // exclusive prefix before this thread's first element
        unsigned first_ev = 0xffffffffu;
        long long Q[kWalkPer];
#pragma unroll
        for (int k = 0; k < kWalkPer; ++k) {
            run += q[k];
            Q[k] = run;
            const unsigned j = j0 + k;
            if (j >= cur && j < len && first_ev == 0xffffffffu) {
                if (evk[k] || K + run >= top) first_ev = j;
            }
        }
        const unsigned c = block_min_u32(first_ev, shu);
        const unsigned stop = c < len ? c : static_cast<unsigned>(len);
#pragma unroll
        for (int k = 0; k < kWalkPer; ++k) {
            const unsigned j = j0 + k;
            if (j >= cur && j < stop && prefix) prefix[j] = from_grid(K + Q[k], eb);
            if (j + 1 == stop && c >= len) sh_next = from_grid(K + Q[k], eb);
        }
        if (c < len && static_cast<unsigned>(j0) <= c && c < static_cast<unsigned>(j0 + kWalkPer)) {
            const int k = c - j0;
            const double prev = (c == cur) ? s : from_grid(K + Q[k] - q[k], eb);
            const double v = __dadd_rn(prev, xr[k]);
            if (prefix) prefix[c] = v;
            sh_next = v;
        }
        __syncthreads();
        s = sh_next;
        __syncthreads();
        if (c >= len) break;
        cur = c + 1;
    }
    return s;
}

// The event-loop walk (used when the windows do not fit their list, or if
// the window walk ever met a value outside the binade it was classified in):
// one CTA chains tile-entry values in order; certain tiles cost O(1), the
// others are folded by the CTA with the event loop.
__device__ void walk_events(const double *x, uint64_t n, double s0, const FoldDesc *desc, uint64_t T,
    double *tstart, int *tmode, double *prefix, double *final_v)
{
    __shared__ double sh_s;
    __shared__ unsigned long long sh_t;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        sh_s = s0;
        sh_t = 0;
    }
    __syncthreads();
    while (true) {
        if (warp == 0) {
            // certain tiles, 32 at a time: lane l takes tile t + l; inside a
            // run of certain tiles of the running sum's binade the entry
            // counts are K + (exclusive prefix of the tiles' A), and the run
            // ends at the first tile that is flagged, of another binade, or
            // would leave the binade (then the CTA folds it exactly)
            double s = sh_s;
            uint64_t t = sh_t;
            while (t < T) {
                const uint64_t mine = t + lane;
                FoldDesc d{0, 1, 0};
                if (mine < T) d = desc[mine];
                const int eb = biased_exp(s);
                const long long K = grid_count(s);
                // inclusive prefix of A over the lanes (unsigned: past the
                // first tile that ends the run the sums are not used)
                unsigned long long P = static_cast<unsigned long long>(d.A);
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned long long n = __shfl_up_sync(0xffffffffu, P, o);
                    if (lane >= o) P += n;
                }
                const bool ok = s > 0.0 && !d.flags && d.eb == eb && d.A >= 0 &&
                                P < static_cast<unsigned long long>(grid_top(eb) - K);
                const unsigned bad = __ballot_sync(0xffffffffu, !ok);
                const int taken = bad ? __ffs(bad) - 1 : 32;
                if (lane < taken) {
                    tstart[mine] = from_grid(K + static_cast<long long>(P) - d.A, eb);
                    tmode[mine] = 0;
                }
                if (taken == 0) break;
                s = from_grid(K + static_cast<long long>(__shfl_sync(0xffffffffu, P, taken - 1)), eb);
                t += taken;
                if (taken < 32) break;
            }
            if (lane == 0) {
                sh_s = s;
                sh_t = t;
            }
        }
        __syncthreads();
        const uint64_t t = sh_t;
        if (t >= T) break;
        // uncertain tile: the whole CTA folds it exactly
        const double sin = sh_s;
        const uint64_t base = t * kFoldTile;
        const uint64_t len = std::min<uint64_t>(kFoldTile, n - base);
        const double sout = fold_tile_exact(x + base, len, sin, prefix ? prefix + base : nullptr);
        if (threadIdx.x == 0) {
            tstart[t] = sin;
            tmode[t] = 1;
            sh_s = sout;
            sh_t = t + 1;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *final_v = sh_s;
}

__device__ void expand_events(const double *x, uint64_t n, const FoldDesc *desc, const double *tstart,
    const int *tmode, double *prefix, uint64_t t, long long *shl)
{
    if (tmode[t] != 0) return;
    const uint64_t base = t * kFoldTile;
    const int eb = desc[t].eb;
    const long long K = grid_count(tstart[t]);
    long long q[kPer];
    long long own = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const uint64_t i = base + threadIdx.x * kPer + k;
        bool e;
        q[k] = (i < n) ? grid_increment(x[i], eb, e) : 0;
        own += q[k];
    }
    long long tot;
    long long run = block_inclusive_sum(own, shl, &tot) - own;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const uint64_t i = base + threadIdx.x * kPer + k;
        run += q[k];
        if (i < n) prefix[i] = from_grid(K + run, eb);
    }
}

constexpr int kStage = 1024;  // window entries staged in shared memory per walk round

// 6. the walk (one CTA): the windows in order; the run before each window is
// one integer step on its binade's grid, the window itself the reference's
// own double add.  Writes the value after every window (mode 0).  When the
// windows did not fit their list, or a run's value is not in the binade it
// was classified in (the margins make that impossible; the check costs two
// compares), the event-loop walk does the fold instead (mode 1).
__global__ void __launch_bounds__(kWalkThreads) k_fold_walk(const double *x, uint64_t n, double s0,
    const FoldDesc *desc, uint64_t T, double *tstart, int *tmode, double *prefix, double *final_v,
    const long long *tot, const int *elast, FoldWindows w, int *mode)
{
    pdl_wait();
    __shared__ unsigned long long sj[kStage];
    __shared__ double sx[kStage];
    __shared__ long long sp[kStage];
    __shared__ int se[kStage];
    __shared__ int sh_ok;
    __shared__ double sh_s;
    __shared__ long long sh_p;
    __shared__ unsigned long long sh_j;
    __shared__ unsigned long long sh_w;
    __shared__ long long sh_q;
    __shared__ int sh_elast;
    // The first round's windows are staged before their count is known
    // (entries past the count are loaded but never read), in the same round
    // trip as the count and the tail's inputs.
    {
        const unsigned m0 = static_cast<unsigned>(w.cap < kStage ? w.cap : kStage);
        for (unsigned k = threadIdx.x; k < m0; k += blockDim.x) {
            sj[k] = w.idx[k];
            sx[k] = w.x[k];
            sp[k] = w.P[k];
            se[k] = w.e[k];
        }
    }
    if (threadIdx.x == 0) {
        const unsigned long long W0 = static_cast<unsigned long long>(tot[1]);
        sh_w = W0;
        sh_q = tot[0];
        sh_elast = *elast;
        sh_ok = W0 <= w.cap ? 1 : 0;
        sh_s = s0;
        sh_p = 0;
        sh_j = 0;
    }
    __syncthreads();
    const unsigned long long W = sh_w;
    for (unsigned long long c0 = 0; sh_ok && c0 < W; c0 += kStage) {
        const unsigned m = static_cast<unsigned>(W - c0 < kStage ? W - c0 : kStage);
        if (c0 > 0) {
            for (unsigned k = threadIdx.x; k < m; k += blockDim.x) {
                sj[k] = w.idx[c0 + k];
                sx[k] = w.x[c0 + k];
                sp[k] = w.P[c0 + k];
                se[k] = w.e[c0 + k];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double s = sh_s;
            long long p = sh_p;
            unsigned long long jn = sh_j;
            int good = 1;
            for (unsigned k = 0; k < m; ++k) {
                if (sj[k] > jn && sp[k] != p) {  // the run jn .. sj[k] - 1 (a zero sum is on binade 0's grid)
                    const int e = se[k];
                    if (!(s >= 0.0) || biased_exp(s) != e) {
                        good = 0;
                        break;
                    }
                    const long long K = grid_count(s) + (sp[k] - p);
                    if (K >= grid_top(e)) {
                        good = 0;
                        break;
                    }
                    s = from_grid(K, e);
                }
                s = __dadd_rn(s, sx[k]);
                w.S[c0 + k] = s;
                p = sp[k];
                jn = sj[k] + 1;
            }
            sh_s = s;
            sh_p = p;
            sh_j = jn;
            sh_ok = good;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && sh_ok) {
        double s = sh_s;
        if (sh_j < n && sh_q != sh_p) {  // the run after the last window, when it adds anything
            const int e = sh_elast;
            const long long K = grid_count(s) + (sh_q - sh_p);
            if (e < 0 || !(s >= 0.0) || biased_exp(s) != e || K >= grid_top(e)) {
                sh_ok = 0;
            } else {
                s = from_grid(K, e);
            }
        }
        if (sh_ok) {
            *final_v = s;
            *mode = 0;
        }
    }
    __syncthreads();
    if (!sh_ok) {
        if (threadIdx.x == 0) *mode = 1;
        walk_events(x, n, s0, desc, T, tstart, tmode, prefix, final_v);
    }
}

// 7. every partial sum, when the caller asks for them: a run element is the
// value after the window before it plus its run's increments on the grid, a
// window element the walk's value.
__global__ void __launch_bounds__(kDescThreads) k_fold_expand(const double *x, uint64_t n, double s0,
    const double *tpre, const double *tpmax, uint64_t T, const long long *pq, const unsigned long long *pw, FoldWindows w,
    const int *mode, const FoldDesc *desc, const double *tstart, const int *tmode, double *prefix)
{
    pdl_wait();
    __shared__ double shd[33];
    __shared__ long long shl[33];
    __shared__ unsigned shu[33];
    const uint64_t t = blockIdx.x;
    if (*mode != 0) {
        expand_events(x, n, desc, tstart, tmode, prefix, t, shl);
        return;
    }
    const uint64_t i0 = t * kFoldTile + static_cast<uint64_t>(threadIdx.x) * kPer;
    double xv[kPer], Ab, own, Mb;
    tile_load(x, n, s0, tpre, tpmax, t, xv, shd, &Ab, &own, &Mb);
    long long q[kPer];
    unsigned win;
    int ep[kPer];
    classify(xv, i0, n, T, s0, Ab, own, Mb, q, win, ep);
    long long qs = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) qs += q[k];
    long long qtot;
    unsigned wtot;
    long long P = pq[t] + block_exclusive_sum(qs, shl, &qtot);
    uint64_t r = pw[t] + block_exclusive_sum(static_cast<unsigned>(__popc(win)), shu, &wtot);
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const uint64_t j = i0 + k;
        if (j >= n) break;
        if ((win >> k) & 1u) {
            prefix[j] = w.S[r];
            ++r;
        } else {
            P += q[k];
            const double Sb = r > 0 ? w.S[r - 1] : s0;
            const long long Pb = r > 0 ? w.P[r - 1] : 0;
            prefix[j] = from_grid(grid_count(Sb) + (P - Pb), biased_exp(Sb));
        }
    }
}

__global__ void k_fold_set(double *v, double s0)
{
    pdl_wait();
    *v = s0;
}

}  // namespace

uint64_t fold_window_cap(uint64_t n)
{
    return std::min<uint64_t>(n + 1, 4096 + n / 256);
}

size_t fold_scratch_bytes(uint64_t n, uint64_t wcap)
{
    const uint64_t T = (n + kFoldTile - 1) / kFoldTile + 1;
    const uint64_t L = wcap == 0 ? T * kFoldLocalCap : 0;
    if (wcap == 0) wcap = fold_window_cap(n);
    return align256(T * sizeof(FoldDesc)) + 4 * align256(T * sizeof(double)) + align256(T * sizeof(int)) +
           align256(T * sizeof(long long)) + align256(T * sizeof(unsigned)) + align256(T * sizeof(long long)) +
           align256(T * sizeof(unsigned long long)) + 256 + align256(wcap * sizeof(unsigned long long)) +
           3 * align256(wcap * sizeof(double)) + align256(wcap * sizeof(int)) + 2 * align256(L * sizeof(int)) +
           2 * align256(L * sizeof(double));
}

FoldScratch fold_scratch_carve(void *base, uint64_t n, uint64_t wcap)
{
    const uint64_t T = (n + kFoldTile - 1) / kFoldTile + 1;
    const unsigned lcap = wcap == 0 ? kFoldLocalCap : 0;
    if (wcap == 0) wcap = fold_window_cap(n);
    char *p = static_cast<char *>(base);
    auto take = [&p](size_t bytes) {
        char *q = p;
        p += align256(bytes);
        return q;
    };
    FoldScratch f;
    f.desc = reinterpret_cast<FoldDesc *>(take(T * sizeof(FoldDesc)));
    f.tsum = reinterpret_cast<double *>(take(T * sizeof(double)));
    f.tpre = reinterpret_cast<double *>(take(T * sizeof(double)));
    f.tpmax = reinterpret_cast<double *>(take(T * sizeof(double)));
    f.tstart = reinterpret_cast<double *>(take(T * sizeof(double)));
    f.tmode = reinterpret_cast<int *>(take(T * sizeof(int)));
    f.tq = reinterpret_cast<long long *>(take(T * sizeof(long long)));
    f.tw = reinterpret_cast<unsigned *>(take(T * sizeof(unsigned)));
    f.pq = reinterpret_cast<long long *>(take(T * sizeof(long long)));
    f.pw = reinterpret_cast<unsigned long long *>(take(T * sizeof(unsigned long long)));
    char *small = take(256);
    f.final_v = reinterpret_cast<double *>(small);
    f.tot = reinterpret_cast<long long *>(small + 64);
    f.elast = reinterpret_cast<int *>(small + 128);
    f.mode = reinterpret_cast<int *>(small + 192);
    f.win.idx = reinterpret_cast<unsigned long long *>(take(wcap * sizeof(unsigned long long)));
    f.win.x = reinterpret_cast<double *>(take(wcap * sizeof(double)));
    f.win.P = reinterpret_cast<long long *>(take(wcap * sizeof(long long)));
    f.win.S = reinterpret_cast<double *>(take(wcap * sizeof(double)));
    f.win.e = reinterpret_cast<int *>(take(wcap * sizeof(int)));
    f.win.cap = wcap;
    const uint64_t L = T * lcap;
    f.loc.off = reinterpret_cast<unsigned *>(take(L * sizeof(unsigned)));
    f.loc.x = reinterpret_cast<double *>(take(L * sizeof(double)));
    f.loc.P = reinterpret_cast<long long *>(take(L * sizeof(long long)));
    f.loc.e = reinterpret_cast<int *>(take(L * sizeof(int)));
    f.loc.cap = lcap;
    return f;
}

int fold_exact(const double *x, uint64_t n, double s0, double *prefix, FoldScratch &fs, cudaStream_t s)
{
    if (n == 0) {
        MB_CUDA(launch_pdl(k_fold_set, 1, 1, 0, s, fs.final_v, s0));
        MB_LAUNCH_CHECK();
        return MCKL_B200_OK;
    }
    const uint64_t T = (n + kFoldTile - 1) / kFoldTile;
    const unsigned nt = static_cast<unsigned>(T);
    MB_CUDA(launch_pdl(k_fold_tilesum, nt, kDescThreads, 0, s, x, n, fs.tsum, fs.tpmax));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_fold_scan_tiles, 1, 1024, 0, s, fs.tsum, T, fs.tpre, fs.tpmax));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_fold_count, nt, kDescThreads, 0, s, x, n, s0, fs.tsum, fs.tpre, fs.tpmax, T, fs.tq, fs.tw,
        fs.desc, fs.elast, fs.loc));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_fold_scan_counts, 1, 1024, 0, s, fs.tq, fs.tw, T, fs.pq, fs.pw, fs.tot));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_fold_emit, nt, kDescThreads, 0, s, x, n, s0, fs.tpre, fs.tpmax, T, fs.pq, fs.pw, fs.tw,
        fs.tot, fs.win, fs.loc));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_fold_walk, 1, kWalkThreads, 0, s, x, n, s0, fs.desc, T, fs.tstart, fs.tmode, prefix,
        fs.final_v, fs.tot, fs.elast, fs.win, fs.mode));
    MB_LAUNCH_CHECK();
    if (prefix) {
        MB_CUDA(launch_pdl(k_fold_expand, nt, kDescThreads, 0, s, x, n, s0, fs.tpre, fs.tpmax, T, fs.pq, fs.pw,
            fs.win, fs.mode, fs.desc, fs.tstart, fs.tmode, prefix));
        MB_LAUNCH_CHECK();
    }
    return MCKL_B200_OK;
}

}  // namespace mckl_b200


using namespace mckl_b200;

extern "C" int mckl_b200_fold_f64(size_t n, const double *x, double s0, double *prefix, double *final_value,
    void *stream)
{
    MB_CHECK_ARG(n == 0 || x != nullptr, "null input");
    MB_CHECK_ARG(final_value != nullptr, "null result");
    cudaStream_t s = as_stream(stream);
    void *base = scratch(1, fold_scratch_bytes(n), s);
    if (!base) {
        set_error("fold scratch allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    FoldScratch fs = fold_scratch_carve(base, n);
    int rc = fold_exact(x, n, s0, prefix, fs, s);
    if (rc != MCKL_B200_OK) return rc;
    MB_CUDA(cudaMemcpyAsync(final_value, fs.final_v, sizeof(double), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return MCKL_B200_OK;
}
