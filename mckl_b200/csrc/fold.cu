// fold.cu -- exact emulation of the sequential double left fold (see fold.cuh).
#include <algorithm>

#include "block_scan.cuh"
#include "common.cuh"
#include "fold.cuh"

namespace mckl_b200 {

namespace {

constexpr int kDescThreads = 256;
constexpr int kPer = kFoldTile / kDescThreads;  // 16 consecutive elements per thread
constexpr int kWalkThreads = 1024;
constexpr int kWalkPer = kFoldTile / kWalkThreads;  // 4
constexpr unsigned kSeqStretch = 256;  // elements folded one at a time after two scan rounds of a tile

__device__ __forceinline__ double ulp_of(double v)
{
    const int eb = biased_exp(v);
    return grid_unit(eb);
}

// 1. approximate tile sums
__global__ void __launch_bounds__(kDescThreads) k_fold_tilesum(const double *x, uint64_t n, double *tsum)
{
    __shared__ double sh[33];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kFoldTile;
    double acc = 0;
    for (int k = 0; k < kPer; ++k) {
        const uint64_t i = base + k * kDescThreads + threadIdx.x;
        if (i < n) acc += x[i];
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) tsum[blockIdx.x] = acc;
}

// 2. exclusive prefix of tile sums (one CTA)
__global__ void __launch_bounds__(1024) k_fold_scan_tiles(const double *tsum, uint64_t T, double *tpre)
{
    __shared__ double sh[33];
    double carry = 0;
    for (uint64_t b = 0; b < T; b += blockDim.x) {
        const uint64_t t = b + threadIdx.x;
        const double v = t < T ? tsum[t] : 0.0;
        double tot;
        const double inc = block_inclusive_sum(v, sh, &tot);
        if (t < T) tpre[t] = carry + (inc - v);
        carry += tot;
    }
}

// 3. tile descriptors: binade certain for the whole tile, no event inside
__global__ void __launch_bounds__(kDescThreads) k_fold_describe(const double *x, uint64_t n, double s0,
    const double *tsum, const double *tpre, uint64_t T, FoldDesc *desc)
{
    __shared__ long long shl[33];
    const uint64_t t = blockIdx.x;
    const uint64_t base = t * kFoldTile;
    const double S = s0 + tpre[t];
    const double hi_est = S + tsum[t];
    // fold error after i additions is below i ulp(s_i) / 2; the tile-sum
    // prefix adds its own few ulps: a generous bound
    const double margin = static_cast<double>(2 * (base + kFoldTile) + 2 * T + 64) * ulp_of(hi_est);
    const double lo = S - margin, hi = hi_est + margin;
    int slow = !(lo > 0.0);
    const int eb = biased_exp(lo);
    if (biased_exp(hi) != eb) slow = 1;
    long long A = 0;
    int ev = 0;
    if (!slow) {
        for (int k = 0; k < kPer; ++k) {
            const uint64_t i = base + threadIdx.x * kPer + k;
            if (i < n) {
                bool e;
                A += grid_increment(x[i], eb, e);
                ev |= e;
            }
        }
    }
    ev = __syncthreads_or(ev);
    A = block_sum(A, shl);
    if (threadIdx.x == 0) {
        desc[t].eb = eb;
        desc[t].flags = (slow || ev) ? 1 : 0;
        desc[t].A = A;
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

// 4. the walker: one CTA chains tile-entry values in order
__global__ void __launch_bounds__(kWalkThreads) k_fold_walk(const double *x, uint64_t n, double s0,
    const FoldDesc *desc, uint64_t T, double *tstart, int *tmode, double *prefix, double *final_v)
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

// 5. expand certain tiles to every partial sum
__global__ void __launch_bounds__(kDescThreads) k_fold_expand(const double *x, uint64_t n, const FoldDesc *desc,
    const double *tstart, const int *tmode, double *prefix)
{
    __shared__ long long shl[33];
    const uint64_t t = blockIdx.x;
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

}  // namespace

size_t fold_scratch_bytes(uint64_t n)
{
    const uint64_t T = (n + kFoldTile - 1) / kFoldTile + 1;
    return align256(T * sizeof(FoldDesc)) + 3 * align256(T * sizeof(double)) + align256(T * sizeof(int)) + 256;
}

FoldScratch fold_scratch_carve(void *base, uint64_t n)
{
    const uint64_t T = (n + kFoldTile - 1) / kFoldTile + 1;
    char *p = static_cast<char *>(base);
    FoldScratch f;
    f.desc = reinterpret_cast<FoldDesc *>(p);
    p += align256(T * sizeof(FoldDesc));
    f.tsum = reinterpret_cast<double *>(p);
    p += align256(T * sizeof(double));
    f.tpre = reinterpret_cast<double *>(p);
    p += align256(T * sizeof(double));
    f.tstart = reinterpret_cast<double *>(p);
    p += align256(T * sizeof(double));
    f.tmode = reinterpret_cast<int *>(p);
    p += align256(T * sizeof(int));
    f.final_v = reinterpret_cast<double *>(p);
    return f;
}

int fold_exact(const double *x, uint64_t n, double s0, double *prefix, FoldScratch &fs, cudaStream_t s)
{
    if (n == 0) {
        MB_CUDA(cudaMemcpyAsync(fs.final_v, &s0, sizeof(double), cudaMemcpyHostToDevice, s));
        return MCKL_B200_OK;
    }
    const uint64_t T = (n + kFoldTile - 1) / kFoldTile;
    k_fold_tilesum<<<static_cast<unsigned>(T), kDescThreads, 0, s>>>(x, n, fs.tsum);
    MB_LAUNCH_CHECK();
    k_fold_scan_tiles<<<1, 1024, 0, s>>>(fs.tsum, T, fs.tpre);
    MB_LAUNCH_CHECK();
    k_fold_describe<<<static_cast<unsigned>(T), kDescThreads, 0, s>>>(x, n, s0, fs.tsum, fs.tpre, T, fs.desc);
    MB_LAUNCH_CHECK();
    k_fold_walk<<<1, kWalkThreads, 0, s>>>(x, n, s0, fs.desc, T, fs.tstart, fs.tmode, prefix, fs.final_v);
    MB_LAUNCH_CHECK();
    if (prefix) {
        k_fold_expand<<<static_cast<unsigned>(T), kDescThreads, 0, s>>>(x, n, fs.desc, fs.tstart, fs.tmode, prefix);
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
