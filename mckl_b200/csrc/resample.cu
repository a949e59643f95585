// resample.cu -- the reference's resampling algorithms (algorithm/resample.hpp)
// on the device, bit-identical in replication counts and parent indices.
//
//   uniform sequences (:63-268)
//     systematic: u_j = fma(j, 1/M, U/M), U one canonical draw (2 words)
//     stratified: u_j = (1/M) (U_j + j), U_j canonical draws per 1024-chunk
//     sorted:     lmax_j = lmax_{j-1} + log(U_j) / (M - j)   (a sequential fold:
//                 negated, it is a fold of nonnegative terms -> fold_exact)
//                 u_j = 1 - exp(lmax_j)
//   replication counts (:374-407): rep_i = LB(c_i) - LB(c_{i-1}) with c_i the
//     exact left fold of W_0..W_i (fold_exact) and LB(v) = #{j : u_j < v}
//     (the reference's merge loop, u nondecreasing); rep_{N-1} = M - LB(c_{N-2})
//   residual (:333-364, :548-566): integer parts of M W_i, residuals summed by
//     the exact fold and scaled by 1 / sum, R = M - sum of integer parts
//     uniforms drawn on the residuals, then rep += integer parts
//   parent indices (:416-466): occupied slots keep their particle; the empty
//     slots, in ascending order, take the surplus copies in source order.  A
//     single-pass decoupled-look-back scan counts empties and surplus copies,
//     each empty slot then finds its source by binary search.
#include <algorithm>

#include "block_scan.cuh"
#include "common.cuh"
#include "crmath.cuh"
#include "fold.cuh"
#include "resample.cuh"
#include "transforms.cuh"

namespace mckl_b200 {

namespace {

unsigned cap_grid(uint64_t n, int threads, int per_sm = 16)
{
    const uint64_t need = (n + threads - 1) / threads;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(need, 148ull * per_sm)));
}

#define GRID_LOOP(i, n) \
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < (n); \
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)

// canonical double uniforms from two u32 words each, stream words from (B, off)
template <class G>
__global__ void k_canonical(G g, Ctr B, uint32_t off, uint64_t n, double *u)
{
    g.prepare();
    GRID_LOOP(i, n)
    {
        const uint64_t a = off + 2 * i;
        uint32_t blk[G::kWords];
        g.block(ctr_add(B, a / G::kWords, G::kCtrWords), blk);
        const uint32_t w0 = blk[a % G::kWords];
        uint32_t w1;
        if ((a + 1) % G::kWords == 0) {
            uint32_t blk2[G::kWords];
            g.block(ctr_add(B, (a + 1) / G::kWords, G::kCtrWords), blk2);
            w1 = blk2[0];
        } else {
            w1 = blk[(a + 1) % G::kWords];
        }
        u[i] = u01_canonical2(w0, w1);
    }
}

__global__ void k_stratified(uint64_t M, double *u)
{
    const double delta = __ddiv_rn(1.0, static_cast<double>(M));
    GRID_LOOP(j, M) { u[j] = __dmul_rn(delta, __dadd_rn(u[j], static_cast<double>(j))); }
}

// sorted, step 1: t_j = -(log(U_j) / (M - j)) >= 0
__global__ void k_sorted_terms(uint64_t M, double *u)
{
    GRID_LOOP(j, M) { u[j] = -__ddiv_rn(dd::log(u[j]), static_cast<double>(M - j)); }
}

// sorted, step 2: u_j = 1 - exp(lmax_j), lmax_j = -prefix_j
__global__ void k_sorted_finish(uint64_t M, const double *prefix, double *u)
{
    GRID_LOOP(j, M) { u[j] = __dsub_rn(1.0, dd::exp(-prefix[j])); }
}

// systematic: one canonical U from two single-word draws at words a0, a0 + 1
template <class G>
__global__ void k_systematic(G g, Ctr B, uint32_t off, uint64_t M, double *u)
{
    g.prepare();
    uint32_t w[2];
    for (int q = 0; q < 2; ++q) {
        const uint64_t a = off + q;
        uint32_t blk[G::kWords];
        g.block(ctr_add(B, a / G::kWords, G::kCtrWords), blk);
        w[q] = blk[a % G::kWords];
    }
    const double U = u01_canonical2(w[0], w[1]);
    const double delta = __ddiv_rn(1.0, static_cast<double>(M));
    const double ud = __dmul_rn(U, delta);
    GRID_LOOP(j, M) { u[j] = __fma_rn(static_cast<double>(j), delta, ud); }
}

// The first k with u[k] >= v in the sorted u[0..M), found by galloping out
// from the guess g (any g in [0, M] gives the same answer) and a binary search
// of the bracket: about 2 log2(|answer - g| + 1) reads.  The uniforms of every
// scheme are sorted and close to evenly spread over [0, 1) -- within one slot
// of j/M for the stratified and systematic sequences -- so g = floor(v M) is
// usually within a step or two, and the reads of a warp are coalesced.
__device__ __forceinline__ uint64_t lower_bound_from(const double *u, uint64_t M, double v, uint64_t g)
{
    uint64_t lo, hi;
    if (g < M && u[g] < v) {  // the answer is in (g, M]
        lo = g + 1;
        hi = M;
        for (uint64_t step = 1;; step <<= 1) {
            const uint64_t probe = lo - 1 + step;
            if (probe >= M) break;
            if (u[probe] >= v) {
                hi = probe;
                break;
            }
            lo = probe + 1;
        }
    } else {  // the answer is in [0, g]
        lo = 0;
        hi = g;
        for (uint64_t step = 1; step <= hi; step <<= 1) {
            const uint64_t probe = hi - step;
            if (u[probe] < v) {
                lo = probe + 1;
                break;
            }
            hi = probe;
        }
    }
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (u[mid] < v) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

__device__ __forceinline__ uint64_t lower_bound(const double *u, uint64_t M, double v)
{
    const double gx = v * static_cast<double>(M);
    const uint64_t g = gx > 0.0 ? (gx < static_cast<double>(M) ? static_cast<uint64_t>(gx) : M) : 0;
    return lower_bound_from(u, M, v, g);
}

// the neighbouring doubles of v >= 0 (v below the largest finite double)
__device__ __forceinline__ double next_up(double v)
{
    return __longlong_as_double(__double_as_longlong(v) + 1);
}

__device__ __forceinline__ double next_down(double v)
{
    return v > 0.0 ? __longlong_as_double(__double_as_longlong(v) - 1) : v;
}

// rep_i from the cumulative weights c (length N - 1) and sorted uniforms u.
// With `ties` set, also counts the uniforms within one representable step of
// a cumulative weight (prev(c_i) <= u_j <= next(c_i)): the comparisons
// u_j < c_i that a cumulative weight one ulp off would decide the other way.
__global__ void k_rep_counts(uint64_t N, uint64_t M, const double *c, const double *u, uint64_t *rep,
    unsigned long long *ties)
{
    pdl_wait();
    __shared__ unsigned long long sh[33];
    unsigned long long nt = 0;
    // the bound below c[i - 1] is the previous lane's bound below c[i]: one
    // search per particle, and one more per warp (the loop bound is the same
    // for the whole CTA, so every lane takes part in the shuffle)
    for (uint64_t b = static_cast<uint64_t>(blockIdx.x) * blockDim.x; b < N;
         b += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t i = b + threadIdx.x;
        uint64_t cur = 0;
        if (i < N) cur = (i + 1 == N) ? M : lower_bound(u, M, c[i]);
        uint64_t prev = __shfl_up_sync(0xffffffffu, cur, 1);
        if (i < N) {
            if ((threadIdx.x & 31) == 0) prev = i == 0 ? 0 : lower_bound(u, M, c[i - 1]);
            rep[i] = cur - prev;
            if (ties && i + 1 < N) {
                const double ci = c[i];
                nt += lower_bound_from(u, M, next_up(next_up(ci)), cur) - lower_bound_from(u, M, next_down(ci), cur);
            }
        }
    }
    if (ties) {
        nt = block_sum(nt, sh);
        if (threadIdx.x == 0 && nt) atomicAdd(ties, nt);
    }
}

__global__ void k_residual_split(uint64_t N, uint64_t M, const double *W, double *resid, uint64_t *integ,
    unsigned long long *isum)
{
    __shared__ unsigned long long sh[33];
    const double coeff = static_cast<double>(M);
    unsigned long long acc = 0;
    GRID_LOOP(i, N)
    {
        const double w = __dmul_rn(coeff, W[i]);
        double ip;
        resid[i] = modf(w, &ip);
        integ[i] = static_cast<uint64_t>(ip);
        acc += static_cast<unsigned long long>(ip);
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) atomicAdd(isum, acc);
}

__global__ void k_residual_scale(uint64_t N, double *resid, const double *sum)
{
    const double mul = __ddiv_rn(1.0, *sum);
    GRID_LOOP(i, N) { resid[i] = __dmul_rn(resid[i], mul); }
}

__global__ void k_add_integ(uint64_t N, uint64_t *rep, const uint64_t *integ)
{
    GRID_LOOP(i, N) { rep[i] += integ[i]; }
}

__global__ void k_fill_rep(uint64_t N, uint64_t M, uint64_t *rep)
{
    pdl_wait();
    GRID_LOOP(i, N) { rep[i] = (N == 1) ? M : 0; }
}

// ---------------------------------------------------------------------------
// rep -> index
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;
constexpr unsigned long long kFlagAgg = 1ull << 62, kFlagInc = 2ull << 62, kValMask = (1ull << 62) - 1;
constexpr long long kSpinLimit = 1ll << 22;  // look-back rounds (each a CTA barrier)

// pair of 31-bit counters packed into 62 bits: low = empties, high = surplus
__device__ __forceinline__ unsigned long long pack(unsigned long long e, unsigned long long s)
{
    return e | (s << 31);
}

// shared-memory index of element o of a scan tile: one pad word per 16
// elements, so the blocked reads (thread t, elements 8t..8t+7) hit distinct
// bank pairs except for a 2-way overlap
__device__ __forceinline__ unsigned scan_pad(unsigned o)
{
    return o + (o >> 4);
}

// Per tile of kScanTile counts: the exclusive prefixes of (empty slot, surplus)
// pairs, and every G-th surplus prefix into `coarse`.  Loads and stores are coalesced through shared memory; each thread
// scans kScanPer consecutive elements.  The tile's offset comes from a
// decoupled look-back done by the whole CTA: its threads read the statuses of
// kScanThreads predecessors at once, wait while any is unpublished, and add
// the aggregates back to the nearest inclusive prefix (tiles before tile 0
// read as an inclusive 0), so with every tile in flight at once a look-back
// takes tiles / kScanThreads rounds.  Tiles are numbered in the order the
// CTAs start (an atomic counter), so every predecessor is running or done.
// The wait is bounded: past kSpinLimit rounds the error word is set and the
// result is invalid (the host reports it).
__global__ void __launch_bounds__(kScanThreads) k_rep_scan(uint64_t N, uint64_t K, const uint64_t *rep,
    uint32_t *ex_empty, uint32_t *ex_surplus, unsigned long long *status, unsigned *tile_counter, int *err,
    uint64_t G, uint32_t *coarse)
{
    pdl_wait();
    __shared__ unsigned long long sh[33];
    __shared__ unsigned shu[33];
    __shared__ unsigned long long sv[kScanTile + kScanTile / 16];
    __shared__ unsigned long long sh_excl;
    __shared__ unsigned sh_tile;
    if (threadIdx.x == 0) sh_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint64_t tile = sh_tile;
    const uint64_t base = tile * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const unsigned o = k * kScanThreads + threadIdx.x;
        const uint64_t i = base + o;
        unsigned long long e = 0, sp = 0;
        if (i < N) {
            const uint64_t r = rep[i];
            if (i < K) {
                e = (r == 0);
                sp = r > 0 ? r - 1 : 0;
            } else {
                sp = r;
            }
        }
        sv[scan_pad(o)] = pack(e, sp);
    }
    __syncthreads();
    unsigned long long v[kScanPer];
    unsigned long long own = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = sv[scan_pad(threadIdx.x * kScanPer + k)];
        own += v[k];
    }
    unsigned long long agg;
    const unsigned long long incl = block_inclusive_sum(own, sh, &agg);
    if (tile == 0) {
        if (threadIdx.x == 0) {
            atomicExch(&status[0], kFlagInc | agg);
            sh_excl = 0;
        }
    } else {
        if (threadIdx.x == 0) atomicExch(&status[tile], kFlagAgg | agg);
        long long p = static_cast<long long>(tile) - 1;
        long long spins = 0;
        bool failed = false;
        unsigned long long excl = 0;
        for (;;) {
            const long long q = p - static_cast<long long>(threadIdx.x);
            unsigned long long st = 2ull << 62;  // kFlagInc, value 0
            if (q >= 0) st = *reinterpret_cast<volatile unsigned long long *>(&status[q]);
            const unsigned long long fl = st & ~kValMask;
            if (__syncthreads_or(fl == 0)) {
                if (++spins > kSpinLimit) {
                    failed = true;
                    break;
                }
                continue;
            }
            const unsigned first = block_min_u32(fl == kFlagInc ? threadIdx.x : 0xffffffffu, shu);
            excl += block_sum(threadIdx.x <= first ? (st & kValMask) : 0ull, sh);
            if (first != 0xffffffffu) break;
            p -= kScanThreads;
        }
        if (threadIdx.x == 0) {
            if (failed) atomicExch(err, 1);
            atomicExch(&status[tile], kFlagInc | (excl + agg));
            sh_excl = excl;
        }
    }
    __syncthreads();
    unsigned long long run = sh_excl + incl - own;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        sv[scan_pad(threadIdx.x * kScanPer + k)] = run;
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        const unsigned o = k * kScanThreads + threadIdx.x;
        const uint64_t i = base + o;
        if (i < N) {
            const unsigned long long x = sv[scan_pad(o)];
            const uint32_t sp = static_cast<uint32_t>((x >> 31) & 0x7fffffffull);
            ex_empty[i] = static_cast<uint32_t>(x & 0x7fffffffull);
            ex_surplus[i] = sp;
            if (i % G == 0) coarse[i / G] = sp;
        }
    }
}

// occupied slots keep their particle; empty slots < K and all slots >= K are
// listed in ascending order
__global__ void k_rep_place(uint64_t N, uint64_t M, uint64_t K, const uint64_t *rep, const uint32_t *ex_empty,
    uint64_t *idx, uint32_t *empty_pos)
{
    pdl_wait();
    const uint64_t n_empty_k = (K == 0) ? 0 : ex_empty[K - 1] + (rep[K - 1] == 0 ? 1 : 0);
    GRID_LOOP(d, M)
    {
        if (d < K) {
            if (rep[d] > 0) {
                idx[d] = d;
            } else {
                empty_pos[ex_empty[d]] = static_cast<uint32_t>(d);
            }
        } else {
            empty_pos[n_empty_k + (d - K)] = static_cast<uint32_t>(d);
        }
    }
}

// The k-th empty slot takes the source whose surplus range holds k: the last
// s with ex_surplus[s] <= k.  One wave of CTAs, each taking 256 consecutive
// empties per round.  A CTA first loads the coarse table of the prefixes,
// coarse[j] = ex_surplus[j G] (at most kCoarse entries, written by the scan),
// and finds in it the cells holding the sources of its first and last empty;
// those bound the sources of all of its empties (ex_surplus is
// nondecreasing).  A bracket of at most kFillStage sources is staged with
// coalesced loads and every lane searches it in shared memory; a wider one is
// searched in global memory, still only between the bounds.
constexpr int kFillThreads = 256, kFillStage = 4096, kCoarse = 2048;

uint64_t coarse_step(uint64_t N)
{
    return std::max<uint64_t>(1, (N + kCoarse - 1) / kCoarse);
}

__device__ __forceinline__ uint64_t surplus_owner(const uint32_t *ex_surplus, uint64_t lo, uint64_t hi, uint64_t k)
{
    // ex_surplus[lo] <= k and (hi == N or ex_surplus[hi] > k)
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (ex_surplus[mid] <= k) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

__global__ void __launch_bounds__(kFillThreads) k_rep_fill(uint64_t N, uint64_t M, uint64_t K, const uint64_t *rep,
    const uint32_t *ex_empty, const uint32_t *ex_surplus, const uint32_t *empty_pos, uint64_t G,
    const uint32_t *coarse, uint64_t *idx)
{
    pdl_wait();
    __shared__ uint32_t sx[kFillStage];
    __shared__ uint32_t sc[kCoarse];
    __shared__ unsigned sh_b[2];
    const uint64_t n_empty = (K == 0 ? 0 : ex_empty[K - 1] + (rep[K - 1] == 0 ? 1 : 0)) + (M - K);
    if (static_cast<uint64_t>(blockIdx.x) * kFillThreads >= n_empty) return;
    const unsigned C = static_cast<unsigned>((N + G - 1) / G);
    for (unsigned j = threadIdx.x; j < C; j += kFillThreads) sc[j] = coarse[j];
    __syncthreads();
    for (uint64_t k0 = static_cast<uint64_t>(blockIdx.x) * kFillThreads; k0 < n_empty;
         k0 += static_cast<uint64_t>(gridDim.x) * kFillThreads) {
        const uint64_t klast = std::min<uint64_t>(n_empty, k0 + kFillThreads) - 1;
        const uint64_t k = k0 + threadIdx.x;
        const uint32_t dst = k <= klast ? empty_pos[k] : 0;  // issued before the searches
        if (threadIdx.x < 2) {
            const uint64_t kk = threadIdx.x == 0 ? k0 : klast;
            unsigned lo = 0, hi = C;  // sc[0] = 0 <= kk
            while (hi - lo > 1) {
                const unsigned mid = (lo + hi) >> 1;
                if (sc[mid] <= kk) {
                    lo = mid;
                } else {
                    hi = mid;
                }
            }
            sh_b[threadIdx.x] = lo;
        }
        __syncthreads();
        const uint64_t slo = sh_b[0] * G, shi = std::min<uint64_t>(N, (sh_b[1] + 1ull) * G);
        const uint64_t len = shi - slo;
        if (len <= kFillStage) {
            for (uint64_t j = threadIdx.x; j < len; j += kFillThreads) sx[j] = ex_surplus[slo + j];
            __syncthreads();
            if (k <= klast) {
                unsigned lo = 0, hi = static_cast<unsigned>(len);
                while (hi - lo > 1) {
                    const unsigned mid = (lo + hi) >> 1;
                    if (sx[mid] <= k) {
                        lo = mid;
                    } else {
                        hi = mid;
                    }
                }
                idx[dst] = slo + lo;
            }
        } else if (k <= klast) {
            idx[dst] = surplus_owner(ex_surplus, slo, shi, k);
        }
        __syncthreads();  // sx and sh_b are rewritten by the next round
    }
}

// idx[i] == i for every occupied slot, and a copy reads only occupied slots,
// so no slot is read after it is written
template <typename T>
__global__ void k_select_inplace(uint64_t N, uint64_t dim, const uint64_t *idx, T *state)
{
    pdl_wait();
    GRID_LOOP(i, N)
    {
        const uint64_t src = idx[i];
        if (src != i)
            for (uint64_t d = 0; d < dim; ++d) state[d * N + i] = state[d * N + src];
    }
}

template <typename T>
__global__ void k_select_copy(uint64_t N, uint64_t M, uint64_t dim, const uint64_t *idx, const T *in, T *out)
{
    pdl_wait();
    GRID_LOOP(i, M)
    {
        const uint64_t src = idx[i];
        for (uint64_t d = 0; d < dim; ++d) out[d * M + i] = in[d * N + src];
    }
}

template <class Fn>
int with_gen(const mckl_b200_engine_t &e, Fn &&fn)
{
    switch (e.kind) {
        case MCKL_B200_PHILOX4X32: {
            PhiloxGen g{static_cast<uint32_t>(e.key[0]), static_cast<uint32_t>(e.key[1])};
            return fn(g);
        }
        case MCKL_B200_THREEFRY4X64: {
            ThreefryGen g = ThreefryGen::make(e.key, e.tweak);
            return fn(g);
        }
        case MCKL_B200_ARS: {
            ArsGen g = ArsGen::make(e.key);
            return fn(g);
        }
        default:
            set_error("resampling needs an engine with 32-bit results (Philox4x32, Threefry4x64, ARS)");
            return MCKL_B200_ERR_ARG;
    }
}

}  // namespace

size_t resample_scratch_bytes(uint64_t N, uint64_t M)
{
    const uint64_t L = std::max<uint64_t>(std::max<uint64_t>(N, M), 1);
    return 1024 + 3 * align256(L * sizeof(double)) + align256(L * sizeof(uint64_t)) + fold_scratch_bytes(L);
}

// Uniform sequence `kind` (0 sorted, 1 stratified, 2 systematic) of length n
// into u (device); advances the engine as the reference's calls do.
int u01_sequence_dev(int kind, mckl_b200_engine_t &e, uint64_t n, double *u, double *tmp, FoldScratch &fs,
    cudaStream_t s)
{
    Ctr B;
    uint32_t off;
    next_position(e, B, off);
    if (kind == 2) {
        const int rc = with_gen(e, [&](auto g) {
            using G = decltype(g);
            k_systematic<G><<<cap_grid(std::max<uint64_t>(n, 1), 256), 256, G::kDynSmem, s>>>(g, B, off, n, u);
            MB_LAUNCH_CHECK();
            return MCKL_B200_OK;
        });
        if (rc != MCKL_B200_OK) return rc;
        advance_call(e, 1);  // U01Distribution<double>{}(rng): two single-word draws
        advance_call(e, 1);
        return MCKL_B200_OK;
    }
    if (n == 0) return MCKL_B200_OK;
    int rc = with_gen(e, [&](auto g) {
        using G = decltype(g);
        k_canonical<G><<<cap_grid(n, 256), 256, G::kDynSmem, s>>>(g, B, off, n, u);
        MB_LAUNCH_CHECK();
        return MCKL_B200_OK;
    });
    if (rc != MCKL_B200_OK) return rc;
    // per 1024-chunk: u01_canonical_distribution -> one call of 2 words per value
    advance_calls(e, n / 1024, 2048);
    advance_call(e, 2 * (n % 1024));
    if (kind == 1) {
        k_stratified<<<cap_grid(n, 256), 256, 0, s>>>(n, u);
        MB_LAUNCH_CHECK();
        return MCKL_B200_OK;
    }
    k_sorted_terms<<<cap_grid(n, 256), 256, 0, s>>>(n, u);
    MB_LAUNCH_CHECK();
    rc = fold_exact(u, n, 0.0, tmp, fs, s);
    if (rc != MCKL_B200_OK) return rc;
    k_sorted_finish<<<cap_grid(n, 256), 256, 0, s>>>(n, tmp, u);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

int resample_dev(int scheme, uint64_t N, uint64_t M, mckl_b200_engine_t &e, const double *W, uint64_t *rep,
    void *scratch_base, cudaStream_t s, unsigned long long *ties_dev)
{
    static const int seq_of[6] = {0, 1, 2, 0, 1, 2};
    const int seq = seq_of[scheme];
    const uint64_t L = std::max<uint64_t>(std::max<uint64_t>(N, M), 1);
    char *p = static_cast<char *>(scratch_base);
    unsigned long long *isum = reinterpret_cast<unsigned long long *>(p);
    double *rsum = reinterpret_cast<double *>(p + 64);
    p += 1024;
    double *u = reinterpret_cast<double *>(p);
    p += align256(L * sizeof(double));
    double *tmp = reinterpret_cast<double *>(p);
    p += align256(L * sizeof(double));
    double *resid = reinterpret_cast<double *>(p);
    p += align256(L * sizeof(double));
    uint64_t *integ = reinterpret_cast<uint64_t *>(p);
    p += align256(L * sizeof(uint64_t));
    FoldScratch fs = fold_scratch_carve(p, L);
    const double *weights = W;
    uint64_t R = M;
    if (scheme >= 3) {
        MB_CUDA(cudaMemsetAsync(isum, 0, sizeof(unsigned long long), s));
        k_residual_split<<<cap_grid(N, 256), 256, 0, s>>>(N, M, W, resid, integ, isum);
        MB_LAUNCH_CHECK();
        int rc = fold_exact(resid, N, 0.0, nullptr, fs, s);
        if (rc != MCKL_B200_OK) return rc;
        MB_CUDA(cudaMemcpyAsync(rsum, fs.final_v, sizeof(double), cudaMemcpyDeviceToDevice, s));
        k_residual_scale<<<cap_grid(N, 256), 256, 0, s>>>(N, resid, rsum);
        MB_LAUNCH_CHECK();
        unsigned long long h = 0;
        MB_CUDA(cudaMemcpyAsync(&h, isum, sizeof(h), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        R = M - h;  // the count of uniforms decides the engine's consumption
        weights = resid;
    }
    int rc = u01_sequence_dev(seq, e, R, u, tmp, fs, s);
    if (rc != MCKL_B200_OK) return rc;
    if (N <= 1 || R == 0) {
        MB_CUDA(launch_pdl(k_fill_rep, cap_grid(N, 256), 256, 0, s, N, R, rep));
        MB_LAUNCH_CHECK();
    } else {
        rc = fold_exact(weights, N - 1, 0.0, tmp, fs, s);  // cumulative weights of particles 0..N-2
        if (rc != MCKL_B200_OK) return rc;
        MB_CUDA(launch_pdl(k_rep_counts, cap_grid(N, 256), 256, 0, s, N, R, tmp, u, rep, ties_dev));
        MB_LAUNCH_CHECK();
    }
    if (scheme >= 3) {
        k_add_integ<<<cap_grid(N, 256), 256, 0, s>>>(N, rep, integ);
        MB_LAUNCH_CHECK();
    }
    return MCKL_B200_OK;
}

ResampleScratch resample_scratch_carve(void *scratch_base, uint64_t N, uint64_t M)
{
    const uint64_t L = std::max<uint64_t>(std::max<uint64_t>(N, M), 1);
    char *p = static_cast<char *>(scratch_base) + 1024;
    ResampleScratch r;
    r.u = reinterpret_cast<double *>(p);
    r.tmp = reinterpret_cast<double *>(p + align256(L * sizeof(double)));
    r.fs = fold_scratch_carve(p + 3 * align256(L * sizeof(double)) + align256(L * sizeof(uint64_t)), L);
    return r;
}

int rep_counts_dev(uint64_t N, uint64_t M, const double *W, const double *u, uint64_t *rep, ResampleScratch &rs,
    cudaStream_t s, unsigned long long *ties_dev)
{
    if (N <= 1 || M == 0) {
        MB_CUDA(launch_pdl(k_fill_rep, cap_grid(N, 256), 256, 0, s, N, M, rep));
        MB_LAUNCH_CHECK();
        return MCKL_B200_OK;
    }
    int rc = fold_exact(W, N - 1, 0.0, rs.tmp, rs.fs, s);  // cumulative weights of particles 0..N-2
    if (rc != MCKL_B200_OK) return rc;
    MB_CUDA(launch_pdl(k_rep_counts, cap_grid(N, 256), 256, 0, s, N, M, rs.tmp, u, rep, ties_dev));
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

size_t rep_index_scratch_bytes(uint64_t N, uint64_t M)
{
    const uint64_t tiles = (N + kScanTile - 1) / kScanTile + 1;
    return 256 + align256(tiles * sizeof(unsigned long long)) + 2 * align256(N * sizeof(uint32_t)) +
           align256(M * sizeof(uint32_t)) + align256(kCoarse * sizeof(uint32_t)) + 256;
}

int rep_to_index_dev(uint64_t N, uint64_t M, const uint64_t *rep, uint64_t *idx, void *scratch_base, int *err_dev,
    cudaStream_t s)
{
    if (N == 0 || M == 0) return MCKL_B200_OK;
    const uint64_t K = std::min(N, M);
    const uint64_t tiles = (N + kScanTile - 1) / kScanTile;
    char *p = static_cast<char *>(scratch_base);
    unsigned *tile_counter = reinterpret_cast<unsigned *>(p);
    p += 256;
    unsigned long long *status = reinterpret_cast<unsigned long long *>(p);
    p += align256((tiles + 1) * sizeof(unsigned long long));
    uint32_t *ex_empty = reinterpret_cast<uint32_t *>(p);
    p += align256(N * sizeof(uint32_t));
    uint32_t *ex_surplus = reinterpret_cast<uint32_t *>(p);
    p += align256(N * sizeof(uint32_t));
    uint32_t *empty_pos = reinterpret_cast<uint32_t *>(p);
    p += align256(M * sizeof(uint32_t));
    uint32_t *coarse = reinterpret_cast<uint32_t *>(p);
    const uint64_t G = coarse_step(N);
    MB_CUDA(cudaMemsetAsync(scratch_base, 0, 256 + align256((tiles + 1) * sizeof(unsigned long long)), s));
    k_rep_scan<<<static_cast<unsigned>(tiles), kScanThreads, 0, s>>>(N, K, rep, ex_empty, ex_surplus, status,
        tile_counter, err_dev, G, coarse);
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_rep_place, cap_grid(M, 256), 256, 0, s, N, M, K, rep, ex_empty, idx, empty_pos));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_rep_fill, cap_grid(M, kFillThreads, 8), kFillThreads, 0, s, N, M, K, rep, ex_empty, ex_surplus, empty_pos,
        G, coarse, idx));
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

template <typename T>
int select_dev(uint64_t N, uint64_t M, uint64_t dim, const uint64_t *idx, const T *in, T *out, cudaStream_t s)
{
    if (N == M && in == out) {
        k_select_inplace<T><<<cap_grid(N, 256), 256, 0, s>>>(N, dim, idx, out);
    } else {
        k_select_copy<T><<<cap_grid(M, 256), 256, 0, s>>>(N, M, dim, idx, in, out);
    }
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

template int select_dev<double>(uint64_t, uint64_t, uint64_t, const uint64_t *, const double *, double *,
    cudaStream_t);
template int select_dev<float>(uint64_t, uint64_t, uint64_t, const uint64_t *, const float *, float *,
    cudaStream_t);

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" {

int mckl_b200_u01_sequence(int kind, mckl_b200_engine_t *e, size_t n, double *u, void *stream)
{
    MB_CHECK_ARG(kind >= 0 && kind <= 2, "kind: 0 sorted, 1 stratified, 2 systematic");
    MB_CHECK_ARG(e != nullptr && kind_valid(e->kind), "invalid engine");
    MB_CHECK_ARG(n == 0 || u != nullptr, "null output");
    cudaStream_t s = as_stream(stream);
    void *base = scratch(3, resample_scratch_bytes(n, n), s);
    if (!base) {
        set_error("scratch allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    const size_t L = std::max<size_t>(n, 1);
    char *p = static_cast<char *>(base) + 1024;
    double *tmp = reinterpret_cast<double *>(p);
    FoldScratch fs = fold_scratch_carve(p + 3 * align256(L * sizeof(double)) + align256(L * sizeof(uint64_t)), L);
    return u01_sequence_dev(kind, *e, n, u, tmp, fs, s);
}

int mckl_b200_resample(int scheme, size_t N, size_t M, mckl_b200_engine_t *rng, const double *W, uint64_t *rep,
    void *stream)
{
    MB_CHECK_ARG(scheme >= 0 && scheme <= 5, "scheme must be 0..5");
    MB_CHECK_ARG(rng != nullptr && kind_valid(rng->kind), "invalid engine");
    MB_CHECK_ARG(N == 0 || (W != nullptr && rep != nullptr), "null pointer");
    MB_CHECK_ARG(N < (1ull << 31) && M < (1ull << 31), "N and M must be below 2^31");
    if (N == 0) return MCKL_B200_OK;
    cudaStream_t s = as_stream(stream);
    void *base = scratch(3, resample_scratch_bytes(N, M), s);
    if (!base) {
        set_error("scratch allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    return resample_dev(scheme, N, M, *rng, W, rep, base, s);
}

int mckl_b200_rep_to_index(size_t N, size_t M, const uint64_t *rep, uint64_t *idx, void *stream)
{
    MB_CHECK_ARG(N == 0 || M == 0 || (rep != nullptr && idx != nullptr), "null pointer");
    MB_CHECK_ARG(N < (1ull << 31) && M < (1ull << 31), "N and M must be below 2^31");
    cudaStream_t s = as_stream(stream);
    void *base = scratch(4, rep_index_scratch_bytes(N, M) + 64, s);
    if (!base) {
        set_error("scratch allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    int *err = reinterpret_cast<int *>(static_cast<char *>(base) + rep_index_scratch_bytes(N, M));
    MB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    int rc = rep_to_index_dev(N, M, rep, idx, base, err, s);
    if (rc != MCKL_B200_OK) return rc;
    int h = 0;
    MB_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    if (h) {
        set_error("rep_to_index: look-back wait exceeded its limit");
        return MCKL_B200_ERR_DEVICE;
    }
    return MCKL_B200_OK;
}

int mckl_b200_select_f64(size_t N, size_t dim, const uint64_t *idx, double *state, void *stream)
{
    MB_CHECK_ARG(N == 0 || dim == 0 || (idx != nullptr && state != nullptr), "null pointer");
    return select_dev<double>(N, N, dim, idx, state, state, as_stream(stream));
}

int mckl_b200_select_f32(size_t N, size_t dim, const uint64_t *idx, float *state, void *stream)
{
    MB_CHECK_ARG(N == 0 || dim == 0 || (idx != nullptr && state != nullptr), "null pointer");
    return select_dev<float>(N, N, dim, idx, state, state, as_stream(stream));
}

}  // extern "C"
