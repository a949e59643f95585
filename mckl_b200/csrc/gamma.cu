// gamma.cu -- Gamma(alpha, beta) transform of an engine stream, exactly as
// the reference's gamma_distribution (random/gamma_distribution.hpp:57-302).
//
// The reference draws in chunks of K = 8192 / sizeof(R) values: one chunk
// consumes a fixed block of engine words (2K uniforms for the T and W
// algorithms, K uniforms + K normals for N, K uniforms for E), keeps the
// accepted values in order, and repeats while more than K values are missing;
// a last chunk covers the remainder and a scalar loop fills what that chunk
// rejected.  Algorithm N also redraws, one scalar normal at a time, every
// normal whose v = 1 + c w is not positive, so its word consumption depends on
// the data.  How many chunks a call needs, and where each chunk's words start,
// therefore depend on the previous chunks: the chunks of one stream run in
// order.  A CTA owns one stream and processes each chunk with all its
// threads: the chunk's words are staged in shared memory, every thread
// transforms K / THREADS values, the N redraws are assigned in index order by
// one warp (the scalar normals they consume form one sequence, evaluated 64 at
// a time), and the accepted values are compacted with a CTA-wide rank.
// Independent streams (gamma_blocks: one stream per block of samples, each on
// its own counter range) run one per CTA across the GPU.
//
// Math: double uses the correctly rounded double-double log/exp/sin/cos of
// crmath.cuh; float evaluates log/exp/sin/cos in double and rounds once (a
// correctly rounded float result except in double-rounding cases, about one
// in 2^28).  Every multiply and add is an explicit _rn operation, fma only
// where the reference calls fma.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "block_scan.cuh"
#include "common.cuh"
#include "dispatch.cuh"
#include "transforms.cuh"

namespace mckl_b200 {

namespace {

template <typename R>
struct GOps;

template <>
struct GOps<double> {
    static constexpr double kTwoPi = 0x1.921fb54442d18p+2;
    static constexpr double k0331 = 0.0331;
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ static double div(double a, double b) { return __ddiv_rn(a, b); }
    __device__ static double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    __device__ static double log(double a) { return dd::log(a); }
    __device__ static double exp(double a) { return dd::exp(a); }
    __device__ static double sqrt(double a) { return __dsqrt_rn(a); }
    __device__ static void sincos(double a, double *s, double *c) { dd::sincos(a, s, c); }
};

template <>
struct GOps<float> {
    static constexpr float kTwoPi = 0x1.921fb6p+2f;
    static constexpr float k0331 = 0.0331f;
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static float div(float a, float b) { return __fdiv_rn(a, b); }
    __device__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    __device__ static float log(float a) { return __double2float_rn(::log(static_cast<double>(a))); }
    __device__ static float exp(float a) { return __double2float_rn(::exp(static_cast<double>(a))); }
    __device__ static float sqrt(float a) { return __fsqrt_rn(a); }
    __device__ static void sincos(float a, float *s, float *c)
    {
        double sd, cd;
        ::sincos(static_cast<double>(a), &sd, &cd);
        *s = __double2float_rn(sd);
        *c = __double2float_rn(cd);
    }
};

// Per-stream constants of GammaDistributionConstant (:57-96), computed on the
// host with the same libm as the reference.
template <typename R>
struct GammaParam {
    R alpha, beta, d, c;
    int alg;  // 0 T (alpha < 0.6), 1 W (alpha < 1), 2 N (alpha > 1), 3 E (alpha == 1)
};

template <typename R>
GammaParam<R> gamma_param(R alpha, R beta)
{
    GammaParam<R> k{alpha, beta, 0, 0, 0};
    if (alpha < static_cast<R>(0.6)) {
        k.alg = 0;
        k.d = 1 - alpha;
        k.c = 1 / alpha;
    } else if (alpha < 1) {
        k.alg = 1;
        const R t = alpha / (1 - alpha);
        k.d = std::pow(alpha, t) * (1 - alpha);
        k.c = 1 / alpha;
    } else if (alpha > 1) {
        k.alg = 2;
        k.d = alpha - static_cast<R>(1) / 3;
        k.c = 1 / (3 * std::sqrt(k.d));
    } else {
        k.alg = 3;
    }
    return k;
}

// CounterEngine state (counter, buffer index) of one stream inside a CTA,
// advanced call by call exactly like the host bookkeeping (advance_call), so
// the representation after the call matches the reference's.
template <int CW>
struct DevEngine {
    Ctr ctr;
    uint32_t idx;

    __device__ void call(uint64_t n, uint32_t M)
    {
        const uint64_t id = idx < M ? idx : M;
        const uint64_t remain = M - id;
        if (n <= remain) {
            idx = static_cast<uint32_t>(id + n);
            return;
        }
        const uint64_t rem2 = n - remain, m = rem2 / M;
        ctr = ctr_add(ctr, m + 1, CW);
        idx = static_cast<uint32_t>(rem2 - m * M);
    }

    // u01_batch of n values from one-word conversions: n / K calls of K
    // (each followed by an empty call) and one of n % K
    __device__ void batch(uint64_t n, uint64_t K, uint32_t M)
    {
        for (uint64_t i = 0; i < n / K; ++i) {
            call(K, M);
            call(0, M);
        }
        call(n % K, M);
    }
};

// Scalar word reader for one thread: word k of the stream (k counted from the
// stream's first word at block B, offset off), one cached block.
template <class G, typename W>
struct ScalarWords {
    static constexpr int WPB = G::kWords / WordView<W>::kPer32;
    const G *g;
    Ctr B;
    uint32_t off;
    uint64_t cached = ~0ull;
    uint32_t blk[G::kWords];

    __device__ W at(uint64_t k)
    {
        const uint64_t a = off + k, b = a / WPB;
        if (b != cached) {
            g->block(ctr_add(B, b, G::kCtrWords), blk);
            cached = b;
        }
        const int j = static_cast<int>(a % WPB);
        W r = 0;
#pragma unroll
        for (int q = 0; q < WPB; ++q)
            if (q == j) r = WordView<W>::get(blk, q);
        return r;
    }
};

// CTA-wide ranks of E predicates per thread in index order, element (t, j)
// having index t + j THREADS: rank[j] = the number of set elements with a
// smaller index, *total the CTA count.  Three barriers for all E (one ballot
// per j; warp 0 scans the E x warps counts).  `sh` holds E THREADS / 32 + 1
// words (at most 64 + 1).
template <int THREADS, int E>
__device__ __forceinline__ void block_rank_multi(const bool (&f)[E], uint32_t *sh, uint32_t (&rank)[E],
    uint32_t *total)
{
    constexpr int NW = THREADS / 32, L = E * NW;
    static_assert(L <= 64, "two counts per lane of warp 0");
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t b[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
        b[j] = __ballot_sync(0xffffffffu, f[j]);
        if (lane == 0) sh[j * NW + warp] = __popc(b[j]);
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t a0 = lane < static_cast<uint32_t>(L) ? sh[lane] : 0u;
        const uint32_t a1 = lane + 32 < static_cast<uint32_t>(L) ? sh[lane + 32] : 0u;
        const uint32_t s0 = warp_inclusive_sum(a0);
        const uint32_t t0 = __shfl_sync(0xffffffffu, s0, 31);
        const uint32_t s1 = warp_inclusive_sum(a1) + t0;
        const uint32_t t1 = __shfl_sync(0xffffffffu, s1, 31);
        __syncwarp();
        if (lane < static_cast<uint32_t>(L)) sh[lane] = s0 - a0;
        if (lane + 32 < static_cast<uint32_t>(L)) sh[lane + 32] = s1 - a1;
        if (lane == 0) sh[L] = t1;
    }
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < E; ++j) rank[j] = sh[j * NW + warp] + __popc(b[j] & lt);
    *total = sh[L];
    __syncthreads();  // `sh` is rewritten by the next call
}

// Scalar normal with the cached second variate (random/normal_distribution.hpp:136-153).
template <typename R>
struct ScalarNormal {
    R saved = 0;
    bool has = false;

    template <class SW>
    __device__ R operator()(SW &sw, uint64_t &k)
    {
        using O = GOps<R>;
        R z;
        if (has) {
            z = saved;
            has = false;
        } else {
            const R a = RealOps<R>::u01(kOC, sw.at(k++));
            const R u1 = O::sqrt(O::mul(static_cast<R>(-2), O::log(a)));
            const R b = RealOps<R>::u01(kOC, sw.at(k++));
            const R u2 = O::mul(O::kTwoPi, b);
            R sn, cs;
            O::sincos(u2, &sn, &cs);
            z = O::mul(u1, cs);
            saved = O::mul(u1, sn);
            has = true;
        }
        return O::add(static_cast<R>(0), O::mul(static_cast<R>(1), z));
    }
};

// Algorithm N's acceptance test of one attempt (uniform u, normal w with
// v = 1 + c w > 0); *r = d v^3 when accepted.
template <typename R>
__device__ __forceinline__ bool gamma_n_accept(const GammaParam<R> &k, R u, R w, R v, R *r)
{
    using O = GOps<R>;
    v = O::mul(O::mul(v, v), v);
    const R w2 = O::mul(w, w);
    R e = O::sub(static_cast<R>(1), O::mul(O::mul(O::k0331, w2), w2));
    if (u < e) {
        *r = O::mul(k.d, v);
        return true;
    }
    e = O::add(O::div(w2, static_cast<R>(2)), O::mul(k.d, O::add(O::sub(static_cast<R>(1), v), O::log(v))));
    if (O::log(u) < e) {
        *r = O::mul(k.d, v);
        return true;
    }
    return false;
}

// GammaDistribution::generate_{t,w,n,e} (:350-459), the scalar fallback.
template <typename R, int ALG, class SW>
__device__ R gamma_scalar(const GammaParam<R> &k, SW &sw, uint64_t &pos)
{
    using O = GOps<R>;
    const R d = k.d, c = k.c;
    R r = 0;
    switch (ALG) {
        case 0:
            for (;;) {
                R u = O::sub(static_cast<R>(1), RealOps<R>::u01(kOO, sw.at(pos++)));
                R e = -O::log(RealOps<R>::u01(kOO, sw.at(pos++)));
                if (u > d) {
                    u = -O::log(O::mul(c, O::sub(static_cast<R>(1), u)));
                    e = O::add(e, u);
                    u = O::add(d, O::mul(k.alpha, u));
                }
                r = O::exp(O::mul(c, O::log(u)));
                if (fabs(r) < e) break;
            }
            break;
        case 1: {
            R u, e;
            do {
                u = -O::log(RealOps<R>::u01(kOO, sw.at(pos++)));
                e = -O::log(RealOps<R>::u01(kOO, sw.at(pos++)));
                r = O::exp(O::mul(c, O::log(u)));
            } while (O::add(u, e) < O::add(d, r));
            break;
        }
        case 2: {
            ScalarNormal<R> rn;
            for (;;) {
                const R u = RealOps<R>::u01(kOO, sw.at(pos++));
                R w, v;
                do {
                    w = rn(sw, pos);
                    v = O::add(static_cast<R>(1), O::mul(c, w));
                } while (v <= 0);
                if (gamma_n_accept(k, u, w, v, &r)) break;
            }
            break;
        }
        default:
            r = -O::log(RealOps<R>::u01(kOO, sw.at(pos++)));
            break;
    }
    return O::mul(k.beta, r);
}

// One attempt of algorithm T (0), W (1) or E (3) of the scalar fallback from
// the words at pos, pos + 1 (E: pos only): these algorithms consume a fixed
// number of words per attempt (kAttemptWords), so attempt j of the fallback
// reads words pos0 + kAttemptWords j whatever the earlier attempts did.
// Returns whether the attempt is accepted; *out = beta r.  The same
// arithmetic as gamma_scalar's loop bodies.
template <int ALG>
struct GammaAttemptWords {
    static constexpr int value = ALG == 3 ? 1 : 2;
};

template <typename R, int ALG, class SW>
__device__ bool gamma_attempt(const GammaParam<R> &k, SW &sw, uint64_t pos, R *out)
{
    using O = GOps<R>;
    const R d = k.d, c = k.c;
    R r;
    bool acc;
    if constexpr (ALG == 0) {
        R u = O::sub(static_cast<R>(1), RealOps<R>::u01(kOO, sw.at(pos)));
        R e = -O::log(RealOps<R>::u01(kOO, sw.at(pos + 1)));
        if (u > d) {
            u = -O::log(O::mul(c, O::sub(static_cast<R>(1), u)));
            e = O::add(e, u);
            u = O::add(d, O::mul(k.alpha, u));
        }
        r = O::exp(O::mul(c, O::log(u)));
        acc = fabs(r) < e;
    } else if constexpr (ALG == 1) {
        const R u = -O::log(RealOps<R>::u01(kOO, sw.at(pos)));
        const R e = -O::log(RealOps<R>::u01(kOO, sw.at(pos + 1)));
        r = O::exp(O::mul(c, O::log(u)));
        acc = !(O::add(u, e) < O::add(d, r));
    } else {
        r = -O::log(RealOps<R>::u01(kOO, sw.at(pos)));
        acc = true;
    }
    *out = O::mul(k.beta, r);
    return acc;
}

// The scalar fallback of algorithms T, W and E on one warp: the warp
// evaluates 32 consecutive attempts at a time and the accepted ones fill the
// `left` outputs in attempt order, which is what the sequential loop of
// gamma_scalar produces.  Returns the words consumed (all lanes agree).
template <typename R, int ALG, class SW>
__device__ uint64_t gamma_scalar_warp(const GammaParam<R> &k, SW &sw, uint64_t pos, uint64_t left, R *o)
{
    constexpr uint64_t WA = GammaAttemptWords<ALG>::value;
    const uint32_t lane = threadIdx.x & 31;
    uint64_t filled = 0, j0 = 0;
    for (;;) {
        R v;
        const bool acc = gamma_attempt<R, ALG>(k, sw, pos + WA * (j0 + lane), &v);
        const uint32_t m = __ballot_sync(0xffffffffu, acc);
        const uint32_t rank = __popc(m & ((1u << lane) - 1u));
        if (acc && filled + rank < left) o[filled + rank] = v;
        const uint32_t cnt = __popc(m);
        if (filled + cnt >= left) {
            // the attempt that fills the last output: the (left - filled)-th
            // accepted lane
            const uint32_t need = static_cast<uint32_t>(left - filled);
            uint32_t mm = m;
            for (uint32_t q = 1; q < need; ++q) mm &= mm - 1;
            const uint32_t last = __ffs(mm) - 1;
            return WA * (j0 + last + 1);
        }
        filled += cnt;
        j0 += 32;
    }
}

// The scalar fallback of algorithm N on one warp.  Each value draws with a
// fresh scalar normal, so a value whose first attempt is accepted with
// v = 1 + c w > 0 consumed exactly three words (its uniform and one
// Box-Muller pair) -- a regular value.  Lane l evaluates value q0 + l as if
// every value before it were regular (its words start at pos + 3 l); the
// values before the first irregular lane are final, and the irregular value
// is then drawn by lane 0 with the sequential loop from its (now known)
// start.  Returns the position after the last value (all lanes agree).
template <typename R, class G, class SW>
__device__ uint64_t gamma_scalar_n_warp(const GammaParam<R> &k, SW &sw, uint64_t pos, uint64_t left, R *o)
{
    using O = GOps<R>;
    const uint32_t lane = threadIdx.x & 31;
    uint64_t q0 = 0;
    while (q0 < left) {
        const uint64_t q = q0 + lane;
        const bool valid = q < left;
        bool reg = false;
        R val = 0;
        if (valid) {
            const uint64_t p = pos + 3 * static_cast<uint64_t>(lane);
            const R u = RealOps<R>::u01(kOO, sw.at(p));
            ScalarNormal<R> rn;
            uint64_t pn = p + 1;
            const R w = rn(sw, pn);
            const R v = O::add(static_cast<R>(1), O::mul(k.c, w));
            R r;
            if (v > 0 && gamma_n_accept(k, u, w, v, &r)) {
                reg = true;
                val = O::mul(k.beta, r);
            }
        }
        const uint32_t irr = __ballot_sync(0xffffffffu, valid && !reg);
        const uint32_t nvalid = static_cast<uint32_t>(min(static_cast<uint64_t>(32), left - q0));
        const uint32_t L = irr ? static_cast<uint32_t>(__ffs(irr) - 1) : nvalid;  // regular values this round
        if (lane < L) o[q] = val;
        pos += 3 * static_cast<uint64_t>(L);
        q0 += L;
        if (irr) {
            uint64_t sp = pos;
            if (lane == 0) o[q0] = gamma_scalar<R, 2>(k, sw, sp);
            pos = __shfl_sync(0xffffffffu, sp, 0);
            q0 += 1;
        }
    }
    return pos;
}

template <typename R>
struct GammaTraits {
    static constexpr int K = 8192 / static_cast<int>(sizeof(R));
};

// Shared memory of the chunk loop (after the generator's own table): the
// staged words of one chunk, reused for the redraw list of algorithm N.
template <class G, typename W, typename R>
struct GammaSmem {
    static constexpr int K = GammaTraits<R>::K;
    static constexpr int WPB = G::kWords / WordView<W>::kPer32;
    static constexpr int kStageBlocks = (2 * K + 2) / WPB + 2;
    static constexpr int kStageBytes = kStageBlocks * G::kWords * 4;
    static constexpr int kListBytes = K * (4 + 2 * static_cast<int>(sizeof(R)));
    static constexpr int kMainBytes = ((kStageBytes > kListBytes ? kStageBytes : kListBytes) + 15) / 16 * 16;
    // plus the batch normals of algorithm N
    static constexpr int kBytes = kMainBytes + K * static_cast<int>(sizeof(R));
};

// One chunk of n <= K values at stream word `pos`; accepted values go to
// out[0, m).  Returns m; advances `pos` and `eng` past the chunk's words.
template <class G, typename W, typename R, int THREADS, int ALG>
__device__ uint32_t gamma_chunk(const G &g, const GammaParam<R> &k, const Ctr &B, uint32_t off, uint64_t &pos,
    DevEngine<G::kCtrWords> &eng, uint32_t n, R *out, unsigned char *smem, uint32_t *shr, uint64_t *sh_pos)
{
    using O = GOps<R>;
    using S = GammaSmem<G, W, R>;
    constexpr int K = S::K, WPB = S::WPB, EPT = K / THREADS;
    constexpr uint32_t M = static_cast<uint32_t>(WPB);
    const R d = k.d, c = k.c, beta = k.beta;
    // ---- stage this chunk's words
    const uint64_t nw = (ALG <= 1) ? 2ull * n : (ALG == 2 ? 2ull * n + ((n & 1u) ? 2 : 0) : n);
    uint32_t *st32 = reinterpret_cast<uint32_t *>(smem);
    const W *st = reinterpret_cast<const W *>(st32);
    const uint64_t a0 = static_cast<uint64_t>(off) + pos, b0 = a0 / WPB;
    const uint32_t s0 = static_cast<uint32_t>(a0 % WPB);
    const int nb = static_cast<int>((s0 + nw + WPB - 1) / WPB);
    for (int i = threadIdx.x; i < nb; i += THREADS) {
        uint32_t blk[G::kWords];
        g.block(ctr_add(B, b0 + i, G::kCtrWords), blk);
#pragma unroll
        for (int q = 0; q < G::kWords; ++q) st32[i * G::kWords + q] = blk[q];
    }
    __syncthreads();
    R x[EPT];
    bool acc[EPT];
    uint32_t got = 0;
    if constexpr (ALG == 3) {
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
            const uint32_t i = threadIdx.x + j * THREADS;
            if (i < n) out[i] = O::mul(-beta, O::log(RealOps<R>::u01(kOO, st[s0 + i])));
        }
        got = n;
        __syncthreads();
    } else if constexpr (ALG <= 1) {
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
            const uint32_t i = threadIdx.x + j * THREADS;
            acc[j] = false;
            if (i >= n) continue;
            R u = RealOps<R>::u01(kOO, st[s0 + i]);
            R e = RealOps<R>::u01(kOO, st[s0 + n + i]);
            if constexpr (ALG == 0) {
                e = O::mul(static_cast<R>(-1), O::log(e));
                if (u > d) {
                    const R t = O::mul(c, O::sub(static_cast<R>(1), u));
                    u = -O::log(t);
                    e = O::add(e, u);
                    u = O::add(d, O::mul(k.alpha, u));
                }
                R xv = O::exp(O::mul(c, O::log(u)));
                const R ua = fabs(xv);
                x[j] = O::mul(beta, xv);
                acc[j] = ua < e;
            } else {
                u = O::mul(static_cast<R>(-1), O::log(u));
                e = O::mul(static_cast<R>(-1), O::log(e));
                const R xv = O::exp(O::mul(c, O::log(u)));
                u = O::add(u, e);
                e = O::add(d, xv);
                x[j] = O::mul(beta, xv);
                acc[j] = u > e;
            }
        }
        __syncthreads();
    } else {
        // ---- algorithm N: the batch normals, one Box-Muller pair per thread
        // and pass into shared memory, then per element u, w, v = fma(c, w, 1)
        R *wbuf = reinterpret_cast<R *>(smem + S::kMainBytes);
        const uint32_t nu = n / 2;
        const uint64_t q0 = s0 + n;  // first normal word in the staging buffer
        for (uint32_t p = threadIdx.x; p < nu; p += THREADS) {
            const R u1 = RealOps<R>::u01(kOC, st[q0 + p]);
            const R u2 = O::mul(O::kTwoPi, RealOps<R>::u01(kOC, st[q0 + nu + p]));
            const R sr = O::sqrt(O::mul(static_cast<R>(-2), O::log(u1)));
            R sn, cs;
            O::sincos(u2, &sn, &cs);
            wbuf[p] = O::mul(sr, sn);
            wbuf[nu + p] = O::mul(sr, cs);
        }
        if ((n & 1u) && threadIdx.x == THREADS - 1) {
            // odd n: the last normal from the two words after the batch
            const R a = RealOps<R>::u01(kOC, st[q0 + n]);
            const R b = RealOps<R>::u01(kOC, st[q0 + n + 1]);
            const R sr = O::mul(static_cast<R>(1), O::sqrt(O::mul(static_cast<R>(-2), O::log(a))));
            R sn, cs;
            O::sincos(O::mul(O::kTwoPi, b), &sn, &cs);
            wbuf[n - 1] = O::add(static_cast<R>(0), O::mul(sr, cs));
        }
        __syncthreads();
        R u[EPT], w[EPT], v[EPT];
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
            const uint32_t i = threadIdx.x + j * THREADS;
            u[j] = w[j] = v[j] = 0;
            if (i >= n) continue;
            u[j] = RealOps<R>::u01(kOO, st[s0 + i]);
            w[j] = wbuf[i];
            v[j] = O::fma(c, w[j], static_cast<R>(1));
        }
        // ---- redraws of v <= 0, in index order, by one thread
        uint32_t *lidx = reinterpret_cast<uint32_t *>(smem);
        R *lw = reinterpret_cast<R *>(smem + K * 4);
        R *lv = lw + K;
        int rk[EPT];
        uint32_t nred = 0;
        {
            bool f[EPT];
            uint32_t r[EPT];
#pragma unroll
            for (int j = 0; j < EPT; ++j) f[j] = threadIdx.x + j * THREADS < n && v[j] <= 0;
            block_rank_multi<THREADS, EPT>(f, shr, r, &nred);  // syncs: staging reads are done
#pragma unroll
            for (int j = 0; j < EPT; ++j) {
                rk[j] = f[j] ? static_cast<int>(r[j]) : -1;
                if (f[j]) lidx[r[j]] = threadIdx.x + j * THREADS;
            }
        }
        if (nred) {
            __syncthreads();
            if (threadIdx.x < 32) {
                // The scalar normals after the batch words form one sequence
                // z_0, z_1, ... (pair j: words 2j, 2j + 1; z_2j = r cos, z_2j+1
                // = r sin, the second returned from the cache); the q-th
                // redrawn element takes the q-th z with 1 + c z > 0.  A warp
                // evaluates 64 z at a time and assigns them by ballot ranks.
                const int lane = threadIdx.x;
                const unsigned lt = (1u << lane) - 1u;
                ScalarWords<G, W> sw{&g, B, off};
                const uint64_t sp0 = pos + nw;
                uint32_t done = 0;
                uint64_t used = 0;  // normals consumed
                for (uint64_t pb = 0; done < nred; pb += 32) {
                    const uint64_t j = pb + lane;
                    uint64_t k = sp0 + 2 * j;
                    ScalarNormal<R> rn;
                    const R z0 = rn(sw, k), z1 = rn(sw, k);
                    const R v0 = O::add(static_cast<R>(1), O::mul(c, z0));
                    const R v1 = O::add(static_cast<R>(1), O::mul(c, z1));
                    const bool a0 = v0 > 0, a1 = v1 > 0;
                    const unsigned m0 = __ballot_sync(0xffffffffu, a0), m1 = __ballot_sync(0xffffffffu, a1);
                    const uint32_t before = __popc(m0 & lt) + __popc(m1 & lt);
                    const uint32_t r0 = before, r1 = before + (a0 ? 1u : 0u);
                    const uint32_t need = nred - done;
                    if (a0 && r0 < need) {
                        lw[done + r0] = z0;
                        lv[done + r0] = v0;
                    }
                    if (a1 && r1 < need) {
                        lw[done + r1] = z1;
                        lv[done + r1] = v1;
                    }
                    const uint32_t tot = __popc(m0) + __popc(m1);
                    if (tot >= need) {
                        // the need-th accepted normal is the last one consumed
                        const bool last0 = a0 && r0 == need - 1, last1 = a1 && r1 == need - 1;
                        const unsigned ml = __ballot_sync(0xffffffffu, last0 || last1);
                        const int src = __ffs(ml) - 1;
                        const uint32_t idx = last0 ? 2u * lane : 2u * lane + 1u;
                        const uint32_t li = __shfl_sync(0xffffffffu, idx, src);
                        used = 2 * pb + li + 1;
                        done = nred;
                    } else {
                        done += tot;
                    }
                }
                // consumed words: two per started pair (a cached second value
                // is dropped with the chunk's normal generator)
                if (lane == 0) *sh_pos = 2 * ((used + 1) / 2);
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < EPT; ++j) {
                if (rk[j] >= 0) {
                    w[j] = lw[rk[j]];
                    v[j] = lv[rk[j]];
                }
            }
        }
        const uint64_t nscalar = nred ? *sh_pos : 0;
        const R db = O::mul(d, beta);
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
            const uint32_t i = threadIdx.x + j * THREADS;
            acc[j] = false;
            if (i >= n) continue;
            R e = O::mul(v[j], v[j]);
            const R vv = O::mul(v[j], e);
            e = O::mul(w[j], w[j]);
            e = O::mul(e, e);
            e = O::fma(-O::k0331, e, static_cast<R>(1));
            x[j] = O::mul(db, vv);
            if (u[j] < e) {
                acc[j] = true;
            } else {
                const R a = O::div(O::mul(w[j], w[j]), static_cast<R>(2));
                const R b = O::add(O::sub(static_cast<R>(1), vv), O::log(vv));
                e = O::add(a, O::mul(d, b));
                acc[j] = O::log(u[j]) < e;
            }
        }
        __syncthreads();  // every thread has read nscalar
        // engine calls of the N chunk: uniforms, normals (+2 odd words), redraw words
        eng.batch(n, K, M);
        if (n == static_cast<uint32_t>(K)) {
            eng.call(K, M);
            eng.call(0, M);
            eng.call(0, M);
        } else {
            eng.call(n, M);
        }
        if (n & 1u) {
            eng.call(1, M);
            eng.call(1, M);
        }
        for (uint64_t q = 0; q < nscalar; ++q) eng.call(1, M);
        pos += nw + nscalar;
    }
    if constexpr (ALG != 2) {
        eng.batch(ALG <= 1 ? 2ull * n : n, K, M);
        pos += nw;
    }
    if constexpr (ALG == 3) return got;
    // ---- compaction of the accepted values, in index order
    uint32_t m = 0, r[EPT];
    block_rank_multi<THREADS, EPT>(acc, shr, r, &m);
#pragma unroll
    for (int j = 0; j < EPT; ++j)
        if (acc[j]) out[r[j]] = x[j];
    return m;
}

// gamma_distribution (:277-302) for `nstreams` streams of n values, all of
// them drawn by algorithm ALG (one instantiation per algorithm keeps the code
// each SM runs small).  Stream list[i] (i when list is null) writes
// r + s * n; its engine starts at (ctr0 with word 1 = s, empty buffer) when
// `blocks` is set, else at the engine state given (one stream), whose final
// state goes to *ctr_out / *idx_out.
constexpr int kGammaThreads = 256;

template <class G, typename W, typename R, int THREADS, int ALG>
__global__ void __launch_bounds__(THREADS, 3) k_gamma(G g, Ctr ctr0, uint32_t idx0, int blocks, uint64_t nstreams,
    const uint32_t *list, uint64_t n, const GammaParam<R> *params, R *r, Ctr *ctr_out, uint32_t *idx_out)
{
    using S = GammaSmem<G, W, R>;
    constexpr int K = S::K;
    constexpr uint32_t M = static_cast<uint32_t>(S::WPB);
    __shared__ uint32_t shr[THREADS / 32 * GammaTraits<float>::K / THREADS + 1];
    __shared__ uint64_t sh_pos;
    extern __shared__ __align__(16) unsigned char gamma_dyn[];
    g.prepare();
    unsigned char *smem = gamma_dyn + G::kDynSmem;
    for (uint64_t i = blockIdx.x; i < nstreams; i += gridDim.x) {
        const uint64_t sidx = list ? list[i] : i;
        const GammaParam<R> k = params[blocks ? sidx : 0];
        DevEngine<G::kCtrWords> eng;
        eng.ctr = ctr0;
        eng.idx = idx0;
        if (blocks) {
            eng.ctr.w[0] = 0;
            eng.ctr.w[1] = sidx;
            eng.ctr.w[2] = eng.ctr.w[3] = 0;
            eng.idx = M;
        }
        // first word of the stream
        Ctr B = eng.ctr;
        uint32_t off = eng.idx;
        if (eng.idx >= M) {
            B = ctr_add(eng.ctr, 1, G::kCtrWords);
            off = 0;
        }
        uint64_t pos = 0, left = n;
        R *o = r + sidx * n;
        while (left > static_cast<uint64_t>(K)) {
            const uint32_t m = gamma_chunk<G, W, R, THREADS, ALG>(g, k, B, off, pos, eng, K, o, smem, shr, &sh_pos);
            if (m == 0) break;
            left -= m;
            o += m;
        }
        const uint32_t m = gamma_chunk<G, W, R, THREADS, ALG>(g, k, B, off, pos, eng, static_cast<uint32_t>(left), o,
            smem, shr, &sh_pos);
        left -= m;
        o += m;
        if constexpr (ALG != 2) {
            if (left && threadIdx.x < 32) {
                ScalarWords<G, W> sw{&g, B, off};
                const uint64_t used = gamma_scalar_warp<R, ALG>(k, sw, pos, left, o);
                if (threadIdx.x == 0)
                    for (uint64_t q = 0; q < used; ++q) eng.call(1, M);
            }
        } else {
            if (left && threadIdx.x < 32) {
                ScalarWords<G, W> sw{&g, B, off};
                const uint64_t sp = gamma_scalar_n_warp<R, G>(k, sw, pos, left, o);
                if (threadIdx.x == 0)
                    for (uint64_t q = pos; q < sp; ++q) eng.call(1, M);
            }
        }
        if (!blocks && threadIdx.x == 0) {
            *ctr_out = eng.ctr;
            *idx_out = eng.idx;
        }
        __syncthreads();
    }
}

template <class G, typename W, typename R, int ALG>
int launch_gamma(const G &g, const Ctr &c0, uint32_t idx0, bool blocks, uint64_t count, const uint32_t *list,
    uint64_t n, const GammaParam<R> *dparams, R *r, Ctr *dctr, uint32_t *didx, cudaStream_t s)
{
    using S = GammaSmem<G, W, R>;
    auto kern = k_gamma<G, W, R, kGammaThreads, ALG>;
    const int dyn = G::kDynSmem + S::kBytes;
    MB_CUDA(allow_dyn_smem(kern, dyn));
    int per_sm = 0;
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGammaThreads, dyn));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t cap = static_cast<uint64_t>(std::max(1, per_sm)) * sms;
    const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(count, cap)));
    kern<<<grid, kGammaThreads, dyn, s>>>(g, c0, idx0, blocks ? 1 : 0, count, list, n, dparams, r, dctr, didx);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

template <class G, typename W, typename R>
int launch_gamma_alg(int alg, const G &g, const Ctr &c0, uint32_t idx0, bool blocks, uint64_t count,
    const uint32_t *list, uint64_t n, const GammaParam<R> *dparams, R *r, Ctr *dctr, uint32_t *didx, cudaStream_t s)
{
    switch (alg) {
        case 0: return launch_gamma<G, W, R, 0>(g, c0, idx0, blocks, count, list, n, dparams, r, dctr, didx, s);
        case 1: return launch_gamma<G, W, R, 1>(g, c0, idx0, blocks, count, list, n, dparams, r, dctr, didx, s);
        case 2: return launch_gamma<G, W, R, 2>(g, c0, idx0, blocks, count, list, n, dparams, r, dctr, didx, s);
        default: return launch_gamma<G, W, R, 3>(g, c0, idx0, blocks, count, list, n, dparams, r, dctr, didx, s);
    }
}

// One launch per algorithm present: the streams of each algorithm are listed
// (device copy) so every CTA runs one algorithm's code.
template <typename R>
int gamma_impl(mckl_b200_engine_t *e, bool blocks, size_t nstreams, size_t n, const GammaParam<R> *hparams,
    size_t nparams, R *r, void *stream)
{
    cudaStream_t s = as_stream(stream);
    std::vector<uint32_t> lists[4];
    if (blocks) {
        for (size_t i = 0; i < nstreams; ++i) lists[hparams[i].alg].push_back(static_cast<uint32_t>(i));
    }
    const size_t pbytes = align256(nparams * sizeof(GammaParam<R>));
    const size_t lbytes = align256(blocks ? nstreams * 4 : 4);
    char *scr = static_cast<char *>(scratch(6, pbytes + lbytes + 256, s));
    if (!scr) return MCKL_B200_ERR_NOMEM;
    auto *dparams = reinterpret_cast<GammaParam<R> *>(scr);
    uint32_t *dlist = reinterpret_cast<uint32_t *>(scr + pbytes);
    Ctr *dctr = reinterpret_cast<Ctr *>(scr + pbytes + lbytes);
    uint32_t *didx = reinterpret_cast<uint32_t *>(scr + pbytes + lbytes + sizeof(Ctr));
    MB_CUDA(cudaMemcpyAsync(dparams, hparams, nparams * sizeof(GammaParam<R>), cudaMemcpyHostToDevice, s));
    std::vector<uint32_t> flat;
    size_t first[4] = {0, 0, 0, 0};
    if (blocks) {
        for (int a = 0; a < 4; ++a) {
            first[a] = flat.size();
            flat.insert(flat.end(), lists[a].begin(), lists[a].end());
        }
        MB_CUDA(cudaMemcpyAsync(dlist, flat.data(), flat.size() * 4, cudaMemcpyHostToDevice, s));
    }
    const Ctr c0 = ctr_of(*e);
    const uint32_t idx0 = e->index;
    const bool w64 = geom(e->kind).rbytes == 8;
    int rc = with_generator(*e, [&](auto g) {
        using G = decltype(g);
        auto run = [&](auto wtag) {
            using W = decltype(wtag);
            if (!blocks) {
                return launch_gamma_alg<G, W, R>(hparams[0].alg, g, c0, idx0, false, 1, nullptr, n, dparams, r, dctr,
                    didx, s);
            }
            for (int a = 0; a < 4; ++a) {
                if (lists[a].empty()) continue;
                const int rc2 = launch_gamma_alg<G, W, R>(a, g, c0, idx0, true, lists[a].size(), dlist + first[a], n,
                    dparams, r, dctr, didx, s);
                if (rc2 != MCKL_B200_OK) return rc2;
            }
            return MCKL_B200_OK;
        };
        if (w64) return run(uint64_t{});
        return run(uint32_t{});
    });
    if (rc != MCKL_B200_OK) return rc;
    if (!blocks) {
        Ctr hc;
        uint32_t hi = 0;
        MB_CUDA(cudaMemcpyAsync(&hc, dctr, sizeof(Ctr), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaMemcpyAsync(&hi, didx, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        set_ctr(*e, hc);
        e->index = hi;
    } else {
        // the host lists must outlive the asynchronous copies
        MB_CUDA(cudaStreamSynchronize(s));
    }
    return MCKL_B200_OK;
}

template <typename R>
int gamma_one(mckl_b200_engine_t *e, size_t n, R *r, R alpha, R beta, void *stream)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    MB_CHECK_ARG(alpha > 0 && beta > 0, "alpha and beta must be positive");
    if (n == 0) return MCKL_B200_OK;
    const GammaParam<R> p = gamma_param<R>(alpha, beta);
    return gamma_impl<R>(e, false, 1, n, &p, 1, r, stream);
}

template <typename R>
int gamma_blocks(const mckl_b200_engine_t *e, size_t nblocks, size_t block, const double *alpha, double beta,
    R *r, void *stream)
{
    MB_CHECK_ARG(e != nullptr && alpha != nullptr, "null argument");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    MB_CHECK_ARG(nblocks == 0 || block == 0 || r != nullptr, "null output");
    MB_CHECK_ARG(beta > 0, "beta must be positive");
    if (nblocks == 0 || block == 0) return MCKL_B200_OK;
    std::vector<GammaParam<R>> p(nblocks);
    for (size_t b = 0; b < nblocks; ++b) {
        MB_CHECK_ARG(alpha[b] > 0, "alpha must be positive");
        p[b] = gamma_param<R>(static_cast<R>(alpha[b]), static_cast<R>(beta));
    }
    mckl_b200_engine_t copy = *e;
    return gamma_impl<R>(&copy, true, nblocks, block, p.data(), nblocks, r, stream);
}

}  // namespace

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" {

int mckl_b200_gamma_f32(mckl_b200_engine_t *e, size_t n, float *r, float alpha, float beta, void *stream)
{
    return gamma_one<float>(e, n, r, alpha, beta, stream);
}

int mckl_b200_gamma_f64(mckl_b200_engine_t *e, size_t n, double *r, double alpha, double beta, void *stream)
{
    return gamma_one<double>(e, n, r, alpha, beta, stream);
}

int mckl_b200_gamma_blocks_f32(const mckl_b200_engine_t *e, size_t nblocks, size_t block, const double *alpha,
    double beta, float *r, void *stream)
{
    return gamma_blocks<float>(e, nblocks, block, alpha, beta, r, stream);
}

int mckl_b200_gamma_blocks_f64(const mckl_b200_engine_t *e, size_t nblocks, size_t block, const double *alpha,
    double beta, double *r, void *stream)
{
    return gamma_blocks<double>(e, nblocks, block, alpha, beta, r, stream);
}

}  // extern "C"
