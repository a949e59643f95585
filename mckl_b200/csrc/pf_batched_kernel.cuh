// pf_batched_kernel.cuh -- the batched particle filter's device code: the
// noise layout, one filter's step (FilterRun) and the persistent kernel
// (k_pf_batched), shared by the library (pf_batched.cu: the built-in AR(1)
// model, its adjoint and its score) and by user instantiations of the model
// hook (include/mckl_b200_batched.cuh).  The comments of pf_batched.cu
// describe the algorithm.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <type_traits>

#include "block_scan.cuh"
#include "common.cuh"
#include "pf_batched.cuh"

namespace mckl_b200 {
namespace batched_detail {

struct WordCache {
    uint64_t blk;
    uint32_t w[4];
};

__device__ __forceinline__ uint32_t word_at(const PhiloxGen &g, uint64_t w, WordCache &c)
{
    const uint64_t b = w >> 2;
    if (b != c.blk) {
        g.block(Ctr{{b + 1, 0, 0, 0}}, c.w);
        c.blk = b;
    }
    return c.w[w & 3];
}

// U01OC<double> of a word, rounded to the propagation type: (w + 1) 2^-32 is
// exact in double; in float it is RN(w + 1) 2^-32, one integer conversion
template <typename R>
__device__ __forceinline__ R u01oc(uint32_t w)
{
    return static_cast<R>(__dadd_rn(__dmul_rn(static_cast<double>(w), 0x1p-32), 0x1p-32));
}

template <>
__device__ __forceinline__ float u01oc<float>(uint32_t w)
{
    return w == 0xFFFFFFFFu ? 1.0f : __fmul_rn(__uint2float_rn(w + 1u), 0x1p-32f);
}

template <typename R>
struct Math;

template <>
struct Math<float> {
    __device__ static float radius(float u) { return sqrtf(-2.0f * logf(u)); }
    __device__ static void sincos2pi(float v, float *s, float *c) { sincospif(2.0f * v, s, c); }
    __device__ static float cos2pi(float v) { return cospif(2.0f * v); }
    // exp2 of the scaled argument (its rounding adds at most 2^-20 relative
    // for the arguments the weights take, |a| <= 20 where it matters): the
    // normaliser's terms and the fixed-point weights, summed in FP64
    __device__ static float exp(float a) { return exp2f(__fmul_rn(a, 1.44269504088896341f)); }
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
};

template <>
struct Math<double> {
    __device__ static double radius(double u) { return sqrt(-2.0 * log(u)); }
    __device__ static void sincos2pi(double v, double *s, double *c) { sincospi(2.0 * v, s, c); }
    __device__ static double cos2pi(double v) { return cospi(2.0 * v); }
    __device__ static double exp(double a) { return ::exp(a); }
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    __device__ static double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
};

// ---------------------------------------------------------------------------
// The model of the filters.  A model is a struct with
//   Param    -- the parameters of one filter (trivially copyable), and
//   Dev<R>   -- those parameters in the propagation type R (float or double),
//               constructed on the device from a Param once per filter, with
//     R init(R e)            x_0 from a standard normal e,
//     R move(R x, R e)       x_t from x_{t-1} and a standard normal e,
//     R log_density(R x, R y) log g(y | x), up to a constant of the filter.
// The noise of every step is Normal(0, 1) from the filter's model stream,
// consumed as normal_distribution does, whatever the model.  Arithmetic in
// Dev should be written with explicit rounding (Math<R>) where the same bits
// are wanted from every build.
// ---------------------------------------------------------------------------
struct Ar1Model {
    // x_0 = sd0 e, x_t = phi x_{t-1} + sx e, log g(y | x) = lconst - (y - x)^2 hinv
    struct Param {
        double phi, sx, sd0, lconst, hinv;
    };
    template <typename R>
    struct Dev {
        R phi, sx, sd0, lconst, hinv;
        __device__ Dev() {}
        __device__ explicit Dev(const Param &p)
            : phi(static_cast<R>(p.phi)), sx(static_cast<R>(p.sx)), sd0(static_cast<R>(p.sd0)),
              lconst(static_cast<R>(p.lconst)), hinv(static_cast<R>(p.hinv))
        {
        }
        __device__ __forceinline__ R init(R e) const { return Math<R>::mul(sd0, e); }
        __device__ __forceinline__ R move(R x, R e) const { return Math<R>::fma(phi, x, Math<R>::mul(sx, e)); }
        __device__ __forceinline__ R log_density(R x, R y) const
        {
            const R r = Math<R>::sub(y, x);
            return Math<R>::fma(-Math<R>::mul(r, r), hinv, lconst);
        }
    };
    __host__ __device__ static Param main(const BatchedFilter &F) { return {F.phi, F.sx, F.sd0, F.lconst, F.hinv}; }
    __host__ __device__ static Param shadow(const BatchedFilter &F)
    {
        return {F.phi_s, F.sx_s, F.sd0_s, F.lconst_s, F.hinv_s};
    }
};

template <typename T>
__device__ __forceinline__ T block_max(T v, T *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_max(v);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nw ? sh[lane] : -INFINITY;
        w = warp_max(w);
        if (lane == 0) sh[32] = w;
    }
    __syncthreads();
    const T r = sh[32];
    __syncthreads();
    return r;
}

// Online log-sum-exp accumulator of one thread: s = sum exp(v - m),
// q = sum exp(2 (v - m)) over the values seen, m their running maximum.  The
// terms are evaluated in the propagation type, summed in FP64; a new maximum
// rescales the sums by an FP64 exp (values arrive in groups of up to eight,
// so this happens a few times per thread and step).
template <typename R>
struct Lse {
    R m = -INFINITY;
    double s = 0.0, q = 0.0;

    template <int K>
    __device__ __forceinline__ void add(const R (&v)[K], int lo, int hi)
    {
        R gm = -INFINITY;
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (k >= lo && k < hi) gm = fmax(gm, v[k]);
        if (gm > m) {
            const double sc = (m == -INFINITY) ? 0.0 : ::exp(static_cast<double>(m) - static_cast<double>(gm));
            s = __dmul_rn(s, sc);
            q = __dmul_rn(q, __dmul_rn(sc, sc));
            m = gm;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (k >= lo && k < hi) {
                const double e = static_cast<double>(Math<R>::exp(Math<R>::sub(v[k], m)));
                s = __dadd_rn(s, e);
                q = __fma_rn(e, e, q);
            }
        }
    }
};

// The combined (max, sum, sum of squares) of a CTA's accumulators.
template <typename R>
__device__ __forceinline__ void block_lse(const Lse<R> &a, R *shr, double *shd, R *M, double *S, double *Q)
{
    const R mm = block_max(a.m, shr);
    const double sc = (a.m == -INFINITY) ? 0.0 : ::exp(static_cast<double>(a.m) - static_cast<double>(mm));
    *M = mm;
    *S = block_sum(__dmul_rn(a.s, sc), shd);
    if (Q) *Q = block_sum(__dmul_rn(a.q, __dmul_rn(sc, sc)), shd);
}

// One Box-Muller pair of one filter at step t: the noise from a radius and an
// angle word, the AR(1) move of particles p0 and p1, their new log-weights
// (old log-weight minus the previous step's maximum, plus the observation's
// log-density; zero old weights after a resampling) and, for the shadow, the
// same in FP64.  Returns the two log-weights in v[0], v[1].
template <typename R, bool SHADOW, class Model = Ar1Model>
struct Step {
    R *x, *l;
    double *xs, *ls;
    typename Model::template Dev<R> m;        // the model in the propagation type
    typename Model::template Dev<double> ms;  // the shadow run's model
    R yt, lshift;
    double yt_d, lshift_s;
    bool init, flat;

    // the move and weight of one particle from its old state (registers)
    __device__ __forceinline__ R move(R e, R x_old, R l_old, R &v) const
    {
        using O = Math<R>;
        if (init) return m.init(e);
        const R xn = m.move(x_old, e);
        const R lo = flat ? R(0) : O::sub(l_old, lshift);
        v = O::add(lo, m.log_density(xn, yt));
        return xn;
    }

    __device__ __forceinline__ double move_shadow(double e, double x_old, double l_old, double &v) const
    {
        using O = Math<double>;
        if (init) return ms.init(e);
        const double xn = ms.move(x_old, e);
        const double lo = flat ? 0.0 : O::sub(l_old, lshift_s);
        v = O::add(lo, ms.log_density(xn, yt_d));
        return xn;
    }

    __device__ __forceinline__ void one(R e, uint64_t p, R &v) const
    {
        const R xn = move(e, init ? R(0) : x[p], (init || flat) ? R(0) : l[p], v);
        x[p] = xn;
        if (!init) l[p] = v;
    }

    __device__ __forceinline__ void one_shadow(double e, uint64_t p, double &v) const
    {
        const double xn = move_shadow(e, init ? 0.0 : xs[p], (init || flat) ? 0.0 : ls[p], v);
        xs[p] = xn;
        if (!init) ls[p] = v;
    }

    // Four pairs of one unit, in two halves: load4 issues every load of the
    // unit before any store (the loads overlap instead of queueing behind the
    // stores), move4 moves and weighs the particles and stores them.
    struct Old {
        R xo[8], lo_[8];
        double xso[8], lso[8];
    };

    __device__ __forceinline__ void load4(const uint32_t (&pa)[4], const uint32_t (&pb)[4], int lo, int hi,
        Old &o) const
    {
        R(&xo)[8] = o.xo;
        R(&lo_)[8] = o.lo_;
        double(&xso)[8] = o.xso;
        double(&lso)[8] = o.lso;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            xo[2 * j] = xo[2 * j + 1] = lo_[2 * j] = lo_[2 * j + 1] = R(0);
            xso[2 * j] = xso[2 * j + 1] = lso[2 * j] = lso[2 * j + 1] = 0.0;
            if (j >= lo && j < hi && !init) {
                xo[2 * j] = x[pa[j]];
                xo[2 * j + 1] = x[pb[j]];
                if (!flat) {
                    lo_[2 * j] = l[pa[j]];
                    lo_[2 * j + 1] = l[pb[j]];
                }
                if constexpr (SHADOW) {
                    xso[2 * j] = xs[pa[j]];
                    xso[2 * j + 1] = xs[pb[j]];
                    if (!flat) {
                        lso[2 * j] = ls[pa[j]];
                        lso[2 * j + 1] = ls[pb[j]];
                    }
                }
            }
        }
    }

    __device__ __forceinline__ void move4(const uint32_t (&wr)[4], const uint32_t (&wa)[4],
        const uint32_t (&pa)[4], const uint32_t (&pb)[4], int lo, int hi, const Old &o, R *v, double *vs) const
    {
        const R(&xo)[8] = o.xo;
        const R(&lo_)[8] = o.lo_;
        const double(&xso)[8] = o.xso;
        const double(&lso)[8] = o.lso;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (j >= lo && j < hi) {
                const R rr = Math<R>::radius(u01oc<R>(wr[j]));
                R sn, cs;
                Math<R>::sincos2pi(u01oc<R>(wa[j]), &sn, &cs);
                const R x0 = move(Math<R>::mul(rr, sn), xo[2 * j], lo_[2 * j], v[2 * j]);
                const R x1 = move(Math<R>::mul(rr, cs), xo[2 * j + 1], lo_[2 * j + 1], v[2 * j + 1]);
                x[pa[j]] = x0;
                x[pb[j]] = x1;
                if (!init) {
                    l[pa[j]] = v[2 * j];
                    l[pb[j]] = v[2 * j + 1];
                }
                if constexpr (SHADOW) {
                    const double rd = Math<double>::radius(u01oc<double>(wr[j]));
                    double snd, csd;
                    Math<double>::sincos2pi(u01oc<double>(wa[j]), &snd, &csd);
                    const double s0 = move_shadow(__dmul_rn(rd, snd), xso[2 * j], lso[2 * j], vs[2 * j]);
                    const double s1 = move_shadow(__dmul_rn(rd, csd), xso[2 * j + 1], lso[2 * j + 1], vs[2 * j + 1]);
                    xs[pa[j]] = s0;
                    xs[pb[j]] = s1;
                    if (!init) {
                        ls[pa[j]] = vs[2 * j];
                        ls[pb[j]] = vs[2 * j + 1];
                    }
                }
            }
        }
    }
};

// Where the Normal(0,1) draws of step t come from.  The draws of a filter
// are 1024-value chunks (radius word i, angle word 512 + i of the chunk, as
// normal_distribution lays them out).  A full chunk is covered by 129 units;
// unit g owns the radius words of Philox block (chunk start / 4) + g and the
// angle words of the block 128 further on, i.e. up to four pairs for two
// Philox blocks (a quarter block per particle).  Units past the full chunks
// are the pairs of the last partial chunk, drawn word by word.
// Placement: a warp owns 32 x 8 consecutive parents per tile and copies them
// into their empty slots; a warp with more than kWarpCopies copies in one tile
// queues its parents (up to kBigParents queued groups) for the whole CTA.
constexpr uint32_t kBigParents = 64;
constexpr uint32_t kWarpParents = 256;
constexpr uint32_t kWarpCopies = 512;
constexpr uint32_t kWs = kWarpParents + 4;  // a warp's staged prefixes (+ the end), 16-byte multiple
// Words of the CTA's uint32 shared buffer: scan scratch, the heavy queue, then
// one staging area per warp (16-byte aligned).
template <int THREADS>
constexpr int shj_words()
{
    return ((THREADS + 35 + kBigParents + 3) / 4) * 4 + (THREADS / 32) * kWs;
}
template <int THREADS>
constexpr int ws_offset()
{
    return ((THREADS + 35 + kBigParents + 3) / 4) * 4;
}

// Eight consecutive elements starting at a 32-byte aligned address (float,
// uint32) or a 64-byte aligned one (double) with vector loads and stores.
// Every filter's particle range starts on a multiple of 32 elements.
__device__ __forceinline__ void ld8(const float *p, float (&v)[8])
{
    const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

__device__ __forceinline__ void ld8(const double *p, double (&v)[8])
{
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double2 a = reinterpret_cast<const double2 *>(p)[q];
        v[2 * q] = a.x;
        v[2 * q + 1] = a.y;
    }
}

__device__ __forceinline__ void ld8(const uint32_t *p, uint32_t (&v)[8])
{
    const uint4 a = reinterpret_cast<const uint4 *>(p)[0], b = reinterpret_cast<const uint4 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

__device__ __forceinline__ void st8(uint32_t *p, const uint32_t (&v)[8])
{
    reinterpret_cast<uint4 *>(p)[0] = make_uint4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<uint4 *>(p)[1] = make_uint4(v[4], v[5], v[6], v[7]);
}

__device__ __forceinline__ void st8(float *p, const float (&v)[8])
{
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
}

__device__ __forceinline__ void st8(double *p, const double (&v)[8])
{
#pragma unroll
    for (int q = 0; q < 4; ++q) reinterpret_cast<double2 *>(p)[q] = make_double2(v[2 * q], v[2 * q + 1]);
}

// A hint that the line holding p is read soon (prefetch.global.L1: nothing
// waits on it and no register is held; p lies inside the buffer)
__device__ __forceinline__ void prefetch_l1(const void *p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

struct NoiseLayout {
    static constexpr uint64_t kUnits = 129;  // units per full chunk (the 32-bit division below uses 129)
    uint64_t N, m, tail, nu_tail, units, per_step;

    __device__ void init(uint64_t n)
    {
        N = n;
        per_step = N + (N & 1) * 2;  // words of one normal_distribution(N) call
        m = N / 1024;
        tail = N % 1024;
        nu_tail = tail / 2;
        units = m * kUnits + nu_tail;
    }

    // Calls pair(wrad, wang, p0, p1, j) for the pairs of unit u at step t
    // (j: slot of the pair inside the unit) and returns the unit's slot range
    // [lo, hi).
    template <class Fn>
    __device__ __forceinline__ void unit(const PhiloxGen &gm, int t, uint64_t u, int *lo_out, int *hi_out,
        Fn &&pair) const
    {
        const uint64_t P = static_cast<uint64_t>(t) * per_step;
        if (u < m * kUnits) {
            // u < 2^28 (N < 2^31): 32-bit division by the constant
            const uint32_t u32 = static_cast<uint32_t>(u), c32 = u32 / 129u;
            const uint64_t c = c32, g = u32 - c32 * 129u;
            const uint64_t base = P + c * 1024;
            const uint64_t B = (base >> 2) + g;
            const int i0 = static_cast<int>(4 * g) - static_cast<int>(base & 3);
            uint32_t wr[4], wa[4];
            gm.block(Ctr{{B + 1, 0, 0, 0}}, wr);
            gm.block(Ctr{{B + 129, 0, 0, 0}}, wa);
            const int lo = i0 < 0 ? -i0 : 0, hi = i0 + 4 > 512 ? 512 - i0 : 4;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j >= lo && j < hi) {
                    const uint64_t p0 = c * 1024 + static_cast<uint64_t>(i0 + j);
                    pair(wr[j], wa[j], p0, p0 + 512, j);
                }
            }
            *lo_out = lo;
            *hi_out = hi;
        } else {
            const uint64_t i = u - m * kUnits, base = P + m * 1024;
            WordCache wc{~0ull, {0, 0, 0, 0}};
            const uint32_t wrad = word_at(gm, base + i, wc);
            const uint32_t wang = word_at(gm, base + nu_tail + i, wc);
            pair(wrad, wang, m * 1024 + i, m * 1024 + nu_tail + i, 0);
            *lo_out = 0;
            *hi_out = 1;
        }
    }

    // The words and particle indices of unit u at step t: pairs j in
    // [lo, hi) use words wr[j], wa[j] and move particles pa[j], pb[j].
    __device__ __forceinline__ void decode(const PhiloxGen &gm, int t, uint64_t u, uint32_t (&wr)[4],
        uint32_t (&wa)[4], uint32_t (&pa)[4], uint32_t (&pb)[4], int *lo_out, int *hi_out) const
    {
        const uint64_t P = static_cast<uint64_t>(t) * per_step;
        if (u < m * kUnits) {
            // u < 2^28 (N < 2^31): 32-bit division by the constant
            const uint32_t u32 = static_cast<uint32_t>(u), c32 = u32 / 129u;
            const uint64_t c = c32, g = u32 - c32 * 129u;
            const uint64_t base = P + c * 1024;
            const uint64_t B = (base >> 2) + g;
            const int i0 = static_cast<int>(4 * g) - static_cast<int>(base & 3);
            gm.block(Ctr{{B + 1, 0, 0, 0}}, wr);
            gm.block(Ctr{{B + 129, 0, 0, 0}}, wa);
            *lo_out = i0 < 0 ? -i0 : 0;
            *hi_out = i0 + 4 > 512 ? 512 - i0 : 4;
            const uint32_t q = static_cast<uint32_t>(c * 1024) + static_cast<uint32_t>(i0);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                pa[j] = q + j;  // only [lo, hi) are used
                pb[j] = q + j + 512;
            }
        } else {
            const uint64_t i = u - m * kUnits, base = P + m * 1024;
            WordCache wc{~0ull, {0, 0, 0, 0}};
            wr[0] = word_at(gm, base + i, wc);
            wa[0] = word_at(gm, base + nu_tail + i, wc);
            pa[0] = static_cast<uint32_t>(m * 1024 + i);
            pb[0] = static_cast<uint32_t>(m * 1024 + nu_tail + i);
            *lo_out = 0;
            *hi_out = 1;
        }
    }

    // The particle slots of unit u at step t (pairs j in [lo, hi) move
    // particles pa[j], pb[j]) and where its words come from (*src: the radius
    // block of a full-chunk unit, the radius word of a tail unit); words()
    // then generates them (decode() in two halves).
    __device__ __forceinline__ void slots(int t, uint32_t u, uint32_t (&pa)[4], uint32_t (&pb)[4], int *lo_out,
        int *hi_out, uint64_t *src) const
    {
        const uint64_t P = static_cast<uint64_t>(t) * per_step;
        if (u < m * kUnits) {
            const uint32_t c32 = u / 129u;
            const uint64_t c = c32, g = u - c32 * 129u;
            const uint64_t base = P + c * 1024;
            *src = (base >> 2) + g;
            const int i0 = static_cast<int>(4 * g) - static_cast<int>(base & 3);
            *lo_out = i0 < 0 ? -i0 : 0;
            *hi_out = i0 + 4 > 512 ? 512 - i0 : 4;
            const uint32_t q = static_cast<uint32_t>(c * 1024) + static_cast<uint32_t>(i0);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                pa[j] = q + j;  // only [lo, hi) are used
                pb[j] = q + j + 512;
            }
        } else {
            const uint64_t i = u - m * kUnits;
            *src = P + m * 1024 + i;
            pa[0] = static_cast<uint32_t>(m * 1024 + i);
            pb[0] = static_cast<uint32_t>(m * 1024 + nu_tail + i);
            *lo_out = 0;
            *hi_out = 1;
        }
    }

    __device__ __forceinline__ void words(const PhiloxGen &gm, uint32_t u, uint64_t src, uint32_t (&wr)[4],
        uint32_t (&wa)[4]) const
    {
        if (u < m * kUnits) {
            gm.block(Ctr{{src + 1, 0, 0, 0}}, wr);
            gm.block(Ctr{{src + 129, 0, 0, 0}}, wa);
        } else {
            WordCache wc{~0ull, {0, 0, 0, 0}};
            wr[0] = word_at(gm, src, wc);
            wa[0] = word_at(gm, src + nu_tail, wc);
        }
    }

    // the two words of the odd last particle (N odd)
    __device__ __forceinline__ void odd_words(const PhiloxGen &gm, int t, uint32_t *w0, uint32_t *w1) const
    {
        const uint64_t P = static_cast<uint64_t>(t) * per_step;
        WordCache wc{~0ull, {0, 0, 0, 0}};
        *w0 = word_at(gm, P + N, wc);
        *w1 = word_at(gm, P + N + 1, wc);
    }
};

// Scalar state of a filter between steps (a checkpoint holds it together
// with the particles and log-weights).
struct FilterScalars {
    double L_prev, ll_sum, Ls_prev, lls_sum, lshift, lshift_s;
    uint64_t events;
    int flat;
};

// One filter run by one CTA: state, and the step of the particle filter.
//
// SHADOW: every particle also carries an FP64 copy, propagated with the same
// uniforms and the shadow parameters, weighted in FP64 and resampled with the
// main run's decisions and parent indices.  With R = float and the same
// parameters its log-likelihood isolates the FP32 arithmetic error from the
// Monte Carlo divergence a flipped ancestor would otherwise start; with
// R = double and perturbed parameters it is the common-random-numbers,
// fixed-ancestor evaluation that finite differences of the estimate need.
template <typename R, int THREADS, bool SHADOW, class Model = Ar1Model>
struct FilterRun {
    NoiseLayout lay;
    PhiloxGen gm, gr;
    Step<R, SHADOW, Model> st;
    R *xc;
    double *xsc;
    double *rec_x = nullptr;  // when set: each step's particles before resampling
    uint32_t *sS, *ep;
    double threshold;
    double L_prev, ll_sum, Ls_prev, lls_sum;
    uint64_t events, n_empty;

    // the built-in AR(1) filters: their parameters are in the descriptor
    __device__ void setup(const BatchedFilter &F, R *xa, R *xb, R *lw, uint32_t *scanS, uint32_t *epos, double *xsa,
        double *xsb, double *lws, double thr)
    {
        setup(F, Ar1Model::main(F), Ar1Model::shadow(F), xa, xb, lw, scanS, epos, xsa, xsb, lws, thr);
    }

    __device__ void setup(const BatchedFilter &F, const typename Model::Param &pm, const typename Model::Param &ps,
        R *xa, R *xb, R *lw, uint32_t *scanS, uint32_t *epos, double *xsa, double *xsb, double *lws, double thr)
    {
        lay.init(F.n);
        gm = PhiloxGen{F.mkey[0], F.mkey[1]};
        gr = PhiloxGen{F.rkey[0], F.rkey[1]};
        (void) xb;
        (void) xsb;
        xc = xa + F.off;
        xsc = SHADOW ? xsa + F.off : nullptr;
        sS = scanS + F.off;
        ep = epos + F.off;
        threshold = thr;
        st.l = lw + F.off;
        st.ls = SHADOW ? lws + F.off : nullptr;
        st.m = typename Model::template Dev<R>(pm);
        st.ms = typename Model::template Dev<double>(ps);
        st.lshift = 0;
        st.lshift_s = 0.0;
        st.flat = true;
        L_prev = log(static_cast<double>(F.n));
        ll_sum = 0.0;
        Ls_prev = L_prev;
        lls_sum = 0.0;
        events = 0;
    }

    __device__ FilterScalars scalars() const
    {
        return FilterScalars{L_prev, ll_sum, Ls_prev, lls_sum, static_cast<double>(st.lshift), st.lshift_s, events,
            st.flat ? 1 : 0};
    }

    __device__ void restore(const FilterScalars &c)
    {
        L_prev = c.L_prev;
        ll_sum = c.ll_sum;
        Ls_prev = c.Ls_prev;
        lls_sum = c.lls_sum;
        st.lshift = static_cast<R>(c.lshift);
        st.lshift_s = c.lshift_s;
        events = c.events;
        st.flat = c.flat != 0;
    }

    // Step t: move, weight, normalise and (when ESS < N threshold) resample;
    // returns whether it resampled.  The resampling is in place (an empty
    // slot takes a copy of an occupied one, which is never overwritten); its
    // placement stays in sS / ep[0, n_empty).  With STAGEX the placement also
    // stages each warp's parent positions in shx (THREADS / 32 x kWarpParents
    // elements of shared memory), so a copy reads its source from there.
    template <bool STAGEX = false>
    __device__ bool step(int t, double yt_d, double *shd, R *shr, unsigned long long *shu, uint32_t *shj,
        R *shx = nullptr)
    {
        const uint64_t N = lay.N;
        st.x = xc;
        st.xs = xsc;
        st.init = (t == 0);
        st.yt_d = yt_d;
        st.yt = static_cast<R>(yt_d);
        Lse<R> acc;
        Lse<double> accs;
        // ---- noise, propagation, log-weights, online normaliser
        const uint32_t fullu = static_cast<uint32_t>(lay.m * NoiseLayout::kUnits);  // units of whole chunks
        for (uint32_t u = threadIdx.x; u < static_cast<uint32_t>(lay.units); u += THREADS) {
            R v[8];
            double vs[8];
            int lo, hi;
            uint32_t wr[4], wa[4], pa[4], pb[4];
            uint64_t src;
            typename Step<R, SHADOW, Model>::Old old;
            // the words first, then the loads: issuing the loads before the
            // generator keeps 16 loaded values live across it, which spills
            // at the 64-register budget of the resident shapes
            lay.slots(t, u, pa, pb, &lo, &hi, &src);
            if (!st.init) {
                // the particles of this thread's next unit, ahead of its loads
                const uint32_t un = u + THREADS;
                if (un < fullu) {
                    const uint32_t c = un / 129u, pn = c * 1024u + 4u * (un - c * 129u);
                    prefetch_l1(st.x + pn);
                    prefetch_l1(st.x + pn + 512);
                    if (!st.flat) {
                        prefetch_l1(st.l + pn);
                        prefetch_l1(st.l + pn + 512);
                    }
                }
            }
            lay.words(gm, u, src, wr, wa);
            st.load4(pa, pb, lo, hi, old);
            st.move4(wr, wa, pa, pb, lo, hi, old, v, vs);
            if (t > 0) {
                acc.add(v, 2 * lo, 2 * hi);
                if constexpr (SHADOW) accs.add(vs, 2 * lo, 2 * hi);
            }
        }
        if ((N & 1) && threadIdx.x == THREADS - 1) {
            uint32_t w0, w1;
            lay.odd_words(gm, t, &w0, &w1);
            R v[1];
            double vs[1];
            st.one(Math<R>::mul(Math<R>::radius(u01oc<R>(w0)), Math<R>::cos2pi(u01oc<R>(w1))), N - 1, v[0]);
            if constexpr (SHADOW)
                st.one_shadow(__dmul_rn(Math<double>::radius(u01oc<double>(w0)), Math<double>::cos2pi(u01oc<double>(w1))),
                    N - 1, vs[0]);
            if (t > 0) {
                acc.add(v, 0, 1);
                if constexpr (SHADOW) accs.add(vs, 0, 1);
            }
        }
        if (t == 0) {
            __syncthreads();
            return false;
        }
        // ---- FP64 normaliser: S = sum exp(l - M), Q = sum exp^2; the log
        // normaliser of the weights relative to M is carried to the next step,
        // whose log-weights start from l - M
        R M;
        double S, Q;
        block_lse(acc, shr, shd, &M, &S, &Q);
        const double L = static_cast<double>(M) + log(S);
        ll_sum += L - L_prev;
        L_prev = log(S);
        if constexpr (SHADOW) {
            double Ms, Ss;
            block_lse<double>(accs, shd, shd, &Ms, &Ss, nullptr);
            lls_sum += Ms + log(Ss) - Ls_prev;
            Ls_prev = log(Ss);
            st.lshift_s = Ms;
        }
        st.lshift = M;
        st.flat = false;
        if (rec_x) {
            for (uint64_t p = threadIdx.x; p < N; p += THREADS) rec_x[p] = static_cast<double>(xc[p]);
            __syncthreads();  // the resampling below overwrites empty slots in place
        }
        const double ess = S * S / Q;
        if (!(ess < static_cast<double>(N) * threshold)) return false;
        // ---- systematic resampling
        ++events;
        uint32_t wr[2];
        {
            WordCache wc{~0ull, {0, 0, 0, 0}};
            const uint64_t a = 2 * (events - 1);
            wr[0] = word_at(gr, a, wc);
            wr[1] = word_at(gr, a + 1, wc);
        }
        const double U = __dadd_rn(__dmul_rn(static_cast<double>(wr[0]), 0x1p-64),
            __dmul_rn(static_cast<double>(wr[1]), 0x1p-32));
        const double invS = 1.0 / S;
        // Exact fixed-point systematic resampling.  The normalised weights
        // become integers W_p = RN(w_p 2^62) (absolute error 2^-63 each) and
        // are summed exactly in 64 bits: the cumulative weights C_p are exact,
        // monotone and independent of the summation order.  The count of grid
        // points (U + j) / N below C_p 2^-62 is then exact integer arithmetic:
        // j_p = clamp(ceil((4 N C_p - U 2^64) / 2^64), 0, N), with U the
        // canonical double of the two resampling words (a multiple of 2^-64).
        // Each thread owns V consecutive particles per tile of THREADS x V.
        // From the counts: replication counts rep_p = j_p - j_{p-1}, the
        // empty slots (rep = 0) in order, and the surplus copies of the
        // parents before p, sS_p = sum_{i<p} max(rep_i - 1, 0) = j_{p-1} - p
        // + E_p with E_p the empty slots before p.
        constexpr int V = 8;
        constexpr uint32_t TILE = THREADS * V;
        const uint64_t U64 = U < 1.0 ? static_cast<uint64_t>(U * 0x1p64) : ~0ull;
        const uint32_t N32 = static_cast<uint32_t>(N);
        // RN(e RN(1/S)) 2^62 == RN(e (RN(1/S) 2^62)): a power-of-two scale
        // commutes with rounding (e RN(1/S) >= 2^-181 when nonzero, far from
        // the subnormals)
        const double invS62 = invS * 0x1p62;
        // grid points (U + i) / N, i < N, at or below c 2^-62, for the
        // cumulative weight c: j = clamp(ceil((X - U64) / 2^64), 0, N) with
        // X = 4 N c, exact and branch-free.  With D = X - (U64 + 1) as a
        // 128-bit difference, j = 0 when D < 0, else (D >> 64) + 1.  N c is
        // formed from two 32 x 32 -> 64-bit products (c < 2^63).
        const uint64_t ulo = U64 + 1;  // U64 + 1 = (uhi, ulo); wraps when U64 = 2^64 - 1
        const int64_t uhi = U64 == ~0ull ? 1 : 0;
        auto count = [N32, ulo, uhi](uint64_t c) -> uint32_t {
            const uint64_t a = static_cast<uint64_t>(N32) * static_cast<uint32_t>(c);
            const uint64_t m = static_cast<uint64_t>(N32) * static_cast<uint32_t>(c >> 32) + (a >> 32);
            // N c = m 2^32 + (a mod 2^32); X = 4 N c = (m >> 30) 2^64 + xlo
            const uint64_t xlo = ((m << 32) | static_cast<uint32_t>(a)) << 2;
            const int64_t dhi = static_cast<int64_t>(m >> 30) - uhi - (xlo < ulo ? 1 : 0);
            return dhi < 0 ? 0u : (dhi + 1 >= static_cast<int64_t>(N32) ? N32 : static_cast<uint32_t>(dhi) + 1u);
        };
        // Two CTA barriers per tile: one per scan.  The scans use different
        // scratch (shu, shj + THREADS + 1), so each scratch's next writer is
        // behind the other scan's barrier.
        unsigned long long *shw64 = shu;
        uint32_t *she = shj + THREADS + 1;
        uint64_t carry = 0;
        uint32_t ecarry = 0;
        for (uint32_t b = 0; b < N32; b += TILE) {
            const uint32_t q0 = b + threadIdx.x * V;
            const bool whole = q0 + V <= N32;  // all V particles exist
            R lv[V];
            if (whole) {
                ld8(st.l + q0, lv);
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k) lv[k] = q0 + k < N32 ? st.l[q0 + k] : R(0);
            }
            unsigned long long C[V];
            unsigned long long acc = 0;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const double w62 = (whole || q0 + k < N32)
                    ? static_cast<double>(Math<R>::exp(Math<R>::sub(lv[k], M))) * invS62 : 0.0;
                acc += __double2ull_rn(w62);
                C[k] = acc;
            }
            unsigned long long tot;
            const uint64_t base = carry + block_inclusive_sum_1b(acc, shw64, &tot) - acc;
            carry += tot;
            // j of the particle before q0: its cumulative weight is base
            // (j_{-1} = 0 from base = 0)
            const uint32_t jm = count(base);
            uint32_t j[V];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const uint32_t p = q0 + k;
                j[k] = (p + 1 >= N32) ? N32 : count(base + C[k]);
            }
            uint32_t ne = 0;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const uint32_t p = q0 + k;
                ne += (p < N32 && j[k] == (k == 0 ? jm : j[k - 1])) ? 1u : 0u;
            }
            uint32_t etot;
            uint32_t E = ecarry + block_inclusive_sum_1b(ne, she, &etot) - ne;
            ecarry += etot;
            uint32_t sv[V];
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const uint32_t p = q0 + k;
                const uint32_t jb = k == 0 ? jm : j[k - 1];
                sv[k] = jb + E - p;
                if ((whole || p < N32) && j[k] == jb) {
                    ep[E] = p;
                    ++E;
                }
            }
            if (whole) {
                st8(sS + q0, sv);
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k)
                    if (q0 + k < N32) sS[q0 + k] = sv[k];
            }
        }
        __syncthreads();
        n_empty = ecarry;
        // Placement: empty slot ep[k] takes a copy of the parent p with
        // sS_p <= k < sS_{p+1} (the k-th surplus copy goes to the k-th empty
        // slot).  Per tile a warp stages the prefixes of its 256 parents in
        // shared memory; its lanes then take the warp's empties 32 at a time
        // (coalesced loads of ep), each finding its parent by a binary search
        // over the staged prefixes.  Parents are occupied slots and never
        // written, so loads and stores need no ordering.  A warp with more
        // than kWarpCopies copies in a tile is queued and copied by the CTA.
        {
            uint32_t *nbig = shj + THREADS + 34;  // queue length, then queued parent groups
            uint32_t *big = nbig + 1;
            const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            uint32_t *wsw = shj + ws_offset<THREADS>() + warp * kWs;
            if (threadIdx.x == 0) *nbig = 0;
            __syncthreads();
            const uint32_t ne = ecarry;
            for (uint32_t b = 0; b < N32; b += TILE) {
                const uint32_t P0 = b + warp * kWarpParents;
                if (P0 >= N32) continue;  // warp-uniform; the loop holds no CTA barrier
                const uint32_t q0 = P0 + lane * V;
                // the warp's parents go to shared memory with their prefixes
                // (STAGEX), read once and coalesced: a copy's source then
                // costs no dependent global load behind the search (an empty
                // slot staged here may be written meanwhile, but an empty
                // slot is no parent)
                R *wx = STAGEX ? shx + warp * kWarpParents : nullptr;
                {
                    uint32_t ss[V];
                    R xv[V];
                    if (q0 + V <= N32) {
                        ld8(sS + q0, ss);
                        if constexpr (STAGEX) ld8(xc + q0, xv);
                    } else {
#pragma unroll
                        for (int k = 0; k < V; ++k) {
                            ss[k] = q0 + k < N32 ? sS[q0 + k] : ne;
                            if constexpr (STAGEX) xv[k] = q0 + k < N32 ? xc[q0 + k] : R(0);
                        }
                    }
                    st8(wsw + lane * V, ss);
                    if constexpr (STAGEX) st8(wx + lane * V, xv);
                }
                if (lane == 31) wsw[kWarpParents] = q0 + V < N32 ? sS[q0 + V] : ne;
                __syncwarp();
                const uint32_t A = wsw[0], B = wsw[kWarpParents];
                uint32_t queued = 0;
                if (B - A > kWarpCopies && lane == 0) {
                    const uint32_t q = atomicAdd(nbig, 1u);
                    if (q < kBigParents) {
                        big[q] = P0;
                        queued = 1;
                    }
                }
                queued = __shfl_sync(0xffffffffu, queued, 0);
                if (!queued) {
                    if constexpr (STAGEX) {
                        for (uint32_t e = A + lane; e < B; e += 32) {
                            uint32_t lo = 0;
#pragma unroll
                            for (uint32_t h = kWarpParents / 2; h >= 1; h >>= 1) lo += wsw[lo + h] <= e ? h : 0;
                            const uint32_t slot = ep[e];
                            xc[slot] = wx[lo];
                            if constexpr (SHADOW) xsc[slot] = xsc[P0 + lo];
                        }
                    } else {
                        for (uint32_t e = A + lane; e < B; e += 32) {
                            uint32_t lo = 0;
#pragma unroll
                            for (uint32_t h = kWarpParents / 2; h >= 1; h >>= 1) lo += wsw[lo + h] <= e ? h : 0;
                            const uint32_t slot = ep[e];
                            xc[slot] = xc[P0 + lo];
                            if constexpr (SHADOW) xsc[slot] = xsc[P0 + lo];
                        }
                    }
                }
                __syncwarp();  // the staging area is rewritten by the next tile
            }
            __syncthreads();
            const uint32_t nb = min(*nbig, kBigParents);
            uint32_t *wsc = shj + ws_offset<THREADS>();  // warp 0's area, now free
            for (uint32_t i = 0; i < nb; ++i) {
                const uint32_t P0 = big[i];
                for (uint32_t k = threadIdx.x; k <= kWarpParents; k += THREADS) wsc[k] = P0 + k < N32 ? sS[P0 + k] : ne;
                __syncthreads();
                const uint32_t A = wsc[0], B = wsc[kWarpParents];
                for (uint32_t e = A + threadIdx.x; e < B; e += THREADS) {
                    uint32_t lo = 0;
#pragma unroll
                    for (uint32_t h = kWarpParents / 2; h >= 1; h >>= 1) lo += wsc[lo + h] <= e ? h : 0;
                    const uint32_t slot = ep[e];
                    xc[slot] = xc[P0 + lo];
                    if constexpr (SHADOW) xsc[slot] = xsc[P0 + lo];
                }
                __syncthreads();
            }
        }
        __syncthreads();
        // the particles now carry equal weights
        st.flat = true;
        L_prev = log(static_cast<double>(N));
        Ls_prev = L_prev;
        return true;
    }
};

// `par` (nullable): the filters' model parameters, which the shadow run
// shares; without it the parameters are the built-in AR(1) model's, from the
// descriptors.
template <typename R, int THREADS, bool SHADOW, int MINB, class Model = Ar1Model>
__global__ void __launch_bounds__(THREADS, MINB) k_pf_batched(const BatchedFilter *filt, const int *order, int nf,
    const double *y, int T, double threshold, R *xa, R *xb, R *lw, uint32_t *scanS, uint32_t *epos,
    double *loglik, uint32_t *nresampled, int *queue, double *xsa, double *xsb, double *lws,
    double *loglik_shadow, const typename Model::Param *par = nullptr)
{
    __shared__ double shd[33];
    __shared__ R shr[33];
    __shared__ unsigned long long shu[33];
    __shared__ __align__(16) uint32_t shj[shj_words<THREADS>()];
    // the placement's staged parent positions, where they fit beside shj in
    // the 48 KB of static shared memory without cutting the residency
    constexpr bool kStageX = THREADS <= 512 && sizeof(R) * (THREADS / 32) * kWarpParents <= 16384;
    __shared__ __align__(16) R shx[kStageX ? (THREADS / 32) * kWarpParents : 1];
    __shared__ int sh_f;
    while (true) {
        if (threadIdx.x == 0) {
            const int k = atomicAdd(queue, 1);
            sh_f = k < nf ? order[k] : -1;
        }
        __syncthreads();
        const int f = sh_f;
        __syncthreads();
        if (f < 0) break;
        FilterRun<R, THREADS, SHADOW, Model> run;
        if (par) {
            run.setup(filt[f], par[f], par[f], xa, xb, lw, scanS, epos, xsa, xsb, lws, threshold);
        } else {
            if constexpr (std::is_same<Model, Ar1Model>::value)
                run.setup(filt[f], xa, xb, lw, scanS, epos, xsa, xsb, lws, threshold);
        }
        const double *yf = y + static_cast<uint64_t>(f) * (T + 1);
        for (int t = 0; t <= T; ++t) run.template step<kStageX>(t, yf[t], shd, shr, shu, shj, shx);
        if (threadIdx.x == 0) {
            loglik[f] = run.ll_sum;
            nresampled[f] = static_cast<uint32_t>(run.events);
            if constexpr (SHADOW) loglik_shadow[f] = run.lls_sum;
        }
        __syncthreads();
    }
}


}  // namespace batched_detail
}  // namespace mckl_b200
