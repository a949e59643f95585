// pf_batched.cu -- the chosen form: many independent AR(1) bootstrap filters
// with uneven particle counts in one persistent kernel.
//
// Each CTA pulls filters from a work queue (largest first) and runs all T
// steps of a filter before taking the next.  Per step and filter:
//   noise      Normal(0,1) from the filter's model stream, consumed exactly as
//              normal_distribution does (random/normal_distribution.hpp:50-101:
//              1024-value chunks, radius word i and angle word K/2 + i, odd n
//              redrawn from two more words), so the plain FP64 path with the
//              same keys sees the same uniforms;
//   propagate  x = phi x + sx eps, log-likelihood, log-weight update: FP32;
//   normalise  max, sum of exp and of exp^2 (ESS), log normaliser and the
//              log-likelihood increment: FP64 accumulation;
//   resample   systematic (algorithm/resample.hpp:258-268) when ESS < N/2,
//              from the filter's resample stream (two words per event):
//              FP64 inclusive scan of the weights, replication counts by the
//              closed-form lower bound of the systematic grid, the reference's
//              slot-preserving parent assignment (:416-466) by two CTA scans
//              and a binary search per empty slot, then the particle gather.
// Particle state (x, log-weights) lives in global memory, contiguous per
// filter; only the filters in flight are touched, so it stays in L2.
#include <algorithm>
#include <cmath>
#include <vector>

#include "block_scan.cuh"
#include "common.cuh"
#include "pf_batched.cuh"

namespace mckl_b200 {

namespace {

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

// U01OC<double> of a word, rounded to the propagation type
template <typename R>
__device__ __forceinline__ R u01oc(uint32_t w)
{
    return static_cast<R>(__dadd_rn(__dmul_rn(static_cast<double>(w), 0x1p-32), 0x1p-32));
}

template <typename R>
struct Math;

template <>
struct Math<float> {
    __device__ static float radius(float u) { return sqrtf(-2.0f * logf(u)); }
    __device__ static void sincos2pi(float v, float *s, float *c) { sincospif(2.0f * v, s, c); }
    __device__ static float cos2pi(float v) { return cospif(2.0f * v); }
    __device__ static float exp(float a) { return expf(a); }
};

template <>
struct Math<double> {
    __device__ static double radius(double u) { return sqrt(-2.0 * log(u)); }
    __device__ static void sincos2pi(double v, double *s, double *c) { sincospi(2.0 * v, s, c); }
    __device__ static double cos2pi(double v) { return cospi(2.0 * v); }
    __device__ static double exp(double a) { return ::exp(a); }
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
            s *= sc;
            q *= sc * sc;
            m = gm;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (k >= lo && k < hi) {
                const double e = static_cast<double>(Math<R>::exp(v[k] - m));
                s += e;
                q += e * e;
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
    *S = block_sum(a.s * sc, shd);
    if (Q) *Q = block_sum(a.q * sc * sc, shd);
}

// One Box-Muller pair of one filter at step t: the noise from a radius and an
// angle word, the AR(1) move of particles p0 and p1, their new log-weights
// (old log-weight minus the previous step's maximum, plus the observation's
// log-density; zero old weights after a resampling) and, for the shadow, the
// same in FP64.  Returns the two log-weights in v[0], v[1].
template <typename R, bool SHADOW>
struct Step {
    R *x, *l;
    double *xs, *ls;
    R phi, sx, sd0, lconst, hinv, yt, lshift;
    double phi_d, sx_d, sd0_d, lconst_d, hinv_d, yt_d, lshift_s;
    bool init, flat;

    __device__ __forceinline__ void pair(uint32_t wrad, uint32_t wang, uint64_t p0, uint64_t p1, R *v, double *vs) const
    {
        const R rr = Math<R>::radius(u01oc<R>(wrad));
        R sn, cs;
        Math<R>::sincos2pi(u01oc<R>(wang), &sn, &cs);
        one(rr * sn, p0, v[0]);
        one(rr * cs, p1, v[1]);
        if constexpr (SHADOW) {
            const double rd = Math<double>::radius(u01oc<double>(wrad));
            double snd, csd;
            Math<double>::sincos2pi(u01oc<double>(wang), &snd, &csd);
            one_shadow(rd * snd, p0, vs[0]);
            one_shadow(rd * csd, p1, vs[1]);
        }
    }

    __device__ __forceinline__ void one(R e, uint64_t p, R &v) const
    {
        if (init) {
            x[p] = sd0 * e;
            return;
        }
        const R xn = phi * x[p] + sx * e;
        x[p] = xn;
        const R r = yt - xn;
        const R lo = flat ? R(0) : l[p] - lshift;
        v = lo + (lconst - r * r * hinv);
        l[p] = v;
    }

    __device__ __forceinline__ void one_shadow(double e, uint64_t p, double &v) const
    {
        if (init) {
            xs[p] = sd0_d * e;
            return;
        }
        const double xn = phi_d * xs[p] + sx_d * e;
        xs[p] = xn;
        const double r = yt_d - xn;
        const double lo = flat ? 0.0 : ls[p] - lshift_s;
        v = lo + (lconst_d - r * r * hinv_d);
        ls[p] = v;
    }
};

// SHADOW (with R = float): every particle also carries an FP64 copy that is
// propagated with the same uniforms, weighted in FP64 and resampled with the
// FP32 run's decisions and parent indices; its log-likelihood isolates the
// FP32 arithmetic error from the Monte Carlo divergence a flipped ancestor
// would otherwise start.
//
// Work split of one step: the Normal(0,1) draws of a filter are 1024-value
// chunks (radius word i, angle word 512 + i of the chunk, as
// normal_distribution lays them out).  A full chunk is covered by 129 units;
// unit g owns the radius words of Philox block (chunk start / 4) + g and the
// angle words of the block 128 further on, i.e. up to four pairs for two
// Philox blocks (a quarter block per particle).  The last partial chunk and an
// odd last particle are drawn word by word.
template <typename R, int THREADS, bool SHADOW>
__global__ void __launch_bounds__(THREADS) k_pf_batched(const BatchedFilter *filt, const int *order, int nf,
    const double *y, int T, double threshold, R *xa, R *xb, R *lw, uint32_t *scanS, uint32_t *epos,
    double *loglik, uint32_t *nresampled, int *queue, double *xsa, double *xsb, double *lws,
    double *loglik_shadow)
{
    __shared__ double shd[33];
    __shared__ R shr[33];
    __shared__ unsigned long long shu[33];
    __shared__ uint32_t shj[THREADS + 1];
    __shared__ int sh_f;
    constexpr uint64_t kUnits = 129;  // units per full chunk
    while (true) {
        if (threadIdx.x == 0) {
            const int k = atomicAdd(queue, 1);
            sh_f = k < nf ? order[k] : -1;
        }
        __syncthreads();
        const int f = sh_f;
        __syncthreads();
        if (f < 0) break;
        const BatchedFilter F = filt[f];
        const uint64_t N = F.n;
        R *xc = xa + F.off, *xn = xb + F.off;
        double *xsc = SHADOW ? xsa + F.off : nullptr, *xsn = SHADOW ? xsb + F.off : nullptr;
        uint32_t *sS = scanS + F.off, *ep = epos + F.off;
        const PhiloxGen gm{F.mkey[0], F.mkey[1]}, gr{F.rkey[0], F.rkey[1]};
        const uint64_t per_step = N + (N & 1) * 2;  // words of one normal_distribution(N) call
        const uint64_t m = N / 1024, tail = N % 1024, nu_tail = tail / 2;
        const uint64_t units = m * kUnits + nu_tail;
        Step<R, SHADOW> st;
        st.l = lw + F.off;
        st.ls = SHADOW ? lws + F.off : nullptr;
        st.phi = static_cast<R>(F.phi);
        st.sx = static_cast<R>(F.sx);
        st.sd0 = static_cast<R>(F.sd0);
        st.lconst = static_cast<R>(F.lconst);
        st.hinv = static_cast<R>(F.hinv);
        st.phi_d = F.phi;
        st.sx_d = F.sx;
        st.sd0_d = F.sd0;
        st.lconst_d = F.lconst;
        st.hinv_d = F.hinv;
        st.lshift = 0;
        st.lshift_s = 0.0;
        st.flat = true;
        double L_prev = log(static_cast<double>(N)), ll_sum = 0.0;
        double Ls_prev = L_prev, lls_sum = 0.0;
        uint64_t events = 0;
        for (int t = 0; t <= T; ++t) {
            const uint64_t P = static_cast<uint64_t>(t) * per_step;
            st.x = xc;
            st.xs = xsc;
            st.init = (t == 0);
            st.yt_d = y[static_cast<uint64_t>(f) * (T + 1) + t];
            st.yt = static_cast<R>(st.yt_d);
            Lse<R> acc;
            Lse<double> accs;
            // ---- noise, propagation, log-weights, online normaliser
            for (uint64_t u = threadIdx.x; u < units; u += THREADS) {
                R v[8];
                double vs[8];
                if (u < m * kUnits) {
                    const uint64_t c = u / kUnits, g = u % kUnits;
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
                            st.pair(wr[j], wa[j], p0, p0 + 512, v + 2 * j, vs + 2 * j);
                        }
                    }
                    if (t > 0) {
                        acc.add(v, 2 * lo, 2 * hi);
                        if constexpr (SHADOW) accs.add(vs, 2 * lo, 2 * hi);
                    }
                } else {
                    const uint64_t i = u - m * kUnits, base = P + m * 1024;
                    WordCache wc{~0ull, {0, 0, 0, 0}};
                    const uint32_t wrad = word_at(gm, base + i, wc);
                    const uint32_t wang = word_at(gm, base + nu_tail + i, wc);
                    st.pair(wrad, wang, m * 1024 + i, m * 1024 + nu_tail + i, v, vs);
                    if (t > 0) {
                        acc.add(v, 0, 2);
                        if constexpr (SHADOW) accs.add(vs, 0, 2);
                    }
                }
            }
            if ((N & 1) && threadIdx.x == THREADS - 1) {
                // odd N: the last particle from the two words after the chunks
                WordCache wc{~0ull, {0, 0, 0, 0}};
                const uint32_t w0 = word_at(gm, P + N, wc), w1 = word_at(gm, P + N + 1, wc);
                R v[1];
                double vs[1];
                st.one(Math<R>::radius(u01oc<R>(w0)) * Math<R>::cos2pi(u01oc<R>(w1)), N - 1, v[0]);
                if constexpr (SHADOW)
                    st.one_shadow(Math<double>::radius(u01oc<double>(w0)) * Math<double>::cos2pi(u01oc<double>(w1)),
                        N - 1, vs[0]);
                if (t > 0) {
                    acc.add(v, 0, 1);
                    if constexpr (SHADOW) accs.add(vs, 0, 1);
                }
            }
            if (t == 0) {
                __syncthreads();
                continue;
            }
            // ---- FP64 normaliser: S = sum exp(l - M), Q = sum exp^2; the
            // log normaliser of the weights relative to M is carried to the
            // next step, whose log-weights start from l - M
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
            const double ess = S * S / Q;
            if (!(ess < static_cast<double>(N) * threshold)) continue;
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
            const double delta = 1.0 / static_cast<double>(N);
            const double ud = U * delta;
            const double invS = 1.0 / S;
            // per tile of THREADS particles: inclusive FP64 scan of the
            // normalised weights, cumulative counts j_p = #{k : u_k < c_p}
            // (the lower bound of c_p on the grid fma(k, delta, ud)), the
            // replication counts j_p - j_{p-1}, and the exclusive scan of
            // (empty slot, surplus copies) that places the parents
            double carry = 0.0;
            unsigned long long carry2 = 0;
            uint32_t jprev = 0;
            for (uint64_t b = 0; b < N; b += THREADS) {
                const uint64_t p = b + threadIdx.x;
                const double w = p < N ? static_cast<double>(Math<R>::exp(st.l[p] - M)) * invS : 0.0;
                double tot;
                const double c = carry + block_inclusive_sum(w, shd, &tot);
                carry += tot;
                uint32_t jp = static_cast<uint32_t>(N);
                if (p + 1 < N) {
                    double jf = ceil((c - ud) * static_cast<double>(N));
                    long long j = jf < 0 ? 0 : (jf > static_cast<double>(N) ? static_cast<long long>(N) : static_cast<long long>(jf));
                    while (j > 0 && fma(static_cast<double>(j - 1), delta, ud) >= c) --j;
                    while (j < static_cast<long long>(N) && fma(static_cast<double>(j), delta, ud) < c) ++j;
                    jp = static_cast<uint32_t>(j);
                }
                shj[threadIdx.x + 1] = jp;
                if (threadIdx.x == 0) shj[0] = jprev;
                __syncthreads();
                const uint32_t rep = p < N ? shj[threadIdx.x + 1] - shj[threadIdx.x] : 0u;
                jprev = shj[THREADS];
                const unsigned long long v = p < N ? ((rep == 0 ? 1ull : 0ull) | (static_cast<unsigned long long>(rep > 0 ? rep - 1 : 0) << 32)) : 0ull;
                unsigned long long tot2;
                const unsigned long long inc = block_inclusive_sum(v, shu, &tot2);
                const unsigned long long ex = carry2 + inc - v;
                carry2 += tot2;
                if (p < N) {
                    sS[p] = static_cast<uint32_t>(ex >> 32);
                    if (rep == 0) {
                        ep[ex & 0xffffffffull] = static_cast<uint32_t>(p);
                    } else {
                        xn[p] = xc[p];  // occupied slots keep their particle
                        if constexpr (SHADOW) xsn[p] = xsc[p];
                    }
                }
            }
            __syncthreads();
            const uint64_t n_empty = carry2 & 0xffffffffull;
            for (uint64_t k = threadIdx.x; k < n_empty; k += THREADS) {
                uint64_t lo = 0, hi = N;  // last source with surplus prefix <= k
                while (hi - lo > 1) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (sS[mid] <= k) {
                        lo = mid;
                    } else {
                        hi = mid;
                    }
                }
                xn[ep[k]] = xc[lo];
                if constexpr (SHADOW) xsn[ep[k]] = xsc[lo];
            }
            __syncthreads();
            // the gathered particles become the current ones, with equal weights
            R *tx = xc;
            xc = xn;
            xn = tx;
            if constexpr (SHADOW) {
                double *ts = xsc;
                xsc = xsn;
                xsn = ts;
            }
            st.flat = true;
            L_prev = log(static_cast<double>(N));
            Ls_prev = L_prev;
        }
        if (threadIdx.x == 0) {
            loglik[f] = ll_sum;
            nresampled[f] = static_cast<uint32_t>(events);
            if constexpr (SHADOW) loglik_shadow[f] = lls_sum;
        }
        __syncthreads();
    }
}

template <typename R, int THREADS, bool SHADOW>
int launch_one(const BatchedArgs &a, const int *order, int nf, int *queue, int ctas, cudaStream_t s)
{
    k_pf_batched<R, THREADS, SHADOW><<<ctas, THREADS, 0, s>>>(a.filt, order, nf, a.y, a.T, a.threshold,
        static_cast<R *>(a.xa), static_cast<R *>(a.xb), static_cast<R *>(a.lw), a.scanS, a.epos,
        a.loglik, a.nresampled, queue, a.xsa, a.xsb, a.lws, a.loglik_shadow);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

template <typename R, int THREADS, bool SHADOW>
int occupancy_one(int *blocks)
{
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_pf_batched<R, THREADS, SHADOW>, THREADS, 0));
    return MCKL_B200_OK;
}

template <typename R, bool SHADOW>
int occupancy_threads(int threads, int *blocks)
{
    switch (threads) {
        case 128: return occupancy_one<R, 128, SHADOW>(blocks);
        case 256: return occupancy_one<R, 256, SHADOW>(blocks);
        case 512: return occupancy_one<R, 512, SHADOW>(blocks);
        default: return occupancy_one<R, 1024, SHADOW>(blocks);
    }
}

template <typename R, bool SHADOW>
int launch_threads(const BatchedArgs &a, const int *order, int nf, int threads, int *queue, int ctas, cudaStream_t s)
{
    switch (threads) {
        case 128: return launch_one<R, 128, SHADOW>(a, order, nf, queue, ctas, s);
        case 256: return launch_one<R, 256, SHADOW>(a, order, nf, queue, ctas, s);
        case 512: return launch_one<R, 512, SHADOW>(a, order, nf, queue, ctas, s);
        default: return launch_one<R, 1024, SHADOW>(a, order, nf, queue, ctas, s);
    }
}

}  // namespace

// resident CTAs per SM of the kernel variant the arguments select
int pf_batched_occupancy(const BatchedArgs &a, int threads, int *blocks)
{
    if (a.fp64) return occupancy_threads<double, false>(threads, blocks);
    if (a.xsa) return occupancy_threads<float, true>(threads, blocks);
    return occupancy_threads<float, false>(threads, blocks);
}

int pf_batched_launch(const BatchedArgs &a, const int *order, int nf, int threads, int ctas_per_sm, int *queue,
    cudaStream_t s)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ctas = std::max(1, std::min(nf, sms * ctas_per_sm));
    MB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), s));
    if (a.fp64) return launch_threads<double, false>(a, order, nf, threads, queue, ctas, s);
    if (a.xsa) return launch_threads<float, true>(a, order, nf, threads, queue, ctas, s);
    return launch_threads<float, false>(a, order, nf, threads, queue, ctas, s);
}

}  // namespace mckl_b200

// ---------------------------------------------------------------------------
// C ABI: a handle owns the uploaded filters, observations and work arrays, so
// the launch itself (mckl_b200_batched_run) is a single capturable kernel.
// ---------------------------------------------------------------------------
struct mckl_b200_batched {
    int F = 0, T = 0;
    uint64_t total = 0;
    double threshold = 0.5;
    int fp64 = 0, threads = 256, ctas_per_sm = 4;
    void *mem = nullptr;
    mckl_b200::BatchedArgs a{};
    int *order = nullptr, *queue = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
};

using namespace mckl_b200;

extern "C" {

int mckl_b200_batched_create(mckl_b200_batched_t **out, size_t F, const size_t *N, size_t T, const double *y,
    const double *phi, const double *sx, const double *sy, const uint32_t *mkeys, const uint32_t *rkeys,
    double threshold, int fp64)
{
    MB_CHECK_ARG(out != nullptr && F > 0 && T > 0, "bad arguments");
    MB_CHECK_ARG(N && y && phi && sx && sy && mkeys && rkeys, "null argument");
    std::vector<BatchedFilter> h(F);
    uint64_t total = 0;
    for (size_t f = 0; f < F; ++f) {
        MB_CHECK_ARG(N[f] >= 1 && N[f] < (1ull << 31), "particle counts must be in [1, 2^31)");
        MB_CHECK_ARG(sy[f] > 0 && phi[f] * phi[f] < 1, "need sy > 0 and |phi| < 1");
        h[f].n = N[f];
        h[f].off = total;
        h[f].phi = phi[f];
        h[f].sx = sx[f];
        h[f].sd0 = sx[f] / std::sqrt(1 - phi[f] * phi[f]);
        h[f].lconst = -std::log(sy[f]) - 0.5 * std::log(2 * 3.14159265358979323846);
        h[f].hinv = 0.5 / (sy[f] * sy[f]);
        h[f].mkey[0] = mkeys[2 * f];
        h[f].mkey[1] = mkeys[2 * f + 1];
        h[f].rkey[0] = rkeys[2 * f];
        h[f].rkey[1] = rkeys[2 * f + 1];
        total += (N[f] + 31) / 32 * 32;
    }
    // largest filters first (longest-processing-time order for the work queue)
    std::vector<int> order(F);
    for (size_t f = 0; f < F; ++f) order[f] = static_cast<int>(f);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return N[a] > N[b]; });
    auto *b = new mckl_b200_batched;
    b->F = static_cast<int>(F);
    b->T = static_cast<int>(T);
    b->total = total;
    b->threshold = threshold;
    const bool shadow = (fp64 == 2);
    b->fp64 = (fp64 == 1) ? 1 : 0;
    const size_t rs = b->fp64 ? 8 : 4;
    const size_t bytes = align256(F * sizeof(BatchedFilter)) + align256(F * (T + 1) * 8) + 3 * align256(total * rs) +
                         2 * align256(total * 4) + align256(F * 8) + align256(F * 4) + align256(F * 4) + 256 +
                         (shadow ? 3 * align256(total * 8) + align256(F * 8) : 0);
    if (cudaMalloc(&b->mem, bytes) != cudaSuccess) {
        delete b;
        set_error("batched filter allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    char *p = static_cast<char *>(b->mem);
    auto take = [&p](size_t n) {
        char *q = p;
        p += align256(n);
        return q;
    };
    b->a.filt = reinterpret_cast<BatchedFilter *>(take(F * sizeof(BatchedFilter)));
    b->a.y = reinterpret_cast<double *>(take(F * (T + 1) * 8));
    b->a.xa = take(total * rs);
    b->a.xb = take(total * rs);
    b->a.lw = take(total * rs);
    b->a.scanS = reinterpret_cast<uint32_t *>(take(total * 4));
    b->a.epos = reinterpret_cast<uint32_t *>(take(total * 4));
    b->a.loglik = reinterpret_cast<double *>(take(F * 8));
    b->a.nresampled = reinterpret_cast<uint32_t *>(take(F * 4));
    b->order = reinterpret_cast<int *>(take(F * 4));
    b->queue = reinterpret_cast<int *>(take(256));
    if (shadow) {
        b->a.xsa = reinterpret_cast<double *>(take(total * 8));
        b->a.xsb = reinterpret_cast<double *>(take(total * 8));
        b->a.lws = reinterpret_cast<double *>(take(total * 8));
        b->a.loglik_shadow = reinterpret_cast<double *>(take(F * 8));
    }
    b->a.T = static_cast<int>(T);
    b->a.threshold = threshold;
    b->a.fp64 = b->fp64;
    MB_CUDA(cudaMemcpy(b->a.filt, h.data(), F * sizeof(BatchedFilter), cudaMemcpyHostToDevice));
    MB_CUDA(cudaMemcpy(b->a.y, y, F * (T + 1) * 8, cudaMemcpyHostToDevice));
    MB_CUDA(cudaMemcpy(b->order, order.data(), F * 4, cudaMemcpyHostToDevice));
    *out = b;
    return MCKL_B200_OK;
}

int mckl_b200_batched_config(mckl_b200_batched_t *b, int threads, int ctas_per_sm)
{
    MB_CHECK_ARG(b != nullptr, "null handle");
    MB_CHECK_ARG(threads == 128 || threads == 256 || threads == 512 || threads == 1024, "threads: 128/256/512/1024");
    MB_CHECK_ARG(ctas_per_sm >= 1 && ctas_per_sm <= 32, "ctas_per_sm in [1, 32]");
    b->threads = threads;
    b->ctas_per_sm = ctas_per_sm;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return MCKL_B200_OK;
}

int mckl_b200_batched_run(mckl_b200_batched_t *b, void *stream)
{
    MB_CHECK_ARG(b != nullptr, "null handle");
    return pf_batched_launch(b->a, b->order, b->F, b->threads, b->ctas_per_sm, b->queue, as_stream(stream));
}

int mckl_b200_batched_run_graph(mckl_b200_batched_t *b, void *stream)
{
    MB_CHECK_ARG(b != nullptr, "null handle");
    cudaStream_t s = as_stream(stream);
    if (!b->exec) {
        cudaStream_t cap;
        MB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        MB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const int rc = pf_batched_launch(b->a, b->order, b->F, b->threads, b->ctas_per_sm, b->queue, cap);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc != MCKL_B200_OK) return rc;
        MB_CUDA(ce);
        b->graph = g;
        MB_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    }
    MB_CUDA(cudaGraphLaunch(b->exec, s));
    count_launch();
    return MCKL_B200_OK;
}

int mckl_b200_batched_autotune(mckl_b200_batched_t *b, int max_trials, int *threads, int *ctas_per_sm,
    float *ms, int *ntrials, void *stream)
{
    MB_CHECK_ARG(b != nullptr && max_trials >= 0, "bad arguments");
    cudaStream_t s = as_stream(stream);
    // candidate block shapes: 4 to 8 warps per scheduler in total, from many
    // small CTAs (small filters keep every thread busy) to few large ones
    // (fewer barriers per particle on the large filters)
    static const int cand[][2] = {{128, 8}, {128, 12}, {256, 4}, {256, 6}, {512, 2}, {512, 3}, {1024, 1}, {1024, 2}};
    int best = -1, n = 0;
    float best_ms = 0.0f;
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    // one untimed run first (module load, caches)
    int rc = pf_batched_launch(b->a, b->order, b->F, 256, 4, b->queue, s);
    for (int k = 0; rc == MCKL_B200_OK && k < static_cast<int>(sizeof(cand) / sizeof(cand[0])); ++k) {
        int fit = 0;
        rc = pf_batched_occupancy(b->a, cand[k][0], &fit);
        if (rc != MCKL_B200_OK) break;
        if (fit < cand[k][1]) continue;  // would not be resident at once
        cudaEventRecord(e0, s);
        rc = pf_batched_launch(b->a, b->order, b->F, cand[k][0], cand[k][1], b->queue, s);
        cudaEventRecord(e1, s);
        if (rc != MCKL_B200_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = MCKL_B200_ERR_CUDA;
            set_error("autotune: kernel failed");
            break;
        }
        float t = 0.0f;
        cudaEventElapsedTime(&t, e0, e1);
        if (n < max_trials) {
            if (threads) threads[n] = cand[k][0];
            if (ctas_per_sm) ctas_per_sm[n] = cand[k][1];
            if (ms) ms[n] = t;
        }
        ++n;
        if (best < 0 || t < best_ms) {
            best = k;
            best_ms = t;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ntrials) *ntrials = n;
    if (rc != MCKL_B200_OK) return rc;
    MB_CHECK_ARG(best >= 0, "autotune: no candidate block shape fits");
    return mckl_b200_batched_config(b, cand[best][0], cand[best][1]);
}

int mckl_b200_batched_set_y(mckl_b200_batched_t *b, const double *y, void *stream)
{
    MB_CHECK_ARG(b != nullptr && y != nullptr, "null argument");
    MB_CUDA(cudaMemcpyAsync(b->a.y, y, static_cast<size_t>(b->F) * (b->T + 1) * 8, cudaMemcpyHostToDevice,
        as_stream(stream)));
    return MCKL_B200_OK;
}

int mckl_b200_batched_shadow(mckl_b200_batched_t *b, double *loglik_fp64, void *stream)
{
    MB_CHECK_ARG(b != nullptr && loglik_fp64 != nullptr, "null argument");
    MB_CHECK_ARG(b->a.loglik_shadow != nullptr, "the handle was not created with fp64 = 2 (shadow)");
    cudaStream_t s = as_stream(stream);
    MB_CUDA(cudaMemcpyAsync(loglik_fp64, b->a.loglik_shadow, b->F * 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return MCKL_B200_OK;
}

int mckl_b200_batched_results(mckl_b200_batched_t *b, double *loglik, uint32_t *nresampled, void *stream)
{
    MB_CHECK_ARG(b != nullptr, "null handle");
    cudaStream_t s = as_stream(stream);
    if (loglik) MB_CUDA(cudaMemcpyAsync(loglik, b->a.loglik, b->F * 8, cudaMemcpyDeviceToHost, s));
    if (nresampled) MB_CUDA(cudaMemcpyAsync(nresampled, b->a.nresampled, b->F * 4, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return MCKL_B200_OK;
}

int mckl_b200_batched_destroy(mckl_b200_batched_t *b)
{
    if (!b) return MCKL_B200_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->mem) cudaFree(b->mem);
    delete b;
    return MCKL_B200_OK;
}

}  // extern "C"
