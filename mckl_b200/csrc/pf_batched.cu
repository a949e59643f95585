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
#include <cstring>
#include <map>
#include <mutex>
#include <cmath>
#include <vector>

#include "block_scan.cuh"
#include "common.cuh"
#include "pf_batched.cuh"
#include "pf_batched_kernel.cuh"

namespace mckl_b200 {

namespace {

using namespace batched_detail;

// ---------------------------------------------------------------------------
// Adjoint: gradient of the FP64 log-likelihood estimate with respect to
// (phi, sx, sy), ancestors and resampling times held fixed.
//
// With the resampling steps r_1 < r_2 < ... fixed, the estimate is
//   logL = sum over segments of [log sum_i exp(l_i at the segment's end) - log N],
// l_i the sum of log g(y_t | x_t^i) over the segment, and x_t^j = phi
// x~_{t-1}^j + sx eps_t^j, x~ the (possibly resampled) particles,
// x_0 = sd0 eps_0 with sd0 = sx / sqrt(1 - phi^2).  Reverse mode, t = T..0,
// with lambda_t = d logL / d x_t and w the softmax of l at the end of the
// segment containing t:
//   mu_t^i     = sum over children j of i of lambda_{t+1}^j  (gather; fixed ancestors)
//   lambda_t^i = phi mu_t^i + w^i (y_t - x_t^i) / sy^2
//   d/dphi  += sum_i x_t^i mu_t^i,   d/dsx += sum_j lambda_t^j eps_t^j,
//   d/dsy   += sum_i w^i (-1/sy + (y_t - x_t^i)^2 / sy^3),
// and at t = 0 the sd0 terms.  The forward pass keeps a checkpoint (particles,
// log-weights, scalars) every C steps; the backward pass replays each block
// of C steps from its checkpoint with the same kernel code -- same counters,
// so the same noise, decisions and ancestors -- recording the particles and
// the parent placement, then sweeps the block backwards.  The noise eps_t is
// recomputed from the counters again in the sweep.  Nothing of size T x N is
// stored.
// ---------------------------------------------------------------------------
struct AdjointArgs {
    int C;                 // checkpoint interval (steps)
    uint64_t total;        // particles over all filters (checkpoint stride)
    double *ck_x, *ck_l;   // checkpoint k of filter f: [k * total + off, + n)
    FilterScalars *ck_s;   // [k * F + f]
    int F;
    // per-CTA work areas, each for nmax particles
    uint64_t nmax;
    double *rec_x, *rec_l; // C x nmax per CTA
    uint32_t *rec_rep, *rec_sS, *rec_ep;
    uint8_t *rec_flag;     // C per CTA
    uint32_t *rec_ne;      // empty slots of each recorded resampling, C per CTA
    double *lam, *mu, *wend;  // nmax per CTA
    double *grad;          // 3 per filter
};

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_pf_adjoint(const BatchedFilter *filt, const int *order, int nf,
    const double *y, int T, double threshold, double *xa, double *xb, double *lw, uint32_t *scanS, uint32_t *epos,
    double *loglik, uint32_t *nresampled, int *queue, AdjointArgs A)
{
    __shared__ double shd[33];
    __shared__ unsigned long long shu[33];
    __shared__ __align__(16) uint32_t shj[shj_words<THREADS>()];
    __shared__ int sh_f;
    const int C = A.C;
    const uint64_t slot = blockIdx.x, cn = static_cast<uint64_t>(C) * A.nmax;
    double *rx = A.rec_x + slot * cn, *rl = A.rec_l + slot * cn;
    uint32_t *rrep = A.rec_rep + slot * cn, *rsS = A.rec_sS + slot * cn, *rep_list = A.rec_ep + slot * cn;
    uint8_t *rflag = A.rec_flag + slot * C;
    uint32_t *rne = A.rec_ne + slot * C;
    double *lam = A.lam + slot * A.nmax, *mu = A.mu + slot * A.nmax, *wend = A.wend + slot * A.nmax;
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
        const double *yf = y + static_cast<uint64_t>(f) * (T + 1);
        const double phi = F.phi, sx = F.sx, sy = F.sy;
        const double sy2inv = 1.0 / (sy * sy);
        FilterRun<double, THREADS, false> run;
        run.setup(F, xa, xb, lw, scanS, epos, nullptr, nullptr, nullptr, threshold);
        auto save = [&](int k) {
            double *cx = A.ck_x + static_cast<uint64_t>(k) * A.total + F.off;
            double *cl = A.ck_l + static_cast<uint64_t>(k) * A.total + F.off;
            for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                cx[p] = run.xc[p];
                cl[p] = run.st.l[p];
            }
            if (threadIdx.x == 0) A.ck_s[static_cast<uint64_t>(k) * A.F + f] = run.scalars();
            __syncthreads();  // the next step overwrites the particles
        };
        // ---- forward pass; checkpoints of the state after steps 0, C, 2C, ...
        for (int t = 0; t <= T; ++t) {
            run.step(t, yf[t], shd, shd, shu, shj);
            if (t % C == 0) save(t / C);
        }
        if (threadIdx.x == 0) {
            loglik[f] = run.ll_sum;
            nresampled[f] = static_cast<uint32_t>(run.events);
        }
        __syncthreads();
        // ---- backward pass
        double g_phi = 0.0, g_sx = 0.0, g_sy = 0.0;
        for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
            lam[p] = 0.0;
            wend[p] = 0.0;
        }
        __syncthreads();
        // noise of step t paired with lambda: sum_j lambda_j eps_j
        auto lam_eps = [&](int t) {
            double acc = 0.0;
            for (uint32_t u = threadIdx.x; u < static_cast<uint32_t>(run.lay.units); u += THREADS) {
                int lo, hi;
                run.lay.unit(run.gm, t, u, &lo, &hi, [&](uint32_t wrad, uint32_t wang, uint64_t p0, uint64_t p1, int) {
                    const double r = Math<double>::radius(u01oc<double>(wrad));
                    double sn, cs;
                    Math<double>::sincos2pi(u01oc<double>(wang), &sn, &cs);
                    acc += lam[p0] * __dmul_rn(r, sn) + lam[p1] * __dmul_rn(r, cs);
                });
            }
            if ((N & 1) && threadIdx.x == THREADS - 1) {
                uint32_t w0, w1;
                run.lay.odd_words(run.gm, t, &w0, &w1);
                acc += lam[N - 1] * __dmul_rn(Math<double>::radius(u01oc<double>(w0)), Math<double>::cos2pi(u01oc<double>(w1)));
            }
            return acc;
        };
        const int nblk = T / C;  // blocks (kC, min(kC + C, T)], k = 0 .. nblk
        for (int k = nblk; k >= 0; --k) {
            const int t0 = k * C, t1 = min(t0 + C, T);
            if (t1 <= t0) continue;
            // replay steps t0+1 .. t1 from checkpoint k, recording them
            {
                const double *cx = A.ck_x + static_cast<uint64_t>(k) * A.total + F.off;
                const double *cl = A.ck_l + static_cast<uint64_t>(k) * A.total + F.off;
                run.setup(F, xa, xb, lw, scanS, epos, nullptr, nullptr, nullptr, threshold);
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                    run.xc[p] = cx[p];
                    run.st.l[p] = cl[p];
                }
                run.restore(A.ck_s[static_cast<uint64_t>(k) * A.F + f]);
                __syncthreads();
            }
            for (int t = t0 + 1; t <= t1; ++t) {
                const uint64_t q = static_cast<uint64_t>(t - t0 - 1);
                double *qx = rx + q * A.nmax, *ql = rl + q * A.nmax;
                run.rec_x = qx;  // the step records its particles before resampling
                const bool res = run.step(t, yf[t], shd, shd, shu, shj);
                run.rec_x = nullptr;
                // record the log-weights and the parent placement (occupied
                // flags, surplus prefix, empties)
                uint32_t *qo = rrep + q * A.nmax, *qs = rsS + q * A.nmax, *qe = rep_list + q * A.nmax;
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                    ql[p] = run.st.l[p];
                    if (res) {
                        qo[p] = 1;
                        qs[p] = run.sS[p];
                    }
                }
                if (threadIdx.x == 0) {
                    rflag[q] = res ? 1 : 0;
                    rne[q] = res ? static_cast<uint32_t>(run.n_empty) : 0u;
                }
                __syncthreads();
                if (res) {
                    for (uint64_t k2 = threadIdx.x; k2 < run.n_empty; k2 += THREADS) {
                        const uint32_t e = run.ep[k2];
                        qe[k2] = e;
                        qo[e] = 0;
                    }
                }
                __syncthreads();
            }
            // sweep t1 .. t0+1
            for (int t = t1; t >= t0 + 1; --t) {
                const uint64_t q = static_cast<uint64_t>(t - t0 - 1);
                const double *xt = rx + q * A.nmax, *lt = rl + q * A.nmax;
                const bool res = rflag[q] != 0;
                // mu_t: children sums of lambda_{t+1} (zero past the last step)
                if (t < T) {
                    // children of parent p: slot p itself when occupied, and
                    // the empty slots el[ss[p], ss[p + 1]) it fills
                    const uint32_t *occ = rrep + q * A.nmax, *ss = rsS + q * A.nmax, *el = rep_list + q * A.nmax;
                    const uint32_t ne = rne[q];
                    for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                        double m_ = lam[p];
                        if (res) {
                            m_ = occ[p] ? lam[p] : 0.0;
                            const uint32_t end = p + 1 < N ? ss[p + 1] : ne;
                            for (uint32_t c = ss[p]; c < end; ++c) m_ += lam[el[c]];
                        }
                        mu[p] = m_;
                        g_phi += xt[p] * m_;
                    }
                } else {
                    for (uint64_t p = threadIdx.x; p < N; p += THREADS) mu[p] = 0.0;
                }
                // weights at the end of the segment containing t
                if (t == T || res) {
                    double mx = -INFINITY;
                    for (uint64_t p = threadIdx.x; p < N; p += THREADS) mx = fmax(mx, lt[p]);
                    mx = block_max(mx, shd);
                    double ssum = 0.0;
                    for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                        const double e = exp(lt[p] - mx);
                        wend[p] = e;
                        ssum += e;
                    }
                    ssum = block_sum(ssum, shd);
                    const double inv = 1.0 / ssum;
                    for (uint64_t p = threadIdx.x; p < N; p += THREADS) wend[p] *= inv;
                }
                __syncthreads();
                const double yt = yf[t];
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                    const double r = yt - xt[p];
                    lam[p] = phi * mu[p] + wend[p] * r * sy2inv;
                    g_sy += wend[p] * (r * r * sy2inv / sy - 1.0 / sy);
                }
                __syncthreads();
                g_sx += lam_eps(t);
                __syncthreads();
            }
        }
        // ---- t = 0: x_0 = sd0 eps_0, no weight; mu_0 = lambda_1 (no resampling at t = 0)
        {
            const double *cx = A.ck_x + F.off;  // checkpoint 0: the particles of step 0
            for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                g_phi += cx[p] * lam[p];
                lam[p] = phi * lam[p];
            }
            __syncthreads();
            const double le = lam_eps(0);
            const double q = 1.0 - phi * phi;
            g_sx += le / sqrt(q);
            g_phi += le * sx * phi / (q * sqrt(q));
        }
        g_phi = block_sum(g_phi, shd);
        g_sx = block_sum(g_sx, shd);
        g_sy = block_sum(g_sy, shd);
        if (threadIdx.x == 0) {
            A.grad[3 * f] = g_phi;
            A.grad[3 * f + 1] = g_sx;
            A.grad[3 * f + 2] = g_sy;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Score by the Fisher identity: grad log p(y_1:T) = E[grad log p(x_0:T, y_1:T)
// | y_1:T], the expectation of an additive functional of the path, estimated
// forward with PaRIS (Olsson and Westerborn 2017, "Efficient particle-based
// online smoothing in general hidden Markov models: the PaRIS algorithm").
// Each particle i of the cloud at t carries tau_t^i, an estimate of
// E[sum_{s<=t} s_s | x_t = xi_t^i, y_1:t]:
//   tau_0^i = s_0(xi_0^i),
//   tau_t^i = (1/K) sum_k [tau_{t-1}^{J_k} + s_t(x_{t-1}^{J_k}, xi_t^i)],
// the J_k drawn from the backward kernel, probability proportional to
// W_{t-1}^j f(xi_t^i | x_{t-1}^j) over the weighted cloud at t - 1 (before its
// resampling).  The J_k are the states after steps 4 and 8 (K = 2) of an
// independent Metropolis-Hastings chain started at the particle's own
// ancestor (Dau and Chopin 2022, "On backward smoothing algorithms"): the
// start is not a draw from the backward kernel (its distribution follows the
// resampling counts), and two steps left a bias of ~12 % of the score at the
// differentiated configuration where eight leave it within the Monte Carlo
// error of a few runs.  Its proposal is an even mixture of the
// ancestor of a uniformly drawn slot and a uniformly drawn particle,
// q(j) = (rep_j + 1) / 2N with rep_j the copies of j after the resampling
// (1 without one): drawn in O(1), and positive wherever the target is (the
// ancestors alone would never propose a particle the resampling dropped, and
// the chain would sample the backward kernel restricted to the survivors).
// The acceptance ratio is
//   W_j' f(xi | x_j') (rep_J + 1) / (W_J f(xi | x_J) (rep_j' + 1)),
// evaluated from lw_j = log W_j - log(rep_j + 1) kept per particle.
// The estimate is sum_i W_T^i tau_T^i.  Additive terms, theta = (phi, sx, sy):
//   transition  d = x_t - phi x_{t-1}:  (d x_{t-1} / sx^2, -1/sx + d^2 / sx^3, 0)
//   observation r = y_t - x_t:           (0, 0, -1/sy + r^2 / sy^3)
//   initial     x_0 ~ N(0, sd0^2), sd0 = sx / sqrt(1 - phi^2):
//               v = x_0^2 / sd0^2 - 1:   (v phi / (1 - phi^2), v / sx, 0)
// The backward draws use Philox4x32 with the filter's resampling key, its
// second word xor 0x9E3779B9, counter (i, t + 2^32 b), b = 0..3: four blocks
// per particle and step (proposal index in [0, 2N) and acceptance uniform of
// each of the eight moves).
// ---------------------------------------------------------------------------
// One 32-byte record per particle: the three components of tau, so that a
// backward draw's tau is one sector
struct __align__(32) ScoreTau {
    double a0, a1, a2, pad;
};

struct ScoreArgs {
    uint64_t nmax;
    double *xb;            // nmax per CTA: the cloud at t before its resampling
    double2 *xw;           // 2 x nmax per CTA: (x_j, lw_j) of the clouds at t - 1 and t, lw_j = log W_j -
                           // log(rep_j + 1), so that a backward draw reads one 16-byte pair
    uint32_t *rep, *anc;   // nmax per CTA: copies of each particle at t - 1, parent of each slot
    ScoreTau *tau;         // 2 x nmax per CTA
    double *score;         // 3 per filter
};

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_pf_score(const BatchedFilter *filt, const int *order, int nf,
    const double *y, int T, double threshold, double *xa, double *xb, double *lw, uint32_t *scanS, uint32_t *epos,
    double *loglik, uint32_t *nresampled, int *queue, ScoreArgs A)
{
    __shared__ double shd[33];
    __shared__ unsigned long long shu[33];
    __shared__ __align__(16) uint32_t shj[shj_words<THREADS>()];
    __shared__ int sh_f;
    const uint64_t slot = blockIdx.x, nm = A.nmax;
    double *xnow = A.xb + slot * nm;
    double2 *xwb[2] = {A.xw + slot * 2 * nm, A.xw + slot * 2 * nm + nm};
    uint32_t *rep = A.rep + slot * nm, *anc = A.anc + slot * nm;
    ScoreTau *taub[2] = {A.tau + slot * 2 * nm, A.tau + slot * 2 * nm + nm};
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
        const uint32_t N32 = static_cast<uint32_t>(N);
        const double *yf = y + static_cast<uint64_t>(f) * (T + 1);
        const double phi = F.phi, sx = F.sx, sy = F.sy;
        const double isx2 = 1.0 / (sx * sx), hsx2 = 0.5 * isx2;
        const double q0 = 1.0 - phi * phi, isd02 = q0 * isx2;
        const PhiloxGen gb{F.rkey[0], F.rkey[1] ^ 0x9E3779B9u};
        FilterRun<double, THREADS, false> run;
        run.setup(F, xa, xb, lw, scanS, epos, nullptr, nullptr, nullptr, threshold);
        // t = 0: the initial cloud, equal weights, no resampling
        run.step(0, yf[0], shd, shd, shu, shj);
        for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
            const double x0 = run.xc[p];
            const double v = x0 * x0 * isd02 - 1.0;
            xwb[0][p] = make_double2(x0, 0.0);
            taub[0][p] = ScoreTau{v * phi / q0, v / sx, 0.0, 0.0};
        }
        __syncthreads();
        int cur = 0;
        // whether the cloud at t - 1 was resampled: otherwise its slots are
        // their own parents (anc = identity, rep = 1) and the arrays are not read
        bool resampled = false;
        for (int t = 1; t <= T; ++t) {
            const double2 *xwp = xwb[(t - 1) & 1];
            double2 *xwn = xwb[t & 1];
            run.rec_x = xnow;  // the step records its cloud before resampling
            const bool res = run.step(t, yf[t], shd, shd, shu, shj);
            run.rec_x = nullptr;
            // PaRIS update of every particle of the cloud at t
            const ScoreTau *tp = taub[cur];
            ScoreTau *tn = taub[cur ^ 1];
            const double yt = yf[t];
            for (uint64_t i = threadIdx.x; i < N; i += THREADS) {
                const double xi = xnow[i];
                uint32_t J = resampled ? anc[i] : static_cast<uint32_t>(i);
                const double2 pJ = xwp[J];
                double xJ = pJ.x;
                double dJ = xi - phi * xJ;
                double lJ = pJ.y;
                double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll 1
                for (int b = 0; b < 4; ++b) {
                    uint32_t wd[4];
                    gb.block(Ctr{{i, static_cast<uint64_t>(t) | (static_cast<uint64_t>(b) << 32), 0, 0}}, wd);
#pragma unroll
                    for (int m = 0; m < 2; ++m) {
                        // k in [0, 2N): the ancestor of slot k, or particle k - N
                        const uint32_t k =
                            static_cast<uint32_t>((static_cast<uint64_t>(wd[2 * m]) * (2ull * N32)) >> 32);
                        const uint32_t jp = k < N32 ? (resampled ? anc[k] : k) : k - N32;
                        const double2 pp = xwp[jp];
                        const double dp = xi - phi * pp.x;
                        const double lp = pp.y;
                        // log of the acceptance ratio
                        const double lr = (dJ * dJ - dp * dp) * hsx2 + lp - lJ;
                        const double u = (static_cast<double>(wd[2 * m + 1]) + 0.5) * 0x1p-32;
                        if (log(u) < lr) {
                            J = jp;
                            xJ = pp.x;
                            dJ = dp;
                            lJ = lp;
                        }
                    }
                    if (b == 1 || b == 3) {  // the states after moves 4 and 8
                        const ScoreTau tJ = tp[J];
                        a0 += tJ.a0 + dJ * xJ * isx2;
                        a1 += tJ.a1 + (dJ * dJ * isx2 - 1.0) / sx;
                        a2 += tJ.a2;
                    }
                }
                const double r = yt - xi;
                tn[i] = ScoreTau{0.5 * a0, 0.5 * a1, 0.5 * a2 + (r * r / (sy * sy) - 1.0) / sy, 0.0};
            }
            cur ^= 1;
            __syncthreads();
            // the cloud at t for the next step: when it was resampled, the
            // parents of the slots and the copies of each particle; then
            // lw = log-weight - log(copies + 1) (the step leaves its
            // log-weights as they were before the resampling; the ratios need
            // no normalisation, and without a resampling the copies are 1)
            resampled = res;
            if (res) {
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) anc[p] = static_cast<uint32_t>(p);
                __syncthreads();
                // slot-preserving placement: parent p keeps slot p when it
                // has copies and fills the empties ep[sS_p .. sS_{p+1})
                const uint32_t ne = static_cast<uint32_t>(run.n_empty);
                for (uint32_t k = threadIdx.x; k < ne; k += THREADS) anc[run.ep[k]] = 0xFFFFFFFFu;
                __syncthreads();
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                    const uint32_t b = run.sS[p], e = p + 1 < N ? run.sS[p + 1] : ne;
                    for (uint32_t c = b; c < e; ++c) anc[run.ep[c]] = static_cast<uint32_t>(p);
                }
                __syncthreads();
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
                    const uint32_t b = run.sS[p], e = p + 1 < N ? run.sS[p + 1] : ne;
                    const uint32_t c = (anc[p] == p ? 1u : 0u) + (e - b);
                    rep[p] = c;
                    xwn[p] = make_double2(xnow[p], run.st.l[p] - log(static_cast<double>(c) + 1.0));
                }
            } else {
                for (uint64_t p = threadIdx.x; p < N; p += THREADS) xwn[p] = make_double2(xnow[p], run.st.l[p]);
            }
            __syncthreads();
        }
        // the estimate: sum_i W_T^i tau_T^i / sum_i W_T^i, W_T the weights
        // of the last cloud (its log-weights relative to their maximum)
        double g0 = 0.0, g1 = 0.0, g2 = 0.0, gw = 0.0;
        const ScoreTau *tT = taub[cur];
        const double mT = run.st.lshift;
        for (uint64_t p = threadIdx.x; p < N; p += THREADS) {
            const double wp = exp(run.st.l[p] - mT);
            const ScoreTau tp = tT[p];
            g0 += wp * tp.a0;
            g1 += wp * tp.a1;
            g2 += wp * tp.a2;
            gw += wp;
        }
        g0 = block_sum(g0, shd);
        g1 = block_sum(g1, shd);
        g2 = block_sum(g2, shd);
        gw = block_sum(gw, shd);
        g0 /= gw;
        g1 /= gw;
        g2 /= gw;
        if (threadIdx.x == 0) {
            loglik[f] = run.ll_sum;
            nresampled[f] = static_cast<uint32_t>(run.events);
            A.score[3 * f] = g0;
            A.score[3 * f + 1] = g1;
            A.score[3 * f + 2] = g2;
        }
        __syncthreads();
    }
}

// Two register budgets per block shape: MINB = 1 (the compiler's choice, 16
// warps per SM at most) and MINB = 1024 / THREADS (64 registers, 32 warps).
template <typename R, int THREADS, bool SHADOW, int MINB>
int launch_one(const BatchedArgs &a, const int *order, int nf, int *queue, int ctas, cudaStream_t s)
{
    k_pf_batched<R, THREADS, SHADOW, MINB><<<ctas, THREADS, 0, s>>>(a.filt, order, nf, a.y, a.T, a.threshold,
        static_cast<R *>(a.xa), static_cast<R *>(a.xb), static_cast<R *>(a.lw), a.scanS, a.epos,
        a.loglik, a.nresampled, queue, a.xsa, a.xsb, a.lws, a.loglik_shadow);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

template <typename R, int THREADS, bool SHADOW, int MINB>
int occupancy_one(int *blocks)
{
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, k_pf_batched<R, THREADS, SHADOW, MINB>, THREADS,
        0));
    return MCKL_B200_OK;
}

// op 0: launch, op 1: occupancy of the variant
template <typename R, int THREADS, bool SHADOW>
int variant(int op, bool capped, const BatchedArgs &a, const int *order, int nf, int *queue, int ctas,
    cudaStream_t s, int *blocks)
{
    constexpr int CAP = 1024 / THREADS;
    if (op == 1) return capped ? occupancy_one<R, THREADS, SHADOW, CAP>(blocks) : occupancy_one<R, THREADS, SHADOW, 1>(blocks);
    return capped ? launch_one<R, THREADS, SHADOW, CAP>(a, order, nf, queue, ctas, s)
                  : launch_one<R, THREADS, SHADOW, 1>(a, order, nf, queue, ctas, s);
}

template <typename R, bool SHADOW>
int dispatch_threads(int op, int threads, bool capped, const BatchedArgs &a, const int *order, int nf, int *queue,
    int ctas, cudaStream_t s, int *blocks)
{
    switch (threads) {
        case 128: return variant<R, 128, SHADOW>(op, capped, a, order, nf, queue, ctas, s, blocks);
        case 256: return variant<R, 256, SHADOW>(op, capped, a, order, nf, queue, ctas, s, blocks);
        case 512: return variant<R, 512, SHADOW>(op, capped, a, order, nf, queue, ctas, s, blocks);
        default: return variant<R, 1024, SHADOW>(op, capped, a, order, nf, queue, ctas, s, blocks);
    }
}

int dispatch(int op, int threads, bool capped, const BatchedArgs &a, const int *order, int nf, int *queue, int ctas,
    cudaStream_t s, int *blocks)
{
    if (a.fp64 && a.xsa) return dispatch_threads<double, true>(op, threads, capped, a, order, nf, queue, ctas, s, blocks);
    if (a.fp64) return dispatch_threads<double, false>(op, threads, capped, a, order, nf, queue, ctas, s, blocks);
    if (a.xsa) return dispatch_threads<float, true>(op, threads, capped, a, order, nf, queue, ctas, s, blocks);
    return dispatch_threads<float, false>(op, threads, capped, a, order, nf, queue, ctas, s, blocks);
}

}  // namespace

// Resident CTAs per SM of the kernel variant that the arguments and block
// shape select, and whether that variant is the register-capped one: the
// uncapped variant when it fits `ctas_per_sm`, else the capped one.
int pf_batched_fit(const BatchedArgs &a, int threads, int ctas_per_sm, bool *capped, int *fit)
{
    int f0 = 0, f1 = 0;
    int rc = dispatch(1, threads, false, a, nullptr, 0, nullptr, 0, nullptr, &f0);
    if (rc != MCKL_B200_OK) return rc;
    rc = dispatch(1, threads, true, a, nullptr, 0, nullptr, 0, nullptr, &f1);
    if (rc != MCKL_B200_OK) return rc;
    *capped = f0 < ctas_per_sm;
    *fit = *capped ? f1 : f0;
    return MCKL_B200_OK;
}

template <int THREADS>
int adjoint_one(const BatchedArgs &a, const int *order, int nf, int *queue, const AdjointArgs &A, int ctas,
    cudaStream_t s)
{
    k_pf_adjoint<THREADS><<<ctas, THREADS, 0, s>>>(a.filt, order, nf, a.y, a.T, a.threshold,
        static_cast<double *>(a.xa), static_cast<double *>(a.xb), static_cast<double *>(a.lw), a.scanS, a.epos,
        a.loglik, a.nresampled, queue, A);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

int pf_adjoint_launch(const BatchedArgs &a, const int *order, int nf, int threads, int *queue, const AdjointArgs &A,
    int ctas, cudaStream_t s)
{
    MB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), s));
    switch (threads) {
        case 128: return adjoint_one<128>(a, order, nf, queue, A, ctas, s);
        case 256: return adjoint_one<256>(a, order, nf, queue, A, ctas, s);
        case 512: return adjoint_one<512>(a, order, nf, queue, A, ctas, s);
        default: return adjoint_one<1024>(a, order, nf, queue, A, ctas, s);
    }
}

template <int THREADS>
int score_one(const BatchedArgs &a, const int *order, int nf, int *queue, const ScoreArgs &A, int ctas,
    cudaStream_t s)
{
    k_pf_score<THREADS><<<ctas, THREADS, 0, s>>>(a.filt, order, nf, a.y, a.T, a.threshold,
        static_cast<double *>(a.xa), static_cast<double *>(a.xb), static_cast<double *>(a.lw), a.scanS, a.epos,
        a.loglik, a.nresampled, queue, A);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

int pf_score_launch(const BatchedArgs &a, const int *order, int nf, int threads, int *queue, const ScoreArgs &A,
    int ctas, cudaStream_t s)
{
    MB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), s));
    switch (threads) {
        case 128: return score_one<128>(a, order, nf, queue, A, ctas, s);
        case 256: return score_one<256>(a, order, nf, queue, A, ctas, s);
        case 512: return score_one<512>(a, order, nf, queue, A, ctas, s);
        default: return score_one<1024>(a, order, nf, queue, A, ctas, s);
    }
}

int pf_batched_launch(const BatchedArgs &a, const int *order, int nf, int threads, int ctas_per_sm, int *queue,
    cudaStream_t s)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    bool capped = false;
    int fit = 0;
    int rc = pf_batched_fit(a, threads, ctas_per_sm, &capped, &fit);
    if (rc != MCKL_B200_OK) return rc;
    const int ctas = std::max(1, std::min(nf, sms * ctas_per_sm));
    MB_CUDA(cudaMemsetAsync(queue, 0, sizeof(int), s));
    return dispatch(0, threads, capped, a, order, nf, queue, ctas, s, nullptr);
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
    std::vector<mckl_b200::BatchedFilter> hf;  // host copy of the filter table
    uint64_t nmax = 0;                         // largest particle count
    void *adj_mem = nullptr;                   // adjoint checkpoints and work areas
    size_t adj_bytes = 0;
    void *score_mem = nullptr;                 // score estimator work areas
    size_t score_bytes = 0;
};

using namespace mckl_b200;

namespace {

// Autotuner picks of this process, by workload: FNV-1a over the device, the
// precision mode, F, T, the threshold and every particle count.
std::mutex g_tune_mu;
std::map<uint64_t, std::pair<int, int>> g_tune;

uint64_t tune_key(const mckl_b200_batched *b)
{
    uint64_t h = 1469598103934665603ull;
    auto mix = [&h](uint64_t v) {
        for (int k = 0; k < 8; ++k) {
            h ^= (v >> (8 * k)) & 0xFF;
            h *= 1099511628211ull;
        }
    };
    int dev = 0;
    cudaGetDevice(&dev);
    uint64_t thr;
    std::memcpy(&thr, &b->threshold, sizeof(thr));
    mix(static_cast<uint64_t>(dev));
    mix(static_cast<uint64_t>(b->fp64) | (b->a.xsa ? 2u : 0u));
    mix(static_cast<uint64_t>(b->F));
    mix(static_cast<uint64_t>(b->T));
    mix(thr);
    for (const auto &f : b->hf) mix(f.n);
    return h;
}

// main-run parameters of one filter and their derived constants
void set_main(BatchedFilter &h, double phi, double sx, double sy)
{
    h.phi = phi;
    h.sx = sx;
    h.sd0 = sx / std::sqrt(1 - phi * phi);
    h.lconst = -std::log(sy) - 0.5 * std::log(2 * 3.14159265358979323846);
    h.hinv = 0.5 / (sy * sy);
    h.sy = sy;
}

// shadow-run parameters of one filter (the same derived constants as the main run's)
void set_shadow(BatchedFilter &h, double phi, double sx, double sy)
{
    h.phi_s = phi;
    h.sx_s = sx;
    h.sd0_s = sx / std::sqrt(1 - phi * phi);
    h.lconst_s = -std::log(sy) - 0.5 * std::log(2 * 3.14159265358979323846);
    h.hinv_s = 0.5 / (sy * sy);
}

}  // namespace

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
        set_main(h[f], phi[f], sx[f], sy[f]);
        set_shadow(h[f], phi[f], sx[f], sy[f]);
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
    MB_CHECK_ARG(fp64 >= 0 && fp64 <= 3, "fp64: 0 FP32, 1 FP64, 2 FP32 + FP64 shadow, 3 FP64 + FP64 shadow");
    const bool shadow = (fp64 >= 2);
    b->fp64 = (fp64 == 1 || fp64 == 3) ? 1 : 0;
    const size_t rs = b->fp64 ? 8 : 4;
    const size_t bytes = align256(F * sizeof(BatchedFilter)) + align256(F * (T + 1) * 8) + 2 * align256(total * rs) +
                         2 * align256(total * 4) + align256(F * 8) + align256(F * 4) + align256(F * 4) + 256 +
                         (shadow ? 2 * align256(total * 8) + align256(F * 8) : 0);
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
    b->a.xb = nullptr;  // the resampling gathers in place
    b->a.lw = take(total * rs);
    b->a.scanS = reinterpret_cast<uint32_t *>(take(total * 4));
    b->a.epos = reinterpret_cast<uint32_t *>(take(total * 4));
    b->a.loglik = reinterpret_cast<double *>(take(F * 8));
    b->a.nresampled = reinterpret_cast<uint32_t *>(take(F * 4));
    b->order = reinterpret_cast<int *>(take(F * 4));
    b->queue = reinterpret_cast<int *>(take(256));
    if (shadow) {
        b->a.xsa = reinterpret_cast<double *>(take(total * 8));
        b->a.xsb = nullptr;
        b->a.lws = reinterpret_cast<double *>(take(total * 8));
        b->a.loglik_shadow = reinterpret_cast<double *>(take(F * 8));
    }
    b->a.T = static_cast<int>(T);
    b->a.threshold = threshold;
    b->a.fp64 = b->fp64;
    MB_CUDA(cudaMemcpy(b->a.filt, h.data(), F * sizeof(BatchedFilter), cudaMemcpyHostToDevice));
    MB_CUDA(cudaMemcpy(b->a.y, y, F * (T + 1) * 8, cudaMemcpyHostToDevice));
    MB_CUDA(cudaMemcpy(b->order, order.data(), F * 4, cudaMemcpyHostToDevice));
    b->hf = h;
    for (size_t f = 0; f < F; ++f) b->nmax = std::max<uint64_t>(b->nmax, N[f]);
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

int mckl_b200_batched_get_config(const mckl_b200_batched_t *b, int *threads, int *ctas_per_sm)
{
    MB_CHECK_ARG(b != nullptr, "null handle");
    if (threads) *threads = b->threads;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
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
    // a workload tuned before in this process (same device, precision mode,
    // filter count, steps, threshold and particle counts) reuses its pick
    const uint64_t key = tune_key(b);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            if (ntrials) *ntrials = 0;
            return mckl_b200_batched_config(b, it->second.first, it->second.second);
        }
    }
    // candidate block shapes: 16 or 32 resident warps per SM (the latter with
    // the register-capped variant), from many small CTAs (small filters keep
    // every thread busy) to few large ones (fewer barriers per particle)
    static const int cand[][2] = {{128, 4}, {128, 8}, {256, 2}, {256, 4}, {512, 1}, {512, 2}, {1024, 1}};
    int best = -1, n = 0;
    float best_ms = 0.0f;
    cudaEvent_t e0, e1;
    MB_CUDA(cudaEventCreate(&e0));
    MB_CUDA(cudaEventCreate(&e1));
    // one untimed run first (module load, caches)
    int rc = pf_batched_launch(b->a, b->order, b->F, 256, 4, b->queue, s);
    for (int k = 0; rc == MCKL_B200_OK && k < static_cast<int>(sizeof(cand) / sizeof(cand[0])); ++k) {
        int fit = 0;
        bool capped = false;
        rc = pf_batched_fit(b->a, cand[k][0], cand[k][1], &capped, &fit);
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
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = {cand[best][0], cand[best][1]};
    }
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

int mckl_b200_batched_shadow_params(mckl_b200_batched_t *b, const double *phi, const double *sx, const double *sy)
{
    MB_CHECK_ARG(b != nullptr && phi && sx && sy, "null argument");
    MB_CHECK_ARG(b->a.xsa != nullptr, "the handle has no shadow run (fp64 = 2 or 3)");
    for (int f = 0; f < b->F; ++f) {
        MB_CHECK_ARG(sy[f] > 0 && phi[f] * phi[f] < 1, "need sy > 0 and |phi| < 1");
        set_shadow(b->hf[f], phi[f], sx[f], sy[f]);
    }
    MB_CUDA(cudaMemcpy(b->a.filt, b->hf.data(), b->hf.size() * sizeof(BatchedFilter), cudaMemcpyHostToDevice));
    return MCKL_B200_OK;
}

int mckl_b200_batched_set_params(mckl_b200_batched_t *b, const double *phi, const double *sx, const double *sy,
    void *stream)
{
    MB_CHECK_ARG(b != nullptr && phi && sx && sy, "null argument");
    for (int f = 0; f < b->F; ++f) {
        MB_CHECK_ARG(sy[f] > 0 && phi[f] * phi[f] < 1, "need sy > 0 and |phi| < 1");
    }
    for (int f = 0; f < b->F; ++f) {
        set_main(b->hf[f], phi[f], sx[f], sy[f]);
        set_shadow(b->hf[f], phi[f], sx[f], sy[f]);
    }
    MB_CUDA(cudaMemcpyAsync(b->a.filt, b->hf.data(), b->hf.size() * sizeof(BatchedFilter), cudaMemcpyHostToDevice,
        as_stream(stream)));
    return MCKL_B200_OK;
}

int mckl_b200_batched_set_keys(mckl_b200_batched_t *b, const uint32_t *mkeys, const uint32_t *rkeys, void *stream)
{
    MB_CHECK_ARG(b != nullptr && mkeys && rkeys, "null argument");
    for (int f = 0; f < b->F; ++f) {
        b->hf[f].mkey[0] = mkeys[2 * f];
        b->hf[f].mkey[1] = mkeys[2 * f + 1];
        b->hf[f].rkey[0] = rkeys[2 * f];
        b->hf[f].rkey[1] = rkeys[2 * f + 1];
    }
    MB_CUDA(cudaMemcpyAsync(b->a.filt, b->hf.data(), b->hf.size() * sizeof(BatchedFilter), cudaMemcpyHostToDevice,
        as_stream(stream)));
    return MCKL_B200_OK;
}

int mckl_b200_batched_adjoint(mckl_b200_batched_t *b, int checkpoint_every, double *loglik, double *grad,
    void *stream)
{
    MB_CHECK_ARG(b != nullptr && grad != nullptr, "null argument");
    MB_CHECK_ARG(b->fp64 == 1 && b->a.xsa == nullptr, "the adjoint needs a handle created with fp64 = 1");
    MB_CHECK_ARG(checkpoint_every >= 1 && checkpoint_every <= 4096, "checkpoint_every in [1, 4096]");
    cudaStream_t s = as_stream(stream);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ctas = std::max(1, std::min(b->F, sms));
    const uint64_t C = static_cast<uint64_t>(checkpoint_every);
    const uint64_t nck = static_cast<uint64_t>(b->T) / C + 1;
    const uint64_t nm = b->nmax;
    // checkpoints + per-CTA replay records + per-CTA adjoint vectors + gradients
    const size_t need = 2 * align256(nck * b->total * 8) + align256(nck * b->F * sizeof(FilterScalars)) +
                        2 * align256(ctas * C * nm * 8) + 3 * align256(ctas * C * nm * 4) + align256(ctas * C) + align256(ctas * C * 4) +
                        3 * align256(ctas * nm * 8) + align256(static_cast<size_t>(b->F) * 24);
    if (b->adj_bytes < need) {
        if (b->adj_mem) cudaFree(b->adj_mem);
        b->adj_mem = nullptr;
        b->adj_bytes = 0;
        if (cudaMalloc(&b->adj_mem, need) != cudaSuccess) {
            set_error("adjoint work memory (" + std::to_string(need >> 20) + " MiB) could not be allocated; "
                      "use a larger checkpoint interval or fewer filters per handle");
            return MCKL_B200_ERR_NOMEM;
        }
        b->adj_bytes = need;
    }
    char *p = static_cast<char *>(b->adj_mem);
    auto take = [&p](size_t n) {
        char *q = p;
        p += align256(n);
        return q;
    };
    AdjointArgs A{};
    A.C = checkpoint_every;
    A.total = b->total;
    A.F = b->F;
    A.nmax = nm;
    A.ck_x = reinterpret_cast<double *>(take(nck * b->total * 8));
    A.ck_l = reinterpret_cast<double *>(take(nck * b->total * 8));
    A.ck_s = reinterpret_cast<FilterScalars *>(take(nck * b->F * sizeof(FilterScalars)));
    A.rec_x = reinterpret_cast<double *>(take(ctas * C * nm * 8));
    A.rec_l = reinterpret_cast<double *>(take(ctas * C * nm * 8));
    A.rec_rep = reinterpret_cast<uint32_t *>(take(ctas * C * nm * 4));
    A.rec_sS = reinterpret_cast<uint32_t *>(take(ctas * C * nm * 4));
    A.rec_ep = reinterpret_cast<uint32_t *>(take(ctas * C * nm * 4));
    A.rec_flag = reinterpret_cast<uint8_t *>(take(ctas * C));
    A.rec_ne = reinterpret_cast<uint32_t *>(take(ctas * C * 4));
    A.lam = reinterpret_cast<double *>(take(ctas * nm * 8));
    A.mu = reinterpret_cast<double *>(take(ctas * nm * 8));
    A.wend = reinterpret_cast<double *>(take(ctas * nm * 8));
    A.grad = reinterpret_cast<double *>(take(static_cast<size_t>(b->F) * 24));
    int rc = pf_adjoint_launch(b->a, b->order, b->F, b->threads, b->queue, A, ctas, s);
    if (rc != MCKL_B200_OK) return rc;
    if (loglik) MB_CUDA(cudaMemcpyAsync(loglik, b->a.loglik, b->F * 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaMemcpyAsync(grad, A.grad, static_cast<size_t>(b->F) * 24, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return MCKL_B200_OK;
}

int mckl_b200_batched_score(mckl_b200_batched_t *b, double *loglik, double *score, void *stream)
{
    MB_CHECK_ARG(b != nullptr && score != nullptr, "null argument");
    MB_CHECK_ARG(b->fp64 == 1 && b->a.xsa == nullptr, "the score needs a handle created with fp64 = 1");
    cudaStream_t s = as_stream(stream);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ctas = std::max(1, std::min(b->F, sms));
    const uint64_t nm = b->nmax;
    const size_t need = align256(ctas * nm * 8) + align256(ctas * 2 * nm * sizeof(double2)) +
                        2 * align256(ctas * nm * 4) + align256(ctas * 2 * nm * sizeof(ScoreTau)) +
                        align256(static_cast<size_t>(b->F) * 24);
    if (b->score_bytes < need) {
        if (b->score_mem) cudaFree(b->score_mem);
        b->score_mem = nullptr;
        b->score_bytes = 0;
        if (cudaMalloc(&b->score_mem, need) != cudaSuccess) {
            set_error("score work memory (" + std::to_string(need >> 20) + " MiB) could not be allocated");
            return MCKL_B200_ERR_NOMEM;
        }
        b->score_bytes = need;
    }
    char *p = static_cast<char *>(b->score_mem);
    auto take = [&p](size_t n) {
        char *q = p;
        p += align256(n);
        return q;
    };
    ScoreArgs A{};
    A.nmax = nm;
    A.xb = reinterpret_cast<double *>(take(ctas * nm * 8));
    A.xw = reinterpret_cast<double2 *>(take(ctas * 2 * nm * sizeof(double2)));
    A.rep = reinterpret_cast<uint32_t *>(take(ctas * nm * 4));
    A.anc = reinterpret_cast<uint32_t *>(take(ctas * nm * 4));
    A.tau = reinterpret_cast<ScoreTau *>(take(ctas * 2 * nm * sizeof(ScoreTau)));
    A.score = reinterpret_cast<double *>(take(static_cast<size_t>(b->F) * 24));
    int rc = pf_score_launch(b->a, b->order, b->F, b->threads, b->queue, A, ctas, s);
    if (rc != MCKL_B200_OK) return rc;
    if (loglik) MB_CUDA(cudaMemcpyAsync(loglik, b->a.loglik, b->F * 8, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaMemcpyAsync(score, A.score, static_cast<size_t>(b->F) * 24, cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return MCKL_B200_OK;
}

int mckl_b200_batched_destroy(mckl_b200_batched_t *b)
{
    if (!b) return MCKL_B200_OK;
    if (b->score_mem) cudaFree(b->score_mem);
    if (b->adj_mem) cudaFree(b->adj_mem);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->mem) cudaFree(b->mem);
    delete b;
    return MCKL_B200_OK;
}

}  // extern "C"
