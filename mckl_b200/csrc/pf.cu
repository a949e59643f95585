// pf.cu -- the plain FP64 bootstrap particle filter for the AR(1) model
//   x_0 ~ N(0, sd0^2),  x_t = phi x_{t-1} + sx eps_t,  y_t = x_t + sy eta_t
// run in the reference's SMCSampler step order (algorithm/smc.hpp:389-406):
// selection (propagate + weight) -> record ESS -> resample iff
// ESS < N * threshold (ResampleEval, algorithm/resample.hpp:494-507) -> next.
// Model noise comes from one sequential engine, as BackendSEQ's eval_range
// does with rng_set[0] (smp/backend_seq.hpp:60-64); resampling uses the
// particle's own engine (core/particle.hpp:364).  Every piece is the
// bit-faithful kernel of its reference function; the loop itself runs on the
// host and waits once per step for the ESS that decides the resampling, as
// the reference's loop does, with the next step's model noise (which does not
// depend on the decision) already queued behind the read-back.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "resample.cuh"
#include "weight.cuh"

namespace mckl_b200 {

namespace {

__global__ void k_fill(uint64_t n, double *a, double v)
{
    pdl_wait();
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        a[i] = v;
    }
}

// x = phi x + sx eps; ll = lconst - (y - x)^2 hinv, each rounding as written
__global__ void k_ar1_propagate(uint64_t n, double *x, const double *eps, double y, double phi, double sx,
    double lconst, double hinv, double *ll)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double a = __dmul_rn(phi, x[i]);
        const double b = __dmul_rn(sx, eps[i]);
        const double xn = __dadd_rn(a, b);
        x[i] = xn;
        const double r = __dsub_rn(y, xn);
        ll[i] = __dsub_rn(lconst, __dmul_rn(__dmul_rn(r, r), hinv));
    }
}

// the same move with y_t read from the device (t = *t_dev), for the captured step
__global__ void k_ar1_propagate_dev(uint64_t n, double *x, const double *eps, const double *y, const int *t_dev,
    double phi, double sx, double lconst, double hinv, double *ll)
{
    pdl_wait();
    const double yt = y[*t_dev];
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double a = __dmul_rn(phi, x[i]);
        const double b = __dmul_rn(sx, eps[i]);
        const double xn = __dadd_rn(a, b);
        x[i] = xn;
        const double r = __dsub_rn(yt, xn);
        ll[i] = __dsub_rn(lconst, __dmul_rn(__dmul_rn(r, r), hinv));
    }
}

__global__ void k_step_inc(int *t_dev)
{
    pdl_wait();
    *t_dev += 1;
}

// Capture the work `fn` enqueues (on a private stream) into an instantiated graph.
template <class Fn>
int capture(cudaGraphExec_t *exec, Fn &&fn)
{
    cudaStream_t cap;
    MB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) {
        cudaStreamDestroy(cap);
        MB_CUDA(ce);
    }
    const int rc = fn(cap);
    cudaGraph_t g = nullptr;
    ce = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rc != MCKL_B200_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    MB_CUDA(ce);
    ce = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    MB_CUDA(ce);
    return MCKL_B200_OK;
}

struct GraphExec {
    cudaGraphExec_t e = nullptr;
    ~GraphExec()
    {
        if (e) cudaGraphExecDestroy(e);
    }
};

// The side stream and events of the weight normaliser's fork (the ESS's dot
// products beside the normaliser's fold), released with the graphs.
// The plain loop's side stream: the next step's noise and the next
// resampling's uniforms are drawn there while the main stream runs the
// current step.  Events: noise[k] -- the noise in buffer k is ready;
// used[k] -- the step that read buffer k is done with it; u_ready / u_used --
// the same for the resampling uniforms.
struct SideWork {
    cudaStream_t s = nullptr;
    cudaEvent_t noise[2] = {nullptr, nullptr}, used[2] = {nullptr, nullptr};
    cudaEvent_t u_ready = nullptr, u_used = nullptr;
    int create()
    {
        MB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        for (cudaEvent_t *e : {&noise[0], &noise[1], &used[0], &used[1], &u_ready, &u_used})
            MB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        return MCKL_B200_OK;
    }
    ~SideWork()
    {
        if (s) cudaStreamSynchronize(s);  // nothing of ours may run past the call
        for (cudaEvent_t e : {noise[0], noise[1], used[0], used[1], u_ready, u_used})
            if (e) cudaEventDestroy(e);
        if (s) cudaStreamDestroy(s);
    }
};

struct OwnedFork {
    WeightFork f{nullptr, nullptr, nullptr};
    int create()
    {
        MB_CUDA(cudaStreamCreateWithFlags(&f.side, cudaStreamNonBlocking));
        MB_CUDA(cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming));
        MB_CUDA(cudaEventCreateWithFlags(&f.join, cudaEventDisableTiming));
        return MCKL_B200_OK;
    }
    ~OwnedFork()
    {
        if (f.join) cudaEventDestroy(f.join);
        if (f.fork) cudaEventDestroy(f.fork);
        if (f.side) cudaStreamDestroy(f.side);
    }
};

unsigned grid_of(uint64_t n)
{
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148 * 16)));
}

// scan ties of the calling thread's last plain-filter run
thread_local uint64_t g_last_ties = 0;

// Page-locked landing place of the per-step (ESS, log normaliser) pair and an
// event marking its copy, one per host thread (allocated once).
struct StepReadback {
    double *h = nullptr;
    cudaEvent_t ev = nullptr;
    ~StepReadback()
    {
        if (ev) cudaEventDestroy(ev);
        if (h) cudaFreeHost(h);
    }
};
thread_local StepReadback g_rb;

}  // namespace

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" int mckl_b200_pf_ar1_plain_f64(size_t N, size_t T, const double *y, double phi, double sx, double sy,
    double sd0, const uint32_t mkey[2], const uint32_t rkey[2], int scheme, double threshold, double *loglik,
    double *ess_hist, uint8_t *resampled, uint64_t *anc_dev, double *x_dev, double *W_dev, void *stream)
{
    MB_CHECK_ARG(N > 0 && N < (1ull << 31), "N must be in [1, 2^31)");
    MB_CHECK_ARG(y != nullptr && mkey != nullptr && rkey != nullptr && loglik != nullptr, "null argument");
    MB_CHECK_ARG(x_dev != nullptr && W_dev != nullptr, "x_dev and W_dev are required");
    MB_CHECK_ARG(scheme >= 0 && scheme <= 5, "scheme must be 0..5");
    MB_CHECK_ARG(sy > 0 && sd0 > 0, "sy and sd0 must be positive");
    cudaStream_t s = as_stream(stream);
    // work buffers: eps, ll, rep, idx, result words
    const size_t wsz = weight_scratch_bytes(N), rsz = resample_scratch_bytes(N, N), isz = rep_index_scratch_bytes(N, N);
    const size_t buf = 5 * align256(N * sizeof(double)) + 512 + align256((T + 1) * sizeof(double));
    char *base = static_cast<char *>(scratch(5, buf + wsz + rsz + isz, s));
    if (!base) {
        set_error("particle filter scratch allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    double *eps = reinterpret_cast<double *>(base);
    double *ll = reinterpret_cast<double *>(base + align256(N * 8));
    uint64_t *rep = reinterpret_cast<uint64_t *>(base + 2 * align256(N * 8));
    uint64_t *idx = reinterpret_cast<uint64_t *>(base + 3 * align256(N * 8));
    double *wres = reinterpret_cast<double *>(base + 4 * align256(N * 8));
    int *err = reinterpret_cast<int *>(base + 4 * align256(N * 8) + 256);
    unsigned long long *ties = reinterpret_cast<unsigned long long *>(base + 4 * align256(N * 8) + 384);
    int *t_dev = reinterpret_cast<int *>(base + 4 * align256(N * 8) + 448);
    double *y_dev = reinterpret_cast<double *>(base + 4 * align256(N * 8) + 512);
    double *eps2 = reinterpret_cast<double *>(base + 4 * align256(N * 8) + 512 + align256((T + 1) * sizeof(double)));
    void *wscr = base + buf;
    void *rscr = base + buf + wsz;
    void *iscr = base + buf + wsz + rsz;

    mckl_b200_engine_t em, er;
    mckl_b200_engine_seed(&em, MCKL_B200_PHILOX4X32, 0);
    mckl_b200_engine_seed(&er, MCKL_B200_PHILOX4X32, 0);
    em.key[0] = mkey[0];
    em.key[1] = mkey[1];
    er.key[0] = rkey[0];
    er.key[1] = rkey[1];

    // constants of the observation density, computed as the reference does on the host
    const double lconst = -std::log(sy) - 0.5 * std::log(2 * 3.14159265358979323846);
    const double hinv = 0.5 / (sy * sy);
    const double equal = 1.0 / static_cast<double>(N);
    MB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    MB_CUDA(cudaMemsetAsync(ties, 0, sizeof(unsigned long long), s));
    k_fill<<<grid_of(N), 256, 0, s>>>(N, W_dev, equal);
    MB_LAUNCH_CHECK();
    if (!g_rb.h) {
        MB_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&g_rb.h), 2 * sizeof(double), cudaHostAllocDefault));
        MB_CUDA(cudaEventCreateWithFlags(&g_rb.ev, cudaEventDisableTiming));
    }
    double ess = static_cast<double>(N), ll_sum = 0.0;
    if (scheme <= 2) {
        // Schemes without residuals: the engine-independent work of a step is
        // two CUDA graphs built once per call -- A: next step, move, weight
        // normalisation, read-back of (ESS, log normaliser); B: the exact
        // cumulative fold, replication counts, rep -> index, select and equal
        // weights -- so a step costs a handful of host calls.  The noise and
        // the resampling uniforms (the engines' positions) are launched as
        // before.
        static const int seq_of[3] = {0, 1, 2};
        ResampleScratch rs = resample_scratch_carve(rscr, N, N);
        MB_CUDA(cudaMemcpyAsync(y_dev, y, (T + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
        MB_CUDA(cudaMemsetAsync(t_dev, 0, sizeof(int), s));
        double *epsb[2] = {eps, eps2};  // step t reads epsb[t & 1]
        SideWork side;
        OwnedFork fork;
        GraphExec ga[2], gb;
        int rc = side.create();
        if (rc != MCKL_B200_OK) return rc;
        rc = fork.create();
        if (rc != MCKL_B200_OK) return rc;
        for (int k = 0; k < 2; ++k) {
            rc = capture(&ga[k].e, [&](cudaStream_t c) {
                k_step_inc<<<1, 1, 0, c>>>(t_dev);
                MB_LAUNCH_CHECK();
                MB_CUDA(launch_pdl(k_ar1_propagate_dev, grid_of(N), 256, 0, c, N, x_dev, epsb[k], y_dev, t_dev, phi, sx, lconst, hinv,
                    ll));
                MB_LAUNCH_CHECK();
                int r = weight_normalize_dev(N, W_dev, ll, 1, wscr, wres, c, 0, &fork.f);
                if (r != MCKL_B200_OK) return r;
                MB_CUDA(cudaMemcpyAsync(g_rb.h, wres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c));
                return MCKL_B200_OK;
            });
            if (rc != MCKL_B200_OK) return rc;
        }
        rc = capture(&gb.e, [&](cudaStream_t c) {
            int r = rep_counts_dev(N, N, W_dev, rs.u, rep, rs, c, ties);
            if (r != MCKL_B200_OK) return r;
            r = rep_to_index_dev(N, N, rep, idx, iscr, err, c);
            if (r != MCKL_B200_OK) return r;
            r = select_dev<double>(N, N, 1, idx, x_dev, x_dev, c);
            if (r != MCKL_B200_OK) return r;
            k_fill<<<grid_of(N), 256, 0, c>>>(N, W_dev, equal);
            MB_LAUNCH_CHECK();
            return MCKL_B200_OK;
        });
        if (rc != MCKL_B200_OK) return rc;
        // The side stream draws, in the engines' own order, the noise of step
        // t + 1 while the main stream runs step t, and the uniforms of the
        // next resampling as soon as the previous one has used its own (they
        // depend only on the resampling engine's position, which moves only
        // at a resampling).  The main stream waits for each before use.
        auto next_uniforms = [&]() -> int {
            MB_CUDA(cudaStreamWaitEvent(side.s, side.u_used, 0));
            const int r = u01_sequence_dev(seq_of[scheme], er, N, rs.u, rs.tmp, rs.fs, side.s);
            if (r != MCKL_B200_OK) return r;
            MB_CUDA(cudaEventRecord(side.u_ready, side.s));
            return MCKL_B200_OK;
        };
        // x_0 on the main stream, then the noise of step 1 and the first
        // uniforms beside it (the model engine's order: x_0, then step 1's draws)
        rc = mckl_b200_normal_f64(&em, N, x_dev, 0.0, sd0, stream);
        if (rc != MCKL_B200_OK) return rc;
        MB_CUDA(cudaEventRecord(side.used[0], s));
        MB_CUDA(cudaStreamWaitEvent(side.s, side.used[0], 0));
        if (T > 0) {
            rc = mckl_b200_normal_f64(&em, N, epsb[1], 0.0, 1.0, side.s);
            if (rc != MCKL_B200_OK) return rc;
            MB_CUDA(cudaEventRecord(side.noise[1], side.s));
        }
        rc = next_uniforms();
        if (rc != MCKL_B200_OK) return rc;
        for (size_t it = 0; it <= T; ++it) {
            if (it > 0) {
                const int k = static_cast<int>(it & 1);
                MB_CUDA(cudaStreamWaitEvent(s, side.noise[k], 0));
                MB_CUDA(cudaGraphLaunch(ga[k].e, s));
                count_launch();
                MB_CUDA(cudaEventRecord(side.used[k], s));
                MB_CUDA(cudaEventRecord(g_rb.ev, s));
                if (it < T) {  // step it + 1's noise, into the buffer step it - 1 read
                    MB_CUDA(cudaStreamWaitEvent(side.s, side.used[k ^ 1], 0));
                    rc = mckl_b200_normal_f64(&em, N, epsb[k ^ 1], 0.0, 1.0, side.s);
                    if (rc != MCKL_B200_OK) return rc;
                    MB_CUDA(cudaEventRecord(side.noise[k ^ 1], side.s));
                }
                MB_CUDA(cudaEventSynchronize(g_rb.ev));
                ess = g_rb.h[0];
                ll_sum += g_rb.h[1];
            }
            if (ess_hist) ess_hist[it] = ess;
            if (resampled) resampled[it] = 0;
            if (ess < static_cast<double>(N) * threshold) {
                MB_CUDA(cudaStreamWaitEvent(s, side.u_ready, 0));
                MB_CUDA(cudaGraphLaunch(gb.e, s));
                count_launch();
                MB_CUDA(cudaEventRecord(side.u_used, s));
                if (it < T) {
                    rc = next_uniforms();
                    if (rc != MCKL_B200_OK) return rc;
                }
                if (anc_dev) {
                    MB_CUDA(cudaMemcpyAsync(anc_dev + it * N, idx, N * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
                }
                ess = static_cast<double>(N);
                if (resampled) resampled[it] = 1;
            }
        }
    } else {
        for (size_t it = 0; it <= T; ++it) {
            if (it == 0) {
                int rc = mckl_b200_normal_f64(&em, N, x_dev, 0.0, sd0, stream);
                if (rc != MCKL_B200_OK) return rc;
                if (T > 0) {
                    rc = mckl_b200_normal_f64(&em, N, eps, 0.0, 1.0, stream);  // the noise of step 1
                    if (rc != MCKL_B200_OK) return rc;
                }
            } else {
                // eps holds this step's noise (drawn during the previous step's
                // round trip): the model stream does not depend on the decisions
                k_ar1_propagate<<<grid_of(N), 256, 0, s>>>(N, x_dev, eps, y[it], phi, sx, lconst, hinv, ll);
                MB_LAUNCH_CHECK();
                int rc = weight_normalize_dev(N, W_dev, ll, 1, wscr, wres, s);
                if (rc != MCKL_B200_OK) return rc;
                MB_CUDA(cudaMemcpyAsync(g_rb.h, wres, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
                MB_CUDA(cudaEventRecord(g_rb.ev, s));
                // the next step's noise keeps the device busy while the host
                // reads the ESS and decides
                if (it < T) {
                    rc = mckl_b200_normal_f64(&em, N, eps, 0.0, 1.0, stream);
                    if (rc != MCKL_B200_OK) return rc;
                }
                MB_CUDA(cudaEventSynchronize(g_rb.ev));
                ess = g_rb.h[0];
                ll_sum += g_rb.h[1];
            }
            if (ess_hist) ess_hist[it] = ess;
            if (resampled) resampled[it] = 0;
            if (ess < static_cast<double>(N) * threshold) {
                int rc = resample_dev(scheme, N, N, er, W_dev, rep, rscr, s, ties);
                if (rc != MCKL_B200_OK) return rc;
                rc = rep_to_index_dev(N, N, rep, idx, iscr, err, s);
                if (rc != MCKL_B200_OK) return rc;
                if (anc_dev) {
                    MB_CUDA(cudaMemcpyAsync(anc_dev + it * N, idx, N * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
                }
                rc = select_dev<double>(N, N, 1, idx, x_dev, x_dev, s);
                if (rc != MCKL_B200_OK) return rc;
                k_fill<<<grid_of(N), 256, 0, s>>>(N, W_dev, equal);
                MB_LAUNCH_CHECK();
                ess = static_cast<double>(N);
                if (resampled) resampled[it] = 1;
            }
        }
    }
    int h = 0;
    unsigned long long nt = 0;
    MB_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaMemcpyAsync(&nt, ties, sizeof(nt), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    if (h) {
        set_error("particle filter: a look-back wait exceeded its limit");
        return MCKL_B200_ERR_DEVICE;
    }
    g_last_ties = nt;
    *loglik = ll_sum;
    return MCKL_B200_OK;
}

extern "C" int mckl_b200_pf_ar1_plain_ties(uint64_t *ties)
{
    MB_CHECK_ARG(ties != nullptr, "null argument");
    *ties = g_last_ties;
    return MCKL_B200_OK;
}
