// weight.cu -- mckl::Weight normalisation on the device (core/weight.hpp:64-227).
//
//   add_log(v):  w_i = log(W_i) + v_i            (:143-148)
//   set_log(v):  w_i = v_i                       (:123-128)
//   normalize:   lmax = max w_i;  w_i = exp(w_i - lmax);
//                accw = left fold of w (std::accumulate over the whole array);
//                essw = left fold over chunks of 1024 of each chunk's own left
//                       fold of w_i * w_i (the cblas_ddot loop);
//                W_i = (1 / accw) * w_i;  ESS = accw * accw / essw.
// log and exp are the double-double versions (crmath.cuh); accw uses the exact
// fold (fold.cuh); the per-chunk dot products are short independent folds,
// one thread each.  The log of the normalising-constant ratio
// log sum_i W_i^old exp(v_i) = lmax + log(accw) is returned alongside.
#include <algorithm>

#include "block_scan.cuh"
#include "common.cuh"
#include "crmath.cuh"
#include "fold.cuh"
#include "weight.cuh"

namespace mckl_b200 {

namespace {

constexpr int kChunk = 1024;  // BufferSize<double> (internal/traits.hpp:171-175)

__global__ void k_weight_prep(uint64_t N, double *W, const double *v, int add_log, long long *lmax_bits)
{
    pdl_wait();
    __shared__ double sh[33];
    double m = -__longlong_as_double(0x7ff0000000000000ll);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double w = add_log ? __dadd_rn(dd::log(W[i]), v[i]) : v[i];
        W[i] = w;
        if (m < w) m = w;  // max_element: NaN never replaces (core/weight.hpp:184-196)
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : -__longlong_as_double(0x7ff0000000000000ll);
        w = warp_max(w);
        if (threadIdx.x == 0) atomicMax(reinterpret_cast<long long *>(lmax_bits), ordered_bits(w));
    }
}

__global__ void k_weight_exp(uint64_t N, double *W, const long long *lmax_bits)
{
    pdl_wait();
    const double lmax = from_ordered_bits(*lmax_bits);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        W[i] = dd::exp(__dsub_rn(W[i], lmax));
    }
}

// one warp per chunk: the lanes form the chunk's products w_i^2 (each
// rounded once, independent of the others) with coalesced loads into shared
// memory, then lane 0 adds them in index order -- that chunk's ddot fold
constexpr int kDotWarps = 4;

__global__ void __launch_bounds__(32 * kDotWarps) k_weight_chunkdot(uint64_t N, const double *W, double *dots)
{
    pdl_wait();
    __shared__ double sq[kDotWarps][kChunk];
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * kDotWarps + warp;
    const uint64_t b = c * kChunk;
    if (b >= N) return;  // warp-uniform; no CTA barrier below
    const unsigned len = static_cast<unsigned>(N - b < kChunk ? N - b : kChunk);
    for (unsigned i = lane; i < len; i += 32) {
        const double w = W[b + i];
        sq[warp][i] = __dmul_rn(w, w);
    }
    __syncwarp();
    if (lane == 0) {
        double s = 0.0;
        for (unsigned i = 0; i < len; ++i) s = __dadd_rn(s, sq[warp][i]);
        dots[c] = s;
    }
}

// the chunk dots are added in order by thread 0 from shared memory, which
// the CTA fills a tile at a time with coalesced loads
constexpr int kFinishThreads = 256, kFinishTile = 2048;

__global__ void __launch_bounds__(kFinishThreads) k_weight_dotsum(uint64_t nchunks, const double *dots, double *essw)
{
    pdl_wait();
    __shared__ double tile[kFinishTile];
    double acc = 0.0;
    for (uint64_t t0 = 0; t0 < nchunks; t0 += kFinishTile) {
        const unsigned len = static_cast<unsigned>(nchunks - t0 < kFinishTile ? nchunks - t0 : kFinishTile);
        for (unsigned i = threadIdx.x; i < len; i += kFinishThreads) tile[i] = dots[t0 + i];
        __syncthreads();
        if (threadIdx.x == 0)
            for (unsigned i = 0; i < len; ++i) acc = __dadd_rn(acc, tile[i]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *essw = acc;
}

__global__ void k_weight_finish(const double *essw, const double *accw, const long long *lmax_bits,
    double *out /* [ess, log_nc, accw, lmax] */)
{
    pdl_wait();
    const double a = *accw;
    const double lmax = from_ordered_bits(*lmax_bits);
    out[0] = __ddiv_rn(__dmul_rn(a, a), *essw);
    out[1] = __dadd_rn(lmax, dd::log(a));
    out[2] = a;
    out[3] = lmax;
}

__global__ void k_weight_reset(long long *lmax_bits, long long v)
{
    pdl_wait();
    *lmax_bits = v;
}

__global__ void k_weight_scale(uint64_t N, double *W, const double *accw)
{
    pdl_wait();
    const double inv = __ddiv_rn(1.0, *accw);
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < N;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        W[i] = __dmul_rn(inv, W[i]);
    }
}

unsigned grid_cap(uint64_t n, int threads)
{
    const uint64_t need = (n + threads - 1) / threads;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(need, 148 * 16)));
}

}  // namespace

size_t weight_scratch_bytes(uint64_t N, uint64_t wcap)
{
    const uint64_t nchunks = (N + kChunk - 1) / kChunk;
    return 256 + align256(nchunks * sizeof(double)) + fold_scratch_bytes(N, wcap);
}

int weight_normalize_dev(uint64_t N, double *W, const double *v, int add_log, void *scratch_base,
    double *result_dev, cudaStream_t s, uint64_t wcap, const WeightFork *fork)
{
    char *p = static_cast<char *>(scratch_base);
    long long *lmax_bits = reinterpret_cast<long long *>(p);
    double *essw = reinterpret_cast<double *>(p + 64);
    const uint64_t nchunks = (N + kChunk - 1) / kChunk;
    double *dots = reinterpret_cast<double *>(p + 256);
    FoldScratch fs = fold_scratch_carve(p + 256 + align256(nchunks * sizeof(double)), N, wcap);
    // the running maximum starts at -inf (a kernel, not a host copy: nothing
    // here reads host memory, so the sequence can be captured in a graph)
    MB_CUDA(launch_pdl(k_weight_reset, 1, 1, 0, s, lmax_bits, ordered_bits(-__builtin_huge_val())));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_weight_prep, grid_cap(N, 256), 256, 0, s, N, W, v, add_log, lmax_bits));
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_weight_exp, grid_cap(N, 256), 256, 0, s, N, W, lmax_bits));
    MB_LAUNCH_CHECK();
    cudaStream_t ds = s;  // the stream of the ESS's dot products
    if (fork) {
        MB_CUDA(cudaEventRecord(fork->fork, s));
        MB_CUDA(cudaStreamWaitEvent(fork->side, fork->fork, 0));
        ds = fork->side;
    }
    const unsigned ndot = static_cast<unsigned>((nchunks + kDotWarps - 1) / kDotWarps);
    if (fork) {  // after an event wait: ordinary launches
        k_weight_chunkdot<<<ndot, 32 * kDotWarps, 0, ds>>>(N, W, dots);
        MB_LAUNCH_CHECK();
        k_weight_dotsum<<<1, kFinishThreads, 0, ds>>>(nchunks, dots, essw);
        MB_LAUNCH_CHECK();
    } else {
        MB_CUDA(launch_pdl(k_weight_chunkdot, ndot, 32 * kDotWarps, 0, s, N, W, dots));
        MB_LAUNCH_CHECK();
        MB_CUDA(launch_pdl(k_weight_dotsum, 1, kFinishThreads, 0, s, nchunks, dots, essw));
        MB_LAUNCH_CHECK();
    }
    if (fork) MB_CUDA(cudaEventRecord(fork->join, fork->side));
    int rc = fold_exact(W, N, 0.0, nullptr, fs, s);
    if (rc != MCKL_B200_OK) return rc;
    if (fork) {
        MB_CUDA(cudaStreamWaitEvent(s, fork->join, 0));
        k_weight_finish<<<1, 1, 0, s>>>(essw, fs.final_v, lmax_bits, result_dev);
    } else {
        MB_CUDA(launch_pdl(k_weight_finish, 1, 1, 0, s, essw, fs.final_v, lmax_bits, result_dev));
    }
    MB_LAUNCH_CHECK();
    MB_CUDA(launch_pdl(k_weight_scale, grid_cap(N, 256), 256, 0, s, N, W, fs.final_v));
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

}  // namespace mckl_b200

using namespace mckl_b200;

static int weight_call(size_t N, double *W, const double *v, int add_log, double *ess, double *log_nc, void *stream)
{
    MB_CHECK_ARG(N > 0, "N must be positive");
    MB_CHECK_ARG(W != nullptr && v != nullptr, "null pointer");
    cudaStream_t s = as_stream(stream);
    void *base = scratch(2, weight_scratch_bytes(N) + 64, s);
    if (!base) {
        set_error("weight scratch allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    double *res = reinterpret_cast<double *>(static_cast<char *>(base) + weight_scratch_bytes(N));
    int rc = weight_normalize_dev(N, W, v, add_log, base, res, s);
    if (rc != MCKL_B200_OK) return rc;
    if (ess || log_nc) {
        double h[4];
        MB_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        if (ess) *ess = h[0];
        if (log_nc) *log_nc = h[1];
    }
    return MCKL_B200_OK;
}

extern "C" int mckl_b200_weight_set_log(size_t N, double *W, const double *v, double *ess, double *log_nc,
    void *stream)
{
    return weight_call(N, W, v, 0, ess, log_nc, stream);
}

extern "C" int mckl_b200_weight_add_log(size_t N, double *W, const double *v, double *ess, double *log_nc_inc,
    void *stream)
{
    return weight_call(N, W, v, 1, ess, log_nc_inc, stream);
}
