// estimator.cu -- SMCEstimator's weighted estimate (algorithm/smc.hpp:90-120)
// on device-resident evaluations: result_j = sum_i W_i u(i, j), the
// reference's cblas_dgemv with the normalised weights.  BLAS leaves the order
// of the sum open; here each CTA sums a contiguous range of particles per
// column (FP64 fma, a fixed order for a given size), and a second pass adds
// the CTA partials in a fixed tree, so the result is deterministic.
//
// Every layout reads u once, coalesced:
//   column-major (u[j n + i]): one CTA per (column, particle chunk);
//   row-major, d <= 256 (u[i d + j]): one CTA per particle chunk walks the
//     chunk's d * rows words flat; thread t always lands on column t mod d
//     (its stride, d * floor(256 / d), is a multiple of d);
//   row-major, d > 256: one CTA per (particle chunk, 256-column tile), a
//     thread per column, rows in order.
#include <algorithm>

#include "block_scan.cuh"
#include "common.cuh"

namespace mckl_b200 {

namespace {

constexpr int kEstThreads = 256;
constexpr uint64_t kEstChunk = 8192;      // particles per CTA (column-major)
constexpr uint64_t kEstChunkNarrow = 2048;  // particles per CTA (row-major, d <= 256): several waves of CTAs
constexpr uint64_t kEstChunkWide = 1024;  // particles per CTA (row-major, d > 256)

// column j = blockIdx.x: the CTAs of one chunk run next to each other and
// share its weights in L2 (the weights are read from DRAM once)
__global__ void __launch_bounds__(kEstThreads) k_est_cols(uint64_t n, uint64_t nb, const double *u, const double *w,
    double *partial)
{
    __shared__ double shd[33];
    const uint64_t j = blockIdx.x;
    const double *uj = u + j * n;
    for (uint64_t c = blockIdx.y; c < nb; c += gridDim.y) {
        const uint64_t b0 = c * kEstChunk, b1 = min(n, b0 + kEstChunk);
        double acc = 0.0;
        for (uint64_t i = b0 + threadIdx.x; i < b1; i += kEstThreads) acc = fma(w[i], uj[i], acc);
        acc = block_sum(acc, shd);
        if (threadIdx.x == 0) partial[j * nb + c] = acc;
    }
}

__global__ void __launch_bounds__(kEstThreads) k_est_rows_narrow(uint64_t n, uint32_t d, const double *u,
    const double *w, double *partial)
{
    __shared__ double sh[kEstThreads];
    const uint32_t q = kEstThreads / d;  // rows per pass
    const uint32_t t = threadIdx.x;
    const uint64_t b0 = blockIdx.x * kEstChunkNarrow, b1 = min(n, b0 + kEstChunkNarrow);
    double acc = 0.0;
    if (t < q * d) {
        const uint32_t j = t % d;
#pragma unroll 4
        for (uint64_t i = b0 + t / d; i < b1; i += q) acc = fma(w[i], u[i * d + j], acc);
    }
    sh[t] = acc;
    __syncthreads();
    if (t < d) {
        double s = 0.0;
        for (uint32_t k = 0; k < q; ++k) s += sh[k * d + t];
        partial[static_cast<uint64_t>(t) * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(kEstThreads) k_est_rows_wide(uint64_t n, uint64_t d, const double *u,
    const double *w, double *partial)
{
    const uint64_t j = blockIdx.y * static_cast<uint64_t>(kEstThreads) + threadIdx.x;
    if (j >= d) return;
    const uint64_t b0 = blockIdx.x * kEstChunkWide, b1 = min(n, b0 + kEstChunkWide);
    double acc = 0.0;
    for (uint64_t i = b0; i < b1; ++i) acc = fma(w[i], u[i * d + j], acc);
    partial[j * gridDim.x + blockIdx.x] = acc;
}

// one CTA per column: thread t adds partials t, t + 256, ... into four
// accumulators (four loads in flight), then a fixed CTA tree
__global__ void __launch_bounds__(kEstThreads) k_est_final(uint64_t nb, const double *partial, double *result)
{
    __shared__ double shd[33];
    const double *pj = partial + static_cast<uint64_t>(blockIdx.x) * nb;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    uint64_t b = threadIdx.x;
    for (; b + 3 * kEstThreads < nb; b += 4 * kEstThreads) {
        a0 += pj[b];
        a1 += pj[b + kEstThreads];
        a2 += pj[b + 2 * kEstThreads];
        a3 += pj[b + 3 * kEstThreads];
    }
    for (; b < nb; b += kEstThreads) a0 += pj[b];
    const double s = block_sum((a0 + a1) + (a2 + a3), shd);
    if (threadIdx.x == 0) result[blockIdx.x] = s;
}

}  // namespace

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" int mckl_b200_weighted_estimate(size_t n, size_t d, int col_major, const double *u, const double *w,
    double *result, void *stream)
{
    MB_CHECK_ARG(d > 0 && d <= 65535 * static_cast<size_t>(kEstThreads), "d in [1, 65535 * 256]");
    MB_CHECK_ARG(!col_major || d <= 65535, "column-major: d in [1, 65535]");
    MB_CHECK_ARG(result != nullptr && (n == 0 || (u != nullptr && w != nullptr)), "null argument");
    cudaStream_t s = as_stream(stream);
    if (n == 0) {
        MB_CUDA(cudaMemsetAsync(result, 0, d * sizeof(double), s));
        return MCKL_B200_OK;
    }
    const bool wide = !col_major && d > static_cast<size_t>(kEstThreads);
    const uint64_t chunk = col_major ? kEstChunk : (wide ? kEstChunkWide : kEstChunkNarrow);
    const uint64_t nb = (n + chunk - 1) / chunk;
    MB_CHECK_ARG(nb <= 0x7fffffffull, "too many particles");
    double *partial = static_cast<double *>(scratch(8, align256(nb * d * sizeof(double)), s));
    if (!partial) return MCKL_B200_ERR_NOMEM;
    if (col_major) {
        const unsigned chunks = static_cast<unsigned>(std::min<uint64_t>(nb, 65535));
        k_est_cols<<<dim3(static_cast<unsigned>(d), chunks), kEstThreads, 0, s>>>(n, nb, u, w, partial);
    } else if (!wide) {
        k_est_rows_narrow<<<static_cast<unsigned>(nb), kEstThreads, 0, s>>>(n, static_cast<uint32_t>(d), u, w,
            partial);
    } else {
        const unsigned tiles = static_cast<unsigned>((d + kEstThreads - 1) / kEstThreads);
        k_est_rows_wide<<<dim3(static_cast<unsigned>(nb), tiles), kEstThreads, 0, s>>>(n, d, u, w, partial);
    }
    MB_LAUNCH_CHECK();
    k_est_final<<<static_cast<unsigned>(d), kEstThreads, 0, s>>>(nb, partial, result);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}
