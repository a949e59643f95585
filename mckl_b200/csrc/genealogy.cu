// genealogy.cu -- ResampleIndex trace-back (algorithm/resample.hpp:597-832)
// on recorded parent indices that stay in device memory.
//
// The reference keeps one parent-index vector per iteration and follows a
// particle's line back with idx = index_[j][idx] (:666-678); its index matrix
// (:752-829) holds, for each particle of iteration iter_back, its ancestors at
// iterations iter..iter_back.  Here every particle's line is one thread: it
// starts from index_[iter_back][i] and gathers backwards through the vectors,
// writing one column per iteration.  Column-major output is coalesced over
// particles as written; for row-major output a CTA stages a few iterations of
// its particles' lines in shared memory and writes whole row segments.
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace mckl_b200 {

namespace {

// Every thread follows kLines particle lines at once (particles i, i + S, ..,
// S the grid's thread count), so kLines dependent gathers are in flight per
// thread.
constexpr int kLines = 2;  // 1, 4 and 8 measured slower

// one step back along a line: a parent index outside the earlier vector would
// read past it, so it records the error and stops the line
__device__ __forceinline__ void step_back(uint64_t r, uint64_t R, const uint64_t *const *index,
    const uint64_t *sizes, uint64_t &idx, bool &live, uint32_t *err)
{
    if (live && r + 1 < R) {
        if (idx >= sizes[r]) {
            atomicOr(err, 1u);
            live = false;
        } else {
            idx = index[r][idx];
        }
    }
}

__global__ void __launch_bounds__(256, 8) k_index_matrix_cols(uint64_t N, uint64_t R, const uint64_t *const *index,
    const uint64_t *sizes, uint64_t *out, uint32_t *err)
{
    const uint64_t S = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i0 = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i0 < N; i0 += S * kLines) {
        uint64_t idx[kLines];
        bool live[kLines];
#pragma unroll
        for (int k = 0; k < kLines; ++k) {
            const uint64_t i = i0 + k * S;
            live[k] = i < N;
            idx[k] = live[k] ? index[R - 1][i] : 0;
        }
        for (uint64_t r = R; r-- > 0;) {
#pragma unroll
            for (int k = 0; k < kLines; ++k) {
                step_back(r, R, index, sizes, idx[k], live[k], err);
                if (live[k]) out[r * N + i0 + k * S] = idx[k];
            }
        }
    }
}

// row-major: a CTA owns 256 * kRowLines consecutive particles and stages
// kRowTile iterations of their lines in shared memory, then writes each
// particle's kRowTile contiguous words with consecutive threads
constexpr int kRowTile = 8;   // 16 measured slower
constexpr int kRowLines = 1;  // 2 measured slower
constexpr int kRowParts = 256 * kRowLines;

__global__ void __launch_bounds__(256) k_index_matrix_rows(uint64_t N, uint64_t R, const uint64_t *const *index,
    const uint64_t *sizes, uint64_t *out, uint32_t *err)
{
    __shared__ uint64_t tile[kRowParts][kRowTile + 1];
    for (uint64_t base = blockIdx.x * static_cast<uint64_t>(kRowParts); base < N;
         base += static_cast<uint64_t>(gridDim.x) * kRowParts) {
        const uint64_t rows = min(static_cast<uint64_t>(kRowParts), N - base);
        uint64_t idx[kRowLines];
        bool live[kRowLines];
#pragma unroll
        for (int k = 0; k < kRowLines; ++k) {
            const uint64_t i = base + threadIdx.x + k * 256;
            live[k] = i < N;
            idx[k] = live[k] ? index[R - 1][i] : 0;
        }
        for (uint64_t hi = R; hi > 0;) {
            const uint64_t lo = hi > static_cast<uint64_t>(kRowTile) ? hi - kRowTile : 0;
            for (uint64_t r = hi; r-- > lo;) {
#pragma unroll
                for (int k = 0; k < kRowLines; ++k) {
                    step_back(r, R, index, sizes, idx[k], live[k], err);
                    tile[threadIdx.x + k * 256][r - lo] = idx[k];
                }
            }
            __syncthreads();
            const uint32_t w = static_cast<uint32_t>(hi - lo);
            for (uint32_t k = threadIdx.x; k < rows * w; k += 256) {
                const uint32_t row = k / w, col = k % w;
                out[(base + row) * R + lo + col] = tile[row][col];
            }
            __syncthreads();
            hi = lo;
        }
    }
}

// Page-locked staging for the upload (vector addresses, sizes, error word)
// and the error read-back: small copies from pageable memory go through the
// driver's staging buffers and cost several microseconds each.  One buffer
// per process, grown on demand, held for the whole call.
std::mutex g_stage_mu;
uint64_t *g_stage = nullptr;
size_t g_stage_words = 0;

uint64_t *stage_words(size_t words)
{
    if (words > g_stage_words) {
        if (g_stage) {
            // a call that failed after queuing its upload may still have
            // it in flight from the old buffer
            cudaDeviceSynchronize();
            cudaFreeHost(g_stage);
        }
        g_stage = nullptr;
        g_stage_words = 0;
        const size_t want = std::max<size_t>(words, 4096);
        if (cudaHostAlloc(reinterpret_cast<void **>(&g_stage), want * sizeof(uint64_t), cudaHostAllocPortable) !=
            cudaSuccess) {
            cudaGetLastError();
            g_stage = nullptr;
            return nullptr;
        }
        g_stage_words = want;
    }
    return g_stage;
}

}  // namespace

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" int mckl_b200_index_matrix(size_t N, size_t R, const uint64_t *const *index_host, const size_t *sizes_host,
    int col_major, uint64_t *out, void *stream)
{
    MB_CHECK_ARG(R > 0 && index_host != nullptr && sizes_host != nullptr, "null index vectors");
    MB_CHECK_ARG(N == 0 || out != nullptr, "null output");
    MB_CHECK_ARG(sizes_host[R - 1] == N, "the last vector must have N entries");
    if (N == 0) return MCKL_B200_OK;
    cudaStream_t s = as_stream(stream);
    // one upload: R vector addresses, R sizes, the error word (zero)
    const size_t words = 2 * R + 1;
    char *scr = static_cast<char *>(scratch(7, align256(words * sizeof(uint64_t)), s));
    if (!scr) return MCKL_B200_ERR_NOMEM;
    auto **dptr = reinterpret_cast<const uint64_t **>(scr);
    auto *dsz = reinterpret_cast<uint64_t *>(scr + R * sizeof(uint64_t));
    auto *derr = reinterpret_cast<uint32_t *>(scr + 2 * R * sizeof(uint64_t));
    for (size_t r = 0; r < R; ++r) {
        MB_CHECK_ARG(index_host[r] != nullptr || sizes_host[r] == 0, "null index vector");
    }
    std::lock_guard<std::mutex> lock(g_stage_mu);  // the staging buffer is reused once this call has synchronized
    uint64_t *up = stage_words(words + 1);
    if (!up) {
        set_error("mckl_b200_index_matrix: page-locked staging buffer allocation failed");
        return MCKL_B200_ERR_NOMEM;
    }
    for (size_t r = 0; r < R; ++r) {
        up[r] = reinterpret_cast<uint64_t>(index_host[r]);
        up[R + r] = sizes_host[r];
    }
    up[2 * R] = 0;
    MB_CUDA(cudaMemcpyAsync(scr, up, words * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // one wave: the resident CTAs, or fewer when the particles run out
    int occ = 1;
    if (col_major) {
        MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_index_matrix_cols, 256, 0));
        const uint64_t blocks = std::min<uint64_t>((N + 256 * kLines - 1) / (256 * kLines),
            static_cast<uint64_t>(sms) * std::max(occ, 1));
        k_index_matrix_cols<<<static_cast<unsigned>(blocks), 256, 0, s>>>(N, R, dptr, dsz, out, derr);
    } else {
        MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_index_matrix_rows, 256, 0));
        const uint64_t blocks = std::min<uint64_t>((N + kRowParts - 1) / kRowParts,
            static_cast<uint64_t>(sms) * std::max(occ, 1));
        k_index_matrix_rows<<<static_cast<unsigned>(blocks), 256, 0, s>>>(N, R, dptr, dsz, out, derr);
    }
    MB_LAUNCH_CHECK();
    uint32_t *herr_p = reinterpret_cast<uint32_t *>(up + words);
    *herr_p = 0;
    MB_CUDA(cudaMemcpyAsync(herr_p, derr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    if (*herr_p) {
        set_error("mckl_b200_index_matrix: a parent index is outside the previous iteration's particles");
        return MCKL_B200_ERR_ARG;
    }
    return MCKL_B200_OK;
}
