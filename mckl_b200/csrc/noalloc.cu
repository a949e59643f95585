// noalloc.cu -- Weight::add_log for callers that cannot allocate device memory.
//
// mckl_b200_weight_add_log needs working memory on the device (the running
// maximum, the per-chunk dot products and the tile bookkeeping of the exact
// sum) and takes it from a buffer the library grows with cudaMalloc.  Some
// host programs cannot let a library do that: plugins whose host owns every
// device allocation through its own pool or budget, code that must not
// synchronize the device (cudaMalloc/cudaFree may), and processes that run
// close to the memory limit and cannot risk a failed allocation in the middle
// of a step.  mckl_b200_weight_add_log_static gives them the same
// normalisation with its working memory in a fixed array compiled into this
// library, so it allocates nothing.
//
// The array below is a host-side symbol: code on the host must not pass its
// name to a kernel (that would hand the GPU a host address).  The device
// address is looked up with cudaGetSymbolAddress once per device, with that
// device current, on the first call made on it, and cached; that first call
// should therefore come before any stream capture.  The cached address
// belongs to the device's primary context: after cudaDeviceReset on a device
// the library's module is loaded again at a new address, so this entry point
// must not be called on that device after a reset in the same process.
#include <mutex>

#include "common.cuh"
#include "weight.cuh"

namespace mckl_b200 {

namespace {

// Largest particle count the fixed working memory serves.
constexpr uint64_t kStaticMaxN = 1ull << 22;
// Window list of the exact sum in the fixed working memory: a sum of
// normalised weights has a few dozen windows; one with more takes the exact
// sum's event-loop path, which needs no list.
constexpr uint64_t kStaticWindows = 256;
// Bytes of fixed working memory per device: the normaliser's scratch for
// kStaticMaxN particles plus 256 bytes of results, rounded up.
constexpr size_t kStaticScratchBytes = 128 * 1024;

static __device__ __align__(256) unsigned char g_weight_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void *g_static_ptr[kMaxDevices] = {nullptr};

// Device address of g_weight_scratch on the current device (looked up once).
int static_scratch(void **out)
{
    int dev = 0;
    MB_CUDA(cudaGetDevice(&dev));
    MB_CHECK_ARG(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (g_static_ptr[dev] == nullptr) {
        // the fixed array must hold the working memory of the largest
        // accepted call plus the results (the sizes come from the
        // normaliser's own layout, so a change there is caught here)
        MB_CHECK_ARG(weight_scratch_bytes(kStaticMaxN, kStaticWindows) + 256 <= kStaticScratchBytes,
            "internal: the fixed working memory is smaller than the largest accepted call needs");
        void *p = nullptr;
        MB_CUDA(cudaGetSymbolAddress(&p, g_weight_scratch));
        g_static_ptr[dev] = p;
    }
    *out = g_static_ptr[dev];
    return MCKL_B200_OK;
}

}  // namespace

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" int mckl_b200_weight_add_log_static(size_t N, double *W, const double *v, double *ess,
    double *log_nc_inc, void *stream)
{
    MB_CHECK_ARG(N > 0, "N must be positive");
    MB_CHECK_ARG(W != nullptr && v != nullptr, "null pointer");
    if (N > kStaticMaxN || weight_scratch_bytes(N, kStaticWindows) + 256 > kStaticScratchBytes) {
        set_error("mckl_b200_weight_add_log_static: N = " + std::to_string(N) +
                  " exceeds the fixed working memory (at most " + std::to_string(kStaticMaxN) +
                  " particles); use mckl_b200_weight_add_log");
        return MCKL_B200_ERR_ARG;
    }
    void *base = nullptr;
    int rc = static_scratch(&base);
    if (rc != MCKL_B200_OK) return rc;
    cudaStream_t s = as_stream(stream);
    double *res = reinterpret_cast<double *>(static_cast<char *>(base) + weight_scratch_bytes(N, kStaticWindows));
    // every value the normaliser reads from its working memory is written
    // first in the same call (the running maximum is reset by a one-thread
    // kernel), so the previous call's leftovers never leak into this one
    rc = weight_normalize_dev(N, W, v, 1, base, res, s, kStaticWindows);
    if (rc != MCKL_B200_OK) return rc;
    if (ess || log_nc_inc) {
        double h[2];
        MB_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, s));
        MB_CUDA(cudaStreamSynchronize(s));
        if (ess) *ess = h[0];
        if (log_nc_inc) *log_nc_inc = h[1];
    }
    return MCKL_B200_OK;
}
