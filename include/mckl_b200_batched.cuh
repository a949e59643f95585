// mckl_b200_batched.cuh -- the model hook of the batched particle filters.
//
// Many bootstrap filters of a user's scalar state-space model run as one
// persistent kernel, instantiated in the user's own CUDA translation unit:
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -std=c++17 --expt-relaxed-constexpr \
//        -I<repo>/include -I<repo>/mckl_b200/csrc my_model.cu
//
// A model is a struct with a parameter type and a device view of it in the
// propagation type (the built-in AR(1) model, mckl_b200::Ar1Model, is the
// example):
//
//   struct MyModel {
//       struct Param { ... };                 // one filter's parameters
//       template <typename R> struct Dev {    // R = float or double
//           __device__ Dev();
//           __device__ explicit Dev(const Param &p);
//           __device__ R init(R e) const;            // x_0 from a standard normal e
//           __device__ R move(R x, R e) const;       // x_t from x_{t-1} and e
//           __device__ R log_density(R x, R y) const; // log g(y | x) up to a constant
//       };
//   };
//
// Everything else is the built-in filters' (SMCSampler with BackendSEQ per
// filter in the reference, algorithm/smc.hpp:389-406): the Normal(0,1) noise
// of each step from the filter's model stream (Philox4x32, consumed as
// normal_distribution does), FP64 normaliser, ESS and log-likelihood,
// systematic resampling at ESS < threshold N from the resampling stream, the
// slot-preserving parent placement.  With Ar1Model, or a user model that
// does the same arithmetic with the same explicit roundings (Math<R>), the
// results equal the built-in filters' (mckl_b200_batched_run) bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "../mckl_b200/csrc/pf_batched_kernel.cuh"

namespace mckl_b200 {

using batched_detail::Ar1Model;
using batched_detail::Math;

namespace batched_detail {

struct DeviceArrays {
    std::vector<void *> p;
    ~DeviceArrays()
    {
        for (void *q : p) cudaFree(q);
    }
    template <typename T>
    cudaError_t take(T **out, size_t count)
    {
        void *q = nullptr;
        const cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        p.push_back(q);
        *out = static_cast<T *>(q);
        return cudaSuccess;
    }
};

template <typename R, class Model>
cudaError_t run_model(int F, const uint64_t *n, const typename Model::Param *par, const double *y, int T,
    const uint32_t *mkey, const uint32_t *rkey, double threshold, double *loglik, uint32_t *nresampled,
    cudaStream_t s)
{
    constexpr int kThreads = 256, kMinBlocks = 4;
    std::vector<BatchedFilter> h(F);
    uint64_t total = 0;
    for (int f = 0; f < F; ++f) {
        h[f] = BatchedFilter{};
        h[f].n = n[f];
        h[f].off = total;  // every filter's range starts on a multiple of 32 particles
        h[f].mkey[0] = mkey[2 * f];
        h[f].mkey[1] = mkey[2 * f + 1];
        h[f].rkey[0] = rkey[2 * f];
        h[f].rkey[1] = rkey[2 * f + 1];
        total += (n[f] + 31) / 32 * 32;
    }
    // largest filters first (longest-processing-time order for the work queue)
    std::vector<int> order(F);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
    DeviceArrays d;
    BatchedFilter *filt;
    int *ord, *queue;
    double *yd, *ll;
    typename Model::Param *pd;
    R *x, *lw;
    uint32_t *scanS, *epos, *nres;
    cudaError_t e;
    if ((e = d.take(&filt, F)) || (e = d.take(&ord, F)) || (e = d.take(&queue, 1)) ||
        (e = d.take(&yd, static_cast<size_t>(F) * (T + 1))) || (e = d.take(&ll, F)) || (e = d.take(&pd, F)) ||
        (e = d.take(&x, total)) || (e = d.take(&lw, total)) || (e = d.take(&scanS, total)) ||
        (e = d.take(&epos, total)) || (e = d.take(&nres, F)))
        return e;
    if ((e = cudaMemcpyAsync(filt, h.data(), F * sizeof(BatchedFilter), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(ord, order.data(), F * sizeof(int), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(yd, y, static_cast<size_t>(F) * (T + 1) * sizeof(double), cudaMemcpyHostToDevice,
             s)) ||
        (e = cudaMemcpyAsync(pd, par, F * sizeof(typename Model::Param), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemsetAsync(queue, 0, sizeof(int), s)))
        return e;
    auto kernel = k_pf_batched<R, kThreads, false, kMinBlocks, Model>;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0)))
        return e;
    const int ctas = std::max(1, std::min(F, sms * std::max(per_sm, 1)));
    kernel<<<ctas, kThreads, 0, s>>>(filt, ord, F, yd, T, threshold, x, x, lw, scanS, epos, ll, nres, queue,
        nullptr, nullptr, nullptr, nullptr, pd);
    if ((e = cudaGetLastError())) return e;
    if ((e = cudaMemcpyAsync(loglik, ll, F * sizeof(double), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(nresampled, nres, F * sizeof(uint32_t), cudaMemcpyDeviceToHost, s)))
        return e;
    return cudaStreamSynchronize(s);
}

}  // namespace batched_detail

// Runs F filters of `Model`: filter f has n[f] particles (1 <= n[f] < 2^31),
// parameters par[f], observations y[f (T + 1) + t] for t = 1..T (y_0 is not
// used), model and resampling keys (mkey[2f], mkey[2f + 1]) and (rkey[2f],
// rkey[2f + 1]) of Philox4x32; systematic resampling when ESS < threshold N.
// fp64: propagate in double, else in float (the normaliser and the
// log-likelihood are FP64 either way).  Host arrays in, host results out:
// loglik[f] (the log of the estimated likelihood of y_1..y_T) and
// nresampled[f] (resampling steps).  Synchronous on `s`; returns the first
// CUDA error.
template <class Model>
cudaError_t batched_run_model(int F, const uint64_t *n, const typename Model::Param *par, const double *y, int T,
    const uint32_t *mkey, const uint32_t *rkey, double threshold, bool fp64, double *loglik, uint32_t *nresampled,
    cudaStream_t s = nullptr)
{
    if (F <= 0 || T < 0) return cudaErrorInvalidValue;
    for (int f = 0; f < F; ++f)
        if (n[f] == 0 || n[f] >= (1ull << 31)) return cudaErrorInvalidValue;
    return fp64 ? batched_detail::run_model<double, Model>(F, n, par, y, T, mkey, rkey, threshold, loglik,
                                                           nresampled, s)
                : batched_detail::run_model<float, Model>(F, n, par, y, T, mkey, rkey, threshold, loglik,
                                                          nresampled, s);
}

}  // namespace mckl_b200
