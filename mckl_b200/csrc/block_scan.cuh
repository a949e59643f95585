// block_scan.cuh -- warp and CTA-wide scans / reductions used by the SMC kernels.
#pragma once

#include <cstdint>
#include <cstring>

namespace mckl_b200 {

template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T n = __shfl_xor_sync(0xffffffffu, v, o);
        v = n > v ? n : v;
    }
    return v;
}

// Inclusive prefix sum over the CTA (blockDim.x a multiple of 32, <= 1024).
// `sh` needs 33 elements of shared scratch; returns the CTA total in *total.
template <typename T>
__device__ __forceinline__ T block_inclusive_sum(T v, T *sh, T *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T inc = warp_inclusive_sum(v);
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nw ? sh[lane] : T(0);
        w = warp_inclusive_sum(w);
        if (lane < nw) sh[lane] = w;
        if (lane == nw - 1) sh[32] = w;
    }
    __syncthreads();
    if (warp > 0) inc += sh[warp - 1];
    *total = sh[32];
    __syncthreads();
    return inc;
}

// Inclusive prefix sum over the CTA with a single barrier: every warp scans
// the warp totals itself.  `sh` needs 32 elements; the caller must separate
// two uses of the same `sh` by another CTA barrier (no trailing barrier here).
template <typename T>
__device__ __forceinline__ T block_inclusive_sum_1b(T v, T *sh, T *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const T inc = warp_inclusive_sum(v);
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    T w = lane < nw ? sh[lane] : T(0);
    w = warp_inclusive_sum(w);
    const T before = __shfl_sync(0xffffffffu, w, warp > 0 ? warp - 1 : 0);
    *total = __shfl_sync(0xffffffffu, w, nw - 1);
    return warp > 0 ? before + inc : inc;
}

// Exclusive prefix sum over the CTA formed without a subtraction: each
// thread's result is a sum of the values of the threads before it only, so
// for floating-point inputs its rounding error is relative to itself (an
// inclusive sum minus the own value would carry the error of the larger
// inclusive sum).  `sh` needs 33 elements; the CTA total goes to *total.
template <typename T>
__device__ __forceinline__ T block_exclusive_sum(T v, T *sh, T *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const T inc = warp_inclusive_sum(v);
    T prev = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) prev = T(0);
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const T w = lane < nw ? sh[lane] : T(0);
        const T wi = warp_inclusive_sum(w);
        T we = __shfl_up_sync(0xffffffffu, wi, 1);
        if (lane == 0) we = T(0);
        if (lane < nw) sh[lane] = we;
        if (lane == nw - 1) sh[32] = wi;
    }
    __syncthreads();
    const T r = warp > 0 ? sh[warp] + prev : prev;
    *total = sh[32];
    __syncthreads();
    return r;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T w = lane < nw ? sh[lane] : T(0);
        w = warp_sum(w);
        if (lane == 0) sh[32] = w;
    }
    __syncthreads();
    const T r = sh[32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ unsigned block_min_u32(unsigned v, unsigned *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = __reduce_min_sync(0xffffffffu, v);
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        unsigned w = lane < nw ? sh[lane] : 0xffffffffu;
        w = __reduce_min_sync(0xffffffffu, w);
        if (lane == 0) sh[32] = w;
    }
    __syncthreads();
    const unsigned r = sh[32];
    __syncthreads();
    return r;
}

// Order-preserving map of doubles to signed 64-bit integers (for atomicMax).
__host__ __device__ __forceinline__ long long ordered_bits(double x)
{
#if defined(__CUDA_ARCH__)
    const long long b = __double_as_longlong(x);
#else
    long long b;
    memcpy(&b, &x, sizeof(b));
#endif
    return b >= 0 ? b : (b ^ 0x7fffffffffffffffll);
}

__device__ __forceinline__ double from_ordered_bits(long long b)
{
    return __longlong_as_double(b >= 0 ? b : (b ^ 0x7fffffffffffffffll));
}

}  // namespace mckl_b200
