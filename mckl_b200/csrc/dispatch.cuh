// dispatch.cuh -- engine kind -> generator dispatch and word views shared by
// the RNG and distribution kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "engines.cuh"

namespace mckl_b200 {

// Allow `kernel` to use `dyn` bytes of dynamic shared memory on top of its
// static shared memory (needed once the sum passes 48 KiB).
template <typename K>
inline cudaError_t allow_dyn_smem(K kernel, int dyn)
{
    if (dyn == 0) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
}

template <typename W>
struct WordView;

template <>
struct WordView<uint32_t> {
    template <int N>
    __device__ static uint32_t get(const uint32_t (&b)[N], int j) { return b[j]; }
    static constexpr int kPer32 = 1;
};

template <>
struct WordView<uint64_t> {
    template <int N>
    __device__ static uint64_t get(const uint32_t (&b)[N], int j)
    {
        return static_cast<uint64_t>(b[2 * j]) | (static_cast<uint64_t>(b[2 * j + 1]) << 32);
    }
    static constexpr int kPer32 = 2;
};

template <class Fn>
inline int with_generator(const mckl_b200_engine_t &e, Fn &&fn)
{
    switch (e.kind) {
        case MCKL_B200_PHILOX4X32:
        case MCKL_B200_PHILOX4X32_64: {
            PhiloxGen g{static_cast<uint32_t>(e.key[0]), static_cast<uint32_t>(e.key[1])};
            return fn(g);
        }
        case MCKL_B200_THREEFRY4X64:
        case MCKL_B200_THREEFRY4X64_64: {
            ThreefryGen g = ThreefryGen::make(e.key, e.tweak);
            return fn(g);
        }
        case MCKL_B200_ARS:
        case MCKL_B200_ARS_64: {
            ArsGen g = ArsGen::make(e.key);
            return fn(g);
        }
        default:
            set_error("unknown engine kind");
            return MCKL_B200_ERR_ARG;
    }
}

}  // namespace mckl_b200
