// transforms.cuh -- device restatements of the reference's word -> real
// conversions (random/internal/u01_generic.hpp:48-198) and of the
// per-element arithmetic of the Normal / Exponential transforms.  Every
// rounding step is written with an explicit _rn intrinsic so the compiler
// cannot contract a multiply and an add into one FMA where the reference
// rounds twice (and vice versa where the reference calls std::fma).
#pragma once

#include <cstdint>

#include "crmath.cuh"

namespace mckl_b200 {

enum U01Variant { kCanonical = 0, kCC = 1, kCO = 2, kOC = 3, kOO = 4 };

// ---- words -> double ---------------------------------------------------------
__device__ __forceinline__ double u01_f64(int v, uint32_t u)
{
    const double d = static_cast<double>(u);
    switch (v) {
        case kCC: return __dmul_rn(__dadd_rn(static_cast<double>(u & 1u), d), 0x1p-32);
        case kCO: return __dmul_rn(d, 0x1p-32);
        case kOC: return __dadd_rn(__dmul_rn(d, 0x1p-32), 0x1p-32);
        case kOO: return __dadd_rn(__dmul_rn(d, 0x1p-32), 0x1p-33);
        default: return __dadd_rn(__dmul_rn(d, 0x1p-32), 0.0);  // canonical, one word (float result only)
    }
}

__device__ __forceinline__ double u01_f64(int v, uint64_t u)
{
    switch (v) {
        case kCC: {
            const uint64_t w = (u << 1) >> 10;
            return __dmul_rn(static_cast<double>((w & 1u) + w), 0x1p-54);
        }
        case kCO: return __dmul_rn(static_cast<double>(u >> 11), 0x1p-53);
        case kOC: return __dadd_rn(__dmul_rn(static_cast<double>(u >> 11), 0x1p-53), 0x1p-53);
        case kOO: return __dadd_rn(__dmul_rn(static_cast<double>(u >> 12), 0x1p-52), 0x1p-53);
        default: return __dadd_rn(__dmul_rn(__ull2double_rn(u), 0x1p-64), 0.0);
    }
}

// canonical double from two u32 words (U01CanonicalGenericImpl with Q = 2)
__device__ __forceinline__ double u01_canonical2(uint32_t u0, uint32_t u1)
{
    const double hi = __dadd_rn(__dmul_rn(static_cast<double>(u1), 0x1p-32), 0.0);
    return __dadd_rn(__dmul_rn(static_cast<double>(u0), 0x1p-64), hi);
}

// ---- words -> float ----------------------------------------------------------
__device__ __forceinline__ float u01_f32(int v, uint32_t u)
{
    switch (v) {
        case kCC: {
            const uint32_t w = (u << 1) >> 7;
            return __fmul_rn(static_cast<float>((w & 1u) + w), 0x1p-25f);
        }
        case kCO: return __fmul_rn(static_cast<float>(u >> 8), 0x1p-24f);
        case kOC: return __fadd_rn(__fmul_rn(static_cast<float>(u >> 8), 0x1p-24f), 0x1p-24f);
        case kOO: return __fadd_rn(__fmul_rn(static_cast<float>(u >> 9), 0x1p-23f), 0x1p-24f);
        default: return __fadd_rn(__fmul_rn(__uint2float_rn(u), 0x1p-32f), 0.0f);
    }
}

__device__ __forceinline__ float u01_f32(int v, uint64_t u)
{
    switch (v) {
        case kCC: {
            const uint64_t w = (u << 1) >> 39;
            return __fmul_rn(static_cast<float>((w & 1u) + w), 0x1p-25f);
        }
        case kCO: return __fmul_rn(static_cast<float>(u >> 40), 0x1p-24f);
        case kOC: return __fadd_rn(__fmul_rn(static_cast<float>(u >> 40), 0x1p-24f), 0x1p-24f);
        case kOO: return __fadd_rn(__fmul_rn(static_cast<float>(u >> 41), 0x1p-23f), 0x1p-24f);
        default: return __fadd_rn(__fmul_rn(__ull2float_rn(u), 0x1p-64f), 0.0f);
    }
}

template <typename R>
struct RealOps;

template <>
struct RealOps<double> {
    static constexpr double kTwoPi = 0x1.921fb54442d18p+2;
    __device__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ static double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    __device__ static double log(double a) { return dd::log(a); }
    __device__ static double exp(double a) { return dd::exp(a); }
    __device__ static double sqrt(double a) { return __dsqrt_rn(a); }
    __device__ static void sincos(double a, double *s, double *c) { dd::sincos(a, s, c); }
    __device__ static double cos(double a) { return dd::cos(a); }
    template <typename W>
    __device__ static double u01(int v, W u) { return u01_f64(v, u); }
};

template <>
struct RealOps<float> {
    static constexpr float kTwoPi = 0x1.921fb6p+2f;
    __device__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    __device__ static float log(float a) { return ::logf(a); }
    __device__ static float exp(float a) { return ::expf(a); }
    __device__ static float sqrt(float a) { return __fsqrt_rn(a); }
    __device__ static void sincos(float a, float *s, float *c) { ::sincosf(a, s, c); }
    __device__ static float cos(float a) { return ::cosf(a); }
    template <typename W>
    __device__ static float u01(int v, W u) { return u01_f32(v, u); }
};

}  // namespace mckl_b200
