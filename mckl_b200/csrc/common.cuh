// common.cuh -- host-side plumbing shared by the CUDA translation units:
// error reporting across the C ABI, engine geometry, and the exact
// CounterEngine state bookkeeping (random/counter.hpp:142-199).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/mckl_b200.h"
#include "engines.cuh"

namespace mckl_b200 {

// ---- error reporting -------------------------------------------------------
void set_error(const std::string &msg);

#define MB_CHECK_ARG(cond, msg)                 \
    do {                                        \
        if (!(cond)) {                          \
            ::mckl_b200::set_error(msg);        \
            return MCKL_B200_ERR_ARG;           \
        }                                       \
    } while (0)

#define MB_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t err_ = (call);                                                 \
        if (err_ != cudaSuccess) {                                                 \
            ::mckl_b200::set_error(std::string(#call) + ": " + cudaGetErrorString(err_)); \
            return MCKL_B200_ERR_CUDA;                                             \
        }                                                                          \
    } while (0)

// Every kernel launch is followed by MB_LAUNCH_CHECK(), which also counts it.
void count_launch();
#define MB_LAUNCH_CHECK()                 \
    do {                                  \
        ::mckl_b200::count_launch();      \
        MB_CUDA(cudaGetLastError());      \
    } while (0)

inline cudaStream_t as_stream(void *s)
{
    return reinterpret_cast<cudaStream_t>(s);
}

// ---- programmatic dependent launch -----------------------------------------
// The SMC step's kernels form long chains of small dependent launches.  A
// kernel of such a chain is launched with programmatic stream serialisation
// (launch_pdl), so that its launch and CTA set-up overlap the end of the
// kernel before it, and begins with pdl_wait(), which returns once that
// kernel has completed and its writes are visible.  pdl_wait() is a no-op in
// a kernel launched the ordinary way, so the same kernels serve both.
__device__ __forceinline__ void pdl_wait()
{
#if defined(__CUDA_ARCH__)
    asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = s == nullptr ? 0 : 1;  // the legacy default stream: an ordinary launch
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...);
}

// ---- engine geometry -------------------------------------------------------
struct Geom {
    int M;          // result words per block
    int rbytes;     // bytes per result word (4 or 8)
    int cwords;     // u64 counter words
    int bwords32;   // u32 words per block
};

inline bool kind_valid(uint32_t kind)
{
    return kind >= MCKL_B200_PHILOX4X32 && kind <= MCKL_B200_ARS_64;
}

inline Geom geom(uint32_t kind)
{
    switch (kind) {
        case MCKL_B200_PHILOX4X32: return {4, 4, 2, 4};
        case MCKL_B200_PHILOX4X32_64: return {2, 8, 2, 4};
        case MCKL_B200_THREEFRY4X64: return {8, 4, 4, 8};
        case MCKL_B200_THREEFRY4X64_64: return {4, 8, 4, 8};
        case MCKL_B200_ARS: return {4, 4, 2, 4};
        case MCKL_B200_ARS_64: return {2, 8, 2, 4};
        default: return {0, 0, 0, 0};
    }
}

inline Ctr ctr_of(const mckl_b200_engine_t &e)
{
    Ctr c;
    for (int i = 0; i < 4; ++i) c.w[i] = e.ctr[i];
    return c;
}

inline void set_ctr(mckl_b200_engine_t &e, const Ctr &c)
{
    for (int i = 0; i < 4; ++i) e.ctr[i] = c.w[i];
}

// Where the next word comes from: word `off` of the block with counter `B`.
inline void next_position(const mckl_b200_engine_t &e, Ctr &B, uint32_t &off)
{
    const Geom g = geom(e.kind);
    const uint32_t idx = e.index < static_cast<uint32_t>(g.M) ? e.index : g.M;
    if (idx < static_cast<uint32_t>(g.M)) {
        B = ctr_of(e);
        off = idx;
    } else {
        B = ctr_add(ctr_of(e), 1, g.cwords);
        off = 0;
    }
}

// State after one CounterEngine::operator()(n, r) call (random/counter.hpp:142-165).
inline void advance_call(mckl_b200_engine_t &e, uint64_t n)
{
    const Geom g = geom(e.kind);
    const uint64_t M = static_cast<uint64_t>(g.M);
    const uint64_t idx = e.index < M ? e.index : M;
    const uint64_t remain = M - idx;
    if (n <= remain) {
        e.index = static_cast<uint32_t>(idx + n);
        return;
    }
    const uint64_t rem2 = n - remain;
    const uint64_t m = rem2 / M;
    set_ctr(e, ctr_add(ctr_of(e), m + 1, g.cwords));
    e.index = static_cast<uint32_t>(rem2 - m * M);
}

// State after `q` consecutive calls of `S` words each (S > words per block,
// so every call after the first starts from a partially used block and ends
// in the canonical form ctr = block of the next word, index = its offset).
inline void advance_calls(mckl_b200_engine_t &e, uint64_t q, uint64_t S)
{
    if (q == 0) return;
    advance_call(e, S);
    if (q == 1) return;
    const Geom g = geom(e.kind);
    const uint64_t M = static_cast<uint64_t>(g.M);
    const uint64_t total = static_cast<uint64_t>(e.index) + (q - 1) * S;
    set_ctr(e, ctr_add(ctr_of(e), total / M, g.cwords));
    e.index = static_cast<uint32_t>(total % M);
}

// Round a byte count up to a multiple of 256 (every carved scratch region
// starts on a 256-byte boundary).
inline size_t align256(size_t n)
{
    return (n + 255) & ~static_cast<size_t>(255);
}

// Working device memory owned by the library: one growable buffer per
// (device, stream, slot), so calls on different streams never share it.
// Returns nullptr when it cannot be obtained (or would have to grow while
// the stream is being captured).
void *scratch(int slot, size_t bytes, cudaStream_t stream);
// Release the buffers of `stream` on the current device.
int scratch_release(cudaStream_t stream);

}  // namespace mckl_b200
