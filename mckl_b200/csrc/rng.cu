// rng.cu -- RNG fills and the U01 / Normal / Exponential transforms on sm_100a.
//
// Every kernel is a pure function of (generator key, first block counter,
// word offset): thread i of the grid computes its blocks straight from the
// counter, so there is no inter-thread dependency and no read traffic.  Two
// shapes cover every call:
//   * aligned: the stream starts on a block boundary and the output is
//     16-byte aligned -> each thread turns whole blocks into 128-bit stores;
//   * staged: any start offset / alignment -> a CTA generates a tile of blocks
//     into shared memory and writes its outputs from there, coalesced.
// The Normal transform pairs the two halves of each 8192-byte chunk
// (random/normal_distribution.hpp:50-78), so one CTA owns one chunk and stages
// the chunk's words in shared memory.
#include <algorithm>
#include <atomic>
#include <type_traits>
#include <cstring>
#include <mutex>
#include <functional>
#include <map>

#include "common.cuh"
#include "dispatch.cuh"
#include "transforms.cuh"

namespace mckl_b200 {

// ---------------------------------------------------------------------------
// error state, scratch
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void set_error(const std::string &msg)
{
    g_last_error = msg;
}

void count_launch()
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

struct ScratchBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct ScratchKey {
    int dev;
    cudaStream_t stream;
    int slot;
    bool operator<(const ScratchKey &o) const
    {
        if (dev != o.dev) return dev < o.dev;
        if (stream != o.stream) return std::less<cudaStream_t>()(stream, o.stream);
        return slot < o.slot;
    }
};

static std::mutex g_scratch_mu;
static std::map<ScratchKey, ScratchBuf> g_scratch;

// One buffer per (device, stream, slot): calls on different streams never
// share working memory, and calls on one stream are ordered by the stream.
// The buffers come from the stream-ordered allocator, so a buffer that must
// grow is released after the work already queued on its stream
// (cudaFreeAsync) and replaced on the same stream without synchronising the
// device.  Growing is refused while the stream is being captured (the
// allocation would belong to the graph).
void *scratch(int slot, size_t bytes, cudaStream_t stream)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    ScratchBuf &b = g_scratch[ScratchKey{dev, stream, slot}];
    if (b.bytes < bytes) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            set_error("working memory must grow during stream capture; make one call of this size on the "
                      "stream before capturing it");
            return nullptr;
        }
        if (b.ptr) {
            if (cudaFreeAsync(b.ptr, stream) != cudaSuccess) return nullptr;
            b.ptr = nullptr;
            b.bytes = 0;
        }
        const size_t want = std::max<size_t>(bytes, 1 << 20);
        if (cudaMallocAsync(&b.ptr, want, stream) != cudaSuccess) {
            b.ptr = nullptr;
            return nullptr;
        }
        b.bytes = want;
    }
    return b.ptr;
}

// Release every working buffer this library holds for `stream` on the
// current device (after the work queued on it).
int scratch_release(cudaStream_t stream)
{
    int dev = 0;
    MB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    for (auto it = g_scratch.begin(); it != g_scratch.end();) {
        if (it->first.dev == dev && it->first.stream == stream) {
            if (it->second.ptr) MB_CUDA(cudaFreeAsync(it->second.ptr, stream));
            it = g_scratch.erase(it);
        } else {
            ++it;
        }
    }
    return MCKL_B200_OK;
}

// ---------------------------------------------------------------------------
// launch geometry
// ---------------------------------------------------------------------------
static int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

static unsigned grid_for(uint64_t work_items, int threads, int ctas_per_sm)
{
    const uint64_t need = (work_items + threads - 1) / threads;
    const uint64_t cap = static_cast<uint64_t>(sm_count()) * ctas_per_sm;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min(need, cap)));
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
// Write block i into a shared staging buffer with 128-bit stores: consecutive
// lanes then fill consecutive 16-byte slots (no bank conflicts).
template <class G>
__device__ __forceinline__ void stage_block(uint32_t *st32, int i, const uint32_t (&blk)[G::kWords])
{
    uint4 *dst = reinterpret_cast<uint4 *>(st32) + i * (G::kWords / 4);
#pragma unroll
    for (int q = 0; q < G::kWords / 4; ++q) {
        dst[q] = make_uint4(blk[4 * q], blk[4 * q + 1], blk[4 * q + 2], blk[4 * q + 3]);
    }
}

// Store N values of R starting at a pointer known to be 16-byte aligned.
template <typename R, int N>
__device__ __forceinline__ void store_aligned(R *p, const R (&v)[N])
{
    if constexpr ((sizeof(R) * N) % 16 == 0) {
        constexpr int Q = static_cast<int>(sizeof(R) * N / 16);
        const uint4 *src = reinterpret_cast<const uint4 *>(v);
        uint4 *dst = reinterpret_cast<uint4 *>(p);
        // streaming stores: the output is written once and not read back here
#pragma unroll
        for (int q = 0; q < Q; ++q) __stcs(dst + q, src[q]);
    } else {
#pragma unroll
        for (int q = 0; q < N; ++q) p[q] = v[q];
    }
}

// ---------------------------------------------------------------------------
// Output functors: how words become outputs.
//   RawOut<W>        one word -> itself
//   U01Out<R,W>      one word -> U01 variant
//   Canon2Out        two u32 words -> canonical double
//   ExpOut<R,W>      one word -> log(U01OC) * (-1/lambda)
// ---------------------------------------------------------------------------
template <typename W>
struct RawOut {
    using out_t = W;
    static constexpr int kIn = 1;
    static constexpr bool kCheap = true;
    __device__ W operator()(const W *w) const { return w[0]; }
};

template <typename R, typename W>
struct U01Out {
    using out_t = R;
    static constexpr int kIn = 1;
    static constexpr bool kCheap = true;
    int variant;
    __device__ R operator()(const W *w) const { return RealOps<R>::u01(variant, w[0]); }
};

struct Canon2Out {
    using out_t = double;
    static constexpr int kIn = 2;
    static constexpr bool kCheap = true;
    __device__ double operator()(const uint32_t *w) const { return u01_canonical2(w[0], w[1]); }
};

template <typename R, typename W>
struct ExpOut {
    using out_t = R;
    static constexpr int kIn = 1;
    static constexpr bool kCheap = false;
    R a;  // -1 / lambda, rounded in R as the reference does
    __device__ R operator()(const W *w) const
    {
        const R u = RealOps<R>::u01(kOC, w[0]);
        return RealOps<R>::mul(a, RealOps<R>::log(u));
    }
};

// Outputs of 32 bytes per block, lane l of a warp holding block bw + l: each
// lane writing its own 32 bytes makes every 128-bit store instruction cover
// half of each sector it touches.  Instead instruction k writes chunk 32k + l
// of the warp's 1 KiB (half l % 2 of block 16k + l / 2, fetched by shuffles),
// so each store is contiguous across the warp.  Returns false, storing
// nothing, unless all 32 blocks of the warp exist (then every lane is here).
template <typename R, int N>
__device__ __forceinline__ bool store_warp32(R *out, uint64_t b, uint64_t nblk, const R (&v)[N])
{
    static_assert(sizeof(R) * N == 32, "32-byte blocks only");
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t bw = b - lane;  // block of lane 0
    if (bw + 31 >= nblk) return false;
    const uint4 c0 = reinterpret_cast<const uint4 *>(v)[0], c1 = reinterpret_cast<const uint4 *>(v)[1];
    uint4 *dst = reinterpret_cast<uint4 *>(out + bw * N);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int src = 16 * k + static_cast<int>(lane >> 1);
        uint4 a, h;
        a.x = __shfl_sync(0xffffffffu, c0.x, src);
        a.y = __shfl_sync(0xffffffffu, c0.y, src);
        a.z = __shfl_sync(0xffffffffu, c0.z, src);
        a.w = __shfl_sync(0xffffffffu, c0.w, src);
        h.x = __shfl_sync(0xffffffffu, c1.x, src);
        h.y = __shfl_sync(0xffffffffu, c1.y, src);
        h.z = __shfl_sync(0xffffffffu, c1.z, src);
        h.w = __shfl_sync(0xffffffffu, c1.w, src);
        __stcs(dst + 32 * k + lane, (lane & 1) ? h : a);
    }
    return true;
}

// Aligned shape: nblk whole blocks starting at counter `base`; block b feeds
// outputs [b * OPB, (b + 1) * OPB).  `out` is 16-byte aligned.
template <class G, typename W, class F, int THREADS = 256>
__global__ void __launch_bounds__(THREADS) k_blocks(G g, Ctr base, uint64_t nblk, typename F::out_t *out, F f)
{
    using R = typename F::out_t;
    constexpr int WPB = G::kWords / WordView<W>::kPer32;  // words per block
    constexpr int OPB = WPB / F::kIn;                     // outputs per block
    g.prepare();
    // four blocks per thread and iteration, a grid stride apart (each store
    // instruction stays coalesced across the warp): independent work to
    // overlap with the stores in flight; one for the transforms whose
    // per-value math (double-double log) needs the registers
    constexpr int U = F::kCheap ? 4 : 1;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t b0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b0 < nblk; b0 += U * stride) {
#pragma unroll
        for (int i = 0; i < U; ++i) {
            const uint64_t b = b0 + i * stride;
            if (b >= nblk) break;
            uint32_t blk[G::kWords];
            g.block(ctr_add(base, b, G::kCtrWords), blk);
            W w[WPB];
#pragma unroll
            for (int j = 0; j < WPB; ++j) w[j] = WordView<W>::get(blk, j);
            R o[OPB];
#pragma unroll
            for (int j = 0; j < OPB; ++j) o[j] = f(w + j * F::kIn);
            // the shuffles pay only where the store, not the generator or the
            // transform, is the limit (Philox with a cheap transform)
            if constexpr (sizeof(R) * OPB == 32 && F::kCheap && std::is_same<G, PhiloxGen>::value) {
                if (store_warp32<R, OPB>(out, b, nblk, o)) continue;
            }
            store_aligned<R, OPB>(out + b * OPB, o);
        }
    }
}

// k_blocks for Philox launches whose block counters differ only in their low
// word (PhiloxLo: the counter-independent products folded once per launch).
template <typename W, class F>
__global__ void __launch_bounds__(256) k_blocks_plo(PhiloxLo p, uint64_t nblk, typename F::out_t *out, F f)
{
    using R = typename F::out_t;
    constexpr int WPB = PhiloxGen::kWords / WordView<W>::kPer32;
    constexpr int OPB = WPB / F::kIn;
    constexpr int U = F::kCheap ? 4 : 1;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t b0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b0 < nblk; b0 += U * stride) {
#pragma unroll
        for (int i = 0; i < U; ++i) {
            const uint64_t b = b0 + i * stride;
            if (b >= nblk) break;
            uint32_t blk[PhiloxGen::kWords];
            p.block(static_cast<uint32_t>(b), blk);
            W w[WPB];
#pragma unroll
            for (int j = 0; j < WPB; ++j) w[j] = WordView<W>::get(blk, j);
            R o[OPB];
#pragma unroll
            for (int j = 0; j < OPB; ++j) o[j] = f(w + j * F::kIn);
            if constexpr (sizeof(R) * OPB == 32 && F::kCheap) {
                if (store_warp32<R, OPB>(out, b, nblk, o)) continue;
            }
            store_aligned<R, OPB>(out + b * OPB, o);
        }
    }
}

// Staged shape: outputs [0, n) consume stream words off + kIn * [0, n) counted
// from word 0 of block `base`.  A CTA stages TB blocks per tile.
template <class G, typename W, class F, int TB>
__global__ void __launch_bounds__(256) k_staged(G g, Ctr base, uint32_t off, uint64_t n, typename F::out_t *out, F f)
{
    constexpr int WPB = G::kWords / WordView<W>::kPer32;
    constexpr int TW = TB * WPB;  // words per tile
    __shared__ __align__(16) uint32_t st32[TB * G::kWords];
    W *st = reinterpret_cast<W *>(st32);
    g.prepare();
    const uint64_t total = static_cast<uint64_t>(off) + n * F::kIn;  // stream words touched, from block start
    const uint64_t ntiles = (total + TW - 1) / TW;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint64_t w0 = t * TW;
        for (int i = threadIdx.x; i < TB; i += blockDim.x) {
            if (w0 + static_cast<uint64_t>(i) * WPB < total) {
                uint32_t blk[G::kWords];
                g.block(ctr_add(base, t * TB + i, G::kCtrWords), blk);
                stage_block<G>(st32, i, blk);
            }
        }
        __syncthreads();
        // outputs whose first word lies in this tile; a 2-word output may
        // straddle into the next tile, which the last thread recomputes.
        for (int j = threadIdx.x; j < TW; j += blockDim.x) {
            const uint64_t s = w0 + j;  // stream word
            if (s < off || s >= total) continue;
            const uint64_t rel = s - off;
            if (rel % F::kIn != 0) continue;
            W w[F::kIn];
            bool ok = true;
#pragma unroll
            for (int q = 0; q < F::kIn; ++q) {
                if (j + q < TW) {
                    w[q] = st[j + q];
                } else {
                    ok = false;
                }
            }
            if (!ok) {
                // word j + 1 is in the next block: generate it directly
                const uint64_t s1 = s + 1;
                uint32_t blk[G::kWords];
                g.block(ctr_add(base, s1 / WPB, G::kCtrWords), blk);
                w[1] = WordView<W>::get(blk, static_cast<int>(s1 % WPB));
            }
            out[rel / F::kIn] = f(w);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Normal: one CTA per 8192-byte chunk.  Chunk c uses stream words
// [c K, c K + K) (relative to the call's first word); word i < K/2 is the
// radius uniform and word K/2 + i the angle uniform of output pair
// (c K + i, c K + K/2 + i).
// ---------------------------------------------------------------------------
template <class G, typename W, typename R, int K>
__global__ void __launch_bounds__(256) k_normal(G g, Ctr base, uint32_t off, uint64_t first_chunk,
    uint64_t nchunks, uint32_t len, R *out, R mean, R sd)
{
    using O = RealOps<R>;
    constexpr int WPB = G::kWords / WordView<W>::kPer32;
    constexpr int NB = K / WPB + 1;  // blocks staged per chunk (one extra for misalignment)
    __shared__ __align__(16) uint32_t st32[NB * G::kWords];
    const W *st = reinterpret_cast<const W *>(st32);
    g.prepare();
    const uint32_t nu = len / 2;
    for (uint64_t cc = blockIdx.x; cc < nchunks; cc += gridDim.x) {
        const uint64_t c = first_chunk + cc;
        const uint64_t a0 = static_cast<uint64_t>(off) + c * K;  // absolute word of the chunk start
        const uint64_t b0 = a0 / WPB;
        const uint32_t s0 = static_cast<uint32_t>(a0 % WPB);
        const int nb = static_cast<int>((s0 + len + WPB - 1) / WPB);
        for (int i = threadIdx.x; i < nb; i += blockDim.x) {
            uint32_t blk[G::kWords];
            g.block(ctr_add(base, b0 + i, G::kCtrWords), blk);
            stage_block<G>(st32, i, blk);
        }
        __syncthreads();
        R *o = out + c * K;
        for (uint32_t p = threadIdx.x; p < nu; p += blockDim.x) {
            const R u1 = O::u01(kOC, st[s0 + p]);
            const R u2 = O::u01(kOC, st[s0 + nu + p]);
            R s = O::sqrt(O::mul(static_cast<R>(-2), O::log(u1)));
            R sn, cs;
            O::sincos(O::mul(O::kTwoPi, u2), &sn, &cs);
            if (sd != static_cast<R>(1)) s = O::mul(sd, s);
            if (mean != static_cast<R>(0)) {
                o[p] = O::fma(s, sn, mean);
                o[nu + p] = O::fma(s, cs, mean);
            } else {
                o[p] = O::mul(s, sn);
                o[nu + p] = O::mul(s, cs);
            }
        }
        if ((len & 1u) && threadIdx.x == 0) {
            o[len - 1] = O::u01(kOC, st[s0 + len - 1]);  // raw U01OC, as the reference leaves it
        }
        __syncthreads();
    }
}

// odd-n fix-up: r[n-1] = mean + (sd * sqrt(-2 log u)) * cos(2 pi v), u and v the
// two words after the last chunk (random/normal_distribution.hpp:93-100)
template <class G, typename W, typename R>
__global__ void k_normal_odd(G g, Ctr base, uint64_t a_u, R *dst, R mean, R sd)
{
    using O = RealOps<R>;
    constexpr int WPB = G::kWords / WordView<W>::kPer32;
    g.prepare();
    if (threadIdx.x != 0) return;
    W wv[2];
    for (int q = 0; q < 2; ++q) {
        const uint64_t a = a_u + q;
        uint32_t blk[G::kWords];
        g.block(ctr_add(base, a / WPB, G::kCtrWords), blk);
        wv[q] = WordView<W>::get(blk, static_cast<int>(a % WPB));
    }
    const R u = O::u01(kOC, wv[0]);
    const R v = O::u01(kOC, wv[1]);
    const R a = O::sqrt(O::mul(static_cast<R>(-2), O::log(u)));
    const R b = O::mul(sd, a);
    const R c = O::cos(O::mul(O::kTwoPi, v));
    *dst = O::add(mean, O::mul(b, c));
}

// ---------------------------------------------------------------------------
// host dispatch
// ---------------------------------------------------------------------------
// Launch the word -> output transform F for n outputs from position (B, off).
template <class G, typename W, class F>
static int launch_words(const G &g, const Ctr &B, uint32_t off, uint64_t n, typename F::out_t *out,
    const F &f, cudaStream_t s)
{
    if (n == 0) return MCKL_B200_OK;
    constexpr int WPB = G::kWords / WordView<W>::kPer32;
    constexpr int OPB = WPB / F::kIn;
    const bool aligned = (off == 0) && (reinterpret_cast<uintptr_t>(out) % 16 == 0);
    // ARS: 32 KiB of table per CTA bounds residency at 6 CTAs per SM
    const int ctas = std::is_same<G, ArsGen>::value ? 6 : 8;
    if (aligned) {
        const uint64_t nblk = n / OPB;
        bool done_blocks = false;
        if constexpr (std::is_same<G, PhiloxGen>::value) {
            // no carry out of the low counter word within this launch
            if (nblk && (B.w[0] & 0xffffffffull) + (nblk - 1) <= 0xffffffffull) {
                k_blocks_plo<W, F><<<grid_for(nblk, 256, ctas), 256, 0, s>>>(PhiloxLo::make(g, B), nblk, out, f);
                MB_LAUNCH_CHECK();
                done_blocks = true;
            }
        }
        if constexpr (std::is_same<G, ArsGen>::value) {
            // ARS with four round tables: one 1024-thread CTA per SM
            if (nblk) {
                MB_CUDA(allow_dyn_smem(k_blocks<ArsGen4, W, F, 1024>, ArsGen4::kDynSmem));
                k_blocks<ArsGen4, W, F, 1024><<<grid_for(nblk, 1024, 1), 1024, ArsGen4::kDynSmem, s>>>(
                    ArsGen4::from(g), B, nblk, out, f);
                MB_LAUNCH_CHECK();
                done_blocks = true;
            }
        }
        if (nblk && !done_blocks) {
            MB_CUDA(allow_dyn_smem(k_blocks<G, W, F>, G::kDynSmem));
            k_blocks<G, W, F><<<grid_for(nblk, 256, ctas), 256, G::kDynSmem, s>>>(g, B, nblk, out, f);
            MB_LAUNCH_CHECK();
        }
        const uint64_t done = nblk * OPB;
        if (done < n) {
            const Ctr B2 = ctr_add(B, nblk, G::kCtrWords);
            MB_CUDA(allow_dyn_smem(k_staged<G, W, F, 256>, G::kDynSmem));
            k_staged<G, W, F, 256><<<1, 256, G::kDynSmem, s>>>(g, B2, 0, n - done, out + done, f);
            MB_LAUNCH_CHECK();
        }
        return MCKL_B200_OK;
    }
    const uint64_t tiles = (static_cast<uint64_t>(off) + n * F::kIn + 256 * WPB - 1) / (256 * WPB);
    MB_CUDA(allow_dyn_smem(k_staged<G, W, F, 256>, G::kDynSmem));
    k_staged<G, W, F, 256><<<grid_for(tiles * 256, 256, ctas), 256, G::kDynSmem, s>>>(g, B, off, n, out, f);
    MB_LAUNCH_CHECK();
    return MCKL_B200_OK;
}

static bool is64(uint32_t kind)
{
    return geom(kind).rbytes == 8;
}

// Engine calls made by the reference's BATCH_0 / BATCH_1 chunking
// (random/internal/common.hpp:89-122): n / K calls of K words (each followed
// by an empty call), then one call of n % K words.
static void advance_chunked(mckl_b200_engine_t &e, uint64_t n, uint64_t K, uint64_t words_per_out)
{
    advance_calls(e, n / K, K * words_per_out);
    advance_call(e, (n % K) * words_per_out);
}

template <typename R>
static int u01_impl(mckl_b200_engine_t *e, int variant, size_t n, R *r, void *stream)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    Ctr B;
    uint32_t off;
    next_position(*e, B, off);
    cudaStream_t s = as_stream(stream);
    const bool canon2 = std::is_same<R, double>::value && variant == kCanonical && !is64(e->kind);
    int rc = with_generator(*e, [&](auto g) {
        using G = decltype(g);
        if (canon2) {
            return launch_words<G, uint32_t>(g, B, off, n, reinterpret_cast<double *>(r), Canon2Out{}, s);
        }
        if (is64(e->kind)) {
            return launch_words<G, uint64_t>(g, B, off, n, r, U01Out<R, uint64_t>{variant}, s);
        }
        return launch_words<G, uint32_t>(g, B, off, n, r, U01Out<R, uint32_t>{variant}, s);
    });
    if (rc != MCKL_B200_OK) return rc;
    advance_chunked(*e, n, 8192 / sizeof(R), canon2 ? 2 : 1);
    return MCKL_B200_OK;
}

template <typename R>
static int exponential_impl(mckl_b200_engine_t *e, size_t n, R *r, R lambda, void *stream)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    MB_CHECK_ARG(lambda > 0, "lambda must be positive");
    Ctr B;
    uint32_t off;
    next_position(*e, B, off);
    cudaStream_t s = as_stream(stream);
    const R a = static_cast<R>(-1) / lambda;
    int rc = with_generator(*e, [&](auto g) {
        using G = decltype(g);
        if (is64(e->kind)) return launch_words<G, uint64_t>(g, B, off, n, r, ExpOut<R, uint64_t>{a}, s);
        return launch_words<G, uint32_t>(g, B, off, n, r, ExpOut<R, uint32_t>{a}, s);
    });
    if (rc != MCKL_B200_OK) return rc;
    advance_chunked(*e, n, 8192 / sizeof(R), 1);
    return MCKL_B200_OK;
}

template <typename R>
static int normal_impl(mckl_b200_engine_t *e, size_t n, R *r, R mean, R sd, void *stream)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    MB_CHECK_ARG(sd > 0, "stddev must be positive");
    constexpr uint64_t K = 8192 / sizeof(R);
    Ctr B;
    uint32_t off;
    next_position(*e, B, off);
    cudaStream_t s = as_stream(stream);
    const uint64_t m = n / K, l = n % K;
    int rc = with_generator(*e, [&](auto g) {
        using G = decltype(g);
        auto run = [&](auto wtag) {
            using W = decltype(wtag);
            MB_CUDA(allow_dyn_smem(k_normal<G, W, R, K>, G::kDynSmem));
            if (m) {
                k_normal<G, W, R, K><<<grid_for(m * 256, 256, 8), 256, G::kDynSmem, s>>>(g, B, off, 0, m, K, r,
                    mean, sd);
                MB_LAUNCH_CHECK();
            }
            if (l) {
                k_normal<G, W, R, K><<<1, 256, G::kDynSmem, s>>>(g, B, off, m, 1, static_cast<uint32_t>(l), r,
                    mean, sd);
                MB_LAUNCH_CHECK();
            }
            if (n % 2) {
                MB_CUDA(allow_dyn_smem(k_normal_odd<G, W, R>, G::kDynSmem));
                k_normal_odd<G, W, R><<<1, 32, G::kDynSmem, s>>>(g, B, static_cast<uint64_t>(off) + n, r + n - 1,
                    mean, sd);
                MB_LAUNCH_CHECK();
            }
            return MCKL_B200_OK;
        };
        if (is64(e->kind)) return run(uint64_t{});
        return run(uint32_t{});
    });
    if (rc != MCKL_B200_OK) return rc;
    // engine calls: per chunk u01_oc(K) -> [K][0]; then u01_oc(l) -> [l];
    // odd n: two single-word draws
    advance_calls(*e, m, K);
    advance_call(*e, l);
    if (n % 2) {
        advance_call(*e, 1);
        advance_call(*e, 1);
    }
    return MCKL_B200_OK;
}

}  // namespace mckl_b200

using namespace mckl_b200;

extern "C" {

const char *mckl_b200_last_error(void)
{
    return g_last_error.c_str();
}

uint64_t mckl_b200_launch_count(void)
{
    return g_launches.load(std::memory_order_relaxed);
}

const char *mckl_b200_version(void)
{
    return "mckl_b200 0.2 (sm_100a)";
}

int mckl_b200_release_stream(void *stream)
{
    return scratch_release(as_stream(stream));
}

int mckl_b200_engine_seed(mckl_b200_engine_t *e, uint32_t kind, uint64_t seed)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(kind), "invalid engine kind");
    std::memset(e, 0, sizeof(*e));
    e->kind = kind;
    const bool k32 = (kind != MCKL_B200_THREEFRY4X64 && kind != MCKL_B200_THREEFRY4X64_64);
    e->key[0] = k32 ? (seed & 0xFFFFFFFFull) : seed;
    e->index = static_cast<uint32_t>(geom(kind).M);
    return MCKL_B200_OK;
}

int mckl_b200_engine_discard(mckl_b200_engine_t *e, uint64_t nskip)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    const Geom g = geom(e->kind);
    const uint64_t M = static_cast<uint64_t>(g.M);
    if (nskip == 0) return MCKL_B200_OK;
    const uint64_t idx = e->index < M ? e->index : M;
    const uint64_t remain = M - idx;
    if (nskip <= remain) {
        e->index = static_cast<uint32_t>(idx + nskip);
        return MCKL_B200_OK;
    }
    nskip -= remain;
    // increment(ctr, nskip / M * rate) with rate = 1 (result block == counter
    // size), including the reference's carry when ctr[0] == max - k
    // (random/internal/increment_generic.hpp:209-217), then one generated block.
    const uint64_t k = nskip / M;
    Ctr c = ctr_of(*e);
    if (c.w[0] < UINT64_MAX - k) {
        c.w[0] += k;
    } else {
        c.w[0] += k;
        for (int i = 1; i < g.cwords; ++i) {
            if (++c.w[i] != 0) break;
        }
    }
    c = ctr_add(c, 1, g.cwords);
    set_ctr(*e, c);
    e->index = static_cast<uint32_t>(nskip % M);
    return MCKL_B200_OK;
}

int mckl_b200_rand(mckl_b200_engine_t *e, size_t n, void *r, void *stream)
{
    MB_CHECK_ARG(e != nullptr, "null engine");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    Ctr B;
    uint32_t off;
    next_position(*e, B, off);
    cudaStream_t s = as_stream(stream);
    int rc = with_generator(*e, [&](auto g) {
        using G = decltype(g);
        if (is64(e->kind)) {
            return launch_words<G, uint64_t>(g, B, off, n, static_cast<uint64_t *>(r), RawOut<uint64_t>{}, s);
        }
        return launch_words<G, uint32_t>(g, B, off, n, static_cast<uint32_t *>(r), RawOut<uint32_t>{}, s);
    });
    if (rc != MCKL_B200_OK) return rc;
    advance_call(*e, n);
    return MCKL_B200_OK;
}

int mckl_b200_philox4x32_kernel(uint64_t ctr[2], size_t n, void *r, const uint32_t key[2], void *stream)
{
    MB_CHECK_ARG(ctr != nullptr && key != nullptr, "null ctr/key");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    Ctr B{{ctr[0], ctr[1], 0, 0}};
    B = ctr_add(B, 1, 2);
    PhiloxGen g{key[0], key[1]};
    int rc = launch_words<PhiloxGen, uint32_t>(g, B, 0, n * 4, static_cast<uint32_t *>(r), RawOut<uint32_t>{},
        as_stream(stream));
    if (rc != MCKL_B200_OK) return rc;
    Ctr E = ctr_add(Ctr{{ctr[0], ctr[1], 0, 0}}, n, 2);
    ctr[0] = E.w[0];
    ctr[1] = E.w[1];
    return MCKL_B200_OK;
}

int mckl_b200_threefry4x64_kernel(uint64_t ctr[4], size_t n, void *r, const uint64_t key[4],
    const uint64_t tweak[2], void *stream)
{
    MB_CHECK_ARG(ctr != nullptr && key != nullptr, "null ctr/key");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    const uint64_t zero[2] = {0, 0};
    ThreefryGen g = ThreefryGen::make(key, tweak ? tweak : zero);
    Ctr C{{ctr[0], ctr[1], ctr[2], ctr[3]}};
    int rc = launch_words<ThreefryGen, uint32_t>(g, ctr_add(C, 1, 4), 0, n * 8, static_cast<uint32_t *>(r),
        RawOut<uint32_t>{}, as_stream(stream));
    if (rc != MCKL_B200_OK) return rc;
    Ctr E = ctr_add(C, n, 4);
    for (int i = 0; i < 4; ++i) ctr[i] = E.w[i];
    return MCKL_B200_OK;
}

int mckl_b200_ars_kernel(uint64_t ctr[2], size_t n, void *r, const uint32_t key[4], void *stream)
{
    MB_CHECK_ARG(ctr != nullptr && key != nullptr, "null ctr/key");
    MB_CHECK_ARG(n == 0 || r != nullptr, "null output");
    const uint64_t k64[4] = {key[0], key[1], key[2], key[3]};
    ArsGen g = ArsGen::make(k64);
    Ctr C{{ctr[0], ctr[1], 0, 0}};
    int rc = launch_words<ArsGen, uint32_t>(g, ctr_add(C, 1, 2), 0, n * 4, static_cast<uint32_t *>(r),
        RawOut<uint32_t>{}, as_stream(stream));
    if (rc != MCKL_B200_OK) return rc;
    Ctr E = ctr_add(C, n, 2);
    ctr[0] = E.w[0];
    ctr[1] = E.w[1];
    return MCKL_B200_OK;
}

#define MB_U01(name, variant)                                                                      \
    int mckl_b200_u01_##name##_f32(mckl_b200_engine_t *e, size_t n, float *r, void *stream)          \
    {                                                                                              \
        return u01_impl<float>(e, variant, n, r, stream);                                          \
    }                                                                                              \
    int mckl_b200_u01_##name##_f64(mckl_b200_engine_t *e, size_t n, double *r, void *stream)         \
    {                                                                                              \
        return u01_impl<double>(e, variant, n, r, stream);                                         \
    }

MB_U01(canonical, kCanonical)
MB_U01(cc, kCC)
MB_U01(co, kCO)
MB_U01(oc, kOC)
MB_U01(oo, kOO)

int mckl_b200_normal_f32(mckl_b200_engine_t *e, size_t n, float *r, float mean, float sd, void *stream)
{
    return normal_impl<float>(e, n, r, mean, sd, stream);
}

int mckl_b200_normal_f64(mckl_b200_engine_t *e, size_t n, double *r, double mean, double sd, void *stream)
{
    return normal_impl<double>(e, n, r, mean, sd, stream);
}

int mckl_b200_exponential_f32(mckl_b200_engine_t *e, size_t n, float *r, float lambda, void *stream)
{
    return exponential_impl<float>(e, n, r, lambda, stream);
}

int mckl_b200_exponential_f64(mckl_b200_engine_t *e, size_t n, double *r, double lambda, void *stream)
{
    return exponential_impl<double>(e, n, r, lambda, stream);
}

}  // extern "C"
