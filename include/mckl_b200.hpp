// mckl_b200.hpp -- C++ host interface over the C ABI (mckl_b200.h), shaped
// like the reference's own classes so MCKL host code can use the B200 path
// with minimal change.  Header-only, C++14, no dependency besides the CUDA
// runtime (for device buffers) and libmckl_b200.so.
//
//  * Generators for mckl::CounterEngine<ResultType, Generator>
//    (random/counter.hpp:47-61): PhiloxGenerator4x32 / Threefry4x64Generator /
//    ARSGenerator have ctr_type, key_type, size(), key(), reset(key) and
//    operator()(ctr, r) / operator()(ctr, n, r).  `mckl::CounterEngine<
//    std::uint32_t, mckl_b200::PhiloxGenerator4x32>` is then a drop-in for
//    mckl::Philox4x32 whose bulk fills run on the GPU; it works with every
//    reference distribution.  Buffers may be host or device memory.
//  * Engine<Kind, ResultType>: device-resident batch API with the reference's
//    names (seed, key, ctr, discard, rand, u01_*_distribution,
//    normal_distribution, exponential_distribution) writing device memory.
//  * Weight, resampling functors and rep_to_index/select over device arrays
//    (core/weight.hpp, algorithm/resample.hpp), mirroring ResampleEval.
// Errors surface as mckl_b200::Error (the reference uses runtime_assert,
// internal/assert.hpp:49-100).
#ifndef MCKL_B200_HPP
#define MCKL_B200_HPP

#include <cuda_runtime_api.h>

#include <array>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mckl_b200.h"

namespace mckl_b200 {

class Error : public std::runtime_error {
  public:
    explicit Error(const std::string &m) : std::runtime_error(m) {}
};

inline void check(int rc)
{
    if (rc != MCKL_B200_OK) throw Error(std::string("mckl_b200: ") + mckl_b200_last_error());
}

inline void check_cuda(cudaError_t e)
{
    if (e != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e));
}

// RAII device buffer
template <typename T>
class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t n) { resize(n); }
    ~DeviceBuffer() { reset(); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    void resize(std::size_t n)
    {
        if (n <= cap_) {
            n_ = n;
            return;
        }
        reset();
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&p_), (n ? n : 1) * sizeof(T)));
        cap_ = n_ = n;
    }
    void reset()
    {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        cap_ = n_ = 0;
    }
    T *data() { return p_; }
    const T *data() const { return p_; }
    std::size_t size() const { return n_; }
    void upload(const T *h, std::size_t n)
    {
        resize(n);
        check_cuda(cudaMemcpy(p_, h, n * sizeof(T), cudaMemcpyHostToDevice));
    }
    void download(T *h, std::size_t n) const
    {
        check_cuda(cudaMemcpy(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost));
    }

  private:
    T *p_ = nullptr;
    std::size_t n_ = 0, cap_ = 0;
};

namespace detail {

// Is `p` directly addressable by the device (device or page-locked memory)?
inline bool device_addressable(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged ||
           (a.type == cudaMemoryTypeHost && a.devicePointer != nullptr);
}

// Run `fill(dst_device, bytes)` into `r`: directly when the device can write
// it, else through a staging buffer copied back to pageable host memory.
template <typename Fill>
void fill_any(void *r, std::size_t bytes, Fill &&fill)
{
    if (bytes == 0) return;
    if (device_addressable(r)) {
        check(fill(r));
        check_cuda(cudaStreamSynchronize(nullptr));
        return;
    }
    thread_local DeviceBuffer<unsigned char> stage;
    stage.resize(bytes);
    check(fill(stage.data()));
    check_cuda(cudaMemcpy(r, stage.data(), bytes, cudaMemcpyDeviceToHost));
}

// Host single-block versions of the three generators, for the reference's
// one-block buffer refills (CounterEngine::operator()(), random/counter.hpp:
// 132-140) and short fills, where a device round trip would cost far more
// than the arithmetic.  Same functions as csrc/engines.cuh.
inline void philox_block_host(std::uint64_t c0, std::uint64_t c1, const std::uint32_t *key, std::uint32_t *out)
{
    std::uint32_t s0 = static_cast<std::uint32_t>(c0), s1 = static_cast<std::uint32_t>(c0 >> 32);
    std::uint32_t s2 = static_cast<std::uint32_t>(c1), s3 = static_cast<std::uint32_t>(c1 >> 32);
    std::uint32_t a = key[0], b = key[1];
    for (int r = 0; r < 10; ++r) {
        const std::uint64_t p2 = static_cast<std::uint64_t>(s2) * 0xCD9E8D57u;
        const std::uint64_t p0 = static_cast<std::uint64_t>(s0) * 0xD2511F53u;
        const std::uint32_t n0 = a ^ s1 ^ static_cast<std::uint32_t>(p2 >> 32);
        const std::uint32_t n2 = b ^ s3 ^ static_cast<std::uint32_t>(p0 >> 32);
        s1 = static_cast<std::uint32_t>(p2);
        s3 = static_cast<std::uint32_t>(p0);
        s0 = n0;
        s2 = n2;
        a += 0x9E3779B9u;
        b += 0xBB67AE85u;
    }
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
    out[3] = s3;
}

inline void threefry_block_host(const std::uint64_t *c, const std::uint64_t *key, const std::uint64_t *tweak,
    std::uint64_t *out)
{
    static const int R0[8] = {14, 52, 23, 5, 25, 46, 58, 32}, R1[8] = {16, 57, 40, 37, 33, 12, 22, 32};
    std::uint64_t par[8] = {key[0], key[1], key[2], key[3],
        0x1BD11BDAA9FC1A22ull ^ key[0] ^ key[1] ^ key[2] ^ key[3], tweak[0], tweak[1], tweak[0] ^ tweak[1]};
    std::uint64_t s[4] = {c[0], c[1], c[2], c[3]};
    auto rotl = [](std::uint64_t x, int r) { return (x << r) | (x >> (64 - r)); };
    for (int N = 0; N <= 20; ++N) {
        if (N > 0) {
            s[0] += s[1];
            s[2] += s[3];
            const std::uint64_t t1 = rotl(s[1], R0[(N - 1) % 8]), t3 = rotl(s[3], R1[(N - 1) % 8]);
            s[1] = s[2] ^ t3;
            s[3] = s[0] ^ t1;
        }
        if (N % 4 == 0) {
            const std::uint64_t S = static_cast<std::uint64_t>(N / 4);
            s[0] += par[S % 5];
            s[1] += par[(S + 1) % 5] + par[5 + S % 3];
            s[2] += par[(S + 2) % 5] + par[5 + (S + 1) % 3];
            s[3] += par[(S + 3) % 5] + S;
        }
    }
    std::memcpy(out, s, sizeof(s));
}

inline std::uint8_t gf_mul_host(std::uint8_t a, std::uint8_t b)
{
    std::uint8_t p = 0;
    for (int i = 0; i < 8; ++i) {
        if (b & 1) p ^= a;
        a = static_cast<std::uint8_t>((a << 1) ^ ((a & 0x80) ? 0x1B : 0));
        b >>= 1;
    }
    return p;
}

inline const std::uint8_t *aes_sbox_host()
{
    static std::uint8_t sb[256];
    static bool ready = false;
    if (!ready) {
        for (int x = 0; x < 256; ++x) {
            std::uint8_t inv = 0;
            for (int y = 1; x && y < 256; ++y) {
                if (gf_mul_host(static_cast<std::uint8_t>(x), static_cast<std::uint8_t>(y)) == 1) {
                    inv = static_cast<std::uint8_t>(y);
                    break;
                }
            }
            std::uint8_t b = inv, t = inv;
            for (int i = 0; i < 4; ++i) {
                b = static_cast<std::uint8_t>((b << 1) | (b >> 7));
                t ^= b;
            }
            sb[x] = static_cast<std::uint8_t>(t ^ 0x63);
        }
        ready = true;
    }
    return sb;
}

// ARS-5: the FIPS-197 round (SubBytes, ShiftRows, MixColumns, AddRoundKey) on
// little-endian column words, round keys as Weyl increments of the key halves
inline void ars_block_host(std::uint64_t c0, std::uint64_t c1, const std::uint32_t *key, std::uint32_t *out)
{
    const std::uint8_t *sb = aes_sbox_host();
    const std::uint64_t klo = key[0] | (static_cast<std::uint64_t>(key[1]) << 32);
    const std::uint64_t khi = key[2] | (static_cast<std::uint64_t>(key[3]) << 32);
    std::uint8_t st[16];
    std::memcpy(st, &c0, 8);
    std::memcpy(st + 8, &c1, 8);
    for (int n = 0; n <= 5; ++n) {
        if (n > 0) {
            std::uint8_t t[16];
            for (int c = 0; c < 4; ++c)
                for (int r = 0; r < 4; ++r) t[4 * c + r] = sb[st[4 * ((c + r) & 3) + r]];  // SubBytes + ShiftRows
            if (n < 5) {
                for (int c = 0; c < 4; ++c) {  // MixColumns
                    const std::uint8_t a0 = t[4 * c], a1 = t[4 * c + 1], a2 = t[4 * c + 2], a3 = t[4 * c + 3];
                    t[4 * c] = gf_mul_host(a0, 2) ^ gf_mul_host(a1, 3) ^ a2 ^ a3;
                    t[4 * c + 1] = a0 ^ gf_mul_host(a1, 2) ^ gf_mul_host(a2, 3) ^ a3;
                    t[4 * c + 2] = a0 ^ a1 ^ gf_mul_host(a2, 2) ^ gf_mul_host(a3, 3);
                    t[4 * c + 3] = gf_mul_host(a0, 3) ^ a1 ^ a2 ^ gf_mul_host(a3, 2);
                }
            }
            std::memcpy(st, t, 16);
        }
        const std::uint64_t k0 = klo + 0x9E3779B97F4A7C15ull * static_cast<std::uint64_t>(n);
        const std::uint64_t k1 = khi + 0xBB67AE8584CAA73Bull * static_cast<std::uint64_t>(n);
        std::uint8_t kb[16];
        std::memcpy(kb, &k0, 8);
        std::memcpy(kb + 8, &k1, 8);
        for (int i = 0; i < 16; ++i) st[i] ^= kb[i];
    }
    std::memcpy(out, st, 16);
}

inline void ctr_inc(std::uint64_t *c, int n)
{
    for (int i = 0; i < n; ++i)
        if (++c[i] != 0) return;
}

// Below this many blocks a fill is computed on the host.
constexpr std::size_t kHostBlocks = 4096;

}  // namespace detail

// ---------------------------------------------------------------------------
// Generators for mckl::CounterEngine (random/counter.hpp:47-61).  Counter and
// key types are the reference's: Counter<u32,4> = std::array<u64,2>,
// Counter<u64,4> = std::array<u64,4>.
// ---------------------------------------------------------------------------
class PhiloxGenerator4x32 {
  public:
    using ctr_type = std::array<std::uint64_t, 2>;
    using key_type = std::array<std::uint32_t, 2>;
    static constexpr std::size_t size() { return 16; }
    key_type key() const { return key_; }
    void reset(const key_type &k) { key_ = k; }
    template <typename R>
    void operator()(ctr_type &ctr, R *r) const { operator()(ctr, 1, r); }
    template <typename R>
    void operator()(ctr_type &ctr, std::size_t n, R *r) const
    {
        std::uint64_t c[2] = {ctr[0], ctr[1]};
        if (n < detail::kHostBlocks && !detail::device_addressable(r)) {
            unsigned char *o = reinterpret_cast<unsigned char *>(r);
            for (std::size_t i = 0; i < n; ++i, o += 16) {
                detail::ctr_inc(c, 2);
                std::uint32_t w[4];
                detail::philox_block_host(c[0], c[1], key_.data(), w);
                std::memcpy(o, w, 16);
            }
        } else {
            detail::fill_any(r, n * size(), [&](void *dst) {
                return mckl_b200_philox4x32_kernel(c, n, dst, key_.data(), nullptr);
            });
        }
        ctr[0] = c[0];
        ctr[1] = c[1];
    }
    friend bool operator==(const PhiloxGenerator4x32 &a, const PhiloxGenerator4x32 &b) { return a.key_ == b.key_; }
    friend bool operator!=(const PhiloxGenerator4x32 &a, const PhiloxGenerator4x32 &b) { return !(a == b); }

  private:
    key_type key_{{0, 0}};
};

class Threefry4x64Generator {
  public:
    using ctr_type = std::array<std::uint64_t, 4>;
    using key_type = std::array<std::uint64_t, 4>;
    static constexpr std::size_t size() { return 32; }
    key_type key() const { return key_; }
    void reset(const key_type &k)
    {
        key_ = k;
        tweak_ = {{0, 0}};
    }
    void tweak(std::uint64_t t0, std::uint64_t t1) { tweak_ = {{t0, t1}}; }
    template <typename R>
    void operator()(ctr_type &ctr, R *r) const { operator()(ctr, 1, r); }
    template <typename R>
    void operator()(ctr_type &ctr, std::size_t n, R *r) const
    {
        if (n < detail::kHostBlocks && !detail::device_addressable(r)) {
            unsigned char *o = reinterpret_cast<unsigned char *>(r);
            for (std::size_t i = 0; i < n; ++i, o += 32) {
                detail::ctr_inc(ctr.data(), 4);
                std::uint64_t w[4];
                detail::threefry_block_host(ctr.data(), key_.data(), tweak_.data(), w);
                std::memcpy(o, w, 32);
            }
            return;
        }
        detail::fill_any(r, n * size(), [&](void *dst) {
            return mckl_b200_threefry4x64_kernel(ctr.data(), n, dst, key_.data(), tweak_.data(), nullptr);
        });
    }
    friend bool operator==(const Threefry4x64Generator &a, const Threefry4x64Generator &b)
    {
        return a.key_ == b.key_ && a.tweak_ == b.tweak_;
    }
    friend bool operator!=(const Threefry4x64Generator &a, const Threefry4x64Generator &b) { return !(a == b); }

  private:
    key_type key_{{0, 0, 0, 0}};
    std::array<std::uint64_t, 2> tweak_{{0, 0}};
};

class ARSGenerator {
  public:
    using ctr_type = std::array<std::uint64_t, 2>;
    using key_type = std::array<std::uint32_t, 4>;
    static constexpr std::size_t size() { return 16; }
    key_type key() const { return key_; }
    void reset(const key_type &k) { key_ = k; }
    template <typename R>
    void operator()(ctr_type &ctr, R *r) const { operator()(ctr, 1, r); }
    template <typename R>
    void operator()(ctr_type &ctr, std::size_t n, R *r) const
    {
        std::uint64_t c[2] = {ctr[0], ctr[1]};
        if (n < detail::kHostBlocks && !detail::device_addressable(r)) {
            unsigned char *o = reinterpret_cast<unsigned char *>(r);
            for (std::size_t i = 0; i < n; ++i, o += 16) {
                detail::ctr_inc(c, 2);
                std::uint32_t w[4];
                detail::ars_block_host(c[0], c[1], key_.data(), w);
                std::memcpy(o, w, 16);
            }
        } else {
            detail::fill_any(r, n * size(), [&](void *dst) {
                return mckl_b200_ars_kernel(c, n, dst, key_.data(), nullptr);
            });
        }
        ctr[0] = c[0];
        ctr[1] = c[1];
    }
    friend bool operator==(const ARSGenerator &a, const ARSGenerator &b) { return a.key_ == b.key_; }
    friend bool operator!=(const ARSGenerator &a, const ARSGenerator &b) { return !(a == b); }

  private:
    key_type key_{{0, 0, 0, 0}};
};

// ---------------------------------------------------------------------------
// Device-resident engines with the reference's batch API (device outputs).
// ---------------------------------------------------------------------------
template <std::uint32_t Kind, typename ResultType>
class Engine {
  public:
    using result_type = ResultType;
    explicit Engine(std::uint64_t s = 1) { seed(s); }
    void seed(std::uint64_t s) { check(mckl_b200_engine_seed(&st_, Kind, s)); }
    void key(const std::array<std::uint64_t, 4> &k)
    {
        for (int i = 0; i < 4; ++i) st_.key[i] = k[i];
        for (int i = 0; i < 4; ++i) st_.ctr[i] = 0;
        st_.index = 0xffffffffu;
    }
    void ctr(const std::array<std::uint64_t, 4> &c)
    {
        for (int i = 0; i < 4; ++i) st_.ctr[i] = c[i];
        st_.index = 0xffffffffu;
    }
    void discard(std::uint64_t n) { check(mckl_b200_engine_discard(&st_, n)); }
    mckl_b200_engine_t &state() { return st_; }
    const mckl_b200_engine_t &state() const { return st_; }

  private:
    mckl_b200_engine_t st_;
};

using Philox4x32 = Engine<MCKL_B200_PHILOX4X32, std::uint32_t>;
using Philox4x32_64 = Engine<MCKL_B200_PHILOX4X32_64, std::uint64_t>;
using Threefry4x64 = Engine<MCKL_B200_THREEFRY4X64, std::uint32_t>;
using Threefry4x64_64 = Engine<MCKL_B200_THREEFRY4X64_64, std::uint64_t>;
using ARS = Engine<MCKL_B200_ARS, std::uint32_t>;
using ARS_64 = Engine<MCKL_B200_ARS_64, std::uint64_t>;

// mckl::rand(rng, n, r) (random/counter.hpp:298-303), r on the device
template <std::uint32_t K, typename R>
void rand(Engine<K, R> &rng, std::size_t n, R *r_dev, cudaStream_t s = nullptr)
{
    check(mckl_b200_rand(&rng.state(), n, r_dev, s));
}

#define MCKL_B200_DEFINE_U01(name)                                                                      \
    template <std::uint32_t K, typename R>                                                              \
    void u01_##name##_distribution(Engine<K, R> &rng, std::size_t n, double *r, cudaStream_t s = nullptr) \
    {                                                                                                   \
        check(mckl_b200_u01_##name##_f64(&rng.state(), n, r, s));                                       \
    }                                                                                                   \
    template <std::uint32_t K, typename R>                                                              \
    void u01_##name##_distribution(Engine<K, R> &rng, std::size_t n, float *r, cudaStream_t s = nullptr) \
    {                                                                                                   \
        check(mckl_b200_u01_##name##_f32(&rng.state(), n, r, s));                                       \
    }
MCKL_B200_DEFINE_U01(canonical)
MCKL_B200_DEFINE_U01(cc)
MCKL_B200_DEFINE_U01(co)
MCKL_B200_DEFINE_U01(oc)
MCKL_B200_DEFINE_U01(oo)
#undef MCKL_B200_DEFINE_U01

// the reference's default U01Distribution is the canonical one (random/u01_distribution.hpp:213-235)
template <std::uint32_t K, typename R, typename T>
void u01_distribution(Engine<K, R> &rng, std::size_t n, T *r, cudaStream_t s = nullptr)
{
    u01_canonical_distribution(rng, n, r, s);
}

template <std::uint32_t K, typename R>
void normal_distribution(Engine<K, R> &rng, std::size_t n, double *r, double mean, double sd, cudaStream_t s = nullptr)
{
    check(mckl_b200_normal_f64(&rng.state(), n, r, mean, sd, s));
}

template <std::uint32_t K, typename R>
void normal_distribution(Engine<K, R> &rng, std::size_t n, float *r, float mean, float sd, cudaStream_t s = nullptr)
{
    check(mckl_b200_normal_f32(&rng.state(), n, r, mean, sd, s));
}

template <std::uint32_t K, typename R>
void exponential_distribution(Engine<K, R> &rng, std::size_t n, double *r, double lambda, cudaStream_t s = nullptr)
{
    check(mckl_b200_exponential_f64(&rng.state(), n, r, lambda, s));
}

template <std::uint32_t K, typename R>
void exponential_distribution(Engine<K, R> &rng, std::size_t n, float *r, float lambda, cudaStream_t s = nullptr)
{
    check(mckl_b200_exponential_f32(&rng.state(), n, r, lambda, s));
}

// ---------------------------------------------------------------------------
// SMC pieces over device arrays
// ---------------------------------------------------------------------------

// mckl::Weight (core/weight.hpp:44-228) with its data on the device
class Weight {
  public:
    explicit Weight(std::size_t N = 0) { resize(N); }
    std::size_t size() const { return data_.size(); }
    void resize(std::size_t N)
    {
        data_.resize(N);
        set_equal();
    }
    double ess() const { return ess_; }
    double log_nc() const { return log_nc_; }
    double *data() { return data_.data(); }
    const double *data() const { return data_.data(); }
    void set_equal()
    {
        std::vector<double> h(size(), 1.0 / static_cast<double>(size()));
        if (size()) data_.upload(h.data(), h.size());
        ess_ = static_cast<double>(size());
    }
    void set_log(const double *v_dev) { check(mckl_b200_weight_set_log(size(), data(), v_dev, &ess_, &log_nc_, nullptr)); }
    void add_log(const double *v_dev) { check(mckl_b200_weight_add_log(size(), data(), v_dev, &ess_, &log_nc_, nullptr)); }

  private:
    DeviceBuffer<double> data_;
    double ess_ = 0, log_nc_ = 0;
};

// ResampleAlgorithm functors (algorithm/resample.hpp:569-593):
// void(N, M, rng, W, rep) with W and rep on the device
template <int Scheme>
struct ResampleAlgorithm {
    template <std::uint32_t K, typename R>
    void operator()(std::size_t N, std::size_t M, Engine<K, R> &rng, const double *W_dev, std::uint64_t *rep_dev) const
    {
        check(mckl_b200_resample(Scheme, N, M, &rng.state(), W_dev, rep_dev, nullptr));
    }
};
using ResampleMultinomial = ResampleAlgorithm<0>;
using ResampleStratified = ResampleAlgorithm<1>;
using ResampleSystematic = ResampleAlgorithm<2>;
using ResampleResidual = ResampleAlgorithm<3>;
using ResampleResidualStratified = ResampleAlgorithm<4>;
using ResampleResidualSystematic = ResampleAlgorithm<5>;

// resample_trans_rep_index (algorithm/resample.hpp:416-466)
inline void resample_trans_rep_index(std::size_t N, std::size_t M, const std::uint64_t *rep_dev, std::uint64_t *idx_dev)
{
    check(mckl_b200_rep_to_index(N, M, rep_dev, idx_dev, nullptr));
}

// ResampleEval::operator() (algorithm/resample.hpp:494-507) for a column-major
// N x dim particle state on the device: counts, parent indices, select, equal weights
template <typename Algorithm, std::uint32_t K, typename R>
void resample(const Algorithm &alg, Engine<K, R> &rng, Weight &w, double *state_dev, std::size_t dim)
{
    const std::size_t N = w.size();
    DeviceBuffer<std::uint64_t> rep(N), idx(N);
    alg(N, N, rng, w.data(), rep.data());
    resample_trans_rep_index(N, N, rep.data(), idx.data());
    check(mckl_b200_select_f64(N, dim, idx.data(), state_dev, nullptr));
    w.set_equal();
}

}  // namespace mckl_b200

#endif  // MCKL_B200_HPP
