// engines.cuh -- sm_100a device implementations of MCKL's three counter-based
// generators.  Each generator maps one counter to one block of random words;
// no state is carried between blocks, so any thread can produce any block of
// any stream from (key, counter) alone.
//
//   Philox4x32-10   random/internal/philox_generic_4x.hpp:40-53,
//                   random/internal/philox_constants.hpp:51-56, 82-87
//   Threefry4x64-20 random/threefry.hpp:109-133,
//                   random/internal/threefry_common.hpp:212-247,
//                   random/internal/threefry_generic_4x64.hpp:40-79,
//                   random/internal/threefry_constants.hpp:51-56, 83-89
//   ARS-5           random/internal/aes_generic.hpp:254-306, 413-491,
//                   random/internal/aes_constants.hpp:289-304
//
// Block words are little-endian u32: a Philox/ARS block is 4 words, a
// Threefry4x64 block is 8 words (lo, hi of each 64-bit lane).  Engines with
// 64-bit results read the same bytes two words at a time.
#pragma once

#include <cstdint>

namespace mckl_b200 {

// 128/256-bit counters in the reference's Counter layout (random/increment.hpp:54-104).
struct Ctr {
    uint64_t w[4];
};

__host__ __device__ inline Ctr ctr_add(const Ctr &c, uint64_t k, int nwords)
{
    Ctr r = c;
    uint64_t s = r.w[0] + k;
    uint64_t carry = (s < r.w[0]) ? 1 : 0;
    r.w[0] = s;
    for (int i = 1; i < nwords && carry; ++i) {
        r.w[i] += 1;
        carry = (r.w[i] == 0) ? 1 : 0;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Philox4x32-10
// ---------------------------------------------------------------------------
struct PhiloxGen {
    static constexpr int kWords = 4;     // u32 words per block
    static constexpr int kCtrWords = 2;  // u64 counter words
    static constexpr int kDynSmem = 0;   // dynamic shared memory bytes per CTA
    uint32_t k0, k1;

    __device__ __forceinline__ void prepare() const {}

    __device__ __forceinline__ void block(const Ctr &c, uint32_t out[4]) const
    {
        uint32_t s0 = static_cast<uint32_t>(c.w[0]);
        uint32_t s1 = static_cast<uint32_t>(c.w[0] >> 32);
        uint32_t s2 = static_cast<uint32_t>(c.w[1]);
        uint32_t s3 = static_cast<uint32_t>(c.w[1] >> 32);
        uint32_t a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            const uint32_t hi2 = __umulhi(s2, 0xCD9E8D57u);
            const uint32_t lo2 = s2 * 0xCD9E8D57u;
            const uint32_t hi0 = __umulhi(s0, 0xD2511F53u);
            const uint32_t lo0 = s0 * 0xD2511F53u;
            s0 = a ^ s1 ^ hi2;
            s1 = lo2;
            s2 = b ^ s3 ^ hi0;
            s3 = lo0;
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        out[0] = s0;
        out[1] = s1;
        out[2] = s2;
        out[3] = s3;
    }
};

__host__ __device__ inline uint32_t mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) >> 32);
#endif
}

// Philox blocks of one launch whose counters differ only in the low 32-bit
// word s0 (s1, s2, s3 fixed): in the first round the product of s2 does not
// depend on the block, so neither do the first round's outputs s0' and s1',
// nor the second round's product of s0'.  Those are folded once per launch
// (make); a block then takes 36 of the 40 multiply halves.  The output is
// the same as PhiloxGen::block on the full counter.
struct PhiloxLo {
    uint32_t lo;            // s0 of block 0 of the launch
    uint32_t k1s3;          // k1 ^ s3 (first round, third word)
    uint32_t ca, cb, lo0c;  // second round: (k0 + W0) ^ s1', (k1 + W1) ^ hi(s0' M0), lo(s0' M0)
    uint32_t a2, b2;        // keys of the third round

    __host__ __device__ static PhiloxLo make(const PhiloxGen &g, const Ctr &base)
    {
        const uint32_t s1 = static_cast<uint32_t>(base.w[0] >> 32);
        const uint32_t s2 = static_cast<uint32_t>(base.w[1]);
        const uint32_t s3 = static_cast<uint32_t>(base.w[1] >> 32);
        const uint32_t s0p = g.k0 ^ s1 ^ mulhi32(s2, 0xCD9E8D57u);
        const uint32_t s1p = s2 * 0xCD9E8D57u;
        PhiloxLo p;
        p.lo = static_cast<uint32_t>(base.w[0]);
        p.k1s3 = g.k1 ^ s3;
        p.ca = (g.k0 + 0x9E3779B9u) ^ s1p;
        p.cb = (g.k1 + 0xBB67AE85u) ^ mulhi32(s0p, 0xD2511F53u);
        p.lo0c = s0p * 0xD2511F53u;
        p.a2 = g.k0 + 2u * 0x9E3779B9u;
        p.b2 = g.k1 + 2u * 0xBB67AE85u;
        return p;
    }

    // block i of the launch (counter low word lo + i, no carry into s1)
    __host__ __device__ __forceinline__ void block(uint32_t i, uint32_t out[4]) const
    {
        const uint32_t s0 = lo + i;
        const uint32_t t2 = k1s3 ^ mulhi32(s0, 0xD2511F53u);  // first round
        const uint32_t t3 = s0 * 0xD2511F53u;
        uint32_t x0 = ca ^ mulhi32(t2, 0xCD9E8D57u);  // second round
        uint32_t x1 = t2 * 0xCD9E8D57u;
        uint32_t x2 = cb ^ t3;
        uint32_t x3 = lo0c;
        uint32_t a = a2, b = b2;
#pragma unroll
        for (int r = 2; r < 10; ++r) {
            const uint32_t hi2 = mulhi32(x2, 0xCD9E8D57u);
            const uint32_t lo2 = x2 * 0xCD9E8D57u;
            const uint32_t hi0 = mulhi32(x0, 0xD2511F53u);
            const uint32_t lo0 = x0 * 0xD2511F53u;
            x0 = a ^ x1 ^ hi2;
            x1 = lo2;
            x2 = b ^ x3 ^ hi0;
            x3 = lo0;
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        out[0] = x0;
        out[1] = x1;
        out[2] = x2;
        out[3] = x3;
    }
};

// ---------------------------------------------------------------------------
// Threefry4x64-20.  The key-injection words of all six injections are
// precomputed on the host (they do not depend on the counter).
// ---------------------------------------------------------------------------
struct ThreefryGen {
    static constexpr int kWords = 8;
    static constexpr int kCtrWords = 4;
    static constexpr int kDynSmem = 0;
    uint64_t inj[6][4];  // inj[S][i] = par[(S+i)%5] + tweak/parity terms, S = round/4

    __host__ static ThreefryGen make(const uint64_t key[4], const uint64_t tweak[2])
    {
        ThreefryGen g;
        uint64_t par[8];
        for (int i = 0; i < 4; ++i) par[i] = key[i];
        par[4] = 0x1BD11BDAA9FC1A22ull ^ key[0] ^ key[1] ^ key[2] ^ key[3];
        par[5] = tweak[0];
        par[6] = tweak[1];
        par[7] = tweak[0] ^ tweak[1];
        for (uint64_t S = 0; S < 6; ++S) {
            g.inj[S][0] = par[(S + 0) % 5];
            g.inj[S][1] = par[(S + 1) % 5] + par[5 + (S + 0) % 3];
            g.inj[S][2] = par[(S + 2) % 5] + par[5 + (S + 1) % 3];
            g.inj[S][3] = par[(S + 3) % 5] + S;
        }
        return g;
    }

    __device__ __forceinline__ void prepare() const {}

    template <int L>
    __device__ __forceinline__ static uint64_t rotl(uint64_t x)
    {
        if constexpr (L == 32) {
            return (x << 32) | (x >> 32);
        } else {
            return (x << L) | (x >> (64 - L));
        }
    }

    template <int L0, int L1>
    __device__ __forceinline__ static void round(uint64_t &s0, uint64_t &s1, uint64_t &s2,
        uint64_t &s3)
    {
        s0 += s1;
        s2 += s3;
        const uint64_t t1 = rotl<L0>(s1);
        const uint64_t t3 = rotl<L1>(s3);
        s1 = s2 ^ t3;
        s3 = s0 ^ t1;
    }

    __device__ __forceinline__ void inject(int S, uint64_t &s0, uint64_t &s1, uint64_t &s2,
        uint64_t &s3) const
    {
        s0 += inj[S][0];
        s1 += inj[S][1];
        s2 += inj[S][2];
        s3 += inj[S][3];
    }

    __device__ __forceinline__ void block(const Ctr &c, uint32_t out[8]) const
    {
        uint64_t s0 = c.w[0], s1 = c.w[1], s2 = c.w[2], s3 = c.w[3];
        inject(0, s0, s1, s2, s3);
#pragma unroll
        for (int cyc = 0; cyc < 5; ++cyc) {
            if (cyc % 2 == 0) {
                round<14, 16>(s0, s1, s2, s3);
                round<52, 57>(s0, s1, s2, s3);
                round<23, 40>(s0, s1, s2, s3);
                round<5, 37>(s0, s1, s2, s3);
            } else {
                round<25, 33>(s0, s1, s2, s3);
                round<46, 12>(s0, s1, s2, s3);
                round<58, 22>(s0, s1, s2, s3);
                round<32, 32>(s0, s1, s2, s3);
            }
            inject(cyc + 1, s0, s1, s2, s3);
        }
        out[0] = static_cast<uint32_t>(s0);
        out[1] = static_cast<uint32_t>(s0 >> 32);
        out[2] = static_cast<uint32_t>(s1);
        out[3] = static_cast<uint32_t>(s1 >> 32);
        out[4] = static_cast<uint32_t>(s2);
        out[5] = static_cast<uint32_t>(s2 >> 32);
        out[6] = static_cast<uint32_t>(s3);
        out[7] = static_cast<uint32_t>(s3 >> 32);
    }
};

// ---------------------------------------------------------------------------
// ARS-5 with table-driven AES rounds from shared memory.
//
// The AES S-box and the round table Te0 (Te0[x] = {2S(x), S(x), S(x), 3S(x)}
// as little-endian bytes) are derived at compile time from GF(2^8)
// arithmetic.  In shared memory Te0 is replicated once per lane
// (tab[x * 32 + lane]), so the 32 lanes of a warp always hit 32 different
// banks; Te1..Te3 are byte rotations of Te0 and the final-round S-box byte is
// byte 1 of Te0.
// ---------------------------------------------------------------------------
struct AesTables {
    uint32_t te0[256];
};

constexpr uint8_t gf_mul(uint8_t a, uint8_t b)
{
    uint8_t p = 0;
    for (int i = 0; i < 8; ++i) {
        if (b & 1) p = static_cast<uint8_t>(p ^ a);
        const bool hi = (a & 0x80) != 0;
        a = static_cast<uint8_t>(a << 1);
        if (hi) a = static_cast<uint8_t>(a ^ 0x1B);
        b = static_cast<uint8_t>(b >> 1);
    }
    return p;
}

constexpr uint8_t gf_inv(uint8_t x)
{
    // x^254 by square-and-multiply (0 maps to 0)
    uint8_t r = 1, base = x;
    int e = 254;
    while (e) {
        if (e & 1) r = gf_mul(r, base);
        base = gf_mul(base, base);
        e >>= 1;
    }
    return x == 0 ? 0 : r;
}

constexpr uint8_t aes_sbox_entry(int x)
{
    uint8_t b = gf_inv(static_cast<uint8_t>(x));
    uint8_t s = b;
    for (int i = 0; i < 4; ++i) {
        b = static_cast<uint8_t>((b << 1) | (b >> 7));
        s = static_cast<uint8_t>(s ^ b);
    }
    return static_cast<uint8_t>(s ^ 0x63);
}

constexpr AesTables make_aes_tables()
{
    AesTables t{};
    for (int x = 0; x < 256; ++x) {
        const uint8_t s = aes_sbox_entry(x);
        t.te0[x] = static_cast<uint32_t>(gf_mul(s, 2)) | (static_cast<uint32_t>(s) << 8) |
                   (static_cast<uint32_t>(s) << 16) | (static_cast<uint32_t>(gf_mul(s, 3)) << 24);
    }
    return t;
}

__constant__ const AesTables kAesTables = make_aes_tables();

// The lane-replicated table lives at the start of the kernel's dynamic shared
// memory; every kernel instantiated with ArsGen is launched with
// ArsGen::kDynSmem bytes of it.
__device__ __forceinline__ uint32_t *ars_smem_table()
{
    extern __shared__ __align__(16) uint32_t mb_dyn_smem[];
    return mb_dyn_smem;
}

struct ArsGen {
    static constexpr int kWords = 4;
    static constexpr int kCtrWords = 2;
    static constexpr int kDynSmem = 256 * 32 * 4;
    uint32_t rk[6][4];

    __host__ static ArsGen make(const uint64_t key[4])
    {
        ArsGen g;
        const uint64_t klo = (key[0] & 0xFFFFFFFFull) | ((key[1] & 0xFFFFFFFFull) << 32);
        const uint64_t khi = (key[2] & 0xFFFFFFFFull) | ((key[3] & 0xFFFFFFFFull) << 32);
        for (uint64_t n = 0; n <= 5; ++n) {
            const uint64_t a = klo + 0x9E3779B97F4A7C15ull * n;
            const uint64_t b = khi + 0xBB67AE8584CAA73Bull * n;
            g.rk[n][0] = static_cast<uint32_t>(a);
            g.rk[n][1] = static_cast<uint32_t>(a >> 32);
            g.rk[n][2] = static_cast<uint32_t>(b);
            g.rk[n][3] = static_cast<uint32_t>(b >> 32);
        }
        return g;
    }

    // Every thread of the CTA must call prepare() before the first block().
    __device__ __forceinline__ void prepare() const
    {
        uint32_t *tab = ars_smem_table();
        for (int i = threadIdx.x; i < 256 * 32; i += blockDim.x) {
            tab[i] = kAesTables.te0[i >> 5];
        }
        __syncthreads();
    }

    // Shared-memory byte address of this lane's copy of Te0[x] is
    // x * 128 + base, base = table + 4 * lane.  Bytes are pulled out and
    // rotated with PRMT (one ALU op each); the address is one multiply-add.
    __device__ __forceinline__ static uint32_t lds(uint32_t addr)
    {
        uint32_t v;
        asm("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
        return v;
    }

    template <int B>
    __device__ __forceinline__ static uint32_t te(uint32_t s, uint32_t base)
    {
        const uint32_t x = __byte_perm(s, 0u, 0x4440u | B);
        uint32_t a;
        asm("mad.lo.u32 %0, %1, 128, %2;" : "=r"(a) : "r"(x), "r"(base));
        return lds(a);
    }

    __device__ __forceinline__ static uint32_t rot8(uint32_t x) { return __byte_perm(x, x, 0x2103u); }
    __device__ __forceinline__ static uint32_t rot16(uint32_t x) { return __byte_perm(x, x, 0x1032u); }
    __device__ __forceinline__ static uint32_t rot24(uint32_t x) { return __byte_perm(x, x, 0x0321u); }

    __device__ __forceinline__ void block(const Ctr &c, uint32_t out[4]) const
    {
        const uint32_t base =
            static_cast<uint32_t>(__cvta_generic_to_shared(ars_smem_table())) + 4u * (threadIdx.x & 31u);
        uint32_t s0 = static_cast<uint32_t>(c.w[0]) ^ rk[0][0];
        uint32_t s1 = static_cast<uint32_t>(c.w[0] >> 32) ^ rk[0][1];
        uint32_t s2 = static_cast<uint32_t>(c.w[1]) ^ rk[0][2];
        uint32_t s3 = static_cast<uint32_t>(c.w[1] >> 32) ^ rk[0][3];
#pragma unroll
        for (int r = 1; r <= 4; ++r) {
            const uint32_t t0 = rk[r][0] ^ te<0>(s0, base) ^ rot8(te<1>(s1, base)) ^ rot16(te<2>(s2, base)) ^
                                rot24(te<3>(s3, base));
            const uint32_t t1 = rk[r][1] ^ te<0>(s1, base) ^ rot8(te<1>(s2, base)) ^ rot16(te<2>(s3, base)) ^
                                rot24(te<3>(s0, base));
            const uint32_t t2 = rk[r][2] ^ te<0>(s2, base) ^ rot8(te<1>(s3, base)) ^ rot16(te<2>(s0, base)) ^
                                rot24(te<3>(s1, base));
            const uint32_t t3 = rk[r][3] ^ te<0>(s3, base) ^ rot8(te<1>(s0, base)) ^ rot16(te<2>(s1, base)) ^
                                rot24(te<3>(s2, base));
            s0 = t0;
            s1 = t1;
            s2 = t2;
            s3 = t3;
        }
        // last round: S-box byte = byte 1 of Te0, placed with PRMT in ShiftRows order
        auto last = [base](uint32_t a, uint32_t b, uint32_t c2, uint32_t d) -> uint32_t {
            const uint32_t x0 = te<0>(a, base), x1 = te<1>(b, base), x2 = te<2>(c2, base), x3 = te<3>(d, base);
            const uint32_t lo = __byte_perm(x0, x1, 0x0051u);  // low bytes: x0.b1, x1.b1
            const uint32_t hi = __byte_perm(x2, x3, 0x0051u);  // low bytes: x2.b1, x3.b1
            return __byte_perm(lo, hi, 0x5410u);
        };
        out[0] = rk[5][0] ^ last(s0, s1, s2, s3);
        out[1] = rk[5][1] ^ last(s1, s2, s3, s0);
        out[2] = rk[5][2] ^ last(s2, s3, s0, s1);
        out[3] = rk[5][3] ^ last(s3, s0, s1, s2);
    }
};

// ARS-5 with four lane-replicated round tables, Te1..Te3 stored rotated
// (Te_t[x] = Te0[x] rotated left by 8t bits) instead of rotated per lookup:
// 48 fewer byte permutes per block, whose ALU pipe is the limit of the
// one-table form, for 128 KiB of shared memory.  Bit-identical to ArsGen;
// used by the aligned fill kernel, launched with 1024-thread CTAs (one per
// SM keeps 32 warps resident).
struct ArsGen4 {
    static constexpr int kWords = 4;
    static constexpr int kCtrWords = 2;
    static constexpr int kTableBytes = 256 * 32 * 4;
    static constexpr int kDynSmem = 4 * kTableBytes;
    uint32_t rk[6][4];

    __host__ static ArsGen4 from(const ArsGen &g)
    {
        ArsGen4 h;
        for (int n = 0; n < 6; ++n)
            for (int k = 0; k < 4; ++k) h.rk[n][k] = g.rk[n][k];
        return h;
    }

    __device__ __forceinline__ void prepare() const
    {
        uint32_t *tab = ars_smem_table();
        for (int i = threadIdx.x; i < 256 * 32; i += blockDim.x) {
            const uint32_t v = kAesTables.te0[i >> 5];
            tab[i] = v;
            tab[i + 256 * 32] = ArsGen::rot8(v);
            tab[i + 2 * 256 * 32] = ArsGen::rot16(v);
            tab[i + 3 * 256 * 32] = ArsGen::rot24(v);
        }
        __syncthreads();
    }

    __device__ __forceinline__ void block(const Ctr &c, uint32_t out[4]) const
    {
        const uint32_t b0 =
            static_cast<uint32_t>(__cvta_generic_to_shared(ars_smem_table())) + 4u * (threadIdx.x & 31u);
        const uint32_t b1 = b0 + kTableBytes, b2 = b0 + 2 * kTableBytes, b3 = b0 + 3 * kTableBytes;
        uint32_t s0 = static_cast<uint32_t>(c.w[0]) ^ rk[0][0];
        uint32_t s1 = static_cast<uint32_t>(c.w[0] >> 32) ^ rk[0][1];
        uint32_t s2 = static_cast<uint32_t>(c.w[1]) ^ rk[0][2];
        uint32_t s3 = static_cast<uint32_t>(c.w[1] >> 32) ^ rk[0][3];
#pragma unroll
        for (int r = 1; r <= 4; ++r) {
            const uint32_t t0 = rk[r][0] ^ ArsGen::te<0>(s0, b0) ^ ArsGen::te<1>(s1, b1) ^ ArsGen::te<2>(s2, b2) ^
                                ArsGen::te<3>(s3, b3);
            const uint32_t t1 = rk[r][1] ^ ArsGen::te<0>(s1, b0) ^ ArsGen::te<1>(s2, b1) ^ ArsGen::te<2>(s3, b2) ^
                                ArsGen::te<3>(s0, b3);
            const uint32_t t2 = rk[r][2] ^ ArsGen::te<0>(s2, b0) ^ ArsGen::te<1>(s3, b1) ^ ArsGen::te<2>(s0, b2) ^
                                ArsGen::te<3>(s1, b3);
            const uint32_t t3 = rk[r][3] ^ ArsGen::te<0>(s3, b0) ^ ArsGen::te<1>(s0, b1) ^ ArsGen::te<2>(s1, b2) ^
                                ArsGen::te<3>(s2, b3);
            s0 = t0;
            s1 = t1;
            s2 = t2;
            s3 = t3;
        }
        // last round from table 0 as in ArsGen: the S-box byte is byte 1 of Te0
        auto last = [b0](uint32_t a, uint32_t b, uint32_t c2, uint32_t d) -> uint32_t {
            const uint32_t x0 = ArsGen::te<0>(a, b0), x1 = ArsGen::te<1>(b, b0), x2 = ArsGen::te<2>(c2, b0),
                           x3 = ArsGen::te<3>(d, b0);
            const uint32_t lo = __byte_perm(x0, x1, 0x0051u);
            const uint32_t hi = __byte_perm(x2, x3, 0x0051u);
            return __byte_perm(lo, hi, 0x5410u);
        };
        out[0] = rk[5][0] ^ last(s0, s1, s2, s3);
        out[1] = rk[5][1] ^ last(s1, s2, s3, s0);
        out[2] = rk[5][2] ^ last(s2, s3, s0, s1);
        out[3] = rk[5][3] ^ last(s3, s0, s1, s2);
    }
};

}  // namespace mckl_b200
