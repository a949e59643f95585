/* oracle.c -- plain-C restatement of MCKL's counter-based RNG / SMC hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each function cites the reference
 * file:line it restates; paths are relative to the MCKL source tree.
 *
 * Build pins (oracle/Makefile): -ffp-contract=off, so every rounding written
 * here is a rounding in the binary; fma() is written out exactly where the
 * reference calls mckl::muladd with MCKL_USE_FMA on (math/vmf.hpp:670-694).
 */
#include "oracle.h"

#include <stdlib.h>
#include <tgmath.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Engines                                                                  */
/* ------------------------------------------------------------------------ */

enum { K_PHILOX = 1, K_PHILOX64 = 2, K_THREEFRY = 3, K_THREEFRY64 = 4, K_ARS = 5, K_ARS64 = 6 };

static unsigned block_bytes(uint32_t kind)
{
    return (kind == K_THREEFRY || kind == K_THREEFRY64) ? 32u : 16u;
}

static unsigned result_bytes(uint32_t kind)
{
    return (kind == K_PHILOX64 || kind == K_THREEFRY64 || kind == K_ARS64) ? 8u : 4u;
}

static unsigned ctr_words(uint32_t kind)
{
    return (kind == K_THREEFRY || kind == K_THREEFRY64) ? 4u : 2u;
}

static unsigned words_per_block(uint32_t kind)
{
    return block_bytes(kind) / result_bytes(kind);
}

/* Philox4x32-10: random/internal/philox_generic_4x.hpp:40-53 (round),
 * random/internal/philox_constants.hpp:51-56, 82-87 (Weyl and multipliers),
 * random/internal/philox_common.hpp:46-73 (PhiloxHiLo returns the low half). */
static void philox4x32_10(const uint64_t *ctr, const uint64_t *key, uint32_t out[4])
{
    uint32_t s0 = (uint32_t) ctr[0], s1 = (uint32_t) (ctr[0] >> 32);
    uint32_t s2 = (uint32_t) ctr[1], s3 = (uint32_t) (ctr[1] >> 32);
    uint32_t k0 = (uint32_t) key[0], k1 = (uint32_t) key[1];
    for (uint32_t r = 0; r != 10; ++r) {
        const uint64_t p2 = (uint64_t) s2 * 0xCD9E8D57u;
        const uint64_t p0 = (uint64_t) s0 * 0xD2511F53u;
        const uint32_t kr0 = k0 + 0x9E3779B9u * r;
        const uint32_t kr1 = k1 + 0xBB67AE85u * r;
        const uint32_t n0 = kr0 ^ s1 ^ (uint32_t) (p2 >> 32);
        const uint32_t n1 = (uint32_t) p2;
        const uint32_t n2 = kr1 ^ s3 ^ (uint32_t) (p0 >> 32);
        const uint32_t n3 = (uint32_t) p0;
        s0 = n0; s1 = n1; s2 = n2; s3 = n3;
    }
    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
}

/* Threefry4x64-20: random/threefry.hpp:109-133 (parity word, tweak),
 * random/internal/threefry_common.hpp:212-247 (key injection),
 * random/internal/threefry_generic_4x64.hpp:40-79 (round with the 1<->3 swap),
 * random/internal/threefry_constants.hpp:51-56, 83-89 (parity, rotations). */
static const int TF_R0[8] = {14, 52, 23, 5, 25, 46, 58, 32};
static const int TF_R1[8] = {16, 57, 40, 37, 33, 12, 22, 32};

static uint64_t rotl64(uint64_t x, int r)
{
    return (x << r) | (x >> (64 - r));
}

static void threefry4x64_20(const uint64_t *ctr, const uint64_t *key, const uint64_t *tweak,
    uint64_t out[4])
{
    uint64_t par[8];
    par[0] = key[0]; par[1] = key[1]; par[2] = key[2]; par[3] = key[3];
    par[4] = 0x1BD11BDAA9FC1A22ull ^ key[0] ^ key[1] ^ key[2] ^ key[3];
    par[5] = tweak[0]; par[6] = tweak[1]; par[7] = tweak[0] ^ tweak[1];
    uint64_t s[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    for (int N = 0; N <= 20; ++N) {
        if (N > 0) {
            const int L0 = TF_R0[(N - 1) % 8], L1 = TF_R1[(N - 1) % 8];
            s[0] += s[1];
            s[2] += s[3];
            const uint64_t t1 = rotl64(s[1], L0);
            const uint64_t t3 = rotl64(s[3], L1);
            s[1] = s[2] ^ t3;
            s[3] = s[0] ^ t1;
        }
        if (N % 4 == 0) {
            const uint64_t S = (uint64_t) (N / 4);
            s[0] += par[(S + 0) % 5];
            s[1] += par[(S + 1) % 5] + par[5 + (S + 0) % 3];
            s[2] += par[(S + 2) % 5] + par[5 + (S + 1) % 3];
            s[3] += par[(S + 3) % 5] + S;
        }
    }
    out[0] = s[0]; out[1] = s[1]; out[2] = s[2]; out[3] = s[3];
}

/* ARS-5: random/internal/aes_generic.hpp:254-306 (round keys: Weyl increments
 * of the two 64-bit key halves, random/internal/aes_constants.hpp:289-304),
 * :413-491 (first xor, four table rounds, last S-box round).  The table-driven
 * round is the FIPS-197 round in little-endian words; the tables are derived
 * here from the field arithmetic instead of being copied. */
static uint32_t aes_te0[256];
static uint8_t aes_sbox[256];
static int aes_ready;

static uint8_t gf_mul(uint8_t a, uint8_t b)
{
    uint8_t p = 0;
    while (b) {
        if (b & 1) p ^= a;
        a = (uint8_t) ((a << 1) ^ ((a & 0x80) ? 0x1B : 0));
        b >>= 1;
    }
    return p;
}

static void aes_init(void)
{
    if (aes_ready) return;
    for (int x = 0; x < 256; ++x) {
        uint8_t inv = 0;
        if (x != 0) {
            for (int y = 1; y < 256; ++y) {
                if (gf_mul((uint8_t) x, (uint8_t) y) == 1) { inv = (uint8_t) y; break; }
            }
        }
        uint8_t b = inv, s = inv;
        for (int i = 1; i <= 4; ++i) {
            b = (uint8_t) ((b << 1) | (b >> 7));
            s ^= b;
        }
        aes_sbox[x] = (uint8_t) (s ^ 0x63);
    }
    for (int x = 0; x < 256; ++x) {
        const uint8_t s = aes_sbox[x];
        aes_te0[x] = (uint32_t) gf_mul(s, 2) | ((uint32_t) s << 8) | ((uint32_t) s << 16) |
                     ((uint32_t) gf_mul(s, 3) << 24);
    }
    aes_ready = 1;
}

static uint32_t rotl32(uint32_t x, int r)
{
    return (x << r) | (x >> (32 - r));
}

static void ars5(const uint64_t *ctr, const uint64_t *key, uint32_t out[4])
{
    aes_init();
    const uint64_t klo = (uint64_t) (uint32_t) key[0] | ((uint64_t) (uint32_t) key[1] << 32);
    const uint64_t khi = (uint64_t) (uint32_t) key[2] | ((uint64_t) (uint32_t) key[3] << 32);
    uint32_t rk[6][4];
    for (int n = 0; n <= 5; ++n) {
        const uint64_t a = klo + 0x9E3779B97F4A7C15ull * (uint64_t) n;
        const uint64_t b = khi + 0xBB67AE8584CAA73Bull * (uint64_t) n;
        rk[n][0] = (uint32_t) a; rk[n][1] = (uint32_t) (a >> 32);
        rk[n][2] = (uint32_t) b; rk[n][3] = (uint32_t) (b >> 32);
    }
    uint32_t s[4] = {(uint32_t) ctr[0], (uint32_t) (ctr[0] >> 32), (uint32_t) ctr[1],
        (uint32_t) (ctr[1] >> 32)};
    for (int j = 0; j < 4; ++j) s[j] ^= rk[0][j];
    for (int r = 1; r <= 4; ++r) {
        uint32_t t[4];
        for (int j = 0; j < 4; ++j) {
            t[j] = rk[r][j] ^ aes_te0[s[j] & 0xFF] ^ rotl32(aes_te0[(s[(j + 1) & 3] >> 8) & 0xFF], 8) ^
                   rotl32(aes_te0[(s[(j + 2) & 3] >> 16) & 0xFF], 16) ^
                   rotl32(aes_te0[s[(j + 3) & 3] >> 24], 24);
        }
        memcpy(s, t, sizeof(t));
    }
    for (int j = 0; j < 4; ++j) {
        out[j] = rk[5][j] ^ (uint32_t) aes_sbox[s[j] & 0xFF] ^
                 ((uint32_t) aes_sbox[(s[(j + 1) & 3] >> 8) & 0xFF] << 8) ^
                 ((uint32_t) aes_sbox[(s[(j + 2) & 3] >> 16) & 0xFF] << 16) ^
                 ((uint32_t) aes_sbox[s[(j + 3) & 3] >> 24] << 24);
    }
}

int orc_block(const orc_engine *e, const uint64_t *ctr, void *out)
{
    switch (e->kind) {
        case K_PHILOX: case K_PHILOX64: philox4x32_10(ctr, e->key, (uint32_t *) out); return 0;
        case K_THREEFRY: case K_THREEFRY64: threefry4x64_20(ctr, e->key, e->tweak, (uint64_t *) out); return 0;
        case K_ARS: case K_ARS64: ars5(ctr, e->key, (uint32_t *) out); return 0;
        default: return -1;
    }
}

/* Counter increment by one block: random/internal/increment_generic.hpp:56-90. */
static void ctr_inc(orc_engine *e)
{
    const unsigned w = ctr_words(e->kind);
    for (unsigned i = 0; i < w; ++i) {
        if (++e->ctr[i] != 0) return;
    }
}

/* CounterEngine::operator()(n, r): random/counter.hpp:142-165.  The buffered
 * block is a pure function of (key, ctr), so it is regenerated, not stored. */
int orc_rand(orc_engine *e, size_t n, void *r)
{
    const unsigned M = words_per_block(e->kind), rb = result_bytes(e->kind);
    unsigned char blk[32];
    unsigned char *out = (unsigned char *) r;
    if (e->index > M) e->index = M;
    const size_t remain = M - e->index;
    if (n <= remain) {
        if (n) {
            orc_block(e, e->ctr, blk);
            memcpy(out, blk + (size_t) e->index * rb, n * rb);
        }
        e->index += (uint32_t) n;
        return 0;
    }
    if (remain) {
        orc_block(e, e->ctr, blk);
        memcpy(out, blk + (size_t) e->index * rb, remain * rb);
        out += remain * rb;
    }
    n -= remain;
    e->index = M;
    const size_t m = n / M;
    for (size_t b = 0; b < m; ++b) {
        ctr_inc(e);
        orc_block(e, e->ctr, out);
        out += (size_t) M * rb;
    }
    n -= m * M;
    ctr_inc(e);
    orc_block(e, e->ctr, blk);
    memcpy(out, blk, n * rb);
    e->index = (uint32_t) n;
    return 0;
}

/* CounterEngine::operator()(): random/counter.hpp:132-140. */
static uint64_t orc_next(orc_engine *e)
{
    const unsigned M = words_per_block(e->kind), rb = result_bytes(e->kind);
    unsigned char blk[32];
    if (e->index >= M) {
        ctr_inc(e);
        e->index = 0;
    }
    orc_block(e, e->ctr, blk);
    uint64_t v = 0;
    memcpy(&v, blk + (size_t) e->index * rb, rb);
    e->index++;
    return v;
}

/* ------------------------------------------------------------------------ */
/* U01 conversions: random/internal/u01_generic.hpp:48-198 with W = 32 or 64  */
/* ------------------------------------------------------------------------ */

static double u01_f64(int variant, uint64_t u, int W)
{
    /* W = 32: M = 53 > W.  W = 64: M = 53 < W. */
    if (W == 32) {
        switch (variant) {
            case 1: return ((double) (u & 1) + (double) u) * 0x1p-32;      /* CC: P = 31, V = 32 */
            case 2: return (double) u * 0x1p-32;                            /* CO */
            case 3: return (double) u * 0x1p-32 + 0x1p-32;                  /* OC */
            case 4: return (double) u * 0x1p-32 + 0x1p-33;                  /* OO */
        }
    } else {
        switch (variant) {
            case 1: { uint64_t v = (u << 1) >> 10; return (double) ((v & 1) + v) * 0x1p-54; } /* P = 53, V = 54, L = 1, R = 9 */
            case 2: return (double) (u >> 11) * 0x1p-53;
            case 3: return (double) (u >> 11) * 0x1p-53 + 0x1p-53;
            case 4: return (double) (u >> 12) * 0x1p-52 + 0x1p-53;
        }
    }
    return 0;
}

static float u01_f32(int variant, uint64_t u, int W)
{
    if (W == 32) {
        const uint32_t x = (uint32_t) u;
        switch (variant) {
            case 1: { uint32_t v = (x << 1) >> 7; return (float) ((v & 1) + v) * 0x1p-25f; } /* P = 24, V = 25 */
            case 2: return (float) (x >> 8) * 0x1p-24f;
            case 3: return (float) (x >> 8) * 0x1p-24f + 0x1p-24f;
            case 4: return (float) (x >> 9) * 0x1p-23f + 0x1p-24f;
        }
    } else {
        switch (variant) {
            case 1: { uint64_t v = (u << 1) >> 39; return (float) ((v & 1) + v) * 0x1p-25f; }
            case 2: return (float) (u >> 40) * 0x1p-24f;
            case 3: return (float) (u >> 40) * 0x1p-24f + 0x1p-24f;
            case 4: return (float) (u >> 41) * 0x1p-23f + 0x1p-24f;
        }
    }
    return 0;
}

/* Read n engine words (u32 or u64 by engine) into a u64 buffer. */
static void rand_words(orc_engine *e, size_t n, uint64_t *buf)
{
    if (result_bytes(e->kind) == 8) {
        orc_rand(e, n, buf);
        return;
    }
    uint32_t *tmp = (uint32_t *) malloc((n ? n : 1) * sizeof(uint32_t));
    orc_rand(e, n, tmp);
    for (size_t i = 0; i < n; ++i) buf[i] = tmp[i];
    free(tmp);
}

static uint64_t next_word(orc_engine *e)
{
    return orc_next(e);
}

/* The float/double instantiations of the distribution code. */
#define REAL double
#define RS(name) name##_f64
#define U01CONV u01_f64
#define KBUF 1024
#define PI2 0x1.921fb54442d18p+2
#include "oracle_real.inc"
#undef REAL
#undef RS
#undef U01CONV
#undef KBUF
#undef PI2

#define REAL float
#define RS(name) name##_f32
#define U01CONV u01_f32
#define KBUF 2048
#define PI2 0x1.921fb6p+2f
#include "oracle_real.inc"
#undef REAL
#undef RS
#undef U01CONV
#undef KBUF
#undef PI2

int orc_u01(orc_engine *e, int variant, int is_f64, size_t n, void *r)
{
    if (variant < 0 || variant > 4) return -2;
    if (is_f64) u01_batch_f64(e, variant, n, (double *) r);
    else u01_batch_f32(e, variant, n, (float *) r);
    return 0;
}

int orc_normal(orc_engine *e, int is_f64, size_t n, void *r, double mean, double sd)
{
    if (is_f64) normal_batch_f64(e, n, (double *) r, mean, sd);
    else normal_batch_f32(e, n, (float *) r, (float) mean, (float) sd);
    return 0;
}

int orc_exponential(orc_engine *e, int is_f64, size_t n, void *r, double lambda)
{
    if (is_f64) exponential_batch_f64(e, n, (double *) r, lambda);
    else exponential_batch_f32(e, n, (float *) r, (float) lambda);
    return 0;
}

int orc_gamma(orc_engine *e, int is_f64, size_t n, void *r, double alpha, double beta)
{
    if (is_f64) gamma_batch_f64(e, n, (double *) r, alpha, beta);
    else gamma_batch_f32(e, n, (float *) r, (float) alpha, (float) beta);
    return 0;
}

int orc_gamma_blocks(const orc_engine *e, int is_f64, size_t nblocks, size_t block,
    const double *alpha, double beta, void *r, int nthreads)
{
    return orc_gamma_blocks_from(e, is_f64, 0, nblocks, block, alpha, beta, r, nthreads);
}

/* Blocks first .. first + nblocks - 1 of the same per-block form: block
 * first + b is written to r + b * block, with shape alpha[b]. */
int orc_gamma_blocks_from(const orc_engine *e, int is_f64, size_t first, size_t nblocks, size_t block,
    const double *alpha, double beta, void *r, int nthreads)
{
    (void) nthreads;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for (long long b = 0; b < (long long) nblocks; ++b) {
        orc_engine s = *e;
        s.ctr[0] = 0; s.ctr[1] = (uint64_t) (first + (size_t) b); s.ctr[2] = s.ctr[3] = 0;
        s.index = 0xFFFFFFFFu;
        if (is_f64) gamma_batch_f64(&s, block, (double *) r + (size_t) b * block, alpha[b], beta);
        else gamma_batch_f32(&s, block, (float *) r + (size_t) b * block, (float) alpha[b], (float) beta);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Weight: core/weight.hpp:64-227                                            */
/* ------------------------------------------------------------------------ */

static void weight_normalize(size_t N, double *w, int use_log, double *ess)
{
    double lmax = 0;
    if (use_log) {
        lmax = -INFINITY;                               /* max_element, :184-196 */
        for (size_t i = 0; i < N; ++i) if (lmax < w[i]) lmax = w[i];
    }
    double accw = 0, essw = 0;
    const size_t K = 1024;
    for (size_t c = 0; c < N; c += K) {                 /* normalize(n, ...), :214-227 */
        const size_t n = (N - c < K) ? N - c : K;
        double *wc = w + c;
        if (use_log) {
            for (size_t i = 0; i < n; ++i) wc[i] = wc[i] - lmax;
            for (size_t i = 0; i < n; ++i) wc[i] = exp(wc[i]);
        }
        for (size_t i = 0; i < n; ++i) accw = accw + wc[i];   /* std::accumulate */
        double d = 0;                                          /* cblas_ddot loop */
        for (size_t i = 0; i < n; ++i) { const double t = wc[i] * wc[i]; d = d + t; }
        essw = essw + d;
    }
    const double inv = 1 / accw;
    for (size_t i = 0; i < N; ++i) w[i] = inv * w[i];
    *ess = accw * accw / essw;
}

int orc_weight_set_log(size_t N, const double *v, double *W, double *ess)
{
    memcpy(W, v, N * sizeof(double));
    weight_normalize(N, W, 1, ess);
    return 0;
}

int orc_weight_add_log(size_t N, double *W, const double *v, double *ess)
{
    for (size_t i = 0; i < N; ++i) W[i] = log(W[i]);
    for (size_t i = 0; i < N; ++i) W[i] = W[i] + v[i];
    weight_normalize(N, W, 1, ess);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Resampling: algorithm/resample.hpp                                        */
/* ------------------------------------------------------------------------ */

/* u01_trans_sorted_impl, :63-80: chunked exponential spacings. */
static void sorted_chunk(size_t n0, size_t n, const double *u01, double *r, size_t N, double *lmax)
{
    if (n0 == n) return;
    double s[1024];
    size_t j = 0, m = N - n0;
    for (size_t i = 0; i < n - n0; ++i) r[i] = log(u01[i]);
    for (size_t i = n0; i != n; ++i, ++j, --m) {
        *lmax = *lmax + r[j] / (double) m;
        s[j] = *lmax;
    }
    for (size_t i = 0; i < n - n0; ++i) s[i] = exp(s[i]);
    for (size_t i = 0; i < n - n0; ++i) r[i] = 1 - s[i];
}

int orc_u01_trans_sorted(size_t N, const double *u01, double *r)
{
    if (N == 0) return 0;
    const size_t k = 1024;
    double lmax = 0;
    size_t n0 = 0;
    for (size_t i = 0; i != N / k; ++i, n0 += k, u01 += k, r += k) sorted_chunk(n0, n0 + k, u01, r, N, &lmax);
    sorted_chunk(n0, N, u01, r, N, &lmax);
    return 0;
}

/* u01_rand_sorted, :216-235: canonical uniforms per chunk, then the spacings. */
static void u01_rand_sorted(orc_engine *e, size_t N, double *r)
{
    if (N == 0) return;
    const size_t k = 1024;
    double lmax = 0;
    size_t n0 = 0;
    for (size_t i = 0; i != N / k; ++i, n0 += k, r += k) {
        u01_batch_f64(e, 0, k, r);
        sorted_chunk(n0, n0 + k, r, r, N, &lmax);
    }
    if (n0 != N) {
        u01_batch_f64(e, 0, N - n0, r);
        sorted_chunk(n0, N, r, r, N, &lmax);
    }
}

/* u01_rand_stratified, :239-254 and u01_trans_stratified_impl, :95-120. */
static void stratified_chunk(orc_engine *e, size_t n0, size_t n, double *r, double delta)
{
    if (n0 == n) return;
    u01_batch_f64(e, 0, n - n0, r);
    for (size_t j = 0; j < n - n0; ++j) r[j] = r[j] + (double) (n0 + j);
    for (size_t j = 0; j < n - n0; ++j) r[j] = delta * r[j];
}

static void u01_rand_stratified(orc_engine *e, size_t N, double *r)
{
    const size_t k = 1024;
    const double delta = 1 / (double) N;
    size_t n0 = 0;
    for (size_t i = 0; i != N / k; ++i, n0 += k, r += k) stratified_chunk(e, n0, n0 + k, r, delta);
    stratified_chunk(e, n0, N, r, delta);
}

/* u01_rand_systematic, :258-268 and u01_trans_systematic_impl, :122-135. */
static void u01_rand_systematic(orc_engine *e, size_t N, double *r)
{
    double u;
    u01_batch_f64(e, 0, 1, &u);   /* U01Distribution<double>{}(rng): 2 words, canonical */
    if (N == 0) return;
    const double delta = 1 / (double) N;
    const double ud = u * delta;
    for (size_t i = 0; i < N; ++i) r[i] = fma((double) i, delta, ud);
}

int orc_u01_sequence(int kind, orc_engine *e, size_t N, double *r)
{
    switch (kind) {
        case 0: u01_rand_sorted(e, N, r); return 0;
        case 1: u01_rand_stratified(e, N, r); return 0;
        case 2: u01_rand_systematic(e, N, r); return 0;
    }
    return -2;
}

/* resample_trans_u01_rep, :374-407. */
int orc_rep_to_u01(size_t N, size_t M, const double *W, const double *u01seq, uint64_t *rep)
{
    if (N == 0) return 0;
    if (N == 1) { rep[0] = M; return 0; }
    memset(rep, 0, N * sizeof(uint64_t));
    if (M == 0) return 0;
    double accw = 0;
    size_t j = 0;
    for (size_t i = 0; i != N - 1; ++i) {
        accw = accw + W[i];
        while (j != M && u01seq[j] < accw) { rep[i] += 1; ++j; }
    }
    rep[N - 1] = M - j;
    return 0;
}

/* resample_trans_residual, :333-364. */
static size_t trans_residual(size_t N, size_t M, const double *W, double *resid, uint64_t *integ)
{
    double sum_resid = 0;
    uint64_t sum_integ = 0;
    const double coeff = (double) M;
    for (size_t i = 0; i < N; ++i) {
        const double w = coeff * W[i];
        double ip;
        resid[i] = modf(w, &ip);
        integ[i] = (uint64_t) ip;
        sum_resid = sum_resid + resid[i];
        sum_integ += integ[i];
    }
    const double mul = 1 / sum_resid;
    for (size_t i = 0; i < N; ++i) resid[i] = resid[i] * mul;
    return M - (size_t) sum_integ;
}

/* ResampleAlgorithm::eval, :527-566; schemes :569-593. */
int orc_resample(int scheme, size_t N, size_t M, orc_engine *e, const double *W, uint64_t *rep)
{
    static const int seq_of[6] = {0, 1, 2, 0, 1, 2};
    if (scheme < 0 || scheme > 5) return -2;
    const int seq = seq_of[scheme];
    if (scheme < 3) {
        double *u = (double *) malloc((M ? M : 1) * sizeof(double));
        orc_u01_sequence(seq, e, M, u);
        orc_rep_to_u01(N, M, W, u, rep);
        free(u);
        return 0;
    }
    double *resid = (double *) malloc((N ? N : 1) * sizeof(double));
    uint64_t *integ = (uint64_t *) malloc((N ? N : 1) * sizeof(uint64_t));
    const size_t R = trans_residual(N, M, W, resid, integ);
    double *u = (double *) malloc((R ? R : 1) * sizeof(double));
    orc_u01_sequence(seq, e, R, u);
    orc_rep_to_u01(N, R, resid, u, rep);
    for (size_t i = 0; i < N; ++i) rep[i] += integ[i];
    free(u); free(resid); free(integ);
    return 0;
}

/* resample_trans_rep_index, :416-466: occupied slots keep their particle; the
 * empty ones, in ascending order, take the surplus copies in source order. */
int orc_rep_index(size_t N, size_t M, const uint64_t *rep, uint64_t *idx)
{
    if (N == 0 || M == 0) return 0;
    const size_t K = N < M ? N : M;
    uint64_t time = 0;
    size_t src = 0;
#define SEEK()                                                                  \
    do {                                                                        \
        if (src < K && rep[src] < time + 2) {                                   \
            time = 0;                                                           \
            do { ++src; } while (src < K && rep[src] < time + 2);               \
        }                                                                       \
        if (src >= K && src < N && rep[src] < time + 1) {                       \
            time = 0;                                                           \
            do { ++src; } while (src < N && rep[src] < time + 1);               \
        }                                                                       \
    } while (0)
    for (size_t dst = 0; dst != K; ++dst) {
        if (rep[dst] > 0) idx[dst] = dst;
        else { SEEK(); idx[dst] = src; ++time; }
    }
    for (size_t dst = K; dst < M; ++dst) { SEEK(); idx[dst] = src; ++time; }
#undef SEEK
    return 0;
}

/* StateMatrix<ColMajor>::select with n == size(): core/state_matrix.hpp:239-253. */
int orc_select_f64(size_t N, size_t dim, const uint64_t *idx, double *state)
{
    for (size_t d = 0; d < dim; ++d) {
        double *col = state + d * N;
        for (size_t i = 0; i < N; ++i) col[i] = col[idx[i]];
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* AR(1) particle filter through the SMCSampler step order                   */
/* (algorithm/smc.hpp:389-406, BackendSEQ: smp/backend_seq.hpp:40-70)        */
/* ------------------------------------------------------------------------ */

static orc_engine philox_engine(const uint32_t key[2])
{
    orc_engine e;
    memset(&e, 0, sizeof(e));
    e.kind = K_PHILOX;
    e.key[0] = key[0];
    e.key[1] = key[1];
    e.index = 4;
    return e;
}

/* Observations: one Normal(0,1) batch of 2T + 2 values from Philox4x32(key):
 * x_0 = sd0 z_0, x_t = phi x_{t-1} + sx z_t, y_t = x_t + sy z_{T+t}. */
int orc_simulate_ar1(size_t T, double phi, double sx, double sy, double sd0,
    const uint32_t key[2], double *x, double *y)
{
    orc_engine e = philox_engine(key);
    double *z = (double *) malloc((2 * T + 2) * sizeof(double));
    normal_batch_f64(&e, 2 * T + 2, z, 0.0, 1.0);
    x[0] = sd0 * z[0];
    y[0] = 0;
    for (size_t t = 1; t <= T; ++t) {
        const double a = phi * x[t - 1];
        const double b = sx * z[t];
        x[t] = a + b;
        const double c = sy * z[T + t];
        y[t] = x[t] + c;
    }
    free(z);
    return 0;
}

int orc_pf_ar1(size_t N, size_t T, const double *y, double phi, double sx, double sy,
    double sd0, const uint32_t mkey[2], const uint32_t rkey[2], int scheme,
    double threshold, double *loglik, double *ess_hist, uint8_t *resampled,
    uint64_t *anc, double *x_out, double *W_out)
{
    orc_engine em = philox_engine(mkey), er = philox_engine(rkey);
    double *x = (double *) malloc(N * sizeof(double));
    double *W = (double *) malloc(N * sizeof(double));
    double *ll = (double *) malloc(N * sizeof(double));
    double *eps = (double *) malloc(N * sizeof(double));
    uint64_t *rep = (uint64_t *) malloc(N * sizeof(uint64_t));
    uint64_t *idx = (uint64_t *) malloc(N * sizeof(uint64_t));
    const double lconst = -log(sy) - 0.5 * log(2 * 3.14159265358979323846);
    const double hinv = 0.5 / (sy * sy);
    double ess = (double) N;
    for (size_t i = 0; i < N; ++i) W[i] = 1.0 / (double) N;   /* Weight::set_equal */
    *loglik = 0;
    for (size_t it = 0; it <= T; ++it) {
        if (it == 0) {
            normal_batch_f64(&em, N, x, 0.0, sd0);
        } else {
            normal_batch_f64(&em, N, eps, 0.0, 1.0);
            const double yt = y[it];
            for (size_t i = 0; i < N; ++i) {
                const double a = phi * x[i];
                const double b = sx * eps[i];
                x[i] = a + b;
                const double r = yt - x[i];
                const double r2 = r * r;
                const double t = r2 * hinv;
                ll[i] = lconst - t;
            }
            double m = -INFINITY;
            for (size_t i = 0; i < N; ++i) m = ll[i] > m ? ll[i] : m;
            double s = 0;
            for (size_t i = 0; i < N; ++i) { const double t = W[i] * exp(ll[i] - m); s = s + t; }
            *loglik = *loglik + (m + log(s));
            orc_weight_add_log(N, W, ll, &ess);
        }
        if (ess_hist) ess_hist[it] = ess;
        if (resampled) resampled[it] = 0;
        if (ess < (double) N * threshold) {
            orc_resample(scheme, N, N, &er, W, rep);
            orc_rep_index(N, N, rep, idx);
            if (anc) memcpy(anc + it * N, idx, N * sizeof(uint64_t));
            if (resampled) resampled[it] = 1;
            orc_select_f64(N, 1, idx, x);
            for (size_t i = 0; i < N; ++i) W[i] = 1.0 / (double) N;
            ess = (double) N;
        }
    }
    if (x_out) memcpy(x_out, x, N * sizeof(double));
    if (W_out) memcpy(W_out, W, N * sizeof(double));
    free(x); free(W); free(ll); free(eps); free(rep); free(idx);
    return 0;
}

/* SMCEstimator::estimate (algorithm/smc.hpp:100-117): result_j =
 * sum_i W_i u(i, j) through cblas_dgemv (ColMajor NoTrans over the row-major
 * evaluations, ColMajor Trans over the column-major ones).  The reference
 * requires a BLAS (internal/cblas.hpp:75, 115-118), which fixes no summation
 * order; this restates the order of the reference BLAS's dgemv loops (alpha =
 * 1, beta = 0): a left fold over particles of the rounded products W_i u(i, j),
 * the same in both layouts. */
int orc_weighted_estimate(size_t n, size_t d, int col_major, const double *u, const double *w, double *out)
{
    for (size_t j = 0; j < d; ++j) {
        double s = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const double v = col_major ? u[j * n + i] : u[i * d + j];
            s = s + w[i] * v;
        }
        out[j] = s;
    }
    return 0;
}

/* Sequential left fold s_i = s_{i-1} + x_i from s_{-1} = s0 (the
 * std::accumulate / `accw += w[i]` loops of core/weight.hpp:221 and
 * algorithm/resample.hpp:395-403); prefix may be NULL. */
int orc_fold(size_t n, const double *x, double s0, double *prefix, double *final_value)
{
    double s = s0;
    for (size_t i = 0; i < n; ++i) {
        s = s + x[i];
        if (prefix) prefix[i] = s;
    }
    *final_value = s;
    return 0;
}

/* glibc's double log (0), exp (1) and sin/cos (2): the functions the
 * reference's transforms call (math/vmf.hpp:1008-1075). */
int orc_math_f64(int fn, size_t n, const double *x, double *y, double *y2)
{
    for (size_t i = 0; i < n; ++i) {
        switch (fn) {
            case 0: y[i] = log(x[i]); break;
            case 1: y[i] = exp(x[i]); break;
            default: y[i] = sin(x[i]); if (y2) y2[i] = cos(x[i]); break;
        }
    }
    return 0;
}

/* Kalman filter for the same model (not part of MCKL): exact log-likelihood
 * and its gradient with respect to (phi, sx, sy), prior x_0 ~ N(0, sd0^2) with
 * the stationary sd0 = sx / sqrt(1 - phi^2). Forward-mode derivatives. */
int orc_kalman_ar1(size_t T, const double *y, double phi, double sx, double sy,
    double *loglik, double *grad)
{
    double m = 0, P = sx * sx / (1 - phi * phi);
    double dm[3] = {0, 0, 0};
    double dP[3];
    dP[0] = sx * sx * 2 * phi / ((1 - phi * phi) * (1 - phi * phi));
    dP[1] = 2 * sx / (1 - phi * phi);
    dP[2] = 0;
    double ll = 0, g[3] = {0, 0, 0};
    for (size_t t = 1; t <= T; ++t) {
        /* predict */
        double mp = phi * m, Pp = phi * phi * P + sx * sx;
        double dmp[3], dPp[3];
        for (int k = 0; k < 3; ++k) { dmp[k] = phi * dm[k]; dPp[k] = phi * phi * dP[k]; }
        dmp[0] += m; dPp[0] += 2 * phi * P; dPp[1] += 2 * sx;
        /* innovation */
        const double S = Pp + sy * sy, v = y[t] - mp;
        double dS[3], dv[3];
        for (int k = 0; k < 3; ++k) { dS[k] = dPp[k]; dv[k] = -dmp[k]; }
        dS[2] += 2 * sy;
        ll += -0.5 * (log(2 * 3.14159265358979323846) + log(S) + v * v / S);
        for (int k = 0; k < 3; ++k) g[k] += -0.5 * (dS[k] / S + 2 * v * dv[k] / S - v * v * dS[k] / (S * S));
        /* update */
        const double Kg = Pp / S;
        double dK[3];
        for (int k = 0; k < 3; ++k) dK[k] = dPp[k] / S - Pp * dS[k] / (S * S);
        m = mp + Kg * v;
        P = (1 - Kg) * Pp;
        for (int k = 0; k < 3; ++k) {
            dm[k] = dmp[k] + dK[k] * v + Kg * dv[k];
            dP[k] = -dK[k] * Pp + (1 - Kg) * dPp[k];
        }
    }
    *loglik = ll;
    if (grad) { grad[0] = g[0]; grad[1] = g[1]; grad[2] = g[2]; }
    return 0;
}
