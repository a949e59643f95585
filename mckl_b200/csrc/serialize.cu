// serialize.cu -- engine state in the reference's text form
// (CounterEngine's operator<< / operator>>, random/counter.hpp:235-272).
//
// The reference writes `M r_0 .. r_{M-1}` (the buffered block of M results),
// `Kc c_0 .. c_{Kc-1}` (the counter), the generator (Philox: its 2-word key;
// Threefry: the 8-word parameter array key[0..3], parity, tweak[0..1],
// tweak parity; ARS: its 4-word key) and the buffer index.  The buffer is a
// pure function of key and counter, so a save recomputes it (when the index
// says it is in use; an unused buffer is written as zeros) and a load checks
// it against the counter.
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mckl_b200.hpp"
#include "common.cuh"

namespace {

using mckl_b200::Geom;
using mckl_b200::geom;

// the block at the engine's counter, as M result words (u32 or u64)
std::vector<uint64_t> buffered_block(const mckl_b200_engine_t &e)
{
    const Geom g = geom(e.kind);
    std::vector<uint64_t> r(g.M);
    uint32_t w32[8] = {0};
    switch (e.kind) {
        case MCKL_B200_PHILOX4X32:
        case MCKL_B200_PHILOX4X32_64: {
            const uint32_t key[2] = {static_cast<uint32_t>(e.key[0]), static_cast<uint32_t>(e.key[1])};
            mckl_b200::detail::philox_block_host(e.ctr[0], e.ctr[1], key, w32);
            break;
        }
        case MCKL_B200_THREEFRY4X64:
        case MCKL_B200_THREEFRY4X64_64: {
            uint64_t w64[4];
            mckl_b200::detail::threefry_block_host(e.ctr, e.key, e.tweak, w64);
            for (int i = 0; i < 4; ++i) {
                w32[2 * i] = static_cast<uint32_t>(w64[i]);
                w32[2 * i + 1] = static_cast<uint32_t>(w64[i] >> 32);
            }
            break;
        }
        default: {
            const uint32_t key[4] = {static_cast<uint32_t>(e.key[0]), static_cast<uint32_t>(e.key[1]),
                static_cast<uint32_t>(e.key[2]), static_cast<uint32_t>(e.key[3])};
            mckl_b200::detail::ars_block_host(e.ctr[0], e.ctr[1], key, w32);
            break;
        }
    }
    for (int i = 0; i < g.M; ++i) {
        r[i] = g.rbytes == 4 ? w32[i] : (static_cast<uint64_t>(w32[2 * i]) | (static_cast<uint64_t>(w32[2 * i + 1]) << 32));
    }
    return r;
}

bool is_threefry(uint32_t k)
{
    return k == MCKL_B200_THREEFRY4X64 || k == MCKL_B200_THREEFRY4X64_64;
}

bool is_ars(uint32_t k)
{
    return k == MCKL_B200_ARS || k == MCKL_B200_ARS_64;
}

}  // namespace

using namespace mckl_b200;

extern "C" int mckl_b200_engine_save(const mckl_b200_engine_t *e, char *buf, size_t cap, size_t *len)
{
    MB_CHECK_ARG(e != nullptr && len != nullptr, "null argument");
    MB_CHECK_ARG(kind_valid(e->kind), "invalid engine kind");
    const Geom g = geom(e->kind);
    std::ostringstream os;
    const bool used = e->index < static_cast<uint32_t>(g.M);
    const std::vector<uint64_t> r = used ? buffered_block(*e) : std::vector<uint64_t>(g.M, 0);
    os << g.M;
    for (int i = 0; i < g.M; ++i) os << ' ' << r[i];
    os << ' ' << g.cwords;
    for (int i = 0; i < g.cwords; ++i) os << ' ' << e->ctr[i];
    if (is_threefry(e->kind)) {
        const uint64_t par4 = 0x1BD11BDAA9FC1A22ull ^ e->key[0] ^ e->key[1] ^ e->key[2] ^ e->key[3];
        os << " 8 " << e->key[0] << ' ' << e->key[1] << ' ' << e->key[2] << ' ' << e->key[3] << ' ' << par4 << ' '
           << e->tweak[0] << ' ' << e->tweak[1] << ' ' << (e->tweak[0] ^ e->tweak[1]);
    } else if (is_ars(e->kind)) {
        os << " 4";
        for (int i = 0; i < 4; ++i) os << ' ' << static_cast<uint32_t>(e->key[i]);
    } else {
        os << " 2 " << static_cast<uint32_t>(e->key[0]) << ' ' << static_cast<uint32_t>(e->key[1]);
    }
    os << ' ' << (e->index < static_cast<uint32_t>(g.M) ? e->index : static_cast<uint32_t>(g.M));
    const std::string s = os.str();
    *len = s.size();
    if (buf == nullptr) return MCKL_B200_OK;  // size query
    MB_CHECK_ARG(cap > s.size(), "buffer too small (see *len)");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return MCKL_B200_OK;
}

extern "C" int mckl_b200_engine_load(mckl_b200_engine_t *e, uint32_t kind, const char *text)
{
    MB_CHECK_ARG(e != nullptr && text != nullptr, "null argument");
    MB_CHECK_ARG(kind_valid(kind), "invalid engine kind");
    const Geom g = geom(kind);
    std::istringstream is(text);
    auto take = [&is](uint64_t &v) { return static_cast<bool>(is >> v); };
    uint64_t m = 0, kc = 0, kg = 0, idx = 0;
    mckl_b200_engine_t t{};
    t.kind = kind;
    std::vector<uint64_t> r;
    bool ok = take(m) && m == static_cast<uint64_t>(g.M);
    for (uint64_t i = 0; ok && i < m; ++i) {
        uint64_t v;
        ok = take(v);
        r.push_back(v);
    }
    ok = ok && take(kc) && kc == static_cast<uint64_t>(g.cwords);
    for (uint64_t i = 0; ok && i < kc; ++i) ok = take(t.ctr[i]);
    ok = ok && take(kg);
    if (ok && is_threefry(kind)) {
        uint64_t par[8];
        ok = kg == 8;
        for (int i = 0; ok && i < 8; ++i) ok = take(par[i]);
        if (ok) {
            for (int i = 0; i < 4; ++i) t.key[i] = par[i];
            t.tweak[0] = par[5];
            t.tweak[1] = par[6];
            ok = par[4] == (0x1BD11BDAA9FC1A22ull ^ par[0] ^ par[1] ^ par[2] ^ par[3]) &&
                 par[7] == (par[5] ^ par[6]);
        }
    } else if (ok) {
        const uint64_t want = is_ars(kind) ? 4 : 2;
        ok = kg == want;
        for (uint64_t i = 0; ok && i < kg; ++i) ok = take(t.key[i]) && t.key[i] <= 0xFFFFFFFFull;
    }
    ok = ok && take(idx) && idx <= static_cast<uint64_t>(g.M);
    MB_CHECK_ARG(ok, "not an engine state of this kind in the reference's text form");
    t.index = static_cast<uint32_t>(idx);
    if (t.index < static_cast<uint32_t>(g.M)) {
        MB_CHECK_ARG(buffered_block(t) == r,
            "the buffered results do not match the counter (only states the engine itself produced can be loaded)");
    }
    *e = t;
    return MCKL_B200_OK;
}
