// crmath.cuh -- double-precision log, exp and sin/cos evaluated in
// double-double arithmetic and rounded once, so the result is the correctly
// rounded value except when the exact result lies within ~2^-70 relative of
// a rounding midpoint.
//
// Why: the reference's transforms call glibc's log/exp/sin/cos, which are
// correctly rounded in all but rare cases.  CUDA's library versions are
// accurate to 1-2 ULP, and Box-Muller's sqrt(-2 log u) * sin(2 pi v) compounds
// those into 3-ULP differences.  Evaluating in double-double makes the device
// agree with the reference to within its own rounding.
//
// Methods (standard, written from the mathematics):
//   log: x = 2^e m, m in [1, 2); a 128-entry table gives inv ~ 1/m with
//        nine bits and -ln(inv) in double-double, r = m inv - 1 exactly,
//        log1p(r) by its series (|r| <= 2^-7); e ln2 with ln2 as a
//        double-double constant.
//   exp: x = k ln2 + r (Cody-Waite, three-part ln2), r/16 through a Taylor
//        series for expm1 in double-double, four squarings of 1 + expm1,
//        scaled by 2^k.
//   sin/cos: x = k pi/2 + r (Cody-Waite with four parts of pi/2, |x| < 1e5),
//        Taylor series of sin r and cos r (|r| <= pi/4) with the leading
//        terms in double-double; the quadrant picks signs and swaps.
// Constants are the exact double / double-double splits of ln 2, pi/2 and the
// series coefficients.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

// The same source compiles for the device (CUDA intrinsics, explicit
// round-to-nearest) and for a host check against the C library (plain
// operators; the host build must use -ffp-contract=off).
#if defined(__CUDACC__)
#define MB_HD __host__ __device__ __forceinline__
#else
#define MB_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define MB_ADD(a, b) __dadd_rn((a), (b))
#define MB_SUB(a, b) __dsub_rn((a), (b))
#define MB_MUL(a, b) __dmul_rn((a), (b))
#define MB_DIV(a, b) __ddiv_rn((a), (b))
#define MB_FMA(a, b, c) __fma_rn((a), (b), (c))
#define MB_RINT(a) rint(a)
#define MB_AS_BITS(x) __double_as_longlong(x)
#define MB_FROM_BITS(b) __longlong_as_double(b)
#define MB_LIB_SINCOS(x, s, c) ::sincos((x), (s), (c))
#else
#define MB_ADD(a, b) ((a) + (b))
#define MB_SUB(a, b) ((a) - (b))
#define MB_MUL(a, b) ((a) * (b))
#define MB_DIV(a, b) ((a) / (b))
#define MB_FMA(a, b, c) std::fma((a), (b), (c))
#define MB_RINT(a) std::rint(a)
#define MB_AS_BITS(x) ::mckl_b200::dd::host_bits(x)
#define MB_FROM_BITS(b) ::mckl_b200::dd::host_double(b)
#define MB_LIB_SINCOS(x, s, c) (*(s) = std::sin(x), *(c) = std::cos(x))
#endif

namespace mckl_b200 {
namespace dd {

#if !defined(__CUDA_ARCH__)
inline long long host_bits(double x)
{
    long long b;
    std::memcpy(&b, &x, sizeof(b));
    return b;
}
inline double host_double(long long b)
{
    double x;
    std::memcpy(&x, &b, sizeof(x));
    return x;
}
#endif

struct DD {
    double hi, lo;
};

MB_HD DD two_sum(double a, double b)
{
    const double s = MB_ADD(a, b);
    const double bb = MB_SUB(s, a);
    const double err = MB_ADD(MB_SUB(a, MB_SUB(s, bb)), MB_SUB(b, bb));
    return {s, err};
}

MB_HD DD fast_two_sum(double a, double b)
{
    const double s = MB_ADD(a, b);
    return {s, MB_SUB(b, MB_SUB(s, a))};
}

MB_HD DD two_prod(double a, double b)
{
    const double p = MB_MUL(a, b);
    return {p, MB_FMA(a, b, -p)};
}

MB_HD DD add(DD a, DD b)
{
    DD s = two_sum(a.hi, b.hi);
    const DD t = two_sum(a.lo, b.lo);
    s.lo = MB_ADD(s.lo, t.hi);
    s = fast_two_sum(s.hi, s.lo);
    s.lo = MB_ADD(s.lo, t.lo);
    return fast_two_sum(s.hi, s.lo);
}

MB_HD DD add_d(DD a, double b)
{
    DD s = two_sum(a.hi, b);
    s.lo = MB_ADD(s.lo, a.lo);
    return fast_two_sum(s.hi, s.lo);
}

MB_HD DD mul(DD a, DD b)
{
    DD p = two_prod(a.hi, b.hi);
    p.lo = MB_FMA(a.hi, b.lo, p.lo);
    p.lo = MB_FMA(a.lo, b.hi, p.lo);
    return fast_two_sum(p.hi, p.lo);
}

MB_HD DD mul_d(DD a, double b)
{
    DD p = two_prod(a.hi, b);
    p.lo = MB_FMA(a.lo, b, p.lo);
    return fast_two_sum(p.hi, p.lo);
}

// ---------------------------------------------------------------------------
constexpr double kLn2Hi = 0x1.62e42fefa39efp-1, kLn2Lo = 0x1.abc9e3b39803fp-56;
constexpr double kThirdHi = 0x1.5555555555555p-2, kThirdLo = 0x1.5555555555555p-56;
constexpr double kSqrt2 = 0x1.6a09e667f3bcdp+0;

// Reduction table of log: {inv_i, -ln(inv_i) hi, lo} (log_table.inc, written
// by gen_log_table.py).  Device copy in global memory (the lanes of a warp
// index it at random: a constant-bank copy would serialise them).
#if defined(__CUDACC__)
static __device__ const double kLogTab[128][3] = {
#include "log_table.inc"
};
#endif
#if !defined(__CUDA_ARCH__)
static const double kLogTabHost[128][3] = {
#include "log_table.inc"
};
#endif
#if defined(__CUDA_ARCH__)
#define MB_LOGTAB(i, k) __ldg(&kLogTab[(i)][(k)])
#else
#define MB_LOGTAB(i, k) kLogTabHost[(i)][(k)]
#endif

// Correctly rounded (see header) natural logarithm of a double.
// x = 2^e m, m in [1, 2); the top seven fraction bits pick inv_i ~ 1/m with
// nine significant bits, so r = m inv_i - 1 is exact (one fma) and
// |r| <= 2^-7; log x = e ln2 + (-ln inv_i) + log1p(r), with
// log1p(r) = r - r^2/2 + r^3 P(r), P the series sum_{n>=3} (-1)^(n+1) r^(n-3)/n
// to n = 12 in double, the rest in double-double.
MB_HD double log(double x)
{
    if (!(x > 0.0)) return x == 0.0 ? -MB_FROM_BITS(0x7ff0000000000000ll) : MB_FROM_BITS(0x7ff8000000000000ll);
    long long bits = MB_AS_BITS(x);
    int ex = static_cast<int>((bits >> 52) & 0x7ff);
    if (ex == 0x7ff) return x;  // +inf
    int e;
    if (ex == 0) {  // subnormal: scale into the normal range
        bits = MB_AS_BITS(MB_MUL(x, 0x1p54));
        ex = static_cast<int>((bits >> 52) & 0x7ff);
        e = ex - 1023 - 54;
    } else {
        e = ex - 1023;
    }
    const double m = MB_FROM_BITS((bits & 0x000fffffffffffffll) | 0x3ff0000000000000ll);
    const int i = static_cast<int>((bits >> 45) & 127);
    const double r = MB_FMA(m, MB_LOGTAB(i, 0), -1.0);  // exact
    double P = -0x1.5555555555555p-4;                   // -1/12
    P = MB_FMA(P, r, 0x1.745d1745d1746p-4);             // 1/11
    P = MB_FMA(P, r, -0x1.999999999999ap-4);            // -1/10
    P = MB_FMA(P, r, 0x1.c71c71c71c71cp-4);             // 1/9
    P = MB_FMA(P, r, -0x1.0000000000000p-3);            // -1/8
    P = MB_FMA(P, r, 0x1.2492492492492p-3);             // 1/7
    P = MB_FMA(P, r, -0x1.5555555555555p-3);            // -1/6
    P = MB_FMA(P, r, 0x1.999999999999ap-3);             // 1/5
    P = MB_FMA(P, r, -0x1.0000000000000p-2);            // -1/4
    P = MB_FMA(P, r, 0x1.5555555555555p-2);             // 1/3
    const DD r2 = two_prod(r, r);
    const double r3p = MB_MUL(MB_MUL(r2.hi, r), P);
    DD lp = two_sum(r, MB_MUL(r2.hi, -0.5));
    lp.lo = MB_ADD(lp.lo, MB_ADD(MB_MUL(r2.lo, -0.5), r3p));
    lp = fast_two_sum(lp.hi, lp.lo);
    const double ed = static_cast<double>(e);
    DD el = two_prod(ed, kLn2Hi);
    el.lo = MB_FMA(ed, kLn2Lo, el.lo);
    el = fast_two_sum(el.hi, el.lo);
    const DD res = add(add(el, DD{MB_LOGTAB(i, 1), MB_LOGTAB(i, 2)}), lp);
    return MB_ADD(res.hi, res.lo);
}

// ---------------------------------------------------------------------------
constexpr double kInvLn2 = 0x1.71547652b82fep+0;
constexpr double kLn2Cw0 = 0x1.62e42fefa3800p-1;  // 42 significant bits: k * kLn2Cw0 is exact
constexpr double kLn2Cw1 = 0x1.ef35793c76730p-45;
constexpr double kLn2Cw2 = 0x1.f97b57a079a19p-103;

MB_HD double scale2(double y, int k)
{
    if (k > 1023) {
        y = MB_MUL(y, 0x1p1023);
        k -= 1023;
        if (k > 1023) k = 1023;
    } else if (k < -1022) {
        y = MB_MUL(y, 0x1p-600);
        k += 600;
        if (k < -1022) k = -1022;
    }
    return MB_MUL(y, MB_FROM_BITS(static_cast<long long>(k + 1023) << 52));
}

// The accurate phase of exp: the double-double evaluation below, correctly
// rounded (see header) for normal results; results in the subnormal range are
// rounded twice.
MB_HD double exp_dd(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return MB_FROM_BITS(0x7ff0000000000000ll);
    if (x < -745.2) return 0.0;
    const double kd = MB_RINT(MB_MUL(x, kInvLn2));
    const int k = static_cast<int>(kd);
    const double r0 = MB_FMA(-kd, kLn2Cw0, x);  // exact
    const DD p1 = two_prod(-kd, kLn2Cw1);
    DD r = two_sum(r0, p1.hi);
    r.lo = MB_ADD(r.lo, p1.lo);
    r.lo = MB_FMA(-kd, kLn2Cw2, r.lo);
    r = fast_two_sum(r.hi, r.lo);
    const DD s{MB_MUL(r.hi, 0.0625), MB_MUL(r.lo, 0.0625)};
    const double sh = s.hi;
    // V = sum_{n=3}^{10} s^(n-3) / n!
    double V = 0x1.27e4fb7789f5cp-22;
    V = MB_FMA(V, sh, 0x1.71de3a556c734p-19);
    V = MB_FMA(V, sh, 0x1.a01a01a01a01ap-16);
    V = MB_FMA(V, sh, 0x1.a01a01a01a01ap-13);
    V = MB_FMA(V, sh, 0x1.6c16c16c16c17p-10);
    V = MB_FMA(V, sh, 0x1.1111111111111p-7);
    V = MB_FMA(V, sh, 0x1.5555555555555p-5);
    V = MB_FMA(V, sh, 0x1.5555555555555p-3);
    const DD inner = add_d(mul_d(s, V), 0.5);
    DD E = add(s, mul(mul(s, s), inner));  // expm1(s)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        E = add(DD{MB_MUL(E.hi, 2.0), MB_MUL(E.lo, 2.0)}, mul(E, E));  // expm1(2s)
    }
    const DD res = add_d(E, 1.0);
    return scale2(MB_ADD(res.hi, res.lo), k);
}

// Table of the quick phase: {hi, lo} of 2^(j/64), j = 0..63 (exp_table.inc,
// written by gen_exp_table.py), in global memory on the device like kLogTab.
#if defined(__CUDACC__)
static __device__ const double kExpTab[64][2] = {
#include "exp_table.inc"
};
#endif
#if !defined(__CUDA_ARCH__)
static const double kExpTabHost[64][2] = {
#include "exp_table.inc"
};
#endif
#if defined(__CUDA_ARCH__)
#define MB_EXPTAB(j, k) __ldg(&kExpTab[(j)][(k)])
#else
#define MB_EXPTAB(j, k) kExpTabHost[(j)][(k)]
#endif

// Ziv's rounding test: v.hi = RN(v.hi + v.lo), and v approximates a value
// to within 2^-62 relative.  True when every value that close rounds to v.hi,
// i.e. when v.hi is the correctly rounded value.  Below a power of two the
// gap to the next double is half as wide, so the test uses a quarter ulp on
// that side.  Zero and subnormal v.hi fail.
MB_HD bool ziv_ok(const DD &v)
{
    const long long b = MB_AS_BITS(v.hi) & 0x7fffffffffffffffll;  // |v.hi|
    const double u = MB_MUL(MB_FROM_BITS(b & 0x7ff0000000000000ll), 0x1p-52);  // ulp(v.hi)
    const bool inward = v.hi > 0.0 ? v.lo < 0.0 : v.lo > 0.0;
    const double half = ((b & 0x000fffffffffffffll) == 0 && inward) ? MB_MUL(u, 0.25) : MB_MUL(u, 0.5);
    const double d = v.lo < 0.0 ? -v.lo : v.lo;
    return MB_ADD(d, MB_MUL(MB_FROM_BITS(b), 0x1p-62)) < half;
}

constexpr double kExpInvL = 0x1.71547652b82fep+6;  // 64 / ln2
constexpr double kExpL1 = 0x1.62e42fefa0000p-7;    // ln2/64 to 36 bits: k * kExpL1 exact for |k| < 2^17
constexpr double kExpL2 = 0x1.cf79abc9e3b3ap-46;   // RN(ln2/64 - kExpL1)

// The quick phase of exp: Tang's table-driven method (P. T. P. Tang, ACM TOMS
// 15(2), 1989) with Ziv's rounding test (A. Ziv, ACM TOMS 17(3), 1991).
// x = k ln2/64 + r, k = 64 m + j, |r| <= ln2/128: the reduction is exact to
// 2^-78 (r_hi = x - k L1 exactly by Sterbenz's lemma, the k L2 term in a
// two_sum), exp(r) - 1 - r_hi is a degree-6 Taylor polynomial (truncation
// below 2^-65) plus r_lo, and 2^(j/64) (1 + r_hi + p) is summed with the
// leading product exact.  The total relative error is below 2^-64.4; the
// result is taken only when the double nearest to the approximation is the
// same for every value within 2^-62 relative of it, which makes it the
// correctly rounded exp(x) -- the value the accurate phase returns there
// too, as the exact result is then far from any rounding midpoint.  About
// one argument in 500 fails the test and goes to the accurate phase; so do
// arguments whose result is not a normal double (outside [-708, 709]).
MB_HD bool exp_quick(double x, double *y)
{
    if (!(x >= -708.0 && x <= 709.0)) return false;
    const double kd = MB_RINT(MB_MUL(x, kExpInvL));
    const int k = static_cast<int>(kd);
    const double rh0 = MB_FMA(-kd, kExpL1, x);  // exact
    const DD r = two_sum(rh0, MB_MUL(-kd, kExpL2));
    const double rh = r.hi;
    double P = 0x1.6c16c16c16c17p-10;         // 1/720
    P = MB_FMA(P, rh, 0x1.1111111111111p-7);  // 1/120
    P = MB_FMA(P, rh, 0x1.5555555555555p-5);  // 1/24
    P = MB_FMA(P, rh, 0x1.5555555555555p-3);  // 1/6
    P = MB_FMA(P, rh, 0.5);
    const double p = MB_FMA(MB_MUL(rh, rh), P, r.lo);  // exp(r) - 1 - r_hi
    const int j = k & 63, m = k >> 6;                   // k = 64 m + j, m = floor(k / 64)
    const double Th = MB_EXPTAB(j, 0), Tl = MB_EXPTAB(j, 1);
    const DD a = two_prod(Th, rh);
    const DD s = two_sum(Th, a.hi);
    const double t = MB_ADD(s.lo, MB_ADD(a.lo, MB_FMA(Th, p, MB_FMA(Tl, MB_ADD(rh, p), Tl))));
    const DD v = fast_two_sum(s.hi, t);
    if (!ziv_ok(v)) return false;
    *y = MB_MUL(v.hi, MB_FROM_BITS(static_cast<long long>(m + 1023) << 52));  // exact: a normal result
    return true;
}

// Correctly rounded (see header) exponential: the quick phase, else the
// accurate one.
MB_HD double exp(double x)
{
    double y;
    if (exp_quick(x, &y)) return y;
    return exp_dd(x);
}

// ---------------------------------------------------------------------------
constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;
constexpr double kPio2P1 = 0x1.921fb54400000p+0;  // 33 significant bits
constexpr double kPio2P2 = 0x1.0b4611a600000p-34; // 33 significant bits
constexpr double kPio2P3 = 0x1.3198a2e037073p-69;
constexpr double kPio2P4 = 0x1.129024e088a68p-123;

// The accurate phase of sincos: sin and cos of a double in double-double,
// correctly rounded (see header) for |x| < 1e5; larger arguments fall back to
// the device library.
MB_HD void sincos_dd(double x, double *sp, double *cp)
{
    if (!(x < 1e5 && x > -1e5)) {
        MB_LIB_SINCOS(x, sp, cp);
        return;
    }
    const double kd = MB_RINT(MB_MUL(x, kTwoOverPi));
    const double t = MB_FMA(-kd, kPio2P1, x);  // exact
    const DD p2 = two_prod(-kd, kPio2P2);
    DD r = two_sum(t, p2.hi);
    r.lo = MB_ADD(r.lo, p2.lo);
    r.lo = MB_FMA(-kd, kPio2P3, r.lo);
    r.lo = MB_FMA(-kd, kPio2P4, r.lo);
    r = fast_two_sum(r.hi, r.lo);
    const DD w = mul(r, r);
    const double wh = w.hi;
    // sin r = r (1 + w(-1/6 + w(1/120 + w(-1/5040 + w S4))))
    double S4 = -0x1.761b41316381ap-75;
    S4 = MB_FMA(S4, wh, 0x1.71b8ef6dcf572p-66);
    S4 = MB_FMA(S4, wh, -0x1.2f49b46814157p-57);
    S4 = MB_FMA(S4, wh, 0x1.952c77030ad4ap-49);
    S4 = MB_FMA(S4, wh, -0x1.ae7f3e733b81fp-41);
    S4 = MB_FMA(S4, wh, 0x1.6124613a86d09p-33);
    S4 = MB_FMA(S4, wh, -0x1.ae64567f544e4p-26);
    S4 = MB_FMA(S4, wh, 0x1.71de3a556c734p-19);
    DD sp3 = add(DD{-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73}, mul_d(w, S4));
    DD sp2 = add(DD{0x1.1111111111111p-7, 0x1.1111111111111p-63}, mul(w, sp3));
    DD sp1 = add(DD{-0x1.5555555555555p-3, -0x1.5555555555555p-57}, mul(w, sp2));
    const DD sn = mul(r, add_d(mul(w, sp1), 1.0));
    // cos r = 1 + w(-1/2 + w(1/24 + w(-1/720 + w C4)))
    double C4 = -0x1.0ce396db7f853p-70;
    C4 = MB_FMA(C4, wh, 0x1.e542ba4020225p-62);
    C4 = MB_FMA(C4, wh, -0x1.6827863b97d97p-53);
    C4 = MB_FMA(C4, wh, 0x1.ae7f3e733b81fp-45);
    C4 = MB_FMA(C4, wh, -0x1.93974a8c07c9dp-37);
    C4 = MB_FMA(C4, wh, 0x1.1eed8eff8d898p-29);
    C4 = MB_FMA(C4, wh, -0x1.27e4fb7789f5cp-22);
    C4 = MB_FMA(C4, wh, 0x1.a01a01a01a01ap-16);
    DD cp3 = add(DD{-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65}, mul_d(w, C4));
    DD cp2 = add(DD{0x1.5555555555555p-5, 0x1.5555555555555p-59}, mul(w, cp3));
    DD cp1 = add_d(mul(w, cp2), -0.5);
    const DD cs = add_d(mul(w, cp1), 1.0);
    const double s = MB_ADD(sn.hi, sn.lo);
    const double c = MB_ADD(cs.hi, cs.lo);
    const int q = static_cast<int>(static_cast<long long>(kd) & 3);
    switch (q) {
        case 0: *sp = s; *cp = c; break;
        case 1: *sp = c; *cp = -s; break;
        case 2: *sp = -s; *cp = -c; break;
        default: *sp = -c; *cp = s; break;
    }
}

// Table of the quick phase: {sin hi, lo, cos hi, lo} of j/64, j = 0..51
// (sincos_table.inc, written by gen_sincos_table.py), in global memory on the
// device like kLogTab.
#if defined(__CUDACC__)
static __device__ const double kSinCosTab[52][4] = {
#include "sincos_table.inc"
};
#endif
#if !defined(__CUDA_ARCH__)
static const double kSinCosTabHost[52][4] = {
#include "sincos_table.inc"
};
#endif
#if defined(__CUDA_ARCH__)
#define MB_SCTAB(j, k) __ldg(&kSinCosTab[(j)][(k)])
#else
#define MB_SCTAB(j, k) kSinCosTabHost[(j)][(k)]
#endif

// The quick phase of sincos: the accurate phase's reduction to r = x - k pi/2
// (a double-double, |r| <= pi/4), then |r| = j/64 + b with |b| <= 1/128
// (b_hi = |r_hi| - j/64 exactly, by Sterbenz's lemma for j >= 1) and the
// angle-addition formulas over the table's sin(j/64), cos(j/64):
//   sin|r| = S + C b_h + [S_l + C_l b_h + C b_l - S b_h b_l + S (cos b_h - 1) + C (sin b_h - b_h)]
//   cos|r| = C - S b_h + [C_l - S_l b_h - S b_l - C b_h b_l + C (cos b_h - 1) - S (sin b_h - b_h)]
// with the leading products exact (two_prod) and cos b_h - 1, sin b_h - b_h
// Taylor polynomials in b_h^2 (truncation below 2^-70 relative).  The
// bracketed tails are below 2^-14 of the results, so their roundings stay
// below 2^-64 relative.  Both values are taken only when Ziv's test passes for
// both (then each is the correctly rounded value, as the accurate phase's);
// otherwise the call goes to the accurate phase.
MB_HD bool sincos_quick(double x, double *sp, double *cp)
{
    if (!(x < 1e5 && x > -1e5)) return false;
    const double kd = MB_RINT(MB_MUL(x, kTwoOverPi));
    const double t = MB_FMA(-kd, kPio2P1, x);  // exact
    const DD p2 = two_prod(-kd, kPio2P2);
    DD r = two_sum(t, p2.hi);
    r.lo = MB_ADD(r.lo, p2.lo);
    r.lo = MB_FMA(-kd, kPio2P3, r.lo);
    r.lo = MB_FMA(-kd, kPio2P4, r.lo);
    r = fast_two_sum(r.hi, r.lo);
    const bool neg = r.hi < 0.0;
    const double ah = neg ? -r.hi : r.hi, bl = neg ? -r.lo : r.lo;  // |r| = ah + bl
    const double jd = MB_RINT(MB_MUL(ah, 64.0));
    if (!(jd <= 51.0)) return false;
    const int j = static_cast<int>(jd);
    const double bh = MB_SUB(ah, MB_MUL(jd, 0.015625));  // exact
    const double w = MB_MUL(bh, bh);
    double Pc = 0x1.a01a01a01a01ap-16;           // 1/40320
    Pc = MB_FMA(Pc, w, -0x1.6c16c16c16c17p-10);  // -1/720
    Pc = MB_FMA(Pc, w, 0x1.5555555555555p-5);    // 1/24
    Pc = MB_FMA(Pc, w, -0.5);
    double Ps = 0x1.71de3a556c734p-19;           // 1/362880
    Ps = MB_FMA(Ps, w, -0x1.a01a01a01a01ap-13);  // -1/5040
    Ps = MB_FMA(Ps, w, 0x1.1111111111111p-7);    // 1/120
    Ps = MB_FMA(Ps, w, -0x1.5555555555555p-3);   // -1/6
    const double cm1 = MB_MUL(w, Pc);             // cos b_h - 1
    const double smb = MB_MUL(bh, MB_MUL(w, Ps));  // sin b_h - b_h
    const double bbl = MB_MUL(bh, bl);
    const double Sh = MB_SCTAB(j, 0), Sl = MB_SCTAB(j, 1), Ch = MB_SCTAB(j, 2), Cl = MB_SCTAB(j, 3);
    const DD p = two_prod(Ch, bh);
    const DD sa = two_sum(Sh, p.hi);
    double ts = MB_FMA(Cl, bh, Sl);
    ts = MB_FMA(-Sh, bbl, ts);
    ts = MB_FMA(Ch, bl, ts);
    ts = MB_FMA(Ch, smb, ts);
    ts = MB_FMA(Sh, cm1, ts);
    ts = MB_ADD(MB_ADD(sa.lo, p.lo), ts);
    const DD sv = fast_two_sum(sa.hi, ts);
    const DD q = two_prod(Sh, bh);
    const DD ca = two_sum(Ch, -q.hi);
    double tc = MB_FMA(-Sl, bh, Cl);
    tc = MB_FMA(-Ch, bbl, tc);
    tc = MB_FMA(-Sh, bl, tc);
    tc = MB_FMA(-Sh, smb, tc);
    tc = MB_FMA(Ch, cm1, tc);
    tc = MB_ADD(MB_SUB(ca.lo, q.lo), tc);
    const DD cv = fast_two_sum(ca.hi, tc);
    if (!ziv_ok(sv) || !ziv_ok(cv)) return false;
    const double s = neg ? -sv.hi : sv.hi, c = cv.hi;
    switch (static_cast<int>(static_cast<long long>(kd) & 3)) {
        case 0: *sp = s; *cp = c; break;
        case 1: *sp = c; *cp = -s; break;
        case 2: *sp = -s; *cp = -c; break;
        default: *sp = -c; *cp = s; break;
    }
    return true;
}

// sin and cos of a double, correctly rounded (see header): the quick phase,
// else the accurate one.
MB_HD void sincos(double x, double *sp, double *cp)
{
    if (sincos_quick(x, sp, cp)) return;
    sincos_dd(x, sp, cp);
}

MB_HD double cos(double x)
{
    double s, c;
    sincos(x, &s, &c);
    return c;
}

MB_HD double sin(double x)
{
    double s, c;
    sincos(x, &s, &c);
    return s;
}

}  // namespace dd
}  // namespace mckl_b200
