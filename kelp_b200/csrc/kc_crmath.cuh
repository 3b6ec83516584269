// Correctly rounded natural logarithm and sine / cosine in double precision,
// for the counter RNG's Box-Muller draws (diffusion.py:233-249: r =
// sqrt(-2 log u1), g1 = r cos(2 pi u2), g2 = r sin(2 pi u2)), whose values
// must equal the reference's bit for bit.  The reference's Numba kernels call
// the host C library; these functions return the double nearest the exact
// value, so they agree with it wherever it rounds correctly (the inputs where
// it does not are the exception tables of kc_rng_exceptions.bin).
//
// Method (published, written here from the mathematics):
//  * double-double arithmetic -- Dekker's exact sum / product (Dekker 1971,
//    "A floating-point technique for extending the available precision"),
//    the product error by one fused multiply-add;
//  * log: table-driven reduction (Tang 1990, "Table-driven implementation of
//    the logarithm function in IEEE floating-point arithmetic"):
//    x = 2^e m, m in [0.6875, 1.375), r = m c_i - 1 exact, |r| < 2^-7,
//    log x = e ln2 - log c_i + log1p(r), log1p by its alternating series to
//    2^-105 in double-double;
//  * sin / cos: Cody-Waite reduction by pi/2 in three 53-bit parts (exact
//    first step by one fused multiply-add), then the Taylor series of sin and
//    cos on |r| <= pi/4 to 2^-105 in double-double (Cody & Waite 1980,
//    "Software Manual for the Elementary Functions");
//  * the double-double result (about 100 correct bits) is rounded once to
//    double, which is the correctly rounded value unless the exact value lies
//    within ~2^-98 (relative) of a rounding boundary (the rounding test of
//    Ziv 1991, "Fast evaluation of elementary mathematical functions with
//    correctly rounded last bit").  `log_cr_checked` / `sincos_cr_checked`
//    report that case; over all 2^32 uniforms the RNG can draw it never
//    occurs (gen_rng_exceptions.cpp counts it).
//
// Every operation is an explicit round-to-nearest intrinsic on the device and
// a plain IEEE operation on the host (compiled without contraction), so the
// host and device builds return the same bits.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "kc_crmath_tables.h"

#if defined(__CUDACC__)
#define KC_CR_HD __host__ __device__ __forceinline__
#else
#define KC_CR_HD inline
#endif

namespace kc {
namespace cr {

#if defined(__CUDACC__)
static __device__ const double g_log_inv[128] = KC_CR_LOG_INV;
static __device__ const double g_log_nlc_hi[128] = KC_CR_LOG_NLC_HI;
static __device__ const double g_log_nlc_lo[128] = KC_CR_LOG_NLC_LO;
static __device__ __align__(32) const double g_tab_sc[208] = KC_CR_TAB_SC;
#endif
static const double h_log_inv[128] = KC_CR_LOG_INV;
static const double h_log_nlc_hi[128] = KC_CR_LOG_NLC_HI;
static const double h_log_nlc_lo[128] = KC_CR_LOG_NLC_LO;
alignas(32) static const double h_tab_sc[208] = KC_CR_TAB_SC;

#if defined(__CUDA_ARCH__)
KC_CR_HD double add(double a, double b) { return __dadd_rn(a, b); }
KC_CR_HD double sub(double a, double b) { return __dsub_rn(a, b); }
KC_CR_HD double mul(double a, double b) { return __dmul_rn(a, b); }
KC_CR_HD double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
KC_CR_HD double log_inv(int i) { return __ldg(&g_log_inv[i]); }
KC_CR_HD double log_nlc_hi(int i) { return __ldg(&g_log_nlc_hi[i]); }
KC_CR_HD double log_nlc_lo(int i) { return __ldg(&g_log_nlc_lo[i]); }
KC_CR_HD uint64_t bits_of(double x) { return (uint64_t)__double_as_longlong(x); }
KC_CR_HD double from_bits(uint64_t b) { return __longlong_as_double((long long)b); }
// sin(j/64) hi, lo, cos(j/64) hi, lo
KC_CR_HD void tab_sc(int j, double& sh, double& sl, double& ch, double& cl) {
    const double2* p = reinterpret_cast<const double2*>(g_tab_sc) + 2 * j;
    const double2 a = __ldg(p), b = __ldg(p + 1);
    sh = a.x; sl = a.y; ch = b.x; cl = b.y;
}
#else
KC_CR_HD double add(double a, double b) { return a + b; }
KC_CR_HD double sub(double a, double b) { return a - b; }
KC_CR_HD double mul(double a, double b) { return a * b; }
KC_CR_HD double fma_(double a, double b, double c) { return std::fma(a, b, c); }
KC_CR_HD double log_inv(int i) { return h_log_inv[i]; }
KC_CR_HD double log_nlc_hi(int i) { return h_log_nlc_hi[i]; }
KC_CR_HD double log_nlc_lo(int i) { return h_log_nlc_lo[i]; }
KC_CR_HD uint64_t bits_of(double x) { uint64_t b; std::memcpy(&b, &x, 8); return b; }
KC_CR_HD double from_bits(uint64_t b) { double x; std::memcpy(&x, &b, 8); return x; }
KC_CR_HD void tab_sc(int j, double& sh, double& sl, double& ch, double& cl) {
    sh = h_tab_sc[4 * j]; sl = h_tab_sc[4 * j + 1]; ch = h_tab_sc[4 * j + 2]; cl = h_tab_sc[4 * j + 3];
}
#endif

struct DD {
    double hi, lo;
};

// a + b = s + e exactly (any magnitudes)
KC_CR_HD DD two_sum(double a, double b) {
    const double s = add(a, b);
    const double bb = sub(s, a);
    const double e = add(sub(a, sub(s, bb)), sub(b, bb));
    return {s, e};
}

// a + b = s + e exactly when |a| >= |b| (or a == 0)
KC_CR_HD DD fast_two_sum(double a, double b) {
    const double s = add(a, b);
    return {s, sub(b, sub(s, a))};
}

// a * b = p + e exactly (no underflow)
KC_CR_HD DD two_prod(double a, double b) {
    const double p = mul(a, b);
    return {p, fma_(a, b, -p)};
}

// double-double sum, relative error ~2^-106 (both parts' errors carried)
KC_CR_HD DD dd_add(DD x, DD y) {
    const DD s = two_sum(x.hi, y.hi);
    const DD t = two_sum(x.lo, y.lo);
    const DD u = fast_two_sum(s.hi, add(s.lo, t.hi));
    return fast_two_sum(u.hi, add(u.lo, t.lo));
}

// double-double product, relative error ~2^-104
KC_CR_HD DD dd_mul(DD x, DD y) {
    const DD p = two_prod(x.hi, y.hi);
    const double cross = fma_(x.hi, y.lo, mul(x.lo, y.hi));
    return fast_two_sum(p.hi, add(p.lo, cross));
}

// Horner evaluation of sum_k (H[k] + L[k]) t^k, k = 0..N-1, in double-double
template <int N>
KC_CR_HD DD horner(const double (&H)[N], const double (&L)[N], DD t) {
    DD p = {H[N - 1], L[N - 1]};
#pragma unroll
    for (int k = N - 2; k >= 0; --k) p = dd_add(dd_mul(p, t), DD{H[k], L[k]});
    return p;
}

// The double-double v rounds to v.hi (the last step was a fast two-sum); the
// exact value rounds to the same double unless it may lie across the rounding
// boundary nearest v: |v.lo| within rel * |v.hi| of half an ulp of v.hi.
KC_CR_HD bool round_ambiguous(DD v, double rel) {
    if (v.hi == 0.0 || !(fabs(v.hi) < 1e300)) return false;
    const uint64_t b = bits_of(fabs(v.hi));
    const double ulp = sub(from_bits(b + 1), from_bits(b));
    return fabs(sub(fabs(v.lo), mul(0.5, ulp))) <= mul(rel, fabs(v.hi));
}

// log(x) to ~2^-100 as a double-double, for positive normal x
KC_CR_HD DD log_dd(double x) {
    const uint64_t ix = bits_of(x);
    int e = (int)((ix >> 52) & 0x7ff) - 1023;
    const int i = (int)((ix >> 45) & 127);   // top 7 mantissa bits
    double m = from_bits((ix & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);   // [1, 2)
    if (i >= 48) {   // m in [0.6875, 1)
        m = mul(m, 0.5);
        e += 1;
    }
    const double c = log_inv(i);
    const DD p = two_prod(m, c);
    const DD r = two_sum(sub(p.hi, 1.0), p.lo);   // m c - 1 exactly (p.hi - 1 is exact: p.hi in [0.5, 2])
    constexpr double L1H[16] = KC_CR_L1P_HI;
    constexpr double L1L[16] = KC_CR_L1P_LO;
    const DD l1p = dd_mul(r, horner<16>(L1H, L1L, r));
    const double ed = (double)e;
    DD acc = two_prod(ed, kCrLn2_2);
    acc = dd_add(DD{mul(ed, kCrLn2_1), 0.0}, DD{acc.hi, add(acc.lo, mul(ed, kCrLn2_3))});   // e ln2 (e * ln2_1 exact)
    acc = dd_add(acc, DD{log_nlc_hi(i), log_nlc_lo(i)});
    return dd_add(acc, l1p);
}

// Fast path of log (Ziv's first step): the same reduction, then
// log1p(r) = r - r^2/2 + r^3 Q(r), the first two terms exact as
// double-doubles and Q (degree 8, to r^11/11) in double, summed by exact
// two-sums.  Absolute error below 2^-74 (the r^3 Q term's evaluation); the
// result is at least 2^-8 in magnitude unless it is log1p(r) itself, whose
// error is relative to r, so the relative error stays below 2^-66.  Returns
// the double-double; round_ambiguous(v, 2^-63) decides whether it rounds
// like the exact value.
KC_CR_HD DD log_fast(double x) {
    const uint64_t ix = bits_of(x);
    int e = (int)((ix >> 52) & 0x7ff) - 1023;
    const int i = (int)((ix >> 45) & 127);
    double m = from_bits((ix & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (i >= 48) {
        m = mul(m, 0.5);
        e += 1;
    }
    const DD p = two_prod(m, log_inv(i));
    const DD r = two_sum(sub(p.hi, 1.0), p.lo);   // m c - 1 exactly
    const DD rr = two_prod(r.hi, r.hi);
    const double rh = r.hi;
    double q = fma_(rh, 1.0 / 11.0, -0.1);
    q = fma_(rh, q, 1.0 / 9.0);
    q = fma_(rh, q, -0.125);
    q = fma_(rh, q, 1.0 / 7.0);
    q = fma_(rh, q, -1.0 / 6.0);
    q = fma_(rh, q, 0.2);
    q = fma_(rh, q, -0.25);
    q = fma_(rh, q, 1.0 / 3.0);
    const double tail = mul(mul(rr.hi, rh), q);
    const double ed = (double)e;
    const double half = mul(-0.5, rr.hi);   // exact
    double small = add(mul(ed, kCrLn2_2), log_nlc_lo(i));
    small = add(small, r.lo);
    small = add(small, mul(-0.5, rr.lo));
    small = sub(small, mul(rh, r.lo));
    small = add(small, tail);
    small = add(small, mul(ed, kCrLn2_3));
    const DD s1 = two_sum(mul(ed, kCrLn2_1), log_nlc_hi(i));   // e * ln2_1 exact
    const DD s2 = two_sum(s1.hi, rh);
    const DD s3 = two_sum(s2.hi, half);
    const double lo = add(add(add(s1.lo, s2.lo), s3.lo), small);
    return fast_two_sum(s3.hi, lo);
}

// The double-double second steps, out of line on the device: they run for a
// few arguments in a thousand, and one copy keeps the callers' code small.
#if defined(__CUDACC__)
#define KC_CR_SLOW static __host__ __device__ __noinline__
#else
#define KC_CR_SLOW static inline
#endif
KC_CR_SLOW double log_slow(double x) { return log_dd(x).hi; }

// Correctly rounded log(x) for positive normal x (the RNG's uniforms are in
// [2^-33, 1)); other arguments take the library log.  The fast path decides
// all but ~0.02 % of arguments; the rest take the double-double path.
KC_CR_HD double log_cr(double x) {
    const uint64_t ix = bits_of(x);
    const unsigned ex = (unsigned)((ix >> 52) & 0x7ff);
    if ((ix >> 63) || ex == 0 || ex == 0x7ff) return log(x);
    const DD v = log_fast(x);
    if (!round_ambiguous(v, 0x1p-63)) return v.hi;
    return log_slow(x);
}

KC_CR_HD double log_cr_checked(double x, bool* ambiguous) {
    const DD v = log_dd(x);
    *ambiguous = round_ambiguous(v, 0x1p-98);
    return v.hi;
}

// sin / cos of x (|x| < 2^20) as double-doubles, by quadrant
KC_CR_HD void sincos_dd(double x, DD& s, DD& c) {
    const double kd = rint(mul(x, kCrTwoOverPi));
    DD r = {x, 0.0};
    if (kd != 0.0) {
        const double rh = fma_(-kd, kCrPio2_1, x);   // exact: a multiple of 2^-52 below 1 in magnitude
        const DD p2 = two_prod(kd, kCrPio2_2);
        r = dd_add(DD{rh, 0.0}, DD{-p2.hi, -p2.lo});
        r = dd_add(r, DD{-mul(kd, kCrPio2_3), 0.0});
    }
    constexpr double SH[15] = KC_CR_SIN_HI;
    constexpr double SL[15] = KC_CR_SIN_LO;
    constexpr double CH[15] = KC_CR_COS_HI;
    constexpr double CL[15] = KC_CR_COS_LO;
    const DD t = dd_mul(r, r);
    const DD sr = dd_mul(r, horner<15>(SH, SL, t));
    const DD cr = horner<15>(CH, CL, t);
    const int q = (int)((long long)kd & 3);
    if (q == 0) { s = sr; c = cr; }
    else if (q == 1) { s = cr; c = DD{-sr.hi, -sr.lo}; }
    else if (q == 2) { s = DD{-sr.hi, -sr.lo}; c = DD{-cr.hi, -cr.lo}; }
    else { s = DD{-cr.hi, -cr.lo}; c = sr; }
}

// Fast path of sin / cos (|x| < 2^20): the Cody-Waite reduction r = x - k
// pi/2 as a double-double, then r = a + t with a = j/64 from a table of
// sin a, cos a (double-double records) and |t| <= 1/128 (t's high part
// exact by Sterbenz's lemma); sin r = sin a cos t + cos a sin t, cos r = cos a
// cos t - sin a sin t with the a-terms, a*t and a*t^2/2 products exact
// (two-products) and the t^3 .. t^8 terms in double.  Absolute error below
// 2^-73; |sin r| >= 2^-7 unless a = 0 (then the error is relative to t) and
// |cos r| >= 0.7, so the relative error stays below 2^-66.  Outputs the
// double-doubles of sin x and cos x.
KC_CR_HD void sincos_fast(double x, DD& s, DD& c) {
    const double kd = rint(mul(x, kCrTwoOverPi));
    double rh = x, rl = 0.0;
    if (kd != 0.0) {
        const double r0 = fma_(-kd, kCrPio2_1, x);   // exact
        const DD p2 = two_prod(kd, kCrPio2_2);
        const DD r1 = two_sum(r0, -p2.hi);
        const DD r2 = fast_two_sum(r1.hi, sub(sub(r1.lo, p2.lo), mul(kd, kCrPio2_3)));
        rh = r2.hi;
        rl = r2.lo;
    }
    const double jd = rint(mul(rh, 64.0));
    const int ja = (int)fabs(jd);
    double sh, sl, ch, cl;
    tab_sc(ja, sh, sl, ch, cl);
    if (jd < 0.0) { sh = -sh; sl = -sl; }
    const double th = sub(rh, mul(jd, 0.015625));   // exact
    const double tl = rl;
    const DD tt = two_prod(th, th);
    const double u = tt.hi;
    const double ttl = add(tt.lo, mul(mul(2.0, th), tl));
    // sin t - t and cos t - 1 + t^2/2
    const double s3 = mul(mul(th, u), fma_(u, fma_(u, -1.0 / 5040.0, 1.0 / 120.0), -1.0 / 6.0));
    const double c4 = mul(mul(u, u), fma_(u, fma_(u, 1.0 / 40320.0, -1.0 / 720.0), 1.0 / 24.0));
    const double half = mul(-0.5, u), half_l = mul(-0.5, ttl);   // -t^2/2
    {   // sin r = sin a + cos a t - sin a t^2/2 + sin a c4 + cos a s3
        const DD b = two_prod(ch, th);
        const DD q = two_prod(sh, half);
        double small = add(add(sl, b.lo), q.lo);
        small = add(small, mul(ch, tl));
        small = add(small, mul(cl, th));
        small = add(small, mul(sh, half_l));
        small = add(small, mul(sl, half));
        small = add(small, mul(sh, c4));
        small = add(small, mul(ch, s3));
        const DD s1 = two_sum(sh, b.hi);
        const DD s2 = two_sum(s1.hi, q.hi);
        s = fast_two_sum(s2.hi, add(add(s1.lo, s2.lo), small));
    }
    {   // cos r = cos a - sin a t - cos a t^2/2 + cos a c4 - sin a s3
        const DD b = two_prod(-sh, th);
        const DD q = two_prod(ch, half);
        double small = add(add(cl, b.lo), q.lo);
        small = sub(small, mul(sh, tl));
        small = sub(small, mul(sl, th));
        small = add(small, mul(ch, half_l));
        small = add(small, mul(cl, half));
        small = add(small, mul(ch, c4));
        small = sub(small, mul(sh, s3));
        const DD c1 = two_sum(ch, b.hi);
        const DD c2 = two_sum(c1.hi, q.hi);
        c = fast_two_sum(c2.hi, add(add(c1.lo, c2.lo), small));
    }
    const int qd = (int)((long long)kd & 3);
    const DD sr = s, cr = c;
    if (qd == 1) { s = cr; c = DD{-sr.hi, -sr.lo}; }
    else if (qd == 2) { s = DD{-sr.hi, -sr.lo}; c = DD{-cr.hi, -cr.lo}; }
    else if (qd == 3) { s = DD{-cr.hi, -cr.lo}; c = sr; }
}

KC_CR_SLOW void sincos_slow(double x, double* sn, double* cs) {
    DD s, c;
    sincos_dd(x, s, c);
    *sn = s.hi;
    *cs = c.hi;
}

// Correctly rounded sin(x), cos(x) for |x| < 2^20 (the RNG's angles are in
// (0, 2 pi)); larger or non-finite arguments take the library functions.
// The fast path decides all but ~0.4 % of arguments; the rest take the
// double-double path.
KC_CR_HD void sincos_cr(double x, double* sn, double* cs) {
    if (!(fabs(x) < 0x1p20)) {
        *sn = sin(x);
        *cs = cos(x);
        return;
    }
    DD s, c;
    sincos_fast(x, s, c);
    if (round_ambiguous(s, 0x1p-63) || round_ambiguous(c, 0x1p-63)) {
        sincos_slow(x, sn, cs);
        return;
    }
    *sn = s.hi;
    *cs = c.hi;
}

KC_CR_HD double cos_cr(double x) {
    double sn, cs;
    sincos_cr(x, &sn, &cs);
    return cs;
}

// Out-of-line entry points for the step kernels: the double-double
// temporaries of the correctly rounded paths then live in the callee instead
// of raising the register pressure of a large kernel body.
#ifndef KC_CR_OUTLINE
#define KC_CR_OUTLINE 1
#endif
#if defined(__CUDACC__)
#if KC_CR_OUTLINE
#define KC_CR_K __device__ __noinline__ static
#else
#define KC_CR_K __device__ __forceinline__ static
#endif
KC_CR_K double cos_cr_k(double x) { return cos_cr(x); }
KC_CR_K double2 sincos_cr_k(double x) {
    double2 r;
    sincos_cr(x, &r.x, &r.y);
    return r;
}
#endif

KC_CR_HD void sincos_cr_checked(double x, double* sn, double* cs, bool* ambiguous) {
    DD s, c;
    sincos_dd(x, s, c);
    *sn = s.hi;
    *cs = c.hi;
    *ambiguous = round_ambiguous(s, 0x1p-98) || round_ambiguous(c, 0x1p-98);
}

}  // namespace cr
}  // namespace kc
