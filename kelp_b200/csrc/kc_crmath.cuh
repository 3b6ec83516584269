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
#endif
static const double h_log_inv[128] = KC_CR_LOG_INV;
static const double h_log_nlc_hi[128] = KC_CR_LOG_NLC_HI;
static const double h_log_nlc_lo[128] = KC_CR_LOG_NLC_LO;

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

// Correctly rounded log(x) for positive normal x (the RNG's uniforms are in
// [2^-33, 1)); other arguments take the library log.
KC_CR_HD double log_cr(double x) {
    const uint64_t ix = bits_of(x);
    const unsigned ex = (unsigned)((ix >> 52) & 0x7ff);
    if ((ix >> 63) || ex == 0 || ex == 0x7ff) return log(x);
    return log_dd(x).hi;
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

// Correctly rounded sin(x), cos(x) for |x| < 2^20 (the RNG's angles are in
// (0, 2 pi)); larger or non-finite arguments take the library functions.
KC_CR_HD void sincos_cr(double x, double* sn, double* cs) {
    if (!(fabs(x) < 0x1p20)) {
        *sn = sin(x);
        *cs = cos(x);
        return;
    }
    DD s, c;
    sincos_dd(x, s, c);
    *sn = s.hi;
    *cs = c.hi;
}

KC_CR_HD void sincos_cr_checked(double x, double* sn, double* cs, bool* ambiguous) {
    DD s, c;
    sincos_dd(x, s, c);
    *sn = s.hi;
    *cs = c.hi;
    *ambiguous = round_ambiguous(s, 0x1p-98) || round_ambiguous(c, 0x1p-98);
}

}  // namespace cr
}  // namespace kc
