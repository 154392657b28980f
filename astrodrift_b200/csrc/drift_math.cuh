// drift_math.cuh -- FP64 special powers used on the integration path.
//
// The reference evaluates pow(r2, -1.5) in every force call, pow(err, 1/8) in
// the DOP853 controller and pow(x, 1.5) in the Miyamoto-Nagai disk, all
// through glibc's pow, which returns the correctly rounded result except in
// rare near-halfway cases.  These routines compute the same powers from IEEE
// sqrt / rsqrt and division plus one Newton correction carried in double-double
// (two-term) arithmetic, so the result is the correctly rounded value unless
// the exact power lies within about 2^-50 ulp of a rounding boundary.  They
// are written from the algebra below; no vendor math code is reproduced.
//
//   x^(3/2):  s = RN(sqrt x), e = x - s^2 exactly (one fma), so
//             sqrt x = s + e/(2s) + O(e^2) and x^(3/2) = x s + x e/(2s)
//             = x s + e s / 2 (1 + O(2^-52)).
//   x^(-3/2): r0 = y^3 with y a Newton-refined rsqrt estimate is within a
//             few ulps; one Newton step on
//             r^-2 = x^3 gives r = r0 (1 + delta / 2) with
//             delta = 1 - r0^2 x^3 formed in double-double (x^3 and r0^2
//             as exact products), leaving an error of order delta^2.
//   x^(1/8):  y0 = sqrt(sqrt(sqrt x)) is within about one ulp; one Newton
//             step on y^8 = x with y0^8 formed in double-double gives
//             y = y0 (1 - (y0^8 - x) / (8 x)).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "drift_math_tables.h"

// 1: the translation unit reproduces the reference's rounding (see
// drift_kernels_exact.cu); 0: multiply-add contraction and a-few-ulp powers.
#ifndef DRIFT_EXACT_ARITH
#define DRIFT_EXACT_ARITH 1
#endif

namespace drift {

// Exact product: a * b == hi + lo.
__device__ __forceinline__ void two_prod(double a, double b, double &hi, double &lo)
{
    hi = a * b;
    lo = fma(a, b, -hi);
}

// x^(3/2) as an unevaluated sum hi + lo, valid for x in [1e-200, 1e200].
__device__ __forceinline__ void pow_1p5_dd(double x, double &hi, double &lo)
{
    double s = sqrt(x);
    double e = fma(-s, s, x);
    two_prod(x, s, hi, lo);
    lo = fma(0.5 * e, s, lo);
}

__device__ __forceinline__ bool in_fast_range(double x)
{
    return __builtin_expect(x > 1e-200 && x < 1e200, 1);
}

// 1/x for x in [1e-300, 1e300] without the division's special-case branch:
// hardware estimate (PTX rcp.approx.ftz.f64) and two Newton steps
// r <- r (2 - x r), within about an ulp of the rounded quotient.  Used only
// where the reference's rounding need not be reproduced.
__device__ __forceinline__ double fast_rcp(double x)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = r * fma(-x, r, 2.0);
    r = r * fma(-x, r, 2.0);
    return r;
}

// x^(3/2), rounded to nearest (pow(x, 1.5) semantics for x >= 0).
static __device__ __noinline__ double pow_1p5_rare(double x);

__device__ __forceinline__ double pow_1p5(double x)
{
    if (in_fast_range(x)) {
        double hi, lo;
        pow_1p5_dd(x, hi, lo);
        return hi + lo;
    }
    return pow_1p5_rare(x);
}

// Arguments outside [1e-200, 1e200], out of line like pow_m1p5_rare.
static __device__ __noinline__ double pow_1p5_rare(double x)
{
    if (x == 0.0) return 0.0;
    if (!(x >= 0.0)) return __longlong_as_double(0x7ff8000000000000LL);  // NaN
    if (isinf(x)) return x;
    // Rescale by an even power of two: x = m 4^k, x^(3/2) = m^(3/2) 8^k.
    int k = (ilogb(x)) / 2;
    double m = scalbn(x, -2 * k);
    double hi, lo;
    pow_1p5_dd(m, hi, lo);
    return scalbn(hi + lo, 3 * k);
}

// Valid for x in [1e-90, 1e90] (x^3 and its low part stay normal).
__device__ __forceinline__ double pow_m1p5_core(double x)
{
    // Hardware estimate (PTX rsqrt.approx.f64, about 2^-23 relative error on
    // normal inputs) refined by two Newton steps y <- y (3 - x y^2) / 2 to a
    // few ulps; the double-double step below then rounds correctly.
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    y = y * fma(-0.5 * x, y * y, 1.5);
    y = y * fma(-0.5 * x, y * y, 1.5);
    double r0 = y * y * y;
    double a, al, b, bl, c, cl, p, pl;
    two_prod(x, x, a, al);      // x^2
    two_prod(a, x, b, bl);      // x^3 = b + bl
    bl = fma(al, x, bl);
    two_prod(r0, r0, c, cl);    // r0^2 = c + cl
    two_prod(c, b, p, pl);      // r0^2 x^3 = p + pl
    pl = fma(c, bl, fma(cl, b, pl));
    double delta = (1.0 - p) - pl;
    return fma(r0, 0.5 * delta, r0);
}

// x^(-3/2), rounded to nearest (pow(x, -1.5) semantics, including the
// special values: +-0 -> +inf, +inf -> +0, x < 0 -> NaN).
//
// The arguments outside (1e-90, 1e90) take an out-of-line path: the force
// is inlined at every stage of a step, and one shared copy of the rescaling
// keeps it out of each copy's instruction stream.
static __device__ __noinline__ double pow_m1p5_rare(double x)
{
    if (x == 0.0) return __longlong_as_double(0x7ff0000000000000LL);  // +inf
    if (!(x >= 0.0)) return __longlong_as_double(0x7ff8000000000000LL);
    if (isinf(x)) return 0.0;
    int k = (ilogb(x)) / 2;
    double m = scalbn(x, -2 * k);
    return scalbn(pow_m1p5_core(m), -3 * k);
}

__device__ __forceinline__ double pow_m1p5(double x)
{
    if (__builtin_expect(x > 1e-90 && x < 1e90, 1)) return pow_m1p5_core(x);
    return pow_m1p5_rare(x);
}

// x^(1/8), rounded to nearest (pow(x, 0.125) semantics for the values the
// controller produces: 0 -> 0, +inf -> +inf, NaN and x < 0 -> NaN).
__device__ __forceinline__ double root8(double x)
{
    double y0 = sqrt(sqrt(sqrt(x)));
    if (__builtin_expect(!(x > 1e-280 && x < 1e300), 0)) return y0;
    double a_h, a_l, b_h, b_l, c_h, c_l;
    two_prod(y0, y0, a_h, a_l);                 // y0^2
    two_prod(a_h, a_h, b_h, b_l);               // y0^4
    b_l = fma(2.0 * a_h, a_l, b_l);
    two_prod(b_h, b_h, c_h, c_l);               // y0^8
    c_l = fma(2.0 * b_h, b_l, c_l);
    double delta = ((c_h - x) + c_l) / x;       // y0^8 / x - 1
    return fma(y0, -0.125 * delta, y0);
}

// ---- few-ulp variants for the contraction unit -------------------------
// Without the double-double correction: y = rsqrt(x) refined by two Newton
// steps is within about an ulp of x^-1/2, and y^3 within a few ulps of
// x^-3/2; sqrt(x) x and sqrt(sqrt(sqrt(x))) likewise.  The contraction unit
// already departs from the reference's rounding in every multiply-add, so
// these save the correction's dozen FP64 instructions per call.
__device__ __forceinline__ double pow_m1p5_few_ulp(double x)
{
    if (__builtin_expect(x > 1e-90 && x < 1e90, 1)) {
        // y = x^-1/2 (1 + d) from the hardware estimate; with
        // e = 1 - x y^2 = 1 - (1 + d)^2 the power is
        // x^-3/2 = y^3 (1 - e)^-3/2 = y^3 (1 + 3/2 e + 15/8 e^2 + 35/16 e^3 + O(e^4)),
        // one correction of depth 6 instead of two Newton steps and a cube.
        double y;
        asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
        const double e = fma(-x * y, y, 1.0);
        const double y3 = y * (y * y);
        return fma(y3, e * fma(fma(2.1875, e, 1.875), e, 1.5), y3);
    }
    return pow_m1p5_rare(x);
}

__device__ __forceinline__ double pow_1p5_few_ulp(double x)
{
    if (in_fast_range(x)) return x * sqrt(x);
    return pow_1p5_rare(x);
}

__device__ __forceinline__ double root8_few_ulp(double x) { return sqrt(sqrt(sqrt(x))); }

// Natural log and exp for the contraction unit, from their series (no
// vendor code): each call site inlines about half the instructions of the
// library functions, which matters where a force is inlined at every stage.
//   log x = k ln2 + 2 atanh(t),  x = 2^k m with m in [sqrt(1/2), sqrt(2)),
//           t = (m - 1) / (m + 1), |t| <= 0.1716, atanh t = sum_j t^(2j+1) / (2j+1);
//           terms to j = 10 leave less than 2^-55 of the sum.
//   exp x = 2^k e^r,  k = rint(x / ln2), r = x - k ln2 with ln2 in two parts,
//           |r| <= 0.3466, e^r = sum_{n <= 13} r^n / n! (remainder < 2^-56 of e^r).
// Within a few ulps for normal positive x (log) and |x| < 708 (exp); every
// other argument takes the library function out of line.
constexpr double LN2_HI = 0.6931471805599453;
constexpr double LN2_LO = 2.3190468138462996e-17;
constexpr double LOG2_E = 1.4426950408889634;

static __device__ __noinline__ double log_rare(double x) { return log(x); }
static __device__ __noinline__ double exp_rare(double x) { return exp(x); }

__device__ __forceinline__ double log_few_ulp(double x)
{
    if (!(x >= 2.2250738585072014e-308 && x <= 1.7976931348623157e308)) return log_rare(x);
    const long long bits = __double_as_longlong(x);
    int k = (int)(bits >> 52) - 1023;
    double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);  // [1, 2)
    if (m > 1.4142135623730951) {
        m *= 0.5;
        k += 1;
    }
    const double t = (m - 1.0) * fast_rcp(m + 1.0);
    const double z = t * t;
    double p = 1.0 / 21.0;
    p = fma(p, z, 1.0 / 19.0);
    p = fma(p, z, 1.0 / 17.0);
    p = fma(p, z, 1.0 / 15.0);
    p = fma(p, z, 1.0 / 13.0);
    p = fma(p, z, 1.0 / 11.0);
    p = fma(p, z, 1.0 / 9.0);
    p = fma(p, z, 1.0 / 7.0);
    p = fma(p, z, 1.0 / 5.0);
    p = fma(p, z, 1.0 / 3.0);
    const double lm = 2.0 * fma(t * z, p, t);  // 2 (t + t^3 p)
    const double kd = (double)k;
    return fma(kd, LN2_HI, fma(kd, LN2_LO, lm));
}

__device__ __forceinline__ double exp_few_ulp(double x)
{
    if (!(fabs(x) < 708.0)) return exp_rare(x);
    const double kd = rint(x * LOG2_E);
    const double r = fma(-kd, LN2_LO, fma(-kd, LN2_HI, x));
    double p = 1.0 / 6227020800.0;          // 1/13!
    p = fma(p, r, 1.0 / 479001600.0);       // 1/12!
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    return p * __longlong_as_double((long long)((int)kd + 1023) << 52);
}

// ---- table-driven log and exp for the contraction unit's Bovy force ----
// The tables (drift_math_tables.h, generated with 60-digit arithmetic) are
// staged in shared memory beside the bulge table; one call reads two (log)
// or one (exp) entry at a per-lane index.
//   log x = k ln2 + L_i + log1p(r),  x = 2^k m, m in [1, 2), i = the top 7
//           bits of m's fraction, r = m * inv_c_i - 1 (one fused multiply-add)
//           with inv_c_i = RN(1 / (1 + i/128)) and L_i = RN(-ln inv_c_i), so
//           |r| < 1/128 and log1p(r) needs terms to r^8 (the next one is
//           below 2^-56 of r).
//   exp x = 2^e T_j e^r,  x = (64 e + j) ln2 / 64 + r with ln2 / 64 in two
//           parts, |r| <= ln2 / 128, T_j = RN(2^(j/64)), e^r - 1 to r^5
//           (the remainder is below 2^-54).
// exp is within a few ulps for |x| < 708; log within a few ulps for normal
// x >= 1 and within about 1e-16 absolute below 1 (near 1 from below the
// k ln2 and L_i terms cancel), which is what its uses need: the halo's
// ln(1 + u) and the bulge's x^s = exp(s ln x).  Other arguments take the
// library function out of line.
constexpr int MATH_TABLE_DOUBLES = 2 * LOG_TABLE_N + EXP_TABLE_N;
constexpr int MATH_LOG_PAIRS = 0;  // (inv_c_i, L_i) pairs, 16-byte aligned
constexpr int MATH_EXP_T = 2 * LOG_TABLE_N;
// ln2 / 64 split so that k * LN2_64_HI is exact for |k| < 2^17
constexpr double LN2_64_HI = 0x1.62e42fefa0000p-7;
constexpr double LN2_64_LO = 0x1.cf79abc9e3b3ap-46;
constexpr double INV_LN2_64 = 0x1.71547652b82fep+6;  // 64 / ln2

// Entry i of the math tables (for the staging loops).
__device__ __forceinline__ double math_table_entry(int i) { return MATH_TABLE_INIT[i]; }

__device__ __forceinline__ double log_tab(const double *T, double x)
{
    if (!(x >= 2.2250738585072014e-308 && x <= 1.7976931348623157e308)) return log_rare(x);
    const long long bits = __double_as_longlong(x);
    const int k = (int)(bits >> 52) - 1023;
    const int i = (int)((bits >> 45) & (LOG_TABLE_N - 1));
    const double m = __longlong_as_double((bits & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    const double2 e = reinterpret_cast<const double2 *>(T + MATH_LOG_PAIRS)[i];  // (inv_c_i, L_i)
    const double r = fma(m, e.x, -1.0);
    double p = -1.0 / 8.0;
    p = fma(p, r, 1.0 / 7.0);
    p = fma(p, r, -1.0 / 6.0);
    p = fma(p, r, 1.0 / 5.0);
    p = fma(p, r, -1.0 / 4.0);
    p = fma(p, r, 1.0 / 3.0);
    p = fma(p, r, -1.0 / 2.0);
    const double lp = fma(p * r, r, r);  // r + r^2 (-1/2 + r/3 - ...)
    const double kd = (double)k;
    return fma(kd, LN2_HI, e.y + fma(kd, LN2_LO, lp));
}

__device__ __forceinline__ double exp_tab(const double *T, double x)
{
    if (!(fabs(x) < 708.0)) return exp_rare(x);
    const double kd = rint(x * INV_LN2_64);
    const double r = fma(-kd, LN2_64_LO, fma(-kd, LN2_64_HI, x));
    const int k = (int)kd;
    const int j = k & (EXP_TABLE_N - 1);
    const int e = k >> 6;  // floor(k / 64)
    double p = 1.0 / 120.0;
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0) * r;  // e^r - 1
    const double t = T[MATH_EXP_T + j];
    return fma(t, p, t) * __longlong_as_double((long long)(e + 1023) << 52);
}

// x^(-1/2) within about an ulp for x in [1e-300, 1e300]: the hardware
// estimate (rsqrt.approx.ftz.f64, relative error near 2^-23) y0 and, with
// e = 1 - x y0^2, y = y0 (1 + e/2 + 3 e^2 / 8) (the omitted term is 5 e^3 / 16).
__device__ __forceinline__ double rsqrt_few_ulp(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);
}

__device__ __forceinline__ double unit_log(double x)
{
#if DRIFT_EXACT_ARITH
    return log(x);
#else
    return log_few_ulp(x);
#endif
}

__device__ __forceinline__ double unit_exp(double x)
{
#if DRIFT_EXACT_ARITH
    return exp(x);
#else
    return exp_few_ulp(x);
#endif
}

// log2(q) for the DOPR54 controller, whose result is only rounded to an
// integer after scaling by 0.1: in the contraction unit the exponent plus a
// single-precision log2 of the mantissa in [1, 2) (absolute error ~1e-7,
// which moves the rounding only when the argument lies that close to a
// half-integer).  0 -> -inf, NaN -> NaN, +inf -> +inf as log2.
__device__ __forceinline__ double log2_for_rounding_few_ulp(double q)
{
    if (!(q > 0.0) || isinf(q)) return log2(q);
    int e;
    const double m = 2.0 * frexp(q, &e);  // q = m 2^(e-1), m in [1, 2)
    return (double)(e - 1) + (double)__log2f((float)m);
}

__device__ __forceinline__ double unit_log2_for_rounding(double q)
{
#if DRIFT_EXACT_ARITH
    return log2(q);
#else
    return log2_for_rounding_few_ulp(q);
#endif
}

// The powers as the integrators call them in this translation unit.
__device__ __forceinline__ double unit_pow_m1p5(double x)
{
#if DRIFT_EXACT_ARITH
    return pow_m1p5(x);
#else
    return pow_m1p5_few_ulp(x);
#endif
}

__device__ __forceinline__ double unit_pow_1p5(double x)
{
#if DRIFT_EXACT_ARITH
    return pow_1p5(x);
#else
    return pow_1p5_few_ulp(x);
#endif
}

__device__ __forceinline__ double unit_root8(double x)
{
#if DRIFT_EXACT_ARITH
    return root8(x);
#else
    return root8_few_ulp(x);
#endif
}

}  // namespace drift
