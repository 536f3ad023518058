// Natural logarithm of a positive, normal, finite double for the FP64
// integrands (the vector potential's log of a ratio of positive sums).
//
// Method (Cody and Waite range reduction, then the atanh series of the
// logarithm): x = 2^e m with m in [sqrt(1/2), sqrt(2)), so that
// log x = e ln 2 + log m and log m = 2 atanh(f), f = (m - 1) / (m + 1),
// |f| <= 0.1716.  2 atanh(f) = 2 f + 2 f^3 / 3 + ... + 2 f^21 / 21 leaves a
// truncation below 1e-17 relative.  The quotient f is formed with its rounding
// error carried (m + 1 is split into a double and its exact rounding error,
// the reciprocal of the approximate MUFU estimate is refined by two Newton
// steps, the residual g - q t is taken exactly by a fused multiply-add, and f's
// own rounding error is kept as a low part); ln 2 is split into a high part of
// at most 32 significant bits (e ln2_hi exact for |e| < 2^11) and the
// remainder, and e ln2_hi + 2 f is summed exactly, so the result is rounded
// once: within 1 ulp of log x and correctly rounded in all but a fraction of a
// percent of cases (checked against the host's log), at about two thirds of
// the cost of CUDA's log in FP64-pipe slots.
//
// Domain: x > 0, normal and finite (no zero, subnormal, infinite or NaN
// handling); every argument the integrands pass is a ratio of positive sums.
#ifndef CCOIL_LOG64_CUH
#define CCOIL_LOG64_CUH

__device__ __forceinline__ double log64(double x)
{
    // ln 2 = ln2_hi + ln2_lo: ln 2 rounded to nearest at 32 significant bits
    // (the nearest such value ends in three more zero bits) and the remainder
    constexpr double kLn2Hi = 0.6931471806019545;     // 0x3FE62E42FF000000
    constexpr double kLn2Lo = -4.2009150726810846e-11;
    const long long bits = __double_as_longlong(x);
    // e = floor(log2(x / sqrt(1/2))): the exponent that brings m into [sqrt(1/2), sqrt(2))
    const long long e = (bits - 0x3FE6A09E667F3BCDLL) >> 52;
    const double m = __longlong_as_double(bits - (e << 52));
    const double g = m - 1.0;          // exact (m within a factor 2 of 1)
    const double t = m + 1.0;
    const double tl = g - (t - 2.0);   // m + 1 - t, exactly
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(t));
    y = fma(y, fma(-t, y, 1.0), y);
    y = fma(y, fma(-t, y, 1.0), y);
    const double q = g * y;
    const double r = fma(-q, tl, fma(-q, t, g));  // g - q (t + tl)
    const double f = fma(r, y, q);
    const double flo = fma(r, y, q - f);          // f's own rounding error
    const double z = f * f;
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
    const double f2 = 2.0 * f;
    const double ed = (double)e;
    // every small term first, then e ln2_hi + 2 f as an exact sum (|e ln2_hi|
    // exceeds |2 f| whenever e != 0), so the result is rounded once
    const double small = fma(ed, kLn2Lo, fma(f2 * z, p, 2.0 * flo));
    const double a = ed * kLn2Hi;
    const double sum = a + f2;
    const double err = f2 - (sum - a);
    return sum + (err + small);
}

// log(n / d) for positive normal n and d: n is brought to d's binary exponent
// (n' = n 2^-k, exact) and, by one factor of 2, to n' / d in [sqrt(1/2),
// sqrt(2)); then log(n / d) = k ln 2 + 2 atanh(f), f = (n' - d) / (n' + d), by
// the series above.  n' - d is exact (Sterbenz: n' and d within a factor 2), so
// f keeps its relative accuracy however close n / d is to 1, which a rounded
// quotient n / d would not; the quotient takes one Newton-Raphson step on the
// reciprocal estimate and a residual correction, and the low parts log64
// carries are dropped: within a few ulp of log(n / d).  Used by the FP64
// refinement forms of the vector potential (a ratio of products of distances).
__device__ __forceinline__ double logRatio64(double n, double d)
{
    constexpr double kLn2 = 0.6931471805599453;
    constexpr double kSqrt2 = 1.4142135623730951, kSqrtHalf = 0.7071067811865476;
    const long long bn = __double_as_longlong(n), bd = __double_as_longlong(d);
    long long k = (bn >> 52) - (bd >> 52);
    double m = __longlong_as_double(bn - (k << 52));
    const bool up = m >= kSqrt2 * d, down = m < kSqrtHalf * d;
    m = up ? 0.5 * m : (down ? 2.0 * m : m);
    k += (long long)up - (long long)down;
    const double g = m - d;  // exact
    const double t = m + d;
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(t));
    y = fma(y, fma(-t, y, 1.0), y);
    const double q = g * y;
    const double f = fma(fma(-q, t, g), y, q);
    const double z = f * f;
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
    const double f2 = 2.0 * f;
    return fma((double)k, kLn2, fma(f2 * z, p, f2));
}

#endif
