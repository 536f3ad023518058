// Reciprocal square root, square root and division in FP64 for FP64 work that
// needs FP64 accuracy but not the reference's operation sequence (the refinement
// pass of FP32_REFINED plans and the FP64 nodes of the FP32 arrangement
// kernels), each from the FP64 estimate of the special-function unit and
// Newton-Raphson steps:
//
//   rsqrt64u(x): 1/sqrt(x) from rsqrt.approx.ftz.f64 and two steps
//                y <- y + y (1/2 - (x/2) y^2), the residual by a fused
//                multiply-add;
//   sqrt64u(x):  sqrt(x) by Goldschmidt's coupled iteration from the same
//                estimate: s = x y, h = y / 2, then twice r = 1/2 - s h,
//                s <- s + s r (and h <- h + h r before the last);
//   div64u(n, d): n / d from rcp.approx.ftz.f64, one step y <- y + y (1 - d y)
//                and the residual correction q + (n - q d) y with n - q d exact
//                in a fused multiply-add (Markstein's final step), which squares
//                the remaining relative error;
//   sqrt64(x), rsqrt64(x): the IEEE path outside [kLo64, kHi64].
//
// The unchecked forms take arguments in [kLo64, kHi64] (positive, normal, far
// from both ends of the exponent range, so no intermediate overflows or
// flushes).  Loops that can bound their arguments beforehand take them through
// the CHECKED template argument: the range check and the IEEE paths are
// branches, and a branch per root keeps the compiler from interleaving
// independent roots.  ccoil_eval_fp64_op exposes the unchecked forms (and
// logRatio64) for accuracy checks against the host.
#ifndef CCOIL_FP64OPS_CUH
#define CCOIL_FP64OPS_CUH

constexpr double kLo64 = 1e-36, kHi64 = 1e36;

__device__ __forceinline__ double rsqrt64u(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double hx = 0.5 * x;
    double e = fma(-hx * y, y, 0.5);
    y = fma(y, e, y);
    e = fma(-hx * y, y, 0.5);
    return fma(y, e, y);
}

__device__ __forceinline__ double sqrt64u(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double s = x * y, h = 0.5 * y;
    double r = fma(-s, h, 0.5);
    s = fma(s, r, s);
    h = fma(h, r, h);
    r = fma(-s, h, 0.5);
    return fma(s, r, s);
}

__device__ __forceinline__ double rsqrt64(double x)
{
    if (!(x > kLo64 && x < kHi64))
        return 1.0 / sqrt(x);
    return rsqrt64u(x);
}

__device__ __forceinline__ double sqrt64(double x)
{
    if (!(x > kLo64 && x < kHi64))
        return sqrt(x);
    return sqrt64u(x);
}

__device__ __forceinline__ double div64u(double n, double d)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    y = fma(y, fma(-d, y, 1.0), y);
    const double q = n * y;
    return fma(fma(-q, d, n), y, q);
}

template <bool CHECKED> __device__ __forceinline__ double rsqrt64t(double x)
{
    return CHECKED ? rsqrt64(x) : rsqrt64u(x);
}

template <bool CHECKED> __device__ __forceinline__ double sqrt64t(double x)
{
    return CHECKED ? sqrt64(x) : sqrt64u(x);
}

template <bool CHECKED> __device__ __forceinline__ double div64t(double n, double d)
{
    return CHECKED ? n / d : div64u(n, d);
}

// Every argument of an angular loop lies in [lo, hi] when the loop forms it as
// base + k c or base - k c with k >= 0 and |c| <= 1 and the bounds are the
// computed base - k and base + k (rounding is monotone).
__device__ __forceinline__ bool inRange64(double lo, double hi) { return lo > kLo64 && hi < kHi64; }

#endif
