// Reciprocal square root and division in FP64 for FP64 work that needs FP64
// accuracy but not the reference's operation sequence (the refinement pass of
// FP32_REFINED plans and the FP64 nodes of the FP32 arrangement kernels):
//
//   rsqrt64u(x): 1/sqrt(x) from the FP64 reciprocal-square-root estimate
//                (rsqrt.approx.ftz.f64) and two Newton-Raphson steps
//                y <- y + y (1 - x y^2) / 2, each squaring the estimate's
//                relative error, the residual 1 - x y^2 taken by a fused
//                multiply-add;
//   div64u(n, d): n / d from the FP64 reciprocal estimate (rcp.approx.ftz.f64),
//                two Newton-Raphson steps y <- y + y (1 - d y) and one residual
//                correction q + (n - q d) y with the residual exact in a fused
//                multiply-add (Markstein's final step);
//   sqrt64(x):   x rsqrt64(x).
//
// The unchecked forms take arguments in [kLo64, kHi64] (positive, normal, far
// from both ends of the exponent range, so no intermediate overflows or
// flushes); rsqrt64 takes the IEEE path outside it.  Loops that can bound
// their arguments beforehand take the unchecked forms through the CHECKED
// template argument: the range check and the IEEE paths are branches, and a
// branch per root keeps the compiler from interleaving independent roots.
// ccoil_eval_rsqrt64 and ccoil_eval_div64 expose the unchecked forms for
// accuracy checks against the host.
#ifndef CCOIL_FP64OPS_CUH
#define CCOIL_FP64OPS_CUH

constexpr double kLo64 = 1e-36, kHi64 = 1e36;

__device__ __forceinline__ double rsqrt64u(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x * y, y, 1.0);
    y = fma(0.5 * y, e, y);
    e = fma(-x * y, y, 1.0);
    return fma(0.5 * y, e, y);
}

__device__ __forceinline__ double rsqrt64(double x)
{
    if (!(x > kLo64 && x < kHi64))
        return 1.0 / sqrt(x);
    return rsqrt64u(x);
}

__device__ __forceinline__ double sqrt64(double x) { return x * rsqrt64(x); }

__device__ __forceinline__ double div64u(double n, double d)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    y = fma(y, fma(-d, y, 1.0), y);
    y = fma(y, fma(-d, y, 1.0), y);
    const double q = n * y;
    return fma(fma(-q, d, n), y, q);
}

template <bool CHECKED> __device__ __forceinline__ double rsqrt64t(double x)
{
    return CHECKED ? rsqrt64(x) : rsqrt64u(x);
}

template <bool CHECKED> __device__ __forceinline__ double sqrt64t(double x) { return x * rsqrt64t<CHECKED>(x); }

template <bool CHECKED> __device__ __forceinline__ double div64t(double n, double d)
{
    return CHECKED ? n / d : div64u(n, d);
}

// Every argument of an angular loop lies in [lo, hi] when the loop forms it as
// base + k c or base - k c with k >= 0 and |c| <= 1 and the bounds are the
// computed base - k and base + k (rounding is monotone).
__device__ __forceinline__ bool inRange64(double lo, double hi) { return lo > kLo64 && hi < kHi64; }

#endif
