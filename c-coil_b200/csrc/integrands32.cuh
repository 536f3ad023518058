// FP32-compensated integrands, shared by the field kernels (fields32.cuh) and
// the arrangement kernels (pairs.cu); included inside their anonymous
// namespaces after integrands64.cuh.
//
// Arithmetic.  Per point and coil the frame transform, the per-thickness-node
// constants and the final sums are FP64; the angular loop runs in FP32 over
// mirror pairs of nodes (phi, pi - phi): each step evaluates both nodes and
// adds w c (f(c) - f(-c)) and w (g(c) + g(-c)) to FP32 running sums.
// Far from the coil f(c) and f(-c) agree to many digits: the vector potential
// and the field form their difference in closed form, as delta = 2 b2 c times a
// cancellation-free expression (below), so its relative error does not grow
// with the distance; the gradient subtracts (its error stays two orders below
// the others').  The vector potential and the field compensate their sums
// (Kahan: it halves their 99th-percentile error); the arrangement kernels add
// plainly (the FP64 sum over the secondary's nodes averages their rounding).
// Both nodes of a pair take every quantity of the form
// Q + b2 (1 - cos) from the same FP32 constants Q and b2 (with their own
// 1 - cos, omc and omcm), so the rounding of Q and b2 is common to the pair.
// The FP32 integrands are
// algebraic rewrites of the reference's (CalculateFieldsFast.cxx,
// CalculateFieldsSlow.cxx) that remove every cancellation FP32 cannot afford:
//   distance^2     D - 2 p r cos  ->  (p - r)^2 + z^2 + 2 p r (1 - cos)
//   G2 - G1        -> dD G1^2 G2^2 / (G1 + G2),  dD = top^2 - bot^2 = 2 z b
//   top G1 - bot G2 (point outside the slab |z| > b/2)
//                  -> rho^2 dD G1^2 G2^2 / (top G1 + bot G2)
//   asinh(top/rho) - asinh(bot/rho) (vector potential)
//                  -> asinh(dD / (top s2 + bot s1)) outside the slab,
//                     asinh((top s2 - bot s1) / rho^2) inside it
//   RZ gradient node (fast) -> p [c (T1 + Y) - k (2 Y + T1)], where
//                     T1 = top G1^3 - bot G2^3, Y = (top G1 - bot G2) / rho^2 and
//                     k = p r sin^2 / rho^2 (in [0, 1]): equal node by node to the
//                     reference's (p / M^2)(top L1 (O J1 + N) - bot L2 (O J2 + N)),
//                     via N = c rho^4 - p r s^2 rho^2 and O = c rho^2 - 2 p r s^2,
//                     without its 1/rho^4 cancellation
// and the azimuthal tables hold one entry per mirror pair (PhiNode32).


// Runs body(k, accumulator set) over the pair entries lane, lane + LANES, ...,
// alternating between two independent accumulator sets so consecutive entries
// do not wait on each other's additions (and each running sum stays short).
template <int LANES, typename Acc, typename Body>
__device__ __forceinline__ void forNodes(int n, int lane, Acc &a0, Acc &a1, Body body)
{
    int k = lane;
    for (; k + LANES < n; k += 2 * LANES)
    {
        body(k, a0);
        body(k + LANES, a1);
    }
    if (k < n)
        body(k, a0);
}

// pair entries of a table slice holding n angular nodes
__device__ __forceinline__ int pairEntries(int n) { return (n + 1) >> 1; }

// Fast method: whether a point lies outside the coil's length slab (|z| > b/2)
// picks between two cancellation-free forms of each integrand.  When every
// active lane agrees the warp runs a loop with that form only (SLAB 1: all
// outside, 2: all inside); otherwise each lane selects (SLAB 0).
template <int V>
struct SlabTag
{
    static constexpr int value = V;
};
// UNIFORM false: always the per-lane form (B, measured no faster with the
// branches, and the arrangement kernels, whose out-of-line quadrature measured
// 35 % slower with the three loop copies).
template <bool UNIFORM, typename Loop>
__device__ __forceinline__ void bySlab(bool outside, Loop loop)
{
    if (!UNIFORM)
    {
        loop(SlabTag<0>{});
        return;
    }
    const unsigned mask = __activemask();
    if (__all_sync(mask, outside))
        loop(SlabTag<1>{});
    else if (__all_sync(mask, !outside))
        loop(SlabTag<2>{});
    else
        loop(SlabTag<0>{});
}
template <int SLAB>
__device__ __forceinline__ bool slabOutside(bool perLane)
{
    return SLAB == 1 ? true : (SLAB == 2 ? false : perLane);
}

// Compensated (Kahan) running sum
struct Kahan
{
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float x)
    {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// Plain running sum, for callers whose error is set elsewhere (the gradient,
// whose pair sums stay far below the FP32 path's error bar, and the
// arrangement kernels, whose FP64 sum over the secondary's nodes averages the
// per-node rounding)
struct PlainSum
{
    float s = 0.0f;
    __device__ __forceinline__ void add(float x) { s += x; }
    __device__ __forceinline__ double value() const { return (double)s; }
};

template <typename S>
struct Acc1
{
    S v;
};
template <typename S>
struct Acc2
{
    S h, z;
};
struct Acc4
{
    float a = 0.0f, b = 0.0f, c = 0.0f, d = 0.0f;
};

// reciprocal: MUFU estimate (within 1 ulp), no special-case handling needed
// since every argument here is a positive normal number
__device__ __forceinline__ float rcpApprox(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// reciprocal square root: the MUFU estimate (relative error below 2^-22.9),
// flush-to-zero form (one instruction; every argument here is a positive
// normal number, a squared distance or 1 + u^2); a Newton-Raphson step
// (CCOIL_RSQRT_NEWTON=1) did not change the measured error of the sums, which
// is set by the far-field cancellation, and costs 4 FMA per call
#ifndef CCOIL_RSQRT_NEWTON
#define CCOIL_RSQRT_NEWTON 0
#endif
__device__ __forceinline__ float rsqrtNR(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
#if CCOIL_RSQRT_NEWTON
    float e = fmaf(-x * y, y, 1.0f);
    y = fmaf(0.5f * y, e, y);
#endif
    return y;
}

// asinh(u): the Maclaurin series sum_n (-1)^n (2n)! / (4^n (n!)^2 (2n+1)) u^(2n+1)
// through n = 6 when every lane of the warp has |u| < 0.25 (truncation below
// 6e-11 relative there); asinhMid up to 1, asinhLarge beyond (CUDA's asinhf
// past 1e18)
__device__ __forceinline__ float asinhSmall(float u)
{
    const float u2 = u * u;
    float p = 0.017352764f;          // 231/13312
    p = fmaf(p, u2, -0.022372159f);  // -63/2816
    p = fmaf(p, u2, 0.030381944f);   // 35/1152
    p = fmaf(p, u2, -0.044642857f);  // -5/112
    p = fmaf(p, u2, 0.075f);         // 3/40
    p = fmaf(p, u2, -0.16666667f);   // -1/6
    return fmaf(p * u2, u, u);
}

// asinh(u) for 0.25 <= |u| < 1e18: log(x) with x = |u| + sqrt(1 + u^2) carried
// as x_hi + x_lo (one Newton step on the square root, the exact residual of
// 1 + u^2 and of the sum), then log(x_hi) by exponent reduction to
// m in [sqrt(1/2), sqrt(2)) and log(m) = 2 atanh(f), f = (m - 1) / (m + 1), as
// 2 (f + f^3/3 + ... + f^9/9) (|f| <= 0.1716: truncation below 3e-9 relative),
// plus x_lo / x_hi; ln 2 is split into a high part exact in e ln2_hi and a low
// part (Cody and Waite).  About 1-2 ulp over the range.
__device__ __forceinline__ float asinhLarge(float u)
{
    const float a = fabsf(u);
    const float y = fmaf(a, a, 1.0f);
    const float ylo = fmaf(a, a, 1.0f - y);  // 1 + a^2 - y (exact while y < 2; negligible beyond)
    const float rs = rsqrtNR(y);
    float sq = y * rs;
    sq = fmaf(0.5f * fmaf(-sq, sq, y), rs, sq);
    const float ds = (fmaf(-sq, sq, y) + ylo) * (0.5f * rs);
    const float xh = sq + a;  // sq >= a: exact rounding error below
    const float xl = (a - (xh - sq)) + ds;
    const int i = __float_as_int(xh);
    const int e = (i - 0x3f3504f3) >> 23;
    const float m = __int_as_float(i - (e << 23));
    const float g = m - 1.0f;  // exact
    const float t = 2.0f + g;
    const float tl = g - (t - 2.0f);  // exact rounding error of t
    const float rc = rcpApprox(t);
    const float q = g * rc;
    const float f = fmaf(rc, fmaf(-q, t, g) - q * tl, q);
    const float z = f * f;
    const float p = fmaf(fmaf(fmaf(0.11111111f, z, 0.14285715f), z, 0.2f), z, 0.33333334f);
    const float f2 = 2.0f * f;
    const float logm = fmaf(f2 * z, p, f2);
    const float ef = (float)e;
    const float r = fmaf(ef, 0.693145751953125f, fmaf(ef, 1.42860682e-06f, logm + xl * rcpApprox(xh)));
    return copysignf(r, u);
}

// asinh(u) for |u| <= 1: u P(u^2), P of degree 8 from a Chebyshev least-squares
// fit of asinh(sqrt(x)) / sqrt(x) on x in [0, 1], computed for this library
// (1.7 ulp at most in FP32 Horner evaluation, checked on 80,000 arguments)
__device__ __forceinline__ float asinhMid(float u)
{
    const float x = u * u;
    float p = 6.495655980e-04f;
    p = fmaf(p, x, -3.737240797e-03f);
    p = fmaf(p, x, 1.025899500e-02f);
    p = fmaf(p, x, -1.902823150e-02f);
    p = fmaf(p, x, 2.937856875e-02f);
    p = fmaf(p, x, -4.446590319e-02f);
    p = fmaf(p, x, 7.498393208e-02f);
    p = fmaf(p, x, -1.666660905e-01f);
    p = fmaf(p, x, 1.0f);
    return u * p;
}

// asinh(u) per lane: asinhMid up to 1, asinhLarge beyond (CUDA's asinhf past 1e18)
__device__ __forceinline__ float asinhAny(float u)
{
    const float au = fabsf(u);
    if (au <= 1.0f)
        return asinhMid(u);
    return au < 1e18f ? asinhLarge(u) : asinhf(u);
}

// asinh(u) in a tier the warp chose beforehand: 0 every lane's argument below
// 0.25, 1 below 1, 2 per lane
__device__ __forceinline__ float asinhTier(float u, int tier)
{
    if (tier == 0)
        return asinhSmall(u);
    if (tier == 1)
        return asinhMid(u);
    return asinhAny(u);
}

__device__ __forceinline__ bool nearWinding(const SegmentHeader &h, const Frame &f)
{
    return f.r > h.near_lo[0] && f.r < h.near_hi[0] && f.z > h.near_lo[1] && f.z < h.near_hi[1];
}

// Mirror-pair differences in closed form.  For the pair (c, -c) the second
// node's squared distances exceed the first's by delta = b2 (omcm - omc); with
// g = 1 / sqrt(D) and g' = 1 / sqrt(D + delta),
//   g - g' = delta e,  e = g^2 g'^2 / (g + g'),
// and every difference below is delta times a sum of terms of one sign, so its
// relative error stays that of a few FP32 roundings however far the point is
// (forming f(c) - f(-c) by subtraction loses the ratio distance / radius).
// The accumulated weight of a difference is w2c2 = 2 w c^2 (= w c delta / b2),
// so b2 multiplies the sums after the loop, in FP64.
struct PairInv
{
    float i1, i2;  // 1 / (x1 + x1'), 1 / (x2 + x2') from one reciprocal
};
__device__ __forceinline__ PairInv pairInverse(float a, float b)
{
    const float r = rcpApprox(a * b);
    return {b * r, a * r};
}

// Vector potential.  Fast method: per node asinh(u) with u = dD / (top s2 + bot s1)
// outside the slab, (top s2 - bot s1) / rho^2 inside it (s the distances to the
// slab's faces); the pair's difference is asinh(u) - asinh(u') =
// asinh((u - u') (u + u') / (u sqrt(1 + u'^2) + u' sqrt(1 + u^2))), with u - u'
// in closed form:
//   outside  (u - u') / delta = dD (top / (s2 + s2') + bot / (s1 + s1')) / (V V'),  V = top s2 + bot s1
//   inside   (u - u') / delta = [top (bot^2 + s2 s2') / (s2 + s2') - bot (top^2 + s1 s1') / (s1 + s1')]
//                               / (rho^2 rho'^2)
// (outside, top and bot share a sign; inside, top > 0 > bot, so every term is
// positive).  u and u' share a sign, so the last denominator does not cancel
// either.
// Slow method: sum w c (g - g') = b2 sum w2c2 e.
// S: the running-sum type of the pair accumulation (Kahan or PlainSum);
// UNIFORM: warp-uniform slab branches (bySlab)
template <int LANES, typename S = Kahan, bool UNIFORM = true>
__device__ __forceinline__ double segmentA32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                             const PhiNode32 *pn, const Frame &f, int lane)
{
    double sum = 0.0;
    const int np = pairEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool same = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot;
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const float dDf = (float)dD, dDl = (float)(dD - (double)dDf);
        bySlab<UNIFORM>(same, [&](auto slab) {
            const bool outside = slabOutside<decltype(slab)::value>(same);
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double q = (t.x - f.r) * (t.x - f.r), b2d = 2.0 * t.x * f.r;
                const float qf = (float)q, b2 = (float)b2d;
                const float d1 = (float)(top * top + q), d2 = (float)(bot * bot + q);
                // |u| decreases with 1 - cos on either side of the slab and the
                // difference's argument stays below max(|u|, |u'|), so |u| at phi = 0
                // bounds every argument of this thickness node: one warp vote picks the
                // asinh form for all of them
                float u0;
                {
                    const float e1 = d1 * rsqrtNR(d1), e2 = d2 * rsqrtNR(d2);
                    u0 = outside ? fabsf(fmaf(dDl, 1.0f, dDf) * rcpApprox(fmaf(topf, e2, botf * e1)))
                                 : fabsf(fmaf(topf, e2, -botf * e1) * rcpApprox(qf));
                }
                const unsigned mask = __activemask();
                const int tier = __all_sync(mask, u0 < 0.25f) ? 0 : (__all_sync(mask, u0 <= 1.0f) ? 1 : 2);
                Acc1<S> a0, a1;
                forNodes<LANES>(np, lane, a0, a1, [&](int k, Acc1<S> &acc) {
                    const PhiNode32 nd = pn[k];
                    const float dom = nd.omcm - nd.omc;  // delta / b2
                    const float den1 = fmaf(b2, nd.omc, d1), den2 = fmaf(b2, nd.omc, d2);
                    const float den1m = fmaf(b2, nd.omcm, d1), den2m = fmaf(b2, nd.omcm, d2);
                    const float s1 = den1 * rsqrtNR(den1), s2 = den2 * rsqrtNR(den2);
                    const float s1m = den1m * rsqrtNR(den1m), s2m = den2m * rsqrtNR(den2m);
                    const PairInv is = pairInverse(s1 + s1m, s2 + s2m);
                    float u, um, du;
                    if (outside)
                    {
                        const float v = fmaf(topf, s2, botf * s1), vm = fmaf(topf, s2m, botf * s1m);
                        const PairInv iv = pairInverse(v, vm);
                        u = fmaf(dDl, iv.i1, dDf * iv.i1);
                        um = fmaf(dDl, iv.i2, dDf * iv.i2);
                        du = fmaf(topf, is.i2, botf * is.i1) * (u * iv.i2);
                    }
                    else
                    {
                        const float rho2 = fmaf(b2, nd.omc, qf), rho2m = fmaf(b2, nd.omcm, qf);
                        const PairInv ir = pairInverse(rho2, rho2m);
                        u = fmaf(topf, s2, -botf * s1) * ir.i1;
                        um = fmaf(topf, s2m, -botf * s1m) * ir.i2;
                        // top (bot^2 + s2 s2') / (s2 + s2') - bot (top^2 + s1 s1') / (s1 + s1'), both terms >= 0
                        du = fmaf(topf * fmaf(botf, botf, s2 * s2m), is.i2, -botf * fmaf(topf, topf, s1 * s1m) * is.i1) *
                             (ir.i1 * ir.i2);
                    }
                    // sqrt(1 + u^2), sqrt(1 + u'^2)
                    const float y = fmaf(u, u, 1.0f), ym = fmaf(um, um, 1.0f);
                    const float sq = y * rsqrtNR(y), sqm = ym * rsqrtNR(ym);
                    const float arg = (du * (b2 * dom)) * ((u + um) * rcpApprox(fmaf(u, sqm, um * sq)));
                    acc.v.add((0.5f * nd.w * dom) * asinhTier(arg, tier));
                });
                sum += t.y * t.x * (a0.v.value() + a1.v.value());
            }
        });
    }
    else
    {
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = l.x + f.z;
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double q = (t.x - f.r) * (t.x - f.r) + zl * zl, b2d = 2.0 * t.x * f.r;
                const float qf = (float)q, b2 = (float)b2d;
                Acc1<S> a0, a1;
                forNodes<LANES>(np, lane, a0, a1, [&](int k, Acc1<S> &acc) {
                    const PhiNode32 nd = pn[k];
                    const float g = rsqrtNR(fmaf(b2, nd.omc, qf)), gm = rsqrtNR(fmaf(b2, nd.omcm, qf));
                    const float gg = g * gm;
                    acc.v.add(nd.w2c2 * (gg * gg * rcpApprox(g + gm)));
                });
                sum += l.y * t.y * t.x * (double)b2 * (a0.v.value() + a1.v.value());
            }
        }
    }
    return sum;
}

// Field.  Fast method, per node: the H integrand over dD w c is
// hv = g1^2 g2^2 / (g1 + g2) and the Z integrand over w is num y with
// num = p^2 - p r c and y = (top g1 - bot g2) / rho^2 (= dD g1^2 g2^2 / (top g1 + bot g2)
// outside the slab; dD multiplies after the loop there).  The pair contributes
//   H: w c (hv - hv') = b2 w2c2 kh,
//      kh = (u1 + u2' + u1^2 / (u2 + u2') + u2'^2 / (u1 + u1')) hv hv'   (u = 1 / g)
//   Z: w (num y + num' y') = w (2 p^2 y' + num (y - y')),  y - y' = delta ey:
//      outside [top g1 g1' (e1 g2^2 + g1' e2 (g2 + g2')) + bot g2 g2' (e1 (g1 + g1') g2 + g1'^2 e2)] / (X X'),
//              X = top g1 + bot g2
//      inside  (top e1 - bot e2 + y') / rho^2.
// Far from the coil, num y + num' y' subtracts two terms ~ p r c y; near the
// winding (y >> y'), p^2 (y + y') - p r c (y - y') does; 2 p^2 y' + num (y - y')
// does neither (num = p (p - r) + p r (1 - c) from the table).
// Slow method: with k3 = (g^3 - g'^3) / delta = e (g^2 + g g' + g'^2),
//   H: w c (g^3 - g'^3) = b2 w2c2 k3,   Z: w (2 p^2 g'^3 + num delta k3).
template <typename S>
struct Acc3
{
    S h, y, e;
};

template <int LANES, typename S = Kahan>
__device__ __forceinline__ void segmentB32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const PhiNode32 *pn, const Frame &f, int lane, double &H, double &Z)
{
    H = 0.0;
    Z = 0.0;
    const int np = pairEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool outside = top * bot > 0.0;  // per lane (slab branches measured no faster for B)
        const float topf = (float)top, botf = (float)bot;
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const double zScale = outside ? dD : 1.0;
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double q = (t.x - f.r) * (t.x - f.r), b2d = 2.0 * t.x * f.r;
            const float qf = (float)q, b2 = (float)b2d;
            const float d1 = (float)(top * top + q), d2 = (float)(bot * bot + q);
            const float n0 = (float)(t.x * (t.x - f.r)), n1 = (float)(t.x * f.r);
            Acc3<S> a0, a1;
            forNodes<LANES>(np, lane, a0, a1, [&](int k, Acc3<S> &acc) {
                const PhiNode32 nd = pn[k];
                const float den1 = fmaf(b2, nd.omc, d1), den2 = fmaf(b2, nd.omc, d2);
                const float den1m = fmaf(b2, nd.omcm, d1), den2m = fmaf(b2, nd.omcm, d2);
                const float g1 = rsqrtNR(den1), g2 = rsqrtNR(den2), g1m = rsqrtNR(den1m), g2m = rsqrtNR(den2m);
                // per node: hv, y and 1 / X from one reciprocal of (g1 + g2) X
                auto node = [&](float a, float b, float rho2, float &hv, float &y, float &ix) {
                    const float gg = a * b, gg2 = gg * gg, s = a + b;
                    const float t1 = topf * a, t2 = botf * b;
                    const float X = outside ? t1 + t2 : rho2;
                    const float R = rcpApprox(s * X);
                    hv = gg2 * (X * R);
                    ix = s * R;
                    y = (outside ? gg2 : t1 - t2) * ix;
                };
                float hv, y, ix, hvm, ym, ixm;
                node(g1, g2, fmaf(b2, nd.omc, qf), hv, y, ix);
                node(g1m, g2m, fmaf(b2, nd.omcm, qf), hvm, ym, ixm);
                const float s1 = g1 + g1m, s2 = g2 + g2m;
                const PairInv is = pairInverse(s1, s2);
                const float p1 = g1 * g1m, p2 = g2 * g2m;
                const float e1 = p1 * p1 * is.i1, e2 = p2 * p2 * is.i2;
                const float u1 = den1 * g1, u2m = den2m * g2m;
                const float kh = ((u1 + u2m) + fmaf(u1 * u1, p2 * is.i2, (u2m * u2m) * (p1 * is.i1))) * (hv * hvm);
                const float ey = outside ? fmaf(topf * p1, fmaf(e1, g2 * g2, g1m * (e2 * s2)),
                                                botf * p2 * fmaf(e1 * s1, g2, g1m * g1m * e2)) *
                                               (ix * ixm)
                                         : (fmaf(topf, e1, -botf * e2) + ym) * ix;
                const float num = fmaf(n1, nd.omc, n0);  // p^2 - p r c = p (p - r) + p r (1 - c)
                acc.h.add(nd.w2c2 * kh);
                acc.y.add(nd.w * ym);
                acc.e.add((nd.w * (nd.omcm - nd.omc)) * (num * ey));
            });
            const double b2f = (double)b2;
            H += t.y * t.x * dD * b2f * (a0.h.value() + a1.h.value());
            Z += t.y * zScale * (2.0 * t.x * t.x * (a0.y.value() + a1.y.value()) + b2f * (a0.e.value() + a1.e.value()));
        }
    }
    else
    {
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = l.x + f.z;
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double q = (t.x - f.r) * (t.x - f.r) + zl * zl, b2d = 2.0 * t.x * f.r;
                const float qf = (float)q, b2 = (float)b2d;
                const float n0 = (float)(t.x * (t.x - f.r)), n1 = (float)(t.x * f.r);
                Acc3<S> a0, a1;
                forNodes<LANES>(np, lane, a0, a1, [&](int k, Acc3<S> &acc) {
                    const PhiNode32 nd = pn[k];
                    const float g = rsqrtNR(fmaf(b2, nd.omc, qf)), gm = rsqrtNR(fmaf(b2, nd.omcm, qf));
                    const float gg = g * gm, g2 = g * g, gm2 = gm * gm;
                    const float k3 = gg * gg * rcpApprox(g + gm) * (g2 + fmaf(g, gm, gm2));
                    const float num = fmaf(n1, nd.omc, n0);
                    acc.h.add(nd.w2c2 * k3);
                    acc.y.add(nd.w * (gm2 * gm));
                    acc.e.add((nd.w * (nd.omcm - nd.omc)) * (num * k3));
                });
                const double w = l.y * t.y, b2f = (double)b2;
                H += w * t.x * zl * b2f * (a0.h.value() + a1.h.value());
                Z += w * (2.0 * t.x * t.x * (a0.y.value() + a1.y.value()) + b2f * (a0.e.value() + a1.e.value()));
            }
        }
    }
}

// {RPhi, RR, RZ, ZZ}
template <int LANES>
__device__ __forceinline__ void segmentG32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const PhiNode32 *pn, const Frame &f, int lane, double *g)
{
    double rphi = 0.0, rr = 0.0, rz = 0.0, zz = 0.0;
    const double r = f.r;
    const int np = pairEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool same = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot, lenf = (float)(2.0 * h.half_length);
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const float dDf = (float)dD;
        bySlab<true>(same, [&](auto slab) {
            const bool outside = slabOutside<decltype(slab)::value>(same);
            // one node: dg = G2 - G1, dg3 = G1^3 - G2^3, cz = T1 + Y (the RZ part
            // multiplying cos) and kz = k (2 Y + T1) / sin2 (sin2 = (b2 / 2) sin^2 is
            // the same for both nodes of a pair).  T1 = top G1^3 - bot G2^3 and
            // Y = (top G1 - bot G2) / rho^2, each in its cancellation-free form for a
            // point outside / inside the slab
            auto node = [&](float rho2, float den1, float den2, float &dg, float &dg3, float &cz, float &kz) {
                const float g1 = rsqrtNR(den1), g2 = rsqrtNR(den2);
                const float gg = g1 * g2, s = g1 + g2;
                const float ddgg = dDf * gg * gg;
                dg = ddgg * rcpApprox(s);
                dg3 = -dg * fmaf(g1, g1, fmaf(g1, g2, g2 * g2));
                const float g13 = g1 * g1 * g1;
                const float T1 = outside ? fmaf(lenf, g13, botf * dg3) : fmaf(topf, g13, -botf * (g2 * g2 * g2));
                const float t1 = topf * g1, t2 = botf * g2;
                const float yn = outside ? ddgg : (t1 - t2);
                const float yd = outside ? (t1 + t2) : rho2;
                const float Y = yn * rcpApprox(yd);
                cz = T1 + Y;
                kz = fmaf(2.0f, Y, T1) * rcpApprox(rho2);
            };
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double q = (t.x - r) * (t.x - r), b2d = 2.0 * t.x * r;
                const float qf = (float)q, b2 = (float)b2d, hb2 = (float)(0.5 * b2d);
                const float d1 = (float)(top * top + q), d2 = (float)(bot * bot + q);
                const float pf = (float)t.x, rf = (float)r;
                // (r - p cos) = (r - p) + p (1 - cos); likewise (p - r cos)
                const float rmp = (float)(r - t.x), pmr = (float)(t.x - r);
                Acc4 a0, a1;
                forNodes<LANES>(np, lane, a0, a1, [&](int k, Acc4 &acc) {
                    const PhiNode32 nd = pn[k];
                    const float wc = 0.5f * nd.w * (nd.omcm - nd.omc);
                    float dg, dg3, cz, kz, dgm, dg3m, czm, kzm;
                    node(fmaf(b2, nd.omc, qf), fmaf(b2, nd.omc, d1), fmaf(b2, nd.omc, d2), dg, dg3, cz, kz);
                    node(fmaf(b2, nd.omcm, qf), fmaf(b2, nd.omcm, d1), fmaf(b2, nd.omcm, d2), dgm, dg3m, czm, kzm);
                    const float sin2 = hb2 * (nd.omc * nd.omcm);  // p r sin^2 = (b2 / 2)(1 - c)(1 + c)
                    acc.a = fmaf(wc, dg - dgm, acc.a);
                    acc.b = fmaf(wc, fmaf(fmaf(pf, nd.omc, rmp), dg3, -fmaf(pf, nd.omcm, rmp) * dg3m), acc.b);
                    acc.d = fmaf(nd.w, fmaf(fmaf(rf, nd.omc, pmr), dg3, fmaf(rf, nd.omcm, pmr) * dg3m), acc.d);
                    acc.c = fmaf(wc, cz - czm, fmaf(-nd.w * sin2, kz + kzm, acc.c));
                });
                const double w = t.y * t.x;
                rphi += w / r * ((double)a0.a + (double)a1.a);
                rr += w * ((double)a0.b + (double)a1.b);
                zz += w * ((double)a0.d + (double)a1.d);
                rz += w * ((double)a0.c + (double)a1.c);
            }
        });
    }
    else
    {
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = l.x + f.z;
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double p = t.x;
                const double q = (p - r) * (p - r) + zl * zl, b2d = 2.0 * p * r;
                const float qf = (float)q, b2 = (float)b2d;
                const float pf = (float)p, rf = (float)r;
                const float rmp = (float)(r - p), pmr = (float)(p - r);
                // RZ node G^5 (p cos (2p^2 + 2r^2 - zl^2 - p r cos) - 3 p^2 r) rewritten as
                // -p (cos G^3 + 3 G^5 (p - r cos)(r - p cos)) (G^5 D = G^3, D the squared
                // distance): its cos G^3 sum is the RPhi sum, so only the second sum is
                // accumulated, and the two are combined in FP64 after the loop
                Acc4 a0, a1;
                forNodes<LANES>(np, lane, a0, a1, [&](int k, Acc4 &acc) {
                    const PhiNode32 nd = pn[k];
                    const float wc = 0.5f * nd.w * (nd.omcm - nd.omc);
                    const float den = fmaf(b2, nd.omc, qf), denm = fmaf(b2, nd.omcm, qf);
                    const float gq = rsqrtNR(den), gqm = rsqrtNR(denm);
                    const float g3 = gq * gq * gq, g5 = g3 * gq * gq;
                    const float g3m = gqm * gqm * gqm, g5m = g3m * gqm * gqm;
                    const float rpc = fmaf(pf, nd.omc, rmp), prc = fmaf(rf, nd.omc, pmr);
                    const float rpcm = fmaf(pf, nd.omcm, rmp), prcm = fmaf(rf, nd.omcm, pmr);
                    acc.a = fmaf(wc, g3 - g3m, acc.a);
                    acc.b = fmaf(wc, fmaf(g5, rpc, -g5m * rpcm), acc.b);
                    acc.d = fmaf(nd.w, fmaf(g5, prc, g5m * prcm), acc.d);
                    acc.c = fmaf(nd.w, fmaf(g5 * prc, rpc, g5m * prcm * rpcm), acc.c);
                });
                const double w = l.y * t.y, ca = (double)a0.a + (double)a1.a;
                rphi += w * p * zl / r * ca;
                rr += -3.0 * w * p * zl * ((double)a0.b + (double)a1.b);
                zz += -3.0 * w * p * zl * ((double)a0.d + (double)a1.d);
                rz += -w * p * (ca + 3.0 * ((double)a0.c + (double)a1.c));
            }
        }
    }
    g[0] = rphi;
    g[1] = rr;
    g[2] = rz;
    g[3] = zz;
}
