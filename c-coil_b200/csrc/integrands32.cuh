// FP32-compensated integrands, shared by the field kernels (fields32.cuh) and
// the arrangement kernels (pairs.cu); included inside their anonymous
// namespaces after integrands64.cuh.
//
// Arithmetic.  Per point and coil the frame transform, the per-thickness-node
// constants and the final sums are FP64; the angular loop runs in FP32 over
// mirror pairs of nodes (phi, pi - phi): each step evaluates both nodes and
// adds w c (f(c) - f(-c)) and w (g(c) + g(-c)) to running sums.
// Far from the coil f(c) and f(-c) agree to many digits: the vector potential
// and the field form their difference in closed form, as delta = 2 b2 c times a
// cancellation-free expression (below), so its relative error does not grow
// with the distance; the gradient subtracts (its error stays two orders below
// the others').  The vector potential and the field compensate their sums
// (each entry's term is added into an FP64 running sum, F64Sum: as accurate as
// a Kahan sum in FP32, which halved their 99th-percentile error against plain
// FP32 sums, and 10 % (B) and 2.5 % (A) faster than it, since the conversion
// and the FP64 add run on the otherwise idle FP64 pipe); the arrangement kernels add
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
// and the azimuthal tables hold two mirror pairs per entry (PhiPair2).


// Runs body(j, accumulator set) over the packed entries (two mirror pairs each)
// lane, lane + LANES, ..., alternating between two independent accumulator
// sets so consecutive entries do not wait on each other's additions (and each
// running sum stays short).
template <int LANES, typename Acc, typename Body>
__device__ __forceinline__ void forEntries(int n, int lane, Acc &a0, Acc &a1, Body body)
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

// One accumulator set, entries in order: fewer live temporaries, for the
// arrangement kernels' field quadrature (its register budget is 56 at 9 CTAs
// per SM; measured 3 % faster there than forEntries)
template <int LANES, typename Acc, typename Body>
__device__ __forceinline__ void forEntriesSerial(int n, int lane, Acc &a0, Acc &, Body body)
{
    for (int k = lane; k < n; k += LANES)
        body(k, a0);
}

// packed entries of a table slice holding n angular nodes: (n + 1) / 2 mirror
// pairs, two per entry
__device__ __forceinline__ int packedEntries(int n) { return (((n + 1) >> 1) + 1) >> 1; }

// Fast method: whether a point lies outside the coil's length slab (|z| > b/2)
// picks between two cancellation-free forms of each integrand.  When every
// active lane agrees the warp runs a loop with that form only (SLAB 1: all
// outside, 2: all inside); otherwise each lane selects (SLAB 0).
template <int V>
struct SlabTag
{
    static constexpr int value = V;
};
// UNIFORM false: always the per-lane form (the arrangement kernels, whose
// out-of-line quadrature measured 35 % slower with the three loop copies)
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

// Packed FP32 arithmetic (sm_100: add/sub/mul/fma.rn.f32x2, one instruction
// for two lanes of a float2); every value of the angular loops is a float2
// holding the same quantity for the two mirror pairs of a packed entry.
using V2 = float2;
__device__ __forceinline__ V2 v2(float a) { return make_float2(a, a); }
__device__ __forceinline__ V2 operator+(V2 a, V2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ V2 operator*(V2 a, V2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ V2 operator-(V2 a, V2 b)
{
    unsigned long long ra, rb, rr;
    memcpy(&ra, &a, 8);
    memcpy(&rb, &b, 8);
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rr) : "l"(ra), "l"(rb));
    V2 r;
    memcpy(&r, &rr, 8);
    return r;
}
__device__ __forceinline__ V2 fma2(V2 a, V2 b, V2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ V2 sel(bool c, V2 a, V2 b) { return c ? a : b; }

// Plain running sums, for callers whose error is set elsewhere (the gradient,
// whose pair sums stay far below the FP32 path's error bar, and the
// arrangement kernels, whose FP64 sum over the secondary's nodes averages the
// per-node rounding)
struct PlainSum
{
    V2 s = {0.0f, 0.0f};
    __device__ __forceinline__ void add(V2 x) { s = s + x; }
    __device__ __forceinline__ double value() const { return (double)s.x + (double)s.y; }
};

// FP64 running sum: each entry's two pair terms are added in FP32 (one
// rounding, relative to that entry's own term), converted and added in FP64,
// on pipes the FP32 integrands leave idle (the conversion built from the
// IEEE fields on the integer pipe instead measured 7 % slower for B)
struct F64Sum
{
    double s = 0.0;
    __device__ __forceinline__ void add(V2 x) { s += (double)(x.x + x.y); }
    __device__ __forceinline__ double value() const { return s; }
};

template <typename S>
struct Acc1
{
    S v;
};
template <typename S>
struct Acc3
{
    S h, y, e;
};
struct Acc4
{
    V2 a = {0.0f, 0.0f}, b = {0.0f, 0.0f}, c = {0.0f, 0.0f}, d = {0.0f, 0.0f};
};
__device__ __forceinline__ double hsum(V2 a) { return (double)a.x + (double)a.y; }

// reciprocal: MUFU estimate (within 1 ulp), no special-case handling needed
// since every argument here is a positive normal number; CCOIL_RCP_NEWTON=1
// adds a Newton-Raphson step (2 FMA), which measured 4-10 % slower for a
// per-field maximum error within 20 % of this form's (128-coil group, 2^20
// points)
#ifndef CCOIL_RCP_NEWTON
#define CCOIL_RCP_NEWTON 0
#endif
__device__ __forceinline__ float rcpApprox(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
#if CCOIL_RCP_NEWTON
    y = fmaf(y, fmaf(-x, y, 1.0f), y);
#endif
    return y;
}

// reciprocal square root: the MUFU estimate (relative error below 2^-22.9),
// flush-to-zero form (one instruction; every argument here is a positive
// normal number, a squared distance or 1 + u^2); a Newton-Raphson step
// (CCOIL_RSQRT_NEWTON=1) costs 4 FMA per call, measured 18 % slower (A, B, G
// of the 128-coil group at 2^20 points), and lowered the maximum error of A
// from 2.6e-6 to 1.4e-6 and of B from 1.2e-6 to 0.9e-6: the FP32 rounding of
// the per-node constants, not the estimate, sets the per-coil error
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

__device__ __forceinline__ bool nearWinding(const SegmentHeader &h, const Frame &f)
{
    return f.r > h.near_lo[0] && f.r < h.near_hi[0] && f.z > h.near_lo[1] && f.z < h.near_hi[1];
}

__device__ __forceinline__ V2 rcp2(V2 x) { return make_float2(rcpApprox(x.x), rcpApprox(x.y)); }
__device__ __forceinline__ V2 rsq2(V2 x) { return make_float2(rsqrtNR(x.x), rsqrtNR(x.y)); }

// asinh of both lanes in a tier the warp chose beforehand: 0 every argument
// below 0.25, 1 below 1, 2 per lane (the series and the polynomial packed)
__device__ __forceinline__ V2 asinhTier2(V2 u, int tier)
{
    if (tier == 0)
    {
        const V2 u2 = u * u;
        V2 p = v2(0.017352764f);
        p = fma2(p, u2, v2(-0.022372159f));
        p = fma2(p, u2, v2(0.030381944f));
        p = fma2(p, u2, v2(-0.044642857f));
        p = fma2(p, u2, v2(0.075f));
        p = fma2(p, u2, v2(-0.16666667f));
        return fma2(p * u2, u, u);
    }
    if (tier == 1)
    {
        const V2 x = u * u;
        V2 p = v2(6.495655980e-04f);
        p = fma2(p, x, v2(-3.737240797e-03f));
        p = fma2(p, x, v2(1.025899500e-02f));
        p = fma2(p, x, v2(-1.902823150e-02f));
        p = fma2(p, x, v2(2.937856875e-02f));
        p = fma2(p, x, v2(-4.446590319e-02f));
        p = fma2(p, x, v2(7.498393208e-02f));
        p = fma2(p, x, v2(-1.666660905e-01f));
        p = fma2(p, x, v2(1.0f));
        return u * p;
    }
    return make_float2(asinhAny(u.x), asinhAny(u.y));
}

// sqrt(1 + x) for 0 <= x < 1/16: 1 + x/2 - x^2/8 + x^3/16 - 5 x^4/128 + 7 x^5/256 - 21 x^6/1024
__device__ __forceinline__ V2 sqrt1pSeries(V2 x)
{
    V2 p = v2(-0.0205078125f);
    p = fma2(p, x, v2(0.02734375f));
    p = fma2(p, x, v2(-0.0390625f));
    p = fma2(p, x, v2(0.0625f));
    p = fma2(p, x, v2(-0.125f));
    p = fma2(p, x, v2(0.5f));
    return fma2(p, x, v2(1.0f));
}

// 1 / a and 1 / b from one reciprocal
struct PairInv
{
    V2 i1, i2;
};
__device__ __forceinline__ PairInv pairInverse(V2 a, V2 b)
{
    const V2 r = rcp2(a * b);
    return {b * r, a * r};
}

// Mirror-pair differences in closed form.  For the pair (c, -c) the second
// node's squared distances exceed the first's by delta = b2 (omcm - omc); with
// g = 1 / sqrt(D) and g' = 1 / sqrt(D + delta),
//   g - g' = delta e,  e = g^2 g'^2 / (g + g'),
// and every difference below is delta times a sum of terms of one sign, so its
// relative error stays that of a few FP32 roundings however far the point is
// (forming f(c) - f(-c) by subtraction loses the ratio distance / radius).
// The accumulated weight of a difference is w2c2 = 2 w c^2 (= w c delta / b2),
// so b2 multiplies the sums after the loop, in FP64.  Every quantity is a
// float2 over the two pairs of a packed entry.

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
// S: the running-sum type of the pair accumulation (F64Sum or PlainSum);
// UNIFORM: warp-uniform slab branches (bySlab)
template <int LANES, typename S = F64Sum, bool UNIFORM = true>
__device__ __forceinline__ double segmentA32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                             const PhiPair2 *pn, const Frame &f, int lane)
{
    double sum = 0.0;
    const int ne = packedEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool same = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot;
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const float dDf = (float)dD, dDl = (float)(dD - (double)dDf);
        const V2 TOP = v2(topf), BOT = v2(botf), NBOT = v2(-botf), DDF = v2(dDf), DDL = v2(dDl);
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
                const V2 B2 = v2(b2), D1 = v2(d1), D2 = v2(d2), Q = v2(qf);
                Acc1<S> a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc1<S> &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 dom = nd.omcm - nd.omc;  // delta / b2
                    const V2 den1 = fma2(B2, nd.omc, D1), den2 = fma2(B2, nd.omc, D2);
                    const V2 den1m = fma2(B2, nd.omcm, D1), den2m = fma2(B2, nd.omcm, D2);
                    const V2 s1 = den1 * rsq2(den1), s2 = den2 * rsq2(den2);
                    const V2 s1m = den1m * rsq2(den1m), s2m = den2m * rsq2(den2m);
                    const V2 ss1 = s1 + s1m, ss2 = s2 + s2m;
                    // 1 / (s1 + s1'), 1 / (s2 + s2') and 1 / V, 1 / V' (outside; inside the
                    // slab 1 / rho^2, 1 / rho'^2) from one reciprocal of the four
                    const V2 va = outside ? fma2(TOP, s2, BOT * s1) : fma2(B2, nd.omc, Q);
                    const V2 vb = outside ? fma2(TOP, s2m, BOT * s1m) : fma2(B2, nd.omcm, Q);
                    const V2 sp = ss1 * ss2, vp = va * vb;
                    const V2 r = rcp2(sp * vp);
                    const V2 rs = vp * r, rv = sp * r;  // 1 / (ss1 ss2), 1 / (va vb)
                    const PairInv is = {ss2 * rs, ss1 * rs}, iv = {vb * rv, va * rv};
                    V2 u, um, du;
                    if (outside)
                    {
                        u = fma2(DDL, iv.i1, DDF * iv.i1);
                        um = fma2(DDL, iv.i2, DDF * iv.i2);
                        du = fma2(TOP, is.i2, BOT * is.i1) * (u * iv.i2);
                    }
                    else
                    {
                        u = fma2(TOP, s2, NBOT * s1) * iv.i1;
                        um = fma2(TOP, s2m, NBOT * s1m) * iv.i2;
                        // top (bot^2 + s2 s2') / (s2 + s2') - bot (top^2 + s1 s1') / (s1 + s1'), both terms >= 0
                        du = fma2(TOP * fma2(BOT, BOT, s2 * s2m), is.i2, NBOT * fma2(TOP, TOP, s1 * s1m) * is.i1) * rv;
                    }
                    // sqrt(1 + u^2), sqrt(1 + u'^2): in tier 0 (|u| < 0.25) the binomial
                    // series through x^6 (x = u^2, truncation below 1e-10), otherwise MUFU
                    V2 sq, sqm;
                    if (tier == 0)
                    {
                        sq = sqrt1pSeries(u * u);
                        sqm = sqrt1pSeries(um * um);
                    }
                    else
                    {
                        const V2 y = fma2(u, u, v2(1.0f)), ym = fma2(um, um, v2(1.0f));
                        sq = y * rsq2(y);
                        sqm = ym * rsq2(ym);
                    }
                    const V2 arg = (du * (B2 * dom)) * ((u + um) * rcp2(fma2(u, sqm, um * sq)));
                    acc.v.add(nd.wc * asinhTier2(arg, tier));
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
                const float b2 = (float)b2d;
                const V2 B2 = v2(b2), Q = v2((float)q);
                Acc1<S> a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc1<S> &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 g = rsq2(fma2(B2, nd.omc, Q)), gm = rsq2(fma2(B2, nd.omcm, Q));
                    const V2 gg = g * gm;
                    acc.v.add(nd.w2c2 * (gg * gg * rcp2(g + gm)));
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
template <int LANES, typename S = F64Sum, bool UNIFORM = true>
__device__ __forceinline__ void segmentB32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const PhiPair2 *pn, const Frame &f, int lane, double &H, double &Z)
{
    H = 0.0;
    Z = 0.0;
    const int ne = packedEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool same = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot;
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const V2 TOP = v2(topf), BOT = v2(botf), NBOT = v2(-botf);
        bySlab<UNIFORM>(same, [&](auto slab) {
            const bool outside = slabOutside<decltype(slab)::value>(same);
            const double zScale = outside ? dD : 1.0;
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double q = (t.x - f.r) * (t.x - f.r), b2d = 2.0 * t.x * f.r;
                const float b2 = (float)b2d;
                const V2 B2 = v2(b2), Q = v2((float)q), D1 = v2((float)(top * top + q)),
                         D2 = v2((float)(bot * bot + q));
                const V2 N0 = v2((float)(t.x * (t.x - f.r))), N1 = v2((float)(t.x * f.r));
                Acc3<S> a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc3<S> &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 den1 = fma2(B2, nd.omc, D1), den2 = fma2(B2, nd.omc, D2);
                    const V2 den1m = fma2(B2, nd.omcm, D1), den2m = fma2(B2, nd.omcm, D2);
                    const V2 g1 = rsq2(den1), g2 = rsq2(den2), g1m = rsq2(den1m), g2m = rsq2(den2m);
                    // per node: hv = g1^2 g2^2 / (g1 + g2), y, and 1 / X, all from 1 / ((g1 + g2) X)
                    const V2 s = g1 + g2, sm = g1m + g2m;
                    const V2 t1 = TOP * g1, t2 = BOT * g2, t1m = TOP * g1m, t2m = BOT * g2m;
                    const V2 X = sel(outside, t1 + t2, fma2(B2, nd.omc, Q));
                    const V2 Xm = sel(outside, t1m + t2m, fma2(B2, nd.omcm, Q));
                    const V2 s1 = g1 + g1m, s2 = g2 + g2m;
                    // 1 / ((g1 + g2) X) per node and 1 / (s1 s2); merging all three into one
                    // reciprocal measured no faster (the FP32 pipe bounds the kernel)
                    const V2 R = rcp2(s * X), Rm = rcp2(sm * Xm), rc = rcp2(s1 * s2);
                    const V2 gg = g1 * g2, gg2 = gg * gg, ggm = g1m * g2m, gg2m = ggm * ggm;
                    const V2 hv = gg2 * (X * R), hvm = gg2m * (Xm * Rm);
                    const V2 ix = s * R, ixm = sm * Rm;
                    const V2 y = sel(outside, gg2, t1 - t2) * ix, ym = sel(outside, gg2m, t1m - t2m) * ixm;
                    const PairInv is = {s2 * rc, s1 * rc};
                    const V2 p1 = g1 * g1m, p2 = g2 * g2m;
                    const V2 e1 = p1 * p1 * is.i1, e2 = p2 * p2 * is.i2;
                    const V2 u1 = den1 * g1, u2m = den2m * g2m;
                    const V2 kh = ((u1 + u2m) + fma2(u1 * u1, p2 * is.i2, (u2m * u2m) * (p1 * is.i1))) * (hv * hvm);
                    const V2 ey = outside ? fma2(TOP * p1, fma2(e1, g2 * g2, g1m * (e2 * s2)),
                                                 BOT * p2 * fma2(e1 * s1, g2, g1m * g1m * e2)) *
                                                (ix * ixm)
                                          : (fma2(TOP, e1, NBOT * e2) + ym) * ix;
                    const V2 num = fma2(N1, nd.omc, N0);  // p^2 - p r c = p (p - r) + p r (1 - c)
                    acc.h.add(nd.w2c2 * kh);
                    acc.y.add(nd.w * ym);
                    acc.e.add(nd.wc * (num * ey));  // w c: the factor 2 after the loop
                });
                const double b2f = (double)b2;
                H += t.y * t.x * dD * b2f * (a0.h.value() + a1.h.value());
                Z += t.y * zScale *
                     (2.0 * t.x * t.x * (a0.y.value() + a1.y.value()) + 2.0 * b2f * (a0.e.value() + a1.e.value()));
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
                const float b2 = (float)b2d;
                const V2 B2 = v2(b2), Q = v2((float)q);
                const V2 N0 = v2((float)(t.x * (t.x - f.r))), N1 = v2((float)(t.x * f.r));
                Acc3<S> a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc3<S> &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 g = rsq2(fma2(B2, nd.omc, Q)), gm = rsq2(fma2(B2, nd.omcm, Q));
                    const V2 gg = g * gm, g2 = g * g, gm2 = gm * gm;
                    const V2 k3 = gg * gg * rcp2(g + gm) * (g2 + fma2(g, gm, gm2));
                    const V2 num = fma2(N1, nd.omc, N0);
                    acc.h.add(nd.w2c2 * k3);
                    acc.y.add(nd.w * (gm2 * gm));
                    acc.e.add(nd.wc * (num * k3));
                });
                const double w = l.y * t.y, b2f = (double)b2;
                H += w * t.x * zl * b2f * (a0.h.value() + a1.h.value());
                Z += w * (2.0 * t.x * t.x * (a0.y.value() + a1.y.value()) + 2.0 * b2f * (a0.e.value() + a1.e.value()));
            }
        }
    }
}

// The vector potential with each mirror pair's difference taken by
// subtraction (asinh(u) - asinh(u'), g - g'), for the arrangement kernels, for
// the reason given at segmentB32Direct.
template <int LANES, typename S = PlainSum>
__device__ __forceinline__ double segmentA32Direct(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                                   const PhiPair2 *pn, const Frame &f, int lane)
{
    double sum = 0.0;
    const int ne = packedEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool outside = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot;
        const float dDf = (float)(2.0 * f.z * (2.0 * h.half_length));
        const V2 TOP = v2(topf), BOT = v2(botf), NBOT = v2(-botf), DDF = v2(dDf);
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double q = (t.x - f.r) * (t.x - f.r), b2d = 2.0 * t.x * f.r;
            const float qf = (float)q, b2 = (float)b2d;
            const float d1 = (float)(top * top + q), d2 = (float)(bot * bot + q);
            float u0;
            {
                const float e1 = d1 * rsqrtNR(d1), e2 = d2 * rsqrtNR(d2);
                u0 = outside ? fabsf(dDf * rcpApprox(fmaf(topf, e2, botf * e1)))
                             : fabsf(fmaf(topf, e2, -botf * e1) * rcpApprox(qf));
            }
            const unsigned mask = __activemask();
            const int tier = __all_sync(mask, u0 < 0.25f) ? 0 : (__all_sync(mask, u0 <= 1.0f) ? 1 : 2);
            const V2 B2 = v2(b2), D1 = v2(d1), D2 = v2(d2), Q = v2(qf);
            Acc1<S> a0, a1;
            forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc1<S> &acc) {
                const PhiPair2 nd = pn[k];
                auto arg = [&](V2 om) {
                    const V2 den1 = fma2(B2, om, D1), den2 = fma2(B2, om, D2);
                    const V2 s1 = den1 * rsq2(den1), s2 = den2 * rsq2(den2);
                    const V2 num = sel(outside, DDF, fma2(TOP, s2, NBOT * s1));
                    const V2 den = sel(outside, fma2(TOP, s2, BOT * s1), fma2(B2, om, Q));
                    return num * rcp2(den);
                };
                const V2 diff = asinhTier2(arg(nd.omc), tier) - asinhTier2(arg(nd.omcm), tier);
                acc.v.add(nd.wc * diff);
            });
            sum += t.y * t.x * (a0.v.value() + a1.v.value());
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
                const V2 B2 = v2((float)b2d), Q = v2((float)q);
                Acc1<S> a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc1<S> &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 g = rsq2(fma2(B2, nd.omc, Q)), gm = rsq2(fma2(B2, nd.omcm, Q));
                    acc.v.add(nd.wc * (g - gm));
                });
                sum += l.y * t.y * t.x * (a0.v.value() + a1.v.value());
            }
        }
    }
    return sum;
}

// The field with each mirror pair's difference taken by subtraction, for the
// arrangement kernels: there every secondary node's field enters a sum over
// the secondary's ring that itself cancels (the flux through a loop is far
// smaller than the sum of |A| or |B| along it), and that cancellation, not the
// per-node error, sets the error of M and F, so the closed forms of
// segmentB32 measured no more accurate there and 57 % slower (F/T).
//   fast:  H w c (hv - hv'), Z w (num y + num' y') with hv = g1^2 g2^2 / (g1 + g2),
//          y = Y / X as in segmentB32 (dD inside Y outside the slab)
//   slow:  H w c (g^3 - g'^3), Z w (num g^3 + num' g'^3)
template <int LANES, typename S = PlainSum>
__device__ __forceinline__ void segmentB32Direct(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                                 const PhiPair2 *pn, const Frame &f, int lane, double &H, double &Z)
{
    H = 0.0;
    Z = 0.0;
    const int ne = packedEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool outside = top * bot > 0.0;
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const V2 TOP = v2((float)top), BOT = v2((float)bot), DDF = v2((float)dD);
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double q = (t.x - f.r) * (t.x - f.r), b2d = 2.0 * t.x * f.r;
            const V2 B2 = v2((float)b2d), Q = v2((float)q), D1 = v2((float)(top * top + q)),
                     D2 = v2((float)(bot * bot + q));
            const V2 N0 = v2((float)(t.x * (t.x - f.r))), N1 = v2((float)(t.x * f.r));
            Acc3<S> a0, a1;
            forEntriesSerial<LANES>(ne, lane, a0, a1, [&](int k, Acc3<S> &acc) {
                const PhiPair2 nd = pn[k];
                auto node = [&](V2 om, V2 &hv, V2 &zv) {
                    const V2 g1 = rsq2(fma2(B2, om, D1)), g2 = rsq2(fma2(B2, om, D2));
                    const V2 gg = g1 * g2, gg2 = gg * gg, s = g1 + g2;
                    const V2 t1 = TOP * g1, t2 = BOT * g2;
                    const V2 X = sel(outside, t1 + t2, fma2(B2, om, Q));
                    const V2 Y = sel(outside, DDF * gg2, t1 - t2);
                    const V2 R = rcp2(s * X);
                    hv = gg2 * (X * R);
                    zv = fma2(N1, om, N0) * Y * (s * R);
                };
                V2 hv, zv, hm, zm;
                node(nd.omc, hv, zv);
                node(nd.omcm, hm, zm);
                acc.h.add(nd.wc * (hv - hm));
                acc.y.add(nd.w * (zv + zm));
            });
            H += t.y * t.x * dD * (a0.h.value() + a1.h.value());
            Z += t.y * (a0.y.value() + a1.y.value());
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
                const V2 B2 = v2((float)b2d), Q = v2((float)q);
                const V2 N0 = v2((float)(t.x * (t.x - f.r))), N1 = v2((float)(t.x * f.r));
                Acc3<S> a0, a1;
                forEntriesSerial<LANES>(ne, lane, a0, a1, [&](int k, Acc3<S> &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 g = rsq2(fma2(B2, nd.omc, Q)), gm = rsq2(fma2(B2, nd.omcm, Q));
                    const V2 g3 = g * g * g, g3m = gm * gm * gm;
                    acc.y.add(nd.w * fma2(g3, fma2(N1, nd.omc, N0), g3m * fma2(N1, nd.omcm, N0)));
                    acc.h.add(nd.wc * (g3 - g3m));
                });
                const double w = l.y * t.y;
                H += w * t.x * zl * (a0.h.value() + a1.h.value());
                Z += w * (a0.y.value() + a1.y.value());
            }
        }
    }
}

// {RPhi, RR, RZ, ZZ}
template <int LANES>
__device__ __forceinline__ void segmentG32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const PhiPair2 *pn, const Frame &f, int lane, double *g)
{
    double rphi = 0.0, rr = 0.0, rz = 0.0, zz = 0.0;
    const double r = f.r;
    const int ne = packedEntries(h.n_phi);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool same = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot, lenf = (float)(2.0 * h.half_length);
        const double dD = 2.0 * f.z * (2.0 * h.half_length);
        const V2 TOP = v2(topf), BOT = v2(botf), NBOT = v2(-botf), LEN = v2(lenf), DDF = v2((float)dD),
                 NDDF = v2(-(float)dD);
        bySlab<true>(same, [&](auto slab) {
            const bool outside = slabOutside<decltype(slab)::value>(same);
            // one node: dg = G2 - G1, dg3 = G1^3 - G2^3, cz = T1 + Y (the RZ part
            // multiplying cos) and kz = k (2 Y + T1) / sin2 (sin2 = (b2 / 2) sin^2 is
            // the same for both nodes of a pair).  T1 = top G1^3 - bot G2^3 and
            // Y = (top G1 - bot G2) / rho^2, each in its cancellation-free form for a
            // point outside / inside the slab
            auto node = [&](V2 rho2, V2 den1, V2 den2, V2 &dg, V2 &dg3, V2 &cz, V2 &kz) {
                const V2 g1 = rsq2(den1), g2 = rsq2(den2);
                const V2 gg = g1 * g2, s = g1 + g2;
                const V2 t1 = TOP * g1, t2 = BOT * g2;
                const V2 yd = sel(outside, t1 + t2, rho2);
                // separate reciprocals: merging the three into one (1/a = bc rcp(abc))
                // measured 2 % slower, with the XU pipe at 75 % and the FP32 pipe at 64 %
                const V2 rs = rcp2(s), ryd = rcp2(yd), rrho = rcp2(rho2);
                const V2 gg2 = gg * gg, ggs = gg2 * rs;
                const V2 ddgg = DDF * gg2;
                dg = DDF * ggs;
                dg3 = (NDDF * ggs) * fma2(g1, g1, fma2(g1, g2, g2 * g2));
                const V2 g13 = g1 * g1 * g1;
                const V2 T1 = outside ? fma2(LEN, g13, BOT * dg3) : fma2(TOP, g13, NBOT * (g2 * g2 * g2));
                const V2 yn = sel(outside, ddgg, t1 - t2);
                const V2 Y = yn * ryd;
                cz = T1 + Y;
                kz = fma2(v2(2.0f), Y, T1) * rrho;
            };
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double q = (t.x - r) * (t.x - r), b2d = 2.0 * t.x * r;
                const V2 B2 = v2((float)b2d), NHB2 = v2(-(float)(0.5 * b2d)), Q = v2((float)q);
                const V2 D1 = v2((float)(top * top + q)), D2 = v2((float)(bot * bot + q));
                const V2 PF = v2((float)t.x), NPF = v2(-(float)t.x), RF = v2((float)r);
                // (r - p cos) = (r - p) + p (1 - cos); likewise (p - r cos)
                const V2 RMP = v2((float)(r - t.x)), NRMP = v2(-(float)(r - t.x)), PMR = v2((float)(t.x - r));
                Acc4 a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc4 &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 wc = nd.wc;
                    V2 dg, dg3, cz, kz, dgm, dg3m, czm, kzm;
                    node(fma2(B2, nd.omc, Q), fma2(B2, nd.omc, D1), fma2(B2, nd.omc, D2), dg, dg3, cz, kz);
                    node(fma2(B2, nd.omcm, Q), fma2(B2, nd.omcm, D1), fma2(B2, nd.omcm, D2), dgm, dg3m, czm, kzm);
                    acc.a = fma2(wc, dg - dgm, acc.a);
                    acc.b = fma2(wc, fma2(fma2(PF, nd.omc, RMP), dg3, fma2(NPF, nd.omcm, NRMP) * dg3m), acc.b);
                    acc.d = fma2(nd.w, fma2(fma2(RF, nd.omc, PMR), dg3, fma2(RF, nd.omcm, PMR) * dg3m), acc.d);
                    acc.c = fma2(wc, cz - czm, fma2(NHB2 * nd.ws2, kz + kzm, acc.c));  // -w p r sin^2 = -(b2 / 2) w (1 - c)(1 + c)
                });
                const double w = t.y * t.x;
                rphi += w / r * (hsum(a0.a) + hsum(a1.a));
                rr += w * (hsum(a0.b) + hsum(a1.b));
                zz += w * (hsum(a0.d) + hsum(a1.d));
                rz += w * (hsum(a0.c) + hsum(a1.c));
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
                const V2 B2 = v2((float)b2d), Q = v2((float)q);
                const V2 PF = v2((float)p), NPF = v2(-(float)p), RF = v2((float)r);
                const V2 RMP = v2((float)(r - p)), NRMP = v2(-(float)(r - p)), PMR = v2((float)(p - r));
                // RZ node G^5 (p cos (2p^2 + 2r^2 - zl^2 - p r cos) - 3 p^2 r) rewritten as
                // -p (cos G^3 + 3 G^5 (p - r cos)(r - p cos)) (G^5 D = G^3, D the squared
                // distance): its cos G^3 sum is the RPhi sum, so only the second sum is
                // accumulated, and the two are combined in FP64 after the loop
                Acc4 a0, a1;
                forEntries<LANES>(ne, lane, a0, a1, [&](int k, Acc4 &acc) {
                    const PhiPair2 nd = pn[k];
                    const V2 wc = nd.wc;
                    const V2 gq = rsq2(fma2(B2, nd.omc, Q)), gqm = rsq2(fma2(B2, nd.omcm, Q));
                    const V2 g3 = gq * gq * gq, g5 = g3 * gq * gq;
                    const V2 g3m = gqm * gqm * gqm, g5m = g3m * gqm * gqm;
                    const V2 rpc = fma2(PF, nd.omc, RMP), prc = fma2(RF, nd.omc, PMR);
                    const V2 rpcm = fma2(PF, nd.omcm, RMP), prcm = fma2(RF, nd.omcm, PMR);
                    acc.a = fma2(wc, g3 - g3m, acc.a);
                    acc.b = fma2(wc, fma2(g5, rpc, g5m * fma2(NPF, nd.omcm, NRMP)), acc.b);
                    acc.d = fma2(nd.w, fma2(g5, prc, g5m * prcm), acc.d);
                    acc.c = fma2(nd.w, fma2(g5 * prc, rpc, g5m * prcm * rpcm), acc.c);
                });
                const double w = l.y * t.y, ca = hsum(a0.a) + hsum(a1.a);
                rphi += w * p * zl / r * ca;
                rr += -3.0 * w * p * zl * (hsum(a0.b) + hsum(a1.b));
                zz += -3.0 * w * p * zl * (hsum(a0.d) + hsum(a1.d));
                rz += -w * p * (ca + 3.0 * (hsum(a0.c) + hsum(a1.c)));
            }
        }
    }
    g[0] = rphi;
    g[1] = rr;
    g[2] = rz;
    g[3] = zz;
}
