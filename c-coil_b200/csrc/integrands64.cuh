// FP64 integrands of the reference's CPU quadrature, node for node, shared by
// the field kernels (fields.cu) and the coil-pair kernels (pairs.cu).  Included
// inside an anonymous namespace.
//
//   A fast  src/Coil/Fields/CalculateFieldsFast.cxx:13-83
//   B fast  src/Coil/Fields/CalculateFieldsFast.cxx:85-160
//   G fast  src/Coil/Fields/CalculateFieldsFast.cxx:162-266
//   A/B/G slow  src/Coil/Fields/CalculateFieldsSlow.cxx:13-265
//   Cartesian wrappers  src/Coil/Fields/CalculateFieldsMethods.cxx:6-84

#include "log64.cuh"

struct Frame
{
    double z, r, cphi, sphi;
};

// point -> coil frame cylindrical coordinates: inverse transform of (p - centre)
// as vec3::Matrix3 * vec3::Vector3 evaluates it (Matrix3.cxx:50-55, left to right,
// no fused multiply-add), then (z, sqrt(x^2 + y^2), atan2(y, x)) as
// Vector3::getAsCylindricalCoords (Vector3.cxx:99-102); cos and sin of the
// azimuth are taken as x/r and y/r
// (T is double, or volatile double for a pose kept in shared memory)
template <typename T>
__device__ __forceinline__ Frame toCoilFrameAt(const T *pos, const T *M, double px, double py, double pz)
{
    double dx = __dsub_rn(px, pos[0]), dy = __dsub_rn(py, pos[1]), dz = __dsub_rn(pz, pos[2]);
    double x = __dadd_rn(__dadd_rn(__dmul_rn(M[0], dx), __dmul_rn(M[1], dy)), __dmul_rn(M[2], dz));
    double y = __dadd_rn(__dadd_rn(__dmul_rn(M[3], dx), __dmul_rn(M[4], dy)), __dmul_rn(M[5], dz));
    Frame f;
    f.z = __dadd_rn(__dadd_rn(__dmul_rn(M[6], dx), __dmul_rn(M[7], dy)), __dmul_rn(M[8], dz));
    f.r = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
    if (f.r > 0.0)
    {
        f.cphi = x / f.r;
        f.sphi = y / f.r;
    }
    else
    {
        f.cphi = 1.0;  // atan2(0, 0) = 0
        f.sphi = 0.0;
    }
    return f;
}

__device__ __forceinline__ Frame toCoilFrame(const SegmentHeader &h, double px, double py, double pz)
{
    return toCoilFrameAt(h.position, h.inv_transform, px, py, pz);
}

// ---------------------------------------------------------------------------
// FP64 segment integrals (cylindrical partial sums for one segment)
//
// Each node's value is computed with the reference's exact sequence of IEEE
// double operations (round-to-nearest multiply/add/divide/sqrt, evaluated left
// to right, no fused multiply-add), because several integrands cancel
// catastrophically inside a node (e + d for d << 0 in A, G2 - G1 in B, the RZ
// bracket of G): any other rounding would be amplified far above 1e-12 there.
// Only the weighting and the accumulation are reassociated.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double sqr(double a) { return __dsqrt_rn(a); }

template <int LANES>
__device__ __forceinline__ double segmentA64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                             const double2 *pt, const Frame &f, int lane)
{
    double sum = 0.0;
    if (h.fast)
    {
        // CalculateFieldsFast.cxx:27-78
        const double top = add(f.z, h.half_length), bot = sub(f.z, h.half_length);
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double cA = mul(mul(2.0, t.x), f.r);
            const double cB = add(mul(t.x, t.x), mul(f.r, f.r));
            double part = 0.0;
            for (int k = lane; k < h.n_phi; k += LANES)
            {
                const double2 q = pt[k];
                const double g = dvd(1.0, sqr(sub(cB, mul(cA, q.x))));
                const double d1 = mul(top, g), d2 = mul(bot, g);
                const double e1 = sqr(add(mul(d1, d1), 1.0)), e2 = sqr(add(mul(d2, d2), 1.0));
                const double lg = log64(dvd(add(e1, d1), add(e2, d2)));
                part += mul(mul(q.y, q.x), lg);
            }
            sum += mul(mul(t.y, t.x), part);
        }
    }
    else
    {
        // CalculateFieldsSlow.cxx:55-78
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = add(l.x, f.z);
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double cA = mul(mul(2.0, t.x), f.r);
                const double cB = add(add(mul(t.x, t.x), mul(f.r, f.r)), mul(zl, zl));
                double part = 0.0;
                for (int k = lane; k < h.n_phi; k += LANES)
                {
                    const double2 q = pt[k];
                    part += mul(q.y, dvd(mul(t.x, q.x), sqr(sub(cB, mul(cA, q.x)))));
                }
                sum += mul(mul(l.y, t.y), part);
            }
        }
    }
    return sum;
}

template <int LANES>
__device__ __forceinline__ void segmentB64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const double2 *pt, const Frame &f, int lane, double &H, double &Z)
{
    H = 0.0;
    Z = 0.0;
    if (h.fast)
    {
        // CalculateFieldsFast.cxx:100-155
        const double top = add(f.z, h.half_length), bot = sub(f.z, h.half_length);
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double cA = mul(t.x, t.x), cB = mul(t.x, f.r);
            const double cC = add(cA, mul(f.r, f.r));
            const double d1 = add(mul(top, top), cC), d2 = add(mul(bot, bot), cC);
            double h0 = 0.0, z0 = 0.0;
            for (int k = lane; k < h.n_phi; k += LANES)
            {
                const double2 q = pt[k];
                const double F = mul(mul(2.0, cB), q.x);
                const double g1 = dvd(1.0, sqr(sub(d1, F))), g2 = dvd(1.0, sqr(sub(d2, F)));
                h0 += mul(mul(q.y, q.x), sub(g2, g1));
                z0 += mul(mul(q.y, dvd(sub(cA, mul(0.5, F)), sub(cC, F))), sub(mul(top, g1), mul(bot, g2)));
            }
            H += mul(mul(t.y, t.x), h0);
            Z += mul(t.y, z0);
        }
    }
    else
    {
        // CalculateFieldsSlow.cxx:129-158
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = add(l.x, f.z);
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double cA = mul(t.x, t.x), cB = mul(t.x, zl), cC = mul(t.x, f.r);
                const double cD = add(add(cA, mul(f.r, f.r)), mul(zl, zl));
                double h0 = 0.0, z0 = 0.0;
                for (int k = lane; k < h.n_phi; k += LANES)
                {
                    const double2 q = pt[k];
                    const double F = mul(mul(2.0, cC), q.x);
                    const double den = sub(cD, F);
                    const double g = dvd(q.y, mul(den, sqr(den)));
                    z0 += mul(g, sub(cA, mul(cC, q.x)));
                    h0 += mul(g, mul(cB, q.x));
                }
                const double w = mul(l.y, t.y);
                H += mul(w, h0);
                Z += mul(w, z0);
            }
        }
    }
}

// {RPhi, RR, RZ, ZZ}
template <int LANES>
__device__ __forceinline__ void segmentG64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const double2 *pt, const Frame &f, int lane, double *g)
{
    double rphi = 0.0, rr = 0.0, rz = 0.0, zz = 0.0;
    const double r = f.r;
    if (h.fast)
    {
        // CalculateFieldsFast.cxx:179-254
        const double top = add(f.z, h.half_length), bot = sub(f.z, h.half_length);
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double A = mul(t.x, t.x), B = mul(r, r), C = mul(t.x, r);
            const double D = add(A, B), E = add(mul(A, A), mul(B, B)), F = mul(C, C);
            const double G1 = add(D, mul(top, top)), G2 = add(D, mul(bot, bot));
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            for (int k = lane; k < h.n_phi; k += LANES)
            {
                const double2 q = pt[k];
                const double c = q.x, c2 = mul(c, c);
                const double pe = mul(mul(2.0, C), c);
                const double J1 = sub(G1, pe), J2 = sub(G2, pe);
                const double K1 = sqr(J1), K2 = sqr(J2);
                const double L1 = dvd(1.0, mul(J1, K1)), L2 = dvd(1.0, mul(J2, K2));
                const double M = sub(D, pe);
                const double N = add(sub(mul(mul(mul(2.0, F), c), add(c2, 2.0)),
                                         mul(mul(C, add(mul(3.0, c2), 1.0)), D)),
                                     mul(c, E));
                const double O = sub(mul(c, D), mul(2.0, C));
                const double w = q.y;
                s0 += mul(mul(w, dvd(mul(t.x, c), r)), sub(dvd(1.0, K2), dvd(1.0, K1)));
                s1 += mul(mul(mul(w, sub(C, mul(A, c))), c), sub(L1, L2));
                s3 += mul(mul(w, sub(A, mul(C, c))), sub(L1, L2));
                s2 += mul(dvd(mul(w, t.x), mul(M, M)),
                          sub(mul(mul(top, L1), add(mul(O, J1), N)), mul(mul(bot, L2), add(mul(O, J2), N))));
            }
            rphi += mul(t.y, s0);
            rr += mul(t.y, s1);
            rz += mul(t.y, s2);
            zz += mul(t.y, s3);
        }
    }
    else
    {
        // CalculateFieldsSlow.cxx:212-251
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = add(l.x, f.z);
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double A = mul(t.x, t.x), B = mul(r, r), C = mul(zl, zl);
                const double D = mul(r, t.x), E = mul(t.x, zl), F = dvd(1.0, r);
                const double G = sub(add(mul(2.0, A), mul(2.0, B)), C), Hh = add(add(A, B), C);
                double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
                for (int k = lane; k < h.n_phi; k += LANES)
                {
                    const double2 q = pt[k];
                    const double c = q.x;
                    const double J = sub(Hh, mul(mul(2.0, D), c));
                    const double sJ = sqr(J);
                    const double X = dvd(q.y, mul(J, sJ));
                    const double Y = dvd(q.y, mul(mul(J, J), sJ));
                    s0 += mul(X, mul(mul(F, E), c));
                    s1 += mul(mul(Y, mul(-3.0, mul(E, sub(r, mul(t.x, c))))), c);
                    s3 += mul(Y, mul(-3.0, mul(E, sub(t.x, mul(r, c)))));
                    s2 += mul(Y, sub(mul(mul(t.x, sub(G, mul(D, c))), c), mul(mul(3.0, A), r)));
                }
                const double w = mul(l.y, t.y);
                rphi += mul(w, s0);
                rr += mul(w, s1);
                rz += mul(w, s2);
                zz += mul(w, s3);
            }
        }
    }
    g[0] = rphi;
    g[1] = rr;
    g[2] = rz;
    g[3] = zz;
}
// ---------------------------------------------------------------------------
// Epilogues: cylindrical partials -> Cartesian, rotated by the coil transform,
// added to the point's accumulators (linear in the partials, so per-lane
// partials can be rotated before the cross-lane reduction).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void addRotated(const SegmentHeader &h, double vx, double vy, double vz, double *acc)
{
    acc[0] += h.transform[0] * vx + h.transform[1] * vy + h.transform[2] * vz;
    acc[1] += h.transform[3] * vx + h.transform[4] * vy + h.transform[5] * vz;
    acc[2] += h.transform[6] * vx + h.transform[7] * vy + h.transform[8] * vz;
}

// CalculateFieldsMethods.cxx:39-84, including the on-axis branch and the T*G
// product of the reference.
__device__ __forceinline__ void addGradient(const SegmentHeader &h, const Frame &f, const double *g, double *acc)
{
    double G[9];
    double rphi = g[0], rr = g[1], rz = g[2], zz = g[3];
    if (f.r / h.inner_radius < 1e-12)
    {
        G[0] = rr; G[1] = 0.0; G[2] = 0.0;
        G[3] = 0.0; G[4] = rr; G[5] = 0.0;
        G[6] = 0.0; G[7] = 0.0; G[8] = zz;
    }
    else
    {
        double c = f.cphi, s = f.sphi;
        double xx = rr * c * c + rphi * s * s;
        double yy = rr * s * s + rphi * c * c;
        double xy = s * c * (rr - rphi);
        double xz = rz * c, yz = rz * s;
        G[0] = xx; G[1] = xy; G[2] = xz;
        G[3] = xy; G[4] = yy; G[5] = yz;
        G[6] = xz; G[7] = yz; G[8] = zz;
    }
    const double *T = h.transform;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            acc[3 * i + j] += T[3 * i] * G[j] + T[3 * i + 1] * G[3 + j] + T[3 * i + 2] * G[6 + j];
}

template <int FIELD, int LANES>
__device__ __forceinline__ void integrateSegment64(const unsigned char *seg, double px, double py, double pz, int lane,
                                                   double *acc)
{
    const SegmentHeader &h = *reinterpret_cast<const SegmentHeader *>(seg);
    const double2 *tt = reinterpret_cast<const double2 *>(seg) + h.off_t;
    const double2 *lt = reinterpret_cast<const double2 *>(seg) + h.off_l;
    const double2 *pt = reinterpret_cast<const double2 *>(seg) + h.off_phi;
    Frame f = toCoilFrame(h, px, py, pz);
    if (FIELD == CCOIL_FIELD_B)
    {
        double H, Z;
        segmentB64<LANES>(h, tt, lt, pt, f, lane, H, Z);
        addRotated(h, H * f.cphi, H * f.sphi, Z, acc);
    }
    else if (FIELD == CCOIL_FIELD_G)
    {
        double g[4];
        segmentG64<LANES>(h, tt, lt, pt, f, lane, g);
        addGradient(h, f, g, acc);
    }
    else
    {
        double a = segmentA64<LANES>(h, tt, lt, pt, f, lane) * h.field_factor;
        addRotated(h, -a * f.sphi, a * f.cphi, 0.0, acc);
    }
}

