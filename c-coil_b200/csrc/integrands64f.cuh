#ifndef CCOIL_INTEGRANDS64F_CUH
#define CCOIL_INTEGRANDS64F_CUH

// Cheaper FP64 forms of the vector potential and the field, for FP64 work that
// needs FP64 accuracy but not the reference's operation sequence (which the
// FP64 field and arrangement kernels keep for 1e-12 parity): the refinement
// pass of FP32_REFINED plans, and the FP64 nodes (near-field and refined) of
// the FP32 arrangement kernels.  Included inside the kernels' anonymous
// namespaces after integrands64.cuh and integrands32.cuh.
//
//   rsqrt64: 1/sqrt(x) from the FP32 MUFU estimate (relative error below
//            2^-22.9) and two Newton-Raphson steps y <- y + y (1 - x y^2) / 2,
//            each squaring the relative error (below 2^-45, then below FP64's
//            rounding); arguments outside FP32's normal range take the IEEE path
//   sqrt64:  x rsqrt64(x)
__device__ __forceinline__ double rsqrt64(double x)
{
    if (!(x > 1e-36 && x < 1e36))
        return 1.0 / sqrt(x);
    double y = (double)rsqrtNR((float)x);
    double e = fma(-x * y, y, 1.0);
    y = fma(0.5 * y, e, y);
    e = fma(-x * y, y, 1.0);
    return fma(0.5 * y, e, y);
}
__device__ __forceinline__ double sqrt64(double x) { return x * rsqrt64(x); }

// The vector potential of one segment at one point, one thread.  Fast method:
// the reference's node value is log((e1 + d1) / (e2 + d2)) =
// asinh(top / sqrt(D)) - asinh(bot / sqrt(D)) (D = p^2 + r^2 - 2 p r c,
// e = sqrt(d^2 + 1)).  With A1 = |top| + s1, A2 = |bot| + s2,
// s = sqrt(top^2 + D) or sqrt(bot^2 + D), it is log(A1 / A2) above the coil's
// length slab (bot >= 0), log(A2 / A1) below it (top < 0) and log(A1 A2 / D)
// inside it: log(num / den) with num and den products of positive terms, so
// nothing cancels (the reference's e + d for d << 0 does), and two square
// roots per node instead of three.  The nodes phi and pi - phi form mirror
// pairs whose weighted cosines are opposite (symmetric Gauss-Legendre nodes
// and weights, up to their rounding), so a pair takes one logarithm:
//   w c lg + w' c' lg' = ((w c - w' c') / 2) log(num den' / (den num')).
// PAIRED: the table holds the mirror pairs as consecutive entries (the field
// plans' FP32-mode order, an odd table's middle node last); otherwise it is in
// the reference's order and the mirror of node k is node n - 1 - k.
// Against 40-digit arithmetic a pair is within 1.1e-11 (relative) where the
// reference's sequence is off by up to 2e-10.
// Slow method: w c p / sqrt(D) per node, as the reference.
template <bool PAIRED>
__device__ __forceinline__ double segmentA64Fast(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                                   const double2 *pt, const Frame &f)
{
    double sum = 0.0;
    const int n = h.n_phi;
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double cA = 2.0 * t.x * f.r, cB = t.x * t.x + f.r * f.r;
            const double T2 = top * top, B2 = bot * bot, aT = fabs(top), aB = fabs(bot);
            const bool above = bot >= 0.0, below = top < 0.0;
            auto ratio = [&](double c, double &num, double &den) {
                const double D = cB - cA * c;
                const double a1 = aT + sqrt64(T2 + D), a2 = aB + sqrt64(B2 + D);
                num = above ? a1 : (below ? a2 : a1 * a2);
                den = above ? a2 : (below ? a1 : D);
            };
            double part = 0.0;
            for (int m = 0; m < n / 2; ++m)
            {
                const double2 q = pt[PAIRED ? 2 * m : m], qm = pt[PAIRED ? 2 * m + 1 : n - 1 - m];
                double n1, e1, n2, e2;
                ratio(q.x, n1, e1);
                ratio(qm.x, n2, e2);
                part += 0.5 * (q.y * q.x - qm.y * qm.x) * log64((n1 * e2) / (e1 * n2));
            }
            if (n & 1)
            {
                // an odd table's middle node
                const double2 q = pt[PAIRED ? n - 1 : n / 2];
                double n1, e1;
                ratio(q.x, n1, e1);
                part += q.y * q.x * log64(n1 / e1);
            }
            sum += t.y * t.x * part;
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
                const double cA = 2.0 * t.x * f.r, cB = t.x * t.x + f.r * f.r + zl * zl;
                double part = 0.0;
                for (int k = 0; k < n; ++k)
                {
                    const double2 q = pt[k];
                    part += q.y * q.x * rsqrt64(cB - cA * q.x);
                }
                sum += l.y * t.y * t.x * part;
            }
        }
    }
    return sum;
}

// The field of one segment at one point, one thread:
// the reference's node values with every 1/sqrt(D) from rsqrt64 (fast method:
// w c (g2 - g1) and w (p^2 - p r c) / rho^2 (top g1 - bot g2); slow method:
// w g^3 (p^2 - p r c) and w g^3 p zl c)
__device__ __forceinline__ void segmentB64Fast(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                                 const double2 *pt, const Frame &f, double &H, double &Z)
{
    H = 0.0;
    Z = 0.0;
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double cA = t.x * t.x, cB = t.x * f.r, cC = cA + f.r * f.r;
            const double d1 = top * top + cC, d2 = bot * bot + cC;
            double h0 = 0.0, z0 = 0.0;
            for (int k = 0; k < h.n_phi; ++k)
            {
                const double2 q = pt[k];
                const double F = 2.0 * cB * q.x;
                const double g1 = rsqrt64(d1 - F), g2 = rsqrt64(d2 - F);
                h0 += q.y * q.x * (g2 - g1);
                z0 += q.y * ((cA - 0.5 * F) / (cC - F)) * (top * g1 - bot * g2);
            }
            H += t.y * t.x * h0;
            Z += t.y * z0;
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
                const double cA = t.x * t.x, cB = t.x * zl, cC = t.x * f.r;
                const double cD = cA + f.r * f.r + zl * zl;
                double h0 = 0.0, z0 = 0.0;
                for (int k = 0; k < h.n_phi; ++k)
                {
                    const double2 q = pt[k];
                    const double g = rsqrt64(cD - 2.0 * cC * q.x);
                    const double wg3 = q.y * (g * g * g);
                    z0 += wg3 * (cA - cC * q.x);
                    h0 += wg3 * (cB * q.x);
                }
                const double w = l.y * t.y;
                H += w * h0;
                Z += w * z0;
            }
        }
    }
}

#endif
