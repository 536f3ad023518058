#ifndef CCOIL_INTEGRANDS64F_CUH
#define CCOIL_INTEGRANDS64F_CUH

#include "fp64ops.cuh"

// Cheaper FP64 forms of the vector potential and the field, for FP64 work that
// needs FP64 accuracy but not the reference's operation sequence (which the
// FP64 field and arrangement kernels keep for 1e-12 parity): the refinement
// pass of FP32_REFINED plans, and the FP64 nodes (near-field and refined) of
// the FP32 arrangement kernels.  Included inside the kernels' anonymous
// namespaces after integrands64.cuh; the reciprocal square roots, square roots
// and divisions come from fp64ops.cuh.

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
// log(n / d): logRatio64 on the unchecked path, log64 of the IEEE quotient on
// the checked one
template <bool CHECKED> __device__ __forceinline__ double logRatio64t(double n, double d)
{
    return CHECKED ? log64(n / d) : logRatio64(n, d);
}

// One thickness node of the fast method: sum over the angular nodes.
template <bool PAIRED, bool CHECKED>
__device__ __forceinline__ double phiLoopA64(const double2 *pt, int n, double cA, double cB, double T2, double B2,
                                             double aT, double aB, bool above, bool below)
{
    auto ratio = [&](double c, double &num, double &den) {
        const double D = cB - cA * c;
        const double a1 = aT + sqrt64t<CHECKED>(T2 + D), a2 = aB + sqrt64t<CHECKED>(B2 + D);
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
        part += 0.5 * (q.y * q.x - qm.y * qm.x) * logRatio64t<CHECKED>(n1 * e2, e1 * n2);
    }
    if (n & 1)
    {
        // an odd table's middle node
        const double2 q = pt[PAIRED ? n - 1 : n / 2];
        double n1, e1;
        ratio(q.x, n1, e1);
        part += q.y * q.x * logRatio64t<CHECKED>(n1, e1);
    }
    return part;
}

template <bool PAIRED>
__device__ __forceinline__ double segmentA64Fast(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                                   const double2 *pt, const Frame &f)
{
    double sum = 0.0;
    const int n = h.n_phi;
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const double T2 = top * top, B2 = bot * bot, aT = fabs(top), aB = fabs(bot);
        const bool above = bot >= 0.0, below = top < 0.0;
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double cA = 2.0 * t.x * f.r, cB = t.x * t.x + f.r * f.r;
            // D in [cB - |cA|, cB + |cA|], the roots' arguments T2 + D and B2 + D
            // above it; D (the divisor inside the slab) and the products of
            // a = |t| + sqrt(t^2 + D) >= sqrt(D) that reach the division stay in
            // FP64's normal range with them
            const double k = fabs(cA);
            const bool fast = inRange64(cB - k, fmax(T2, B2) + (cB + k));
            const double part = fast ? phiLoopA64<PAIRED, false>(pt, n, cA, cB, T2, B2, aT, aB, above, below)
                                     : phiLoopA64<PAIRED, true>(pt, n, cA, cB, T2, B2, aT, aB, above, below);
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
                if (inRange64(cB - fabs(cA), cB + fabs(cA)))
                    for (int k = 0; k < n; ++k)
                    {
                        const double2 q = pt[k];
                        part += q.y * q.x * rsqrt64u(cB - cA * q.x);
                    }
                else
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
template <bool CHECKED>
__device__ __forceinline__ void phiLoopB64(const double2 *pt, int n, double cA, double cB, double cC, double d1,
                                           double d2, double top, double bot, double &h0, double &z0)
{
    for (int k = 0; k < n; ++k)
    {
        const double2 q = pt[k];
        const double F = 2.0 * cB * q.x;
        const double g1 = rsqrt64t<CHECKED>(d1 - F), g2 = rsqrt64t<CHECKED>(d2 - F);
        h0 += q.y * q.x * (g2 - g1);
        z0 += q.y * div64t<CHECKED>(cA - 0.5 * F, cC - F) * (top * g1 - bot * g2);
    }
}

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
            // F = 2 cB c in [-2 cB, 2 cB]: the roots' arguments d - F and the
            // divisor cC - F (<= both) lie in [cC - 2 cB, max(d1, d2) + 2 cB]
            if (inRange64(cC - 2.0 * fabs(cB), fmax(d1, d2) + 2.0 * fabs(cB)))
                phiLoopB64<false>(pt, h.n_phi, cA, cB, cC, d1, d2, top, bot, h0, z0);
            else
                phiLoopB64<true>(pt, h.n_phi, cA, cB, cC, d1, d2, top, bot, h0, z0);
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
                auto node = [&](const double2 q, double g) {
                    const double wg3 = q.y * (g * g * g);
                    z0 += wg3 * (cA - cC * q.x);
                    h0 += wg3 * (cB * q.x);
                };
                if (inRange64(cD - 2.0 * fabs(cC), cD + 2.0 * fabs(cC)))
                    for (int k = 0; k < h.n_phi; ++k)
                        node(pt[k], rsqrt64u(cD - 2.0 * cC * pt[k].x));
                else
                    for (int k = 0; k < h.n_phi; ++k)
                        node(pt[k], rsqrt64(cD - 2.0 * cC * pt[k].x));
                const double w = l.y * t.y;
                H += w * h0;
                Z += w * z0;
            }
        }
    }
}

#endif
