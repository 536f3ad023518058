// Coil-pair kernels: mutual inductance and force/torque over many arrangements
// (the reference's CPU general case, evaluated for every arrangement at once).
//
// Reference algorithm per arrangement and primary (CPU path):
//   Coil::calculateMutualInductanceGeneral  src/Coil/MInductance/CalculateMInductanceGeneral.cxx:8-117
//   Coil::calculateForceTorqueGeneral       src/Coil/ForceAndTorque/CalculateForceGeneral.cxx:9-131
//   ring nodes  Coil::calculateRingIncrementPosition  src/Coil/Utils/SupportFunctions.cxx:72-122
//   coplanar axes  Coil::improvedPrecisionCase       src/Coil/Utils/SupportFunctions.cxx:124-161
//   group sums  CoilGroup::computeMutualInductance / computeForceTorque
//               src/CoilGroup/MInductance/ComputeMInductance.cxx:4-20,
//               src/CoilGroup/ForceAndTorque/ComputeForce.cxx:4-28
// The secondary is a cloud of nodes (length x thickness x azimuth); at each
// node the primary's A (for M) or B (for F/T) is the full field quadrature:
// FP64 (integrands64.cuh), or FP32-compensated (integrands32.cuh) with FP64
// for secondary nodes in the primary's near-field box.
//
// Mapping.  One warp per arrangement (grid-stride); the 32 lanes split the
// secondary's nodes, each lane evaluates the primary's whole quadrature at its
// node; the node tables are read from global memory (all lanes read the same
// primary node: L1 broadcast).  A fixed-order shuffle reduction per primary
// gives a deterministic result; primaries of a group are summed in order.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace ccoil
{
namespace
{
#include "integrands64.cuh"
#include "integrands32.cuh"
#include "integrands64f.cuh"

constexpr double kPi = 3.14159265358979323846;
constexpr double kMuReduced = 1e-7;

// One primary of a pair, followed in the blob by its tables.
struct alignas(16) PairHeader
{
    SegmentHeader prim;  // primary geometry (its own pose, used when primaries do not move) and node counts
    double m_factor;     // 2 pi N2 / (I1 lB tB aB): mutual inductance scale
    double f_factor;     // 2 pi I2 N2 / (lB tB aB): force/torque scale
    double prim_y_angle; // the primary's own orientation (used when primaries do not move)
    double prim_z_angle;
    int s_nl, s_nt, s_na, s_ablocks;  // secondary node counts and angular blocks
    int off_sl, off_st, off_sa;       // secondary tables (16-byte units from the header)
    int full_ring;                    // 1: always integrate the whole secondary ring (the reference's GPU
                                      // kernels), 0: half ring for coplanar axes (its CPU path)
    // parameter-gradient tables (16-byte units; 0 when absent): d(node position)/d(dimension)
    // of the primary's thickness and length nodes and of the secondary's length and
    // thickness nodes, i.e. the nodes' positions on [0, 1] (thickness) or [-1/2, 1/2] (length)
    int off_tu, off_lu, off_slu, off_stu;
};
static_assert(sizeof(PairHeader) % 16 == 0, "pair header alignment");

struct alignas(16) SecAngular
{
    double bpos;  // angular block index + 0.5
    double x;     // Gauss-Legendre node in [-1, 1]
    double w;     // its weight
    double pad;
};

struct Pose
{
    double pos[3];
    double T[9];
    double Ti[9];
};

// Coil::calculateTransformationMatrices (src/Coil/Utils/CalculateAttributes.cxx:65-78)
__device__ __forceinline__ void poseFromAngles(const double *p, Pose &o)
{
    o.pos[0] = p[0];
    o.pos[1] = p[1];
    o.pos[2] = p[2];
    double sY, cY, sZ, cZ;
    sincos(p[3], &sY, &cY);
    sincos(p[4], &sZ, &cZ);
    o.T[0] = cZ * cZ * cY - sZ * sZ;  o.T[1] = -sZ * cZ * cY - sZ * cZ;  o.T[2] = cZ * sY;
    o.T[3] = sZ * cZ * cY + sZ * cZ;  o.T[4] = cZ * cZ - sZ * sZ * cY;   o.T[5] = sZ * sY;
    o.T[6] = -sY * cZ;                o.T[7] = sY * sZ;                  o.T[8] = cY;
    o.Ti[0] = cZ * cZ * cY - sZ * sZ; o.Ti[1] = sZ * cZ * cY + sZ * cZ;  o.Ti[2] = -cZ * sY;
    o.Ti[3] = -sZ * cZ * cY - sZ * cZ; o.Ti[4] = cZ * cZ - sZ * sZ * cY; o.Ti[5] = sZ * sY;
    o.Ti[6] = sY * cZ;                o.Ti[7] = sY * sZ;                 o.Ti[8] = cY;
}

__device__ __forceinline__ void cross3(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// improvedPrecisionCase: when the two axes and the centre offset are coplanar
// the reference integrates half of the secondary ring starting at `offset`
__device__ __forceinline__ bool improvedCase(const double *pp, const double *sp, double &offset)
{
    const double pn[3] = {sin(pp[3]) * cos(pp[4]), sin(pp[3]) * sin(pp[4]), cos(pp[3])};
    const double sn[3] = {sin(sp[3]) * cos(sp[4]), sin(sp[3]) * sin(sp[4]), cos(sp[3])};
    const double d[3] = {pp[0] - sp[0], pp[1] - sp[1], pp[2] - sp[2]};
    double pl[3];
    cross3(pn, d, pl);
    const double dot = pl[0] * sn[0] + pl[1] * sn[1] + pl[2] * sn[2];
    offset = 0.0;
    if (!(fabs(dot) <= 1e-14))
        return false;
    if (pl[0] == 0.0 && pl[1] == 0.0 && pl[2] == 0.0)
        cross3(sn, d, pl);
    if (pl[0] == 0.0 && pl[1] == 0.0 && pl[2] == 0.0)
        cross3(sn, pn, pl);
    offset = atan2(cos(sp[3]) * (pl[0] * cos(sp[4]) + pl[1] * sin(sp[4])) - pl[2] * sin(sp[3]),
                   pl[0] * sin(sp[4]) - pl[1] * cos(sp[4]));
    return true;
}

// Coil::isZAxisCase (src/Coil/Utils/SupportFunctions.cxx:55-70)
__device__ __forceinline__ bool zAxisCase(const double *pp, const double *sp, double primR)
{
    return fabs(pp[0] / primR) < 1e-12 && fabs(pp[1] / primR) < 1e-12 && fabs(sp[0] / primR) < 1e-12 &&
           fabs(sp[1] / primR) < 1e-12 && fabs(pp[3] / (2 * kPi)) < 1e-12 && fabs(sp[3] / (2 * kPi)) < 1e-12;
}

// A_phi of the primary at a point and its derivatives in r and z (coil frame):
//   fast node  a = r' c [asinh(top/rho) - asinh(bot/rho)],
//              da/dz = r' c (g1 - g2),  da/dr = -r' c (r - r' c)(top g1 - bot g2) / rho^2
//   slow node  a = r' c / sqrt(D),  da/dz = -r' c zl D^-3/2,  da/dr = -r' c (r - r' c) D^-3/2
// (the value `a` uses the reference's operation sequence, as segmentA64)
__device__ __forceinline__ void segmentAGrad64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                               const double2 *pt, const Frame &f, double &A, double &Ar, double &Az)
{
    A = segmentA64<1>(h, tt, lt, pt, f, 0);
    Ar = 0.0;
    Az = 0.0;
    const double r = f.r;
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            double sr = 0.0, sz = 0.0;
            for (int k = 0; k < h.n_phi; ++k)
            {
                const double2 q = pt[k];
                const double c = q.x;
                const double rho2 = t.x * t.x + r * r - 2.0 * t.x * r * c;
                const double g1 = rsqrt(rho2 + top * top), g2 = rsqrt(rho2 + bot * bot);
                sz += q.y * c * (g1 - g2);
                sr -= q.y * c * (r - t.x * c) * (top * g1 - bot * g2) / rho2;
            }
            Ar += t.y * t.x * sr;
            Az += t.y * t.x * sz;
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
                double sr = 0.0, sz = 0.0;
                for (int k = 0; k < h.n_phi; ++k)
                {
                    const double2 q = pt[k];
                    const double c = q.x;
                    const double D = t.x * t.x + r * r - 2.0 * t.x * r * c + zl * zl;
                    const double g = rsqrt(D), g3 = g * g * g;
                    sz -= q.y * c * zl * g3;
                    sr -= q.y * c * (r - t.x * c) * g3;
                }
                Ar += l.y * t.y * t.x * sr;
                Az += l.y * t.y * t.x * sz;
            }
        }
    }
}

// Derivatives of the primary's A_phi(r, z) at one point (coil frame) for the
// parameter gradient, given its value a: with respect to r and z (for the
// Jacobian) and to the primary's inner radius R, thickness a and length b.
// With the current density N I / (a b) folded into the node weights, the
// thickness integral (a / 2) sum w_i f(r'_i) makes the weights independent of
// a, so d/dR = sum w_i df/dr', d/da = sum w_i u_i df/dr' (u_i = dr'_i/da), and
// for the fast method d/db = -a/b + the derivative of the length limits
// (top, bot = z +- b/2); for the slow method d/db moves the length nodes.
//   fast node  f = r' c V,  V = asinh(top/rho) - asinh(bot/rho)
//              df/dr' = c V - r' c (r' - r c)(top g1 - bot g2) / rho^2,  dV/db = (g1 + g2) / 2
//   slow node  f = r' c g,  g = D^-1/2
//              df/dr' = c g - r' c (r' - r c) g^3,  df/dzl = -r' c zl g^3
// out: {dA/dr, dA/dz, dA/dR, dA/da, dA/db}
__device__ __noinline__ void segmentAParams64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                              const double2 *pt, const double2 *tu, const double2 *lu,
                                              const Frame &f, double a, double *out)
{
    const double r = f.r;
    double Ar = 0.0, Az = 0.0, dR = 0.0, dA = 0.0, dB = 0.0;
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double p = t.x;
            double sr = 0.0, sz = 0.0, sp = 0.0, sb = 0.0;
            for (int k = 0; k < h.n_phi; ++k)
            {
                const double2 q = pt[k];
                const double c = q.x;
                const double rho2 = p * p + r * r - 2.0 * p * r * c;
                const double g1 = rsqrt(rho2 + top * top), g2 = rsqrt(rho2 + bot * bot);
                const double irho = rsqrt(rho2);
                const double V = asinh(top * irho) - asinh(bot * irho);
                const double tg = top * g1 - bot * g2;
                sz += q.y * c * (g1 - g2);
                sr -= q.y * c * (r - p * c) * tg / rho2;
                sp += q.y * c * (V - p * (p - r * c) * tg / rho2);
                sb += q.y * c * 0.5 * (g1 + g2);
            }
            Ar += t.y * p * sr;
            Az += t.y * p * sz;
            dR += t.y * sp;
            dA += t.y * tu[j].x * sp;
            dB += t.y * p * sb;
        }
        dB -= a / (2.0 * h.half_length);
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
                double sr = 0.0, sz = 0.0, sp = 0.0;
                for (int k = 0; k < h.n_phi; ++k)
                {
                    const double2 q = pt[k];
                    const double c = q.x;
                    const double D = p * p + r * r - 2.0 * p * r * c + zl * zl;
                    const double g = rsqrt(D), g3 = g * g * g;
                    sz -= q.y * c * zl * g3;
                    sr -= q.y * c * (r - p * c) * g3;
                    sp += q.y * (c * g - p * c * (p - r * c) * g3);
                }
                const double w = l.y * t.y;
                Ar += w * p * sr;
                Az += w * p * sz;
                dR += w * sp;
                dA += w * tu[j].x * sp;
                dB += w * lu[i].x * p * sz;
            }
        }
    }
    out[0] = Ar;
    out[1] = Az;
    out[2] = dR;
    out[3] = dA;
    out[4] = dB;
}

// The same five derivatives with the primary's quadrature in FP32 (mirror
// pairs, two per packed step, differences by subtraction as in the FP32
// arrangement integrands; the FP64 sum over the secondary's nodes follows).
// Per node h(c) multiplies c, so a pair adds w c (h(c) - h(-c)):
//   fast  h_z = g1 - g2 = -dD g1^2 g2^2 / (g1 + g2),  h_r = -(r - p c) y,
//         h_p = V - p (p - r c) y,  h_b = (g1 + g2) / 2,
//         y = (top g1 - bot g2) / rho^2 (its cancellation-free form outside the slab),
//         V = asinh(u) in the single-asinh form of segmentA32Direct
//   slow  h_z = -zl g^3,  h_r = -(r - p c) g^3,  h_p = g - p (p - r c) g^3
__device__ __noinline__ void segmentAParams32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                              const PhiPair2 *pn, const double2 *tu, const double2 *lu,
                                              const Frame &f, double a, double *out)
{
    const double r = f.r;
    const int ne = packedEntries(h.n_phi);
    double Ar = 0.0, Az = 0.0, dR = 0.0, dA = 0.0, dB = 0.0;
    const V2 RF = v2((float)r);
    if (h.fast)
    {
        const double top = f.z + h.half_length, bot = f.z - h.half_length;
        const bool outside = top * bot > 0.0;
        const float topf = (float)top, botf = (float)bot;
        const float dDf = (float)(2.0 * f.z * (2.0 * h.half_length));
        const V2 TOP = v2(topf), BOT = v2(botf), NBOT = v2(-botf), DDF = v2(dDf), NDDF = v2(-dDf);
        for (int j = 0; j < h.n_t; ++j)
        {
            const double2 t = tt[j];
            const double p = t.x, q = (p - r) * (p - r), b2d = 2.0 * p * r;
            const float qf = (float)q, d1 = (float)(top * top + q), d2 = (float)(bot * bot + q);
            float u0;
            {
                const float e1 = d1 * rsqrtNR(d1), e2 = d2 * rsqrtNR(d2);
                u0 = outside ? fabsf(dDf * rcpApprox(fmaf(topf, e2, botf * e1)))
                             : fabsf(fmaf(topf, e2, -botf * e1) * rcpApprox(qf));
            }
            const unsigned mask = __activemask();
            const int tier = __all_sync(mask, u0 < 0.25f) ? 0 : (__all_sync(mask, u0 <= 1.0f) ? 1 : 2);
            const V2 B2 = v2((float)b2d), Q = v2(qf), D1 = v2(d1), D2 = v2(d2), PF = v2((float)p);
            const V2 RMP = v2((float)(r - p)), PMR = v2((float)(p - r));
            Acc4 a0, a1;
            forEntries<1>(ne, 0, a0, a1, [&](int k, Acc4 &acc) {
                const PhiPair2 nd = pn[k];
                auto node = [&](V2 om, V2 &hz, V2 &hr, V2 &hp, V2 &hb) {
                    const V2 den1 = fma2(B2, om, D1), den2 = fma2(B2, om, D2), rho2 = fma2(B2, om, Q);
                    const V2 g1 = rsq2(den1), g2 = rsq2(den2);
                    const V2 s = g1 + g2, gg = g1 * g2, gg2 = gg * gg;
                    const V2 t1 = TOP * g1, t2 = BOT * g2;
                    const V2 X = sel(outside, t1 + t2, rho2);
                    const V2 R = rcp2(s * X);
                    const V2 y = sel(outside, DDF * gg2, t1 - t2) * (s * R);
                    const V2 s1 = den1 * g1, s2 = den2 * g2;
                    const V2 u = sel(outside, DDF, fma2(TOP, s2, NBOT * s1)) *
                                 rcp2(sel(outside, fma2(TOP, s2, BOT * s1), rho2));
                    const V2 V = asinhTier2(u, tier);
                    hz = NDDF * gg2 * (X * R);
                    hr = v2(0.0f) - fma2(PF, om, RMP) * y;
                    hp = V - PF * fma2(RF, om, PMR) * y;
                    hb = v2(0.5f) * s;
                };
                V2 hz, hr, hp, hb, hzm, hrm, hpm, hbm;
                node(nd.omc, hz, hr, hp, hb);
                node(nd.omcm, hzm, hrm, hpm, hbm);
                const V2 wc = nd.wc;
                acc.a = fma2(wc, hz - hzm, acc.a);
                acc.b = fma2(wc, hr - hrm, acc.b);
                acc.c = fma2(wc, hp - hpm, acc.c);
                acc.d = fma2(wc, hb - hbm, acc.d);
            });
            const double sz = hsum(a0.a) + hsum(a1.a), sr = hsum(a0.b) + hsum(a1.b);
            const double sp = hsum(a0.c) + hsum(a1.c), sb = hsum(a0.d) + hsum(a1.d);
            Ar += t.y * p * sr;
            Az += t.y * p * sz;
            dR += t.y * sp;
            dA += t.y * tu[j].x * sp;
            dB += t.y * p * sb;
        }
        dB -= a / (2.0 * h.half_length);
    }
    else
    {
        for (int i = 0; i < h.n_l; ++i)
        {
            const double2 l = lt[i];
            const double zl = l.x + f.z;
            const V2 NZL = v2(-(float)zl);
            for (int j = 0; j < h.n_t; ++j)
            {
                const double2 t = tt[j];
                const double p = t.x, q = (p - r) * (p - r) + zl * zl, b2d = 2.0 * p * r;
                const V2 B2 = v2((float)b2d), Q = v2((float)q), PF = v2((float)p);
                const V2 RMP = v2((float)(r - p)), PMR = v2((float)(p - r));
                Acc4 a0, a1;
                forEntries<1>(ne, 0, a0, a1, [&](int k, Acc4 &acc) {
                    const PhiPair2 nd = pn[k];
                    auto node = [&](V2 om, V2 &hz, V2 &hr, V2 &hp) {
                        const V2 g = rsq2(fma2(B2, om, Q)), g3 = g * g * g;
                        hz = NZL * g3;
                        hr = v2(0.0f) - fma2(PF, om, RMP) * g3;
                        hp = g - PF * fma2(RF, om, PMR) * g3;
                    };
                    V2 hz, hr, hp, hzm, hrm, hpm;
                    node(nd.omc, hz, hr, hp);
                    node(nd.omcm, hzm, hrm, hpm);
                    const V2 wc = nd.wc;
                    acc.a = fma2(wc, hz - hzm, acc.a);
                    acc.b = fma2(wc, hr - hrm, acc.b);
                    acc.c = fma2(wc, hp - hpm, acc.c);
                });
                const double sz = hsum(a0.a) + hsum(a1.a), sr = hsum(a0.b) + hsum(a1.b);
                const double sp = hsum(a0.c) + hsum(a1.c);
                const double w = l.y * t.y;
                Ar += w * p * sr;
                Az += w * p * sz;
                dR += w * sp;
                dA += w * tu[j].x * sp;
                dB += w * lu[i].x * p * sz;
            }
        }
    }
    out[0] = Ar;
    out[1] = Az;
    out[2] = dR;
    out[3] = dA;
    out[4] = dB;
}

// d T / d(y axis angle) and d T / d(z axis angle) of poseFromAngles' transform
__device__ __forceinline__ void transformDerivatives(double yA, double zA, double *dTy, double *dTz)
{
    double sY, cY, sZ, cZ;
    sincos(yA, &sY, &cY);
    sincos(zA, &sZ, &cZ);
    dTy[0] = -cZ * cZ * sY; dTy[1] = sZ * cZ * sY;  dTy[2] = cZ * cY;
    dTy[3] = -sZ * cZ * sY; dTy[4] = sZ * sZ * sY;  dTy[5] = sZ * cY;
    dTy[6] = -cY * cZ;      dTy[7] = cY * sZ;       dTy[8] = -sY;
    const double c2 = cZ * cZ - sZ * sZ, s2 = 2.0 * sZ * cZ;
    dTz[0] = -s2 * (cY + 1.0); dTz[1] = -c2 * (cY + 1.0); dTz[2] = -sZ * sY;
    dTz[3] = c2 * (cY + 1.0);  dTz[4] = -s2 * (1.0 + cY); dTz[5] = cZ * sY;
    dTz[6] = sY * sZ;          dTz[7] = sY * cZ;          dTz[8] = 0.0;
}

#ifndef CCOIL_PAIR_MIN_BLOCKS
#define CCOIL_PAIR_MIN_BLOCKS 6
#endif
// the same for the FP32 variants (M and F/T, packed integrands with the
// subtracted mirror differences): 9 measured best against 6 (M 69.6 and
// 75.2 ms at 2^18 arrangements; F/T 48.0 and 48.5 ms); their lanes wait on
// fixed-latency chains, which more resident warps hide
#ifndef CCOIL_PAIR32_MIN_BLOCKS
#define CCOIL_PAIR32_MIN_BLOCKS 9
#endif
// the FP32_REFINED variants, whose refined nodes run the FP64 forms: 9 measured
// as fast as 8, 7 and 6 (80 registers) at the fractions that reach 1e-7 (M
// 124.4 against 124.7-126.5 ms at 2^18 arrangements; F/T 104.1 against
// 103.0-104.1 ms), and faster at the default fraction (M 72.1 against 73.9-76.0)
#ifndef CCOIL_PAIR32R_MIN_BLOCKS
#define CCOIL_PAIR32R_MIN_BLOCKS 9
#endif
// FP32_REFINED arrangements: the largest scratch of node contributions (the
// grid shrinks to fit it)
constexpr size_t kPairRefineScratchBytes = size_t(1) << 30;
// largest single-primary blob staged in shared memory (0 turns staging off)
#ifndef CCOIL_PAIR_STAGE_MAX_BYTES
#define CCOIL_PAIR_STAGE_MAX_BYTES (48 * 1024)
#endif

// What a warp needs of its current arrangement and primary, written by lane 0
// into shared memory and read back by all lanes inside the secondary-node loop
// (volatile: kept out of registers, which the primary quadrature needs)
struct WarpPose
{
    double pos[3], T[9], Ti[9];  // primary pose
    double sp[3];                // secondary centre
    double sA, cA, sB, cB;       // sin / cos of the secondary's y and z axis angles
    double offset, ablk;         // secondary azimuth offset and angular block size
    double dTy[9], dTz[9];       // d(primary transform)/d(y, z axis angle) (parameter gradient only)
    int skip;                    // coaxial pair left to the z-axis pass
};

// FP64 primary quadrature at one secondary node, out of line for the FP32
// kernel (which takes it only for near-field nodes) so that its register
// budget does not carry the FP64 integrands.  The point's frame coordinates
// pass by value (the quadrature reads z and r only), so nothing of the
// caller's has to sit in memory for the call.
__device__ __forceinline__ Frame frameZR(double z, double r)
{
    Frame f;
    f.z = z;
    f.r = r;
    f.cphi = 1.0;
    f.sphi = 0.0;
    return f;
}

__device__ __noinline__ double pairA64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                       const double2 *pt, double z, double r)
{
    return segmentA64<1>(h, tt, lt, pt, frameZR(z, r), 0);
}

__device__ __noinline__ double2 pairB64(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                        const double2 *pt, double z, double r)
{
    double H, Z;
    segmentB64<1>(h, tt, lt, pt, frameZR(z, r), 0, H, Z);
    return make_double2(H, Z);
}

// The FP32 kernels' FP64 nodes (near-field and refined): FP64 accuracy without
// the reference's operation sequence, in the cheaper forms of
// integrands64f.cuh (the table is in the reference's order)
__device__ __noinline__ double pairA64Fast(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                           const double2 *pt, double z, double r)
{
    return segmentA64Fast<false>(h, tt, lt, pt, frameZR(z, r));
}

__device__ __noinline__ double2 pairB64Fast(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                            const double2 *pt, double z, double r)
{
    double H, Z;
    segmentB64Fast(h, tt, lt, pt, frameZR(z, r), H, Z);
    return make_double2(H, Z);
}

// The FP32 primary quadrature, out of line as well: the loop over the
// primary's nodes gets the whole register budget.  Its pair sums are plain
// FP32: the FP64 sum over the secondary's nodes averages their rounding
// (measured: the same error statistics against FP64 as with compensated sums,
// at 7-18 % less time)
__device__ __noinline__ double pairA32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                       const PhiPair2 *pn, double z, double r)
{
    return segmentA32Direct<1, PlainSum>(h, tt, lt, pn, frameZR(z, r), 0);
}

__device__ __noinline__ double2 pairB32(const SegmentHeader &h, const double2 *tt, const double2 *lt,
                                        const PhiPair2 *pn, double z, double r)
{
    double H, Z;
    segmentB32Direct<1, PlainSum>(h, tt, lt, pn, frameZR(z, r), 0, H, Z);
    return make_double2(H, Z);
}

// 1: the FP64 kernel calls the out-of-line FP64 quadrature too
#ifndef CCOIL_PAIR_CALL_FP64
#define CCOIL_PAIR_CALL_FP64 0
#endif

// stagedBytes > 0: there is one primary and its whole pair blob (stagedBytes,
// a multiple of 16) is copied into shared memory once per CTA, so the inner
// quadrature reads its tables from shared memory instead of through L1.
//
// FP32 (mutual inductance and force/torque only): the primary quadrature at a
// secondary node runs in the FP32-compensated integrands, except for nodes in
// the primary's near-field box: the warp defers those to a list in shared
// memory and evaluates them with the FP64 integrands 32 at a time, so the FP64
// work runs on full warps instead of dragging whole mixed iterations along;
// the secondary-node sums and the cross-lane reduction stay FP64.
//
// REFINE (FP32_REFINED, M and F/T): each secondary node's FP32 contribution is
// also written to the warp's region of nodeScratch (node-major, W doubles per
// node; deferred near-field nodes as zeros).  Once the warp has the primary's
// total, every node whose contribution exceeds `fraction` of it (for F/T: of
// the force or of the torque) is taken out of the sums and evaluated again
// with the FP64 integrands, 32 at a time like the near-field nodes: the nodes
// that dominate an arrangement whose ring sum cancels, whose FP32 errors the
// cancellation magnifies.
template <int QTY, bool FP32, bool REFINE = false>
__global__ void __launch_bounds__(128, FP32 ? (REFINE ? CCOIL_PAIR32R_MIN_BLOCKS : CCOIL_PAIR32_MIN_BLOCKS)
                                               : CCOIL_PAIR_MIN_BLOCKS)
    pairKernel64(const unsigned char *__restrict__ blob, const long long *__restrict__ primOffsets, int nprim,
                 const double *__restrict__ primPoses, const double *__restrict__ secPoses, long long count,
                 double *__restrict__ out, unsigned long long *__restrict__ zAxisCount, int stagedBytes,
                 const long long *__restrict__ zOffsets, long long *__restrict__ zList,
                 unsigned long long *__restrict__ zListCount, double *__restrict__ nodeScratch, int scratchNodes,
                 double fraction)
{
    extern __shared__ __align__(16) unsigned char stagedPair[];
    __shared__ WarpPose warpPoses[4];
    __shared__ int nearLists[4][64];  // FP32: each warp's deferred near-field secondary nodes
    constexpr int W = QTY == 0 ? 1 : QTY == 1 ? 6 : QTY == 2 ? 3 : 14;
    // Running sums in shared memory: each thread's sums over its secondary nodes
    // (one column per thread, so a warp's accesses hit 32 consecutive doubles)
    // and each warp's sums over the primaries (lane 0).  Held in registers they
    // stayed live across the out-of-line quadrature call and spilled to local
    // memory at the register budget of 9 CTAs per SM.
    __shared__ double laneSums[W][128];
    __shared__ double warpSums[4][W];
    if (stagedBytes > 0)
    {
        const int4 *src = reinterpret_cast<const int4 *>(blob + primOffsets[0]);
        int4 *dst = reinterpret_cast<int4 *>(stagedPair);
        for (int i = threadIdx.x; i < stagedBytes / 16; i += blockDim.x)
            dst[i] = src[i];
        __syncthreads();
    }
    const int lane = threadIdx.x % 32;
    volatile WarpPose &S = warpPoses[threadIdx.x / 32];
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const long long warps = (long long)gridDim.x * blockDim.x / 32;
    double *part = &laneSums[0][threadIdx.x];  // part[128 i]: this thread's sum i
    double *total = warpSums[threadIdx.x / 32];
    for (long long a = warp; a < count; a += warps)
    {
        if (lane == 0)
            for (int i = 0; i < W; ++i)
                total[i] = 0.0;
        bool hasZ = false;  // lane 0: some primary of this arrangement is left to the z-axis pass
        for (int j = 0; j < nprim; ++j)
        {
            const unsigned char *base = stagedBytes > 0 ? stagedPair : blob + primOffsets[j];
            const PairHeader &ph = *reinterpret_cast<const PairHeader *>(base);
            const SegmentHeader &h = ph.prim;
            const double2 *tt = reinterpret_cast<const double2 *>(base) + h.off_t;
            const double2 *lt = reinterpret_cast<const double2 *>(base) + h.off_l;
            const double2 *pt = reinterpret_cast<const double2 *>(base) + h.off_phi;
            const double2 *sl = reinterpret_cast<const double2 *>(base) + ph.off_sl;
            const double2 *st = reinterpret_cast<const double2 *>(base) + ph.off_st;
            const SecAngular *sa = reinterpret_cast<const SecAngular *>(reinterpret_cast<const double2 *>(base) +
                                                                        ph.off_sa);
            const PhiPair2 *pn = reinterpret_cast<const PhiPair2 *>(reinterpret_cast<const double2 *>(base) +
                                                                    h.off_f32);
            __syncwarp();  // every lane is done with the previous pose
            if (lane == 0)
            {
                const double *sp = secPoses + 5 * a;
                Pose P;
                double ppose[5], spose[5];
                for (int i = 0; i < 5; ++i)
                    spose[i] = sp[i];
                if (primPoses)
                {
                    for (int i = 0; i < 5; ++i)
                        ppose[i] = primPoses[5 * a + i];
                    poseFromAngles(ppose, P);
                }
                else
                {
                    for (int i = 0; i < 3; ++i)
                        P.pos[i] = ppose[i] = h.position[i];
                    for (int i = 0; i < 9; ++i)
                    {
                        P.T[i] = h.transform[i];
                        P.Ti[i] = h.inv_transform[i];
                    }
                    ppose[3] = ph.prim_y_angle;
                    ppose[4] = ph.prim_z_angle;
                }
                const bool isZ = zAxisCase(ppose, spose, h.inner_radius);
                if (zAxisCount && isZ)
                    atomicAdd(zAxisCount, 1ull);
                const bool skip = isZ && zOffsets && zOffsets[j] >= 0;
                S.skip = skip ? 1 : 0;
                hasZ = hasZ || skip;
                double offset = 0.0;
                const bool improved = QTY != 1 && !ph.full_ring ? improvedCase(ppose, spose, offset) : false;
                for (int i = 0; i < 3; ++i)
                {
                    S.pos[i] = P.pos[i];
                    S.sp[i] = spose[i];
                }
                for (int i = 0; i < 9; ++i)
                {
                    S.T[i] = P.T[i];
                    S.Ti[i] = P.Ti[i];
                }
                double sA, cA, sB, cB;
                sincos(spose[3], &sA, &cA);
                sincos(spose[4], &sB, &cB);
                S.sA = sA;
                S.cA = cA;
                S.sB = sB;
                S.cB = cB;
                S.offset = offset;
                S.ablk = (improved ? kPi : 2 * kPi) / ph.s_ablocks;
                if (QTY == 3)
                {
                    double dTy[9], dTz[9];
                    transformDerivatives(ppose[3], ppose[4], dTy, dTz);
                    for (int i = 0; i < 9; ++i)
                    {
                        S.dTy[i] = dTy[i];
                        S.dTz[i] = dTz[i];
                    }
                }
            }
            __syncwarp();
            if (S.skip)
                continue;  // warp-uniform: the z-axis pass adds this primary
            const int nsec = ph.s_nl * ph.s_nt * ph.s_na;
            for (int i = 0; i < W; ++i)
                part[128 * i] = 0.0;
            // every lane runs the same number of iterations (warp-uniform choices
            // below); a lane past the end evaluates the last node and drops it
            // One secondary node per lane.  mode 0: the FP64 kernel; mode 1: the FP32
            // pass, which defers near-field nodes to the warp's list; mode 2: a batch
            // of deferred nodes, in FP64, one per lane
            int nNear = 0;
            int *list = nearLists[threadIdx.x / 32];
            // REFINE: this warp's node contributions
            double *scr = REFINE ? nodeScratch + (size_t)warp * (size_t)scratchNodes * W : nullptr;
            auto node = [&](int n, bool valid, int mode) {
                const int k = n % ph.s_na, lt_i = n / ph.s_na;
                const int t = lt_i % ph.s_nt, l = lt_i / ph.s_nt;
                const double2 L = sl[l], R = st[t];
                const SecAngular A = sa[k];
                const double ablk = S.ablk;
                const double phi = (S.offset + ablk * A.bpos) + (ablk * 0.5) * A.x;
                double sP, cP;
                sincos(phi, &sP, &cP);
                const double sA = S.sA, cA = S.cA, sB = S.sB, cB = S.cB;
                const double ringP[3] = {cB * cA * cP - sB * sP, sB * cA * cP + cB * sP, -sA * cP};
                const double tan[3] = {-cB * cA * sP - sB * cP, -sB * cA * sP + cB * cP, sA * sP};
                const double q[3] = {S.sp[0] + L.x * sA * cB + R.x * ringP[0],
                                     S.sp[1] + L.x * sA * sB + R.x * ringP[1], S.sp[2] + L.x * cA + R.x * ringP[2]};
                const double w = 0.125 * R.x * L.y * R.y * A.w;
                const Frame f = toCoilFrameAt(S.pos, S.Ti, q[0], q[1], q[2]);
                const bool far = mode == 1;
                if (mode == 1)
                {
                    const bool near = valid && nearWinding(h, f);
                    const unsigned bal = __ballot_sync(0xffffffffu, near);
                    if (bal)
                    {
                        if (near)
                            list[nNear + __popc(bal & ((1u << lane) - 1u))] = n;
                        nNear += __popc(bal);
                        valid = valid && !near;
                    }
                    if (REFINE && near)
                        for (int i = 0; i < W; ++i)
                            scr[(size_t)n * W + i] = 0.0;
                }
                if (QTY == 0)
                {
                    double av;
                    if (!FP32)
                        av = CCOIL_PAIR_CALL_FP64 ? pairA64(h, tt, lt, pt, f.z, f.r) : segmentA64<1>(h, tt, lt, pt, f, 0);
                    else if (far)
                        av = pairA32(h, tt, lt, pn, f.z, f.r);
                    else
                        av = pairA64Fast(h, tt, lt, pt, f.z, f.r);
                    const double vx = -av * f.sphi, vy = av * f.cphi;
                    const double Ax = S.T[0] * vx + S.T[1] * vy, Ay = S.T[3] * vx + S.T[4] * vy,
                                 Az = S.T[6] * vx + S.T[7] * vy;
                    const double c = (Ax * tan[0] + Ay * tan[1] + Az * tan[2]) * w;
                    if (valid)
                    {
                        part[0] += c;
                        if (REFINE && far)
                            scr[n] = c;
                    }
                }
                else if (QTY == 3)
                {
                    // parameter gradient: per secondary node, the derivative of
                    // w (A(q) . t) with respect to every coil parameter
                    const double2 *tu = reinterpret_cast<const double2 *>(base) + ph.off_tu;
                    const double2 *lu = reinterpret_cast<const double2 *>(base) + ph.off_lu;
                    const double ul = (reinterpret_cast<const double2 *>(base) + ph.off_slu)[l].x;
                    const double ut = (reinterpret_cast<const double2 *>(base) + ph.off_stu)[t].x;
                    double av, d[5];
                    if (FP32 && far)
                    {
                        av = pairA32(h, tt, lt, pn, f.z, f.r);
                        segmentAParams32(h, tt, lt, pn, tu, lu, f, av, d);
                    }
                    else
                    {
                        av = pairA64(h, tt, lt, pt, f.z, f.r);
                        segmentAParams64(h, tt, lt, pt, tu, lu, f, av, d);
                    }
                    const double ar = d[0], az = d[1];
                    const double c = f.cphi, s_ = f.sphi;
                    const double ao = f.r > 0.0 ? av / f.r : ar;
                    const double J[9] = {s_ * c * (ao - ar), -s_ * s_ * ar - c * c * ao, -s_ * az,
                                         c * c * ar + s_ * s_ * ao, s_ * c * (ar - ao), c * az,
                                         0.0, 0.0, 0.0};
                    double e[3], u[3], v[3], gp[3];
                    for (int i = 0; i < 3; ++i)
                        e[i] = -S.T[3 * i] * s_ + S.T[3 * i + 1] * c;                      // T (-sin, cos, 0)
                    for (int i = 0; i < 3; ++i)
                        u[i] = S.T[i] * tan[0] + S.T[3 + i] * tan[1] + S.T[6 + i] * tan[2];  // T^T t
                    for (int i = 0; i < 3; ++i)
                        v[i] = J[i] * u[0] + J[3 + i] * u[1] + J[6 + i] * u[2];           // J^T u
                    for (int i = 0; i < 3; ++i)
                        gp[i] = S.T[3 * i] * v[0] + S.T[3 * i + 1] * v[1] + S.T[3 * i + 2] * v[2];
                    const double et = e[0] * tan[0] + e[1] * tan[1] + e[2] * tan[2];
                    double g[14];
                    g[0] = av * et;
                    g[1] = d[2] * et;
                    g[2] = d[3] * et;
                    g[3] = d[4] * et;
                    // primary orientation: (dT A_loc) . t + (J_loc dT^T (q - c)) . (T^T t)
                    const double aloc[2] = {-s_ * av, c * av};
                    const double dv[3] = {q[0] - S.pos[0], q[1] - S.pos[1], q[2] - S.pos[2]};
                    for (int k = 0; k < 2; ++k)
                    {
                        double dT[9];
                        for (int i = 0; i < 9; ++i)
                            dT[i] = k == 0 ? S.dTy[i] : S.dTz[i];
                        double y[3], gk = 0.0;
                        for (int j = 0; j < 3; ++j)
                            y[j] = dT[j] * dv[0] + dT[3 + j] * dv[1] + dT[6 + j] * dv[2];
                        for (int i = 0; i < 3; ++i)
                        {
                            gk += (dT[3 * i] * aloc[0] + dT[3 * i + 1] * aloc[1]) * tan[i];
                            gk += (J[3 * i] * y[0] + J[3 * i + 1] * y[1] + J[3 * i + 2] * y[2]) * u[i];
                        }
                        g[4 + k] = gk;
                    }
                    // secondary inner radius, thickness, length (node positions; the
                    // weight is proportional to the ring radius)
                    const double axis[3] = {sA * cB, sA * sB, cA};
                    g[6] = av * et / R.x + ringP[0] * gp[0] + ringP[1] * gp[1] + ringP[2] * gp[2];
                    g[7] = ut * g[6];
                    g[8] = ul * (axis[0] * gp[0] + axis[1] * gp[1] + axis[2] * gp[2]);
                    g[9] = gp[0];
                    g[10] = gp[1];
                    g[11] = gp[2];
                    // secondary orientation: node position and tangent move
                    const double A_[3] = {av * e[0], av * e[1], av * e[2]};
                    const double dE1A[3] = {-cB * sA, -sB * sA, -cA}, dAxA[3] = {cA * cB, cA * sB, -sA};
                    const double dE1B[3] = {-sB * cA, cB * cA, 0.0}, dE2B[3] = {-cB, -sB, 0.0},
                                 dAxB[3] = {-sA * sB, sA * cB, 0.0};
                    double gA = 0.0, gB = 0.0;
                    for (int i = 0; i < 3; ++i)
                    {
                        const double dqA = L.x * dAxA[i] + R.x * cP * dE1A[i], dtA = -sP * dE1A[i];
                        const double dqB = L.x * dAxB[i] + R.x * (cP * dE1B[i] + sP * dE2B[i]),
                                     dtB = -sP * dE1B[i] + cP * dE2B[i];
                        gA += dqA * gp[i] + A_[i] * dtA;
                        gB += dqB * gp[i] + A_[i] * dtB;
                    }
                    g[12] = gA;
                    g[13] = gB;
                    if (valid)
                        for (int i = 0; i < 14; ++i)
                            part[128 * i] += g[i] * w;
                }
                else if (QTY == 2)
                {
                    // dM/d(secondary position) = factor sum_n w_n J_A(q_n)^T t_n,
                    // J_A = T J_loc T^T; J_loc of A_loc = a(r, z) (-sin, cos, 0)
                    double av, ar, az;
                    segmentAGrad64(h, tt, lt, pt, f, av, ar, az);
                    const double c = f.cphi, s_ = f.sphi;
                    const double ao = f.r > 0.0 ? av / f.r : ar;
                    const double J[9] = {s_ * c * (ao - ar), -s_ * s_ * ar - c * c * ao, -s_ * az,
                                         c * c * ar + s_ * s_ * ao, s_ * c * (ar - ao), c * az,
                                         0.0, 0.0, 0.0};
                    // T J^T T^T t
                    double u[3], v[3], o[3];
                    for (int i = 0; i < 3; ++i)
                        u[i] = S.T[i] * tan[0] + S.T[3 + i] * tan[1] + S.T[6 + i] * tan[2];  // T^T t
                    for (int i = 0; i < 3; ++i)
                        v[i] = J[i] * u[0] + J[3 + i] * u[1] + J[6 + i] * u[2];           // J^T u
                    for (int i = 0; i < 3; ++i)
                        o[i] = S.T[3 * i] * v[0] + S.T[3 * i + 1] * v[1] + S.T[3 * i + 2] * v[2];
                    if (valid)
                        for (int i = 0; i < 3; ++i)
                            part[128 * i] += o[i] * w;
                }
                else
                {
                    double H, Z;
                    if (!FP32 && !CCOIL_PAIR_CALL_FP64)
                        segmentB64<1>(h, tt, lt, pt, f, 0, H, Z);
                    else
                    {
                        const double2 hz = !FP32 ? pairB64(h, tt, lt, pt, f.z, f.r)
                                                 : far ? pairB32(h, tt, lt, pn, f.z, f.r)
                                                       : pairB64Fast(h, tt, lt, pt, f.z, f.r);
                        H = hz.x;
                        Z = hz.y;
                    }
                    const double vx = H * f.cphi, vy = H * f.sphi;
                    const double B[3] = {S.T[0] * vx + S.T[1] * vy + S.T[2] * Z, S.T[3] * vx + S.T[4] * vy + S.T[5] * Z,
                                         S.T[6] * vx + S.T[7] * vy + S.T[8] * Z};
                    double dF[3], dT[3];
                    cross3(tan, B, dF);
                    for (int i = 0; i < 3; ++i)
                        dF[i] *= w;
                    const double rel[3] = {q[0] - S.sp[0], q[1] - S.sp[1], q[2] - S.sp[2]};
                    cross3(rel, dF, dT);
                    if (valid)
                        for (int i = 0; i < 3; ++i)
                        {
                            part[128 * i] += dF[i];
                            part[128 * (3 + i)] += dT[i];
                            if (REFINE && far)
                            {
                                scr[(size_t)n * W + i] = dF[i];
                                scr[(size_t)n * W + 3 + i] = dT[i];
                            }
                        }
                }
            };
            // 32 listed nodes (or the last few) in FP64
            auto fp64Batch = [&]() {
                __syncwarp();
                const bool v = lane < nNear;
                node(list[v ? lane : 0], v, 2);
                const int rest = nNear > 32 ? nNear - 32 : 0;
                const int moved = lane < rest ? list[32 + lane] : 0;
                __syncwarp();
                if (lane < rest)
                    list[lane] = moved;
                __syncwarp();
                nNear = rest;
            };
            // REFINE at fraction 0 refines every node: each node in the FP64 forms
            // directly, without the FP32 pass
            const bool allFp64 = REFINE && !(fraction > 0.0);
            if (!FP32)
                for (int n0 = 0; n0 < nsec; n0 += 32)
                    node(n0 + lane < nsec ? n0 + lane : nsec - 1, n0 + lane < nsec, 0);
            else if (allFp64)
                for (int n0 = 0; n0 < nsec; n0 += 32)
                    node(n0 + lane < nsec ? n0 + lane : nsec - 1, n0 + lane < nsec, 2);
            else
                for (int n0 = 0; n0 < nsec || nNear > 0;)
                {
                    if (nNear >= 32 || n0 >= nsec)
                        fp64Batch();  // deferred near-field nodes
                    else
                    {
                        node(n0 + lane < nsec ? n0 + lane : nsec - 1, n0 + lane < nsec, 1);
                        n0 += 32;
                    }
                }
            if (REFINE && !allFp64)
            {
                // the primary's totals (every lane), then the dominating nodes in FP64;
                // node n was evaluated, and its contribution stored, by lane n % 32
                double lim[2] = {0.0, 0.0};
                for (int g = 0; g < (QTY == 0 ? 1 : 2); ++g)
                {
                    double n2 = 0.0;
                    for (int i = 0; i < (QTY == 0 ? 1 : 3); ++i)
                    {
                        double v = part[128 * (3 * g + i)];
#pragma unroll
                        for (int off = 16; off > 0; off /= 2)
                            v += __shfl_xor_sync(0xffffffffu, v, off);
                        n2 += v * v;
                    }
                    lim[g] = fraction * fraction * n2;  // not finite: nothing is picked
                }
                for (int b0 = 0; b0 < nsec; b0 += 32)
                {
                    const int n = b0 + lane;
                    bool pick = false;
                    if (n < nsec)
                    {
                        double c[W];
                        for (int i = 0; i < W; ++i)
                            c[i] = scr[(size_t)n * W + i];
                        if (QTY == 0)
                            pick = c[0] * c[0] > lim[0];
                        else
                            pick = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] > lim[0] ||
                                   c[3] * c[3] + c[4] * c[4] + c[5] * c[5] > lim[1];
                        if (pick)
                            for (int i = 0; i < W; ++i)
                                part[128 * i] -= c[i];
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, pick);
                    if (pick)
                        list[nNear + __popc(bal & ((1u << lane) - 1u))] = n;
                    nNear += __popc(bal);
                    if (nNear >= 32)
                        fp64Batch();
                }
                while (nNear > 0)
                    fp64Batch();
            }
            const double scale = QTY == 1 ? ph.f_factor : ph.m_factor;
#pragma unroll
            for (int i = 0; i < W; ++i)
            {
                double v = part[128 * i];
#pragma unroll
                for (int off = 16; off > 0; off /= 2)
                    v += __shfl_xor_sync(0xffffffffu, v, off);
                if (lane == 0)
                    total[i] += v * scale;
            }
        }
        if (lane == 0)
        {
#pragma unroll
            for (int i = 0; i < W; ++i)
                out[W * a + i] = total[i];
            if (hasZ)
                zList[atomicAdd(zListCount, 1ull)] = a;
        }
    }
}

void put(std::vector<unsigned char> &blob, const void *p, size_t n)
{
    const unsigned char *c = static_cast<const unsigned char *>(p);
    blob.insert(blob.end(), c, c + n);
}

// The primary's field tables: thickness nodes {r', constant w} with the
// integrator's constant folded in, length nodes {z, w} (slow method) and
// angular nodes {cos, w}, as the reference's field integrators lay them out
// (CalculateFieldsFast.cxx:17-55, CalculateFieldsSlow.cxx:17-66).
void primaryTables(const Coil &prim, const PrecisionArgs &pp, std::vector<double> &pt_, std::vector<double> &pl_,
                   std::vector<double> &pa_)
{
    const bool fast = prim.use_fast_method != 0;
    const double tBlock = prim.thickness / pp.thickness_blocks, aBlock = kPi / pp.angular_blocks;
    const double constant = fast ? kMuReduced * prim.current_density * tBlock * aBlock * 2 * 0.25
                                 : kMuReduced * prim.current_density * (prim.length / pp.length_blocks) * tBlock *
                                       aBlock * 2 * 0.125;
    const double *tx = legendreNodes(pp.thickness_increments), *tw = legendreWeights(pp.thickness_increments);
    for (int b = 0; b < pp.thickness_blocks; ++b)
        for (int i = 0; i < pp.thickness_increments; ++i)
        {
            pt_.push_back(prim.inner_radius + tBlock * (b + 0.5) + (tBlock * 0.5) * tx[i]);
            pt_.push_back(constant * tw[i]);
        }
    if (!fast)
    {
        const double lBlock = prim.length / pp.length_blocks;
        const double *lx = legendreNodes(pp.length_increments), *lw = legendreWeights(pp.length_increments);
        for (int b = 0; b < pp.length_blocks; ++b)
            for (int i = 0; i < pp.length_increments; ++i)
            {
                pl_.push_back(-prim.length * 0.5 + lBlock * (b + 0.5) + (lBlock * 0.5) * lx[i]);
                pl_.push_back(lw[i]);
            }
    }
    const double *ax = legendreNodes(pp.angular_increments), *aw = legendreWeights(pp.angular_increments);
    for (int b = 0; b < pp.angular_blocks; ++b)
        for (int i = 0; i < pp.angular_increments; ++i)
        {
            pa_.push_back(std::cos(aBlock * (b + 0.5) + (aBlock * 0.5) * ax[i]));
            pa_.push_back(aw[i]);
        }
}

// Primary tables as the reference's field integrators lay them out
// (CalculateFieldsFast.cxx:17-55, CalculateFieldsSlow.cxx:17-66), secondary
// cloud as CalculateMInductanceGeneral.cxx:41-103 builds it.
bool buildPair(const Coil &prim, const Coil &sec, const PrecisionArgs &pp, const PrecisionArgs &spa, bool fp32,
               bool units, const PairOptions &opt, std::vector<unsigned char> &blob, std::string &err)
{
    if (!validArgs(pp) || !validArgs(spa))
    {
        err = "pair precision arguments out of range (increments 1..100, blocks >= 1)";
        return false;
    }
    if (!(prim.inner_radius > 0.0) || !(prim.thickness > 0.0) || !(prim.length > 0.0) || !(sec.inner_radius > 0.0) ||
        !(sec.thickness > 0.0) || !(sec.length > 0.0) || prim.current == 0.0)
    {
        err = "coil dimensions must be positive and the primary current non-zero";
        return false;
    }
    const size_t start = blob.size();
    const bool fast = prim.use_fast_method != 0;
    std::vector<double> pt_, pl_, pa_;
    primaryTables(prim, pp, pt_, pl_, pa_);
    // secondary cloud tables
    std::vector<double> sl_, st_;
    std::vector<SecAngular> sa_;
    const double lbs = sec.length / spa.length_blocks, tbs = sec.thickness / spa.thickness_blocks;
    const double *slx = legendreNodes(spa.length_increments), *slw = legendreWeights(spa.length_increments);
    for (int b = 0; b < spa.length_blocks; ++b)
        for (int i = 0; i < spa.length_increments; ++i)
        {
            sl_.push_back(-sec.length * 0.5 + lbs * (b + 0.5) + (lbs * 0.5) * slx[i]);
            sl_.push_back(slw[i]);
        }
    const double *stx = legendreNodes(spa.thickness_increments), *stw = legendreWeights(spa.thickness_increments);
    for (int b = 0; b < spa.thickness_blocks; ++b)
        for (int i = 0; i < spa.thickness_increments; ++i)
        {
            st_.push_back(sec.inner_radius + tbs * (b + 0.5) + (tbs * 0.5) * stx[i]);
            st_.push_back(stw[i]);
        }
    const double *sax = legendreNodes(spa.angular_increments), *saw = legendreWeights(spa.angular_increments);
    for (int b = 0; b < spa.angular_blocks; ++b)
        for (int i = 0; i < spa.angular_increments; ++i)
            sa_.push_back({b + 0.5, sax[i], saw[i], 0.0});

    PairHeader ph;
    std::memset(&ph, 0, sizeof(ph));
    SegmentHeader &h = ph.prim;
    for (int i = 0; i < 3; ++i)
        h.position[i] = prim.position[i];
    std::memcpy(h.transform, prim.transform, sizeof(h.transform));
    std::memcpy(h.inv_transform, prim.inverse_transform, sizeof(h.inv_transform));
    h.half_length = prim.length * 0.5;
    h.field_factor = 1.0;
    h.inner_radius = prim.inner_radius;
    h.n_t = (int)pt_.size() / 2;
    h.n_l = (int)pl_.size() / 2;
    h.n_phi = (int)pa_.size() / 2;
    h.fast = fast ? 1 : 0;
    const int hdr16 = (int)sizeof(PairHeader) / 16;
    h.off_t = hdr16;
    h.off_l = h.off_t + h.n_t;
    h.off_phi = h.off_l + h.n_l;
    ph.s_nl = (int)sl_.size() / 2;
    ph.s_nt = (int)st_.size() / 2;
    ph.s_na = (int)sa_.size();
    ph.s_ablocks = spa.angular_blocks;
    ph.off_sl = h.off_phi + h.n_phi;
    ph.off_st = ph.off_sl + ph.s_nl;
    ph.off_sa = ph.off_st + ph.s_nt;
    std::vector<PhiPair2> p32;
    if (fp32)
    {
        // FP32 angular mirror-pair table (entries of two pairs) after the secondary tables
        std::vector<PhiNode32> single;
        buildPhiPairs32(pp, single);
        packPhiPairs2(single.data(), (int)single.size(), p32);
        h.off_f32 = ph.off_sa + 2 * ph.s_na;
        setNearBox(prim, h);
    }
    // parameter-gradient tables: each node's position per unit of its layer's
    // dimension, {u, 0} (thickness on [0, 1], length on [-1/2, 1/2])
    std::vector<double> tu_, lu_, slu_, stu_;
    if (units)
    {
        auto thicknessUnits = [](const PrecisionArgs &a, std::vector<double> &o) {
            const double *x = legendreNodes(a.thickness_increments);
            for (int b = 0; b < a.thickness_blocks; ++b)
                for (int i = 0; i < a.thickness_increments; ++i)
                    o.insert(o.end(), {((b + 0.5) + 0.5 * x[i]) / a.thickness_blocks, 0.0});
        };
        auto lengthUnits = [](const PrecisionArgs &a, std::vector<double> &o) {
            const double *x = legendreNodes(a.length_increments);
            for (int b = 0; b < a.length_blocks; ++b)
                for (int i = 0; i < a.length_increments; ++i)
                    o.insert(o.end(), {-0.5 + ((b + 0.5) + 0.5 * x[i]) / a.length_blocks, 0.0});
        };
        thicknessUnits(pp, tu_);
        if (!fast)
            lengthUnits(pp, lu_);
        lengthUnits(spa, slu_);
        thicknessUnits(spa, stu_);
        const int base16 = ph.off_sa + 2 * ph.s_na + (int)(sizeof(PhiPair2) / 16 * p32.size());
        ph.off_tu = base16;
        ph.off_lu = ph.off_tu + (int)tu_.size() / 2;
        ph.off_slu = ph.off_lu + (int)lu_.size() / 2;
        ph.off_stu = ph.off_slu + (int)slu_.size() / 2;
    }
    const double blocks = double(spa.length_blocks) * spa.thickness_blocks * spa.angular_blocks;
    ph.m_factor = 2 * kPi * sec.num_turns / prim.current / blocks * opt.scale;
    ph.f_factor = 2 * kPi * (sec.current * sec.num_turns) / blocks * opt.scale;
    ph.full_ring = opt.full_ring ? 1 : 0;
    ph.prim_y_angle = prim.y_axis_angle;
    ph.prim_z_angle = prim.z_axis_angle;
    put(blob, &ph, sizeof(ph));
    put(blob, pt_.data(), sizeof(double) * pt_.size());
    put(blob, pl_.data(), sizeof(double) * pl_.size());
    put(blob, pa_.data(), sizeof(double) * pa_.size());
    put(blob, sl_.data(), sizeof(double) * sl_.size());
    put(blob, st_.data(), sizeof(double) * st_.size());
    put(blob, sa_.data(), sizeof(SecAngular) * sa_.size());
    put(blob, p32.data(), sizeof(PhiPair2) * p32.size());
    put(blob, tu_.data(), sizeof(double) * tu_.size());
    put(blob, lu_.data(), sizeof(double) * lu_.size());
    put(blob, slu_.data(), sizeof(double) * slu_.size());
    put(blob, stu_.data(), sizeof(double) * stu_.size());
    (void)start;
    return true;
}

#include "zaxis.cuh"

// Stream-ordered temporary from the library's memory pool: no device-wide
// synchronisation and no driver mapping work per call
struct DevBuf
{
    void *p = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t alloc(size_t bytes, cudaStream_t s)
    {
        st = s;
        return scratchAlloc(&p, bytes, s);
    }
    ~DevBuf()
    {
        if (p)
            cudaFreeAsync(p, st);
    }
};
} // namespace

int cudaFail(cudaError_t e, const char *what);
} // namespace ccoil

using namespace ccoil;

int ccoil::pairArrangements(const ccoil_coil_t *primaries, int primary_count, const ccoil_coil_t *secondary,
                            const ccoil_precision_args_t *secondary_precisions,
                            const ccoil_precision_args_t *zaxis_precisions, const ccoil_pose_t *primary_poses,
                            const ccoil_pose_t *secondary_poses, long long count, int quantity, int precision,
                            double *out, long long *z_axis_count, int memory, void *stream, const PairOptions &opt)
{
    if (primary_count < 0 || (primary_count > 0 && (!primaries || !secondary_precisions)) || !secondary)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "null coils or negative primary_count");
    if (count < 0 || (count > 0 && (!secondary_poses || !out)))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "count < 0 or null poses/out");
    if (primary_poses && primary_count != 1)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "per-arrangement primary poses need exactly one primary");
    if (quantity != CCOIL_PAIR_MUTUAL_INDUCTANCE && quantity != CCOIL_PAIR_FORCE_TORQUE &&
        quantity != CCOIL_PAIR_MUTUAL_INDUCTANCE_GRADIENT && quantity != CCOIL_PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "unknown pair quantity");
    if (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT && count > 0 && (primary_count != 1 || !primary_poses))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT,
                           "the parameter gradient needs exactly one primary with per-arrangement poses");
    if (precision != CCOIL_PRECISION_FP64 && precision != CCOIL_PRECISION_FP32_COMPENSATED &&
        precision != CCOIL_PRECISION_FP32_REFINED)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "unknown precision mode");
    if (precision == CCOIL_PRECISION_FP32_COMPENSATED && quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE_GRADIENT)
        return failMessage(CCOIL_ERR_NOT_SUPPORTED,
                           "the position gradient is evaluated in FP64 only (the parameter gradient has an FP32 form)");
    if (precision == CCOIL_PRECISION_FP32_REFINED && quantity != CCOIL_PAIR_MUTUAL_INDUCTANCE &&
        quantity != CCOIL_PAIR_FORCE_TORQUE)
        return failMessage(CCOIL_ERR_NOT_SUPPORTED, "FP32_REFINED covers mutual inductance and force/torque");
    const bool fp32 = precision != CCOIL_PRECISION_FP64;
    const bool refine = precision == CCOIL_PRECISION_FP32_REFINED;
    if (memory != CCOIL_MEMORY_HOST && memory != CCOIL_MEMORY_DEVICE)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "memory must be HOST or DEVICE");
    if (z_axis_count)
        *z_axis_count = 0;
    const int width = quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE            ? 1
                      : quantity == CCOIL_PAIR_FORCE_TORQUE               ? 6
                      : quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE_GRADIENT ? 3
                                                                          : 14;
    if (count == 0)
        return CCOIL_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (primary_count == 0)
    {
        cudaError_t e = memory == CCOIL_MEMORY_HOST ? cudaSuccess : cudaMemsetAsync(out, 0, sizeof(double) * width * count, st);
        if (memory == CCOIL_MEMORY_HOST)
            std::memset(out, 0, sizeof(double) * width * count);
        return e == cudaSuccess ? CCOIL_OK : cudaFail(e, "memset");
    }

    std::vector<unsigned char> blob;
    std::vector<long long> offsets;
    std::string err;
    for (int j = 0; j < primary_count; ++j)
    {
        offsets.push_back((long long)blob.size());
        if (!buildPair(primaries[j], *secondary, primaries[j].precision, secondary_precisions[j], fp32,
                       quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT, opt, blob, err))
            return fail(CCOIL_ERR_INVALID_ARGUMENT, "primary " + std::to_string(j) + ": " + err);
    }
    const size_t generalBytes = blob.size();
    // coaxial pairs: the z-axis tables of every primary (M and F/T only)
    const bool zPass = zaxis_precisions && (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE ||
                                            quantity == CCOIL_PAIR_FORCE_TORQUE);
    std::vector<long long> zOffsets(primary_count, -1);
    if (zPass)
        for (int j = 0; j < primary_count; ++j)
        {
            zOffsets[j] = (long long)blob.size();
            if (!buildZAxis(primaries[j], *secondary, zaxis_precisions[2 * j], zaxis_precisions[2 * j + 1], blob, err))
                return fail(CCOIL_ERR_INVALID_ARGUMENT, "primary " + std::to_string(j) + ": " + err);
        }
    DevBuf dBlob, dOff, dPrim, dSec, dOut, dZ, dZOff, dZList, dZCount, dScratch;
    cudaError_t e = dBlob.alloc(blob.size(), st);
    if (e == cudaSuccess)
        e = dOff.alloc(sizeof(long long) * offsets.size(), st);
    if (e == cudaSuccess)
        e = dZ.alloc(sizeof(unsigned long long), st);
    if (e == cudaSuccess && zPass)
    {
        e = dZOff.alloc(sizeof(long long) * primary_count, st);
        if (e == cudaSuccess)
            e = dZList.alloc(sizeof(long long) * count, st);
        if (e == cudaSuccess)
            e = dZCount.alloc(sizeof(unsigned long long), st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dZOff.p, zOffsets.data(), sizeof(long long) * primary_count, cudaMemcpyHostToDevice,
                                st);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(dZCount.p, 0, sizeof(unsigned long long), st);
    }
    if (e == cudaSuccess && memory == CCOIL_MEMORY_HOST)
    {
        e = dSec.alloc(sizeof(double) * 5 * count, st);
        if (e == cudaSuccess && primary_poses)
            e = dPrim.alloc(sizeof(double) * 5 * count, st);
        if (e == cudaSuccess)
            e = dOut.alloc(sizeof(double) * width * count, st);
    }
    if (e != cudaSuccess)
        return cudaFail(e, "scratch allocation");
    e = cudaMemcpyAsync(dBlob.p, blob.data(), blob.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dOff.p, offsets.data(), sizeof(long long) * offsets.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(dZ.p, 0, sizeof(unsigned long long), st);
    const double *secP = reinterpret_cast<const double *>(secondary_poses);
    const double *primP = reinterpret_cast<const double *>(primary_poses);
    double *o = out;
    if (e == cudaSuccess && memory == CCOIL_MEMORY_HOST)
    {
        e = cudaMemcpyAsync(dSec.p, secondary_poses, sizeof(double) * 5 * count, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && primary_poses)
            e = cudaMemcpyAsync(dPrim.p, primary_poses, sizeof(double) * 5 * count, cudaMemcpyHostToDevice, st);
        secP = static_cast<const double *>(dSec.p);
        primP = primary_poses ? static_cast<const double *>(dPrim.p) : nullptr;
        o = static_cast<double *>(dOut.p);
    }
    if (e != cudaSuccess)
        return cudaFail(e, "host->device copy");
    // one primary whose tables fit: stage them in shared memory
    const int stagedBytes = (primary_count == 1 && generalBytes <= CCOIL_PAIR_STAGE_MAX_BYTES &&
                             generalBytes % 16 == 0)
                                ? (int)generalBytes
                                : 0;
    const long long warpsNeeded = count;
    long long blocks = (warpsNeeded + 3) / 4;
    if (blocks > 148LL * 64)
        blocks = 148LL * 64;
    // FP32_REFINED: every warp's region of node contributions (the grid strides over
    // the arrangements, so the scratch is sized by the grid, not by the count)
    int scratchNodes = 0;
    if (refine)
    {
        for (long long off : offsets)
        {
            const PairHeader *ph = reinterpret_cast<const PairHeader *>(blob.data() + off);
            scratchNodes = std::max(scratchNodes, ph->s_nl * ph->s_nt * ph->s_na);
        }
        // at most kPairRefineScratchBytes: a secondary with many nodes runs on fewer
        // warps (each keeps 1 or 6 doubles per node), never fewer than one CTA per SM
        const size_t perBlock = sizeof(double) * (size_t)width * (size_t)scratchNodes * 4;
        const long long fit = (long long)(kPairRefineScratchBytes / perBlock);
        blocks = std::max(1LL, std::min(blocks, std::max(fit, 148LL)));
        e = dScratch.alloc(perBlock * (size_t)blocks, st);
        if (e != cudaSuccess)
            return cudaFail(e, "refinement scratch");
    }
    const double fraction = refineFraction();
    auto *scratch = static_cast<double *>(dScratch.p);
    auto *zc = static_cast<unsigned long long *>(dZ.p);
    const auto *dB = static_cast<const unsigned char *>(dBlob.p);
    const auto *dO = static_cast<const long long *>(dOff.p);
    const size_t smem = (size_t)stagedBytes;
    const auto *zO = static_cast<const long long *>(dZOff.p);
    auto *zL = static_cast<long long *>(dZList.p);
    auto *zN = static_cast<unsigned long long *>(dZCount.p);
#define CCOIL_PAIR_LAUNCH(Q, F, ...)                                                                                   \
    pairKernel64<Q, F, ##__VA_ARGS__><<<(unsigned)blocks, 128, smem, st>>>(                                          \
        dB, dO, primary_count, primP, secP, count, o, zc, stagedBytes, zO, zL, zN, scratch, scratchNodes, fraction)
    if (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE && !fp32)
        CCOIL_PAIR_LAUNCH(0, false);
    else if (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE && refine)
        CCOIL_PAIR_LAUNCH(0, true, true);
    else if (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE)
        CCOIL_PAIR_LAUNCH(0, true);
    else if (quantity == CCOIL_PAIR_FORCE_TORQUE && !fp32)
        CCOIL_PAIR_LAUNCH(1, false);
    else if (quantity == CCOIL_PAIR_FORCE_TORQUE && refine)
        CCOIL_PAIR_LAUNCH(1, true, true);
    else if (quantity == CCOIL_PAIR_FORCE_TORQUE)
        CCOIL_PAIR_LAUNCH(1, true);
    else if (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE_GRADIENT)
        CCOIL_PAIR_LAUNCH(2, false);
    else if (!fp32)
        CCOIL_PAIR_LAUNCH(3, false);
    else
        CCOIL_PAIR_LAUNCH(3, true);
#undef CCOIL_PAIR_LAUNCH
    if (zPass && cudaGetLastError() == cudaSuccess)
    {
        // the z-axis pass: one warp per recorded arrangement
        if (quantity == CCOIL_PAIR_MUTUAL_INDUCTANCE)
            zAxisKernel<0><<<148 * 8, 128, 0, st>>>(dB, dO, zO, primary_count, primP, secP, zL, zN, o);
        else
            zAxisKernel<1><<<148 * 8, 128, 0, st>>>(dB, dO, zO, primary_count, primP, secP, zL, zN, o);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return cudaFail(e, "pair kernel launch");
    if (memory == CCOIL_MEMORY_HOST)
        e = cudaMemcpyAsync(out, o, sizeof(double) * width * count, cudaMemcpyDeviceToHost, st);
    unsigned long long zcount = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&zcount, zc, sizeof(zcount), cudaMemcpyDeviceToHost, st);
    // the call is synchronous, as the reference's: host outputs and the z-axis count
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, "pair arrangements");
    if (z_axis_count)
        *z_axis_count = (long long)zcount;
    return CCOIL_OK;
}

extern "C" int ccoil_pair_arrangements_zaxis(const ccoil_coil_t *primaries, int primary_count,
                                             const ccoil_coil_t *secondary,
                                             const ccoil_precision_args_t *secondary_precisions,
                                             const ccoil_precision_args_t *zaxis_precisions,
                                             const ccoil_pose_t *primary_poses, const ccoil_pose_t *secondary_poses,
                                             long long count, int quantity, int precision, double *out,
                                             long long *z_axis_count, int memory, void *stream)
{
    return pairArrangements(primaries, primary_count, secondary, secondary_precisions, zaxis_precisions,
                            primary_poses, secondary_poses, count, quantity, precision, out, z_axis_count, memory,
                            stream, PairOptions{});
}

extern "C" int ccoil_pair_arrangements(const ccoil_coil_t *primaries, int primary_count, const ccoil_coil_t *secondary,
                                       const ccoil_precision_args_t *secondary_precisions,
                                       const ccoil_pose_t *primary_poses, const ccoil_pose_t *secondary_poses,
                                       long long count, int quantity, int precision, double *out,
                                       long long *z_axis_count, int memory, void *stream)
{
    return ccoil_pair_arrangements_zaxis(primaries, primary_count, secondary, secondary_precisions, nullptr,
                                         primary_poses, secondary_poses, count, quantity, precision, out,
                                         z_axis_count, memory, stream);
}
