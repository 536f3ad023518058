// Adjoint of the coil-group B field with respect to every coil's parameters
// {R, a, b, N*I, x, y, z, yAxisAngle, zAxisAngle}, for every coil type: the fast
// method (RECTANGULAR and THIN, analytic length integral,
// src/Coil/Fields/CalculateFieldsFast.cxx:85-160) and the slow method (FLAT and
// FILAMENT, length nodes, src/Coil/Fields/CalculateFieldsSlow.cxx:86-165).
//
// Given points p and the upstream gradient v(p) = dL/dB(p), it accumulates
// dL/dtheta_c = sum_p v(p) . dB_c(p)/dtheta_c.  Nothing from the forward pass
// is stored: every node is recomputed here (the quadrature is cheap to redo and
// would cost n x nodes x 12 words to keep).
//
// Fast method, per node (weight w, node radius r', azimuth cos c; point at
// radius r, height z; top/bot = z +- b/2; rho^2 = r'^2 + r^2 - 2 r' r c;
// g1,2 = (rho^2 + top^2, bot^2)^-1/2):
//   H node  r' c (g2 - g1)                     (radial field, the reference's H term)
//   Z node  (r'^2 - r' r c) / rho^2 (top g1 - bot g2)
//   d/dr'   H: c (g2 - g1) + r' c (r' - r c)(g1^3 - g2^3)
//           Z: [(2r' - r c) E + N dE/dr'] / rho^2 - 2 N E (r' - r c) / rho^4,
//              E = top g1 - bot g2, N = r'^2 - r' r c, dE/dr' = -(r' - r c)(top g1^3 - bot g2^3)
//   d/dtop  H: r' c top g1^3       Z: N g1^3
//   d/dbot  H: -r' c bot g2^3      Z: -N g2^3
//   local Jacobian (RPhi, RR, RZ, ZZ) = (H/r, dH/dr, dH/dz, dZ/dz) in the stable
//   forms r' c (g2 - g1) / r, r' c (r - r' c)(g1^3 - g2^3), r' c (top g1^3 - bot g2^3),
//   (r'^2 - r' r c)(g1^3 - g2^3).
// With r' = R + a u (u the node's fraction of the thickness), B = K sum w h and
// K = 1e-7 (N I / (a b)) (a / tB) (pi / aB) / 2 (the reference's constant):
//   dB/dR = K sum w dh/dr',  dB/da = K sum w u dh/dr',
//   dB/db = -B/b + K sum w (dh/dtop - dh/dbot) / 2,  dB/d(NI) = B / (NI).
// Slow method, per node at height zl = z + l (l = b v the length node, v in
// [-1/2, 1/2]; G = (r'^2 + r^2 + zl^2 - 2 r' r c)^-1/2):
//   H node  r' c zl G^3,  Z node N G^3,
//   d/dr'   H: c zl G^3 - 3 r' c zl (r' - r c) G^5,  Z: (2 r' - r c) G^3 - 3 N (r' - r c) G^5
//   d/dzl   H: r' c G^3 - 3 r' c zl^2 G^5 (= the RZ node),  Z: -3 N zl G^5 (= the ZZ node)
//   RR node -3 r' c zl (r - r' c) G^5
// and K = 1e-7 N I (pi / aB) / (4 lB tB) does not depend on a or b:
//   dB/da = K sum w u dh/dr',  dB/db = K sum w v dh/dzl.
// Thin dimensions are 1e-25 R as in the reference (src/Coil/Coil.cxx:27-28); the
// derivative with respect to such a dimension is the one at that value.
// Globally B = T Bloc(T^T (p - pos)): dB/dpos = -T Gloc T^T,
// dB/dangle = T' Bloc + T Gloc T'^T (p - pos).
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <algorithm>

#include <cmath>
#include <cstring>
#include <vector>

namespace ccoil
{
int cudaFail(cudaError_t e, const char *what);

namespace
{
constexpr double kPi = 3.14159265358979323846;
constexpr int kAdjLanes = 4;
constexpr int kAdjThreads = 128;
constexpr int kAdjPoints = kAdjThreads / kAdjLanes;

struct alignas(16) AdjCoil
{
    double R, a, b, K1, half_b, NI;  // K1 = K / (N I): the constant per unit N I
    double pos[3];
    double T[9], Ta[9], Tb[9];  // transform and its derivatives by yAxisAngle, zAxisAngle
    int nt, nphi, off_t, off_phi;  // tables in 16-byte units from the record start
    int nl, off_l, fast, pad2;     // slow method: length nodes
};

// thickness node {r', w, u}; length node {l, w, v}
struct alignas(16) AdjT
{
    double rp, w, u, pad;
};

__device__ __forceinline__ void matvec(const double *M, const double *v, double *o)
{
    o[0] = M[0] * v[0] + M[1] * v[1] + M[2] * v[2];
    o[1] = M[3] * v[0] + M[4] * v[1] + M[5] * v[2];
    o[2] = M[6] * v[0] + M[7] * v[1] + M[8] * v[2];
}

__device__ __forceinline__ void matTvec(const double *M, const double *v, double *o)
{
    o[0] = M[0] * v[0] + M[3] * v[1] + M[6] * v[2];
    o[1] = M[1] * v[0] + M[4] * v[1] + M[7] * v[2];
    o[2] = M[2] * v[0] + M[5] * v[1] + M[8] * v[2];
}

__global__ void __launch_bounds__(kAdjThreads) adjointKernel(const unsigned char *__restrict__ blob,
                                                             const long long *__restrict__ offsets, int ncoils,
                                                             const double *__restrict__ points,
                                                             const double *__restrict__ gradB, long long npts,
                                                             double *__restrict__ partial)
{
    __shared__ double red[kAdjThreads / 32][9];
    const int lane = threadIdx.x % kAdjLanes;
    const long long p = (long long)blockIdx.x * kAdjPoints + threadIdx.x / kAdjLanes;
    const bool active = p < npts;
    double P[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    if (active)
        for (int i = 0; i < 3; ++i)
        {
            P[i] = points[3 * p + i];
            v[i] = gradB[3 * p + i];
        }
    // blockIdx.x: a tile of kAdjPoints points; blockIdx.y (grid-strided): the coil
    for (int c = blockIdx.y; c < ncoils; c += gridDim.y)
    {
        const unsigned char *base = blob + offsets[c];
        const AdjCoil &C = *reinterpret_cast<const AdjCoil *>(base);
        const AdjT *tt = reinterpret_cast<const AdjT *>(reinterpret_cast<const double2 *>(base) + C.off_t);
        const double2 *pt = reinterpret_cast<const double2 *>(base) + C.off_phi;
        double d[3] = {P[0] - C.pos[0], P[1] - C.pos[1], P[2] - C.pos[2]};
        double xl[3];
        matTvec(C.T, d, xl);
        const double r = sqrt(xl[0] * xl[0] + xl[1] * xl[1]), z = xl[2];
        const double cph = r > 0.0 ? xl[0] / r : 1.0, sph = r > 0.0 ? xl[1] / r : 0.0;
        const double top = z + C.half_b, bot = z - C.half_b;
        // H, Z, dH/dR, dZ/dR, dH/da, dZ/da, dH/db', dZ/db', RPhi*r, RR, RZ, ZZ
        double s[12];
        for (int i = 0; i < 12; ++i)
            s[i] = 0.0;
        if (C.fast)
            for (int j = 0; j < C.nt; ++j)
            {
                const AdjT t = tt[j];
                const double rp = t.rp;
                double a[10];
                for (int i = 0; i < 10; ++i)
                    a[i] = 0.0;
                for (int k = lane; k < C.nphi; k += kAdjLanes)
                {
                    const double2 q = pt[k];
                    const double cc = q.x, w = q.y;
                    const double rho2 = rp * rp + r * r - 2.0 * rp * r * cc;
                    const double g1 = rsqrt(rho2 + top * top), g2 = rsqrt(rho2 + bot * bot);
                    const double g13 = g1 * g1 * g1, g23 = g2 * g2 * g2;
                    const double N = rp * rp - rp * r * cc, E = top * g1 - bot * g2;
                    const double hH = rp * cc * (g2 - g1), hZ = N / rho2 * E;
                    const double rmc = rp - r * cc;
                    const double dHdr = cc * (g2 - g1) + rp * cc * rmc * (g13 - g23);
                    const double dE = -rmc * (top * g13 - bot * g23);
                    const double dZdr = ((2.0 * rp - r * cc) * E + N * dE) / rho2 - 2.0 * N * E * rmc / (rho2 * rho2);
                    const double dHdb = 0.5 * (rp * cc * top * g13 + rp * cc * bot * g23);
                    const double dZdb = 0.5 * (N * g13 + N * g23);
                    a[0] += w * hH;
                    a[1] += w * hZ;
                    a[2] += w * dHdr;
                    a[3] += w * dZdr;
                    a[4] += w * dHdb;
                    a[5] += w * dZdb;
                    a[6] += w * hH;                                     // RPhi * r
                    a[7] += w * rp * cc * (r - rp * cc) * (g13 - g23);  // RR
                    a[8] += w * rp * cc * (top * g13 - bot * g23);      // RZ
                    a[9] += w * N * (g13 - g23);                        // ZZ
                }
                s[0] += t.w * a[0];
                s[1] += t.w * a[1];
                s[2] += t.w * a[2];
                s[3] += t.w * a[3];
                s[4] += t.w * t.u * a[2];
                s[5] += t.w * t.u * a[3];
                s[6] += t.w * a[4];
                s[7] += t.w * a[5];
                s[8] += t.w * a[6];
                s[9] += t.w * a[7];
                s[10] += t.w * a[8];
                s[11] += t.w * a[9];
            }
        else
        {
            const AdjT *lt = reinterpret_cast<const AdjT *>(reinterpret_cast<const double2 *>(base) + C.off_l);
            for (int l = 0; l < C.nl; ++l)
            {
                const AdjT L = lt[l];
                const double zl = z + L.rp;
                for (int j = 0; j < C.nt; ++j)
                {
                    const AdjT t = tt[j];
                    const double rp = t.rp;
                    double a[8];
                    for (int i = 0; i < 8; ++i)
                        a[i] = 0.0;
                    for (int k = lane; k < C.nphi; k += kAdjLanes)
                    {
                        const double2 q = pt[k];
                        const double cc = q.x, w = q.y;
                        const double G = rsqrt(rp * rp + r * r + zl * zl - 2.0 * rp * r * cc);
                        const double G3 = G * G * G, G5 = G3 * G * G;
                        const double N = rp * rp - rp * r * cc, rmc = rp - r * cc;
                        const double hH = rp * cc * zl * G3;
                        a[0] += w * hH;
                        a[1] += w * N * G3;
                        a[2] += w * (cc * zl * G3 - 3.0 * rp * cc * zl * rmc * G5);
                        a[3] += w * ((2.0 * rp - r * cc) * G3 - 3.0 * N * rmc * G5);
                        a[4] += w * (rp * cc * G3 - 3.0 * rp * cc * zl * zl * G5);  // dH/dzl = RZ
                        a[5] += w * (-3.0 * N * zl * G5);                         // dZ/dzl = ZZ
                        a[6] += w * hH;                                           // RPhi * r
                        a[7] += w * (-3.0 * rp * cc * zl * (r - rp * cc) * G5);   // RR
                    }
                    const double lw = L.w * t.w;
                    s[0] += lw * a[0];
                    s[1] += lw * a[1];
                    s[2] += lw * a[2];
                    s[3] += lw * a[3];
                    s[4] += lw * t.u * a[2];
                    s[5] += lw * t.u * a[3];
                    s[6] += lw * L.u * a[4];
                    s[7] += lw * L.u * a[5];
                    s[8] += lw * a[6];
                    s[9] += lw * a[7];
                    s[10] += lw * a[4];
                    s[11] += lw * a[5];
                }
            }
        }
        for (int off = kAdjLanes / 2; off > 0; off /= 2)
            for (int i = 0; i < 12; ++i)
                s[i] += __shfl_xor_sync(0xffffffffu, s[i], off);
        double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (active && lane == 0)
        {
            const double K = C.K1 * C.NI;
            const double H = K * s[0], Z = K * s[1];
            const double Bl[3] = {H * cph, H * sph, Z};
            const double Bu[3] = {C.K1 * s[0] * cph, C.K1 * s[0] * sph, C.K1 * s[1]};  // per unit N I
            double B[3];
            matvec(C.T, Bu, B);
            double Tv[3];
            matTvec(C.T, v, Tv);  // local components of v
            // dB/dR, dB/da, dB/db (local components, rotated by T: v.T x = (T^T v).x)
            const double dR[3] = {K * s[2] * cph, K * s[2] * sph, K * s[3]};
            const double da[3] = {K * s[4] * cph, K * s[4] * sph, K * s[5]};
            // the fast method's constant holds 1 / b (its length integral is analytic)
            const double ib = C.fast ? 1.0 / C.b : 0.0;
            const double db[3] = {-Bl[0] * ib + K * s[6] * cph, -Bl[1] * ib + K * s[6] * sph, -Bl[2] * ib + K * s[7]};
            g[0] = Tv[0] * dR[0] + Tv[1] * dR[1] + Tv[2] * dR[2];
            g[1] = Tv[0] * da[0] + Tv[1] * da[1] + Tv[2] * da[2];
            g[2] = Tv[0] * db[0] + Tv[1] * db[1] + Tv[2] * db[2];
            g[3] = v[0] * B[0] + v[1] * B[1] + v[2] * B[2];
            // local Jacobian
            double G[9];
            const double rphi = K * s[8], rr = K * s[9], rz = K * s[10], zz = K * s[11];
            if (r / C.R < 1e-12)
            {
                G[0] = rr; G[1] = 0; G[2] = 0; G[3] = 0; G[4] = rr; G[5] = 0; G[6] = 0; G[7] = 0; G[8] = zz;
            }
            else
            {
                const double rp_ = rphi / r;
                G[0] = rr * cph * cph + rp_ * sph * sph;
                G[4] = rr * sph * sph + rp_ * cph * cph;
                G[1] = G[3] = sph * cph * (rr - rp_);
                G[2] = G[6] = rz * cph;
                G[5] = G[7] = rz * sph;
                G[8] = zz;
            }
            // position: -(T G T^T)^T v = -T G (T^T v)   (G symmetric)
            double GTv[3], pg[3];
            matvec(G, Tv, GTv);
            matvec(C.T, GTv, pg);
            g[4] = -pg[0];
            g[5] = -pg[1];
            g[6] = -pg[2];
            // angles: v . (T' Bl + T G T'^T d)
            for (int m = 0; m < 2; ++m)
            {
                const double *Tp = m == 0 ? C.Ta : C.Tb;
                double t1[3], u1[3], u2[3];
                matvec(Tp, Bl, t1);
                matTvec(Tp, d, u1);
                matvec(G, u1, u2);
                double t2[3];
                matvec(C.T, u2, t2);
                g[7 + m] = v[0] * (t1[0] + t2[0]) + v[1] * (t1[1] + t2[1]) + v[2] * (t1[2] + t2[2]);
            }
        }
        // CTA sum over its points: lanes of a warp (offsets kAdjLanes..16), then warps
        for (int off = kAdjLanes; off < 32; off *= 2)
            for (int i = 0; i < 9; ++i)
                g[i] += __shfl_xor_sync(0xffffffffu, g[i], off);
        if (threadIdx.x % 32 == 0)
            for (int i = 0; i < 9; ++i)
                red[threadIdx.x / 32][i] = g[i];
        __syncthreads();
        if (threadIdx.x < 9)
        {
            double sum = 0.0;
            for (int w = 0; w < kAdjThreads / 32; ++w)
                sum += red[w][threadIdx.x];
            partial[((long long)blockIdx.x * ncoils + c) * 9 + threadIdx.x] = sum;
        }
        __syncthreads();
    }
}

// fixed-order sum of the CTA partials
__global__ void adjointReduce(const double *__restrict__ partial, int blocks, int ncoils, double *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncoils * 9)
        return;
    double s = 0.0;
    for (int b = 0; b < blocks; ++b)
        s += partial[(long long)b * ncoils * 9 + i];
    out[i] = s;
}

void putBytes(std::vector<unsigned char> &blob, const void *p, size_t n)
{
    const unsigned char *c = static_cast<const unsigned char *>(p);
    blob.insert(blob.end(), c, c + n);
}

struct DBuf  // stream-ordered temporary from the library's memory pool
{
    void *p = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t alloc(size_t bytes, cudaStream_t s)
    {
        st = s;
        return scratchAlloc(&p, bytes, s);
    }
    ~DBuf()
    {
        if (p)
            cudaFreeAsync(p, st);
    }
};
} // namespace
} // namespace ccoil

using namespace ccoil;

extern "C" int ccoil_b_field_adjoint(const double *params, const ccoil_precision_args_t *precisions, int coil_count,
                                     const double *points, long long point_count, const double *grad_b,
                                     double *grad_params, void *stream)
{
    if (coil_count < 0 || (coil_count > 0 && (!params || !precisions)))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "null params/precisions or coil_count < 0");
    if (point_count < 0 || (point_count > 0 && (!points || !grad_b)) || (coil_count > 0 && !grad_params))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "null device buffers or point_count < 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (coil_count == 0)
        return CCOIL_OK;
    std::vector<unsigned char> blob;
    std::vector<long long> offsets;
    for (int c = 0; c < coil_count; ++c)
    {
        const double *q = params + 9 * c;
        const PrecisionArgs &pa = precisions[c];
        if (!validArgs(pa))
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "precision arguments out of range");
        const double R = q[0], NI = q[3];
        if (!(R > 0.0) || !(q[1] >= 0.0) || !(q[2] >= 0.0) || !std::isfinite(NI))
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "coil parameters need R > 0, a >= 0, b >= 0, finite N*I");
        // thin dimensions as the reference's Coil replaces them; b / R >= 1e-7 selects the fast method
        const double thin = 1e-7;
        const double a = q[1] / R < thin ? 1e-18 * R * thin : q[1];
        const double b = q[2] / R < thin ? 1e-18 * R * thin : q[2];
        const bool fast = q[2] / R >= thin;
        AdjCoil C;
        std::memset(&C, 0, sizeof(C));
        C.R = R;
        C.a = a;
        C.b = b;
        C.NI = NI;
        C.fast = fast ? 1 : 0;
        if (fast)
            C.K1 = 1e-7 * (1.0 / b) * (1.0 / pa.thickness_blocks) * (kPi / pa.angular_blocks) * 0.5;
        else
            C.K1 = 1e-7 * (kPi / pa.angular_blocks) * 0.25 / (pa.length_blocks * pa.thickness_blocks);
        C.half_b = 0.5 * b;
        C.pos[0] = q[4];
        C.pos[1] = q[5];
        C.pos[2] = q[6];
        const double cY = std::cos(q[7]), sY = std::sin(q[7]), cZ = std::cos(q[8]), sZ = std::sin(q[8]);
        const double T[9] = {cZ * cZ * cY - sZ * sZ, -sZ * cZ * cY - sZ * cZ, cZ * sY,
                             sZ * cZ * cY + sZ * cZ, cZ * cZ - sZ * sZ * cY, sZ * sY,
                             -sY * cZ, sY * sZ, cY};
        const double Ta[9] = {-cZ * cZ * sY, sZ * cZ * sY, cZ * cY,
                              -sZ * cZ * sY, sZ * sZ * sY, sZ * cY,
                              -cY * cZ, cY * sZ, -sY};
        const double k1 = cY + 1.0, dc = cZ * cZ - sZ * sZ;
        const double Tb[9] = {-2.0 * sZ * cZ * k1, -dc * k1, -sZ * sY,
                              dc * k1, -2.0 * sZ * cZ * k1, cZ * sY,
                              sY * sZ, sY * cZ, 0.0};
        std::memcpy(C.T, T, sizeof(T));
        std::memcpy(C.Ta, Ta, sizeof(Ta));
        std::memcpy(C.Tb, Tb, sizeof(Tb));
        C.nt = pa.thickness_blocks * pa.thickness_increments;
        C.nphi = pa.angular_blocks * pa.angular_increments;
        C.nl = fast ? 0 : pa.length_blocks * pa.length_increments;
        C.off_t = (int)(sizeof(AdjCoil) / 16);
        C.off_phi = C.off_t + 2 * C.nt;
        C.off_l = C.off_phi + C.nphi;
        offsets.push_back((long long)blob.size());
        putBytes(blob, &C, sizeof(C));
        const double tb = a / pa.thickness_blocks, ab = kPi / pa.angular_blocks;
        const double *tx = legendreNodes(pa.thickness_increments), *tw = legendreWeights(pa.thickness_increments);
        for (int bt = 0; bt < pa.thickness_blocks; ++bt)
            for (int i = 0; i < pa.thickness_increments; ++i)
            {
                const double u = (bt + 0.5 + 0.5 * tx[i]) / pa.thickness_blocks;
                AdjT e{R + tb * (bt + 0.5) + (tb * 0.5) * tx[i], tw[i], u, 0.0};
                putBytes(blob, &e, sizeof(e));
            }
        const double *ax = legendreNodes(pa.angular_increments), *aw = legendreWeights(pa.angular_increments);
        for (int bp = 0; bp < pa.angular_blocks; ++bp)
            for (int i = 0; i < pa.angular_increments; ++i)
            {
                double e[2] = {std::cos(ab * (bp + 0.5) + (ab * 0.5) * ax[i]), aw[i]};
                putBytes(blob, e, sizeof(e));
            }
        if (!fast)
        {
            // length nodes l = b v, v in [-1/2, 1/2] (CalculateFieldsSlow.cxx's length layer)
            const double lb = b / pa.length_blocks;
            const double *lx = legendreNodes(pa.length_increments), *lw = legendreWeights(pa.length_increments);
            for (int bl = 0; bl < pa.length_blocks; ++bl)
                for (int i = 0; i < pa.length_increments; ++i)
                {
                    const double l = -0.5 * b + lb * (bl + 0.5) + (lb * 0.5) * lx[i];
                    AdjT e{l, lw[i], -0.5 + (bl + 0.5 + 0.5 * lx[i]) / pa.length_blocks, 0.0};
                    putBytes(blob, &e, sizeof(e));
                }
        }
    }
    const long long blocks = point_count > 0 ? (point_count + kAdjPoints - 1) / kAdjPoints : 1;
    if (blocks > (1LL << 24))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "point_count too large for the adjoint's partial sums");
    DBuf dBlob, dOff, dPartial;
    cudaError_t e = dBlob.alloc(blob.size(), st);
    if (e == cudaSuccess)
        e = dOff.alloc(sizeof(long long) * offsets.size(), st);
    if (e == cudaSuccess)
        e = dPartial.alloc(sizeof(double) * 9 * coil_count * blocks, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dBlob.p, blob.data(), blob.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dOff.p, offsets.data(), sizeof(long long) * offsets.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
        return cudaFail(e, "adjoint set-up");
    if (point_count == 0)
        e = cudaMemsetAsync(dPartial.p, 0, sizeof(double) * 9 * coil_count, st);
    else
        adjointKernel<<<dim3((unsigned)blocks, (unsigned)std::min(coil_count, 65535)), kAdjThreads, 0, st>>>(
            static_cast<const unsigned char *>(dBlob.p), static_cast<const long long *>(dOff.p), coil_count, points,
            grad_b, point_count, static_cast<double *>(dPartial.p));
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e == cudaSuccess)
        adjointReduce<<<(coil_count * 9 + 255) / 256, 256, 0, st>>>(static_cast<const double *>(dPartial.p),
                                                                    (int)blocks, coil_count, grad_params);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);  // results in grad_params when the call returns
    return e == cudaSuccess ? CCOIL_OK : cudaFail(e, "adjoint");
}
