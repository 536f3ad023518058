// Self inductance of many coils (Coil::computeAndSetSelfInductance,
// src/Coil/MInductance/ComputeMInductanceMethods.cxx:55-81).
//
// The reference centres the coil and takes the z-axis pair arguments of the
// coil with itself.  A FLAT coil goes through the coaxial mutual inductance
// of the coil with itself: here, the z-axis pass of the arrangement kernels.
// RECTANGULAR and THIN coils use the closed form of
// Coil::calculateSelfInductance (src/Coil/MInductance/CalculateMInductanceZAxis.cxx:233-319):
// a triple sum over a unit-thickness radial layer, the coil's thickness nodes
// and its angular nodes.  FILAMENT has no self inductance (the integral
// diverges) and is rejected.  One CTA per coil; the terms follow the
// reference's operation order, and the CTA reduces them in a fixed order.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace ccoil
{
namespace
{
constexpr double kPi = 3.14159265358979323846;
constexpr double kMuReduced = 1e-7;

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double sqr(double a) { return __dsqrt_rn(a); }

// Per coil: this header, then {radial position, w}, {thickness position, w}, {cos, w}
struct alignas(16) SelfHeader
{
    double constant;  // g_MiReduced J tBlock aBlock radialBlock 2 0.125
    double length;
    double scale;     // 2 pi N / (I length)
    double pad;
    int n_r, n_t, n_phi, pad1;
};
static_assert(sizeof(SelfHeader) % 16 == 0, "self-inductance header alignment");

__global__ void __launch_bounds__(256) selfInductanceKernel(const unsigned char *__restrict__ blob,
                                                            const long long *__restrict__ offsets,
                                                            double *__restrict__ out)
{
    __shared__ double warpSums[8];
    const unsigned char *base = blob + offsets[blockIdx.x];
    const SelfHeader &h = *reinterpret_cast<const SelfHeader *>(base);
    const double2 *rn = reinterpret_cast<const double2 *>(base + sizeof(SelfHeader));
    const double2 *tn = rn + h.n_r, *pn = tn + h.n_t;
    const double b = h.length, b2 = mul(b, b);
    const long long n = (long long)h.n_r * h.n_t * h.n_phi;
    double part = 0.0;
    for (long long e = threadIdx.x; e < n; e += blockDim.x)
    {
        const int k = (int)(e % h.n_phi);
        const long long ij = e / h.n_phi;
        const int j = (int)(ij % h.n_t), i = (int)(ij / h.n_t);
        const double2 R = rn[i], T = tn[j], P = pn[k];
        const double tempConst = mul(mul(h.constant, R.y), T.y);
        const double A = mul(mul(2.0, T.x), R.x);
        const double B = add(mul(T.x, T.x), mul(R.x, R.x));
        const double C = sub(B, mul(A, P.x));
        const double D = sqr(C), E = sqr(add(C, b2));
        const double F = dvd(b, D), G = sqr(add(mul(F, F), 1.0));
        const double H = log(add(F, G));
        part += mul(mul(mul(mul(tempConst, P.y), A), P.x), add(sub(D, E), mul(b, H)));
    }
#pragma unroll
    for (int off = 16; off > 0; off /= 2)
        part += __shfl_xor_sync(0xffffffffu, part, off);
    if (threadIdx.x % 32 == 0)
        warpSums[threadIdx.x / 32] = part;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w)
            s += warpSums[w];
        out[blockIdx.x] = mul(s, h.scale);
    }
}

void put(std::vector<unsigned char> &blob, const void *p, size_t n)
{
    const unsigned char *c = static_cast<const unsigned char *>(p);
    blob.insert(blob.end(), c, c + n);
}

// the tables of Coil::calculateSelfInductance for one coil at pair arguments (p, s)
void buildSelf(const Coil &k, const PrecisionArgs &p, const PrecisionArgs &s, std::vector<unsigned char> &blob)
{
    const double thicknessBlock = k.thickness / p.thickness_blocks;
    const double angularBlock = kPi / p.angular_blocks;
    const double radialBlock = 1.0 / s.thickness_blocks;
    SelfHeader h;
    std::memset(&h, 0, sizeof(h));
    h.constant = kMuReduced * k.current_density * thicknessBlock * angularBlock * radialBlock * 2 * 0.125;
    h.length = k.length;
    h.scale = 2 * kPi * k.num_turns / (k.current * k.length);
    std::vector<double> r, t, f;
    const double *rx = legendreNodes(s.thickness_increments), *rw = legendreWeights(s.thickness_increments);
    for (int bR = 0; bR < s.thickness_blocks; ++bR)
    {
        const double blockPositionR = k.inner_radius + radialBlock * k.thickness * (bR + 0.5);
        for (int i = 0; i < s.thickness_increments; ++i)
            r.insert(r.end(), {blockPositionR + (radialBlock * k.thickness * 0.5) * rx[i], rw[i]});
    }
    const double *tx = legendreNodes(p.thickness_increments), *tw = legendreWeights(p.thickness_increments);
    for (int bT = 0; bT < p.thickness_blocks; ++bT)
    {
        const double blockPositionT = k.inner_radius + thicknessBlock * (bT + 0.5);
        for (int i = 0; i < p.thickness_increments; ++i)
            t.insert(t.end(), {blockPositionT + (thicknessBlock * 0.5) * tx[i], tw[i]});
    }
    const double *ax = legendreNodes(p.angular_increments), *aw = legendreWeights(p.angular_increments);
    for (int bP = 0; bP < p.angular_blocks; ++bP)
    {
        const double blockPositionPhi = angularBlock * (bP + 0.5);
        for (int i = 0; i < p.angular_increments; ++i)
            f.insert(f.end(), {std::cos(blockPositionPhi + (angularBlock * 0.5) * ax[i]), aw[i]});
    }
    h.n_r = (int)r.size() / 2;
    h.n_t = (int)t.size() / 2;
    h.n_phi = (int)f.size() / 2;
    put(blob, &h, sizeof(h));
    put(blob, r.data(), sizeof(double) * r.size());
    put(blob, t.data(), sizeof(double) * t.size());
    put(blob, f.data(), sizeof(double) * f.size());
}

// stream-ordered temporary from the library's memory pool
struct Buf
{
    void *p = nullptr;
    cudaStream_t st = nullptr;
    cudaError_t alloc(size_t bytes, cudaStream_t s)
    {
        st = s;
        return scratchAlloc(&p, bytes, s);
    }
    ~Buf()
    {
        if (p)
            cudaFreeAsync(p, st);
    }
};
} // namespace

int cudaFail(cudaError_t e, const char *what);
} // namespace ccoil

using namespace ccoil;

extern "C" int ccoil_self_inductances(const ccoil_coil_t *coils, const ccoil_precision_args_t *pair_precisions,
                                      int count, double *out, void *stream)
{
    if (count < 0 || (count > 0 && (!coils || !pair_precisions || !out)))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "null coils, precisions or output, or count < 0");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<unsigned char> blob;
    std::vector<long long> offsets;
    std::vector<int> closedForm;  // index into the kernel's output, or -1 for a FLAT coil
    for (int c = 0; c < count; ++c)
    {
        const Coil &k = coils[c];
        const PrecisionArgs &p = pair_precisions[2 * c], &s = pair_precisions[2 * c + 1];
        if (k.coil_type == 3)
            return fail(CCOIL_ERR_INVALID_ARGUMENT, "coil " + std::to_string(c) +
                                                        ": a filament's self inductance is not defined "
                                                        "(the integral diverges)");
        if (!validArgs(p) || !validArgs(s))
            return fail(CCOIL_ERR_INVALID_ARGUMENT, "coil " + std::to_string(c) + ": precision arguments out of range");
        if (!(k.inner_radius > 0.0) || !(k.thickness > 0.0) || !(k.length > 0.0) || k.current == 0.0)
            return fail(CCOIL_ERR_INVALID_ARGUMENT, "coil " + std::to_string(c) + ": invalid dimensions or zero current");
        if (k.coil_type == 2)
        {
            closedForm.push_back(-1);
            continue;
        }
        closedForm.push_back((int)offsets.size());
        offsets.push_back((long long)blob.size());
        buildSelf(k, p, s, blob);
    }
    // FLAT coils: the coaxial mutual inductance of the centred coil with itself
    for (int c = 0; c < count; ++c)
    {
        if (closedForm[c] >= 0)
            continue;
        const Coil &src = coils[c];
        Coil k;
        const double origin[3] = {0.0, 0.0, 0.0};
        initCoil(src.inner_radius, src.thickness, src.length, src.num_turns, src.current, src.sine_frequency, origin,
                 0.0, 0.0, k);
        const ccoil_precision_args_t zargs[2] = {pair_precisions[2 * c], pair_precisions[2 * c + 1]};
        k.precision = zargs[0];
        ccoil_pose_t pose = {{0.0, 0.0, 0.0}, 0.0, 0.0};
        const int rc = ccoil_pair_arrangements_zaxis(&k, 1, &k, &zargs[1], zargs, &pose, &pose, 1,
                                                     CCOIL_PAIR_MUTUAL_INDUCTANCE, CCOIL_PRECISION_FP64, &out[c],
                                                     nullptr, CCOIL_MEMORY_HOST, stream);
        if (rc != CCOIL_OK)
            return rc;
    }
    if (offsets.empty())
        return CCOIL_OK;
    Buf dBlob, dOff, dOut;
    cudaError_t e = dBlob.alloc(blob.size(), st);
    if (e == cudaSuccess)
        e = dOff.alloc(sizeof(long long) * offsets.size(), st);
    if (e == cudaSuccess)
        e = dOut.alloc(sizeof(double) * offsets.size(), st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dBlob.p, blob.data(), blob.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dOff.p, offsets.data(), sizeof(long long) * offsets.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
        return cudaFail(e, "self-inductance buffers");
    selfInductanceKernel<<<(unsigned)offsets.size(), 256, 0, st>>>(static_cast<const unsigned char *>(dBlob.p),
                                                                   static_cast<const long long *>(dOff.p),
                                                                   static_cast<double *>(dOut.p));
    e = cudaGetLastError();
    std::vector<double> res(offsets.size());
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(res.data(), dOut.p, sizeof(double) * res.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, "self-inductance kernel");
    for (int c = 0; c < count; ++c)
        if (closedForm[c] >= 0)
            out[c] = res[closedForm[c]];
    return CCOIL_OK;
}
