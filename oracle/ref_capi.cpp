// Test infrastructure only (never linked into the product).
//
// A C-ABI over the reference's own, unmodified CPU implementation (C-Coil,
// src/Coil, src/CoilGroup, src/Tensor, src/LegendreMatrix), compiled in place by
// oracle/Makefile into oracle/_ref/libccoil_ref.so.  The tests and the CPU
// baseline of bench.py call it through ctypes to obtain the reference's double
// precision results on the same seeded inputs as the CUDA path.
//
// Coils are passed as 11 doubles:
//   {R, a, b, N, I, f, x, y, z, yAxisAngle, zAxisAngle}
// which feed the reference constructor Coil(R, a, b, N, I, f, PrecisionFactor,
// threads, position, yAngle, zAngle) (src/Coil/Coil.h:293-295).
// Points are interleaved xyz doubles (the memory layout of vec3::Vector3Array).
// Every function returns 0 on success and -1 if the reference threw.
#include "Coil.h"
#include "CoilGroup.h"
#include "LegendreMatrix.h"

#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

namespace
{
int g_threads = 8;

enum Quantity { QTY_A = 0, QTY_B = 1, QTY_E = 2, QTY_G = 3 };

std::unique_ptr<Coil> makeCoil(const double *c, double pf)
{
    return std::make_unique<Coil>(c[0], c[1], c[2], int(c[3]), c[4], c[5], PrecisionFactor(pf), g_threads,
                                  vec3::Vector3(c[6], c[7], c[8]), c[9], c[10]);
}

std::shared_ptr<Coil> makeSharedCoil(const double *c, double pf)
{
    return std::make_shared<Coil>(c[0], c[1], c[2], int(c[3]), c[4], c[5], PrecisionFactor(pf), g_threads,
                                  vec3::Vector3(c[6], c[7], c[8]), c[9], c[10]);
}

vec3::Vector3Array toArray(long long n, const double *p)
{
    vec3::Vector3Array arr;
    arr.reserve(n);
    for (long long i = 0; i < n; ++i)
        arr.append(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    return arr;
}

void putVectors(const vec3::Vector3Array &arr, double *out)
{
    for (size_t i = 0; i < arr.size(); ++i)
    {
        out[3 * i] = arr[i].x;
        out[3 * i + 1] = arr[i].y;
        out[3 * i + 2] = arr[i].z;
    }
}

void putMatrices(const vec3::Matrix3Array &arr, double *out)
{
    for (size_t i = 0; i < arr.size(); ++i)
    {
        const vec3::Matrix3 &m = arr[i];
        double v[9] = {m.xx, m.xy, m.xz, m.yx, m.yy, m.yz, m.zx, m.zy, m.zz};
        std::memcpy(out + 9 * i, v, sizeof(v));
    }
}

PrecisionArguments toArgs(const int *p)
{
    return PrecisionArguments(p[0], p[1], p[2], p[3], p[4], p[5]);
}

void fromArgs(const PrecisionArguments &a, int *out)
{
    out[0] = a.angularBlocks;
    out[1] = a.thicknessBlocks;
    out[2] = a.lengthBlocks;
    out[3] = a.angularIncrements;
    out[4] = a.thicknessIncrements;
    out[5] = a.lengthIncrements;
}

// 0 = CPU_ST, 1 = CPU_MT, 2 = GPU (a build with USE_GPU, linked against
// libccoil_b200.so, whose exports stand in for the reference's CUDA kernels)
ComputeMethod toMethod(int m) { return m == 2 ? GPU : (m == 1 ? CPU_MT : CPU_ST); }

void coilFields(const Coil &coil, const PrecisionArguments &prec, int qty, ComputeMethod method,
                const vec3::Vector3Array &pts, double *out, bool accumulate)
{
    long long n = (long long)pts.size();
    int width = qty == QTY_G ? 9 : 3;
    std::vector<double> tmp((size_t)n * width);
    switch (qty)
    {
        case QTY_A: putVectors(coil.computeAllAPotentialVectors(pts, prec, method), tmp.data()); break;
        case QTY_B: putVectors(coil.computeAllBFieldVectors(pts, prec, method), tmp.data()); break;
        case QTY_E: putVectors(coil.computeAllEFieldVectors(pts, prec, method), tmp.data()); break;
        default: putMatrices(coil.computeAllBGradientMatrices(pts, prec, method), tmp.data()); break;
    }
    for (size_t i = 0; i < tmp.size(); ++i)
        out[i] = accumulate ? out[i] + tmp[i] : tmp[i];
}
} // namespace

extern "C" {

int ref_set_threads(int n)
{
    g_threads = n < 1 ? 1 : n;
    return 0;
}

int ref_legendre(int order, double *pos, double *w)
{
    if (order < 1 || order > Legendre::maxLegendreOrder)
        return -1;
    for (int i = 0; i < order; ++i)
    {
        pos[i] = Legendre::positionMatrix[order - 1][i];
        w[i] = Legendre::weightsMatrix[order - 1][i];
    }
    return 0;
}

// derived attributes: {thickness, length, currentDensity, current, useFastMethod,
// coilType, transform[9], inverseTransform[9]}
int ref_coil_info(const double *c, double *out)
{
    try
    {
        auto coil = makeCoil(c, 5.0);
        out[0] = coil->getThickness();
        out[1] = coil->getLength();
        out[2] = coil->getCurrentDensity();
        out[3] = coil->getCurrent();
        out[4] = coil->isUsingFastMethod() ? 1.0 : 0.0;
        out[5] = double(int(coil->getCoilType()));
        vec3::Matrix3 t = coil->getTransformationMatrix();
        vec3::Matrix3 it = coil->getInverseTransformationMatrix();
        double tv[18] = {t.xx, t.xy, t.xz, t.yx, t.yy, t.yz, t.zx, t.zy, t.zz,
                         it.xx, it.xy, it.xz, it.yx, it.yy, it.yz, it.zx, it.zy, it.zz};
        std::memcpy(out + 6, tv, sizeof(tv));
        return 0;
    } catch (...) { return -1; }
}

int ref_precision_args(const double *c, double pf, int gpu, int *out6)
{
    try
    {
        auto coil = makeCoil(c, pf);
        fromArgs(gpu ? coil->getPrecisionSettingsGPU() : coil->getPrecisionSettingsCPU(), out6);
        return 0;
    } catch (...) { return -1; }
}

int ref_secondary_precision_gpu(const double *c, double pf, int *out6)
{
    try
    {
        auto coil = makeCoil(c, pf);
        fromArgs(PrecisionArguments::getSecondaryCoilPrecisionArgumentsGPU(*coil, PrecisionFactor(pf)), out6);
        return 0;
    } catch (...) { return -1; }
}

int ref_pair_args(const double *p, const double *s, double pf, int gpu, int zAxis, int pureGPU, int *out12)
{
    try
    {
        auto prim = makeCoil(p, pf);
        auto sec = makeCoil(s, pf);
        CoilPairArguments a = CoilPairArguments::getAppropriateCoilPairArguments(
            *prim, *sec, PrecisionFactor(pf), gpu ? GPU : CPU_ST, zAxis != 0, pureGPU != 0);
        fromArgs(a.primaryPrecision, out12);
        fromArgs(a.secondaryPrecision, out12 + 6);
        return 0;
    } catch (...) { return -1; }
}

// One coil: fields at n points with explicit precision args (prec6) or, if prec6
// is null, the coil's default CPU precision at pf.  method 0 = CPU_ST, 1 = CPU_MT,
// 2 = GPU.
int ref_coil_fields(const double *c, double pf, const int *prec6, int qty, int method, long long n,
                    const double *pts, double *out)
{
    try
    {
        auto coil = makeCoil(c, pf);
        PrecisionArguments prec = prec6 ? toArgs(prec6) : coil->getPrecisionSettingsCPU();
        coilFields(*coil, prec, qty, toMethod(method), toArray(n, pts), out, false);
        return 0;
    } catch (...) { return -1; }
}

// A group as CoilGroup::computeAll*(points, CPU_ST) evaluates it
// (src/CoilGroup/Fields/ComputeFields.cxx:60-71): member coils in order, each at
// its own default CPU precision for the group's PrecisionFactor, summed point by
// point.  method 1 runs each member with CPU_MT (the per-member MT path), which
// avoids the group MTD path and its doubled output length.
int ref_group_fields(int ncoils, const double *coils, double pf, int qty, int method, long long n,
                     const double *pts, double *out)
{
    try
    {
        vec3::Vector3Array arr = toArray(n, pts);
        int width = qty == QTY_G ? 9 : 3;
        std::memset(out, 0, sizeof(double) * (size_t)n * width);
        for (int k = 0; k < ncoils; ++k)
        {
            auto coil = makeCoil(coils + 11 * k, pf);
            coilFields(*coil, coil->getPrecisionSettingsCPU(), qty, toMethod(method), arr, out, true);
        }
        return 0;
    } catch (...) { return -1; }
}

// A group through the reference's own group dispatch, CoilGroup::computeAll*(points, method)
// (src/CoilGroup/Fields/ComputeFields.cxx): with method 2 (GPU) its glue packs every member
// at its GPU precision for pf (src/CoilGroup/Utils/GPUArgumentGeneration.cxx:17-95) and calls
// Calculate_hardware_accelerated_*_group.
int ref_group_fields_dispatch(int ncoils, const double *coils, double pf, int qty, int method, long long n,
                              const double *pts, double *out)
{
    try
    {
        std::vector<std::shared_ptr<Coil>> members;
        for (int k = 0; k < ncoils; ++k)
            members.push_back(makeSharedCoil(coils + 11 * k, pf));
        CoilGroup group(members, PrecisionFactor(pf), g_threads);
        vec3::Vector3Array arr = toArray(n, pts);
        switch (qty)
        {
            case QTY_A: putVectors(group.computeAllAPotentialVectors(arr, toMethod(method)), out); break;
            case QTY_B: putVectors(group.computeAllBFieldVectors(arr, toMethod(method)), out); break;
            case QTY_E: putVectors(group.computeAllEFieldVectors(arr, toMethod(method)), out); break;
            default: putMatrices(group.computeAllBGradientMatrices(arr, toMethod(method)), out); break;
        }
        return 0;
    } catch (...) { return -1; }
}

int ref_mutual_inductance(const double *p, const double *s, double pf, int method, double *out)
{
    try
    {
        auto prim = makeCoil(p, pf);
        auto sec = makeCoil(s, pf);
        *out = Coil::computeMutualInductance(*prim, *sec, PrecisionFactor(pf), toMethod(method));
        return 0;
    } catch (...) { return -1; }
}

int ref_mutual_inductance_args(const double *p, const double *s, const int *args12, int method, double *out)
{
    try
    {
        auto prim = makeCoil(p, 5.0);
        auto sec = makeCoil(s, 5.0);
        CoilPairArguments a(toArgs(args12), toArgs(args12 + 6));
        *out = Coil::computeMutualInductance(*prim, *sec, a, toMethod(method));
        return 0;
    } catch (...) { return -1; }
}

int ref_force_torque(const double *p, const double *s, double pf, int method, double *out6)
{
    try
    {
        auto prim = makeCoil(p, pf);
        auto sec = makeCoil(s, pf);
        auto ft = Coil::computeForceTorque(*prim, *sec, PrecisionFactor(pf), toMethod(method));
        double v[6] = {ft.first.x, ft.first.y, ft.first.z, ft.second.x, ft.second.y, ft.second.z};
        std::memcpy(out6, v, sizeof(v));
        return 0;
    } catch (...) { return -1; }
}

int ref_force_torque_args(const double *p, const double *s, const int *args12, int method, double *out6)
{
    try
    {
        auto prim = makeCoil(p, 5.0);
        auto sec = makeCoil(s, 5.0);
        CoilPairArguments a(toArgs(args12), toArgs(args12 + 6));
        auto ft = Coil::computeForceTorque(*prim, *sec, a, toMethod(method));
        double v[6] = {ft.first.x, ft.first.y, ft.first.z, ft.second.x, ft.second.y, ft.second.z};
        std::memcpy(out6, v, sizeof(v));
        return 0;
    } catch (...) { return -1; }
}

// Coil::computeAll{MutualInductance,ForceTorque}Arrangements
// (src/Coil/MInductance/ComputeMInductanceMethods.cxx:83-143,
//  src/Coil/ForceAndTorque/ComputeForceMethods.cxx:58-117).
// Angles are arrays of length n; positions interleaved xyz.
int ref_m_arrangements(const double *p, const double *s, long long n, const double *primPos, const double *secPos,
                       const double *pY, const double *pZ, const double *sY, const double *sZ, double pf, int method,
                       double *out)
{
    try
    {
        auto prim = makeCoil(p, pf);
        auto sec = makeCoil(s, pf);
        auto res = Coil::computeAllMutualInductanceArrangements(
            *prim, *sec, toArray(n, primPos), toArray(n, secPos), std::vector<double>(pY, pY + n),
            std::vector<double>(pZ, pZ + n), std::vector<double>(sY, sY + n), std::vector<double>(sZ, sZ + n),
            PrecisionFactor(pf), toMethod(method));
        for (long long i = 0; i < n; ++i)
            out[i] = res[i];
        return 0;
    } catch (...) { return -1; }
}

int ref_ft_arrangements(const double *p, const double *s, long long n, const double *primPos, const double *secPos,
                        const double *pY, const double *pZ, const double *sY, const double *sZ, double pf, int method,
                        double *out)
{
    try
    {
        auto prim = makeCoil(p, pf);
        auto sec = makeCoil(s, pf);
        auto res = Coil::computeAllForceTorqueArrangements(
            *prim, *sec, toArray(n, primPos), toArray(n, secPos), std::vector<double>(pY, pY + n),
            std::vector<double>(pZ, pZ + n), std::vector<double>(sY, sY + n), std::vector<double>(sZ, sZ + n),
            PrecisionFactor(pf), toMethod(method));
        for (long long i = 0; i < n; ++i)
        {
            out[6 * i] = res[i].first.x;
            out[6 * i + 1] = res[i].first.y;
            out[6 * i + 2] = res[i].first.z;
            out[6 * i + 3] = res[i].second.x;
            out[6 * i + 4] = res[i].second.y;
            out[6 * i + 5] = res[i].second.z;
        }
        return 0;
    } catch (...) { return -1; }
}

// CoilGroup::computeAll{MutualInductance,ForceTorque}Arrangements
// (src/CoilGroup/MInductance/ComputeMInductance.cxx:23-64,
//  src/CoilGroup/ForceAndTorque/ComputeForce.cxx:47-89).  secMember >= 0 makes the
// secondary that group member (which the group then leaves out of its own sum);
// otherwise the secondary is the separate coil `s`.
int ref_group_m_arrangements(int ncoils, const double *coils, const double *s, int secMember, long long n,
                             const double *secPos,
                             const double *sY, const double *sZ, double pf, int method, double *out)
{
    try
    {
        std::vector<std::shared_ptr<Coil>> members;
        for (int k = 0; k < ncoils; ++k)
            members.push_back(makeSharedCoil(coils + 11 * k, pf));
        CoilGroup group(members, PrecisionFactor(pf), g_threads);
        auto own = makeCoil(s, pf);
        const Coil &sec = secMember >= 0 ? group[secMember] : *own;
        auto res = group.computeAllMutualInductanceArrangements(
            sec, toArray(n, secPos), std::vector<double>(sY, sY + n), std::vector<double>(sZ, sZ + n),
            PrecisionFactor(pf), toMethod(method));
        for (long long i = 0; i < n; ++i)
            out[i] = res[i];
        return 0;
    } catch (...) { return -1; }
}

int ref_group_ft_arrangements(int ncoils, const double *coils, const double *s, int secMember, long long n,
                             const double *secPos,
                              const double *sY, const double *sZ, double pf, int method, double *out)
{
    try
    {
        std::vector<std::shared_ptr<Coil>> members;
        for (int k = 0; k < ncoils; ++k)
            members.push_back(makeSharedCoil(coils + 11 * k, pf));
        CoilGroup group(members, PrecisionFactor(pf), g_threads);
        auto own = makeCoil(s, pf);
        const Coil &sec = secMember >= 0 ? group[secMember] : *own;
        auto res = group.computeAllForceTorqueArrangements(
            sec, toArray(n, secPos), std::vector<double>(sY, sY + n), std::vector<double>(sZ, sZ + n),
            PrecisionFactor(pf), toMethod(method));
        for (long long i = 0; i < n; ++i)
        {
            out[6 * i] = res[i].first.x;
            out[6 * i + 1] = res[i].first.y;
            out[6 * i + 2] = res[i].first.z;
            out[6 * i + 3] = res[i].second.x;
            out[6 * i + 4] = res[i].second.y;
            out[6 * i + 5] = res[i].second.z;
        }
        return 0;
    } catch (...) { return -1; }
}

int ref_self_inductance(const double *c, double pf, double *out)
{
    try
    {
        auto coil = makeCoil(c, pf);
        *out = coil->computeAndSetSelfInductance(PrecisionFactor(pf));
        return 0;
    } catch (...) { return -1; }
}

} // extern "C"
