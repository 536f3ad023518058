// The reference's own GPU entry points (include/ccoil_reference_abi.h) on top
// of this library's kernels: the reference's host glue links against them
// unchanged.  Each call rebuilds the coil descriptors the C-ABI takes from the
// reference's table structs, checks that the tables are the Gauss-Legendre
// tables the glue always writes (the kernels regenerate them at full
// precision from the node counts), and evaluates in FP64, synchronously, on
// the default stream.
#include "ccoil_internal.h"
#include "../../include/ccoil_reference_abi.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace ccoil
{
namespace
{
constexpr double kPi = 3.14159265358979323846;
constexpr double kMuReduced = 1e-7;  // g_MiReduced
constexpr int kIncrements = CCOIL_REFERENCE_GPU_INCREMENTS;
// the glue's tables are Legendre::positionMatrix / weightsMatrix entries (and
// cosines of their angles), which agree with this library's to ~1e-16
constexpr double kTableTolerance = 1e-13;

[[noreturn]] void raise(const std::string &where, const std::string &what)
{
    throw std::runtime_error(where + ": " + what);
}

void check(int status, const char *where)
{
    if (status != CCOIL_OK)
        raise(where, ccoil_last_error_message());
}

void checkCount(int n, const char *name, const char *where)
{
    if (n < 1 || n > kIncrements)
        raise(where, std::string(name) + " must lie in [1, " + std::to_string(kIncrements) + "], got " +
                         std::to_string(n));
}

// nodes[i] (and weights[i]) of order n must be the Gauss-Legendre table of that order
void checkLegendre(const double *nodes, const double *weights, int n, const char *name, const char *where)
{
    const double *x = legendreNodes(n), *w = legendreWeights(n);
    for (int i = 0; i < n; ++i)
        if (!(std::fabs(nodes[i] - x[i]) <= kTableTolerance) || !(std::fabs(weights[i] - w[i]) <= kTableTolerance))
            raise(where, std::string(name) + " is not the Gauss-Legendre table of order " + std::to_string(n));
}

// cos(pi / 2 (1 + x_i)) and w_i, the angular table of generateCoilData
void checkCosines(const double *cosines, const double *weights, int n, const char *name, const char *where)
{
    const double *x = legendreNodes(n), *w = legendreWeights(n);
    for (int i = 0; i < n; ++i)
        if (!(std::fabs(cosines[i] - std::cos(0.5 * kPi * (1.0 + x[i]))) <= kTableTolerance) ||
            !(std::fabs(weights[i] - w[i]) <= kTableTolerance))
            raise(where, std::string(name) + " is not the angular table of order " + std::to_string(n));
}

ccoil_precision_args_t singleBlock(int angular, int thickness, int length)
{
    ccoil_precision_args_t p;
    p.angular_blocks = p.thickness_blocks = p.length_blocks = 1;
    p.angular_increments = angular;
    p.thickness_increments = thickness;
    p.length_increments = length;
    return p;
}

// The current density whose constant this library's tables fold in equals the
// glue's constFactor: mu0/4pi J a pi/2 (fast) or mu0/4pi J a b pi/2 (slow).
double currentDensity(double constFactor, double thickness, double length, bool fast)
{
    return constFactor / (kMuReduced * thickness * (fast ? 1.0 : length) * kPi * 0.5);
}

// A primary (field source) from its CoilData.  The reference's GPU kernels run
// the slow method without a length layer (the length is folded into
// constFactor): one length node at the centre is the same quadrature.
Coil coilFromData(const CoilData &d, const char *where)
{
    checkCount(d.angularIncrements, "angularIncrements", where);
    checkCount(d.thicknessIncrements, "thicknessIncrements", where);
    checkCosines(d.cosPrecomputeArray, d.angularWeightArray, d.angularIncrements, "the angular table", where);
    checkLegendre(d.thicknessPositionArray, d.thicknessWeightArray, d.thicknessIncrements, "the thickness table",
                  where);
    if (!(d.innerRadius > 0.0) || !(d.thickness > 0.0) || !(d.length > 0.0))
        raise(where, "inner radius, thickness and length must be positive");
    Coil k{};
    k.inner_radius = d.innerRadius;
    k.thickness = d.thickness;
    k.length = d.length;
    k.use_fast_method = d.useFastMethod ? 1 : 0;
    k.current_density = currentDensity(d.constFactor, d.thickness, d.length, d.useFastMethod);
    k.current = d.current;
    k.sine_frequency = d.frequency;
    for (int i = 0; i < 3; ++i)
        k.position[i] = d.positionVector[i];
    for (int i = 0; i < 9; ++i)
    {
        k.transform[i] = d.transformArray[i];
        k.inverse_transform[i] = d.invTransformArray[i];
    }
    k.num_turns = 1;
    k.coil_type = d.useFastMethod ? kRectangular : kFlat;
    k.precision = singleBlock(d.angularIncrements, d.thicknessIncrements, 1);
    return k;
}

template <typename Result>
void fields(const Coil *coils, int count, long long opCount, const VectorData *posArr, Result *resArr, int field,
            const char *where)
{
    if (opCount < 0)
        raise(where, "negative point count");
    if (opCount == 0)
        return;
    if (!posArr)
        raise(where, "null position array");
    constexpr int width = sizeof(Result) / sizeof(double);
    // a null result array still evaluates (the reference leaves the result on the device)
    std::vector<double> discard;
    double *out = reinterpret_cast<double *>(resArr);
    if (!out)
    {
        discard.resize((size_t)opCount * width);
        out = discard.data();
    }
    check(ccoil_compute_fields(coils, count, reinterpret_cast<const double *>(posArr), opCount, field,
                               CCOIL_PRECISION_FP64, out, CCOIL_MEMORY_HOST, nullptr),
          where);
}

template <typename Result>
void singleField(long long opCount, const CoilData &coil, const VectorData *posArr, Result *resArr, int field,
                 const char *where)
{
    const Coil k = coilFromData(coil, where);
    fields(&k, 1, opCount, posArr, resArr, field, where);
}

template <typename Result>
void groupField(long long coilCount, long long opCount, const CoilData *coilArr, const VectorData *posArr,
                Result *resArr, int field, const char *where)
{
    if (coilCount < 0 || coilCount > (1LL << 30) || (coilCount > 0 && !coilArr))
        raise(where, "bad coil count or null coil array");
    std::vector<Coil> coils;
    coils.reserve((size_t)coilCount);
    for (long long i = 0; i < coilCount; ++i)
        coils.push_back(coilFromData(coilArr[i], where));
    if (coilCount == 0)
    {
        if (resArr && opCount > 0)
            for (long long i = 0; i < opCount; ++i)
                resArr[i] = Result{};
        return;
    }
    fields(coils.data(), (int)coilCount, opCount, posArr, resArr, field, where);
}

// The secondary of a pair: unit turns and current, so the kernel's scale is
// 2 pi (over I1 for the mutual inductance) and the glue's correctionFactor
// multiplies the result.
Coil secondaryCoil(double R, double a, double b, int nA, int nT, int nL, const char *where)
{
    checkCount(nA, "secondary angularIncrements", where);
    checkCount(nT, "secondary thicknessIncrements", where);
    checkCount(nL, "secondary lengthIncrements", where);
    if (!(R > 0.0) || !(a > 0.0) || !(b > 0.0))
        raise(where, "secondary inner radius, thickness and length must be positive");
    Coil s{};
    s.inner_radius = R;
    s.thickness = a;
    s.length = b;
    s.current = 1.0;
    s.num_turns = 1;
    s.use_fast_method = 1;
    s.transform[0] = s.transform[4] = s.transform[8] = 1.0;
    s.inverse_transform[0] = s.inverse_transform[4] = s.inverse_transform[8] = 1.0;
    s.precision = singleBlock(nA, nT, nL);
    return s;
}

void pairs(const Coil *prims, int primCount, const Coil &sec, const std::vector<ccoil_pose_t> *primPoses,
           const std::vector<ccoil_pose_t> &secPoses, int quantity, double correctionFactor, double *out,
           const char *where)
{
    const long long count = (long long)secPoses.size();
    std::vector<ccoil_precision_args_t> secPrec((size_t)primCount, sec.precision);
    PairOptions opt;
    opt.full_ring = true;
    opt.scale = correctionFactor / (2.0 * kPi);
    check(pairArrangements(prims, primCount, &sec, secPrec.data(), nullptr, primPoses ? primPoses->data() : nullptr,
                           secPoses.data(), count, quantity, CCOIL_PRECISION_FP64, out, nullptr, CCOIL_MEMORY_HOST,
                           nullptr, opt),
          where);
}

ccoil_pose_t pose(const double *pos, double yAngle, double zAngle)
{
    ccoil_pose_t p;
    for (int i = 0; i < 3; ++i)
        p.position[i] = pos[i];
    p.y_axis_angle = yAngle;
    p.z_axis_angle = zAngle;
    return p;
}

template <typename Result>
void coilPairs(long long configCount, long long pointCount, const CoilPairArgumentsData *pair,
               const CoilPairPositionData *configArr, Result *resArr, int quantity, const char *where)
{
    if (configCount < 0 || !pair || (configCount > 0 && !configArr))
        raise(where, "negative configuration count or null argument");
    const CoilPairArgumentsData &d = *pair;
    checkCount(d.primAngularIncrements, "primAngularIncrements", where);
    checkCount(d.primThicknessIncrements, "primThicknessIncrements", where);
    checkCosines(d.primCosPrecomputeArray, d.primAngularWeightArray, d.primAngularIncrements,
                 "the primary's angular table", where);
    checkLegendre(d.primThicknessPositionArray, d.primThicknessWeightArray, d.primThicknessIncrements,
                  "the primary's thickness table", where);
    const Coil sec = secondaryCoil(d.secInnerRadius, d.secThickness, d.secLength, d.secAngularIncrements,
                                   d.secThicknessIncrements, d.secLengthIncrements, where);
    checkLegendre(d.secAngularPositionArray, d.secAngularWeightArray, d.secAngularIncrements,
                  "the secondary's angular table", where);
    checkLegendre(d.secThicknessPositionArray, d.secThicknessWeightArray, d.secThicknessIncrements,
                  "the secondary's thickness table", where);
    checkLegendre(d.secLengthPositionArray, d.secLengthWeightArray, d.secLengthIncrements,
                  "the secondary's length table", where);
    if (pointCount != (long long)d.secAngularIncrements * d.secThicknessIncrements * d.secLengthIncrements)
        raise(where, "pointCount must be the secondary's node count");
    if (!(d.primInnerRadius > 0.0) || !(d.primThickness > 0.0) || !(d.primLength > 0.0))
        raise(where, "primary inner radius, thickness and length must be positive");
    if (configCount == 0)
        return;
    Coil prim{};
    prim.inner_radius = d.primInnerRadius;
    prim.thickness = d.primThickness;
    prim.length = d.primLength;
    prim.use_fast_method = d.useFastMethod ? 1 : 0;
    prim.current_density = currentDensity(d.constFactor, d.primThickness, d.primLength, d.useFastMethod);
    prim.current = 1.0;  // the glue's correctionFactor already holds 1 / I1 where it applies
    prim.num_turns = 1;
    prim.coil_type = d.useFastMethod ? kRectangular : kFlat;
    prim.transform[0] = prim.transform[4] = prim.transform[8] = 1.0;
    prim.inverse_transform[0] = prim.inverse_transform[4] = prim.inverse_transform[8] = 1.0;
    prim.precision = singleBlock(d.primAngularIncrements, d.primThicknessIncrements, 1);
    std::vector<ccoil_pose_t> pp, sp;
    pp.reserve((size_t)configCount);
    sp.reserve((size_t)configCount);
    for (long long i = 0; i < configCount; ++i)
    {
        const CoilPairPositionData &c = configArr[i];
        pp.push_back(pose(c.primPositionVector, c.primAlphaAngle, c.primBetaAngle));
        sp.push_back(pose(c.secPositionVector, c.secAlphaAngle, c.secBetaAngle));
    }
    constexpr int width = sizeof(Result) / sizeof(double);
    std::vector<double> discard;
    double *out = reinterpret_cast<double *>(resArr);
    if (!out)
    {
        discard.resize((size_t)configCount * width);
        out = discard.data();
    }
    pairs(&prim, 1, sec, &pp, sp, quantity, d.correctionFactor, out, where);
}

template <typename Result>
void groupPairs(long long coilCount, long long configCount, long long pointCount, const SecondaryCoilData &s,
                const CoilData *coils, const SecondaryCoilPositionData *positions, Result *resArr, int quantity,
                const char *where)
{
    if (coilCount < 0 || coilCount > (1LL << 30) || configCount < 0 || (coilCount > 0 && !coils) ||
        (configCount > 0 && !positions))
        raise(where, "negative count or null argument");
    const Coil sec = secondaryCoil(s.innerRadius, s.thickness, s.length, s.angularIncrements, s.thicknessIncrements,
                                   s.lengthIncrements, where);
    checkLegendre(s.angularPositionArray, s.angularWeightArray, s.angularIncrements, "the secondary's angular table",
                  where);
    checkLegendre(s.thicknessPositionArray, s.thicknessWeightArray, s.thicknessIncrements,
                  "the secondary's thickness table", where);
    checkLegendre(s.lengthPositionArray, s.lengthWeightArray, s.lengthIncrements, "the secondary's length table",
                  where);
    if (pointCount != (long long)s.angularIncrements * s.thicknessIncrements * s.lengthIncrements)
        raise(where, "pointCount must be the secondary's node count");
    std::vector<Coil> prims;
    prims.reserve((size_t)coilCount);
    for (long long i = 0; i < coilCount; ++i)
    {
        Coil k = coilFromData(coils[i], where);
        // the group mutual-inductance kernel divides by each coil's current; the force kernel does not
        if (quantity == CCOIL_PAIR_FORCE_TORQUE)
            k.current = 1.0;
        else if (k.current == 0.0)
            raise(where, "coil " + std::to_string(i) + " has zero current (the mutual inductance divides by it)");
        prims.push_back(k);
    }
    if (configCount == 0)
        return;
    constexpr int width = sizeof(Result) / sizeof(double);
    std::vector<double> discard;
    double *out = reinterpret_cast<double *>(resArr);
    if (!out)
    {
        discard.resize((size_t)configCount * width);
        out = discard.data();
    }
    if (coilCount == 0)
    {
        for (size_t i = 0; i < (size_t)configCount * width; ++i)
            out[i] = 0.0;
        return;
    }
    std::vector<ccoil_pose_t> sp;
    sp.reserve((size_t)configCount);
    for (long long i = 0; i < configCount; ++i)
        sp.push_back(pose(positions[i].positionVector, positions[i].alphaAngle, positions[i].betaAngle));
    pairs(prims.data(), (int)coilCount, sec, nullptr, sp, quantity, s.correctionFactor, out, where);
}
} // namespace
} // namespace ccoil

using namespace ccoil;

void Calculate_hardware_accelerated_a(long long opCount, CoilData coil, const VectorData *posArr, VectorData *resArr)
{
    singleField(opCount, coil, posArr, resArr, CCOIL_FIELD_A, "Calculate_hardware_accelerated_a");
}

void Calculate_hardware_accelerated_b(long long opCount, CoilData coil, const VectorData *posArr, VectorData *resArr)
{
    singleField(opCount, coil, posArr, resArr, CCOIL_FIELD_B, "Calculate_hardware_accelerated_b");
}

void Calculate_hardware_accelerated_g(long long opCount, CoilData coil, const VectorData *posArr, MatrixData *resArr)
{
    singleField(opCount, coil, posArr, resArr, CCOIL_FIELD_G, "Calculate_hardware_accelerated_g");
}

void Calculate_mutual_inductance_configurations(long long configCount, long long pointCount,
                                                const CoilPairArgumentsData *coilPair,
                                                const CoilPairPositionData *configArr, double *inductanceArr)
{
    coilPairs(configCount, pointCount, coilPair, configArr, inductanceArr, CCOIL_PAIR_MUTUAL_INDUCTANCE,
              "Calculate_mutual_inductance_configurations");
}

void Calculate_force_and_torque_configurations(long long configCount, long long pointCount,
                                               const CoilPairArgumentsData *coilPair,
                                               const CoilPairPositionData *configArr, ForceTorqueData *forceTorqueArr)
{
    coilPairs(configCount, pointCount, coilPair, configArr, forceTorqueArr, CCOIL_PAIR_FORCE_TORQUE,
              "Calculate_force_and_torque_configurations");
}

void Calculate_hardware_accelerated_a_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, VectorData *resArr)
{
    groupField(coilCount, opCount, coilArr, posArr, resArr, CCOIL_FIELD_A, "Calculate_hardware_accelerated_a_group");
}

void Calculate_hardware_accelerated_b_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, VectorData *resArr)
{
    groupField(coilCount, opCount, coilArr, posArr, resArr, CCOIL_FIELD_B, "Calculate_hardware_accelerated_b_group");
}

void Calculate_hardware_accelerated_e_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, VectorData *resArr)
{
    groupField(coilCount, opCount, coilArr, posArr, resArr, CCOIL_FIELD_E, "Calculate_hardware_accelerated_e_group");
}

void Calculate_hardware_accelerated_g_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, MatrixData *resArr)
{
    groupField(coilCount, opCount, coilArr, posArr, resArr, CCOIL_FIELD_G, "Calculate_hardware_accelerated_g_group");
}

void Calculate_mutual_inductance_configurations_group(long long coilCount, long long configCount,
                                                      long long pointCount, SecondaryCoilData secondaryCoil,
                                                      const CoilData *coils,
                                                      const SecondaryCoilPositionData *secondaryPositions,
                                                      double *inductanceArr)
{
    groupPairs(coilCount, configCount, pointCount, secondaryCoil, coils, secondaryPositions, inductanceArr,
               CCOIL_PAIR_MUTUAL_INDUCTANCE, "Calculate_mutual_inductance_configurations_group");
}

void Calculate_force_and_torque_configurations_group(long long coilCount, long long configCount,
                                                     long long pointCount, SecondaryCoilData secondaryCoil,
                                                     const CoilData *coils,
                                                     const SecondaryCoilPositionData *secondaryPositions,
                                                     ForceTorqueData *forceTorqueArr)
{
    groupPairs(coilCount, configCount, pointCount, secondaryCoil, coils, secondaryPositions, forceTorqueArr,
               CCOIL_PAIR_FORCE_TORQUE, "Calculate_force_and_torque_configurations_group");
}
