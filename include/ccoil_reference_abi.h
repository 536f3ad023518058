/*
 * ccoil_reference_abi.h -- the reference's own GPU entry points, exported by
 * libccoil_b200.so with their C++ signatures, so that the reference's host glue
 * links against this library unchanged (no .cu files of the reference are
 * compiled).
 *
 * The reference declares these functions in
 *   src/Coil/CUDAKernels/CoilAcceleration.h:8-29
 *   src/CoilGroup/CUDAKernels/CoilGroupAcceleration.h:7-37
 * over the structs of src/CUDAUtils/ConstantsAndStructs/CoilDataStructs.h:5-255.
 * Those structs hold TYPE fields; this library implements the TYPE=double
 * layout with GPU_INCREMENTS = CCOIL_REFERENCE_GPU_INCREMENTS (80, the
 * reference's CMake default), so the glue must be built with -DTYPE=double and
 * that GPU_INCREMENTS.  The struct definitions below reproduce that layout
 * member for member (the reference's default constructors aside, which do not
 * change it); a translation unit that already included the reference's
 * CoilDataStructs.h gets a size check instead.
 *
 * Semantics: each function evaluates the quadrature that the reference's
 * kernel of the same name defines on the tables it is given (the caller's
 * node counts, constant factors and correction factors), in FP64, and returns
 * after the results are in the host arrays -- as the reference's functions
 * do.  Differences from the reference's kernels, all deliberate:
 *   - results come from this library's FP64 kernels, which follow the
 *     reference's CPU integrands (src/Coil/Fields/CalculateFieldsFast.cxx,
 *     CalculateFieldsSlow.cxx) operation for operation; the reference's kernels
 *     use single-block tables with the same integrands, so on the same tables
 *     the two agree to rounding;
 *   - the gradient's on-axis branch applies where r / R < 1e-12, as on the CPU
 *     (src/Coil/Fields/CalculateFieldsMethods.cxx:60), not r / R <= 1e-5 as in
 *     src/Coil/CUDAKernels/FieldG.cu;
 *   - arrangement sums are reduced in a fixed order (no atomics), so results
 *     are reproducible run to run;
 *   - a failure throws std::runtime_error with the library's message instead
 *     of ending the process (src/CUDAUtils/ErrorCheck/ErrorCheck.cu:15).
 * Host-side quirks of the reference's glue (the force path's correction
 * factor 2 pi N2 / I1 at coil level, the halved PrecisionFactor of the group
 * arrangement paths, the GPU_INCREMENTS cap) live in the glue, before these
 * calls, and are therefore reproduced as they are.
 */
#ifndef CCOIL_REFERENCE_ABI_H
#define CCOIL_REFERENCE_ABI_H

#ifdef __cplusplus

#ifndef CCOIL_REFERENCE_GPU_INCREMENTS
#define CCOIL_REFERENCE_GPU_INCREMENTS 80
#endif

#ifndef GENERAL_COIL_PROGRAM_COILDATA_H
#define GENERAL_COIL_PROGRAM_COILDATA_H

/* One coil's tables as Coil::generateCoilData (src/Coil/Utils/SupportFunctions.cxx:167-223)
 * and CoilGroup::generateCoilDataArray (src/CoilGroup/Utils/GPUArgumentGeneration.cxx:17-95)
 * fill them. */
struct CoilData
{
    double constFactor;
    double current;
    double frequency;
    bool useFastMethod;
    double innerRadius;
    double thickness;
    double length;
    int angularIncrements;
    int lengthIncrements;
    int thicknessIncrements;
    double thicknessPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double thicknessWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double cosPrecomputeArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double angularWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double positionVector[3];
    double transformArray[9];
    double invTransformArray[9];
};

struct VectorData
{
    double x, y, z;
};

struct MatrixData
{
    double xx, xy, xz, yx, yy, yz, zx, zy, zz;
};

struct ForceTorqueData
{
    double forceX, forceY, forceZ;
    double torqueX, torqueY, torqueZ;
};

/* The secondary of a group arrangement (CoilGroup::generateSecondaryData,
 * src/CoilGroup/Utils/GPUArgumentGeneration.cxx:98-135). */
struct SecondaryCoilData
{
    double innerRadius;
    double thickness;
    double length;
    double correctionFactor;
    int angularIncrements;
    int lengthIncrements;
    int thicknessIncrements;
    double angularPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double angularWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double thicknessPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double thicknessWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double lengthPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double lengthWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
};

struct SecondaryCoilPositionData
{
    double positionVector[3];
    double alphaAngle;
    double betaAngle;
};

struct CoilPairPositionData
{
    double primPositionVector[3];
    double primAlphaAngle;
    double primBetaAngle;
    double secPositionVector[3];
    double secAlphaAngle;
    double secBetaAngle;
};

/* A coil pair's tables as Coil::generateCoilPairArgumentsData
 * (src/Coil/Utils/SupportFunctions.cxx:226-300) fills them. */
struct CoilPairArgumentsData
{
    double constFactor;
    double correctionFactor;
    bool useFastMethod;
    double primInnerRadius;
    double primThickness;
    double primLength;
    int primAngularIncrements;
    int primLengthIncrements;
    int primThicknessIncrements;
    double secInnerRadius;
    double secThickness;
    double secLength;
    int secAngularIncrements;
    int secLengthIncrements;
    int secThicknessIncrements;
    double primThicknessPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double primThicknessWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double primCosPrecomputeArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double primAngularWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double secAngularPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double secAngularWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double secThicknessPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double secThicknessWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double secLengthPositionArray[CCOIL_REFERENCE_GPU_INCREMENTS];
    double secLengthWeightArray[CCOIL_REFERENCE_GPU_INCREMENTS];
};
#endif /* GENERAL_COIL_PROGRAM_COILDATA_H */

/* The TYPE=double layout at CCOIL_REFERENCE_GPU_INCREMENTS: 4 tables of doubles
 * and 30 eight-byte slots (6 doubles, the bool padded to 8 bytes, the 3 ints
 * padded to 16, 21 position and matrix entries). */
static_assert(sizeof(CoilData) == (4 * CCOIL_REFERENCE_GPU_INCREMENTS + 30) * 8,
              "CoilData must have the reference's TYPE=double layout");
static_assert(sizeof(VectorData) == 24 && sizeof(MatrixData) == 72 && sizeof(ForceTorqueData) == 48,
              "result structs must have the reference's TYPE=double layout");

/* Coil-level entry points (src/Coil/CUDAKernels/CoilAcceleration.h:8-29).
 * Fields of one coil at opCount points; resArr == nullptr evaluates without
 * copying back, as the reference does. */
void Calculate_hardware_accelerated_a(long long opCount, CoilData coil, const VectorData *posArr,
                                      VectorData *resArr = nullptr);
void Calculate_hardware_accelerated_b(long long opCount, CoilData coil, const VectorData *posArr,
                                      VectorData *resArr = nullptr);
void Calculate_hardware_accelerated_g(long long opCount, CoilData coil, const VectorData *posArr,
                                      MatrixData *resArr = nullptr);
/* Mutual inductance (force/torque) of the pair for configCount arrangements of
 * both coils; pointCount is the secondary's node count (length x thickness x
 * angular increments) and must agree with the pair's tables. */
void Calculate_mutual_inductance_configurations(long long configCount, long long pointCount,
                                                const CoilPairArgumentsData *coilPair,
                                                const CoilPairPositionData *configArr, double *inductanceArr = nullptr);
void Calculate_force_and_torque_configurations(long long configCount, long long pointCount,
                                               const CoilPairArgumentsData *coilPair,
                                               const CoilPairPositionData *configArr,
                                               ForceTorqueData *forceTorqueArr = nullptr);

/* Group entry points (src/CoilGroup/CUDAKernels/CoilGroupAcceleration.h:7-37).
 * Sums over coilCount coils; E is 2 pi f A per coil. */
void Calculate_hardware_accelerated_a_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, VectorData *resArr = nullptr);
void Calculate_hardware_accelerated_b_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, VectorData *resArr = nullptr);
void Calculate_hardware_accelerated_e_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, VectorData *resArr = nullptr);
void Calculate_hardware_accelerated_g_group(long long coilCount, long long opCount, const CoilData *coilArr,
                                            const VectorData *posArr, MatrixData *resArr = nullptr);
/* The secondary at configCount positions against the coilCount coils at their
 * own positions (the group without the secondary). */
void Calculate_mutual_inductance_configurations_group(long long coilCount, long long configCount,
                                                      long long pointCount, SecondaryCoilData secondaryCoil,
                                                      const CoilData *coils,
                                                      const SecondaryCoilPositionData *secondaryPositions,
                                                      double *inductanceArr = nullptr);
void Calculate_force_and_torque_configurations_group(long long coilCount, long long configCount,
                                                     long long pointCount, SecondaryCoilData secondaryCoil,
                                                     const CoilData *coils,
                                                     const SecondaryCoilPositionData *secondaryPositions,
                                                     ForceTorqueData *forceTorqueArr = nullptr);

#endif /* __cplusplus */

#endif /* CCOIL_REFERENCE_ABI_H */
