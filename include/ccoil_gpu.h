/*
 * ccoil_gpu.h -- C-ABI of the B200 (sm_100a) field and coil-pair hot path of
 * C-Coil.  Plain C types only: pointers, sizes, enums and POD structs.
 *
 * The library (libccoil_b200.so) replaces the reference's CUDA entry points
 *   src/Coil/CUDAKernels/CoilAcceleration.h:8-29
 *   src/CoilGroup/CUDAKernels/CoilGroupAcceleration.h:7-37
 * and the host-side precision logic they depend on
 *   src/Coil/PrecisionArguments/PrecisionArguments.cxx:57-288
 *   src/Coil/PrecisionArguments/CoilPairArguments.cxx:20-255.
 *
 * Conventions
 *   - Every entry point returns ccoil_status_t (0 = success) and never exits
 *     the process.  ccoil_last_error_message() describes the last failure on
 *     the calling thread.
 *   - Points are interleaved xyz doubles (the memory layout of the reference's
 *     vec3::Vector3Array).  Vector outputs are xyz doubles per point; gradient
 *     outputs are 9 doubles per point in row-major order (xx xy xz yx ... zz),
 *     the layout of vec3::Matrix3.
 *   - `memory` says whether points/outputs are host pointers (the call copies
 *     them and returns after the result is back in host memory) or device
 *     pointers (the call is asynchronous on `stream`).  Coil descriptors are
 *     always host memory.
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *     stream).
 */
#ifndef CCOIL_GPU_H
#define CCOIL_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCOIL_ABI_VERSION 1

typedef enum ccoil_status
{
    CCOIL_OK = 0,
    CCOIL_ERR_INVALID_ARGUMENT = 1,
    CCOIL_ERR_CUDA = 2,
    CCOIL_ERR_OUT_OF_MEMORY = 3,
    CCOIL_ERR_NOT_SUPPORTED = 4,
    CCOIL_ERR_TIMEOUT = 5,
    CCOIL_ERR_NO_DEVICE = 6
} ccoil_status_t;

/* Arithmetic of the quadrature.  FP64 reproduces the reference's double CPU
 * path; FP32_COMPENSATED runs the bulk of the nodes in FP32 with compensated
 * accumulation and keeps FP64 for near-field points and the final sums;
 * FP32_REFINED (field plans, and mutual inductance and force/torque
 * arrangements) is FP32_COMPENSATED in which every (point, coil) contribution
 * (arrangements: every secondary node's contribution) whose norm exceeds a set
 * fraction of the norm of the total is replaced by its FP64 value
 * (ccoil_set_refine_fraction): where the contributions cancel, those that
 * dominate carry errors that the cancellation magnifies, and those are
 * re-evaluated. */
typedef enum ccoil_precision
{
    CCOIL_PRECISION_FP64 = 0,
    CCOIL_PRECISION_FP32_COMPENSATED = 1,
    CCOIL_PRECISION_FP32_REFINED = 2
} ccoil_precision_t;

typedef enum ccoil_field
{
    CCOIL_FIELD_A = 0, /* vector potential               (Coil::computeAllAPotentialVectors) */
    CCOIL_FIELD_B = 1, /* magnetic flux density          (Coil::computeAllBFieldVectors)     */
    CCOIL_FIELD_E = 2, /* electric field amplitude 2pi f A (Coil::computeAllEFieldVectors)   */
    CCOIL_FIELD_G = 3  /* B gradient, T*G as the reference (Coil::computeAllBGradientMatrices) */
} ccoil_field_t;

typedef enum ccoil_memory
{
    CCOIL_MEMORY_HOST = 0,
    CCOIL_MEMORY_DEVICE = 1
} ccoil_memory_t;

/* PrecisionArguments (src/Coil/Coil.h:47-94): blocks and Gauss-Legendre
 * increments per layer (angular = phi, thickness = a, length = b). */
typedef struct ccoil_precision_args
{
    int angular_blocks;
    int thickness_blocks;
    int length_blocks;
    int angular_increments;
    int thickness_increments;
    int length_increments;
} ccoil_precision_args_t;

/* One coil as the reference's Coil object holds it (src/Coil/Coil.h:152-196):
 * thin dimensions are already replaced by 1e-25*R (src/Coil/Coil.cxx:27-28),
 * current_density = I*N/(a*b), transform/inverse_transform are the row-major
 * matrices of Coil::calculateTransformationMatrices
 * (src/Coil/Utils/CalculateAttributes.cxx:65-78). */
typedef struct ccoil_coil
{
    double inner_radius;
    double thickness;
    double length;
    double current_density;
    double current;
    double sine_frequency;
    double position[3];
    double y_axis_angle;
    double z_axis_angle;
    double transform[9];
    double inverse_transform[9];
    int num_turns;
    int use_fast_method; /* RECTANGULAR/THIN: 1, FLAT/FILAMENT: 0 */
    int coil_type;       /* 0 RECTANGULAR, 1 THIN, 2 FLAT, 3 FILAMENT (src/Coil/EnumsAndConstants/CoilType.h) */
    ccoil_precision_args_t precision; /* precision used for this coil's fields */
} ccoil_coil_t;

/* Library identity. */
int ccoil_abi_version(void);
const char *ccoil_last_error_message(void);

/* ------------------------------------------------------------------------ *
 * Host-side mirrors of the reference's coil set-up and precision balancing  *
 * ------------------------------------------------------------------------ */

/* Coil::Coil(R, a, b, N, I, f, PrecisionFactor, threads, position, yAngle,
 * zAngle) (src/Coil/Coil.cxx:46-67): fills `out` including the CPU precision
 * arguments for precision_factor (gpu_increments == 0) or the GPU ones
 * (gpu_increments = the reference's GPU_INCREMENTS cap). */
int ccoil_coil_init(double inner_radius, double thickness, double length, int num_turns, double current,
                    double sine_frequency, const double position[3], double y_axis_angle, double z_axis_angle,
                    double precision_factor, int gpu_increments, ccoil_coil_t *out);

/* PrecisionArguments::getCoilPrecisionArguments{CPU,GPU}
 * (src/Coil/PrecisionArguments/PrecisionArguments.cxx:57-185);
 * gpu_increments == 0 selects the CPU variant. */
int ccoil_precision_arguments(const ccoil_coil_t *coil, double precision_factor, int gpu_increments,
                              ccoil_precision_args_t *out);

/* CoilPairArguments::getAppropriateCoilPairArguments
 * (src/Coil/PrecisionArguments/CoilPairArguments.cxx:49-255);
 * gpu_increments == 0 selects computeMethod != GPU. */
int ccoil_pair_arguments(const ccoil_coil_t *primary, const ccoil_coil_t *secondary, double precision_factor,
                         int gpu_increments, int z_axis_case, int pure_gpu, ccoil_precision_args_t *primary_out,
                         ccoil_precision_args_t *secondary_out);

/* Gauss-Legendre nodes and weights of order 1..100 in ascending node order
 * (the content of src/LegendreMatrix/LegendreMatrix.cxx, computed). */
int ccoil_legendre(int order, double *nodes, double *weights);

/* ------------------------------------------------------------------------ *
 * Fields of a coil or a coil group at many points                          *
 * ------------------------------------------------------------------------ */

/* Sum over `coil_count` coils of field `field` at `point_count` points, each
 * coil at its own `precision` arguments.  coil_count == 1 is the single-coil
 * path (Coil::computeAll*), coil_count > 1 the group path
 * (CoilGroup::computeAll*).  Replaces Calculate_hardware_accelerated_{a,b,g}
 * (src/Coil/CUDAKernels/CoilAcceleration.h:8-18) and
 * Calculate_hardware_accelerated_{a,b,e,g}_group
 * (src/CoilGroup/CUDAKernels/CoilGroupAcceleration.h:7-25). */
int ccoil_compute_fields(const ccoil_coil_t *coils, int coil_count, const double *points, long long point_count,
                         int field, int precision, double *out, int memory, void *stream);

/* A prepared coil set: node tables built and resident in device memory, so
 * repeated evaluations only move points and results.  Plans and one-shot calls
 * take their device memory from the library's stream-ordered pool on the
 * current device, which keeps up to 16 GiB of freed blocks mapped for reuse
 * until the process exits (an FP32_REFINED evaluation of 2^20 points of a
 * 128-coil group takes about 5 GB of scratch). */
typedef struct ccoil_field_plan ccoil_field_plan_t;

int ccoil_field_plan_create(const ccoil_coil_t *coils, int coil_count, int field, int precision,
                            ccoil_field_plan_t **plan);
/* lanes_per_point: 0 = automatic, else 1, 2, 4, 8, 16 or 32 threads share one point. */
int ccoil_field_plan_execute(ccoil_field_plan_t *plan, const double *points, long long point_count, double *out,
                             int memory, int lanes_per_point, void *stream);
int ccoil_field_plan_destroy(ccoil_field_plan_t *plan);
/* Number of segments (a coil's geometry with a slice of its node tables; a
 * coil whose tables exceed one staging buffer spans several) the plan
 * evaluates per point. */
int ccoil_field_plan_segment_count(const ccoil_field_plan_t *plan, int *count);

/* Point ordering of the FP32 plans (process-wide, read when a plan executes;
 * on by default): an FP32_COMPENSATED or FP32_REFINED plan given at least
 * 16,384 points (and at most 2^30) sorts them along a Morton curve over their
 * bounding box, evaluates them in that order and writes every result to the
 * caller's index.  Warps of nearby points agree more often on the integrands'
 * per-warp choices, which measured 4-8 % faster on points spread through a
 * volume.  The order is deterministic; results differ from unordered
 * evaluation only by FP32 rounding (within the mode's error).  The FP64 mode,
 * the batched plans and ccoil_fields_fp32c_static keep the caller's order. */
int ccoil_set_point_ordering(int enabled);
int ccoil_point_ordering(void);

/* FP32_REFINED's fraction (process-wide, read when a plan executes; finite,
 * >= 0; default 0.1): a (point, coil segment) pair is re-evaluated in FP64 when
 * the norm of its FP32 contribution exceeds `fraction` times the norm of the
 * point's total.  Smaller fractions refine more pairs; 0 refines every pair
 * with a non-zero contribution.  The plan stores every contribution of a chunk
 * of points (at most 4 GiB, plus a list of at most 2 GiB; larger calls run in
 * several chunks).  Points with
 * a non-finite total are not refined.  ccoil_field_plan_refined_pairs reports
 * how many pairs the plan's last execution re-evaluated (synchronous). */
int ccoil_set_refine_fraction(double fraction);
double ccoil_refine_fraction(void);
int ccoil_field_plan_refined_pairs(ccoil_field_plan_t *plan, long long *count);

/* ------------------------------------------------------------------------ *
 * Coil pairs over many arrangements                                         *
 * ------------------------------------------------------------------------ */

typedef enum ccoil_pair_quantity
{
    CCOIL_PAIR_MUTUAL_INDUCTANCE = 0, /* M, one double per arrangement */
    CCOIL_PAIR_FORCE_TORQUE = 1,      /* Fx Fy Fz Tx Ty Tz on the secondary, six doubles per arrangement */
    CCOIL_PAIR_MUTUAL_INDUCTANCE_GRADIENT = 2, /* dM/d(secondary position): the exact derivative of the M
                                                  quadrature (adjoint of M; no counterpart in the reference),
                                                  three doubles per arrangement */
    CCOIL_PAIR_MUTUAL_INDUCTANCE_PARAMETER_GRADIENT = 3 /* M and its exact derivatives with respect to both
                                                           coils' parameters (no counterpart in the reference),
                                                           14 doubles per arrangement:
                                                           M, dM/dR1, dM/da1, dM/db1, dM/dyAngle1, dM/dzAngle1,
                                                           dM/dR2, dM/da2, dM/db2, dM/dx2, dM/dy2, dM/dz2,
                                                           dM/dyAngle2, dM/dzAngle2 (1 = primary, 2 = secondary;
                                                           R inner radius, a thickness, b length).  The primary's
                                                           position gradient is -dM/d(x2, y2, z2) and
                                                           dM/dN = M / N for either coil.  One primary with
                                                           per-arrangement poses; FP64 or FP32_COMPENSATED. */
} ccoil_pair_quantity_t;

/* Position and orientation of a coil (Coil::setPositionAndOrientation,
 * src/Coil/Coil.cxx:245-252). */
typedef struct ccoil_pose
{
    double position[3];
    double y_axis_angle;
    double z_axis_angle;
} ccoil_pose_t;

/* Mutual inductance or force/torque of the secondary with `primary_count`
 * primaries, for `count` arrangements, with the reference's CPU general-case
 * algorithm (Coil::calculateMutualInductanceGeneral,
 * src/Coil/MInductance/CalculateMInductanceGeneral.cxx:8-117, and
 * Coil::calculateForceTorqueGeneral,
 * src/Coil/ForceAndTorque/CalculateForceGeneral.cxx:9-131, including the
 * half-ring rule for coplanar axes).  primaries[j].precision is the primary's
 * precision for pair j and secondary_precisions[j] the secondary's (as from
 * ccoil_pair_arguments).  With primary_poses (one per arrangement, exactly one
 * primary) both coils move: Coil::computeAll{MutualInductance,ForceTorque}Arrangements
 * (src/Coil/MInductance/ComputeMInductanceMethods.cxx:200-260).  With
 * primary_poses == NULL the primaries keep their own poses and are summed in
 * order: CoilGroup::computeAll*Arrangements
 * (src/CoilGroup/MInductance/ComputeMInductance.cxx:23-64).  Replaces
 * Calculate_mutual_inductance_configurations[_group] and
 * Calculate_force_and_torque_configurations[_group]
 * (src/Coil/CUDAKernels/CoilAcceleration.h:21-29,
 * src/CoilGroup/CUDAKernels/CoilGroupAcceleration.h:27-37).
 * (primary, arrangement) pairs that are exact z-axis cases (Coil::isZAxisCase)
 * are evaluated here with the general formula (ccoil_pair_arrangements_zaxis
 * uses the reference's z-axis formulas); their number is returned in
 * *z_axis_count.
 * precision: CCOIL_PRECISION_FP64 follows the reference's double arithmetic;
 * CCOIL_PRECISION_FP32_COMPENSATED (mutual inductance, force/torque and the
 * parameter gradient; CCOIL_ERR_NOT_SUPPORTED for the position gradient)
 * evaluates the primary's quadrature
 * in FP32 with compensated sums, except where a secondary node lies within the
 * primary's near-field box (winding cross-section inflated by 0.1 R), which
 * is evaluated in FP64; sums over secondary nodes and primaries are FP64.
 * CCOIL_PRECISION_FP32_REFINED (mutual inductance and force/torque) also
 * re-evaluates in FP64 every secondary node whose contribution exceeds the
 * refinement fraction of the arrangement's M (of its force or of its torque);
 * it keeps each warp's node contributions in up to 1 GiB of device scratch.
 * At fraction 0 every node is refined, so the FP32 pass is skipped: each node
 * is evaluated once in those FP64 forms (within about 1e-11 of
 * CCOIL_PRECISION_FP64, in about half its time). */
int ccoil_pair_arrangements(const ccoil_coil_t *primaries, int primary_count, const ccoil_coil_t *secondary,
                            const ccoil_precision_args_t *secondary_precisions, const ccoil_pose_t *primary_poses,
                            const ccoil_pose_t *secondary_poses, long long count, int quantity, int precision,
                            double *out, long long *z_axis_count, int memory, void *stream);

/* The same with the reference CPU path's per-pair dispatch for coaxial pairs
 * (Coil::computeMutualInductance, src/Coil/MInductance/ComputeMInductanceMethods.cxx:7-30;
 * Coil::computeForceTorque, src/Coil/ForceAndTorque/ComputeForceMethods.cxx:4-23):
 * a (primary, arrangement) pair that Coil::isZAxisCase accepts is evaluated
 * with the z-axis formulas (src/Coil/MInductance/CalculateMInductanceZAxis.cxx:17-232,
 * src/Coil/ForceAndTorque/CalculateForceZAxis.cxx:16-219) at the z-axis pair
 * arguments zaxis_precisions[2j] (primary) and [2j+1] (secondary), as from
 * ccoil_pair_arguments(..., z_axis_case = 1, ...); its force is (0, 0, Fz)
 * and its torque zero.  Mutual inductance and force/torque only (the
 * gradients use the general formula); zaxis_precisions == NULL is
 * ccoil_pair_arrangements. */
int ccoil_pair_arrangements_zaxis(const ccoil_coil_t *primaries, int primary_count, const ccoil_coil_t *secondary,
                                  const ccoil_precision_args_t *secondary_precisions,
                                  const ccoil_precision_args_t *zaxis_precisions, const ccoil_pose_t *primary_poses,
                                  const ccoil_pose_t *secondary_poses, long long count, int quantity, int precision,
                                  double *out, long long *z_axis_count, int memory, void *stream);

/* Self inductance of `count` coils (Coil::computeAndSetSelfInductance,
 * src/Coil/MInductance/ComputeMInductanceMethods.cxx:55-81):
 * pair_precisions[2c] and [2c+1] are the coil's pair arguments with itself in
 * the z-axis case (ccoil_pair_arguments(&coil, &coil, pf, 0, 1, 0, ...)).
 * RECTANGULAR and THIN coils use the closed form of Coil::calculateSelfInductance
 * (src/Coil/MInductance/CalculateMInductanceZAxis.cxx:233-319), FLAT coils the
 * coaxial mutual inductance of the centred coil with itself; a FILAMENT is
 * rejected (CCOIL_ERR_INVALID_ARGUMENT: the integral diverges).  out: host
 * array of count doubles; synchronous on `stream`. */
int ccoil_self_inductances(const ccoil_coil_t *coils, const ccoil_precision_args_t *pair_precisions, int count,
                           double *out, void *stream);

/* ------------------------------------------------------------------------ *
 * Batched independent systems                                               *
 * ------------------------------------------------------------------------ */

/* Many independent coil systems (each what the reference evaluates with one
 * CoilGroup::computeAll*(points, GPU), src/CoilGroup/Fields/CalculateFieldsGPU.cxx:11-196)
 * evaluated by one persistent launch, replayed from a captured CUDA graph.
 * System s owns coils [system_coil_offsets[s], system_coil_offsets[s+1]) and
 * points [system_point_offsets[s], system_point_offsets[s+1]) of the flat
 * arrays; fields_mask combines 1<<CCOIL_FIELD_A, 1<<CCOIL_FIELD_B and
 * 1<<CCOIL_FIELD_G; every requested field is computed in the same launch. */
typedef struct ccoil_batch_plan ccoil_batch_plan_t;

int ccoil_batch_plan_create(const ccoil_coil_t *coils, const int *system_coil_offsets,
                            const long long *system_point_offsets, int system_count, int fields_mask, int precision,
                            ccoil_batch_plan_t **plan);
/* points, out_a/out_b/out_g: device pointers (outputs of unrequested fields may
 * be NULL); the first call with a given set of pointers captures the graph,
 * later calls replay it; ordered after and before `stream`. */
int ccoil_batch_plan_execute(ccoil_batch_plan_t *plan, const double *points, double *out_a, double *out_b,
                             double *out_g, void *stream);
/* Autotuner: times the batch with each candidate item split (the minimum number
 * of work items per system and field before more lanes per point stop being
 * added) and keeps the fastest; reports it and its time. */
int ccoil_batch_plan_tune(ccoil_batch_plan_t *plan, const double *points, double *out_a, double *out_b,
                          double *out_g, int *chosen_split, float *best_ms);
int ccoil_batch_plan_set_split(ccoil_batch_plan_t *plan, int split);
int ccoil_batch_plan_destroy(ccoil_batch_plan_t *plan);

/* ------------------------------------------------------------------------ *
 * Adjoint                                                                   *
 * ------------------------------------------------------------------------ */

/* Gradient of a loss L(B) with respect to each coil's parameters, given
 * grad_b = dL/dB at the points (no counterpart in the reference, which has no
 * derivatives).  params: coil_count x 9 host doubles
 * {R, a, b, N*I, x, y, z, yAxisAngle, zAxisAngle} with the fixed precision
 * arguments `precisions` (host); points, grad_b (point_count x 3) and
 * grad_params (coil_count x 9) are device pointers.  Fast-method coils only
 * (RECTANGULAR, THIN); FP64; deterministic. */
int ccoil_b_field_adjoint(const double *params, const ccoil_precision_args_t *precisions, int coil_count,
                          const double *points, long long point_count, const double *grad_b, double *grad_params,
                          void *stream);

/* Number of device-side wait timeouts seen since the library was loaded (the
 * bounded waits of the staging pipeline; a non-zero value also makes the
 * failing call return CCOIL_ERR_TIMEOUT). */
long long ccoil_timeout_count(void);

/* Failure-path checks, no counterpart in the reference (whose CUDA error path
 * ends the process, src/CUDAUtils/ErrorCheck/ErrorCheck.cu:15).
 * ccoil_check_bounded_wait runs the staging pipeline's bounded mbarrier wait on
 * a barrier that nothing completes, for at most limit_cycles GPU clock cycles
 * (<= 4e9, about 2 s): it returns CCOIL_ERR_TIMEOUT, counts the timeout in
 * ccoil_timeout_count(), and leaves the context usable.  Synchronous on
 * `stream`.
 * ccoil_inject_allocation_failures makes the next `count` device allocations
 * of the library's memory pool fail (as out of memory), so a caller can check
 * that its calls return CCOIL_ERR_OUT_OF_MEMORY and that later calls work;
 * count = 0 clears it. */
int ccoil_check_bounded_wait(long long limit_cycles, void *stream);
int ccoil_inject_allocation_failures(int count);

/* FP32_COMPENSATED field evaluation that allocates nothing.  No counterpart in
 * the reference.  For callers that cannot allocate device memory: plugins
 * inside a host program that owns every device allocation (and budgets the
 * device memory itself), real-time loops that must not stall on an
 * allocation.
 * Same arguments as ccoil_compute_fields with precision FP32_COMPENSATED,
 * except that `points` and `out` must be device pointers and the call is
 * asynchronous on `stream`; the same results up to 16,383 points (from 16,384
 * on, ccoil_compute_fields evaluates the points in Morton order, see
 * ccoil_set_point_ordering, and the two differ by FP32 rounding; this entry
 * point keeps the caller's order).
 *
 * Its scratch (node tables, segment list, near-field work list) is one fixed
 * 3 MiB array in device memory, held by every GPU that loads the library until
 * the process exits.  Limits: at most 1 MiB of node tables (about 400 coils at
 * PrecisionFactor 5), 8192 segments and 2^31-1 points; larger requests return
 * CCOIL_ERR_INVALID_ARGUMENT with a message.  A call on a stream that is being
 * captured returns CCOIL_ERR_NOT_SUPPORTED: every call stages the node tables
 * through one shared host buffer, which a graph replay would read after later
 * calls had overwritten it.  The first call on a device looks up the array's
 * device address and keeps it for the life of the process, so
 * cudaDeviceReset is not supported while the library is in use.  All calls
 * share the array: calls that overlap on the GPU (other streams or host
 * threads) race and must be ordered by the caller. */
int ccoil_fields_fp32c_static(const ccoil_coil_t *coils, int coil_count, const double *points,
                              long long point_count, int field, double *out, void *stream);

/* Diagnostic with no counterpart in the reference: measured throughput of the
 * pipes that bound the field kernels on the current device -- FP64 FMA and
 * FP32 FMA (TFLOP/s, an FMA counted as 2 flops) and MUFU reciprocal square
 * root (tera-ops/s).  Used as roofline denominators. */
int ccoil_measure_pipe_peaks(double *fp64_tflops, double *fp32_tflops, double *mufu_tops);

/* Diagnostic with no counterpart in the reference: measured rates (operations
 * per second, whole device) of rates[0] FP64-pipe instructions (FMA),
 * rates[1] __ddiv_rn, rates[2] __dsqrt_rn, rates[3] the FP64 integrands'
 * logarithm (see ccoil_eval_log64),
 * rates[4] FP32 FMA instructions, rates[5] MUFU reciprocal square root and,
 * when count >= 7, rates[6] packed FP32 FMA instructions (fma.rn.f32x2, two
 * FMAs each).  count must be >= 6.  The roofline model of the field kernels charges each
 * divide, square root and logarithm rates[0] / rates[k] FP64-pipe slots. */
int ccoil_measure_op_rates(double *rates, int count);

/* Diagnostic with no counterpart in the reference: evaluates the natural
 * logarithm that the FP64 vector-potential integrand uses (Cody-Waite range
 * reduction and the atanh series, within about 1 ulp) at n points, for checks
 * against other implementations.  x and out are device pointers of n doubles;
 * every x must be positive, normal and finite.  Synchronous on `stream`. */
int ccoil_eval_log64(const double *x, double *out, long long n, void *stream);

/* Diagnostic with no counterpart in the reference: the FP64 forms that the
 * FP32_REFINED refinement pass and the FP64 nodes of the FP32 arrangement
 * kernels use (FP64 estimates refined by Newton-Raphson steps), at n points,
 * for checks against other implementations.  op 0: out[i] = 1 / sqrt(a[i]);
 * 1: sqrt(a[i]); 2: a[i] / b[i]; 3: log(a[i] / b[i]) (b unused and may be NULL
 * for ops 0 and 1).  All pointers are device pointers of n doubles; a (ops 0,
 * 1) and b (op 2) must lie in [1e-36, 1e36], a in op 2 be finite, a and b in
 * op 3 be positive, normal and finite.  Synchronous on `stream`. */
int ccoil_eval_fp64_op(int op, const double *a, const double *b, double *out, long long n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CCOIL_GPU_H */
