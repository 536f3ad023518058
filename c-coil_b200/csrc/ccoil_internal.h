// Internal declarations shared by the host code and the CUDA kernels.
#ifndef CCOIL_INTERNAL_H
#define CCOIL_INTERNAL_H

#include "../../include/ccoil_gpu.h"

#include <cstdint>
#include <string>
#include <vector>

namespace ccoil
{
using Coil = ccoil_coil_t;
using PrecisionArgs = ccoil_precision_args_t;

constexpr int kMaxOrder = 100;   // Legendre::maxLegendreOrder
constexpr int kRectangular = 0, kThin = 1, kFlat = 2, kFilament = 3;

// ---------------------------------------------------------------------------
// Segment blobs.  A field evaluation is a list of segments; each segment is one
// coil's geometry plus a slice of its angular nodes and all of its thickness
// (and length) nodes, laid out contiguously so one bulk copy stages it in
// shared memory.  Segments are independent: the kernel converts each
// segment's cylindrical partial sums to Cartesian and adds them to the point's
// running total, so a coil whose node tables exceed one segment simply spans
// several segments.
// ---------------------------------------------------------------------------
constexpr int kSegmentBytes = 16384;  // staging buffer per pipeline stage
constexpr int kSegmentStages = 2;

struct alignas(16) SegmentHeader
{
    double position[3];
    double inv_transform[9];
    double transform[9];
    double half_length;   // b/2 (fast method)
    double field_factor;  // 2 pi f for E, 1 otherwise
    double inner_radius;  // R, for the on-axis test of the gradient
    double near_r2;       // FP32 path: squared near-field radius around the winding (in the coil frame)
    double near_lo[2];    // FP32 path: winding cross-section box {r_min, z_min} ...
    double near_hi[2];    // ... and {r_max, z_max}
    int n_t;              // thickness nodes
    int n_l;              // length nodes (slow method)
    int n_phi;            // angular nodes in this segment
    int fast;             // 1 = analytic length integral (RECTANGULAR/THIN)
    int off_t;            // table offsets in 16-byte units from the header start
    int off_l;
    int off_phi;
    int off_f32;          // FP32 tables (0 when absent)
};
static_assert(sizeof(SegmentHeader) % 16 == 0, "segment header must keep 16-byte alignment");

struct SegmentDesc
{
    long long offset;  // byte offset of the blob in the device buffer (multiple of 16)
    int bytes;         // multiple of 16, <= kSegmentBytes
    int coil;          // source coil index
};

// FP32 angular tables, appended after the FP64 tables (16 bytes per entry).
// One entry describes a mirror pair of nodes: node k of the first half of
// [0, pi] and node n-1-k (phi -> pi - phi), whose cosine is the exact negation.
// Every squared distance the integrands use is Q + b2 (1 - cos), so the second
// node's exceed the first's by the same delta = b2 (omcm - omc) = 2 b2 c.  The
// FP32 integrands form f(c) - f(-c) as delta times a cancellation-free
// expression and g(c) + g(-c) directly; the entry carries the weights of
// such terms, computed in FP64 from the FP32 values of omc and omcm (so that
// they match the distances the kernels form from them) and rounded once:
// w2c2 = w (omcm - omc)^2 / 2 = 2 w c^2, the weight of a difference divided by
// b2; wc = w (omcm - omc) / 2 = w c; ws2 = w omc omcm = w sin^2.  With an odd
// node count the middle node (c = 0) is an entry of its own with half its
// weight (evaluated twice, w2c2 = wc = 0).
struct alignas(16) PhiNode32
{
    float w2c2;  // w (omcm - omc)^2 / 2 (0 for the middle node)
    float omc;   // 1 - cos(phi_k) = 2 sin^2(phi_k / 2)
    float omcm;  // 1 - cos(phi_{n-1-k}) = 2 sin^2(phi_{n-1-k} / 2) (about 2 - omc)
    float w;     // w_phi (halved for the middle node)
    float wc;    // w (omcm - omc) / 2
    float ws2;   // w omc omcm
};

// Device layout of the FP32 angular table: two consecutive mirror pairs per
// 48-byte entry, every field a float2 {pair 2m, pair 2m + 1}, so the integrands
// evaluate both pairs with packed FP32 (f32x2) instructions.  A table with an
// odd pair count ends in an entry whose second pair has zero weights and the
// first pair's nodes (its values stay finite and add nothing).  The weights
// wc and ws2 save the integrands 2-5 packed instructions per entry, for one
// more 16-byte load.
struct alignas(16) PhiPair2
{
    float2 omc, omcm, w, w2c2, wc, ws2;
};
static_assert(sizeof(PhiPair2) == 48, "FP32 angular entries are 48 bytes");
void packPhiPairs2(const PhiNode32 *pairs, int count, std::vector<PhiPair2> &out);

// Node order of the FP64 angular table in FP32 mode: position j holds node
// j/2 (j even) or its mirror n-1-j/2 (j odd), so that any even-length slice of
// the table covers whole mirror pairs; with odd n the middle node comes last.
inline int pairOrderNode(int j, int n) { return (j & 1) ? n - 1 - (j >> 1) : (j >> 1); }

// Host-built device tables for a coil set.
struct SegmentSet
{
    std::vector<unsigned char> blob;  // host copy, 16-byte aligned entries
    std::vector<SegmentDesc> segs;
    int max_bytes = 0;
};

// Destination of the segment builder: the blob bytes, appended in order (every
// entry keeps 16-byte alignment), and one descriptor per finished segment.  A
// sink with fixed capacity returns false when full; overflowMessage() then
// names the limit that was reached.
struct SegmentSink
{
    virtual bool append(const void *p, size_t n) = 0;
    virtual size_t size() const = 0;
    virtual bool segment(const SegmentDesc &d) = 0;
    virtual std::string overflowMessage() const = 0;

  protected:
    ~SegmentSink() = default;
};

// Builds the segment list for `coils` (each at its own precision) for field
// evaluation; precision selects whether FP32 tables are appended.
bool buildFieldSegments(const Coil *coils, int count, int field, int precision, SegmentSet &out, std::string &err);
// The same layout written into any sink (the allocation-free entry point's
// fixed staging buffers use this form).
bool buildFieldSegments(const Coil *coils, int count, int field, int precision, SegmentSink &out, std::string &err);
// FP32 angular pair table of a coil at precision p: (n + 1) / 2 entries, entry i
// for nodes i and n-1-i of the FP64 table in its reference order
void buildPhiPairs32(const PrecisionArgs &p, std::vector<PhiNode32> &out);
// entry k (0 <= k < (n + 1) / 2) of that table
PhiNode32 phiPair32(const PrecisionArgs &p, int k);
// FP32 path's near-field box of a coil, into h.near_lo / near_hi / near_r2
void setNearBox(const Coil &k, SegmentHeader &h);

// host_coil.cpp
const double *legendreNodes(int order);
const double *legendreWeights(int order);
PrecisionArgs coilPrecision(const Coil &coil, double pf, int gpuCap);
void pairPrecision(const Coil &prim, const Coil &sec, double pf, int gpuCap, bool zAxis, bool pureGPU,
                   PrecisionArgs &primOut, PrecisionArgs &secOut);
void initCoil(double R, double a, double b, int N, double I, double f, const double pos[3], double yAngle,
              double zAngle, Coil &out);
bool validArgs(const PrecisionArgs &p);

// errors (thread-local message)
void setError(const std::string &msg);
int fail(int status, const std::string &msg);
int failMessage(int status, const char *msg);  // same, without building a std::string

// Device memory for the library's temporaries and plans, from a memory pool of
// the library's own (one per device, created on first use) that keeps up to
// 4 GiB of freed blocks for reuse: after the first calls, allocating and
// freeing costs no driver mapping work and no device-wide synchronisation.
// scratchAlloc/cudaFreeAsync are ordered on `st`.
cudaError_t scratchAlloc(void **p, size_t bytes, cudaStream_t st);

// kernels (fields.cu)
struct FieldLaunch
{
    const unsigned char *d_blob;
    const SegmentDesc *d_segs;
    int nseg;
    const double *d_points;
    long long npts;
    double *d_out;
    int field;
    int precision;
    int lanes;
    // FP32_COMPENSATED: near-field work list (scratch) and its counter
    void *d_work = nullptr;                 // NearPair[work_capacity] (8 bytes each)
    unsigned long long work_capacity = 0;
    unsigned long long *d_work_count = nullptr;
    int near_blocks = 0;                    // grid of the near-field pass
    // FP32_REFINED: every (point, segment) FP32 contribution whose norm exceeds
    // refine_fraction times the norm of the point's total is replaced by its
    // FP64 value; the FP32 pass stores the contributions in d_contrib
    // (nseg x npts x W doubles, scratch), the selection lists the pairs in the
    // work list (which then needs room for them) and counts them in
    // d_refined_total (not reset between calls)
    double refine_fraction = 0.0;
    double *d_contrib = nullptr;
    unsigned long long *d_refine_segs = nullptr;  // nseg counters (scratch)
    unsigned long long *d_refined_total = nullptr;
};
constexpr size_t kNearPairBytes = 8;
// default fraction of FP32_REFINED (ccoil_set_refine_fraction): on the 128-coil
// benchmark group it re-evaluates about 12 % of the (point, coil) pairs in FP64
// and brings the maximum relative error of A and B below 1e-7
constexpr double kDefaultRefineFraction = 0.1;
double refineFraction();  // the process-wide fraction (ccoil_set_refine_fraction)
// FP32_REFINED evaluates the points in chunks whose stored contributions fit
// this many bytes (the 128-coil benchmark group's A and B at 2^20 points take
// 3.8 GB: one chunk), and lists at most kRefineListPairs pairs per chunk (8
// bytes each; every pair of a chunk of A, B or E fits)
constexpr size_t kRefineContribBytes = size_t(1) << 32;
constexpr unsigned long long kRefineListPairs = 1ULL << 28;
int launchFields(const FieldLaunch &L, void *stream);
int readTimeouts(long long &count);

// Point ordering of the FP32 field plans (ordering.cu): sort the points along
// a Morton curve over their bounding box so that each warp's points lie close
// together, evaluate them in that order, scatter the results back.
// orderPoints writes the permutation (order[i] = caller's index of sorted
// point i) and the sorted points; scratch holds pointOrderScratchBytes(n).
constexpr long long kPointOrderMinPoints = 1LL << 14;
constexpr long long kPointOrderMaxPoints = 1LL << 30;
size_t pointOrderScratchBytes(long long n);
int orderPoints(const double *pts, long long n, void *scratch, size_t scratchBytes, int *order, double *sortedPts,
                void *stream);
int scatterResults(const double *sorted, const int *order, long long n, int width, double *out, void *stream);
int checkBoundedWait(long long limitCycles, void *stream);

// batched persistent launch (fields.cu, batch.cuh)
struct BatchLaunch
{
    const unsigned char *d_blob;
    const SegmentDesc *d_segs;
    const void *d_items;  // BatchItem[nitems]
    int nitems;
    unsigned *d_next;     // item counter (scratch)
    const double *d_points;
    double *d_outA, *d_outB, *d_outG;
    int precision;
    int grid;
    void *d_work = nullptr;
    unsigned long long work_capacity = 0;
    unsigned long long *d_work_count = nullptr;
};
constexpr size_t kBatchItemBytes = 32;

// pairs.cu: the arrangement evaluator behind ccoil_pair_arrangements_zaxis,
// with two options its C-ABI callers leave at their defaults: full_ring makes
// every arrangement integrate the whole secondary ring (the reference's GPU
// kernels never take the CPU path's half-ring rule for coplanar axes), and
// scale multiplies the result.
struct PairOptions
{
    bool full_ring = false;
    double scale = 1.0;
};
int pairArrangements(const ccoil_coil_t *primaries, int primary_count, const ccoil_coil_t *secondary,
                     const ccoil_precision_args_t *secondary_precisions, const ccoil_precision_args_t *zaxis_precisions,
                     const ccoil_pose_t *primary_poses, const ccoil_pose_t *secondary_poses, long long count,
                     int quantity, int precision, double *out, long long *z_axis_count, int memory, void *stream,
                     const PairOptions &opt);
int launchBatch(const BatchLaunch &B, void *stream);
int batchBlocksPerSM(int precision);
} // namespace ccoil

#endif
