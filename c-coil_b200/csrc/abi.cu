// The C-ABI entry points (include/ccoil_gpu.h): argument checks, device
// buffers, host<->device staging and kernel dispatch.  Nothing here exits the
// process: every failure becomes a status code plus a thread-local message.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

namespace ccoil
{
namespace
{
// last error message of the calling thread (fixed storage: reporting an error
// never allocates)
thread_local char t_error[512] = "";

// Grow-only device buffer owned by a plan.
struct DeviceBuffer
{
    void *ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t n);
    void release()
    {
        if (ptr)
        {
            cudaDeviceSynchronize();
            cudaFreeAsync(ptr, nullptr);
            cudaStreamSynchronize(nullptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
};
} // namespace

void setError(const std::string &msg) { failMessage(CCOIL_OK, msg.c_str()); }

int fail(int status, const std::string &msg) { return failMessage(status, msg.c_str()); }

int failMessage(int status, const char *msg)
{
    std::snprintf(t_error, sizeof(t_error), "%s", msg ? msg : "");
    return status;
}

int cudaFail(cudaError_t e, const char *what)
{
    if (e == cudaErrorMemoryAllocation)
        return fail(CCOIL_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return fail(CCOIL_ERR_NO_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
    return fail(CCOIL_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace
{
std::mutex g_poolMutex;
constexpr int kMaxDevices = 64;
cudaMemPool_t g_pools[kMaxDevices] = {};
// allocations still to fail on purpose (ccoil_inject_allocation_failures)
std::atomic<int> g_failAllocations{0};
// FP32_REFINED: re-evaluate in FP64 every (point, segment) pair whose FP32
// contribution's norm exceeds this fraction of the norm of the point's total
std::atomic<double> g_refineFraction{kDefaultRefineFraction};
// device-side wait timeouts already reported to a caller
std::atomic<long long> g_timeoutsReported{0};
// FP32 plans sort their points along a Morton curve (ccoil_set_point_ordering)
std::atomic<int> g_pointOrdering{1};
} // namespace

cudaError_t scratchAlloc(void **p, size_t bytes, cudaStream_t st)
{
    for (int n = g_failAllocations.load(); n > 0;)
        if (g_failAllocations.compare_exchange_weak(n, n - 1))
            return cudaErrorMemoryAllocation;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= kMaxDevices)
        return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_poolMutex);
        if (!g_pools[dev])
        {
            cudaMemPoolProps props;
            std::memset(&props, 0, sizeof(props));
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&g_pools[dev], &props);
            if (e != cudaSuccess)
            {
                g_pools[dev] = nullptr;
                return e;
            }
            // freed blocks up to 16 GiB stay mapped for the next allocation: a
            // one-shot FP32_REFINED call frees and takes again ~5 GB of scratch
            // (with 4 GiB kept, the remapping made those calls 1.5x slower)
            unsigned long long keep = 1ULL << 34;
            e = cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess)
                return e;
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

namespace
{
// plan buffers: allocated and released in the order of the legacy default
// stream, which waits for all blocking streams; release waits for the device
// so that no kernel on any stream still reads the buffer
int DeviceBuffer::reserve(size_t n)
{
    if (n <= bytes)
        return CCOIL_OK;
    release();
    cudaError_t e = scratchAlloc(&ptr, n, nullptr);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess)
    {
        ptr = nullptr;
        return cudaFail(e, "device buffer");
    }
    bytes = n;
    return CCOIL_OK;
}

int autoLanes(long long npts)
{
    // enough threads to fill the 148 SMs several times over; below that, split
    // the angular nodes of each point across lanes
    const long long target = 148LL * 1024;
    int lanes = 1;
    while (lanes < 8 && npts * lanes < target)
        lanes *= 2;
    return lanes;
}

bool validLanes(int l) { return l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32; }
} // namespace
} // namespace ccoil

using namespace ccoil;

struct ccoil_field_plan
{
    int field = 0;
    int precision = 0;
    int coil_count = 0;
    SegmentSet set;
    DeviceBuffer blob, segs, points, out, work, workCount;
    DeviceBuffer contrib, refineSegs, refinedTotal;  // FP32_REFINED
    DeviceBuffer orderScratch, order, sortedPoints, sortedOut;  // point ordering
};

extern "C" {

int ccoil_abi_version(void) { return CCOIL_ABI_VERSION; }

const char *ccoil_last_error_message(void) { return t_error; }

int ccoil_coil_init(double inner_radius, double thickness, double length, int num_turns, double current,
                    double sine_frequency, const double position[3], double y_axis_angle, double z_axis_angle,
                    double precision_factor, int gpu_increments, ccoil_coil_t *out)
{
    if (!out)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "out is null");
    if (!(inner_radius > 0.0) || thickness < 0.0 || length < 0.0 || num_turns < 1 || gpu_increments < 0 ||
        gpu_increments > kMaxOrder)
        return fail(CCOIL_ERR_INVALID_ARGUMENT,
                    "coil needs inner_radius > 0, thickness >= 0, length >= 0, num_turns >= 1, "
                    "gpu_increments in [0, 100]");
    initCoil(inner_radius, thickness, length, num_turns, current, sine_frequency, position, y_axis_angle,
             z_axis_angle, *out);
    out->precision = coilPrecision(*out, precision_factor, gpu_increments);
    return CCOIL_OK;
}

int ccoil_precision_arguments(const ccoil_coil_t *coil, double precision_factor, int gpu_increments,
                              ccoil_precision_args_t *out)
{
    if (!coil || !out)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "null argument");
    if (gpu_increments < 0 || gpu_increments > kMaxOrder)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "gpu_increments must be in [0, 100]");
    *out = coilPrecision(*coil, precision_factor, gpu_increments);
    return CCOIL_OK;
}

int ccoil_pair_arguments(const ccoil_coil_t *primary, const ccoil_coil_t *secondary, double precision_factor,
                         int gpu_increments, int z_axis_case, int pure_gpu, ccoil_precision_args_t *primary_out,
                         ccoil_precision_args_t *secondary_out)
{
    if (!primary || !secondary || !primary_out || !secondary_out)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "null argument");
    if (gpu_increments < 0 || gpu_increments > kMaxOrder)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "gpu_increments must be in [0, 100]");
    pairPrecision(*primary, *secondary, precision_factor, gpu_increments, z_axis_case != 0, pure_gpu != 0,
                  *primary_out, *secondary_out);
    return CCOIL_OK;
}

int ccoil_legendre(int order, double *nodes, double *weights)
{
    if (order < 1 || order > kMaxOrder || !nodes || !weights)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "order must be in [1, 100] and buffers non-null");
    std::memcpy(nodes, legendreNodes(order), sizeof(double) * order);
    std::memcpy(weights, legendreWeights(order), sizeof(double) * order);
    return CCOIL_OK;
}

int ccoil_field_plan_create(const ccoil_coil_t *coils, int coil_count, int field, int precision,
                            ccoil_field_plan_t **plan)
{
    if (!plan)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "plan is null");
    *plan = nullptr;
    if (coil_count < 0 || (coil_count > 0 && !coils))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "coil_count < 0 or coils null");
    if (field < CCOIL_FIELD_A || field > CCOIL_FIELD_G)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "field must be A, B, E or G");
    if (precision != CCOIL_PRECISION_FP64 && precision != CCOIL_PRECISION_FP32_COMPENSATED &&
        precision != CCOIL_PRECISION_FP32_REFINED)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "precision must be FP64, FP32_COMPENSATED or FP32_REFINED");

    ccoil_field_plan *p = new (std::nothrow) ccoil_field_plan();
    if (!p)
        return fail(CCOIL_ERR_OUT_OF_MEMORY, "host allocation failed");
    p->field = field;
    p->precision = precision;
    p->coil_count = coil_count;
    std::string err;
    const int tables = precision == CCOIL_PRECISION_FP64 ? CCOIL_PRECISION_FP64 : CCOIL_PRECISION_FP32_COMPENSATED;
    if (!buildFieldSegments(coils, coil_count, field, tables, p->set, err))
    {
        delete p;
        return fail(CCOIL_ERR_INVALID_ARGUMENT, err);
    }
    if (!p->set.segs.empty())
    {
        int rc = p->blob.reserve(p->set.blob.size());
        if (rc == CCOIL_OK)
            rc = p->segs.reserve(sizeof(SegmentDesc) * p->set.segs.size());
        if (rc != CCOIL_OK)
        {
            ccoil_field_plan_destroy(p);
            return rc;
        }
        cudaError_t e = cudaMemcpy(p->blob.ptr, p->set.blob.data(), p->set.blob.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(p->segs.ptr, p->set.segs.data(), sizeof(SegmentDesc) * p->set.segs.size(),
                           cudaMemcpyHostToDevice);
        if (e != cudaSuccess)
        {
            ccoil_field_plan_destroy(p);
            return cudaFail(e, "cudaMemcpy");
        }
    }
    *plan = p;
    return CCOIL_OK;
}

int ccoil_field_plan_execute(ccoil_field_plan_t *plan, const double *points, long long point_count, double *out,
                             int memory, int lanes_per_point, void *stream)
{
    if (!plan)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "plan is null");
    if (point_count < 0 || (point_count > 0 && (!points || !out)))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "point_count < 0 or null points/out");
    if (memory != CCOIL_MEMORY_HOST && memory != CCOIL_MEMORY_DEVICE)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "memory must be HOST or DEVICE");
    if (lanes_per_point != 0 && !validLanes(lanes_per_point))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "lanes_per_point must be 0, 1, 2, 4, 8, 16 or 32");
    if (point_count == 0)
        return CCOIL_OK;
    // grid.x limit: 2^31-1 CTAs of 128/lanes points
    if (point_count > (1LL << 36))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "point_count above 2^36");

    const int width = plan->field == CCOIL_FIELD_G ? 9 : 3;
    const size_t inBytes = sizeof(double) * 3 * (size_t)point_count;
    const size_t outBytes = sizeof(double) * width * (size_t)point_count;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    const double *dPoints = points;
    double *dOut = out;
    if (memory == CCOIL_MEMORY_HOST)
    {
        int rc = plan->points.reserve(inBytes);
        if (rc == CCOIL_OK)
            rc = plan->out.reserve(outBytes);
        if (rc != CCOIL_OK)
            return rc;
        cudaError_t e = cudaMemcpyAsync(plan->points.ptr, points, inBytes, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess)
            return cudaFail(e, "host->device copy of points");
        dPoints = static_cast<const double *>(plan->points.ptr);
        dOut = static_cast<double *>(plan->out.ptr);
    }

    FieldLaunch L;
    L.d_blob = static_cast<const unsigned char *>(plan->blob.ptr);
    L.d_segs = static_cast<const SegmentDesc *>(plan->segs.ptr);
    L.nseg = (int)plan->set.segs.size();
    L.d_points = dPoints;
    L.npts = point_count;
    L.d_out = dOut;
    L.field = plan->field;
    L.precision = plan->precision;
    L.lanes = lanes_per_point ? lanes_per_point : autoLanes(point_count);
    // FP32_REFINED runs in chunks of points whose stored contributions fit
    // kRefineContribBytes and whose pairs fit a list of kRefineListPairs
    const bool refined = plan->precision == CCOIL_PRECISION_FP32_REFINED && L.nseg > 0;
    long long chunk = point_count;
    if (refined)
    {
        const size_t perPoint = (size_t)L.nseg * (size_t)width * sizeof(double);
        long long maxChunk = (long long)(kRefineContribBytes / perPoint);
        const long long byList = (long long)(kRefineListPairs / (unsigned long long)L.nseg);
        maxChunk = std::max(1LL, std::min(maxChunk, byList));
        const long long chunks = (point_count + maxChunk - 1) / maxChunk;
        chunk = (point_count + chunks - 1) / chunks;
        if (L.lanes > 8)
            L.lanes = 8;  // the refining kernel is compiled for 1 to 8 lanes per point
    }
    if (plan->precision == CCOIL_PRECISION_FP32_COMPENSATED || plan->precision == CCOIL_PRECISION_FP32_REFINED)
    {
        // near-field work list: room for every (point, segment) pair up to 4 Mi
        // entries (32 MiB; FP32_REFINED: every pair of a chunk, up to
        // kRefineListPairs); near-field pairs beyond it are integrated in FP64 in
        // place
        unsigned long long want = (unsigned long long)chunk * (unsigned long long)L.nseg;
        const unsigned long long limit = refined ? kRefineListPairs : (1ULL << 22);
        unsigned long long cap = want < limit ? want : limit;
        if (cap == 0)
            cap = 1;
        int rc0 = plan->work.reserve(cap * kNearPairBytes);
        if (rc0 == CCOIL_OK)
            rc0 = plan->workCount.reserve(sizeof(unsigned long long));
        if (rc0 != CCOIL_OK)
            return rc0;
        L.d_work = plan->work.ptr;
        L.work_capacity = plan->work.bytes / kNearPairBytes;
        L.d_work_count = static_cast<unsigned long long *>(plan->workCount.ptr);
        L.near_blocks = 148 * 8;
    }
    if (refined)
    {
        int rc0 = plan->contrib.reserve((size_t)chunk * (size_t)L.nseg * (size_t)width * sizeof(double));
        if (rc0 == CCOIL_OK)
            rc0 = plan->refineSegs.reserve(sizeof(unsigned long long) * (size_t)L.nseg);
        if (rc0 == CCOIL_OK)
            rc0 = plan->refinedTotal.reserve(sizeof(unsigned long long));
        if (rc0 != CCOIL_OK)
            return rc0;
        cudaError_t e = cudaMemsetAsync(plan->refinedTotal.ptr, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess)
            return cudaFail(e, "refinement count");
        L.refine_fraction = g_refineFraction.load();
        L.d_contrib = static_cast<double *>(plan->contrib.ptr);
        L.d_refine_segs = static_cast<unsigned long long *>(plan->refineSegs.ptr);
        L.d_refined_total = static_cast<unsigned long long *>(plan->refinedTotal.ptr);
    }
    // FP32 modes: evaluate the points in Morton order (ordering.cu)
    const bool ordered = g_pointOrdering.load() != 0 && plan->precision != CCOIL_PRECISION_FP64 &&
                         point_count >= kPointOrderMinPoints && point_count <= kPointOrderMaxPoints;
    if (ordered)
    {
        const size_t scratch = pointOrderScratchBytes(point_count);
        int rc0 = plan->orderScratch.reserve(scratch);
        if (rc0 == CCOIL_OK)
            rc0 = plan->order.reserve(sizeof(int) * (size_t)point_count);
        if (rc0 == CCOIL_OK)
            rc0 = plan->sortedPoints.reserve(inBytes);
        if (rc0 == CCOIL_OK)
            rc0 = plan->sortedOut.reserve(outBytes);
        if (rc0 == CCOIL_OK)
            rc0 = orderPoints(dPoints, point_count, plan->orderScratch.ptr, plan->orderScratch.bytes,
                              static_cast<int *>(plan->order.ptr), static_cast<double *>(plan->sortedPoints.ptr),
                              stream);
        if (rc0 != CCOIL_OK)
            return rc0;
        L.d_points = static_cast<const double *>(plan->sortedPoints.ptr);
        L.d_out = static_cast<double *>(plan->sortedOut.ptr);
    }
    int rc = CCOIL_OK;
    for (long long off = 0; off < point_count && rc == CCOIL_OK; off += chunk)
    {
        FieldLaunch C = L;
        C.d_points = L.d_points + 3 * off;
        C.d_out = L.d_out + (long long)width * off;
        C.npts = std::min(chunk, point_count - off);
        rc = launchFields(C, stream);
    }
    if (rc == CCOIL_OK && ordered)
        rc = scatterResults(static_cast<const double *>(plan->sortedOut.ptr), static_cast<const int *>(plan->order.ptr),
                            point_count, width, dOut, stream);
    if (rc != CCOIL_OK)
        return rc;

    if (memory == CCOIL_MEMORY_HOST)
    {
        cudaError_t e = cudaMemcpyAsync(out, dOut, outBytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            return cudaFail(e, "field evaluation");
        long long timeouts = 0;
        rc = readTimeouts(timeouts);
        if (rc != CCOIL_OK)
            return rc;
        if (timeouts > g_timeoutsReported.load())
        {
            g_timeoutsReported.store(timeouts);
            return fail(CCOIL_ERR_TIMEOUT, "a staging wait in the field kernel timed out");
        }
    }
    return CCOIL_OK;
}

int ccoil_field_plan_segment_count(const ccoil_field_plan_t *plan, int *count)
{
    if (!plan || !count)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "null plan or count");
    *count = (int)plan->set.segs.size();
    return CCOIL_OK;
}

int ccoil_field_plan_destroy(ccoil_field_plan_t *plan)
{
    if (!plan)
        return CCOIL_OK;
    plan->blob.release();
    plan->segs.release();
    plan->points.release();
    plan->out.release();
    plan->work.release();
    plan->workCount.release();
    plan->contrib.release();
    plan->refineSegs.release();
    plan->refinedTotal.release();
    plan->orderScratch.release();
    plan->order.release();
    plan->sortedPoints.release();
    plan->sortedOut.release();
    delete plan;
    return CCOIL_OK;
}

int ccoil_compute_fields(const ccoil_coil_t *coils, int coil_count, const double *points, long long point_count,
                         int field, int precision, double *out, int memory, void *stream)
{
    // the execute step's own checks, before any device work
    if (point_count < 0 || (point_count > 0 && (!points || !out)))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "point_count < 0 or null points/out");
    if (memory != CCOIL_MEMORY_HOST && memory != CCOIL_MEMORY_DEVICE)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "memory must be HOST or DEVICE");
    ccoil_field_plan_t *plan = nullptr;
    int rc = ccoil_field_plan_create(coils, coil_count, field, precision, &plan);
    if (rc != CCOIL_OK)
        return rc;
    rc = ccoil_field_plan_execute(plan, points, point_count, out, memory, 0, stream);
    if (memory == CCOIL_MEMORY_DEVICE && rc == CCOIL_OK)
    {
        // the plan's device tables must outlive the asynchronous kernel
        cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        if (e != cudaSuccess)
            rc = cudaFail(e, "field evaluation");
    }
    ccoil_field_plan_destroy(plan);
    return rc;
}

int ccoil_check_bounded_wait(long long limit_cycles, void *stream)
{
    if (limit_cycles < 0 || limit_cycles > 4000000000LL)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "limit_cycles must lie in [0, 4e9]");
    const int rc = checkBoundedWait(limit_cycles, stream);
    // this call reports its own timeout; field calls report only theirs
    long long count = 0;
    if (readTimeouts(count) == CCOIL_OK)
        g_timeoutsReported.store(count);
    return rc;
}

int ccoil_set_point_ordering(int enabled)
{
    g_pointOrdering.store(enabled ? 1 : 0);
    return CCOIL_OK;
}

int ccoil_point_ordering(void) { return g_pointOrdering.load(); }

}  // extern "C"

double ccoil::refineFraction() { return g_refineFraction.load(); }

extern "C" {

int ccoil_set_refine_fraction(double fraction)
{
    if (!(fraction >= 0.0) || !std::isfinite(fraction))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "the refinement fraction must be finite and >= 0");
    g_refineFraction.store(fraction);
    return CCOIL_OK;
}

double ccoil_refine_fraction(void) { return g_refineFraction.load(); }

int ccoil_field_plan_refined_pairs(ccoil_field_plan_t *plan, long long *count)
{
    if (!plan || !count)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "null plan or count");
    *count = 0;
    if (plan->precision != CCOIL_PRECISION_FP32_REFINED || !plan->refinedTotal.ptr)
        return CCOIL_OK;
    unsigned long long v = 0;
    cudaError_t e = cudaMemcpy(&v, plan->refinedTotal.ptr, sizeof(v), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cudaFail(e, "refinement count");
    *count = (long long)v;
    return CCOIL_OK;
}

int ccoil_inject_allocation_failures(int count)
{
    if (count < 0)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "count < 0");
    g_failAllocations.store(count);
    return CCOIL_OK;
}

long long ccoil_timeout_count(void)
{
    long long v = 0;
    if (readTimeouts(v) != CCOIL_OK)
        return -1;
    return v;
}

} // extern "C"
