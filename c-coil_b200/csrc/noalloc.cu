// ccoil_fields_fp32c_static: the FP32-compensated field evaluation for callers
// that cannot allocate device memory -- plugins living inside a host
// application that owns (and budgets) every device allocation, or real-time
// loops where an allocation could stall.  It allocates
// nothing: the scratch the kernel needs (the coil node tables, the segment list,
// the near-field work list and its counter) lives in one file-scope __device__
// array of fixed size, and the node tables are built on the host into a fixed
// staging buffer.
//
// The array is a module global: every GPU that loads the library holds its
// 3 MiB until the process exits, and every call shares it.  Calls that overlap
// on the GPU (two streams, or two host threads) therefore race on it; callers
// must order them, for example by issuing them on one stream.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

namespace ccoil
{
namespace
{
constexpr size_t kStaticBlobBytes = 1u << 20;        // node tables
constexpr int kStaticMaxSegments = 8192;              // segment descriptors (128 KiB)
constexpr size_t kStaticWorkEntries = 1u << 18;       // near-field work list (2 MiB)
constexpr size_t kOffSegs = kStaticBlobBytes;
constexpr size_t kOffWork = kOffSegs + sizeof(SegmentDesc) * kStaticMaxSegments;
constexpr size_t kOffCount = kOffWork + kNearPairBytes * kStaticWorkEntries;
constexpr size_t kStaticScratchBytes = kOffCount + 256;
constexpr int kMaxDevices = 64;

// The scratch.  In host code this name is only a stand-in: its device address
// comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_staticScratch[kStaticScratchBytes];

// host staging for the node tables and segment list (shared by all calls)
unsigned char g_hostBlob[kStaticBlobBytes];
SegmentDesc g_hostSegs[kStaticMaxSegments];
std::mutex g_hostMutex;

unsigned char *g_deviceScratch[kMaxDevices] = {};
std::mutex g_setupMutex;

// The fixed host staging buffers as a segment sink: the node-table layout is
// the plan path's own (buildFieldSegments), only its destination differs.
struct StaticSink final : SegmentSink
{
    size_t used = 0;
    int nseg = 0;
    bool tablesFull = false, segmentsFull = false;
    bool append(const void *p, size_t n) override
    {
        if (used + n > kStaticBlobBytes)
        {
            tablesFull = true;
            return false;
        }
        std::memcpy(g_hostBlob + used, p, n);
        used += n;
        return true;
    }
    size_t size() const override { return used; }
    bool segment(const SegmentDesc &d) override
    {
        if (nseg >= kStaticMaxSegments)
        {
            segmentsFull = true;
            return false;
        }
        g_hostSegs[nseg++] = d;
        return true;
    }
    std::string overflowMessage() const override
    {
        return segmentsFull ? "coil set needs more than 8192 segments; the static entry point's limit"
                            : "coil set needs more than 1 MiB of node tables; the static entry point's limit";
    }
};

// Builds the FP32-compensated segment layout of `coils` into the staging buffers.
int buildStatic(const Coil *coils, int count, int field, size_t &blobBytes, int &nseg)
{
    StaticSink sink;
    std::string err;
    if (!buildFieldSegments(coils, count, field, CCOIL_PRECISION_FP32_COMPENSATED, sink, err))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, err);
    blobBytes = sink.used;
    nseg = sink.nseg;
    return CCOIL_OK;
}

// Device address of the scratch array on the current device, looked up once per
// device with that device current.  The address stays cached for the life of
// the process: cudaDeviceReset, which unloads the module, is not supported while
// the library is in use.
int scratchAddress(unsigned char **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return failMessage(CCOIL_ERR_NO_DEVICE, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return failMessage(CCOIL_ERR_NOT_SUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_deviceScratch[dev])
    {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_staticScratch);
        if (e != cudaSuccess || !ptr)
            return failMessage(CCOIL_ERR_CUDA, e != cudaSuccess ? cudaGetErrorString(e)
                                                                 : "cudaGetSymbolAddress returned a null address");
        g_deviceScratch[dev] = static_cast<unsigned char *>(ptr);
    }
    *out = g_deviceScratch[dev];
    return CCOIL_OK;
}
} // namespace
} // namespace ccoil

using namespace ccoil;

extern "C" int ccoil_fields_fp32c_static(const ccoil_coil_t *coils, int coil_count, const double *points,
                                         long long point_count, int field, double *out, void *stream)
{
    if (coil_count < 0 || (coil_count > 0 && !coils))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "coil_count < 0 or coils null");
    if (field < CCOIL_FIELD_A || field > CCOIL_FIELD_G)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "field must be A, B, E or G");
    if (point_count < 0 || point_count > 2147483647LL || (point_count > 0 && (!points || !out)))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "point_count must be in [0, 2^31-1] with non-null points/out");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int width = field == CCOIL_FIELD_G ? 9 : 3;
    if (point_count == 0)
        return CCOIL_OK;
    // a captured call would record copies from the shared host staging buffers,
    // which a replay reads after later calls have overwritten them
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    const cudaError_t ce = cudaStreamIsCapturing(st, &capture);
    if (ce != cudaSuccess)
        return failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(ce));
    if (capture != cudaStreamCaptureStatusNone)
        return failMessage(CCOIL_ERR_NOT_SUPPORTED, "not supported during stream capture");

    unsigned char *scratch = nullptr;
    int rc = scratchAddress(&scratch);
    if (rc != CCOIL_OK)
        return rc;

    std::lock_guard<std::mutex> lock(g_hostMutex);
    size_t blobBytes = 0;
    int nseg = 0;
    rc = buildStatic(coils, coil_count, field, blobBytes, nseg);
    if (rc != CCOIL_OK)
        return rc;
    cudaError_t e;
    if (nseg == 0)
    {
        e = cudaMemsetAsync(out, 0, sizeof(double) * width * (size_t)point_count, st);
        return e == cudaSuccess ? CCOIL_OK : failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    }
    // the staging buffers are pageable host memory: each copy has consumed them
    // when cudaMemcpyAsync returns, so the next call may overwrite them
    e = cudaMemcpyAsync(scratch, g_hostBlob, blobBytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scratch + kOffSegs, g_hostSegs, sizeof(SegmentDesc) * nseg, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess)
        return failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));

    FieldLaunch L;
    L.d_blob = scratch;
    L.d_segs = reinterpret_cast<const SegmentDesc *>(scratch + kOffSegs);
    L.nseg = nseg;
    L.d_points = points;
    L.npts = point_count;
    L.d_out = out;
    L.field = field;
    L.precision = CCOIL_PRECISION_FP32_COMPENSATED;
    L.lanes = point_count >= 148LL * 1024 ? 1 : point_count >= 148LL * 512 ? 2 : point_count >= 148LL * 256 ? 4 : 8;
    L.d_work = scratch + kOffWork;
    L.work_capacity = kStaticWorkEntries;
    L.d_work_count = reinterpret_cast<unsigned long long *>(scratch + kOffCount);  // zeroed by launchFields
    L.near_blocks = 148 * 8;
    return launchFields(L, stream);
}
