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
constexpr double kPi = 3.14159265358979323846;
constexpr double kMuReduced = 1e-7;
constexpr double kNearMarginStatic = 0.1;  // same near-field box as the plan path's default

// The scratch.  In host code this name is only a stand-in: its device address
// comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_staticScratch[kStaticScratchBytes];

// host staging for the node tables and segment list (shared by all calls)
unsigned char g_hostBlob[kStaticBlobBytes];
SegmentDesc g_hostSegs[kStaticMaxSegments];
std::mutex g_hostMutex;

unsigned char *g_deviceScratch[kMaxDevices] = {};
std::mutex g_setupMutex;

struct Writer
{
    unsigned char *base;
    size_t cap, used = 0;
    bool ok = true;
    void put(const void *p, size_t n)
    {
        if (!ok || used + n > cap)
        {
            ok = false;
            return;
        }
        std::memcpy(base + used, p, n);
        used += n;
    }
};

// Builds the same segment layout as buildFieldSegments (segments.cpp) for the
// FP32-compensated path, computing every node on the fly instead of holding
// per-coil tables.
int buildStatic(const Coil *coils, int count, int field, size_t &blobBytes, int &nseg)
{
    Writer w{g_hostBlob, kStaticBlobBytes};
    nseg = 0;
    for (int ci = 0; ci < count; ++ci)
    {
        const Coil &k = coils[ci];
        const PrecisionArgs &p = k.precision;
        if (!validArgs(p))
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT,
                               "a coil's precision arguments are out of range (increments 1..100, blocks >= 1)");
        if (!(k.inner_radius > 0.0) || !(k.thickness > 0.0) || !(k.length > 0.0))
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "inner radius, thickness and length must be positive");
        const bool fast = k.use_fast_method != 0;
        const double tBlock = k.thickness / p.thickness_blocks, aBlock = kPi / p.angular_blocks;
        const double constant = fast ? kMuReduced * k.current_density * tBlock * aBlock * 2 * 0.25
                                     : kMuReduced * k.current_density * (k.length / p.length_blocks) * tBlock *
                                           aBlock * 2 * 0.125;
        const int nt = p.thickness_blocks * p.thickness_increments;
        const int nl = fast ? 0 : p.length_blocks * p.length_increments;
        const int nphi = p.angular_blocks * p.angular_increments;
        const int headerBytes = (int)sizeof(SegmentHeader);
        const int fixedBytes = headerBytes + 16 * (nt + nl);
        // 16 bytes per FP64 node plus 16 per FP32 mirror-pair entry; segments cut
        // at even node counts so that no mirror pair is split
        const int maxPhi = 2 * ((kSegmentBytes - fixedBytes) / 48);
        if (maxPhi < 1)
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "a coil's thickness/length node tables exceed one segment");
        const double *tx = legendreNodes(p.thickness_increments), *tw = legendreWeights(p.thickness_increments);
        const double *ax = legendreNodes(p.angular_increments), *aw = legendreWeights(p.angular_increments);
        auto phiOf = [&](int j) {
            return aBlock * (j / p.angular_increments + 0.5) + (aBlock * 0.5) * ax[j % p.angular_increments];
        };
        for (int start = 0; start < nphi; start += maxPhi)
        {
            const int cnt = nphi - start < maxPhi ? nphi - start : maxPhi;
            if (nseg >= kStaticMaxSegments)
                return failMessage(CCOIL_ERR_INVALID_ARGUMENT,
                                   "coil set needs more than 8192 segments; the static entry point's limit");
            SegmentHeader h;
            std::memset(&h, 0, sizeof(h));
            std::memcpy(h.position, k.position, sizeof(h.position));
            std::memcpy(h.inv_transform, k.inverse_transform, sizeof(h.inv_transform));
            std::memcpy(h.transform, k.transform, sizeof(h.transform));
            h.half_length = k.length * 0.5;
            h.field_factor = field == CCOIL_FIELD_E ? 2 * kPi * k.sine_frequency : 1.0;
            h.inner_radius = k.inner_radius;
            h.n_t = nt;
            h.n_l = nl;
            h.n_phi = cnt;
            h.fast = fast ? 1 : 0;
            h.off_t = headerBytes / 16;
            h.off_l = h.off_t + nt;
            h.off_phi = h.off_l + nl;
            h.off_f32 = h.off_phi + cnt;
            const double margin = kNearMarginStatic * k.inner_radius;
            h.near_lo[0] = k.inner_radius - margin;
            h.near_hi[0] = k.inner_radius + k.thickness + margin;
            h.near_lo[1] = -0.5 * k.length - margin;
            h.near_hi[1] = 0.5 * k.length + margin;
            h.near_r2 = margin * margin;

            SegmentDesc &d = g_hostSegs[nseg];
            d.offset = (long long)w.used;
            d.coil = ci;
            w.put(&h, sizeof(h));
            for (int bt = 0; bt < p.thickness_blocks; ++bt)
                for (int i = 0; i < p.thickness_increments; ++i)
                {
                    double e[2] = {k.inner_radius + tBlock * (bt + 0.5) + (tBlock * 0.5) * tx[i], constant * tw[i]};
                    w.put(e, sizeof(e));
                }
            if (!fast)
            {
                const double lBlock = k.length / p.length_blocks;
                const double *lx = legendreNodes(p.length_increments), *lw = legendreWeights(p.length_increments);
                for (int bl = 0; bl < p.length_blocks; ++bl)
                    for (int i = 0; i < p.length_increments; ++i)
                    {
                        double e[2] = {-k.length * 0.5 + lBlock * (bl + 0.5) + (lBlock * 0.5) * lx[i], lw[i]};
                        w.put(e, sizeof(e));
                    }
            }
            // the FP64 table in mirror-pair order, then the pair entries it covers
            for (int j = start; j < start + cnt; ++j)
            {
                const int node = pairOrderNode(j, nphi);
                double e[2] = {std::cos(phiOf(node)), aw[node % p.angular_increments]};
                w.put(e, sizeof(e));
            }
            for (int i = start / 2; i < (start + cnt + 1) / 2; ++i)
            {
                const PhiNode32 nd = phiPair32(p, i);
                w.put(&nd, sizeof(nd));
            }
            d.bytes = (int)(w.used - (size_t)d.offset);
            if (!w.ok)
                return failMessage(CCOIL_ERR_INVALID_ARGUMENT,
                                   "coil set needs more than 1 MiB of node tables; the static entry point's limit");
            ++nseg;
        }
    }
    blobBytes = w.used;
    return CCOIL_OK;
}

// Device address of the scratch array on the current device, looked up once per
// device with that device current.
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
