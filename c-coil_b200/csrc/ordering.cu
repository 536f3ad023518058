// Point ordering for the FP32 field plans.
//
// The FP32 integrands make warp-wide choices per (point tile, coil segment):
// which side of the coil's length slab the points lie on, which asinh tier
// their arguments need, which (point, coil) pairs are deferred to the FP64
// near-field pass.  A warp whose 32 points lie close together agrees on those
// choices more often and runs the cheaper uniform form.  So before the field
// kernels run, the plan sorts the points along a Morton (Z-order) curve over
// their bounding box (30-bit keys, 10 bits per axis), evaluates them in that
// order, and writes each result back to the caller's index.  The sort is a
// stable radix sort on (key, index), so the order, and with it every result,
// is the same on every run.
#include "ccoil_internal.h"

#include <cub/device/device_radix_sort.cuh>

namespace ccoil
{
int cudaFail(cudaError_t e, const char *what);

namespace
{
// order-preserving map of a double onto 64-bit unsigned integers
__device__ __forceinline__ unsigned long long orderedBits(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double fromOrderedBits(unsigned long long b)
{
    return __longlong_as_double((long long)((b >> 63) ? (b & 0x7fffffffffffffffull) : ~b));
}

// bbox[0..2]: minimum, bbox[3..5]: maximum of the finite coordinates, as
// orderedBits (initialised to all ones and all zeros)
__global__ void boundsKernel(const double *__restrict__ pts, long long n, unsigned long long *__restrict__ bbox)
{
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        for (int k = 0; k < 3; ++k)
        {
            const double v = pts[3 * i + k];
            if (isfinite(v))
            {
                const unsigned long long b = orderedBits(v);
                lo[k] = b < lo[k] ? b : lo[k];
                hi[k] = b > hi[k] ? b : hi[k];
            }
        }
    for (int k = 0; k < 3; ++k)
        for (int off = 16; off > 0; off /= 2)
        {
            const unsigned long long l = __shfl_xor_sync(0xffffffffu, lo[k], off);
            const unsigned long long h = __shfl_xor_sync(0xffffffffu, hi[k], off);
            lo[k] = l < lo[k] ? l : lo[k];
            hi[k] = h > hi[k] ? h : hi[k];
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k)
        {
            atomicMin(&bbox[k], lo[k]);
            atomicMax(&bbox[3 + k], hi[k]);
        }
}

// the low 10 bits of x moved to every third bit (bit i to bit 3 i)
__device__ __forceinline__ unsigned spread10(unsigned x)
{
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// keys[i] = Morton code of point i in its 1024^3 cell grid over the bounding
// box (points with a non-finite coordinate last), idx[i] = i
__global__ void mortonKernel(const double *__restrict__ pts, long long n, const unsigned long long *__restrict__ bbox,
                             unsigned *__restrict__ keys, int *__restrict__ idx)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    unsigned key = 0;
    bool finite = true;
    for (int k = 0; k < 3; ++k)
    {
        const double v = pts[3 * i + k];
        finite = finite && isfinite(v);
        const bool any = bbox[k] <= bbox[3 + k];  // some finite coordinate exists
        const double lo = any ? fromOrderedBits(bbox[k]) : 0.0, hi = any ? fromOrderedBits(bbox[3 + k]) : 0.0;
        const double ext = hi - lo;
        const double scale = ext > 0.0 && isfinite(ext) ? 1024.0 / ext : 0.0;
        double t = (v - lo) * scale;
        if (!(t >= 0.0))  // negative or NaN
            t = 0.0;
        if (t > 1023.0)
            t = 1023.0;
        key |= spread10((unsigned)t) << k;
    }
    keys[i] = finite ? key : 0x3fffffffu;
    idx[i] = (int)i;
}

__global__ void gatherPointsKernel(const double *__restrict__ pts, const int *__restrict__ order, long long n,
                                   double *__restrict__ sorted)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * n)
        return;
    const long long i = e / 3;
    sorted[e] = pts[3 * (long long)order[i] + (e - 3 * i)];
}

__global__ void scatterResultsKernel(const double *__restrict__ sorted, const int *__restrict__ order, long long n,
                                     int width, double *__restrict__ out)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)width * n)
        return;
    const long long i = e / width;
    out[(long long)width * order[i] + (e - (long long)width * i)] = sorted[e];
}

constexpr size_t kAlign = 256;
size_t roundUp(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

size_t sortTempBytes(long long n)
{
    size_t temp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<const unsigned *>(nullptr),
                                    static_cast<unsigned *>(nullptr), static_cast<const int *>(nullptr),
                                    static_cast<int *>(nullptr), (int)n, 0, 30, (cudaStream_t)0);
    return temp;
}
} // namespace

size_t pointOrderScratchBytes(long long n)
{
    // bbox | keys in | keys out | indices in | radix-sort temporary storage
    return roundUp(6 * sizeof(unsigned long long)) + 3 * roundUp(sizeof(unsigned) * (size_t)n) + sortTempBytes(n);
}

int orderPoints(const double *pts, long long n, void *scratch, size_t scratchBytes, int *order, double *sortedPts,
                void *stream)
{
    if (n <= 0 || n > kPointOrderMaxPoints)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "point ordering: point count out of range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *s = static_cast<unsigned char *>(scratch);
    auto *bbox = reinterpret_cast<unsigned long long *>(s);
    s += roundUp(6 * sizeof(unsigned long long));
    auto *keysIn = reinterpret_cast<unsigned *>(s);
    s += roundUp(sizeof(unsigned) * (size_t)n);
    auto *keysOut = reinterpret_cast<unsigned *>(s);
    s += roundUp(sizeof(unsigned) * (size_t)n);
    auto *idxIn = reinterpret_cast<int *>(s);
    s += roundUp(sizeof(unsigned) * (size_t)n);
    size_t temp = sortTempBytes(n);
    if ((size_t)(s - static_cast<unsigned char *>(scratch)) + temp > scratchBytes)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "point ordering: scratch buffer too small");
    cudaError_t e = cudaMemsetAsync(bbox, 0xff, 3 * sizeof(unsigned long long), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(bbox + 3, 0, 3 * sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return cudaFail(e, "point ordering");
    const long long want = (n + 255) / 256;
    boundsKernel<<<(unsigned)(want < 148 * 8 ? want : 148 * 8), 256, 0, st>>>(pts, n, bbox);
    mortonKernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pts, n, bbox, keysIn, idxIn);
    e = cub::DeviceRadixSort::SortPairs(s, temp, keysIn, keysOut, idxIn, order, (int)n, 0, 30, st);
    if (e == cudaSuccess)
    {
        gatherPointsKernel<<<(unsigned)((3 * n + 255) / 256), 256, 0, st>>>(pts, order, n, sortedPts);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? CCOIL_OK : cudaFail(e, "point ordering");
}

int scatterResults(const double *sorted, const int *order, long long n, int width, double *out, void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    scatterResultsKernel<<<(unsigned)((width * n + 255) / 256), 256, 0, st>>>(sorted, order, n, width, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CCOIL_OK : cudaFail(e, "result scatter");
}
} // namespace ccoil
