// Field kernels: coils x points, Gauss-Legendre quadrature over each coil's
// cross-section and azimuth, on CUDA cores (the integrand is transcendental,
// there is no dense contraction for the tensor cores).
//
// Tiling.  A CTA owns a tile of points (blockDim / LANES points, LANES threads
// per point) and walks the whole segment list.  By default every warp reads the
// segment blobs (coil geometry + node tables, see ccoil_internal.h) straight
// from global memory: all warps of an SM read the same node at the same time, a
// warp-uniform load that L1 serves (the table set stays L1/L2-resident), and no
// warp ever waits for another.  The alternative that stages each segment into
// shared memory with the bulk-copy engine (cp.async.bulk, completion on an
// mbarrier, double buffered, one CTA barrier per segment) is still compiled
// behind CCOIL_FP64_STAGE=1 / CCOIL_FP32_STAGE=1; it measured 1.15x (FP64) and
// 1.9x (FP32) slower on B200, because of the per-segment CTA barrier and the
// mbarrier polls.  The LANES threads of a point split the angular nodes; each
// keeps Cartesian accumulators and the LANES partial results are combined with
// warp shuffles once, at the end.
//
// Integrands follow the reference's CPU code line for line in FP64:
//   A fast  src/Coil/Fields/CalculateFieldsFast.cxx:13-83
//   B fast  src/Coil/Fields/CalculateFieldsFast.cxx:85-160
//   G fast  src/Coil/Fields/CalculateFieldsFast.cxx:162-266
//   A/B/G slow  src/Coil/Fields/CalculateFieldsSlow.cxx:13-265
//   Cartesian wrappers  src/Coil/Fields/CalculateFieldsMethods.cxx:6-84
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <algorithm>

namespace ccoil
{
int cudaFail(cudaError_t e, const char *what);

namespace
{
__device__ unsigned long long g_timeouts = 0;

constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz: bounded mbarrier wait

__device__ __forceinline__ unsigned smemAddr(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarInit(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fenceBarrierInit()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Producer side: announce the byte count and start the bulk copy global -> shared.
__device__ __forceinline__ void stageSegment(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbarTryWait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smemAddr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bounded wait: returns false after `limit` clock cycles (~2 s by default)
// without completion.
__device__ __forceinline__ bool mbarWait(unsigned long long *bar, unsigned parity, long long limit = kWaitCycles)
{
    if (mbarTryWait(bar, parity))
        return true;
    long long start = clock64();
    while (!mbarTryWait(bar, parity))
    {
        if (clock64() - start > limit)
            return false;
    }
    return true;
}

// Exercises the bounded wait on an mbarrier that nothing completes: one thread
// initialises it for one arrival that never comes and waits at most `limit`
// cycles; a wait that gives up is counted in g_timeouts and reported in *status
// (1), and the kernel returns normally.  No copy is in flight on the barrier.
__global__ void boundedWaitKernel(long long limit, int *status)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0)
        return;
    mbarInit(&bar, 1);
    fenceBarrierInit();
    const bool ok = mbarWait(&bar, 0, limit);
    if (!ok)
        atomicAdd(&g_timeouts, 1ull);
    *status = ok ? 0 : 1;
}

#include "integrands64.cuh"

// 6 CTAs of 128 threads per SM (80 registers; measured best on B200)
#ifndef CCOIL_FP64_MIN_BLOCKS
#define CCOIL_FP64_MIN_BLOCKS 6
#endif
// 1: segments staged into shared memory (double-buffered bulk copies, one CTA
// barrier per segment); 0 (default): each warp reads the tables from global
// memory through L1, with no barrier between warps
#ifndef CCOIL_FP64_STAGE
#define CCOIL_FP64_STAGE 0
#endif

template <int FIELD, int LANES>
__global__ void __launch_bounds__(128, CCOIL_FP64_MIN_BLOCKS) fieldsKernel64(const unsigned char *__restrict__ blob,
                                                      const SegmentDesc *__restrict__ segs, int nseg,
                                                      const double *__restrict__ points, long long npts,
                                                      double *__restrict__ out)
{
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bars[kSegmentStages];

    const int lane = threadIdx.x % LANES;
    const long long p = (long long)blockIdx.x * (blockDim.x / LANES) + threadIdx.x / LANES;
    const bool active = p < npts;

#if CCOIL_FP64_STAGE
    if (threadIdx.x == 0)
    {
        for (int s = 0; s < kSegmentStages; ++s)
            mbarInit(&bars[s], 1);
        fenceBarrierInit();
        for (int s = 0; s < kSegmentStages && s < nseg; ++s)
            stageSegment(smem + s * kSegmentBytes, blob + segs[s].offset, (unsigned)segs[s].bytes, &bars[s]);
    }
    __syncthreads();
#endif

    double px = 0.0, py = 0.0, pz = 0.0;
    if (active)
    {
        px = points[3 * p];
        py = points[3 * p + 1];
        pz = points[3 * p + 2];
    }
    double acc[W];
#pragma unroll
    for (int i = 0; i < W; ++i)
        acc[i] = 0.0;

    for (int s = 0; s < nseg; ++s)
    {
#if !CCOIL_FP64_STAGE
        if (active)
            integrateSegment64<FIELD, LANES>(blob + segs[s].offset, px, py, pz, lane, acc);
#else
        const int stage = s % kSegmentStages;
        const unsigned parity = (unsigned)((s / kSegmentStages) & 1);
        bool ok = mbarWait(&bars[stage], parity);
        if (__syncthreads_or(!ok))
        {
            if (threadIdx.x == 0)
            {
                atomicAdd(&g_timeouts, 1ull);
                // let the copies still in flight land before the CTA exits: the
                // newest segment issued into each stage is the largest j <= last
                // with j % stages == stage
                int last = min(s + kSegmentStages - 1, nseg - 1);
                for (int t = 0; t < kSegmentStages; ++t)
                {
                    int j = last - ((last - t) % kSegmentStages + kSegmentStages) % kSegmentStages;
                    if (j >= 0)
                        mbarWait(&bars[t], (unsigned)((j / kSegmentStages) & 1));
                }
            }
            return;
        }
        if (active)
            integrateSegment64<FIELD, LANES>(smem + stage * kSegmentBytes, px, py, pz, lane, acc);
        __syncthreads();
        if (threadIdx.x == 0 && s + kSegmentStages < nseg)
            stageSegment(smem + stage * kSegmentBytes, blob + segs[s + kSegmentStages].offset,
                         (unsigned)segs[s + kSegmentStages].bytes, &bars[stage]);
#endif
    }

    // combine the LANES partial sums of each point (fixed order -> reproducible)
#pragma unroll
    for (int off = LANES / 2; off > 0; off /= 2)
#pragma unroll
        for (int i = 0; i < W; ++i)
            acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
    if (active && lane == 0)
    {
#pragma unroll
        for (int i = 0; i < W; ++i)
            out[W * p + i] = acc[i];
    }
}

#include "fields32.cuh"
#include "batch.cuh"

template <int FIELD>
cudaError_t launchField(const FieldLaunch &L, cudaStream_t st)
{
    const int threads = 128;
    const int ppb = threads / L.lanes;
    long long blocks = (L.npts + ppb - 1) / ppb;
    if (blocks > 2147483647LL)
        return cudaErrorInvalidConfiguration;
    const bool fp32 = L.precision == CCOIL_PRECISION_FP32_COMPENSATED || L.precision == CCOIL_PRECISION_FP32_REFINED;
    const bool refine =
        L.precision == CCOIL_PRECISION_FP32_REFINED && L.d_contrib && L.d_refine_segs && L.d_refined_total;
    // the refining kernel is compiled for 1 to 8 lanes per point
    if (refine && L.lanes > 8)
        return cudaErrorInvalidValue;
    const bool staged = fp32 ? CCOIL_FP32_STAGE : CCOIL_FP64_STAGE;
    const size_t smem = staged ? (size_t)kSegmentStages * kSegmentBytes : 0;
    NearPair *work = reinterpret_cast<NearPair *>(L.d_work);
    switch (L.lanes)
    {
#define CCOIL_LAUNCH32(N, R)                                                                                      \
    fieldsKernel32<FIELD, N, R><<<(unsigned)blocks, threads, smem, st>>>(                                         \
        L.d_blob, L.d_segs, L.nseg, L.d_points, L.npts, L.d_out, work, L.work_capacity, L.d_work_count,           \
        R ? L.d_contrib : nullptr)
#define CCOIL_CASE(N, REFINING)                                                                                   \
    case N:                                                                                                       \
        if (refine)                                                                                               \
            CCOIL_LAUNCH32(N, REFINING);                                                                          \
        else if (fp32)                                                                                            \
            CCOIL_LAUNCH32(N, false);                                                                             \
        else                                                                                                      \
            fieldsKernel64<FIELD, N><<<(unsigned)blocks, threads, smem, st>>>(L.d_blob, L.d_segs, L.nseg,         \
                                                                              L.d_points, L.npts, L.d_out);       \
        break;
        CCOIL_CASE(1, true)
        CCOIL_CASE(2, true)
        CCOIL_CASE(4, true)
        CCOIL_CASE(8, true)
        CCOIL_CASE(16, false)
        CCOIL_CASE(32, false)
#undef CCOIL_CASE
#undef CCOIL_LAUNCH32
        default: return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !fp32)
        return e;
    // near-field pairs in FP64; the grid loops over the device-side count, so no
    // host synchronisation is needed between the passes
    nearFieldKernel<FIELD><<<L.near_blocks, 256, 0, st>>>(L.d_blob, L.d_segs, L.d_points, L.d_out, work,
                                                            L.work_capacity, L.d_work_count);
    e = cudaGetLastError();
    if (e != cudaSuccess || !refine)
        return e;
    // FP32_REFINED: with the near-field pairs in, select the dominating
    // contributions into a segment-major list (the work list is reused), take
    // them out of the totals and add them back in FP64
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    e = cudaMemsetAsync(L.d_refine_segs, 0, sizeof(unsigned long long) * (size_t)L.nseg, st);
    if (e != cudaSuccess)
        return e;
    const long long selectBlocks = std::min<long long>((L.npts + 255) / 256, 148LL * 16);
    refineCountKernel<W><<<(unsigned)selectBlocks, 256, 0, st>>>(L.d_out, L.d_contrib, L.npts, L.nseg,
                                                                 L.refine_fraction, L.d_refine_segs);
    refineScanKernel<<<1, 1024, 0, st>>>(L.d_refine_segs, L.nseg, L.work_capacity, L.d_work_count,
                                         L.d_refined_total);
    refineSelectKernel<W><<<(unsigned)selectBlocks, 256, 0, st>>>(L.d_out, L.d_contrib, L.npts, L.nseg,
                                                                  L.refine_fraction, L.d_refine_segs, work,
                                                                  L.work_capacity);
    refinePairsKernel64<FIELD><<<148 * refineMinBlocks(FIELD), 128, 0, st>>>(L.d_blob, L.d_segs, L.d_points, L.d_out,
                                                                           work, L.work_capacity, L.d_work_count);
    return cudaGetLastError();
}
} // namespace

int launchFields(const FieldLaunch &L, void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (L.npts == 0)
        return CCOIL_OK;
    if (L.nseg == 0)
    {
        int w = L.field == CCOIL_FIELD_G ? 9 : 3;
        cudaError_t e = cudaMemsetAsync(L.d_out, 0, sizeof(double) * (size_t)L.npts * w, st);
        return e == cudaSuccess ? CCOIL_OK : failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaError_t e;
    if (L.precision == CCOIL_PRECISION_FP32_COMPENSATED || L.precision == CCOIL_PRECISION_FP32_REFINED)
    {
        if (L.npts > 2147483647LL)
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "FP32_COMPENSATED supports at most 2^31-1 points per call");
        if (!L.d_work || !L.d_work_count)
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "FP32_COMPENSATED needs a near-field work list");
        e = cudaMemsetAsync(L.d_work_count, 0, sizeof(unsigned long long), st);
        if (e != cudaSuccess)
            return failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    }
    switch (L.field)
    {
        case CCOIL_FIELD_A:
        case CCOIL_FIELD_E: e = launchField<CCOIL_FIELD_A>(L, st); break;
        case CCOIL_FIELD_B: e = launchField<CCOIL_FIELD_B>(L, st); break;
        case CCOIL_FIELD_G: e = launchField<CCOIL_FIELD_G>(L, st); break;
        default: return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "unknown field");
    }
    if (e != cudaSuccess)
        return failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    return CCOIL_OK;
}

int launchBatch(const BatchLaunch &B, void *stream)
{
    static_assert(sizeof(BatchItem) == kBatchItemBytes, "batch item layout");
    return launchBatchImpl(B, static_cast<cudaStream_t>(stream));
}

int batchBlocksPerSM(int precision)
{
    int n = 0;
    cudaError_t e = precision == CCOIL_PRECISION_FP64
                        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batchKernel<CCOIL_PRECISION_FP64>, 128, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                              &n, batchKernel<CCOIL_PRECISION_FP32_COMPENSATED>, 128, 0);
    return (e == cudaSuccess && n > 0) ? n : 1;
}

int checkBoundedWait(long long limitCycles, void *stream)
{
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *dStatus = nullptr;
    cudaError_t e = scratchAlloc(reinterpret_cast<void **>(&dStatus), sizeof(int), st);
    if (e != cudaSuccess)
        return cudaFail(e, "status word");
    int status = 0;
    boundedWaitKernel<<<1, 32, 0, st>>>(limitCycles, dStatus);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&status, dStatus, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(dStatus, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, "bounded wait");
    return status ? fail(CCOIL_ERR_TIMEOUT, "the bounded wait gave up (nothing completed the barrier)") : CCOIL_OK;
}

int readTimeouts(long long &count)
{
    unsigned long long v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_timeouts, sizeof(v));
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    count = (long long)v;
    return CCOIL_OK;
}
} // namespace ccoil
