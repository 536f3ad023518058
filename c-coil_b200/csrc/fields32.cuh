// FP32-compensated field kernels (included by fields.cu inside its anonymous
// namespace, so they share the staging pipeline and the FP64 integrands);
// the integrands themselves are in integrands32.cuh.
//
// Near field.  A point inside a coil's winding box (inflated by a margin) is
// not integrated by the FP32 loop: its (point, segment) pair goes to a work
// list and a second kernel evaluates it with the FP64 integrands, so warps
// never diverge between the two paths.  If the list is full the pair is
// integrated in FP64 in place.

#include "integrands32.cuh"

// Integrates one segment for one lane and returns the norm of the lane's
// contribution (Frobenius norm for the gradient), taken from the cylindrical
// partial sums before the rotation, which keeps it: the refinement test adds
// these norms up per point.
template <int FIELD, int LANES>
__device__ __forceinline__ double integrateSegment32(const unsigned char *seg, const Frame &f, int lane, double *acc)
{
    const SegmentHeader &h = *reinterpret_cast<const SegmentHeader *>(seg);
    const double2 *tt = reinterpret_cast<const double2 *>(seg) + h.off_t;
    const double2 *lt = reinterpret_cast<const double2 *>(seg) + h.off_l;
    const PhiPair2 *pn = reinterpret_cast<const PhiPair2 *>(reinterpret_cast<const double2 *>(seg) + h.off_f32);
    if (FIELD == CCOIL_FIELD_B)
    {
        double H, Z;
        segmentB32<LANES>(h, tt, lt, pn, f, lane, H, Z);
        addRotated(h, H * f.cphi, H * f.sphi, Z, acc);
        return sqrt(H * H + Z * Z);
    }
    else if (FIELD == CCOIL_FIELD_G)
    {
        double g[4];
        segmentG32<LANES>(h, tt, lt, pn, f, lane, g);
        addGradient(h, f, g, acc);
        return sqrt(g[0] * g[0] + g[1] * g[1] + 2.0 * g[2] * g[2] + g[3] * g[3]);
    }
    else
    {
        double a = segmentA32<LANES>(h, tt, lt, pn, f, lane) * h.field_factor;
        addRotated(h, -a * f.sphi, a * f.cphi, 0.0, acc);
        return fabs(a);
    }
}

// FP64 integration of one segment for a pair that did not fit the work list;
// kept out of line so the FP32 kernel's register budget does not carry it.
template <int FIELD, int LANES>
__device__ __noinline__ void integrateSegment64Fallback(const unsigned char *seg, double px, double py, double pz,
                                                        int lane, double *acc)
{
    integrateSegment64<FIELD, LANES>(seg, px, py, pz, lane, acc);
}

// Near-field work list entry: (point, segment)
struct NearPair
{
    int point;
    int segment;
};

// CTAs per SM the register allocation targets (128 threads each): the packed
// FP32 integrands hold two mirror pairs per value, and these are the highest
// occupancies at which they compile without spills -- 5 for the vector
// potential (96 registers), 4 for the field and the gradient (128 registers)
#ifndef CCOIL_FP32_MIN_BLOCKS_A
#define CCOIL_FP32_MIN_BLOCKS_A 5
#endif
#ifndef CCOIL_FP32_MIN_BLOCKS_B
#define CCOIL_FP32_MIN_BLOCKS_B 4
#endif
#ifndef CCOIL_FP32_MIN_BLOCKS_G
#define CCOIL_FP32_MIN_BLOCKS_G 4
#endif
constexpr int fp32MinBlocks(int field)
{
    return field == CCOIL_FIELD_B ? CCOIL_FP32_MIN_BLOCKS_B
                                  : (field == CCOIL_FIELD_G ? CCOIL_FP32_MIN_BLOCKS_G : CCOIL_FP32_MIN_BLOCKS_A);
}
// 1: segments are staged into shared memory by bulk copies (double-buffered,
// one CTA barrier per segment); 0 (default, 1.9x faster on B200): each warp
// reads the segment tables from global memory through L1 -- the same table
// bytes are read by every warp of the SM, so they stay L1/L2-resident -- and
// warps never wait for each other
#ifndef CCOIL_FP32_STAGE
#define CCOIL_FP32_STAGE 0
#endif

template <int FIELD, int LANES>
__global__ void __launch_bounds__(128, fp32MinBlocks(FIELD)) fieldsKernel32(const unsigned char *__restrict__ blob,
                                                      const SegmentDesc *__restrict__ segs, int nseg,
                                                      const double *__restrict__ points, long long npts,
                                                      double *__restrict__ out, NearPair *__restrict__ work,
                                                      unsigned long long workCapacity,
                                                      unsigned long long *__restrict__ workCount,
                                                      double *__restrict__ cabs)
{
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) unsigned long long bars[kSegmentStages];
    __shared__ int timedOut;

    const int lane = threadIdx.x % LANES;
    const long long p = (long long)blockIdx.x * (blockDim.x / LANES) + threadIdx.x / LANES;
    const bool active = p < npts;

#if CCOIL_FP32_STAGE
    if (threadIdx.x == 0)
    {
        timedOut = 0;
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
    double cn = 0.0;  // sum of the segments' contribution norms (refinement test)

    for (int s = 0; s < nseg; ++s)
    {
#if CCOIL_FP32_STAGE
        const int stage = s % kSegmentStages;
        const unsigned parity = (unsigned)((s / kSegmentStages) & 1);
        const bool ok = mbarWait(&bars[stage], parity);
        if (!ok)
            timedOut = 1;
        const unsigned char *seg = smem + stage * kSegmentBytes;
#else
        const bool ok = true;
        const unsigned char *seg = blob + segs[s].offset;
#endif
        if (active && ok)
        {
            const SegmentHeader &h = *reinterpret_cast<const SegmentHeader *>(seg);
            const Frame f = toCoilFrame(h, px, py, pz);
            if (!nearWinding(h, f))
                cn += integrateSegment32<FIELD, LANES>(seg, f, lane, acc);
            else
            {
                bool queued = false;
                if (lane == 0)
                {
                    unsigned long long slot = atomicAdd(workCount, 1ull);
                    if (slot < workCapacity)
                    {
                        work[slot].point = (int)p;
                        work[slot].segment = s;
                        queued = true;
                    }
                }
                // all lanes of the point learn whether the pair was queued
                const unsigned groupMask = LANES == 32 ? 0xffffffffu
                                                       : (((1u << LANES) - 1u) << ((threadIdx.x % 32) / LANES * LANES));
                queued = __shfl_sync(groupMask, queued, (threadIdx.x % 32) / LANES * LANES);
                if (!queued)
                    integrateSegment64Fallback<FIELD, LANES>(seg, px, py, pz, lane, acc);
            }
        }
#if CCOIL_FP32_STAGE
        __syncthreads();
        if (timedOut)
        {
            // a stage never arrived: drain what is in flight (bounded) and leave
            if (threadIdx.x == 0)
            {
                atomicAdd(&g_timeouts, 1ull);
                int last = min(s + kSegmentStages - 1, nseg - 1);
                for (int t = 0; t < kSegmentStages; ++t)
                {
                    int j = last - ((last - t) % kSegmentStages + kSegmentStages) % kSegmentStages;
                    if (j >= s)
                        mbarWait(&bars[t], (unsigned)((j / kSegmentStages) & 1));
                }
            }
            return;
        }
        if (threadIdx.x == 0 && s + kSegmentStages < nseg)
            stageSegment(smem + stage * kSegmentBytes, blob + segs[s + kSegmentStages].offset,
                         (unsigned)segs[s + kSegmentStages].bytes, &bars[stage]);
#endif
    }

#pragma unroll
    for (int off = LANES / 2; off > 0; off /= 2)
    {
#pragma unroll
        for (int i = 0; i < W; ++i)
            acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
        cn += __shfl_xor_sync(0xffffffffu, cn, off);
    }
    if (active && lane == 0)
    {
#pragma unroll
        for (int i = 0; i < W; ++i)
            out[W * p + i] = acc[i];
        if (cabs)
            cabs[p] = cn;
    }
}

// Second pass: one warp per near-field (point, segment) pair, FP64 integrands
// read from the segment blob in global memory, result added to the point's
// output (FP64 atomics; each pair adds once).
template <int FIELD>
__global__ void __launch_bounds__(256) nearFieldKernel(const unsigned char *__restrict__ blob,
                                                       const SegmentDesc *__restrict__ segs,
                                                       const double *__restrict__ points, double *__restrict__ out,
                                                       const NearPair *__restrict__ work,
                                                       unsigned long long workCapacity,
                                                       const unsigned long long *__restrict__ workCount)
{
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    const unsigned long long n = min(*workCount, workCapacity);
    const int lane = threadIdx.x % 32;
    const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const unsigned long long warps = (unsigned long long)gridDim.x * blockDim.x / 32;
    for (unsigned long long i = warp; i < n; i += warps)
    {
        const NearPair e = work[i];
        const unsigned char *seg = blob + segs[e.segment].offset;
        const long long p = e.point;
        double acc[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            acc[k] = 0.0;
        integrateSegment64<FIELD, 32>(seg, points[3 * p], points[3 * p + 1], points[3 * p + 2], lane, acc);
#pragma unroll
        for (int off = 16; off > 0; off /= 2)
#pragma unroll
            for (int k = 0; k < W; ++k)
                acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
        if (lane == 0)
        {
#pragma unroll
            for (int k = 0; k < W; ++k)
                atomicAdd(&out[W * p + k], acc[k]);
        }
    }
}

// Refinement test: a point whose FP32-evaluated contributions have norms that
// add up to more than `ratio` times the norm of its total (the coils' fields
// cancel there, and the total's relative error grows by that ratio; the
// near-field pairs, evaluated in FP64, do not count) is listed for
// re-evaluation in FP64.
template <int W>
__global__ void __launch_bounds__(256) refineTestKernel(const double *__restrict__ out,
                                                        const double *__restrict__ cabs, long long npts, double ratio,
                                                        int *__restrict__ list, unsigned long long capacity,
                                                        unsigned long long *__restrict__ count)
{
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npts;
         p += (long long)gridDim.x * blockDim.x)
    {
        double n2 = 0.0;
#pragma unroll
        for (int k = 0; k < W; ++k)
            n2 += out[W * p + k] * out[W * p + k];
        // !(a <= b) also lists points whose values are not finite
        if (!(cabs[p] <= ratio * sqrt(n2)))
        {
            const unsigned long long slot = atomicAdd(count, 1ull);
            if (slot < capacity)
                list[slot] = (int)p;
        }
    }
}

// FP64 re-evaluation of the listed points: all segments with the FP64
// integrands, LANES threads per point splitting the angular nodes, the result
// overwriting the point's output.  Grid-stride over the device-side count (no
// host synchronisation between the passes); a list that overflowed leaves the
// remaining points at their FP32 values, which the caller learns from the count.
template <int FIELD, int LANES>
__global__ void __launch_bounds__(128) refineKernel64(const unsigned char *__restrict__ blob,
                                                      const SegmentDesc *__restrict__ segs, int nseg,
                                                      const double *__restrict__ points, double *__restrict__ out,
                                                      const int *__restrict__ list, unsigned long long capacity,
                                                      const unsigned long long *__restrict__ count)
{
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    const unsigned long long n = min(*count, capacity);
    const int lane = threadIdx.x % LANES;
    const unsigned long long groups = (unsigned long long)gridDim.x * (blockDim.x / LANES);
    for (unsigned long long i = (unsigned long long)blockIdx.x * (blockDim.x / LANES) + threadIdx.x / LANES;
         i < n; i += groups)
    {
        const long long p = list[i];
        double acc[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            acc[k] = 0.0;
        const double px = points[3 * p], py = points[3 * p + 1], pz = points[3 * p + 2];
        for (int s = 0; s < nseg; ++s)
            integrateSegment64<FIELD, LANES>(blob + segs[s].offset, px, py, pz, lane, acc);
        const unsigned groupMask = LANES == 32 ? 0xffffffffu
                                               : (((1u << LANES) - 1u) << ((threadIdx.x % 32) / LANES * LANES));
#pragma unroll
        for (int off = LANES / 2; off > 0; off /= 2)
#pragma unroll
            for (int k = 0; k < W; ++k)
                acc[k] += __shfl_xor_sync(groupMask, acc[k], off);
        if (lane == 0)
        {
#pragma unroll
            for (int k = 0; k < W; ++k)
                out[W * p + k] = acc[k];
        }
    }
}
