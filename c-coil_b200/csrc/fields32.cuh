// FP32-compensated field kernels (included by fields.cu inside its anonymous
// namespace, so they share the staging pipeline and the FP64 integrands);
// the integrands themselves are in integrands32.cuh.
//
// Near field.  A point inside a coil's winding box (inflated by a margin) is
// not integrated by the FP32 loop: its (point, segment) pair goes to a work
// list and a second kernel evaluates it with the FP64 integrands, so warps
// never diverge between the two paths.  If the list is full the pair is
// integrated in FP64 in place.
//
// FP32_REFINED.  The FP32 kernel also stores every (point, segment)
// contribution; once the point's total is known, a selection kernel removes
// each contribution whose norm exceeds a set fraction of the total's norm
// (the contributions that dominate a point where the coils' fields cancel,
// whose FP32 errors the cancellation magnifies) and lists the pair, and the
// near-field kernel adds those pairs back evaluated with the FP64 integrands.

#include "integrands32.cuh"
#include "integrands64f.cuh"

// Integrates one segment for one lane and adds the lane's contribution to acc.
template <int FIELD, int LANES>
__device__ __forceinline__ void integrateSegment32(const unsigned char *seg, const Frame &f, int lane, double *acc)
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
    }
    else if (FIELD == CCOIL_FIELD_G)
    {
        double g[4];
        segmentG32<LANES>(h, tt, lt, pn, f, lane, g);
        addGradient(h, f, g, acc);
    }
    else
    {
        double a = segmentA32<LANES>(h, tt, lt, pn, f, lane) * h.field_factor;
        addRotated(h, -a * f.sphi, a * f.cphi, 0.0, acc);
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

// REFINE (FP32_REFINED): every (point, segment) contribution is also written
// to contrib, segment-major ([segment][point][W], so a warp's stores for one
// segment are contiguous), near-field pairs as zeros (they are FP64 already)
template <int FIELD, int LANES, bool REFINE>
__global__ void __launch_bounds__(128, fp32MinBlocks(FIELD)) fieldsKernel32(const unsigned char *__restrict__ blob,
                                                      const SegmentDesc *__restrict__ segs, int nseg,
                                                      const double *__restrict__ points, long long npts,
                                                      double *__restrict__ out, NearPair *__restrict__ work,
                                                      unsigned long long workCapacity,
                                                      unsigned long long *__restrict__ workCount,
                                                      double *__restrict__ contrib)
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
    // the lanes of one point
    auto groupMask = [] {
        return LANES == 32 ? 0xffffffffu : (((1u << LANES) - 1u) << ((threadIdx.x % 32) / LANES * LANES));
    };

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
            const bool nearPair = nearWinding(h, f);
            if (!nearPair && !REFINE)
                integrateSegment32<FIELD, LANES>(seg, f, lane, acc);
            else if (!nearPair)
            {
                // the segment's contribution on its own: combined over the point's
                // lanes (all of them take this branch), added to the total by lane 0
                // and stored for the selection
                double c[W];
#pragma unroll
                for (int i = 0; i < W; ++i)
                    c[i] = 0.0;
                integrateSegment32<FIELD, LANES>(seg, f, lane, c);
#pragma unroll
                for (int off = LANES / 2; off > 0; off /= 2)
#pragma unroll
                    for (int i = 0; i < W; ++i)
                        c[i] += __shfl_xor_sync(groupMask(), c[i], off);
                if (lane == 0)
                {
                    double *dst = contrib + ((size_t)s * (size_t)npts + (size_t)p) * W;
#pragma unroll
                    for (int i = 0; i < W; ++i)
                    {
                        acc[i] += c[i];
                        dst[i] = c[i];
                    }
                }
            }
            else
            {
                if (REFINE && lane == 0)
                {
                    double *dst = contrib + ((size_t)s * (size_t)npts + (size_t)p) * W;
#pragma unroll
                    for (int i = 0; i < W; ++i)
                        dst[i] = 0.0;
                }
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
                queued = __shfl_sync(groupMask(), queued, (threadIdx.x % 32) / LANES * LANES);
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

// One segment at one point for the refinement pass: the vector potential (and
// E) and the field with the forms above, the gradient with the FP64 field
// integrands
template <int FIELD>
__device__ __forceinline__ void integrateSegmentRefine(const unsigned char *seg, double px, double py, double pz,
                                                       double *acc)
{
    if (FIELD == CCOIL_FIELD_G)
    {
        integrateSegment64<FIELD, 1>(seg, px, py, pz, 0, acc);
        return;
    }
    const SegmentHeader &h = *reinterpret_cast<const SegmentHeader *>(seg);
    const double2 *tt = reinterpret_cast<const double2 *>(seg) + h.off_t;
    const double2 *lt = reinterpret_cast<const double2 *>(seg) + h.off_l;
    const double2 *pt = reinterpret_cast<const double2 *>(seg) + h.off_phi;
    const Frame f = toCoilFrame(h, px, py, pz);
    if (FIELD == CCOIL_FIELD_B)
    {
        double H, Z;
        segmentB64Fast(h, tt, lt, pt, f, H, Z);
        addRotated(h, H * f.cphi, H * f.sphi, Z, acc);
    }
    else
    {
        const double a = segmentA64Fast<true>(h, tt, lt, pt, f) * h.field_factor;
        addRotated(h, -a * f.sphi, a * f.cphi, 0.0, acc);
    }
}

// FP32_REFINED's FP64 pass: one thread per listed (point, segment) pair, the
// whole segment in FP64 (integrateSegmentRefine; each thickness node's set-up
// serves all its angular nodes, as in the FP64 field kernel, where one warp
// per pair measured 1.2x the time), the result added to the point's output
// (FP64 atomics).  The selection lists the pairs segment-major, so the lanes
// of a warp read one segment's tables and run loops of the same length.
// Grid-stride over the device-side count.
// CTAs per SM of the FP64 pair pass: the most at which each field's FP64
// integrands compile without spills (vector potential 78 registers, field 96,
// gradient 122)
#ifndef CCOIL_REFINE_MIN_BLOCKS_B
#define CCOIL_REFINE_MIN_BLOCKS_B 5
#endif
constexpr int refineMinBlocks(int field)
{
    return field == CCOIL_FIELD_B ? CCOIL_REFINE_MIN_BLOCKS_B : (field == CCOIL_FIELD_G ? 4 : 6);
}
template <int FIELD>
__global__ void __launch_bounds__(128, refineMinBlocks(FIELD)) refinePairsKernel64(
    const unsigned char *__restrict__ blob, const SegmentDesc *__restrict__ segs, const double *__restrict__ points,
    double *__restrict__ out, const NearPair *__restrict__ work, unsigned long long workCapacity,
    const unsigned long long *__restrict__ workCount)
{
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    const unsigned long long n = min(*workCount, workCapacity);
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    {
        const NearPair e = work[i];
        const long long p = e.point;
        double acc[W];
#pragma unroll
        for (int k = 0; k < W; ++k)
            acc[k] = 0.0;
        integrateSegmentRefine<FIELD>(blob + segs[e.segment].offset, points[3 * p], points[3 * p + 1],
                                      points[3 * p + 2], acc);
#pragma unroll
        for (int k = 0; k < W; ++k)
            atomicAdd(&out[W * p + k], acc[k]);
    }
}

// FP32_REFINED selection.  A pair is picked when its stored contribution's
// norm exceeds `fraction` times the norm of the point's total (near-field FP64
// pairs included); a non-finite total picks nothing.  Both passes below make
// the same decision from the same data.
template <int W>
__device__ __forceinline__ bool refinePick(const double *total, const double *c, double fraction)
{
    double n2 = 0.0, c2 = 0.0;
#pragma unroll
    for (int i = 0; i < W; ++i)
    {
        n2 += total[i] * total[i];
        c2 += c[i] * c[i];
    }
    return c2 > fraction * fraction * n2;
}

// Pass 1, one thread per point: picks per segment (segCount, zeroed before).
// Whole warps iterate (base is the warp's first point), so each warp adds once
// per segment.
template <int W>
__global__ void __launch_bounds__(256) refineCountKernel(const double *__restrict__ out,
                                                         const double *__restrict__ contrib, long long npts, int nseg,
                                                         double fraction, unsigned long long *__restrict__ segCount)
{
    const int lane = threadIdx.x % 32;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < npts; base += stride)
    {
        const long long p = base + lane;
        const bool active = p < npts;
        double total[W];
#pragma unroll
        for (int i = 0; i < W; ++i)
            total[i] = active ? out[W * p + i] : 0.0;
        for (int s = 0; s < nseg; ++s)
        {
            double c[W];
#pragma unroll
            for (int i = 0; i < W; ++i)
                c[i] = active ? contrib[((size_t)s * (size_t)npts + (size_t)p) * W + i] : 0.0;
            const unsigned mask = __ballot_sync(0xffffffffu, active && refinePick<W>(total, c, fraction));
            if (mask != 0u && lane == 0)
                atomicAdd(&segCount[s], (unsigned long long)__popc(mask));
        }
    }
}

// Pass 2, one block: segCount becomes each segment's first list slot (exclusive
// prefix sum in segment order), *count the number of picks (the list length,
// read by the FP64 pass), *refined grows by the picks that fit the list.
__global__ void __launch_bounds__(1024) refineScanKernel(unsigned long long *__restrict__ segCount, int nseg,
                                                         unsigned long long capacity,
                                                         unsigned long long *__restrict__ count,
                                                         unsigned long long *__restrict__ refined)
{
    __shared__ unsigned long long part[1024];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0)
        carry = 0;
    __syncthreads();
    for (int base = 0; base < nseg; base += 1024)
    {
        const int s = base + threadIdx.x;
        const unsigned long long v = s < nseg ? segCount[s] : 0ull;
        part[threadIdx.x] = v;
        __syncthreads();
        // Hillis-Steele inclusive scan of the block's slice
        for (int off = 1; off < 1024; off *= 2)
        {
            const unsigned long long add = threadIdx.x >= off ? part[threadIdx.x - off] : 0ull;
            __syncthreads();
            part[threadIdx.x] += add;
            __syncthreads();
        }
        if (s < nseg)
            segCount[s] = carry + part[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023)
            carry += part[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        *count = carry;
        *refined += carry < capacity ? carry : capacity;
    }
}

// Pass 3, one thread per point: every picked pair takes the next slot of its
// segment's range (one atomic per warp and segment), is listed if the slot
// fits the list, and then leaves the point's total; the list comes out
// segment-major, so the FP64 pass's warps read one segment's tables.
template <int W>
__global__ void __launch_bounds__(256) refineSelectKernel(double *__restrict__ out,
                                                          const double *__restrict__ contrib, long long npts, int nseg,
                                                          double fraction, unsigned long long *__restrict__ segNext,
                                                          NearPair *__restrict__ work, unsigned long long capacity)
{
    const int lane = threadIdx.x % 32;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x - lane); base < npts; base += stride)
    {
        const long long p = base + lane;
        const bool active = p < npts;
        double total[W], picked[W];
#pragma unroll
        for (int i = 0; i < W; ++i)
        {
            total[i] = active ? out[W * p + i] : 0.0;
            picked[i] = 0.0;
        }
        for (int s = 0; s < nseg; ++s)
        {
            double c[W];
#pragma unroll
            for (int i = 0; i < W; ++i)
                c[i] = active ? contrib[((size_t)s * (size_t)npts + (size_t)p) * W + i] : 0.0;
            const bool pick = active && refinePick<W>(total, c, fraction);
            const unsigned mask = __ballot_sync(0xffffffffu, pick);
            if (mask == 0u)
                continue;
            unsigned long long first = 0;
            if (lane == 0)
                first = atomicAdd(&segNext[s], (unsigned long long)__popc(mask));
            first = __shfl_sync(0xffffffffu, first, 0);
            const unsigned long long slot = first + (unsigned long long)__popc(mask & ((1u << lane) - 1u));
            if (pick && slot < capacity)
            {
                work[slot].point = (int)p;
                work[slot].segment = s;
#pragma unroll
                for (int i = 0; i < W; ++i)
                    picked[i] += c[i];
            }
        }
        if (active)
        {
#pragma unroll
            for (int i = 0; i < W; ++i)
                out[W * p + i] = total[i] - picked[i];
        }
    }
}
