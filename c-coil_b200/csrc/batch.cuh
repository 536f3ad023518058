// Batched persistent field kernel (included by fields.cu inside its anonymous
// namespace, after fields32.cuh).
//
// Many independent coil systems of uneven size in one launch.  The host cuts
// every (system, field) into work items -- a tile of up to 128/L points of one
// system, L lanes per point -- and sorts them longest first.  A grid sized to
// the machine (CTAs per SM x 148) pulls items from an atomic counter until the
// list is exhausted, so long items start first and short ones fill the tail.
// An item reads its system's segment tables straight from global memory
// (through L1, as the single-system kernels do), so warps synchronise only to
// take the next item.  In FP32_COMPENSATED mode near-field pairs go to the
// work list with the field in the top bits of the segment index.

struct BatchItem
{
    int seg_begin;    // the system's segments [seg_begin, seg_end)
    int seg_end;
    int point_begin;  // first point of the item (global index)
    int point_count;  // points in the item (<= 128 / lanes)
    int lanes;        // 1, 4 or 32 threads per point
    int field;        // CCOIL_FIELD_A, _B, _E or _G
    int pad0, pad1;
};

constexpr int kFieldShift = 28;  // NearPair.segment = segment | field << 28

template <int PREC, int FIELD, int LANES>
__device__ __forceinline__ void batchItem(const BatchItem &I, const unsigned char *__restrict__ blob,
                                          const SegmentDesc *__restrict__ segs, const double *__restrict__ points,
                                          double *__restrict__ out, NearPair *__restrict__ work,
                                          unsigned long long workCapacity, unsigned long long *__restrict__ workCount)
{
    constexpr int W = FIELD == CCOIL_FIELD_G ? 9 : 3;
    const int lane = threadIdx.x % LANES;
    const int local = threadIdx.x / LANES;
    const bool active = local < I.point_count;
    const long long p = (long long)I.point_begin + local;
    const int nseg = I.seg_end - I.seg_begin;

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

    for (int s = 0; s < nseg && active; ++s)
    {
        const unsigned char *seg = blob + segs[I.seg_begin + s].offset;
        if (PREC == CCOIL_PRECISION_FP64)
            integrateSegment64<FIELD, LANES>(seg, px, py, pz, lane, acc);
        else
        {
            const SegmentHeader &h = *reinterpret_cast<const SegmentHeader *>(seg);
            const Frame f = toCoilFrame(h, px, py, pz);
            if (!nearWinding(h, f))
                integrateSegment32<FIELD, LANES>(seg, f, lane, acc);
            else
            {
                bool queued = false;
                if (lane == 0)
                {
                    unsigned long long slot = atomicAdd(workCount, 1ull);
                    if (slot < workCapacity)
                    {
                        work[slot].point = (int)p;
                        work[slot].segment = (I.seg_begin + s) | (FIELD << kFieldShift);
                        queued = true;
                    }
                }
                const unsigned groupMask = LANES == 32 ? 0xffffffffu
                                                       : (((1u << LANES) - 1u) << ((threadIdx.x % 32) / LANES * LANES));
                queued = __shfl_sync(groupMask, queued, (threadIdx.x % 32) / LANES * LANES);
                if (!queued)
                    integrateSegment64Fallback<FIELD, LANES>(seg, px, py, pz, lane, acc);
            }
        }
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

template <int PREC, int FIELD>
__device__ __forceinline__ void batchItemLanes(const BatchItem &I, const unsigned char *blob, const SegmentDesc *segs,
                                               const double *points, double *out, NearPair *work,
                                               unsigned long long cap, unsigned long long *count)
{
    switch (I.lanes)
    {
        case 1: batchItem<PREC, FIELD, 1>(I, blob, segs, points, out, work, cap, count); break;
        case 4: batchItem<PREC, FIELD, 4>(I, blob, segs, points, out, work, cap, count); break;
        default: batchItem<PREC, FIELD, 32>(I, blob, segs, points, out, work, cap, count); break;
    }
}

// CTAs per SM the register allocation targets, per precision.  FP32: 4
// (128 registers, no spills) measured best for B + G over 2,048 systems on
// B200: 2.00 s per step against 2.29 s at 5 and 2.54 s at 6
#ifndef CCOIL_BATCH_MIN_BLOCKS
#define CCOIL_BATCH_MIN_BLOCKS 5
#endif
#ifndef CCOIL_BATCH32_MIN_BLOCKS
#define CCOIL_BATCH32_MIN_BLOCKS 4
#endif

constexpr int batchMinBlocks(int prec)
{
    return prec == CCOIL_PRECISION_FP64 ? CCOIL_BATCH_MIN_BLOCKS : CCOIL_BATCH32_MIN_BLOCKS;
}

template <int PREC>
__global__ void __launch_bounds__(128, batchMinBlocks(PREC)) batchKernel(const unsigned char *__restrict__ blob,
                                                      const SegmentDesc *__restrict__ segs,
                                                      const BatchItem *__restrict__ items, int nitems,
                                                      unsigned *__restrict__ next, const double *__restrict__ points,
                                                      double *__restrict__ outA, double *__restrict__ outB,
                                                      double *__restrict__ outG, NearPair *__restrict__ work,
                                                      unsigned long long workCapacity,
                                                      unsigned long long *__restrict__ workCount)
{
    __shared__ int itemIndex;
    for (;;)
    {
        if (threadIdx.x == 0)
            itemIndex = (int)atomicAdd(next, 1u);
        __syncthreads();
        const int it = itemIndex;
        __syncthreads();  // every thread has read the index before it is replaced
        if (it >= nitems)
            break;
        const BatchItem I = items[it];
        if (I.field == CCOIL_FIELD_B)
            batchItemLanes<PREC, CCOIL_FIELD_B>(I, blob, segs, points, outB, work, workCapacity, workCount);
        else if (I.field == CCOIL_FIELD_G)
            batchItemLanes<PREC, CCOIL_FIELD_G>(I, blob, segs, points, outG, work, workCapacity, workCount);
        else
            batchItemLanes<PREC, CCOIL_FIELD_A>(I, blob, segs, points, outA, work, workCapacity, workCount);
    }
}

// near-field pass of the batched kernel: the field is in the segment's top bits
__global__ void __launch_bounds__(256) batchNearKernel(const unsigned char *__restrict__ blob,
                                                       const SegmentDesc *__restrict__ segs,
                                                       const double *__restrict__ points, double *__restrict__ outA,
                                                       double *__restrict__ outB, double *__restrict__ outG,
                                                       const NearPair *__restrict__ work,
                                                       unsigned long long workCapacity,
                                                       const unsigned long long *__restrict__ workCount)
{
    const unsigned long long n = min(*workCount, workCapacity);
    const int lane = threadIdx.x % 32;
    const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const unsigned long long warps = (unsigned long long)gridDim.x * blockDim.x / 32;
    for (unsigned long long i = warp; i < n; i += warps)
    {
        const NearPair e = work[i];
        const int field = e.segment >> kFieldShift;
        const int segIdx = e.segment & ((1 << kFieldShift) - 1);
        const unsigned char *seg = blob + segs[segIdx].offset;
        const long long p = e.point;
        double acc[9];
        for (int k = 0; k < 9; ++k)
            acc[k] = 0.0;
        const double px = points[3 * p], py = points[3 * p + 1], pz = points[3 * p + 2];
        int W;
        double *out;
        if (field == CCOIL_FIELD_G)
        {
            integrateSegment64<CCOIL_FIELD_G, 32>(seg, px, py, pz, lane, acc);
            W = 9;
            out = outG;
        }
        else if (field == CCOIL_FIELD_B)
        {
            integrateSegment64<CCOIL_FIELD_B, 32>(seg, px, py, pz, lane, acc);
            W = 3;
            out = outB;
        }
        else
        {
            integrateSegment64<CCOIL_FIELD_A, 32>(seg, px, py, pz, lane, acc);
            W = 3;
            out = outA;
        }
        for (int off = 16; off > 0; off /= 2)
            for (int k = 0; k < 9; ++k)
                acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], off);
        if (lane == 0)
            for (int k = 0; k < W; ++k)
                atomicAdd(&out[W * p + k], acc[k]);
    }
}

// Launch of one batched execution: counters reset, persistent kernel, near pass.
int launchBatchImpl(const BatchLaunch &B, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(B.d_next, 0, sizeof(unsigned), st);
    if (e == cudaSuccess && B.precision == CCOIL_PRECISION_FP32_COMPENSATED)
        e = cudaMemsetAsync(B.d_work_count, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess)
        return failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    if (B.nitems == 0)
        return CCOIL_OK;
    NearPair *work = reinterpret_cast<NearPair *>(B.d_work);
    const BatchItem *items = static_cast<const BatchItem *>(B.d_items);
    if (B.precision == CCOIL_PRECISION_FP64)
        batchKernel<CCOIL_PRECISION_FP64><<<B.grid, 128, 0, st>>>(B.d_blob, B.d_segs, items, B.nitems, B.d_next,
                                                                     B.d_points, B.d_outA, B.d_outB, B.d_outG, work,
                                                                     B.work_capacity, B.d_work_count);
    else
        batchKernel<CCOIL_PRECISION_FP32_COMPENSATED><<<B.grid, 128, 0, st>>>(
            B.d_blob, B.d_segs, items, B.nitems, B.d_next, B.d_points, B.d_outA, B.d_outB, B.d_outG, work,
            B.work_capacity, B.d_work_count);
    e = cudaGetLastError();
    if (e == cudaSuccess && B.precision == CCOIL_PRECISION_FP32_COMPENSATED)
    {
        batchNearKernel<<<148 * 8, 256, 0, st>>>(B.d_blob, B.d_segs, B.d_points, B.d_outA, B.d_outB, B.d_outG, work,
                                                 B.work_capacity, B.d_work_count);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? CCOIL_OK : failMessage(CCOIL_ERR_CUDA, cudaGetErrorString(e));
}
