// Host side of the batched launch: item list, autotuner, CUDA graph.
//
// A batch is a list of independent coil systems (the reference would make one
// CoilGroup per system and call computeAll*(points, GPU) per system,
// src/CoilGroup/Fields/CalculateFieldsGPU.cxx:11-196, one kernel per coil).
// Here every system and requested field is cut into work items that one
// persistent launch consumes (batch.cuh).  The launch sequence is captured in
// a CUDA graph per set of device pointers and replayed.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace ccoil
{
int cudaFail(cudaError_t e, const char *what);

namespace
{
struct Item
{
    int seg_begin, seg_end, point_begin, point_count, lanes, field, pad0, pad1;
};
static_assert(sizeof(Item) == kBatchItemBytes, "item layout");

struct Buf
{
    void *p = nullptr;
    size_t n = 0;
    int reserve(size_t bytes)
    {
        if (bytes <= n)
            return CCOIL_OK;
        if (p)
            cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess)
            return cudaFail(e, "cudaMalloc");
        n = bytes;
        return CCOIL_OK;
    }
    ~Buf()
    {
        if (p)
            cudaFree(p);
    }
};
} // namespace
} // namespace ccoil

using namespace ccoil;

struct ccoil_batch_plan
{
    int precision = 0;
    int fields_mask = 0;
    int systems = 0;
    long long points = 0;
    std::vector<int> sysSegBegin, sysSegEnd;
    std::vector<long long> sysPointBegin, sysPointEnd;
    std::vector<double> sysNodes;  // angular x thickness(-length) nodes summed over the system's coils
    SegmentSet set;
    Buf blob, segs, items, next, work, workCount;
    int nitems = 0;
    int split = 16;  // minimum items per (system, field) before lanes stop growing
    int grid = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t evIn = nullptr, evOut = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void *key[4] = {nullptr, nullptr, nullptr, nullptr};
    int keySplit = -1;
};

namespace
{
double fieldWeight(int f) { return f == CCOIL_FIELD_G ? 2.5 : f == CCOIL_FIELD_B ? 1.0 : 1.5; }

int buildItems(ccoil_batch_plan *P)
{
    std::vector<Item> items;
    std::vector<double> cost;
    for (int s = 0; s < P->systems; ++s)
    {
        const long long n = P->sysPointEnd[s] - P->sysPointBegin[s];
        if (n <= 0 || P->sysSegEnd[s] <= P->sysSegBegin[s])
            continue;
        for (int f : {CCOIL_FIELD_A, CCOIL_FIELD_B, CCOIL_FIELD_G})
        {
            if (!(P->fields_mask & (1 << f)))
                continue;
            // fewest lanes per point that still cut the system into `split` items
            int lanes = 1;
            for (int L : {1, 4, 32})
            {
                lanes = L;
                if ((n * L + 127) / 128 >= P->split)
                    break;
            }
            const int tile = 128 / lanes;
            for (long long b = 0; b < n; b += tile)
            {
                Item it{};
                it.seg_begin = P->sysSegBegin[s];
                it.seg_end = P->sysSegEnd[s];
                it.point_begin = (int)(P->sysPointBegin[s] + b);
                it.point_count = (int)std::min<long long>(tile, n - b);
                it.lanes = lanes;
                it.field = f;
                items.push_back(it);
                cost.push_back(P->sysNodes[s] * fieldWeight(f) * it.point_count / lanes);
            }
        }
    }
    // longest first
    std::vector<int> order(items.size());
    for (size_t i = 0; i < order.size(); ++i)
        order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<Item> sorted;
    sorted.reserve(items.size());
    for (int i : order)
        sorted.push_back(items[i]);
    P->nitems = (int)sorted.size();
    if (P->nitems == 0)
        return CCOIL_OK;
    int rc = P->items.reserve(sizeof(Item) * sorted.size());
    if (rc != CCOIL_OK)
        return rc;
    cudaError_t e = cudaMemcpy(P->items.p, sorted.data(), sizeof(Item) * sorted.size(), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? CCOIL_OK : cudaFail(e, "cudaMemcpy");
}

BatchLaunch launchOf(ccoil_batch_plan *P, const double *pts, double *a, double *b, double *g)
{
    BatchLaunch B;
    B.d_blob = static_cast<const unsigned char *>(P->blob.p);
    B.d_segs = static_cast<const SegmentDesc *>(P->segs.p);
    B.d_items = P->items.p;
    B.nitems = P->nitems;
    B.d_next = static_cast<unsigned *>(P->next.p);
    B.d_points = pts;
    B.d_outA = a;
    B.d_outB = b;
    B.d_outG = g;
    B.precision = P->precision;
    B.grid = P->grid;
    if (P->precision == CCOIL_PRECISION_FP32_COMPENSATED)
    {
        B.d_work = P->work.p;
        B.work_capacity = P->work.n / kNearPairBytes;
        B.d_work_count = static_cast<unsigned long long *>(P->workCount.p);
    }
    return B;
}

int zeroOutputs(ccoil_batch_plan *P, double *a, double *b, double *g, cudaStream_t st)
{
    // the near-field pass adds into the outputs; every point is also written by its item
    (void)P;
    (void)a;
    (void)b;
    (void)g;
    (void)st;
    return CCOIL_OK;
}
} // namespace

extern "C" {

int ccoil_batch_plan_create(const ccoil_coil_t *coils, const int *system_coil_offsets,
                            const long long *system_point_offsets, int system_count, int fields_mask, int precision,
                            ccoil_batch_plan_t **plan)
{
    if (!plan)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "plan is null");
    *plan = nullptr;
    if (system_count < 0 || (system_count > 0 && (!system_coil_offsets || !system_point_offsets)))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "system_count < 0 or null offsets");
    if (fields_mask <= 0 || (fields_mask & ~((1 << CCOIL_FIELD_A) | (1 << CCOIL_FIELD_B) | (1 << CCOIL_FIELD_G))))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "fields_mask must combine 1<<A, 1<<B and 1<<G");
    if (precision != CCOIL_PRECISION_FP64 && precision != CCOIL_PRECISION_FP32_COMPENSATED)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "precision must be FP64 or FP32_COMPENSATED");
    const int ncoils = system_count > 0 ? system_coil_offsets[system_count] : 0;
    const long long npts = system_count > 0 ? system_point_offsets[system_count] : 0;
    if (ncoils < 0 || npts < 0 || npts > 2147483647LL || (ncoils > 0 && !coils))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "bad totals: coils >= 0, 0 <= points < 2^31");
    for (int s = 0; s < system_count; ++s)
        if (system_coil_offsets[s] > system_coil_offsets[s + 1] || system_point_offsets[s] > system_point_offsets[s + 1] ||
            system_coil_offsets[s] < 0 || system_point_offsets[s] < 0)
            return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "system offsets must be non-decreasing from 0");

    ccoil_batch_plan *P = new (std::nothrow) ccoil_batch_plan();
    if (!P)
        return failMessage(CCOIL_ERR_OUT_OF_MEMORY, "host allocation failed");
    P->precision = precision;
    P->fields_mask = fields_mask;
    P->systems = system_count;
    P->points = npts;
    std::string err;
    if (!buildFieldSegments(coils, ncoils, CCOIL_FIELD_B, precision, P->set, err))
    {
        delete P;
        return fail(CCOIL_ERR_INVALID_ARGUMENT, err);
    }
    // map systems to their segment ranges (segments are emitted coil by coil)
    std::vector<int> coilFirstSeg(ncoils + 1, (int)P->set.segs.size());
    for (int i = (int)P->set.segs.size() - 1; i >= 0; --i)
        coilFirstSeg[P->set.segs[i].coil] = i;
    for (int c = ncoils - 1; c >= 0; --c)
        coilFirstSeg[c] = std::min(coilFirstSeg[c], coilFirstSeg[c + 1]);
    for (int s = 0; s < system_count; ++s)
    {
        P->sysSegBegin.push_back(coilFirstSeg[system_coil_offsets[s]]);
        P->sysSegEnd.push_back(coilFirstSeg[system_coil_offsets[s + 1]]);
        P->sysPointBegin.push_back(system_point_offsets[s]);
        P->sysPointEnd.push_back(system_point_offsets[s + 1]);
        double nodes = 0.0;
        for (int c = system_coil_offsets[s]; c < system_coil_offsets[s + 1]; ++c)
        {
            const ccoil_precision_args_t &p = coils[c].precision;
            nodes += double(p.angular_blocks) * p.angular_increments * p.thickness_blocks * p.thickness_increments *
                     (coils[c].use_fast_method ? 1.0 : double(p.length_blocks) * p.length_increments);
        }
        P->sysNodes.push_back(nodes);
    }
    int rc = CCOIL_OK;
    if (!P->set.segs.empty())
    {
        rc = P->blob.reserve(P->set.blob.size());
        if (rc == CCOIL_OK)
            rc = P->segs.reserve(sizeof(SegmentDesc) * P->set.segs.size());
        if (rc == CCOIL_OK)
        {
            cudaError_t e = cudaMemcpy(P->blob.p, P->set.blob.data(), P->set.blob.size(), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = cudaMemcpy(P->segs.p, P->set.segs.data(), sizeof(SegmentDesc) * P->set.segs.size(),
                               cudaMemcpyHostToDevice);
            if (e != cudaSuccess)
                rc = cudaFail(e, "cudaMemcpy");
        }
    }
    if (rc == CCOIL_OK)
        rc = P->next.reserve(256);
    if (rc == CCOIL_OK && precision == CCOIL_PRECISION_FP32_COMPENSATED)
    {
        rc = P->work.reserve(kNearPairBytes * (1u << 22));
        if (rc == CCOIL_OK)
            rc = P->workCount.reserve(sizeof(unsigned long long));
    }
    if (rc == CCOIL_OK)
        rc = buildItems(P);
    if (rc == CCOIL_OK)
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        P->grid = sms * batchBlocksPerSM(precision);
        cudaError_t e = cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&P->evIn, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&P->evOut, cudaEventDisableTiming);
        if (e != cudaSuccess)
            rc = cudaFail(e, "stream/event creation");
    }
    if (rc != CCOIL_OK)
    {
        ccoil_batch_plan_destroy(P);
        return rc;
    }
    *plan = P;
    return CCOIL_OK;
}

int ccoil_batch_plan_execute(ccoil_batch_plan_t *P, const double *points, double *out_a, double *out_b,
                             double *out_g, void *stream)
{
    if (!P)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "plan is null");
    if ((P->points > 0 && !points) || ((P->fields_mask & (1 << CCOIL_FIELD_A)) && !out_a) ||
        ((P->fields_mask & (1 << CCOIL_FIELD_B)) && !out_b) || ((P->fields_mask & (1 << CCOIL_FIELD_G)) && !out_g))
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "points and the requested outputs must be device pointers");
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    cudaError_t e;
    const void *key[4] = {points, out_a, out_b, out_g};
    if (!P->exec || std::memcmp(key, P->key, sizeof(key)) != 0 || P->keySplit != P->split)
    {
        if (P->exec)
        {
            cudaGraphExecDestroy(P->exec);
            P->exec = nullptr;
        }
        // capture the launch sequence once for these buffers
        cudaGraph_t graph = nullptr;
        e = cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess)
            return cudaFail(e, "begin capture");
        int rc = launchBatch(launchOf(P, points, out_a, out_b, out_g), P->stream);
        e = cudaStreamEndCapture(P->stream, &graph);
        if (rc != CCOIL_OK)
        {
            if (graph)
                cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess)
            return cudaFail(e, "end capture");
        e = cudaGraphInstantiate(&P->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess)
        {
            P->exec = nullptr;
            return cudaFail(e, "graph instantiate");
        }
        std::memcpy(P->key, key, sizeof(key));
        P->keySplit = P->split;
    }
    // order the graph after the caller's stream and the caller's stream after it
    e = cudaEventRecord(P->evIn, user);
    if (e == cudaSuccess)
        e = cudaStreamWaitEvent(P->stream, P->evIn, 0);
    if (e == cudaSuccess)
        e = cudaGraphLaunch(P->exec, P->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(P->evOut, P->stream);
    if (e == cudaSuccess)
        e = cudaStreamWaitEvent(user, P->evOut, 0);
    return e == cudaSuccess ? CCOIL_OK : cudaFail(e, "graph launch");
}

int ccoil_batch_plan_tune(ccoil_batch_plan_t *P, const double *points, double *out_a, double *out_b, double *out_g,
                          int *chosen_split, float *best_ms)
{
    if (!P)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "plan is null");
    // candidate minimum item counts per (system, field); each is timed on the real
    // batch (one warm-up, then the best of two graph launches) and the fastest kept
    const int candidates[] = {2, 8, 32, 128};
    int bestSplit = P->split;
    float best = 1e30f;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return failMessage(CCOIL_ERR_CUDA, "event creation failed");
    int rc = CCOIL_OK;
    for (int c : candidates)
    {
        P->split = c;
        rc = buildItems(P);
        if (rc != CCOIL_OK)
            break;
        rc = ccoil_batch_plan_execute(P, points, out_a, out_b, out_g, nullptr);
        if (rc != CCOIL_OK)
            break;
        float ms = 1e30f;
        for (int r = 0; r < 2; ++r)
        {
            cudaEventRecord(e0, P->stream);
            cudaGraphLaunch(P->exec, P->stream);
            cudaEventRecord(e1, P->stream);
            cudaEventSynchronize(e1);
            float t = 0.0f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        if (ms < best)
        {
            best = ms;
            bestSplit = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != CCOIL_OK)
        return rc;
    P->split = bestSplit;
    rc = buildItems(P);
    if (chosen_split)
        *chosen_split = bestSplit;
    if (best_ms)
        *best_ms = best;
    cudaError_t e = cudaDeviceSynchronize();
    return rc != CCOIL_OK ? rc : (e == cudaSuccess ? CCOIL_OK : cudaFail(e, "tune"));
}

int ccoil_batch_plan_set_split(ccoil_batch_plan_t *P, int split)
{
    if (!P || split < 1)
        return failMessage(CCOIL_ERR_INVALID_ARGUMENT, "plan null or split < 1");
    P->split = split;
    return buildItems(P);
}

int ccoil_batch_plan_destroy(ccoil_batch_plan_t *P)
{
    if (!P)
        return CCOIL_OK;
    if (P->stream)
        cudaStreamSynchronize(P->stream);
    if (P->exec)
        cudaGraphExecDestroy(P->exec);
    if (P->evIn)
        cudaEventDestroy(P->evIn);
    if (P->evOut)
        cudaEventDestroy(P->evOut);
    if (P->stream)
        cudaStreamDestroy(P->stream);
    delete P;
    return CCOIL_OK;
}

} // extern "C"
