// Pipe-throughput microbenchmark used as the roofline denominators of the
// field kernels, which are bound by CUDA-core pipes (FP64 FMA, FP32 FMA, and
// the MUFU/XU special-function unit), not by HBM or the tensor cores.
//
// Each thread runs 8 independent dependency chains so the pipes, not the
// latency, limit the rate; the grid is 4 CTAs of 256 threads per SM.
// ccoil_measure_op_rates adds the rates of the FP64 divide, square root and
// logarithm the FP64 field kernels use, which expand to several FP64-pipe
// instructions each; the roofline model charges them at these measured rates.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

#include "fp64ops.cuh"
#include "log64.cuh"

namespace ccoil
{
namespace
{
constexpr int kChains = 8;

__global__ void fma64Kernel(double *sink, int iters, double a, double b)
{
    double v[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        v[i] = threadIdx.x * 1e-3 + i;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i)
            v[i] = fma(v[i], a, b);
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        s += v[i];
    if (s == 1.2345)  // never true; keeps the chains alive
        sink[0] = s;
}

__global__ void fma32Kernel(float *sink, int iters, float a, float b)
{
    float v[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        v[i] = threadIdx.x * 1e-3f + i;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i)
            v[i] = fmaf(v[i], a, b);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        s += v[i];
    if (s == 1.2345f)
        sink[0] = s;
}

// packed FP32 (sm_100 fma.rn.f32x2): one instruction, two FMAs
__global__ void fma32x2Kernel(float *sink, int iters, float a, float b)
{
    float2 v[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        v[i] = make_float2(threadIdx.x * 1e-3f + i, threadIdx.x * 2e-3f + i);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i)
            v[i] = __ffma2_rn(v[i], a2, b2);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        s += v[i].x + v[i].y;
    if (s == 1.2345f)
        sink[0] = s;
}

__global__ void mufuKernel(float *sink, int iters)
{
    float v[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        v[i] = 1.0f + threadIdx.x * 1e-3f + i;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i)
        {
            float r;
            asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v[i]));
            v[i] = r + 1.0f;
        }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        s += v[i];
    if (s == 1.2345f)
        sink[0] = s;
}

// One double-precision operation per chain and iteration, followed by one add
// that keeps the values in range (each iteration is a contraction with a fixed
// point near 1.6 - 3.2); the add's FP64 pipe slot is removed from the rate.
// OP 0: __ddiv_rn(1, v), 1: __dsqrt_rn(v), 2: log(v)
template <int OP>
__global__ void op64Kernel(double *sink, int iters)
{
    double v[kChains];
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        v[i] = 1.5 + threadIdx.x * 1e-4 + i * 1e-2;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int i = 0; i < kChains; ++i)
        {
            if (OP == 0)
                v[i] = __dadd_rn(__ddiv_rn(1.0, v[i]), 1.0);
            else if (OP == 1)
                v[i] = __dadd_rn(__dsqrt_rn(v[i]), 1.0);
            else
                v[i] = __dadd_rn(log64(v[i]), 2.0);  // the integrands' logarithm
        }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < kChains; ++i)
        s += v[i];
    if (s == 1.2345)
        sink[0] = s;
}

__global__ void log64Kernel(const double *__restrict__ x, double *__restrict__ out, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = log64(x[i]);
}

// op 0: 1/sqrt(a), 1: sqrt(a), 2: a / b, 3: log(a / b), by the FP64 forms of
// the refinement pass
__global__ void fp64OpKernel(int op, const double *__restrict__ a, const double *__restrict__ b,
                             double *__restrict__ out, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = op == 0 ? rsqrt64u(a[i]) : op == 1 ? sqrt64u(a[i]) : op == 2 ? div64u(a[i], b[i]) : logRatio64(a[i], b[i]);
}

template <typename Launch>
float timeIt(Launch launch)
{
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();  // warm-up
    cudaEventRecord(e0);
    launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}
} // namespace
} // namespace ccoil

using namespace ccoil;

extern "C" int ccoil_measure_op_rates(double *rates, int count)
{
    if (!rates || count < 6)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "rates needs at least 6 entries");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_NO_DEVICE, cudaGetErrorString(e));
    void *sink = nullptr;
    e = cudaMalloc(&sink, 64);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_OUT_OF_MEMORY, cudaGetErrorString(e));
    const int blocks = sms * 4, threads = 256;
    const double lanes = double(blocks) * threads * kChains;
    const int it64 = 4096, it32 = 16384, itMufu = 4096, itOp = 512;
    float ms64 = timeIt([&] { fma64Kernel<<<blocks, threads>>>((double *)sink, it64, 0.999999, 1e-7); });
    float ms32 = timeIt([&] { fma32Kernel<<<blocks, threads>>>((float *)sink, it32, 0.999999f, 1e-7f); });
    float msMu = timeIt([&] { mufuKernel<<<blocks, threads>>>((float *)sink, itMufu); });
    float msDiv = timeIt([&] { op64Kernel<0><<<blocks, threads>>>((double *)sink, itOp); });
    float msSqrt = timeIt([&] { op64Kernel<1><<<blocks, threads>>>((double *)sink, itOp); });
    float msLog = timeIt([&] { op64Kernel<2><<<blocks, threads>>>((double *)sink, itOp); });
    float ms32x2 = count > 6 ? timeIt([&] { fma32x2Kernel<<<blocks, threads>>>((float *)sink, it32, 0.999999f, 1e-7f); })
                             : 0.0f;
    e = cudaGetLastError();
    cudaFree(sink);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    const double dfma = lanes * it64 / (ms64 * 1e-3);  // FP64 pipe instructions per second
    const double opLanes = lanes * itOp;
    const double addSeconds = opLanes / dfma;           // the loop's own add per iteration
    auto rate = [&](float ms) {
        const double t = ms * 1e-3 - addSeconds;
        return t > 0.0 ? opLanes / t : 0.0;
    };
    rates[0] = dfma;
    rates[1] = rate(msDiv);
    rates[2] = rate(msSqrt);
    rates[3] = rate(msLog);
    rates[4] = lanes * it32 / (ms32 * 1e-3);             // FP32 FMA instructions per second
    rates[5] = lanes * itMufu / (msMu * 1e-3);           // MUFU rsqrt per second
    if (count > 6)
        rates[6] = lanes * it32 / (ms32x2 * 1e-3);       // packed FP32 FMA instructions (2 FMAs each) per second
    return CCOIL_OK;
}

extern "C" int ccoil_measure_pipe_peaks(double *fp64_tflops, double *fp32_tflops, double *mufu_tops)
{
    if (!fp64_tflops || !fp32_tflops || !mufu_tops)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "null output");
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_NO_DEVICE, cudaGetErrorString(e));
    void *sink = nullptr;
    e = cudaMalloc(&sink, 64);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_OUT_OF_MEMORY, cudaGetErrorString(e));
    const int blocks = sms * 4, threads = 256;
    const double lanes = double(blocks) * threads * kChains;
    const int it64 = 4096, it32 = 16384, itMufu = 4096;
    float ms64 = timeIt([&] { fma64Kernel<<<blocks, threads>>>((double *)sink, it64, 0.999999, 1e-7); });
    float ms32 = timeIt([&] { fma32Kernel<<<blocks, threads>>>((float *)sink, it32, 0.999999f, 1e-7f); });
    float msMu = timeIt([&] { mufuKernel<<<blocks, threads>>>((float *)sink, itMufu); });
    e = cudaGetLastError();
    cudaFree(sink);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_CUDA, cudaGetErrorString(e));
    *fp64_tflops = 2.0 * lanes * it64 / (ms64 * 1e-3) / 1e12;
    *fp32_tflops = 2.0 * lanes * it32 / (ms32 * 1e-3) / 1e12;
    *mufu_tops = lanes * itMufu / (msMu * 1e-3) / 1e12;
    return CCOIL_OK;
}

// grid-stride launch of an element-wise evaluation kernel over n elements,
// synchronous on the stream
template <typename Launch>
int evalElementwise(long long n, bool pointersOk, void *stream, Launch launch)
{
    if (n < 0 || (n > 0 && !pointersOk))
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "null input or output, or n < 0");
    if (n == 0)
        return CCOIL_OK;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
        return fail(CCOIL_ERR_NO_DEVICE, cudaGetErrorString(e));
    const long long want = (n + 255) / 256, cap = 8LL * sms;
    launch((unsigned)(want < cap ? want : cap), static_cast<cudaStream_t>(stream));
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? CCOIL_OK : fail(CCOIL_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" int ccoil_eval_log64(const double *x, double *out, long long n, void *stream)
{
    return evalElementwise(n, x && out, stream,
                           [&](unsigned grid, cudaStream_t st) { log64Kernel<<<grid, 256, 0, st>>>(x, out, n); });
}

extern "C" int ccoil_eval_fp64_op(int op, const double *a, const double *b, double *out, long long n, void *stream)
{
    if (op < 0 || op > 3)
        return fail(CCOIL_ERR_INVALID_ARGUMENT, "op must be 0 (rsqrt), 1 (sqrt), 2 (divide) or 3 (log of a ratio)");
    return evalElementwise(n, a && out && (op < 2 || b), stream, [&](unsigned grid, cudaStream_t st) {
        fp64OpKernel<<<grid, 256, 0, st>>>(op, a, b, out, n);
    });
}
