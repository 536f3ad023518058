// Pipe-throughput microbenchmark used as the roofline denominators of the
// field kernels, which are bound by CUDA-core pipes (FP64 FMA, FP32 FMA, and
// the MUFU/XU special-function unit), not by HBM or the tensor cores.
//
// Each thread runs 8 independent dependency chains so the pipes, not the
// latency, limit the rate; the grid is 4 CTAs of 256 threads per SM.
#include "ccoil_internal.h"

#include <cuda_runtime.h>

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
