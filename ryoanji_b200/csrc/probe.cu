/*
 * ryoanji-b200: calibration kernels for the roofline denominators that the driver's peak file does not carry.
 *
 * The traversal is bound by the FP32 pipe; its peak is measured here with independent FMA chains (one float FMA
 * per instruction, and the packed f32x2 FMA of sm_100a that issues two per instruction), at the clocks of the run.
 * A streaming copy gives an HBM figure measured the same way as the build kernels run.
 */
#include "internal.hpp"

namespace ryo
{

constexpr int kProbeChains = 8;

__global__ void __launch_bounds__(256) fmaChains(float* out, int iters, float a, float b)
{
    float v[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
        v[c] = threadIdx.x * 1e-3f + c;
    for (int i = 0; i < iters; ++i)
    {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c)
            v[c] = fmaf(v[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
        s += v[c];
    if (s == 1234.5f) out[threadIdx.x] = s; // keeps the chains alive
}

__global__ void __launch_bounds__(256) fma2Chains(float* out, int iters, float a, float b)
{
    unsigned long long v[kProbeChains];
    unsigned long long av, bv;
    asm("mov.b64 %0, {%1, %1};" : "=l"(av) : "f"(a));
    asm("mov.b64 %0, {%1, %1};" : "=l"(bv) : "f"(b));
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
    {
        float lo = threadIdx.x * 1e-3f + c, hi = lo + 0.5f;
        asm("mov.b64 %0, {%1, %2};" : "=l"(v[c]) : "f"(lo), "f"(hi));
    }
    for (int i = 0; i < iters; ++i)
    {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c)
            asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(v[c]) : "l"(av), "l"(bv));
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
    {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v[c]));
        s += lo + hi;
    }
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void copyKernel(const float4* __restrict__ in, float4* __restrict__ out, size_t n)
{
    size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = in[i];
}

//! FP32 peak in TFLOP/s (2 flops per FMA lane) for scalar FMA and packed f32x2 FMA, and copy GB/s (read + write)
void measurePeaks(int smCount, double* fp32, double* fp32x2, double* copyGBs, cudaStream_t s)
{
    float* out;
    RYO_CUDA(cudaMalloc(&out, 1024 * sizeof(float)));
    cudaEvent_t e0, e1;
    RYO_CUDA(cudaEventCreate(&e0));
    RYO_CUDA(cudaEventCreate(&e1));
    const int blocks = smCount * 8, threads = 256, iters = 1 << 14;
    auto timeIt = [&](auto launch) -> double
    {
        launch(); // warm-up
        RYO_CUDA(cudaEventRecord(e0, s));
        launch();
        RYO_CUDA(cudaEventRecord(e1, s));
        RYO_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        RYO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms * 1e-3;
    };
    double flops = double(blocks) * threads * iters * kProbeChains * 2.0;
    double t1 = timeIt([&] {
        fmaChains<<<blocks, threads, 0, s>>>(out, iters, 0.999f, 1e-3f);
        RYO_LAUNCH_CHECK();
    });
    double t2 = timeIt([&] {
        fma2Chains<<<blocks, threads, 0, s>>>(out, iters, 0.999f, 1e-3f);
        RYO_LAUNCH_CHECK();
    });
    *fp32   = flops / t1 * 1e-12;
    *fp32x2 = 2.0 * flops / t2 * 1e-12;

    size_t n = size_t(1) << 26; // 1 GiB per buffer
    float4 *a, *b;
    RYO_CUDA(cudaMalloc(&a, n * sizeof(float4)));
    RYO_CUDA(cudaMalloc(&b, n * sizeof(float4)));
    RYO_CUDA(cudaMemsetAsync(a, 0, n * sizeof(float4), s));
    double tc = timeIt([&] {
        copyKernel<<<smCount * 16, 256, 0, s>>>(a, b, n);
        RYO_LAUNCH_CHECK();
    });
    *copyGBs  = 2.0 * n * sizeof(float4) / tc * 1e-9;
    RYO_CUDA(cudaStreamSynchronize(s));
    cudaFree(a);
    cudaFree(b);
    cudaFree(out);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

} // namespace ryo
