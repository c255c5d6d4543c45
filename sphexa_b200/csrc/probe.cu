// Measured CUDA-core FMA throughput (roofline denominator for the FP32 / FP64 neighbour sums).
#include "common.cuh"
#include "primitives.cuh"

namespace sphb
{

namespace
{

constexpr int kProbeChains = 8;   // independent FMA chains per thread hide the pipeline latency
constexpr int kProbeIters  = 4096;

template<class T>
__global__ void __launch_bounds__(256) fmaProbeKernel(T* out, T seed)
{
    T a[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
    {
        a[c] = seed + T(threadIdx.x + c);
    }
    const T mul = T(0.999999);
    const T add = T(1e-7);
#pragma unroll 16
    for (int it = 0; it < kProbeIters; ++it)
    {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c)
        {
            a[c] = fma(a[c], mul, add);
        }
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c)
    {
        s += a[c];
    }
    if (s == T(-1)) { out[blockIdx.x] = s; } // never true; keeps the chains live
}

//! the same FMA count in packed FP32 (sm_100 FFMA2): kProbeChains / 2 chains of float2
__global__ void __launch_bounds__(256) ffma2ProbeKernel(float* out, float seed)
{
    float2 a[kProbeChains / 2];
#pragma unroll
    for (int c = 0; c < kProbeChains / 2; ++c)
    {
        a[c] = make_float2(seed + float(threadIdx.x + 2 * c), seed + float(threadIdx.x + 2 * c + 1));
    }
    const float2 mul = make_float2(0.999999f, 0.999999f);
    const float2 add = make_float2(1e-7f, 1e-7f);
#pragma unroll 16
    for (int it = 0; it < kProbeIters; ++it)
    {
#pragma unroll
        for (int c = 0; c < kProbeChains / 2; ++c)
        {
            a[c] = __ffma2_rn(a[c], mul, add);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains / 2; ++c)
    {
        s += a[c].x + a[c].y;
    }
    if (s == -1.f) { out[blockIdx.x] = s; } // never true; keeps the chains live
}

template<class T, bool kPacked = false>
int probe(double* tflops)
{
    int blocks = smCount() * 8;
    T* out     = nullptr;
    SPHB_CUDA_TRY(cudaMalloc(&out, blocks * sizeof(T)));
    cudaEvent_t e0, e1;
    SPHB_CUDA_TRY(cudaEventCreate(&e0));
    SPHB_CUDA_TRY(cudaEventCreate(&e1));
    auto launch = [&]() {
        if constexpr (kPacked) { ffma2ProbeKernel<<<blocks, 256>>>(out, 1.0f); }
        else { fmaProbeKernel<T><<<blocks, 256>>>(out, T(1)); }
    };
    for (int w = 0; w < 3; ++w)
    {
        launch();
    }
    const int reps = 10;
    SPHB_CUDA_TRY(cudaEventRecord(e0));
    for (int r = 0; r < reps; ++r)
    {
        launch();
    }
    SPHB_CUDA_TRY(cudaEventRecord(e1));
    SPHB_CUDA_TRY(cudaEventSynchronize(e1));
    countLaunch(3 + reps);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    double flops = 2.0 * double(kProbeChains) * kProbeIters * 256.0 * blocks * reps;
    *tflops      = flops / (ms * 1e-3) / 1e12;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return kOk;
}

} // namespace

} // namespace sphb

extern "C" int sphb_probe_fma_peak(int which, double* tflops)
{
    if (!tflops || which < 0 || which > 2) { return SPHB_ERR_ARG; }
    if (which == 2) { return sphb::probe<float, true>(tflops); }
    return which == 0 ? sphb::probe<float>(tflops) : sphb::probe<double>(tflops);
}
