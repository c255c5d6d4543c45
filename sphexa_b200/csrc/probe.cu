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

template<class T>
int probe(double* tflops)
{
    int blocks = smCount() * 8;
    T* out     = nullptr;
    SPHB_CUDA_TRY(cudaMalloc(&out, blocks * sizeof(T)));
    cudaEvent_t e0, e1;
    SPHB_CUDA_TRY(cudaEventCreate(&e0));
    SPHB_CUDA_TRY(cudaEventCreate(&e1));
    for (int w = 0; w < 3; ++w)
    {
        fmaProbeKernel<T><<<blocks, 256>>>(out, T(1));
    }
    const int reps = 10;
    SPHB_CUDA_TRY(cudaEventRecord(e0));
    for (int r = 0; r < reps; ++r)
    {
        fmaProbeKernel<T><<<blocks, 256>>>(out, T(1));
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
    if (!tflops || (which != 0 && which != 1)) { return SPHB_ERR_ARG; }
    return which == 0 ? sphb::probe<float>(tflops) : sphb::probe<double>(tflops);
}
