// Hilbert space-filling-curve keys on sm_100a.
//
// One thread per particle, FP64 quantisation with every rounding step explicit (no FMA contraction), so the integer
// coordinates and keys are bit-identical to the reference's CPU path (cstone/sfc/sfc.hpp:141-178) compiled without
// floating-point contraction.
#include "common.cuh"
#include "sfc.cuh"

namespace sphb
{

__global__ void sfcKeysKernel(const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, uint64_t* __restrict__ keys, size_t n, DevBox box)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    if (keys[i] == kRemoveKey) { return; } // particles flagged for removal keep their key (sfc.hpp:271-274)
    keys[i] = hilbertKeyOf(x[i], y[i], z[i], box);
}

int launchSfcKeys(const double* x, const double* y, const double* z, uint64_t* keys, size_t n, const DevBox& box,
                  cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    sfcKeysKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(x, y, z, keys, n, box);
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

} // namespace sphb

extern "C" int sphb_compute_sfc_keys(const double* x, const double* y, const double* z, uint64_t* keys, size_t n,
                                     const sphb_box* box, void* stream)
{
    if (!box || (n && (!x || !y || !z || !keys))) { return SPHB_ERR_ARG; }
    return sphb::launchSfcKeys(x, y, z, keys, n, sphb::makeDevBox(*box), static_cast<cudaStream_t>(stream));
}
