// Spatial target groups (cstone computeGroupSplits, cstone/traversal/groups_gpu.cu:58-137 and groups_gpu.cuh:37-216,
// used by the SPH propagators through sph::computeSpatialGroups, sph/include/sph/groups.hpp:41-55, tolFactor 2,
// groups of 32): the particles are cut into fixed runs of groupSize SFC-consecutive particles, and each run is split
// after every particle whose successor lies farther away than min(tolFactor * smallest leaf edge of the run, 2 h)
// (all lengths relative to the box). One warp per fixed run tests its 32 (or 64) consecutive distances with
// shuffles and a ballot; a scan of the per-run counts places the sub-groups, whose boundaries are then written
// directly (the reference writes their sizes and scans them; the boundaries are the same).
//
// The threshold arithmetic follows the reference exactly, in the precision of h (float with its default SphTypes,
// double in the FP64 build), because the split decisions are compared bit for bit with its kernel.
#include "groups.cuh"

namespace sphb
{
namespace
{

constexpr int kMaxTreeLevel = 21;

//! level of a cornerstone node from its key range (a power of 8; cstone treeLevel, sfc/common.hpp)
__device__ __forceinline__ int levelOfRange(uint64_t range) { return kMaxTreeLevel - (63 - __clzll(range)) / 3; }

//! first index i in [0, n) with layout[i] > v, minus one: the leaf holding particle v
__device__ __forceinline__ int leafOf(const uint32_t* layout, int n, uint32_t v)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (layout[mid] <= v) { lo = mid + 1; }
        else { hi = mid; }
    }
    return lo - 1;
}

template<class T>
__device__ __forceinline__ T loadH(const void* h, size_t i)
{
    return static_cast<const T*>(h)[i];
}

/*! One warp per fixed run of kN * 32 particles: masks[w] (kN words, bit b of word k: split after lane b of segment
 *  k) and counts[w] = 1 + number of splits. Lanes past `last` repeat the last particle (zero distance: no split). */
template<int kN, class T>
__global__ void groupSplitsKernel(size_t first, size_t last, const double* x, const double* y, const double* z,
                                  const void* h, const uint64_t* leaves, int numLeaves, const uint32_t* layout,
                                  DevBox box, float tolFactor, uint32_t* masks, int* counts)
{
    size_t warp   = (blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5;
    unsigned lane = threadIdx.x & 31;
    if (warp * kN * 32 >= last - first) { return; }

    size_t body[kN];
#pragma unroll
    for (int k = 0; k < kN; ++k)
    {
        body[k] = min(first + warp * kN * 32 + k * 32 + lane, last - 1);
    }
    // the smallest leaf volume of the run, in the unit box; the reference takes the leaf of the first segment's
    // particle for every segment (groups_gpu.cuh:188-193)
    int leaf0 = leafOf(layout, numLeaves, uint32_t(body[0]));
    T nodeVolume = T(1);
#pragma unroll
    for (int k = 0; k < kN; ++k)
    {
        int level    = levelOfRange(leaves[leaf0 + 1] - leaves[leaf0]);
        // centerAndSize in the unit box: half edge = (edge in integer units) * 0.5 / 2^21
        T halfUnit   = T(0.5) * (T(1) / T(1u << kMaxTreeLevel)) * T(1);
        T size       = T(1u << (kMaxTreeLevel - level)) * halfUnit;
        T vol        = 8 * size * size * size;
        nodeVolume   = min(vol, nodeVolume);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        nodeVolume = min(nodeVolume, __shfl_xor_sync(0xffffffffu, nodeVolume, off));
    }
    double distCrit = cbrt(nodeVolume) * tolFactor;

    double minExt = min(min(box.len[0], box.len[1]), box.len[2]);
    double px[kN], py[kN], pz[kN], ph[kN];
#pragma unroll
    for (int k = 0; k < kN; ++k)
    {
        px[k] = x[body[k]] * box.ilen[0];
        py[k] = y[body[k]] * box.ilen[1];
        pz[k] = z[body[k]] * box.ilen[2];
        ph[k] = h ? double(2) * double(loadH<T>(h, body[k])) / minExt : double(1);
    }
    double critSq = distCrit * distCrit;
#pragma unroll
    for (int k = 0; k < kN; ++k)
    {
        // the successor of each lane: the next lane, for lane 31 the first lane of the next segment (the last lane
        // of the last segment keeps itself: distance zero)
        double nx = __shfl_down_sync(0xffffffffu, px[k], 1);
        double ny = __shfl_down_sync(0xffffffffu, py[k], 1);
        double nz = __shfl_down_sync(0xffffffffu, pz[k], 1);
        if (k < kN - 1)
        {
            double sx = __shfl_sync(0xffffffffu, px[k + 1 < kN ? k + 1 : k], 0);
            double sy = __shfl_sync(0xffffffffu, py[k + 1 < kN ? k + 1 : k], 0);
            double sz = __shfl_sync(0xffffffffu, pz[k + 1 < kN ? k + 1 : k], 0);
            if (lane == 31)
            {
                nx = sx;
                ny = sy;
                nz = sz;
            }
        }
        double dx     = nx - px[k];
        double dy     = ny - py[k];
        double dz     = nz - pz[k];
        double distSq = dx * dx + dy * dy + dz * dz;
        bool split    = distSq > min(critSq, ph[k] * ph[k]);
        uint32_t mask = __ballot_sync(0xffffffffu, split);
        if (lane == 0) { masks[warp * kN + k] = mask; }
        ph[k] = __popc(mask); // reuse: split count of segment k
    }
    if (lane == 0)
    {
        int numSub = 1;
#pragma unroll
        for (int k = 0; k < kN; ++k)
        {
            numSub += int(ph[k]);
        }
        counts[warp] = numSub;
    }
}

//! boundaries of the sub-groups of fixed run w: its start, then one past every split, at offsets[w]
template<int kN>
__global__ void writeBoundsKernel(size_t first, size_t last, const uint32_t* masks, const int* offsets,
                                  size_t numFixed, uint32_t* bounds)
{
    size_t w = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (w > numFixed) { return; }
    if (w == numFixed)
    {
        bounds[offsets[numFixed]] = uint32_t(last);
        return;
    }
    size_t start = first + w * kN * 32;
    int o        = offsets[w];
    bounds[o++]  = uint32_t(start);
#pragma unroll
    for (int k = 0; k < kN; ++k)
    {
        uint32_t m = masks[w * kN + k];
        while (m)
        {
            int b       = __ffs(m) - 1;
            bounds[o++] = uint32_t(start + k * 32 + b + 1);
            m &= m - 1;
        }
    }
}

template<int kN, class T>
int splitsT(size_t first, size_t last, const double* x, const double* y, const double* z, const void* h,
            const uint64_t* leaves, int numLeaves, const uint32_t* layout, const DevBox& box, float tolFactor,
            DeviceBuffer<int>& scratch, DeviceBuffer<uint32_t>& bounds, unsigned* numGroups, cudaStream_t st)
{
    size_t numFixed = (last - first + kN * 32 - 1) / (kN * 32);
    // scratch: masks (kN per run), counts and their scan (numFixed + 1 each), scan temporaries
    size_t maskInts = numFixed * kN + 1;
    size_t need     = maskInts + 2 * (numFixed + 1) + scanTempInts(numFixed + 1);
    SPHB_TRY(scratch.reserve(need));
    uint32_t* masks = reinterpret_cast<uint32_t*>(scratch.data());
    int* counts     = scratch.data() + maskInts;
    int* offsets    = counts + numFixed + 1;
    int* tmp        = offsets + numFixed + 1;
    groupSplitsKernel<kN, T><<<ceilDiv(numFixed * 32, 256), 256, 0, st>>>(first, last, x, y, z, h, leaves,
                                                                          numLeaves, layout, box, tolFactor, masks,
                                                                          counts);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_TRY(exclusiveScan(counts, offsets, numFixed, tmp, st));
    int total = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&total, offsets + numFixed, sizeof(int), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    SPHB_TRY(bounds.reserve(size_t(total) + 1));
    writeBoundsKernel<kN><<<ceilDiv(numFixed + 1, 256), 256, 0, st>>>(first, last, masks, offsets, numFixed,
                                                                      bounds.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    *numGroups = unsigned(total);
    return kOk;
}

} // namespace

int computeGroupSplits(size_t first, size_t last, const double* x, const double* y, const double* z, const void* h,
                       int hType, const uint64_t* leaves, int numLeaves, const uint32_t* layout, const DevBox& box,
                       unsigned groupSize, float tolFactor, DeviceBuffer<int>& scratch, DeviceBuffer<uint32_t>& bounds,
                       unsigned* numGroups, cudaStream_t stream)
{
    if (last < first || numLeaves <= 0 || (hType != SPHB_F32 && hType != SPHB_F64)) { return kErrArg; }
    if (last == first)
    {
        SPHB_TRY(bounds.reserve(1));
        uint32_t v = uint32_t(last);
        SPHB_CUDA_TRY(cudaMemcpyAsync(bounds.data(), &v, sizeof(v), cudaMemcpyHostToDevice, stream));
        SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
        *numGroups = 0;
        return kOk;
    }
    bool f32 = hType == SPHB_F32;
    if (groupSize == 32)
    {
        return f32 ? splitsT<1, float>(first, last, x, y, z, h, leaves, numLeaves, layout, box, tolFactor, scratch,
                                       bounds, numGroups, stream)
                   : splitsT<1, double>(first, last, x, y, z, h, leaves, numLeaves, layout, box, tolFactor, scratch,
                                        bounds, numGroups, stream);
    }
    if (groupSize == 64)
    {
        return f32 ? splitsT<2, float>(first, last, x, y, z, h, leaves, numLeaves, layout, box, tolFactor, scratch,
                                       bounds, numGroups, stream)
                   : splitsT<2, double>(first, last, x, y, z, h, leaves, numLeaves, layout, box, tolFactor, scratch,
                                        bounds, numGroups, stream);
    }
    return kErrArg;
}

} // namespace sphb

extern "C" int sphb_compute_group_splits(size_t first, size_t last, const double* x, const double* y, const double* z,
                                         const void* h, int h_dtype, const uint64_t* leaves, size_t num_leaves,
                                         const uint32_t* layout, const sphb_box* box, unsigned group_size,
                                         float tol_factor, uint32_t* groups, size_t capacity, size_t* num_groups,
                                         void* stream)
{
    using namespace sphb;
    if (!box || !num_groups || !leaves || !layout || num_leaves == 0 || num_leaves >= (size_t(1) << 31)) { return SPHB_ERR_ARG; }
    if (last > first && (!x || !y || !z)) { return SPHB_ERR_ARG; }
    auto st = static_cast<cudaStream_t>(stream);
    DeviceBuffer<int> scratch;
    DeviceBuffer<uint32_t> bounds;
    unsigned num = 0;
    SPHB_TRY(computeGroupSplits(first, last, x, y, z, h, h_dtype, leaves, int(num_leaves), layout, makeDevBox(*box),
                                group_size, tol_factor, scratch, bounds, &num, st));
    *num_groups = num;
    if (groups && size_t(num) + 1 <= capacity)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(groups, bounds.data(), (size_t(num) + 1) * sizeof(uint32_t),
                                      cudaMemcpyDeviceToDevice, st));
    }
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    return groups && size_t(num) + 1 > capacity ? SPHB_ERR_CAPACITY : SPHB_OK;
}
