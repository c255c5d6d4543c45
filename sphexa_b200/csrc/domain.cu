// Halo discovery of one rank of a multi-rank domain on the shared global tree: the search box of every assigned
// leaf (its particles' coordinates widened by 2 h times the search extension) and the remote leaves it overlaps.
//
// The reference discovers halos on its focus tree (cstone::FocusedOctree::discoverHalos,
// domain/include/cstone/focus/octree_focus_mpi.hpp:513-571: computeBoundingBoxGpu, focus/source_center_gpu.cu:23-92,
// then findHalosGpu, traversal/collisions.hpp:40-104). Here every rank holds the same global cornerstone tree, so the
// leaves flagged are leaves of that tree and their indices mean the same on every rank.
#include <cstring>

#include "octree.cuh"
#include "neighbors.cuh"
#include "sfc.cuh"

namespace sphb
{
namespace
{

/*! search box of each assigned leaf, one warp per leaf: the smallest box holding the leaf's geometric centre and every
 *  particle's cube x +- r, r = h * scale rounded in h's own type (computeBoundingBox, focus/source_center.hpp:28-43,
 *  which starts its min/max from the leaf centre) */
template<class Th>
__global__ void searchBoxKernel(const double* x, const double* y, const double* z, const Th* h,
                                const uint32_t* layout, int firstLeaf, int numAssigned, const int* leafToNode,
                                const double* centers, Th scale, double* boxCenter, double* boxSize)
{
    int warp = int((blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (warp >= numAssigned) { return; }
    int node = leafToNode[firstLeaf + warp];
    double mn[3], mx[3];
    for (int k = 0; k < 3; ++k)
    {
        mn[k] = centers[3 * node + k];
        mx[k] = mn[k];
    }
    for (uint32_t i = layout[warp] + lane; i < layout[warp + 1]; i += 32)
    {
        double r    = double(Th(h[i] * scale));
        double p[3] = {x[i], y[i], z[i]};
        for (int k = 0; k < 3; ++k)
        {
            mn[k] = fmin(mn[k], p[k] - r);
            mx[k] = fmax(mx[k], p[k] + r);
        }
    }
    for (int off = 16; off > 0; off >>= 1)
    {
        for (int k = 0; k < 3; ++k)
        {
            mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], off));
            mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], off));
        }
    }
    if (lane == 0)
    {
        for (int k = 0; k < 3; ++k)
        {
            boxCenter[3 * warp + k] = __dmul_rn(__dadd_rn(mx[k], mn[k]), 0.5);
            boxSize[3 * warp + k]   = __dmul_rn(__dsub_rn(mx[k], mn[k]), 0.5);
        }
    }
}

//! the two boxes overlap, with the minimum image on periodic axes (overlap, traversal/boxoverlap.hpp:280-292)
__device__ inline bool boxesOverlap(const double* aCenter, const double* aSize, const double* bCenter,
                                    const double* bSize, const DevBox& box)
{
    bool all = true;
    for (int k = 0; k < 3; ++k)
    {
        double d = fabs(minImage(__dsub_rn(bCenter[k], aCenter[k]), box.len[k], box.ilen[k], box.periodic[k]));
        all      = all && __dsub_rn(__dsub_rn(d, aSize[k]), bSize[k]) < 0.0;
    }
    return all;
}

//! depth of the explicit traversal stack: 8 entries per level below the root (21 levels of 63-bit keys) and a margin
constexpr int kHaloStack = 8 * 22 + 8;

/*! one thread per assigned leaf: depth-first traversal of the linked octree from the root, descending into nodes that
 *  overlap the leaf's search box and are not inside the assigned key range [lowKey, highKey); every such leaf is
 *  flagged (findCollisions, traversal/collisions.hpp:23-47, with findHalos' exclusion of the assigned range) */
__global__ void findHalosKernel(const uint64_t* prefixes, const int* childOffsets, const int* nodeToLeaf,
                                const double* centers, const double* sizes, int numAssigned,
                                const double* boxCenter, const double* boxSize, DevBox box, uint64_t lowKey,
                                uint64_t highKey, uint8_t* leafFlags, unsigned* status)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= numAssigned) { return; }
    double tc[3] = {boxCenter[3 * t], boxCenter[3 * t + 1], boxCenter[3 * t + 2]};
    double ts[3] = {boxSize[3 * t], boxSize[3 * t + 1], boxSize[3 * t + 2]};
    int stack[kHaloStack];
    int sp      = 0;
    stack[sp++] = 0;
    while (sp > 0)
    {
        int node        = stack[--sp];
        uint64_t prefix = prefixes[node];
        uint64_t start  = prefixStart(prefix);
        uint64_t end    = start + nodeRangeAt(prefixLevel(prefix));
        if (start >= lowKey && end <= highKey) { continue; }
        if (!boxesOverlap(centers + 3 * node, sizes + 3 * node, tc, ts, box)) { continue; }
        int child = childOffsets[node];
        if (child == 0)
        {
            leafFlags[nodeToLeaf[node]] = 1;
            continue;
        }
        if (sp + 8 > kHaloStack)
        {
            atomicOr(status, 1u);
            return;
        }
        for (int c = 7; c >= 0; --c)
        {
            stack[sp++] = child + c;
        }
    }
}

} // namespace
} // namespace sphb

extern "C" int sphb_find_halos(const uint64_t* leaves, size_t num_leaves, const double* x, const double* y,
                               const double* z, const void* h, int h_dtype, const uint32_t* layout, size_t first_leaf,
                               size_t last_leaf, const sphb_box* box, float search_ext, uint8_t* flags, void* stream)
{
    using namespace sphb;
    if (!leaves || num_leaves == 0 || num_leaves >= (size_t(1) << 30) || !layout || !box || !flags ||
        first_leaf >= last_leaf || last_leaf > num_leaves || (h_dtype != SPHB_F32 && h_dtype != SPHB_F64) ||
        !(search_ext > 0.0f))
    {
        return SPHB_ERR_ARG;
    }
    for (int k = 0; k < 3; ++k)
    {
        if (!(box->hi[k] > box->lo[k])) { return SPHB_ERR_ARG; }
    }
    auto st        = static_cast<cudaStream_t>(stream);
    int numLeaves  = int(num_leaves);
    int numAssigned = int(last_leaf - first_leaf);
    uint32_t range[2];
    SPHB_CUDA_TRY(cudaMemcpyAsync(range, layout, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(range + 1, layout + numAssigned, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    uint64_t keyRange[2];
    SPHB_CUDA_TRY(cudaMemcpyAsync(keyRange, leaves + first_leaf, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(keyRange + 1, leaves + last_leaf, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    if (range[1] < range[0] || (range[1] > range[0] && (!x || !y || !z || !h))) { return SPHB_ERR_ARG; }

    LinkedOctree t;
    TreeScratch sc;
    SPHB_TRY(buildLinkedOctree(leaves, numLeaves, t, sc, st));
    DevBox dbox = makeDevBox(*box);
    SPHB_TRY(computeGeoCenters(t, dbox, st));
    DeviceBuffer<double> boxCenter, boxSize;
    DeviceBuffer<unsigned> status;
    SPHB_TRY(boxCenter.reserve(3 * size_t(numAssigned)));
    SPHB_TRY(boxSize.reserve(3 * size_t(numAssigned)));
    SPHB_TRY(status.reserve(1));
    SPHB_CUDA_TRY(cudaMemsetAsync(status.data(), 0, sizeof(unsigned), st));
    SPHB_CUDA_TRY(cudaMemsetAsync(flags, 0, num_leaves, st));

    unsigned blocks = ceilDiv(size_t(numAssigned) * 32, 256);
    // the reference's scale Th(2 * searchExtFact), with searchExtFact a float
    float scale = 2.0f * search_ext;
    if (h_dtype == SPHB_F32)
    {
        searchBoxKernel<float><<<blocks, 256, 0, st>>>(x, y, z, static_cast<const float*>(h), layout, int(first_leaf),
                                                       numAssigned, t.leafToNode.data(), t.centers.data(), scale,
                                                       boxCenter.data(), boxSize.data());
    }
    else
    {
        searchBoxKernel<double><<<blocks, 256, 0, st>>>(x, y, z, static_cast<const double*>(h), layout,
                                                        int(first_leaf), numAssigned, t.leafToNode.data(),
                                                        t.centers.data(), double(scale), boxCenter.data(),
                                                        boxSize.data());
    }
    countLaunch();
    findHalosKernel<<<ceilDiv(numAssigned, 128), 128, 0, st>>>(t.prefixes.data(), t.childOffsets.data(),
                                                               t.nodeToLeaf.data(), t.centers.data(), t.sizes.data(),
                                                               numAssigned, boxCenter.data(), boxSize.data(), dbox,
                                                               keyRange[0], keyRange[1], flags, status.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    unsigned err = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&err, status.data(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    return err ? SPHB_ERR_CAPACITY : SPHB_OK;
}
