// TEST ORACLE ONLY (never shipped as product code): the reference's own spatial-group kernels, groupSplitsKernel and
// makeSplitsKernel of cstone/traversal/groups_gpu.cuh:117-216, compiled with nvcc from the reference headers where
// they lie (oracle/Makefile) and launched on the GPU as cstone::computeGroupSplitsImpl does
// (cstone/traversal/groups_gpu.cu:58-106). The two exclusive scans between them, which the reference runs with its
// CUB-based exclusiveScanGpu, run on the host here. Inputs and outputs are host arrays.
#include <cstdint>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "cstone/traversal/groups_gpu.cuh"

namespace
{

template<class T>
T* toDevice(const T* h, size_t n)
{
    T* d = nullptr;
    if (cudaMalloc(&d, (n ? n : 1) * sizeof(T)) != cudaSuccess) { return nullptr; }
    if (n) { cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice); }
    return d;
}

template<unsigned groupSize, class T>
int run(size_t first, size_t last, const double* x, const double* y, const double* z, const T* h,
        const uint64_t* leaves, int numLeaves, const unsigned* layout, const double* b, int pbc, float tolFactor,
        unsigned* out, size_t cap, size_t* numGroupsOut)
{
    using cstone::GpuConfig;
    using cstone::LocalIndex;
    using Mask = util::array<GpuConfig::ThreadMask, groupSize / GpuConfig::warpSize>;
    size_t n   = last;
    auto bt    = pbc ? cstone::BoundaryType::periodic : cstone::BoundaryType::open;
    cstone::Box<double> box(b[0], b[1], b[2], b[3], b[4], b[5], bt, bt, bt);

    double *dx = toDevice(x, n), *dy = toDevice(y, n), *dz = toDevice(z, n);
    T* dh                = h ? toDevice(h, n) : nullptr;
    uint64_t* dleaves    = toDevice(leaves, size_t(numLeaves) + 1);
    unsigned* dlayout    = toDevice(layout, size_t(numLeaves) + 1);
    LocalIndex numFixed  = (last - first + groupSize - 1) / groupSize;
    Mask* dmasks         = nullptr;
    LocalIndex* dsplits  = nullptr;
    cudaMalloc(&dmasks, (numFixed + 1) * sizeof(Mask));
    cudaMalloc(&dsplits, (numFixed + 1) * sizeof(LocalIndex));
    unsigned numThreads = 256;
    unsigned gridSize   = numFixed * GpuConfig::warpSize;
    if (numFixed > 0)
    {
        cstone::groupSplitsKernel<groupSize><<<(gridSize + numThreads - 1) / numThreads, numThreads>>>(
            LocalIndex(first), LocalIndex(last), dx, dy, dz, dh, dleaves, numLeaves, dlayout, box, tolFactor, dmasks,
            dsplits, numFixed);
    }
    std::vector<LocalIndex> splits(numFixed), offsets(numFixed + 1, 0);
    cudaMemcpy(splits.data(), dsplits, numFixed * sizeof(LocalIndex), cudaMemcpyDeviceToHost);
    std::exclusive_scan(splits.begin(), splits.end(), offsets.begin(), LocalIndex(0));
    offsets[numFixed]    = numFixed ? offsets[numFixed - 1] + splits[numFixed - 1] : 0;
    LocalIndex numGroups = offsets[numFixed];
    LocalIndex* doffsets = toDevice(offsets.data(), numFixed + 1);
    LocalIndex* dsizes   = nullptr;
    cudaMalloc(&dsizes, (numGroups + 1) * sizeof(LocalIndex));
    if (numFixed > 0) { cstone::makeSplitsKernel<<<numFixed, numThreads>>>(dmasks, doffsets, numFixed, dsizes); }
    std::vector<LocalIndex> sizes(numGroups), groups(numGroups + 1);
    cudaMemcpy(sizes.data(), dsizes, numGroups * sizeof(LocalIndex), cudaMemcpyDeviceToHost);
    std::exclusive_scan(sizes.begin(), sizes.end(), groups.begin(), LocalIndex(first));
    groups[numGroups] = LocalIndex(last);
    int rc            = cudaDeviceSynchronize() == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : 2;
    *numGroupsOut     = numGroups;
    if (rc == 0 && numGroups + 1 <= cap) { std::copy(groups.begin(), groups.end(), out); }
    for (void* p : {(void*)dx, (void*)dy, (void*)dz, (void*)dh, (void*)dleaves, (void*)dlayout, (void*)dmasks,
                    (void*)dsplits, (void*)doffsets, (void*)dsizes})
    {
        if (p) { cudaFree(p); }
    }
    return rc;
}

} // namespace

/*! Reference group boundaries (num_groups + 1 values into out when they fit). h_is_float: h holds float (the
 *  reference's default SphTypes) or double; h may be null. box6: xmin, xmax, ymin, ymax, zmin, zmax. */
extern "C" int ref_group_splits(size_t first, size_t last, const double* x, const double* y, const double* z,
                                const void* h, int h_is_float, const uint64_t* leaves, int num_leaves,
                                const unsigned* layout, const double* box6, int pbc, unsigned group_size,
                                float tol_factor, unsigned* out, size_t cap, size_t* num_groups)
{
    if (group_size == 32)
    {
        return h_is_float ? run<32, float>(first, last, x, y, z, static_cast<const float*>(h), leaves, num_leaves,
                                           layout, box6, pbc, tol_factor, out, cap, num_groups)
                          : run<32, double>(first, last, x, y, z, static_cast<const double*>(h), leaves, num_leaves,
                                            layout, box6, pbc, tol_factor, out, cap, num_groups);
    }
    if (group_size == 64)
    {
        return h_is_float ? run<64, float>(first, last, x, y, z, static_cast<const float*>(h), leaves, num_leaves,
                                           layout, box6, pbc, tol_factor, out, cap, num_groups)
                          : run<64, double>(first, last, x, y, z, static_cast<const double*>(h), leaves, num_leaves,
                                            layout, box6, pbc, tol_factor, out, cap, num_groups);
    }
    return 1;
}
