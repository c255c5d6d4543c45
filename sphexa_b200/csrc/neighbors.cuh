// Fixed-count neighbour search with smoothing-length iteration (see neighbors.cu).
#pragma once

#include "common.cuh"

namespace sphb
{

//! read-only view of the focus tree used by the traversal (cstone OctreeNsView, cstone/tree/octree.hpp:258-281)
struct TreeView
{
    const int* childOffsets;
    const int* nodeToLeaf;
    const double* centers; // 3 per node
    const double* sizes;   // 3 per node
    const int* layout;     // first particle per leaf, numLeaves+1
    int numNodes;
};

/*! Neighbour lists are stored per group of 32 consecutive particles, slot-major: the k-th neighbour of particle
 *  i = 32 g + lane sits at nidx[(g * ngmax + k) * 32 + lane], so one slot of a warp is one 128-byte line. */
__host__ __device__ inline size_t nidxSlot(size_t group, unsigned ngmax, unsigned k, unsigned lane)
{
    return ((group * ngmax + k) << 5) + lane;
}

struct NeighborParams
{
    unsigned ng0;
    unsigned ngmax;
    int maxIterations; // smoothing-length updates (10 in the reference, sph/include/sph/find_neighbors.hpp:19)
};

/*! Search all particles: updates h where the count left [ng0/4, ngmax+1], writes nc (count incl. self) and lists.
 *  status[0] is set to a non-zero value if a per-warp buffer overflowed (the search then returns SPHB_ERR_CAPACITY). */
int findNeighbors(const double* x, const double* y, const double* z, double* h, size_t n, const TreeView& tree,
                  const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc, unsigned* status,
                  cudaStream_t stream);

} // namespace sphb
