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
    const float4* blockLo; // per run of kBlockSize consecutive particles: bounding box relative to the box corner
    const float4* blockHi;
    int numNodes;
};

//! particles per bounding-box block used to prune the candidates of the search below leaf resolution
constexpr int kBlockSize = 8;

//! bounding boxes of the runs of kBlockSize consecutive particles (ceil(n / kBlockSize) entries each)
int computeBlockBoxes(const double* x, const double* y, const double* z, size_t n, const DevBox& box, float4* lo,
                      float4* hi, cudaStream_t stream);

//! neighbours per list chunk: one 32-byte sector of indices
constexpr unsigned kNbChunk = 8;

//! list capacity per particle rounded up to whole chunks
__host__ __device__ inline unsigned paddedNgmax(unsigned ngmax) { return (ngmax + kNbChunk - 1) / kNbChunk * kNbChunk; }

/*! Neighbour lists are stored per group of 32 consecutive particles in chunks of 8: the k-th neighbour of particle
 *  i = 32 g + lane sits at nidx[((g * (P/8) + k/8) * 32 + lane) * 8 + k%8], P = paddedNgmax(ngmax). Each chunk of a
 *  particle is one full 32-byte sector (written at once by the search, read with two 16-byte loads by the J-loops),
 *  and chunk row k/8 of a warp is 1 KB of contiguous memory. */
__host__ __device__ inline size_t nidxAt(size_t group, unsigned paddedNg, unsigned k, unsigned lane)
{
    return (((group * (paddedNg / kNbChunk) + k / kNbChunk) << 5) + lane) * kNbChunk + (k % kNbChunk);
}

struct NeighborParams
{
    unsigned ng0;
    unsigned ngmax;
    int maxIterations; // smoothing-length updates (10 in the reference, sph/include/sph/find_neighbors.hpp:19)
};

/*! Search all particles (x, y, z and the same coordinates packed as pos = (x, y, z, m)): updates h where the count left [ng0/4, ngmax+1], writes nc (count incl. self) and lists.
 *  status[0] is set to a non-zero value if a per-warp buffer overflowed (the search then returns SPHB_ERR_CAPACITY).
 *  An ensemble passes views (one tree per instance, on the device) and inst (instance per slot, kGhost for
 *  padding): each group searches its instance's tree, padding slots are skipped. */
int findNeighbors(const double* x, const double* y, const double* z, const double4* pos, double* h, size_t n,
                  const TreeView& tree, const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc,
                  unsigned* status, cudaStream_t stream, const TreeView* views = nullptr,
                  const uint8_t* inst = nullptr);

} // namespace sphb
