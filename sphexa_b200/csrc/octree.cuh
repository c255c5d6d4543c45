// Cornerstone leaf trees and their linked octrees on the GPU (see octree.cu).
#pragma once

#include <vector>

#include "common.cuh"
#include "primitives.cuh"

namespace sphb
{

/*! Linked octree over a cornerstone leaf array, in the reference's node order (cstone/tree/octree.hpp:283-358):
 *  nodes sorted by placeholder-bit prefix, i.e. by level, then by key; children of a node are 8 consecutive
 *  nodes in key order. */
struct LinkedOctree
{
    int numLeaves{0};
    int numInternal{0};
    int numNodes{0};
    DeviceBuffer<uint64_t> prefixes;     // [numNodes] placeholder-bit keys
    DeviceBuffer<int> childOffsets;      // [numNodes] first child, 0 for leaves
    DeviceBuffer<int> parents;           // [(numNodes-1)/8] parent of each sibling group
    DeviceBuffer<int> nodeToLeaf;        // [numNodes] leaf index, negative for internal nodes
    DeviceBuffer<int> leafToNode;        // [numLeaves]
    DeviceBuffer<unsigned> nodeCounts;   // [numNodes] particles per node
    DeviceBuffer<double> centers;        // [3*numNodes] geometric centre (x,y,z interleaved)
    DeviceBuffer<double> sizes;          // [3*numNodes] half edge lengths
    DeviceBuffer<int> levelRangeD;       // [kMaxLevel + 2] the first node index per level
};

//! scratch shared by the tree routines
struct TreeScratch
{
    DeviceBuffer<int> ints;
    DeviceBuffer<int> ints2;
    DeviceBuffer<int> scanTmp;
    DeviceBuffer<uint64_t> keys;
    DeviceBuffer<char> sortTmp;
    DeviceBuffer<unsigned> flags; // small device status words
};

/*! Build (or rebuild) the linked octree of `leaves` (numLeaves + 1 keys, device) into `tree`. */
int buildLinkedOctree(const uint64_t* leaves, int numLeaves, LinkedOctree& tree, TreeScratch& s, cudaStream_t stream);

/*! counts[i] = number of sorted keys in [leaves[i], leaves[i+1]) (cstone/tree/csarray.hpp:76-86,181-235) */
int computeLeafCounts(const uint64_t* leaves, int numLeaves, const uint64_t* keys, size_t n, unsigned* counts,
                      cudaStream_t stream);

/*! node counts of every octree node from the leaf counts (sum over each node's leaf range) */
int computeNodeCounts(const uint64_t* leaves, const unsigned* leafCounts, LinkedOctree& tree, TreeScratch& s,
                      cudaStream_t stream);

/*! geometric centres and half sizes of every node inside `box` (cstone/focus/source_center.hpp:147-158) */
int computeGeoCenters(LinkedOctree& tree, const DevBox& box, cudaStream_t stream);

//! Global (domain-decomposition) cornerstone tree: leaves + counts, advanced by csarray rebalance steps.
struct GlobalTree
{
    DeviceBuffer<uint64_t> leaves;
    DeviceBuffer<uint64_t> leavesAlt;
    DeviceBuffer<unsigned> counts;
    int numLeaves{0};
    unsigned bucket{0};
    bool firstCall{true};
    std::vector<uint64_t> hostLeaves;
    bool hostStale{true}; // hostLeaves lag the device leaves
};

int initGlobalTree(GlobalTree& g, unsigned bucket, cudaStream_t stream);

/*! one updateOctreeGlobal step (cstone/tree/update_mpi.hpp:64-99): rebalance on the current counts, recount.
 *  Returns through *maxCount 0 if the decision changed nothing, else the largest leaf count. */
int globalTreeStep(GlobalTree& g, const uint64_t* keys, size_t n, TreeScratch& s, cudaStream_t stream,
                   unsigned* maxCount);

/*! GlobalAssignment::assign's tree part (cstone/domain/assignment.hpp:114-123) for sorted keys */
int updateGlobalTree(GlobalTree& g, const uint64_t* keys, size_t n, TreeScratch& s, cudaStream_t stream);

//! Focused (neighbour-search) tree at one rank: the whole key range is the focus area.
struct FocusTree
{
    DeviceBuffer<uint64_t> leaves;
    DeviceBuffer<uint64_t> leavesAlt;
    DeviceBuffer<unsigned> leafCounts;
    DeviceBuffer<int> layout; // [numLeaves+1] first particle of each leaf (exclusive scan of leafCounts)
    LinkedOctree tree;
    int numLeaves{0};
    unsigned bucket{64};
    bool firstCall{true};
};

int initFocusTree(FocusTree& f, unsigned bucket, TreeScratch& s, cudaStream_t stream);

/*! FocusedOctree::updateTree at one rank (cstone/focus/octree_focus_mpi.hpp:100-175 via
 *  CombinedUpdate::updateFocus, octree_focus.hpp:61-129): decision from the previous node counts, mandatory
 *  global leaves, ancestor protection, rebalance, forced injection if needed. *converged = tree unchanged. */
int focusUpdateTree(FocusTree& f, const GlobalTree& g, TreeScratch& s, cudaStream_t stream, bool* converged);

/*! FocusedOctree::updateCounts at one rank (octree_focus_mpi.hpp:192-251) + layout (cstone/domain/layout.hpp) */
int focusUpdateCounts(FocusTree& f, const uint64_t* keys, size_t n, TreeScratch& s, cudaStream_t stream);

} // namespace sphb
