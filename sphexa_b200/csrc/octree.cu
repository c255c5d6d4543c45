// Cornerstone trees on the GPU: leaf counts, csarray rebalance (global tree), focus-tree update at one rank,
// the linked octree (level-major node order) and node geometry.
//
// The O(n) work (binary searches over the particle keys) and all O(nodes) decisions run as kernels; the host only
// reads a few status words per update to drive the convergence loops, as the reference's loops do
// (cstone/domain/assignment.hpp:114-123, cstone/focus/octree_focus_mpi.hpp:582-599).
#include <algorithm>
#include <cstring>
#include <vector>

#include "octree.cuh"
#include "sfc.cuh"
#include "sort.cuh"

namespace sphb
{

namespace
{

__device__ inline size_t lowerBound(const uint64_t* a, size_t n, uint64_t v)
{
    size_t lo = 0, hi = n;
    while (lo < hi)
    {
        size_t mid = (lo + hi) >> 1;
        if (a[mid] < v) { lo = mid + 1; }
        else { hi = mid; }
    }
    return lo;
}

//! level of the coarsest node that starts at key (number of leading octal digits up to the last non-zero one)
__host__ __device__ inline unsigned alignmentLevel(uint64_t key)
{
    if (key == 0) { return 0; }
#ifdef __CUDA_ARCH__
    unsigned tz = __ffsll((long long)key) - 1;
#else
    unsigned tz = __builtin_ctzll(key);
#endif
    return (63u - tz + 2u) / 3u;
}

__host__ __device__ inline unsigned octalDigitAt(uint64_t key, unsigned level)
{
    return unsigned(key >> (3u * (kMaxLevel - level))) & 7u;
}

// ---------------------------------------------------------------------------------------------------------------
// linked octree construction
// ---------------------------------------------------------------------------------------------------------------

__global__ void internalCountKernel(const uint64_t* leaves, int numLeaves, int* cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > numLeaves) { return; }
    if (i == numLeaves)
    {
        cnt[i] = 0;
        return;
    }
    uint64_t key   = leaves[i];
    unsigned level = treeLevelOf(leaves[i + 1] - key);
    unsigned a     = alignmentLevel(key);
    cnt[i]         = level > a ? int(level - a) : 0;
}

__global__ void emitNodesKernel(const uint64_t* leaves, int numLeaves, int numInternal, const int* offsets,
                                uint64_t* prefixes, uint32_t* ids)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numLeaves) { return; }
    uint64_t key   = leaves[i];
    unsigned level = treeLevelOf(leaves[i + 1] - key);
    unsigned a     = alignmentLevel(key);
    prefixes[numInternal + i] = encodePrefix(key, level);
    ids[numInternal + i]      = uint32_t(numInternal + i);
    int off                   = offsets[i];
    for (unsigned l = a; l < level && off < numInternal; ++l, ++off)
    {
        prefixes[off] = encodePrefix(key, l);
        ids[off]      = uint32_t(off);
    }
}

__global__ void mapNodesKernel(const uint32_t* ids, int numNodes, int numInternal, int* nodeToLeaf, int* leafToNode)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= numNodes) { return; }
    int leaf      = int(ids[p]) - numInternal;
    nodeToLeaf[p] = leaf;
    if (leaf >= 0) { leafToNode[leaf] = p; }
}

__global__ void levelRangeKernel(const uint64_t* prefixes, int numNodes, int* levelRange)
{
    int l = threadIdx.x;
    if (l <= int(kMaxLevel)) { levelRange[l] = int(lowerBound(prefixes, numNodes, uint64_t(1) << (3 * l))); }
    if (l == int(kMaxLevel) + 1) { levelRange[l] = numNodes; }
}

struct LevelRange
{
    int r[kMaxLevel + 2];
};

__global__ void linkKernel(const uint64_t* prefixes, const int* nodeToLeaf, int numNodes, const int* levelRange,
                           int* childOffsets, int* parents)
{
    __shared__ LevelRange lr;
    if (threadIdx.x < kMaxLevel + 2) { lr.r[threadIdx.x] = levelRange[threadIdx.x]; }
    __syncthreads();
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= numNodes) { return; }
    if (nodeToLeaf[p] >= 0)
    {
        childOffsets[p] = 0;
        return;
    }
    uint64_t prefix = prefixes[p];
    unsigned level  = prefixLevel(prefix);
    uint64_t child  = encodePrefix(prefixStart(prefix), level + 1);
    int b           = lr.r[level + 1];
    int e           = lr.r[level + 2];
    int c = b + int(lowerBound(prefixes + b, size_t(e - b), child));
    if (c >= e || c + 8 > numNodes || prefixes[c] != child)
    {
        childOffsets[p] = 0; // malformed leaf array: leave the node childless rather than link out of range
        return;
    }
    childOffsets[p]      = c;
    parents[(c - 1) / 8] = p;
}

// ---------------------------------------------------------------------------------------------------------------
// counts and geometry
// ---------------------------------------------------------------------------------------------------------------

__global__ void leafCountsKernel(const uint64_t* leaves, int numLeaves, const uint64_t* keys, size_t n,
                                 unsigned* counts)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= numLeaves) { return; }
    size_t b  = lowerBound(keys, n, leaves[i]);
    size_t e  = lowerBound(keys, n, leaves[i + 1]);
    counts[i] = unsigned(e - b);
}

__global__ void nodeCountsKernel(const uint64_t* prefixes, int numNodes, const uint64_t* leaves, int numLeaves,
                                 const int* leafScan, unsigned* nodeCounts)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= numNodes) { return; }
    uint64_t prefix = prefixes[p];
    unsigned level  = prefixLevel(prefix);
    uint64_t start  = prefixStart(prefix);
    uint64_t end    = start + nodeRangeAt(level);
    size_t b        = lowerBound(leaves, size_t(numLeaves) + 1, start);
    size_t e        = lowerBound(leaves, size_t(numLeaves) + 1, end);
    nodeCounts[p]   = unsigned(leafScan[e] - leafScan[b]);
}

__global__ void geoKernel(const uint64_t* prefixes, int numNodes, DevBox box, double* centers, double* sizes)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= numNodes) { return; }
    uint64_t prefix = prefixes[p];
    unsigned level  = prefixLevel(prefix);
    unsigned ixyz[3];
    hilbertDecode(prefixStart(prefix), ixyz);
    unsigned edge = (1u << kMaxLevel) >> level;
    unsigned mask = ~(edge - 1u);
    for (int k = 0; k < 3; ++k)
    {
        unsigned lo     = ixyz[k] & mask;
        unsigned hi     = lo + edge;
        double halfUnit = 0.5 * (1.0 / double(1u << kMaxLevel)) * box.len[k];
        centers[3 * p + k] = box.lo[k] + double(hi + lo) * halfUnit;
        sizes[3 * p + k]   = double(hi - lo) * halfUnit;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// global tree: csarray rebalance (cstone/tree/csarray.hpp:248-389)
// ---------------------------------------------------------------------------------------------------------------

__global__ void csNodeOpsKernel(const uint64_t* leaves, const unsigned* counts, int numLeaves, unsigned bucket,
                                int* ops, unsigned* flags)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > numLeaves) { return; }
    if (i == numLeaves)
    {
        ops[i] = 0;
        return;
    }
    uint64_t key   = leaves[i];
    unsigned level = treeLevelOf(leaves[i + 1] - key);
    int op         = 1;
    bool decided   = false;
    if (level > 0)
    {
        int sib = int(octalDigitAt(key, level));
        // the 8 siblings are all leaves if the group spans exactly one parent node
        bool siblings = sib > 0 && leaves[i - sib + 8] == leaves[i - sib] + nodeRangeAt(level - 1);
        if (siblings)
        {
            const unsigned* g = counts + i - sib;
            size_t parentCount = 0;
            for (int k = 0; k < 8; ++k)
            {
                parentCount += g[k];
            }
            if (parentCount <= size_t(bucket))
            {
                op      = 0;
                decided = true;
            }
        }
    }
    if (!decided)
    {
        unsigned c = counts[i];
        if (c > bucket * 512u && level + 3 < kMaxLevel) { op = 4096; }
        else if (c > bucket * 64u && level + 2 < kMaxLevel) { op = 512; }
        else if (c > bucket * 8u && level + 1 < kMaxLevel) { op = 64; }
        else if (c > bucket && level < kMaxLevel) { op = 8; }
    }
    ops[i] = op;
    if (op != 1) { atomicOr(flags, 1u); }
}

//! new leaves from scanned ops (processNode, cstone/tree/csarray.hpp:340-366)
__global__ void rebalanceKernel(const uint64_t* leaves, int numLeaves, const int* scan, uint64_t* newLeaves)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > numLeaves) { return; }
    if (i == numLeaves)
    {
        newLeaves[scan[numLeaves]] = leaves[numLeaves];
        return;
    }
    uint64_t key   = leaves[i];
    unsigned level = treeLevelOf(leaves[i + 1] - key);
    int op         = scan[i + 1] - scan[i];
    int out        = scan[i];
    if (op == 1) { newLeaves[out] = key; }
    else if (op > 1)
    {
        unsigned levelDiff = op == 8 ? 1 : op == 64 ? 2 : op == 512 ? 3 : 4;
        uint64_t step      = nodeRangeAt(level + levelDiff);
        for (int s = 0; s < op; ++s)
        {
            newLeaves[out + s] = key + uint64_t(s) * step;
        }
    }
}

__global__ void maxCountKernel(const unsigned* counts, int n, unsigned* flags)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned v = i < n ? counts[i] : 0u;
    for (int off = 16; off > 0; off >>= 1)
    {
        v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    if ((threadIdx.x & 31) == 0 && v) { atomicMax(flags + 1, v); }
}

// ---------------------------------------------------------------------------------------------------------------
// focus tree update at one rank (cstone/focus/rebalance.hpp, octree_focus.hpp:61-129)
// ---------------------------------------------------------------------------------------------------------------

enum Resolution : unsigned
{
    kConverged   = 0,
    kCancelMerge = 1,
    kRebalance   = 2,
    kFailed      = 3,
};

/*! mergeCountAndMacOp (rebalance.hpp:31-75) with the whole key range in focus: every node is inside the focus and
 *  every sibling group is in the fringe, so the MAC never decides and only particle counts do. */
__global__ void focusOpsKernel(const uint64_t* prefixes, const int* childOffsets, const int* parents,
                               const unsigned* counts, int numNodes, unsigned bucket, int* ops)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= numNodes) { return; }
    if (p > 0)
    {
        int parent = parents[(p - 1) / 8];
        if (counts[parent] <= bucket)
        {
            ops[p] = 0;
            return;
        }
    }
    unsigned level = prefixLevel(prefixes[p]);
    int op         = 1;
    if (childOffsets[p] == 0)
    {
        unsigned c = counts[p];
        if (level + 3 < kMaxLevel && c > 4096u * bucket) { op = 4096; }
        else if (level + 2 < kMaxLevel && c > 512u * bucket) { op = 512; }
        else if (level + 1 < kMaxLevel && c > 64u * bucket) { op = 64; }
        else if (level < kMaxLevel && c > bucket) { op = 8; }
    }
    ops[p] = op;
}

//! smallest existing node containing the node with placeholder-bit key `want` (octree.hpp:199-216)
__device__ int containingNodeOf(uint64_t want, const uint64_t* prefixes, const int* childOffsets)
{
    unsigned wantLevel = prefixLevel(want);
    uint64_t key       = prefixStart(want);
    int node           = 0;
    for (unsigned l = 1; l <= wantLevel; ++l)
    {
        if (childOffsets[node] == 0 || prefixes[node] == want) { break; }
        node = childOffsets[node] + int(octalDigitAt(key, l));
    }
    return node;
}

/*! enforceKeySingle (rebalance.hpp:161-212) for every mandatory key in parallel. Sibling resets only ever turn 0
 *  into 1 and splits take the maximum, so the final ops and the maximum status do not depend on key order. */
__global__ void enforceKeysKernel(const uint64_t* keys, int numKeys, const uint64_t* prefixes, const int* childOffsets,
                                  const int* parents, int* ops, unsigned* status)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= numKeys) { return; }
    uint64_t key = keys[t];
    if (key == 0 || key == kRootRange) { return; }

    unsigned lastNz    = kMaxLevel - unsigned(__ffsll((long long)key) - 1) / 3u;
    uint64_t want      = encodePrefix(key, lastNz);
    int node           = containingNodeOf(want, prefixes, childOffsets);
    uint64_t have      = prefixes[node];
    unsigned haveLevel = prefixLevel(have);

    unsigned st     = kConverged;
    bool trySplit   = have != want && haveLevel < kMaxLevel;
    bool undoMerges = ops[node] == 0 || trySplit;
    if (undoMerges && node > 0)
    {
        st         = kCancelMerge;
        int parent = node;
        do
        {
            parent    = parents[(parent - 1) / 8];
            int first = childOffsets[parent];
            for (int s = first; s < first + 8; ++s)
            {
                atomicCAS(ops + s, 0, 1); // 0 -> 1 only; must not undo a concurrent split of the same node
            }
        } while (parent != 0);
    }
    if (trySplit)
    {
        int levelDiff = int(lastNz) - int(haveLevel);
        st            = levelDiff > 1 ? kFailed : kRebalance;
        atomicMax(ops + node, 8);
    }
    if (st != kConverged) { atomicMax(status, st); }
}

//! nzAncestorOp (rebalance.hpp:96-116): merged nodes are kept only as the left-most descendant of a kept ancestor
__global__ void protectKernel(const uint64_t* prefixes, const int* parents, const int* opsIn, int numNodes,
                              int* opsOut, unsigned* numChanges)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= numNodes) { return; }
    int res;
    if (p == 0) { res = opsIn[0]; }
    else
    {
        int anc = p;
        while (opsIn[anc] == 0)
        {
            anc = parents[(anc - 1) / 8];
        }
        res = prefixStart(prefixes[p]) == prefixStart(prefixes[anc]) ? opsIn[anc] : 0;
    }
    opsOut[p] = res;
    if (res != 1) { atomicAdd(numChanges, 1u); }
}

__global__ void leafOpsKernel(const int* nodeOps, const int* leafToNode, int numLeaves, int* leafOps,
                              unsigned* numNotOne)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > numLeaves) { return; }
    if (i == numLeaves)
    {
        leafOps[i] = 0;
        return;
    }
    int op     = nodeOps[leafToNode[i]];
    leafOps[i] = op;
    if (op != 1) { atomicAdd(numNotOne, 1u); }
}

__global__ void setLeavesKernel(uint64_t* leaves, unsigned* counts, unsigned initialCount)
{
    leaves[0] = 0;
    leaves[1] = kRootRange;
    if (counts) { counts[0] = initialCount; }
}

//! the canonical cornerstone cover of [a, b): largest aligned nodes, greedy from a (host, used for key injection)
void spanRange(uint64_t a, uint64_t b, std::vector<uint64_t>& out)
{
    while (a < b)
    {
        unsigned level = alignmentLevel(a);
        while (a + nodeRangeAt(level) > b)
        {
            ++level;
        }
        out.push_back(a);
        a += nodeRangeAt(level);
    }
}

} // namespace

// -------------------------------------------------------------------------------------------------------------------

int buildLinkedOctree(const uint64_t* leaves, int numLeaves, LinkedOctree& t, TreeScratch& s, cudaStream_t stream)
{
    t.numLeaves   = numLeaves;
    t.numInternal = (numLeaves - 1) / 7;
    t.numNodes    = t.numLeaves + t.numInternal;
    int nn        = t.numNodes;

    SPHB_TRY(t.prefixes.reserve(nn));
    SPHB_TRY(t.childOffsets.reserve(nn + 1));
    SPHB_TRY(t.parents.reserve(std::max(1, (nn - 1) / 8)));
    SPHB_TRY(t.nodeToLeaf.reserve(nn));
    SPHB_TRY(t.leafToNode.reserve(numLeaves));
    SPHB_TRY(t.nodeCounts.reserve(nn));
    SPHB_TRY(t.centers.reserve(3 * size_t(nn)));
    SPHB_TRY(t.sizes.reserve(3 * size_t(nn)));
    SPHB_TRY(s.ints.reserve(std::max(numLeaves + 1, int(kMaxLevel) + 2)));
    SPHB_TRY(s.ints2.reserve(std::max(nn, numLeaves + 1) + 1));
    SPHB_TRY(s.scanTmp.reserve(scanTempInts(numLeaves + 1) + 1));
    SPHB_TRY(s.sortTmp.reserve(sortScratchBytes(nn)));

    unsigned nb = ceilDiv(numLeaves + 1, 256);
    internalCountKernel<<<nb, 256, 0, stream>>>(leaves, numLeaves, s.ints.data());
    SPHB_TRY(exclusiveScan(s.ints.data(), s.ints.data(), numLeaves, s.scanTmp.data(), stream));
    uint32_t* ids = reinterpret_cast<uint32_t*>(s.ints2.data());
    emitNodesKernel<<<ceilDiv(numLeaves, 256), 256, 0, stream>>>(leaves, numLeaves, t.numInternal, s.ints.data(),
                                                                 t.prefixes.data(), ids);
    countLaunch(2);
    SPHB_CUDA_TRY(cudaGetLastError());
    if (nn > 1)
    {
        SPHB_TRY(sortByKey(t.prefixes.data(), ids, nn, false, s.sortTmp.data(), s.sortTmp.capacity(), stream));
    }
    mapNodesKernel<<<ceilDiv(nn, 256), 256, 0, stream>>>(ids, nn, t.numInternal, t.nodeToLeaf.data(),
                                                         t.leafToNode.data());
    // the level ranges stay on the device: the link kernel reads them there (no host round trip per tree build)
    SPHB_TRY(t.levelRangeD.reserve(kMaxLevel + 2));
    levelRangeKernel<<<1, 32, 0, stream>>>(t.prefixes.data(), nn, t.levelRangeD.data());
    countLaunch(2);
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_CUDA_TRY(cudaMemsetAsync(t.parents.data(), 0, sizeof(int) * std::max(1, (nn - 1) / 8), stream));
    linkKernel<<<ceilDiv(nn, 256), 256, 0, stream>>>(t.prefixes.data(), t.nodeToLeaf.data(), nn,
                                                     t.levelRangeD.data(), t.childOffsets.data(), t.parents.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int computeLeafCounts(const uint64_t* leaves, int numLeaves, const uint64_t* keys, size_t n, unsigned* counts,
                      cudaStream_t stream)
{
    leafCountsKernel<<<ceilDiv(numLeaves, 256), 256, 0, stream>>>(leaves, numLeaves, keys, n, counts);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int computeNodeCounts(const uint64_t* leaves, const unsigned* leafCounts, LinkedOctree& t, TreeScratch& s,
                      cudaStream_t stream)
{
    SPHB_TRY(s.ints.reserve(t.numLeaves + 1));
    SPHB_TRY(s.scanTmp.reserve(scanTempInts(t.numLeaves + 1) + 1));
    SPHB_TRY(exclusiveScan(reinterpret_cast<const int*>(leafCounts), s.ints.data(), t.numLeaves, s.scanTmp.data(),
                           stream));
    nodeCountsKernel<<<ceilDiv(t.numNodes, 256), 256, 0, stream>>>(t.prefixes.data(), t.numNodes, leaves,
                                                                  t.numLeaves, s.ints.data(), t.nodeCounts.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int computeGeoCenters(LinkedOctree& t, const DevBox& box, cudaStream_t stream)
{
    geoKernel<<<ceilDiv(t.numNodes, 256), 256, 0, stream>>>(t.prefixes.data(), t.numNodes, box, t.centers.data(),
                                                           t.sizes.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

// -------------------------------------------------------------------------------------------------------------------

int initGlobalTree(GlobalTree& g, unsigned bucket, cudaStream_t stream)
{
    // one root leaf with count bucket-1 (GlobalAssignment constructor, cstone/domain/assignment.hpp:57-74)
    g.bucket    = bucket;
    g.numLeaves = 1;
    g.firstCall = true;
    g.hostStale = true;
    SPHB_TRY(g.leaves.reserve(2));
    SPHB_TRY(g.counts.reserve(1));
    setLeavesKernel<<<1, 1, 0, stream>>>(g.leaves.data(), g.counts.data(), bucket - 1);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int globalTreeStep(GlobalTree& g, const uint64_t* keys, size_t n, TreeScratch& s, cudaStream_t stream,
                   unsigned* maxCount)
{
    int L = g.numLeaves;
    SPHB_TRY(s.ints.reserve(L + 2));
    SPHB_TRY(s.scanTmp.reserve(scanTempInts(L + 1) + 1));
    SPHB_TRY(s.flags.reserve(4));
    SPHB_CUDA_TRY(cudaMemsetAsync(s.flags.data(), 0, 4 * sizeof(unsigned), stream));
    csNodeOpsKernel<<<ceilDiv(L + 1, 256), 256, 0, stream>>>(g.leaves.data(), g.counts.data(), L, g.bucket,
                                                             s.ints.data(), s.flags.data());
    countLaunch();
    SPHB_TRY(exclusiveScan(s.ints.data(), s.ints.data(), L + 1, s.scanTmp.data(), stream));
    // the counts of the current leaves, before knowing whether they change: in the steady state nothing splits or
    // merges and one read back serves both decisions
    SPHB_TRY(computeLeafCounts(g.leaves.data(), L, keys, n, g.counts.data(), stream));
    maxCountKernel<<<ceilDiv(L, 256), 256, 0, stream>>>(g.counts.data(), L, s.flags.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    unsigned msg[3]; // new leaf count, any op, largest count
    SPHB_TRY(readBack(stream, {{msg, s.ints.data() + L, sizeof(int)}, {msg + 1, s.flags.data(), 2 * sizeof(unsigned)}}));
    int newL       = int(msg[0]);
    unsigned anyOp = msg[1];
    if (anyOp)
    {
        // every op 1 would give the same leaves: the rebalance runs only when a node splits or merges
        SPHB_TRY(g.leavesAlt.reserve(newL + 1));
        rebalanceKernel<<<ceilDiv(L + 1, 256), 256, 0, stream>>>(g.leaves.data(), L, s.ints.data(),
                                                                 g.leavesAlt.data());
        countLaunch();
        SPHB_CUDA_TRY(cudaGetLastError());
        g.leaves.swap(g.leavesAlt);
        g.numLeaves = newL;
        g.hostStale = true;
        SPHB_TRY(g.counts.reserve(newL));
        SPHB_TRY(computeLeafCounts(g.leaves.data(), newL, keys, n, g.counts.data(), stream));
        SPHB_CUDA_TRY(cudaMemsetAsync(s.flags.data() + 1, 0, sizeof(unsigned), stream));
        maxCountKernel<<<ceilDiv(newL, 256), 256, 0, stream>>>(g.counts.data(), newL, s.flags.data());
        countLaunch();
        SPHB_CUDA_TRY(cudaGetLastError());
        SPHB_TRY(readBack(stream, {{msg + 2, s.flags.data() + 1, sizeof(unsigned)}}));
    }
    *maxCount = anyOp ? msg[2] : 0u;
    return kOk;
}

int updateGlobalTree(GlobalTree& g, const uint64_t* keys, size_t n, TreeScratch& s, cudaStream_t stream)
{
    if (g.hostLeaves.empty()) { g.hostStale = true; }
    unsigned maxCount = 0;
    SPHB_TRY(globalTreeStep(g, keys, n, s, stream, &maxCount));
    if (g.firstCall || maxCount >= 8 * g.bucket)
    {
        g.firstCall = false;
        int guard   = 0;
        do
        {
            SPHB_TRY(globalTreeStep(g, keys, n, s, stream, &maxCount));
            if (++guard > 64) { return kErrNotConverged; }
        } while (maxCount > g.bucket);
    }
    if (g.hostStale)
    {
        // the host copy of the leaves (mandatory keys of a failed focus update) follows only changes
        g.hostLeaves.resize(g.numLeaves + 1);
        SPHB_CUDA_TRY(cudaMemcpyAsync(g.hostLeaves.data(), g.leaves.data(), (g.numLeaves + 1) * sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost, stream));
        SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
        g.hostStale = false;
    }
    return kOk;
}

// -------------------------------------------------------------------------------------------------------------------

int initFocusTree(FocusTree& f, unsigned bucket, TreeScratch& s, cudaStream_t stream)
{
    // FocusedOctree constructor (octree_focus_mpi.hpp:63-88): root leaf, counts bucket+1
    f.bucket    = bucket;
    f.numLeaves = 1;
    f.firstCall = true;
    SPHB_TRY(f.leaves.reserve(2));
    SPHB_TRY(f.leafCounts.reserve(1));
    SPHB_TRY(f.layout.reserve(2));
    setLeavesKernel<<<1, 1, 0, stream>>>(f.leaves.data(), f.leafCounts.data(), bucket + 1);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_TRY(buildLinkedOctree(f.leaves.data(), 1, f.tree, s, stream));
    unsigned c = bucket + 1;
    SPHB_CUDA_TRY(cudaMemcpyAsync(f.tree.nodeCounts.data(), &c, sizeof(unsigned), cudaMemcpyHostToDevice, stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
    return kOk;
}

int focusUpdateTree(FocusTree& f, const GlobalTree& g, TreeScratch& s, cudaStream_t stream, bool* converged)
{
    LinkedOctree& t = f.tree;
    int nn          = t.numNodes;
    int L           = f.numLeaves;
    SPHB_TRY(s.ints.reserve(nn + L + 2));
    SPHB_TRY(s.ints2.reserve(nn + L + 2));
    SPHB_TRY(s.scanTmp.reserve(scanTempInts(L + 1) + 1));
    SPHB_TRY(s.flags.reserve(4));
    int* ops    = s.ints.data();
    int* opsOut = s.ints2.data();
    SPHB_CUDA_TRY(cudaMemsetAsync(s.flags.data(), 0, 4 * sizeof(unsigned), stream));

    focusOpsKernel<<<ceilDiv(nn, 256), 256, 0, stream>>>(t.prefixes.data(), t.childOffsets.data(), t.parents.data(),
                                                         t.nodeCounts.data(), nn, f.bucket, ops);
    // mandatory keys: the global leaves (the focus start 0 and end 2^63 are always converged)
    enforceKeysKernel<<<ceilDiv(g.numLeaves + 1, 128), 128, 0, stream>>>(
        g.leaves.data(), g.numLeaves + 1, t.prefixes.data(), t.childOffsets.data(), t.parents.data(), ops,
        s.flags.data());
    protectKernel<<<ceilDiv(nn, 256), 256, 0, stream>>>(t.prefixes.data(), t.parents.data(), ops, nn, opsOut,
                                                        s.flags.data() + 1);
    int* leafOps = ops; // node ops no longer needed
    leafOpsKernel<<<ceilDiv(L + 1, 256), 256, 0, stream>>>(opsOut, t.leafToNode.data(), L, leafOps,
                                                           s.flags.data() + 2);
    countLaunch(4);
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_TRY(exclusiveScan(leafOps, leafOps, L + 1, s.scanTmp.data(), stream));
    int newL = 0;
    unsigned flags[3];
    SPHB_TRY(readBack(stream, {{&newL, leafOps + L, sizeof(int)}, {flags, s.flags.data(), sizeof(flags)}}));
    unsigned status = flags[0];
    bool conv       = flags[1] == 0;
    if (status == kCancelMerge) { conv = flags[2] == 0; }
    else if (status == kRebalance) { conv = false; }
    if (status != kFailed && flags[2] == 0 && newL == L)
    {
        // every leaf keeps its op 1: the leaves, and so the linked octree, stay as they are
        *converged = conv;
        return kOk;
    }

    SPHB_TRY(f.leavesAlt.reserve(newL + 1));
    rebalanceKernel<<<ceilDiv(L + 1, 256), 256, 0, stream>>>(f.leaves.data(), L, leafOps, f.leavesAlt.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    f.leaves.swap(f.leavesAlt);
    f.numLeaves = newL;

    if (status == kFailed)
    {
        // injectKeys (cstone/focus/inject.hpp): merge the spanning tree of the mandatory keys into the leaves
        conv = false;
        std::vector<uint64_t> leaves(newL + 1);
        SPHB_CUDA_TRY(cudaMemcpyAsync(leaves.data(), f.leaves.data(), (newL + 1) * sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost, stream));
        SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
        std::vector<uint64_t> mand(g.hostLeaves.begin(), g.hostLeaves.end());
        mand.push_back(0);
        mand.push_back(kRootRange);
        std::sort(mand.begin(), mand.end());
        mand.erase(std::unique(mand.begin(), mand.end()), mand.end());
        std::vector<uint64_t> span;
        for (size_t k = 0; k + 1 < mand.size(); ++k)
        {
            spanRange(mand[k], mand[k + 1], span);
        }
        span.push_back(kRootRange);
        leaves.insert(leaves.end(), span.begin(), span.end());
        std::sort(leaves.begin(), leaves.end());
        leaves.erase(std::unique(leaves.begin(), leaves.end()), leaves.end());
        newL = int(leaves.size()) - 1;
        SPHB_TRY(f.leaves.reserve(newL + 1));
        SPHB_CUDA_TRY(cudaMemcpyAsync(f.leaves.data(), leaves.data(), leaves.size() * sizeof(uint64_t),
                                      cudaMemcpyHostToDevice, stream));
        SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
        f.numLeaves = newL;
    }
    SPHB_TRY(buildLinkedOctree(f.leaves.data(), f.numLeaves, f.tree, s, stream));
    *converged = conv;
    return kOk;
}

int focusUpdateCounts(FocusTree& f, const uint64_t* keys, size_t n, TreeScratch& s, cudaStream_t stream)
{
    int L = f.numLeaves;
    SPHB_TRY(f.leafCounts.reserve(L));
    SPHB_TRY(f.layout.reserve(L + 1));
    SPHB_TRY(s.scanTmp.reserve(scanTempInts(L + 1) + 1));
    SPHB_TRY(computeLeafCounts(f.leaves.data(), L, keys, n, f.leafCounts.data(), stream));
    SPHB_TRY(computeNodeCounts(f.leaves.data(), f.leafCounts.data(), f.tree, s, stream));
    SPHB_TRY(exclusiveScan(reinterpret_cast<const int*>(f.leafCounts.data()), f.layout.data(), L, s.scanTmp.data(),
                           stream));
    return kOk;
}

} // namespace sphb

extern "C" int sphb_compute_octree(const uint64_t* sorted_keys, size_t n, unsigned bucket, uint64_t* leaves,
                                   uint32_t* counts, size_t capacity, size_t* num_leaves, void* stream)
{
    using namespace sphb;
    if (!num_leaves || bucket == 0 || (n && !sorted_keys)) { return SPHB_ERR_ARG; }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // computeOctree (csarray.hpp:432-440): start from the root with count n and step until no change
    GlobalTree g;
    TreeScratch s;
    SPHB_TRY(initGlobalTree(g, bucket, st));
    unsigned c = unsigned(n);
    SPHB_CUDA_TRY(cudaMemcpyAsync(g.counts.data(), &c, sizeof(unsigned), cudaMemcpyHostToDevice, st));
    unsigned maxCount = 1;
    int guard         = 0;
    while (maxCount != 0)
    {
        SPHB_TRY(globalTreeStep(g, sorted_keys, n, s, st, &maxCount));
        if (++guard > 1000) { return SPHB_ERR_NOT_CONVERGED; }
        if (maxCount == 0) { break; }
    }
    *num_leaves = size_t(g.numLeaves);
    if (size_t(g.numLeaves) + 1 <= capacity && leaves && counts)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(leaves, g.leaves.data(), (g.numLeaves + 1) * sizeof(uint64_t),
                                      cudaMemcpyDeviceToDevice, st));
        SPHB_CUDA_TRY(cudaMemcpyAsync(counts, g.counts.data(), g.numLeaves * sizeof(unsigned),
                                      cudaMemcpyDeviceToDevice, st));
    }
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    return size_t(g.numLeaves) + 1 <= capacity ? SPHB_OK : SPHB_ERR_CAPACITY;
}

// ------------------------------------------------------------------------------------------------------------------
// The linked octree in the reference's OctreeData layout (cstone/tree/octree.hpp:283-358)
// ------------------------------------------------------------------------------------------------------------------
namespace sphb
{
namespace
{

//! digitWeight of the reference's binary-radix to octree index map (cstone/sfc/common.hpp:318-322)
__device__ __forceinline__ int refDigitWeight(int digit)
{
    int fourGeqMask = -int(digit >= 4);
    return ((7 - digit) & fourGeqMask) - (digit & ~fourGeqMask);
}

/*! internalToLeaf / leafToInternal in the reference's unsorted-index convention (createUnsortedLayoutCpu,
 *  octree.hpp:77-99 and buildOctreeCpu, :170-196): the unsorted index of leaf l is numInternal + l, that of the
 *  internal node found at leaf boundary tid (common prefix a multiple of 3 bits) is
 *  (tid + binaryKeyWeight(key, level)) / 7; internalToLeaf[sorted] = unsorted - numInternal,
 *  leafToInternal[unsorted] = sorted. */
__global__ void refNodeMapKernel(const uint64_t* leaves, int numLeaves, int numInternal, const uint64_t* prefixes,
                                 int numNodes, const int* leafToNode, int* internalToLeaf, int* leafToInternal)
{
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= numLeaves) { return; }
    int sortedLeaf                       = leafToNode[tid];
    internalToLeaf[sortedLeaf]           = tid;
    leafToInternal[numInternal + tid]    = sortedLeaf;
    if (tid >= numLeaves - 1) { return; }
    uint64_t key     = leaves[tid];
    int prefixLength = int(__clzll(key ^ leaves[tid + 1])) - 1;
    if (prefixLength % 3 != 0) { return; }
    int level  = prefixLength / 3;
    int weight = 0;
    for (int l = 1; l <= level + 1; ++l)
    {
        weight += refDigitWeight(int((key >> (3 * (int(kMaxLevel) - l))) & 7u));
    }
    int octIndex    = (tid + weight) / 7;
    uint64_t prefix = (uint64_t(1) << prefixLength) | (key >> (3 * int(kMaxLevel) - prefixLength));
    // sorted position of this internal node: prefixes are unique and sorted
    int lo = 0, hi = numNodes;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (prefixes[mid] < prefix) { lo = mid + 1; }
        else { hi = mid; }
    }
    internalToLeaf[lo]       = octIndex - numInternal;
    leafToInternal[octIndex] = lo;
}

} // namespace
} // namespace sphb

extern "C" int sphb_build_octree(const uint64_t* leaves, size_t num_leaves, uint64_t* prefixes, int* child_offsets,
                                 int* parents, int* level_range, int* internal_to_leaf, int* leaf_to_internal,
                                 void* stream)
{
    using namespace sphb;
    if (!leaves || num_leaves == 0 || num_leaves >= (size_t(1) << 30) || !prefixes || !child_offsets || !parents ||
        !level_range || !internal_to_leaf || !leaf_to_internal)
    {
        return SPHB_ERR_ARG;
    }
    auto st = static_cast<cudaStream_t>(stream);
    LinkedOctree t;
    TreeScratch sc;
    SPHB_TRY(buildLinkedOctree(leaves, int(num_leaves), t, sc, st));
    int nn = t.numNodes;
    SPHB_CUDA_TRY(cudaMemcpyAsync(prefixes, t.prefixes.data(), nn * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(child_offsets, t.childOffsets.data(), nn * sizeof(int), cudaMemcpyDeviceToDevice,
                                  st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(parents, t.parents.data(), std::max(1, (nn - 1) / 8) * sizeof(int),
                                  cudaMemcpyDeviceToDevice, st));
    refNodeMapKernel<<<ceilDiv(num_leaves, 256), 256, 0, st>>>(leaves, t.numLeaves, t.numInternal, t.prefixes.data(),
                                                                 nn, t.leafToNode.data(), internal_to_leaf,
                                                                 leaf_to_internal);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    SPHB_CUDA_TRY(
        cudaMemcpy(level_range, t.levelRangeD.data(), (kMaxLevel + 2) * sizeof(int), cudaMemcpyDeviceToHost));
    return SPHB_OK;
}

// ------------------------------------------------------------------------------------------------------------------
// One step of the multi-rank global tree: the caller sums the leaf counts of every rank between the steps
// (cstone::updateOctreeGlobal, cstone/tree/update_mpi.hpp:64-99)
// ------------------------------------------------------------------------------------------------------------------

extern "C" int sphb_leaf_counts(const uint64_t* leaves, size_t num_leaves, const uint64_t* sorted_keys, size_t n,
                                uint32_t* counts, void* stream)
{
    using namespace sphb;
    if (!leaves || !counts || num_leaves == 0 || num_leaves >= (size_t(1) << 30) || (n && !sorted_keys))
    {
        return SPHB_ERR_ARG;
    }
    return computeLeafCounts(leaves, int(num_leaves), sorted_keys, n, counts, static_cast<cudaStream_t>(stream));
}

extern "C" int sphb_rebalance_tree(const uint64_t* leaves, size_t num_leaves, const uint32_t* counts, unsigned bucket,
                                   uint64_t* new_leaves, size_t capacity, size_t* num_new, int* converged,
                                   void* stream)
{
    using namespace sphb;
    if (!leaves || !counts || !new_leaves || !num_new || !converged || bucket == 0 || num_leaves == 0 ||
        num_leaves >= (size_t(1) << 30) || new_leaves == leaves)
    {
        return SPHB_ERR_ARG;
    }
    auto st = static_cast<cudaStream_t>(stream);
    int L   = int(num_leaves);
    TreeScratch s;
    SPHB_TRY(s.ints.reserve(L + 2));
    SPHB_TRY(s.scanTmp.reserve(scanTempInts(L + 1) + 1));
    SPHB_TRY(s.flags.reserve(1));
    SPHB_CUDA_TRY(cudaMemsetAsync(s.flags.data(), 0, sizeof(unsigned), st));
    csNodeOpsKernel<<<ceilDiv(L + 1, 256), 256, 0, st>>>(leaves, counts, L, bucket, s.ints.data(), s.flags.data());
    countLaunch();
    SPHB_TRY(exclusiveScan(s.ints.data(), s.ints.data(), L + 1, s.scanTmp.data(), st));
    int newL       = 0;
    unsigned anyOp = 0;
    SPHB_TRY(readBack(st, {{&newL, s.ints.data() + L, sizeof(int)}, {&anyOp, s.flags.data(), sizeof(unsigned)}}));
    *num_new   = size_t(newL);
    *converged = anyOp ? 0 : 1;
    if (size_t(newL) + 1 > capacity) { return SPHB_ERR_CAPACITY; }
    rebalanceKernel<<<ceilDiv(L + 1, 256), 256, 0, st>>>(leaves, L, s.ints.data(), new_leaves);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    return SPHB_OK;
}
