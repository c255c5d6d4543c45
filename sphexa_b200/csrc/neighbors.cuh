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
    // bound on how far any particle has moved since the tree was built (block time steps drift particles between
    // tree builds): node boxes are widened by it, so a particle outside its cell is still found
    double ext{0.0};
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

//! d folded to the nearest periodic image: d - L * rint(d / L), rounded like the reference's uncontracted CPU code
__device__ inline double minImage(double d, double len, double ilen, int periodic)
{
    if (!periodic) { return d; }
    return __dsub_rn(d, __dmul_rn(len, rint(__dmul_rn(d, ilen))));
}

//! smoothing-length update h * 0.5 * (1 + 1023 ng0 / nc)^(1/10) (sph/include/sph/kernels.hpp:27-33)
__device__ inline double updateH(unsigned ng0, unsigned nc, double h)
{
    double ratio = __ddiv_rn(__dmul_rn(1023.0, double(ng0)), double(nc));
    return __dmul_rn(__dmul_rn(h, 0.5), pow(__dadd_rn(1.0, ratio), 0.1));
}

//! the exact pair test of the reference (cstone/findneighbors.hpp:33-51): minimum-image squared distance, summed in
//! the reference's order without contraction
__device__ inline double exactDistSq(double xj, double yj, double zj, double xi, double yi, double zi,
                                     const DevBox& box)
{
    double ex = minImage(xj - xi, box.len[0], box.ilen[0], box.periodic[0]);
    double ey = minImage(yj - yi, box.len[1], box.ilen[1], box.periodic[1]);
    double ez = minImage(zj - zi, box.len[2], box.ilen[2], box.periodic[2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
}

//! the reference's squared search radius (2h)^2 = 4 h h
__device__ inline double searchRadiusSq(double h) { return __dmul_rn(__dmul_rn(4.0, h), h); }

/*! Candidate lists kept across steps ("skin" lists): for every particle, each j whose distance was below
 *  R_i = 2 h_i (1 + skin) when the lists were built, in ascending index order, at most `cap` of them (chunked like
 *  the neighbour lists, with `cap` as the padded width). count[i] is the number found, which can exceed cap: the row
 *  is then incomplete and never used. dist holds, beside each entry, its distance at the build in units of
 *  R_i / kSkinDistUnits, rounded to nearest (16 bits, same chunked layout). */
struct SkinLists
{
    uint32_t* rows;
    unsigned* count;
    double* radius;
    unsigned cap;
    uint16_t* dist;
};

//! units of the quantised build distance per R_i
constexpr double kSkinDistUnits = 65535.0;

/*! Search all particles (x, y, z and the same coordinates packed as pos = (x, y, z, m)): updates h where the count
 *  left [ng0/4, ngmax+1], writes nc (count incl. self) and lists. With gate set, the launch does nothing unless bit
 *  *gate of gateMask is set (a mode chosen on the device, for a captured graph).
 *  status[0] is set to a non-zero value if a per-warp buffer overflowed (the search then returns SPHB_ERR_CAPACITY).
 *  An ensemble passes views (one tree per instance, on the device) and inst (instance per slot, kGhost for
 *  padding): each group searches its instance's tree, padding slots are skipped. */
int findNeighbors(const double* x, const double* y, const double* z, const double4* pos, double* h, size_t n,
                  const TreeView& tree, const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc,
                  unsigned* status, cudaStream_t stream, const TreeView* views = nullptr,
                  const uint8_t* inst = nullptr, const unsigned* gate = nullptr, unsigned gateMask = 0);

/*! The same search for the groups listed in groups[0 .. *numListed) only (a device count: the launch covers every
 *  group and the warps past the count return at once). */
int findNeighborsListed(const double* x, const double* y, const double* z, const double4* pos, double* h, size_t n,
                        const TreeView& tree, const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc,
                        unsigned* status, const unsigned* groups, const unsigned* numListed, cudaStream_t stream,
                        const TreeView* views = nullptr, const uint8_t* inst = nullptr);

/*! Build the skin lists at the current positions and smoothing lengths: R_i = 2 h_i (1 + skin). Row i holds exactly
 *  the j != i whose FP64 minimum-image squared distance is below R_i * R_i, ascending. h is read only. */
int buildSkinLists(const double* x, const double* y, const double* z, const double4* pos, const double* h, size_t n,
                   const TreeView& tree, const DevBox& box, NeighborParams prm, double skin, SkinLists sl,
                   unsigned* status, cudaStream_t stream, const TreeView* views = nullptr,
                   const uint8_t* inst = nullptr, const unsigned* gate = nullptr, unsigned gateMask = 0);

//! inputs of the per-step refilter of the skin lists (skin.cu)
struct SkinFilterArgs
{
    const double4* pos; // current packed positions (x, y, z, m)
    const int4* posq;   // fixed-point positions (mixed precision), or null: every candidate is tested in FP64
    float qscale[3];    // fixed-point unit per axis as FP32
    float qunit;        // the largest fixed-point unit (sets the width of the FP32 uncertainty band)
    double* h;
    unsigned* nc;
    uint32_t* nidx;
    SkinLists sl;
    const double* xb; // positions at the build, by build index
    const double* yb;
    const double* zb;
    const uint32_t* moved;   // bit i: index i holds another particle than at the build (null: none moved)
    const unsigned* dispGrid; // per cell of a kSkinGrid^3 grid over the box: largest displacement (FP32 bits);
                              // an ensemble: one grid per instance, instance k at dispGrid + k kSkinCells
    unsigned* groupD;         // per group: the check's result (D as FP32 bits, or all ones: deferred)
    unsigned* worklist;       // groups the check defers, for findNeighborsListed
    unsigned* numWorklist;
    unsigned* worklist2;      // groups whose smoothing-length iteration leaves their rows
    unsigned* numWorklist2;
    size_t n;
    DevBox box;
    NeighborParams prm;
    const uint8_t* inst;   // an ensemble: instance per slot (kGhost: padding, skipped), else null
    const unsigned* gate;  // if set: the launch runs only when *gate == kSkinModeFilter
};

//! neighbour-stage modes of a simulation stepped without host reads (ensemble), chosen on the device
enum SkinMode : unsigned
{
    kSkinModeTree   = 0, // tree search of every group, no rows
    kSkinModeBuild  = 1, // tree search of every group and a build of the rows
    kSkinModeFilter = 2  // refilter of the rows, tree search of the deferred groups
};

//! words of the device-side control block of skinDecide
enum SkinCtl : int
{
    kCtlMode, kCtlValid, kCtlAge, kCtlHoldoff, kCtlDeferredA, kCtlDeferredB, kCtlGroups, kCtlDeferredTotal,
    kCtlTreeSearches, kCtlBuilds, kCtlFilterSteps, kCtlWords
};

/*! Choose this step's mode into ctl[kCtlMode] from the previous step's deferred counts (ctl[kCtlDeferredA/B], which
 *  the check and the filter increment as worklist counters and which this call resets). */
int skinDecide(unsigned* ctl, cudaStream_t stream);

//! in a build step (ctl[kCtlMode] == kSkinModeBuild): record build positions and the identity index map
int skinCommit(const double* x, const double* y, const double* z, size_t n, double* xb, double* yb, double* zb,
               uint32_t* buildOf, uint32_t* moved, unsigned* ctl, cudaStream_t stream);

//! cells per axis of the displacement grid, and cells per grid (an ensemble has one grid per instance)
constexpr int kSkinGrid  = 32;
constexpr int kSkinCells = kSkinGrid * kSkinGrid * kSkinGrid;

/*! Largest displacement since the build per cell of the grid (cells by current position). buildOf maps the current
 *  index to the build index (null: the identity). dispGrid must be zero on entry. With inst (an ensemble), each
 *  instance has its own grid (instance k at dispGrid + k kSkinCells): members do not interact. */
int skinDisplacement(const double4* pos, const double* xb, const double* yb, const double* zb,
                     const uint32_t* buildOf, size_t n, const DevBox& box, unsigned* dispGrid, cudaStream_t stream,
                     const uint8_t* inst = nullptr, const unsigned* gate = nullptr);

/*! After a sort that moved particles: buildNew[i] = buildOld[order[i]] (buildOld null: the identity) and bit i of
 *  moved = (buildNew[i] != i). */
int skinRemap(const uint32_t* order, const uint32_t* buildOld, uint32_t* buildNew, uint32_t* moved, size_t n,
              cudaStream_t stream);

//! *flag = 1 if a[i] != b[i] for some i < n, else 0 (device flag)
int idsDiffer(const uint64_t* a, const uint64_t* b, size_t n, unsigned* flag, cudaStream_t stream);

/*! Decide per group whether the skin rows can serve it: only when they are provably complete for the current
 *  positions and h, 2 h_i + |displacement of i| + (largest displacement of any particle near the group) <= R_i, and
 *  no particle of the group or of its rows changed index since the build. The others go to the worklist, untouched
 *  (h, nc unchanged), for the tree search. */
int checkSkinGroups(const SkinFilterArgs& a, cudaStream_t stream);

/*! Neighbour lists, counts and the smoothing-length iteration from the skin rows, for the groups the check kept. A
 *  group whose new h leaves its rows goes to worklist2, untouched. The results are those of findNeighbors. */
int filterSkinLists(const SkinFilterArgs& a, cudaStream_t stream);

} // namespace sphb
