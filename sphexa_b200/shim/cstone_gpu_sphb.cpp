/* The cstone GPU primitives of the domain sync implemented on sphb200, for keys uint64_t and coordinates double.
 *
 * A maintainer of the reference builds this file into the reference in place of the definitions in
 * cstone/sfc/sfc_gpu.cu, the sort of cstone/primitives/primitives_gpu.cu and the node counts of
 * cstone/tree/csarray_gpu.cu (declared in cstone/sfc/sfc_gpu.h:23-24, cstone/primitives/primitives_gpu.h:78-86 and
 * cstone/tree/csarray_gpu.h:38-44), adds include/ of this repository to the include path and links libsphb200.so.
 * Errors throw std::runtime_error instead of exiting (cstone/cuda/errorcheck.cuh:15-26).
 *
 * The multi-rank global tree step and the halo search on the global tree are here too, as functions the
 * domain calls in place of updateOctreeGlobalGpu (cstone/tree/update_mpi_gpu.cuh:34-85) and of the focus tree's
 * discoverHalos (cstone/focus/octree_focus_mpi.hpp:513-571).
 */
#include <algorithm>
#include <cstdint>
#include <limits>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>
#include <mpi.h>

#include "cstone/cuda/device_vector.h"
#include "cstone/primitives/primitives_gpu.h"
#include "cstone/sfc/sfc_gpu.h"
#include "cstone/tree/csarray_gpu.h"
#include "sphb200.h"

namespace cstone
{
namespace
{
void check(int rc, const char* what)
{
    if (rc != SPHB_OK) { throw std::runtime_error(std::string(what) + " failed with sphb status " + std::to_string(rc)); }
}

sphb_box toSphbBox(const Box<double>& box)
{
    sphb_box b;
    b.lo[0]       = box.xmin();
    b.hi[0]       = box.xmax();
    b.lo[1]       = box.ymin();
    b.hi[1]       = box.ymax();
    b.lo[2]       = box.zmin();
    b.hi[2]       = box.zmax();
    b.periodic[0] = box.boundaryX() == BoundaryType::periodic;
    b.periodic[1] = box.boundaryY() == BoundaryType::periodic;
    b.periodic[2] = box.boundaryZ() == BoundaryType::periodic;
    return b;
}
} // namespace

template<>
void computeSfcKeysGpu<uint64_t, double>(const double* x, const double* y, const double* z, uint64_t* keys,
                                         size_t numKeys, const Box<double>& box)
{
    sphb_box b = toSphbBox(box);
    check(sphb_compute_sfc_keys(x, y, z, keys, numKeys, &b, nullptr), "computeSfcKeysGpu");
}

template<>
uint64_t sortByKeyTempStorage<uint64_t, unsigned>(uint64_t numElements)
{
    return sphb_sort_by_key_scratch_bytes(numElements);
}

//! the values are carried along with their keys, as CUB's SortPairs does; keyBuf and valueBuf are not needed (the
//! sort works in place with its scratch)
template<>
void sortByKeyGpu<uint64_t, unsigned>(uint64_t* first, uint64_t* last, unsigned* values, uint64_t* /*keyBuf*/,
                                      unsigned* /*valueBuf*/, void* scratch, uint64_t scratchBytes)
{
    check(sphb_sort_by_key(first, values, size_t(last - first), /*init_values=*/0, scratch, scratchBytes, nullptr),
          "sortByKeyGpu");
}

/*! the leaf counts of sorted device keys; the counts are exact, so maxCount (the cap of the reference's capped MPI
 *  sum) must be the unsigned maximum, which every caller of the reference passes */
template<>
void computeNodeCountsGpu<uint64_t>(const uint64_t* tree, unsigned* counts, TreeNodeIndex numNodes,
                                    std::span<const uint64_t> keys, unsigned maxCount, bool /*useCountsAsGuess*/)
{
    if (maxCount != std::numeric_limits<unsigned>::max())
    {
        throw std::invalid_argument("computeNodeCountsGpu: sphb200 counts are not capped");
    }
    check(sphb_leaf_counts(tree, size_t(numNodes), keys.data(), keys.size(), counts, nullptr), "computeNodeCountsGpu");
}

/*! One step of the multi-rank global tree (updateOctreeGlobalGpu, cstone/tree/update_mpi_gpu.cuh:34-85): rebalance
 *  the device leaves d_csTree on the all-reduced counts d_counts, then count this rank's sorted device keys per new
 *  leaf and sum the counts over the ranks (MPI_Allreduce into host memory and back). Returns 0 if the rebalance
 *  changed nothing, else the largest count, as GlobalAssignment::assign's loop expects
 *  (cstone/domain/assignment.hpp:114-123). DevKeyVec / DevCountVec: device vectors with data(), size(), resize()
 *  (cstone::DeviceVector). The linked octree is not built: the halo search below builds its own. */
template<class DevKeyVec, class DevCountVec>
unsigned sphbUpdateOctreeGlobal(std::span<const uint64_t> keys, unsigned bucketSize, DevKeyVec& d_csTree,
                                DevKeyVec& d_tmpTree, DevCountVec& d_counts)
{
    size_t numLeaves = d_csTree.size() - 1;
    size_t numNew    = 0;
    int converged    = 0;
    d_tmpTree.resize(8 * numLeaves + 1);
    int rc = sphb_rebalance_tree(d_csTree.data(), numLeaves, d_counts.data(), bucketSize, d_tmpTree.data(),
                                 d_tmpTree.size(), &numNew, &converged, nullptr);
    if (rc == SPHB_ERR_CAPACITY)
    {
        d_tmpTree.resize(numNew + 1);
        rc = sphb_rebalance_tree(d_csTree.data(), numLeaves, d_counts.data(), bucketSize, d_tmpTree.data(),
                                 d_tmpTree.size(), &numNew, &converged, nullptr);
    }
    check(rc, "sphb_rebalance_tree");
    d_tmpTree.resize(numNew + 1);
    using std::swap;
    swap(d_csTree, d_tmpTree); // the vectors' own swap where they have one (DeviceVector exchanges its buffers)

    d_counts.resize(numNew);
    check(sphb_leaf_counts(d_csTree.data(), numNew, keys.data(), keys.size(), d_counts.data(), nullptr),
          "sphb_leaf_counts");
    std::vector<unsigned> counts(numNew);
    if (cudaMemcpy(counts.data(), d_counts.data(), numNew * sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess)
    {
        throw std::runtime_error("sphbUpdateOctreeGlobal: count download failed");
    }
    MPI_Allreduce(MPI_IN_PLACE, counts.data(), int(numNew), MPI_UNSIGNED, MPI_SUM, MPI_COMM_WORLD);
    if (cudaMemcpy(d_counts.data(), counts.data(), numNew * sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess)
    {
        throw std::runtime_error("sphbUpdateOctreeGlobal: count upload failed");
    }
    return converged ? 0u : *std::max_element(counts.begin(), counts.end());
}

template unsigned sphbUpdateOctreeGlobal<DeviceVector<uint64_t>, DeviceVector<unsigned>>(
    std::span<const uint64_t>, unsigned, DeviceVector<uint64_t>&, DeviceVector<uint64_t>&, DeviceVector<unsigned>&);

/*! Halo flags of this rank per leaf of the global tree (discoverHalos' bounding boxes and findHalos,
 *  cstone/focus/octree_focus_mpi.hpp:513-571, on the global tree): the rank owns leaves [firstLeaf, lastLeaf) with
 *  its SFC-sorted particles x, y, z, h, leaf firstLeaf + i holding [layout[i], layout[i + 1]). Device arrays. */
template<class Th>
void sphbFindHaloLeaves(const uint64_t* leaves, size_t numLeaves, const double* x, const double* y, const double* z,
                        const Th* h, const unsigned* layout, TreeNodeIndex firstLeaf, TreeNodeIndex lastLeaf,
                        const Box<double>& box, float searchExtFact, uint8_t* flags)
{
    static_assert(std::is_same_v<Th, float> || std::is_same_v<Th, double>);
    sphb_box b = toSphbBox(box);
    check(sphb_find_halos(leaves, numLeaves, x, y, z, h, std::is_same_v<Th, float> ? SPHB_F32 : SPHB_F64, layout,
                          size_t(firstLeaf), size_t(lastLeaf), &b, searchExtFact, flags, nullptr),
          "sphb_find_halos");
}

template void sphbFindHaloLeaves<float>(const uint64_t*, size_t, const double*, const double*, const double*,
                                        const float*, const unsigned*, TreeNodeIndex, TreeNodeIndex,
                                        const Box<double>&, float, uint8_t*);
template void sphbFindHaloLeaves<double>(const uint64_t*, size_t, const double*, const double*, const double*,
                                         const double*, const unsigned*, TreeNodeIndex, TreeNodeIndex,
                                         const Box<double>&, float, uint8_t*);

} // namespace cstone
