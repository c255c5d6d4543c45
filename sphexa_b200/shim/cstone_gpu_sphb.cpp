/* The cstone GPU primitives of the domain sync implemented on sphb200, for keys uint64_t and coordinates double.
 *
 * A maintainer of the reference builds this file into the reference in place of the definitions in
 * cstone/sfc/sfc_gpu.cu and the sort of cstone/primitives/primitives_gpu.cu (declared in cstone/sfc/sfc_gpu.h:23-24 and
 * cstone/primitives/primitives_gpu.h:78-86), adds include/ of this repository to the include path and links
 * libsphb200.so. Errors throw std::runtime_error instead of exiting (cstone/cuda/errorcheck.cuh:15-26).
 */
#include <cstdint>
#include <stdexcept>
#include <string>

#include "cstone/primitives/primitives_gpu.h"
#include "cstone/sfc/sfc_gpu.h"
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

} // namespace cstone
