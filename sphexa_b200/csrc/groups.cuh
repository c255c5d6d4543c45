// Spatial target groups: SFC-consecutive runs of at most 32 (or 64) particles, split where consecutive particles are
// far apart (see groups.cu).
#pragma once

#include "common.cuh"
#include "primitives.cuh"

namespace sphb
{

/*! Boundaries of the spatial groups of particles [first, last): group g is [bounds[g], bounds[g + 1]), numGroups
 *  groups, bounds[numGroups] = last. Particles are in SFC order; h is FP32 or FP64 (hType SPHB_F32 / SPHB_F64, the
 *  precision of the split threshold as in the reference) and may be null (no h criterion). leaves (numLeaves + 1
 *  keys) and layout (first particle of each leaf) are the focus tree's. groupSize is 32 or 64. Host-blocking (reads
 *  the group count). The scratch buffers grow as needed. */
int computeGroupSplits(size_t first, size_t last, const double* x, const double* y, const double* z, const void* h,
                       int hType, const uint64_t* leaves, int numLeaves, const uint32_t* layout, const DevBox& box,
                       unsigned groupSize, float tolFactor, DeviceBuffer<int>& scratch, DeviceBuffer<uint32_t>& bounds,
                       unsigned* numGroups, cudaStream_t stream);

} // namespace sphb
