// Radix sort interface (see sort.cu).
#pragma once

#include "common.cuh"

namespace sphb
{

size_t sortScratchBytes(size_t n);

//! stable in-place sort of (key, value) pairs; values set to 0..n-1 first if initValues
int sortByKey(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
              cudaStream_t stream);

/*! The same stable sort for keys that are nearly in order (the previous step's order of slowly moving particles):
 *  values are set to 0..n-1; if no adjacent pair is out of order, nothing moves and *identity is set; otherwise the
 *  tiles that hold inversions are sorted in shared memory (two overlapping tilings), and the full radix sort runs
 *  only if that left any inversion. The result equals sortByKey's. */
int sortNearlySorted(uint64_t* keys, uint32_t* values, size_t n, void* scratch, size_t scratchBytes, bool* identity,
                     cudaStream_t stream);

/*! The same sort without any host synchronisation (stream-capturable): runs exactly the passes of passMask (bit p
 *  = byte p of the key, from the least significant) and ORs a look-back timeout into *errorOut (device) if set. */
int sortByKeyAsync(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
                   unsigned passMask, uint32_t* errorOut, cudaStream_t stream, const uint32_t* gate = nullptr);

/*! The local repair of sortNearlySorted for an array of contiguous segments (seg[i] ascending; a slot never leaves
 *  its segment), without any host synchronisation: values = 0..n-1, flags[0] = number of adjacent pairs of one
 *  segment out of key order, then the tiles holding such pairs are sorted stably by (segment, key) in shared memory
 *  (two overlapping tilings), flags[1] = pairs still out of order. If flags[1] is 0, keys/values are the stable
 *  sort by (segment, key); otherwise a full sort of the repaired sequence (gated on flags + 1) completes it. */
int repairSegmentedAsync(uint64_t* keys, uint32_t* values, const uint64_t* seg, size_t n, uint32_t* flags,
                         cudaStream_t stream);

} // namespace sphb
