// Radix sort interface (see sort.cu).
#pragma once

#include "common.cuh"

namespace sphb
{

size_t sortScratchBytes(size_t n);

//! stable in-place sort of (key, value) pairs; values set to 0..n-1 first if initValues
int sortByKey(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
              cudaStream_t stream);

/*! The same sort without any host synchronisation (stream-capturable): runs exactly the passes of passMask (bit p
 *  = byte p of the key, from the least significant) and ORs a look-back timeout into *errorOut (device) if set. */
int sortByKeyAsync(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
                   unsigned passMask, uint32_t* errorOut, cudaStream_t stream);

} // namespace sphb
