// Radix sort interface (see sort.cu).
#pragma once

#include "common.cuh"

namespace sphb
{

size_t sortScratchBytes(size_t n);

//! stable in-place sort of (key, value) pairs; values set to 0..n-1 first if initValues
int sortByKey(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
              cudaStream_t stream);

} // namespace sphb
