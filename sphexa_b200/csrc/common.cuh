// Shared device/host helpers of the sm_100a hydro library.
#pragma once
#include <initializer_list>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <utility>
#include <cuda_runtime.h>

#include "../../include/sphb200.h"

namespace sphb
{

//! Hilbert keys: 21 bits per dimension, 63 bits in total (cstone/tree/definitions.h:45-75)
constexpr unsigned kMaxLevel  = 21;
constexpr uint64_t kRootRange = uint64_t(1) << 63;
//! the key that flags a particle for removal; it sorts after every valid key (definitions.h:70-75)
constexpr uint64_t kRemoveKey = uint64_t(1) << 63;

//! instance index of a padding slot in a batched ensemble
constexpr uint8_t kGhost = 255;

/*! Per-slot instance map and per-instance values of a batched ensemble step (all null for one simulation). Instances
 *  occupy 32-aligned runs of slots, padded with ghost slots, so a warp group never spans two instances. */
struct BatchView
{
    const uint8_t* inst{nullptr};         // per slot: instance index, kGhost for padding
    const double* gamma{nullptr};         // per instance
    const double* cv{nullptr};            // per instance
    const double* dt{nullptr};            // per instance: the step being taken (AV switches: the previous one)
    const double* dtm1{nullptr};          // per instance: the step before
    unsigned long long* reduce{nullptr};  // per instance: [2k] max divv, [2k+1] min Courant dt (ordered bits)
};
constexpr int kTableSize      = 20000;
constexpr int kWarp           = 32;

//! status codes shared with the C ABI
enum Status : int
{
    kOk            = SPHB_OK,
    kErrArg        = SPHB_ERR_ARG,
    kErrCuda       = SPHB_ERR_CUDA,
    kErrCapacity   = SPHB_ERR_CAPACITY,
    kErrNotConverged = SPHB_ERR_NOT_CONVERGED,
    kErrState        = SPHB_ERR_STATE,
    kErrTimeout      = SPHB_ERR_TIMEOUT,
};

#define SPHB_CUDA_TRY(expr)                                                                                            \
    do                                                                                                                 \
    {                                                                                                                  \
        cudaError_t err_ = (expr);                                                                                     \
        if (err_ != cudaSuccess)                                                                                       \
        {                                                                                                              \
            std::fprintf(stderr, "sphb200: %s failed at %s:%d: %s\n", #expr, __FILE__, __LINE__,                      \
                         cudaGetErrorString(err_));                                                                    \
            return SPHB_ERR_CUDA;                                                                                      \
        }                                                                                                              \
    } while (0)

#define SPHB_TRY(expr)                                                                                                 \
    do                                                                                                                 \
    {                                                                                                                  \
        int st_ = (expr);                                                                                              \
        if (st_ != SPHB_OK) { return st_; }                                                                            \
    } while (0)

//! Coordinate box with inverse lengths and per-axis periodicity (cstone/sfc/box.hpp:94-174)
struct DevBox
{
    double lo[3];
    double hi[3];
    double len[3];
    double ilen[3];
    int periodic[3];
};

inline DevBox makeDevBox(const sphb_box& b)
{
    DevBox d;
    for (int k = 0; k < 3; ++k)
    {
        d.lo[k]       = b.lo[k];
        d.hi[k]       = b.hi[k];
        d.len[k]      = b.hi[k] - b.lo[k];
        d.ilen[k]     = 1.0 / (b.hi[k] - b.lo[k]);
        d.periodic[k] = b.periodic[k] ? 1 : 0;
    }
    return d;
}

inline unsigned ceilDiv(size_t a, unsigned b) { return unsigned((a + b - 1) / b); }

//! number of SMs of the current device, cached per process
int smCount();

/*! A small block of pinned host memory of the calling thread (kReadbackWords words, usable from every device), for
 *  the small reads of the per-step host decisions: a copy into pageable memory returns only when it has completed, so
 *  two of them wait for the stream twice, while copies into pinned memory queue behind the kernels and one
 *  synchronisation serves them all. Null if the allocation failed. */
constexpr int kReadbackWords = 16;
unsigned long long* pinnedReadback();

//! one small read of readBack: bytes of device memory at src, for host memory at dst
struct ReadItem
{
    void* dst;
    const void* src;
    size_t bytes;
};

/*! the items copied through pinnedReadback() with one wait on the stream (at most kReadbackWords * 8 bytes in all;
 *  through pageable memory, one wait per item, if the pinned block is missing) */
int readBack(cudaStream_t stream, std::initializer_list<ReadItem> items);

} // namespace sphb
