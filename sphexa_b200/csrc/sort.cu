// Stable LSD radix sort of (uint64 key, uint32 value) pairs: one histogram sweep for all digits, then one
// "onesweep" pass per 8-bit digit in which each tile ranks its keys, resolves its global digit offsets through a
// decoupled look-back over the preceding tiles, and scatters. Passes whose digit is identical for every key are
// skipped. Replaces the reference's CUB DeviceRadixSort::SortPairs (cstone/primitives/primitives_gpu.cu:308-339).
//
// Tile = 8 warps x 16 keys x 32 lanes = 4096 keys. Within a warp, key k of lane l is element warpBase + k*32 + l, and
// ranking walks k then l, so ranks follow input order (stability). The look-back status word per (tile, digit) is
// 32 bits: 2 flag bits (0 = empty, 1 = tile aggregate, 2 = inclusive prefix) and a 30-bit count, so n < 2^30.
// Every spin on a predecessor's status is bounded; on timeout the pass records an error word that the host reads.
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "sort.cuh"

namespace sphb
{

namespace
{

constexpr int kRadixBits   = 8;
constexpr int kRadix       = 1 << kRadixBits;
constexpr int kSortWarps   = 8;
constexpr int kSortThreads = kSortWarps * kWarp;
constexpr int kItems       = 16;
constexpr int kTile        = kSortThreads * kItems;
constexpr int kPasses      = 8;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;
constexpr long kSpinLimit   = 1L << 24;

struct SortScratch
{
    uint64_t* keysAlt;
    uint32_t* valsAlt;
    uint32_t* hist;       // [kPasses][kRadix] counts, then exclusive offsets
    uint32_t* status;     // [numTiles][kRadix]
    uint32_t* counters;   // [0] tile counter, [1] error word
};

size_t alignUp(size_t x, size_t a) { return (x + a - 1) / a * a; }

size_t numTilesOf(size_t n) { return (n + kTile - 1) / kTile; }

SortScratch carve(void* base, size_t n)
{
    char* p = static_cast<char*>(base);
    SortScratch s;
    s.keysAlt = reinterpret_cast<uint64_t*>(p);
    p += alignUp(n * sizeof(uint64_t), 256);
    s.valsAlt = reinterpret_cast<uint32_t*>(p);
    p += alignUp(n * sizeof(uint32_t), 256);
    s.hist = reinterpret_cast<uint32_t*>(p);
    p += alignUp(kPasses * kRadix * sizeof(uint32_t), 256);
    s.status = reinterpret_cast<uint32_t*>(p);
    p += alignUp(numTilesOf(n) * kRadix * sizeof(uint32_t), 256);
    s.counters = reinterpret_cast<uint32_t*>(p);
    return s;
}

//! digit histograms of all 8 byte positions in one sweep over the keys
__global__ void __launch_bounds__(256) histogramKernel(const uint64_t* __restrict__ keys, size_t n,
                                                       uint32_t* __restrict__ hist, const uint32_t* gate)
{
    if (gate && *gate == 0) { return; }
    __shared__ uint32_t sh[kPasses][kRadix];
    for (int t = threadIdx.x; t < kPasses * kRadix; t += blockDim.x)
    {
        (&sh[0][0])[t] = 0;
    }
    __syncthreads();
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        uint64_t k = keys[i];
#pragma unroll
        for (int p = 0; p < kPasses; ++p)
        {
            atomicAdd(&sh[p][(k >> (p * kRadixBits)) & (kRadix - 1)], 1u);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < kPasses * kRadix; t += blockDim.x)
    {
        uint32_t c = (&sh[0][0])[t];
        if (c) { atomicAdd(hist + t, c); }
    }
}

//! exclusive scan of each pass's 256 digit counts, in place (one block per pass)
__global__ void histScanKernel(uint32_t* hist, const uint32_t* gate)
{
    if (gate && *gate == 0) { return; }
    __shared__ uint32_t sh[kRadix];
    uint32_t* h = hist + blockIdx.x * kRadix;
    int t       = threadIdx.x;
    uint32_t v  = h[t];
    sh[t]       = v;
    __syncthreads();
    for (int off = 1; off < kRadix; off <<= 1)
    {
        uint32_t add = t >= off ? sh[t - off] : 0;
        __syncthreads();
        sh[t] += add;
        __syncthreads();
    }
    h[t] = sh[t] - v;
}

__global__ void iotaKernel(uint32_t* v, size_t n)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i < n) { v[i] = uint32_t(i); }
}

//! *count += number of adjacent pairs with keys[i] > keys[i + 1] (one atomic per block)
__global__ void __launch_bounds__(256) inversionsKernel(const uint64_t* __restrict__ keys, size_t n,
                                                        uint32_t* count)
{
    uint32_t c = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i + 1 < n; i += size_t(gridDim.x) * blockDim.x)
    {
        c += keys[i] > keys[i + 1] ? 1u : 0u;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ uint32_t warpSum[8];
    if ((threadIdx.x & 31) == 0) { warpSum[threadIdx.x >> 5] = c; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint32_t s = 0;
        for (int w = 0; w < 8; ++w)
        {
            s += warpSum[w];
        }
        if (s) { atomicAdd(count, s); }
    }
}

constexpr int kRepairTile    = 2048;
constexpr int kRepairThreads = 256;

/*! Stable sort of one tile of (key, value) pairs in shared memory, tile t covering [offset + t T, offset + (t+1) T),
 *  skipped when the tile and its left neighbour pair are already in order. Bitonic network on (key, position in the
 *  tile), so equal keys keep their order; positions past n are padded with the largest key. */
__global__ void __launch_bounds__(kRepairThreads) repairTilesKernel(uint64_t* keys, uint32_t* vals, size_t n,
                                                                   size_t offset)
{
    __shared__ uint64_t sk[kRepairTile];
    __shared__ uint32_t sv[kRepairTile];
    __shared__ uint16_t sp[kRepairTile];
    size_t t0 = offset + size_t(blockIdx.x) * kRepairTile;
    if (t0 >= n) { return; }
    size_t len = min(size_t(kRepairTile), n - t0);
    bool d     = false;
    for (size_t q = threadIdx.x; q + 1 < len; q += kRepairThreads)
    {
        d = d || keys[t0 + q] > keys[t0 + q + 1];
    }
    if (__syncthreads_or(d) == 0) { return; }
    for (int q = threadIdx.x; q < kRepairTile; q += kRepairThreads)
    {
        bool in = size_t(q) < len;
        sk[q]   = in ? keys[t0 + q] : ~uint64_t(0);
        sv[q]   = in ? vals[t0 + q] : 0u;
        sp[q]   = uint16_t(q);
    }
    __syncthreads();
    for (int size = 2; size <= kRepairTile; size <<= 1)
    {
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for (int q = threadIdx.x; q < kRepairTile; q += kRepairThreads)
            {
                int p = q ^ stride;
                if (p > q)
                {
                    bool up      = (q & size) == 0;
                    bool greater = sk[q] > sk[p] || (sk[q] == sk[p] && sp[q] > sp[p]);
                    if (greater == up)
                    {
                        uint64_t k = sk[q];
                        sk[q]      = sk[p];
                        sk[p]      = k;
                        uint32_t v = sv[q];
                        sv[q]      = sv[p];
                        sv[p]      = v;
                        uint16_t o = sp[q];
                        sp[q]      = sp[p];
                        sp[p]      = o;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (size_t q = threadIdx.x; q < len; q += kRepairThreads)
    {
        keys[t0 + q] = sk[q];
        vals[t0 + q] = sv[q];
    }
}

//! *count += adjacent pairs of one segment out of key order: seg[i] == seg[i + 1] and keys[i] > keys[i + 1]
__global__ void __launch_bounds__(256) inversionsSegKernel(const uint64_t* __restrict__ keys,
                                                           const uint64_t* __restrict__ seg, size_t n,
                                                           uint32_t* count)
{
    uint32_t c = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i + 1 < n; i += size_t(gridDim.x) * blockDim.x)
    {
        c += (keys[i] > keys[i + 1] && seg[i] == seg[i + 1]) ? 1u : 0u;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    __shared__ uint32_t warpSum[8];
    if ((threadIdx.x & 31) == 0) { warpSum[threadIdx.x >> 5] = c; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint32_t s = 0;
        for (int w = 0; w < 8; ++w)
        {
            s += warpSum[w];
        }
        if (s) { atomicAdd(count, s); }
    }
}

/*! repairTilesKernel for an array of contiguous segments (slot ranges that keep their segment): the tile is sorted
 *  stably by (segment, key), so a tile that straddles two segments keeps each segment's slots within it. */
__global__ void __launch_bounds__(kRepairThreads) repairTilesSegKernel(uint64_t* keys, uint32_t* vals,
                                                                      const uint64_t* seg, size_t n, size_t offset)
{
    __shared__ uint64_t sk[kRepairTile];
    __shared__ uint32_t sv[kRepairTile];
    __shared__ uint16_t sp[kRepairTile];
    __shared__ uint8_t sg[kRepairTile];
    size_t t0 = offset + size_t(blockIdx.x) * kRepairTile;
    if (t0 >= n) { return; }
    size_t len = min(size_t(kRepairTile), n - t0);
    bool d     = false;
    for (size_t q = threadIdx.x; q + 1 < len; q += kRepairThreads)
    {
        d = d || (keys[t0 + q] > keys[t0 + q + 1] && seg[t0 + q] == seg[t0 + q + 1]);
    }
    if (__syncthreads_or(d) == 0) { return; }
    // segments are ranked by their order within the tile (they are contiguous and ascending)
    uint64_t seg0 = seg[t0];
    for (int q = threadIdx.x; q < kRepairTile; q += kRepairThreads)
    {
        bool in = size_t(q) < len;
        sk[q]   = in ? keys[t0 + q] : ~uint64_t(0);
        sv[q]   = in ? vals[t0 + q] : 0u;
        sp[q]   = uint16_t(q);
        sg[q]   = in ? uint8_t(min(seg[t0 + q] - seg0, uint64_t(254))) : uint8_t(255);
    }
    __syncthreads();
    for (int size = 2; size <= kRepairTile; size <<= 1)
    {
        for (int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for (int q = threadIdx.x; q < kRepairTile; q += kRepairThreads)
            {
                int p = q ^ stride;
                if (p > q)
                {
                    bool up      = (q & size) == 0;
                    bool greater = sg[q] > sg[p] ||
                                   (sg[q] == sg[p] && (sk[q] > sk[p] || (sk[q] == sk[p] && sp[q] > sp[p])));
                    if (greater == up)
                    {
                        uint64_t k = sk[q];
                        sk[q]      = sk[p];
                        sk[p]      = k;
                        uint32_t v = sv[q];
                        sv[q]      = sv[p];
                        sv[p]      = v;
                        uint16_t o = sp[q];
                        sp[q]      = sp[p];
                        sp[p]      = o;
                        uint8_t g  = sg[q];
                        sg[q]      = sg[p];
                        sg[p]      = g;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (size_t q = threadIdx.x; q < len; q += kRepairThreads)
    {
        keys[t0 + q] = sk[q];
        vals[t0 + q] = sv[q];
    }
}

/*! One onesweep pass over bits [shift, shift+8).
 *
 * Shared memory: per-warp digit counters (8 x 256), the tile's exclusive digit prefix (256) and the tile index.
 */
__global__ void __launch_bounds__(kSortThreads) onesweepKernel(const uint64_t* __restrict__ keysIn,
                                                               const uint32_t* __restrict__ valsIn,
                                                               uint64_t* __restrict__ keysOut,
                                                               uint32_t* __restrict__ valsOut, size_t n, int shift,
                                                               const uint32_t* __restrict__ digitOffsets,
                                                               uint32_t* status, uint32_t* counters,
                                                               const uint32_t* gate)
{
    if (gate && *gate == 0) { return; } // the whole pass is skipped: no tile waits on another
    __shared__ uint32_t warpCount[kSortWarps][kRadix];
    __shared__ uint32_t tilePrefix[kRadix];
    __shared__ uint32_t tileIdxSh;

    const int lane = threadIdx.x & (kWarp - 1);
    const int warp = threadIdx.x / kWarp;

    if (threadIdx.x == 0) { tileIdxSh = atomicAdd(counters, 1u); }
    for (int t = threadIdx.x; t < kSortWarps * kRadix; t += kSortThreads)
    {
        (&warpCount[0][0])[t] = 0;
    }
    __syncthreads();
    const size_t tile     = tileIdxSh;
    const size_t tileBase = tile * kTile;
    const size_t warpBase = tileBase + size_t(warp) * kItems * kWarp;

    uint64_t key[kItems];
    uint32_t val[kItems];
    uint32_t rank[kItems];
#pragma unroll
    for (int k = 0; k < kItems; ++k)
    {
        size_t idx = warpBase + size_t(k) * kWarp + lane;
        bool valid = idx < n;
        key[k]     = valid ? keysIn[idx] : ~uint64_t(0);
        val[k]     = valid ? valsIn[idx] : 0u;
    }

    // warp-local stable ranking: peers with equal digits are found with match.any
#pragma unroll
    for (int k = 0; k < kItems; ++k)
    {
        size_t idx      = warpBase + size_t(k) * kWarp + lane;
        bool valid      = idx < n;
        uint32_t digit  = uint32_t(key[k] >> shift) & (kRadix - 1);
        uint32_t active = __ballot_sync(0xffffffffu, valid);
        uint32_t peers  = __match_any_sync(0xffffffffu, valid ? digit : 0xffffffffu);
        peers &= active;
        uint32_t before = 0;
        if (valid)
        {
            before = warpCount[warp][digit];
        }
        __syncwarp();
        if (valid)
        {
            uint32_t lowerPeers = peers & ((1u << lane) - 1u);
            rank[k]             = before + __popc(lowerPeers);
            if (lowerPeers == 0) { warpCount[warp][digit] = before + __popc(peers); }
        }
        __syncwarp();
    }
    __syncthreads();

    // per digit: exclusive scan over warps, tile total, then look-back across tiles (thread t owns digit t)
    {
        const int d    = threadIdx.x;
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w)
        {
            uint32_t c     = warpCount[w][d];
            warpCount[w][d] = total;
            total += c;
        }
        uint32_t* myStatus = status + tile * kRadix + d;
        if (tile == 0) { atomicExch(myStatus, kFlagInc | total); }
        else { atomicExch(myStatus, kFlagAgg | total); }
        __threadfence();

        uint32_t exclusive = 0;
        if (tile > 0)
        {
            long pred = long(tile) - 1;
            long spins = 0;
            while (pred >= 0)
            {
                uint32_t s = *((volatile uint32_t*)(status + size_t(pred) * kRadix + d));
                uint32_t flag = s & ~kValMask;
                if (flag == 0)
                {
                    if (++spins > kSpinLimit)
                    {
                        atomicExch(counters + 1, 1u);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                exclusive += s & kValMask;
                if (flag == kFlagInc) { break; }
                --pred;
            }
            atomicExch(myStatus, kFlagInc | ((exclusive + total) & kValMask));
        }
        tilePrefix[d] = digitOffsets[d] + exclusive;
    }
    __syncthreads();

#pragma unroll
    for (int k = 0; k < kItems; ++k)
    {
        size_t idx = warpBase + size_t(k) * kWarp + lane;
        if (idx < n)
        {
            uint32_t digit = uint32_t(key[k] >> shift) & (kRadix - 1);
            uint32_t pos   = tilePrefix[digit] + warpCount[warp][digit] + rank[k];
            if (pos < n)
            {
                keysOut[pos] = key[k];
                valsOut[pos] = val[k];
            }
            else { atomicExch(counters + 1, 2u); } // inconsistent offsets: report instead of writing
        }
    }
}

} // namespace

size_t sortScratchBytes(size_t n)
{
    return alignUp(n * sizeof(uint64_t), 256) + alignUp(n * sizeof(uint32_t), 256) +
           alignUp(kPasses * kRadix * sizeof(uint32_t), 256) + alignUp(numTilesOf(n) * kRadix * sizeof(uint32_t), 256) +
           256;
}

namespace
{
int runPasses(uint64_t* keys, uint32_t* values, size_t n, const SortScratch& s, unsigned passMask,
              cudaStream_t stream, const uint32_t* gate = nullptr);

__global__ void orErrorKernel(const uint32_t* err, uint32_t* out)
{
    if (*err) { atomicOr(out, 1u); }
}
} // namespace

int sortByKey(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
              cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    if (n >= (size_t(1) << 30)) { return kErrArg; }
    if (!scratch || scratchBytes < sortScratchBytes(n)) { return kErrCapacity; }
    SortScratch s = carve(scratch, n);

    if (initValues)
    {
        iotaKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(values, n);
        SPHB_CUDA_TRY(cudaGetLastError());
    }

    SPHB_CUDA_TRY(cudaMemsetAsync(s.hist, 0, kPasses * kRadix * sizeof(uint32_t), stream));
    unsigned histBlocks = unsigned(std::min<size_t>(ceilDiv(n, 256 * 16), size_t(smCount()) * 4));
    histogramKernel<<<histBlocks, 256, 0, stream>>>(keys, n, s.hist, nullptr);
    SPHB_CUDA_TRY(cudaGetLastError());

    // decide on the host which passes are trivial (one digit holds every key)
    uint32_t h[kPasses * kRadix];
    SPHB_CUDA_TRY(cudaMemcpyAsync(h, s.hist, sizeof(h), cudaMemcpyDeviceToHost, stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
    bool doPass[kPasses];
    for (int p = 0; p < kPasses; ++p)
    {
        doPass[p] = true;
        for (int d = 0; d < kRadix; ++d)
        {
            if (h[p * kRadix + d] == n) { doPass[p] = false; }
        }
    }

    unsigned mask = 0;
    for (int p = 0; p < kPasses; ++p)
    {
        mask |= doPass[p] ? (1u << p) : 0u;
    }
    SPHB_TRY(runPasses(keys, values, n, s, mask, stream));
    uint32_t err = 0;
    // a plain read: this path serves sphb_sort_by_key_static, which must call no allocating routine (the pinned
    // block of readBack is allocated on its first use in a thread)
    SPHB_CUDA_TRY(cudaMemcpyAsync(&err, s.counters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
    // 1: a look-back wait gave up; 2: offsets left inconsistent by such a wait (nothing else produces them)
    return err ? kErrTimeout : kOk;
}

int sortNearlySorted(uint64_t* keys, uint32_t* values, size_t n, void* scratch, size_t scratchBytes, bool* identity,
                     cudaStream_t stream)
{
    *identity = false;
    if (n == 0)
    {
        *identity = true;
        return kOk;
    }
    if (n >= (size_t(1) << 30)) { return kErrArg; }
    if (!scratch || scratchBytes < sortScratchBytes(n)) { return kErrCapacity; }
    SortScratch s = carve(scratch, n);
    iotaKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(values, n);
    SPHB_CUDA_TRY(cudaGetLastError());
    unsigned blocks = unsigned(std::min<size_t>(ceilDiv(n, 256 * 8), size_t(smCount()) * 8));
    auto countInversions = [&](uint32_t* out) -> int {
        SPHB_CUDA_TRY(cudaMemsetAsync(s.counters, 0, sizeof(uint32_t), stream));
        inversionsKernel<<<blocks, 256, 0, stream>>>(keys, n, s.counters);
        SPHB_CUDA_TRY(cudaGetLastError());
        SPHB_TRY(readBack(stream, {{out, s.counters, sizeof(uint32_t)}}));
        return kOk;
    };
    uint32_t inv = 0;
    SPHB_TRY(countInversions(&inv));
    if (inv == 0)
    {
        *identity = true;
        return kOk;
    }
    // sparse, local disorder: stable sorts of the dirty tiles, then of the tiles shifted by half a tile
    size_t tiles = ceilDiv(n, size_t(kRepairTile));
    repairTilesKernel<<<unsigned(tiles), kRepairThreads, 0, stream>>>(keys, values, n, 0);
    repairTilesKernel<<<unsigned(ceilDiv(n, size_t(kRepairTile))), kRepairThreads, 0, stream>>>(keys, values, n,
                                                                                               kRepairTile / 2);
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_TRY(countInversions(&inv));
    if (inv == 0) { return kOk; }
    // otherwise the full radix sort; the repaired sequence kept equal keys in their original order, so a stable
    // sort of it is the stable sort of the original
    return sortByKey(keys, values, n, false, scratch, scratchBytes, stream);
}

int sortByKeyAsync(uint64_t* keys, uint32_t* values, size_t n, bool initValues, void* scratch, size_t scratchBytes,
                   unsigned passMask, uint32_t* errorOut, cudaStream_t stream, const uint32_t* gate)
{
    if (n == 0) { return kOk; }
    if (n >= (size_t(1) << 30)) { return kErrArg; }
    if (!scratch || scratchBytes < sortScratchBytes(n)) { return kErrCapacity; }
    SortScratch s = carve(scratch, n);
    if (initValues)
    {
        iotaKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(values, n);
        SPHB_CUDA_TRY(cudaGetLastError());
    }
    SPHB_CUDA_TRY(cudaMemsetAsync(s.hist, 0, kPasses * kRadix * sizeof(uint32_t), stream));
    unsigned histBlocks = unsigned(std::min<size_t>(ceilDiv(n, 256 * 16), size_t(smCount()) * 4));
    histogramKernel<<<histBlocks, 256, 0, stream>>>(keys, n, s.hist, gate);
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_TRY(runPasses(keys, values, n, s, passMask, stream, gate));
    if (errorOut) { orErrorKernel<<<1, 1, 0, stream>>>(s.counters + 1, errorOut); }
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

namespace
{

//! keys/values from the alternate buffers, unless the gate is closed (the passes did not run)
__global__ void gatedCopyKernel(const uint64_t* kIn, const uint32_t* vIn, uint64_t* kOut, uint32_t* vOut, size_t n,
                                const uint32_t* gate)
{
    if (*gate == 0) { return; }
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        kOut[i] = kIn[i];
        vOut[i] = vIn[i];
    }
}

//! scan the histograms and run the passes of passMask (bit p: digit p), leaving the result in keys/values; with a
//! gate, every kernel returns at once when *gate is 0 (device-side decision, capturable)
int runPasses(uint64_t* keys, uint32_t* values, size_t n, const SortScratch& s, unsigned passMask,
              cudaStream_t stream, const uint32_t* gate)
{
    histScanKernel<<<kPasses, kRadix, 0, stream>>>(s.hist, gate);
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_CUDA_TRY(cudaMemsetAsync(s.counters + 1, 0, sizeof(uint32_t), stream));

    size_t tiles      = numTilesOf(n);
    uint64_t* kIn     = keys;
    uint32_t* vIn     = values;
    uint64_t* kOut    = s.keysAlt;
    uint32_t* vOut    = s.valsAlt;
    for (int p = 0; p < kPasses; ++p)
    {
        if (!(passMask & (1u << p))) { continue; }
        SPHB_CUDA_TRY(cudaMemsetAsync(s.status, 0, tiles * kRadix * sizeof(uint32_t), stream));
        SPHB_CUDA_TRY(cudaMemsetAsync(s.counters, 0, sizeof(uint32_t), stream));
        onesweepKernel<<<unsigned(tiles), kSortThreads, 0, stream>>>(kIn, vIn, kOut, vOut, n, p * kRadixBits,
                                                                      s.hist + p * kRadix, s.status, s.counters,
                                                                      gate);
        SPHB_CUDA_TRY(cudaGetLastError());
        std::swap(kIn, kOut);
        std::swap(vIn, vOut);
    }
    if (kIn != keys && gate)
    {
        unsigned blocks = unsigned(std::min<size_t>(ceilDiv(n, 256), size_t(smCount()) * 8));
        gatedCopyKernel<<<blocks, 256, 0, stream>>>(kIn, vIn, keys, values, n, gate);
        SPHB_CUDA_TRY(cudaGetLastError());
    }
    else if (kIn != keys)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(keys, kIn, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, stream));
        SPHB_CUDA_TRY(cudaMemcpyAsync(values, vIn, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, stream));
    }
    return kOk;
}

} // namespace

int repairSegmentedAsync(uint64_t* keys, uint32_t* values, const uint64_t* seg, size_t n, uint32_t* flags,
                         cudaStream_t stream)
{
    SPHB_CUDA_TRY(cudaMemsetAsync(flags, 0, 2 * sizeof(uint32_t), stream));
    if (n == 0) { return kOk; }
    unsigned blocks = unsigned(std::min<size_t>(ceilDiv(n, 256 * 8), size_t(smCount()) * 8));
    iotaKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(values, n);
    inversionsSegKernel<<<blocks, 256, 0, stream>>>(keys, seg, n, flags);
    repairTilesSegKernel<<<unsigned(ceilDiv(n, size_t(kRepairTile))), kRepairThreads, 0, stream>>>(keys, values, seg,
                                                                                                   n, 0);
    repairTilesSegKernel<<<unsigned(ceilDiv(n, size_t(kRepairTile))), kRepairThreads, 0, stream>>>(
        keys, values, seg, n, kRepairTile / 2);
    inversionsSegKernel<<<blocks, 256, 0, stream>>>(keys, seg, n, flags + 1);
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

// ---------------------------------------------------------------------------------------------------------------
// Allocation-free variant: the scratch lives in a fixed device array of this library (see sphb_sort_by_key_static)
// ---------------------------------------------------------------------------------------------------------------

//! largest n accepted by the allocation-free sort
constexpr size_t kStaticSortMaxN = size_t(1) << 20;

constexpr size_t alignUpC(size_t x, size_t a) { return (x + a - 1) / a * a; }

constexpr size_t kStaticSortBytes = alignUpC(kStaticSortMaxN * sizeof(uint64_t), 256) +
                                    alignUpC(kStaticSortMaxN * sizeof(uint32_t), 256) +
                                    alignUpC(kPasses * kRadix * sizeof(uint32_t), 256) +
                                    alignUpC((kStaticSortMaxN + kTile - 1) / kTile * kRadix * sizeof(uint32_t), 256) +
                                    256;

/*! Scratch of the allocation-free sort: ~12.6 MB of device memory that every GPU which loads this library holds until
 *  the process exits. Host code must not use the symbol itself as a device address; it asks the runtime for the
 *  device address of this array once per device (staticSortScratch below). */
static __device__ __align__(256) unsigned char gStaticSortScratch[kStaticSortBytes];

namespace
{

//! one looked-up address per CUDA context: a context created after cudaDeviceReset gets its own entry
struct StaticScratchEntry
{
    CUcontext ctx;
    void* addr;
};
constexpr int kMaxContexts = 64;
std::mutex gStaticScratchMutex;
StaticScratchEntry gStaticScratch[kMaxContexts] = {};
int gStaticScratchNext                          = 0;
PFN_cuCtxGetCurrent_v4000 gCtxGetCurrent        = nullptr;

/*! Device address of gStaticSortScratch in the current context, looked up with the context's device current on the
 *  first call in that context. The driver's cuCtxGetCurrent is reached through the runtime's entry-point query, so
 *  this library does not link libcuda. */
int staticSortScratch(void** ptr)
{
    std::lock_guard<std::mutex> lock(gStaticScratchMutex);
    if (!gCtxGetCurrent)
    {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SPHB_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) { return kErrCuda; }
        gCtxGetCurrent = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    }
    CUcontext ctx = nullptr;
    if (gCtxGetCurrent(&ctx) != CUDA_SUCCESS) { return kErrCuda; }
    if (!ctx)
    {
        // no context is current on this thread yet: make the current device's primary context current
        int dev = 0;
        SPHB_CUDA_TRY(cudaGetDevice(&dev));
        SPHB_CUDA_TRY(cudaSetDevice(dev));
        if (gCtxGetCurrent(&ctx) != CUDA_SUCCESS || !ctx) { return kErrCuda; }
    }
    for (const StaticScratchEntry& e : gStaticScratch)
    {
        if (e.ctx == ctx && e.addr)
        {
            *ptr = e.addr;
            return kOk;
        }
    }
    void* p = nullptr;
    SPHB_CUDA_TRY(cudaGetSymbolAddress(&p, gStaticSortScratch));
    gStaticScratch[gStaticScratchNext] = {ctx, p};
    gStaticScratchNext                 = (gStaticScratchNext + 1) % kMaxContexts;
    *ptr                               = p;
    return kOk;
}

} // namespace

} // namespace sphb

extern "C" size_t sphb_sort_by_key_static_max(void) { return sphb::kStaticSortMaxN; }

extern "C" int sphb_sort_by_key_static(uint64_t* keys, uint32_t* values, size_t n, int init_values, void* stream)
{
    if (n && (!keys || !values)) { return SPHB_ERR_ARG; }
    if (n > sphb::kStaticSortMaxN)
    {
        std::fprintf(stderr, "sphb_sort_by_key_static: n = %zu exceeds the fixed scratch capacity of %zu pairs\n", n,
                     sphb::kStaticSortMaxN);
        return SPHB_ERR_CAPACITY;
    }
    void* scratch = nullptr;
    int rc        = sphb::staticSortScratch(&scratch);
    if (rc != SPHB_OK) { return rc; }
    return sphb::sortByKey(keys, values, n, init_values != 0, scratch, sphb::kStaticSortBytes,
                           static_cast<cudaStream_t>(stream));
}

extern "C" size_t sphb_sort_by_key_scratch_bytes(size_t n) { return sphb::sortScratchBytes(n); }

extern "C" int sphb_sort_by_key(uint64_t* keys, uint32_t* values, size_t n, int init_values, void* scratch,
                                size_t scratch_bytes, void* stream)
{
    if (n && (!keys || !values)) { return SPHB_ERR_ARG; }
    return sphb::sortByKey(keys, values, n, init_values != 0, scratch, scratch_bytes,
                           static_cast<cudaStream_t>(stream));
}

extern "C" int sphb_sort_by_key_nearly_sorted(uint64_t* keys, uint32_t* values, size_t n, void* scratch,
                                              size_t scratch_bytes, int* identity, void* stream)
{
    if (!identity || (n && (!keys || !values))) { return SPHB_ERR_ARG; }
    bool id = false;
    int rc  = sphb::sortNearlySorted(keys, values, n, scratch, scratch_bytes, &id, static_cast<cudaStream_t>(stream));
    *identity = id ? 1 : 0;
    return rc;
}
