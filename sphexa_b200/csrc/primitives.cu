// Scans and gathers (see primitives.cuh).
#include <cstring>

#include "primitives.cuh"

namespace sphb
{

uint64_t& launchCounter()
{
    static uint64_t counter = 0;
    return counter;
}

int smCount()
{
    static int sms = 0;
    if (sms == 0)
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) { sms = 148; }
    }
    return sms;
}

unsigned long long* pinnedReadback()
{
    struct Block
    {
        unsigned long long* p{nullptr};
        Block()
        {
            if (cudaHostAlloc(reinterpret_cast<void**>(&p), kReadbackWords * sizeof(unsigned long long),
                              cudaHostAllocPortable) != cudaSuccess)
            {
                p = nullptr;
                cudaGetLastError();
            }
        }
        ~Block()
        {
            if (p) { cudaFreeHost(p); }
        }
    };
    thread_local Block block;
    return block.p;
}

int readBack(cudaStream_t stream, std::initializer_list<ReadItem> items)
{
    unsigned long long* pin = pinnedReadback();
    size_t total            = 0;
    for (const ReadItem& it : items)
    {
        total += (it.bytes + 7) / 8 * 8;
    }
    if (!pin || total > kReadbackWords * sizeof(unsigned long long))
    {
        for (const ReadItem& it : items)
        {
            SPHB_CUDA_TRY(cudaMemcpyAsync(it.dst, it.src, it.bytes, cudaMemcpyDeviceToHost, stream));
        }
        SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
        return kOk;
    }
    size_t off = 0;
    for (const ReadItem& it : items)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(pin) + off, it.src, it.bytes, cudaMemcpyDeviceToHost,
                                      stream));
        off += (it.bytes + 7) / 8 * 8;
    }
    SPHB_CUDA_TRY(cudaStreamSynchronize(stream));
    off = 0;
    for (const ReadItem& it : items)
    {
        std::memcpy(it.dst, reinterpret_cast<const char*>(pin) + off, it.bytes);
        off += (it.bytes + 7) / 8 * 8;
    }
    return kOk;
}

namespace
{

constexpr int kScanThreads = 1024;
constexpr int kScanItems   = 4;
constexpr int kScanTile    = kScanThreads * kScanItems;

//! block-wide exclusive scan of one value per thread; returns the block total through *total
__device__ int blockExclusiveScan(int v, int* total)
{
    __shared__ int warpSums[33]; // 32 warp offsets + the block total
    int lane = threadIdx.x & 31;
    int warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1)
    {
        int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) { incl += t; }
    }
    if (lane == 31) { warpSums[warp] = incl; }
    __syncthreads();
    if (warp == 0)
    {
        int nw = blockDim.x >> 5;
        int s  = lane < nw ? warpSums[lane] : 0;
        int si = s;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            int t = __shfl_up_sync(0xffffffffu, si, off);
            if (lane >= off) { si += t; }
        }
        if (lane < nw) { warpSums[lane] = si - s; }
        if (lane == nw - 1) { warpSums[32] = si; }
    }
    __syncthreads();
    int res = incl - v + warpSums[warp];
    int tot = warpSums[32];
    __syncthreads();
    *total = tot;
    return res;
}

__global__ void __launch_bounds__(kScanThreads) tileSumKernel(const int* in, size_t n, int* tileSums)
{
    size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
    int s       = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        if (base + k < n) { s += in[base + k]; }
    }
    int total;
    blockExclusiveScan(s, &total);
    if (threadIdx.x == 0) { tileSums[blockIdx.x] = total; }
}

__global__ void __launch_bounds__(kScanThreads) scanTileSumsKernel(int* tileSums, int numTiles)
{
    // numTiles <= kScanThreads * kScanItems
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int idx = threadIdx.x * kScanItems + k;
        v[k]    = idx < numTiles ? tileSums[idx] : 0;
        s += v[k];
    }
    int total;
    int ex = blockExclusiveScan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        int idx = threadIdx.x * kScanItems + k;
        if (idx < numTiles) { tileSums[idx] = ex; }
        ex += v[k];
    }
    if (threadIdx.x == 0) { tileSums[numTiles] = total; }
}

__global__ void __launch_bounds__(kScanThreads) scanTilesKernel(const int* in, int* out, size_t n,
                                                                 const int* tileOffsets, int numTiles)
{
    size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int ex = blockExclusiveScan(s, &total) + tileOffsets[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        if (base + k < n) { out[base + k] = ex; }
        ex += v[k];
    }
    if (blockIdx.x == numTiles - 1 && threadIdx.x == 0) { out[n] = tileOffsets[numTiles]; }
}

struct Gather8Args
{
    const uint64_t* src[16];
    uint64_t* dst[16];
};

__global__ void gather8Kernel(const uint32_t* __restrict__ order, size_t n, int numFields, Gather8Args a)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    uint32_t j = order[i];
    for (int f = 0; f < numFields; ++f)
    {
        a.dst[f][i] = __ldg(a.src[f] + j);
    }
}

} // namespace

size_t scanTempInts(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

int exclusiveScan(const int* in, int* out, size_t n, int* tmp, cudaStream_t stream)
{
    if (n == 0)
    {
        SPHB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int), stream));
        return kOk;
    }
    size_t numTiles = (n + kScanTile - 1) / kScanTile;
    if (numTiles > size_t(kScanTile)) { return kErrCapacity; }
    tileSumKernel<<<unsigned(numTiles), kScanThreads, 0, stream>>>(in, n, tmp);
    scanTileSumsKernel<<<1, kScanThreads, 0, stream>>>(tmp, int(numTiles));
    scanTilesKernel<<<unsigned(numTiles), kScanThreads, 0, stream>>>(in, out, n, tmp, int(numTiles));
    countLaunch(3);
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int gather8(const uint32_t* order, size_t n, int numFields, const void* const* src, void* const* dst,
            cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    for (int f0 = 0; f0 < numFields; f0 += 16)
    {
        Gather8Args a;
        int nf = std::min(16, numFields - f0);
        for (int f = 0; f < nf; ++f)
        {
            a.src[f] = static_cast<const uint64_t*>(src[f0 + f]);
            a.dst[f] = static_cast<uint64_t*>(dst[f0 + f]);
        }
        gather8Kernel<<<ceilDiv(n, 256), 256, 0, stream>>>(order, n, nf, a);
        countLaunch();
        SPHB_CUDA_TRY(cudaGetLastError());
    }
    return kOk;
}

} // namespace sphb

extern "C" int sphb_gather8(const uint32_t* order, size_t n, int num_fields, const void* const* src,
                            void* const* dst, void* stream)
{
    if (num_fields < 0 || (n && num_fields && (!order || !src || !dst))) { return SPHB_ERR_ARG; }
    return sphb::gather8(order, n, num_fields, src, dst, static_cast<cudaStream_t>(stream));
}
