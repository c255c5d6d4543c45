// Device functions for Hilbert keys and the cornerstone key arithmetic.
#pragma once

#include "common.cuh"

namespace sphb
{

/*! 3D Hilbert key from 21-bit integer coordinates.
 *
 * Same curve as cstone::iHilbert (cstone/sfc/hilbert.hpp:43-94, after Miki & Umemura, GOTHIC): walking from the
 * coarsest level, each level appends the Hilbert digit of the Morton octant (x<<2 | y<<1 | z) through the table
 * {0,1,3,2,7,6,4,5}, then reflects and permutes the remaining coordinate bits. The steps have to be the same for the
 * keys to be identical; the table is packed into one 32-bit constant (4 bits per octant).
 */
__host__ __device__ inline uint64_t hilbertKey(unsigned px, unsigned py, unsigned pz)
{
    constexpr uint32_t octantToDigit = 0x54672310u; // nibble o holds the Hilbert digit of Morton octant o
    uint64_t key                     = 0;
#pragma unroll
    for (int level = kMaxLevel - 1; level >= 0; --level)
    {
        unsigned xi = (px >> level) & 1u;
        unsigned yi = (py >> level) & 1u;
        unsigned zi = (pz >> level) & 1u;

        unsigned octant = (xi << 2) | (yi << 1) | zi;
        key             = (key << 3) | ((octantToDigit >> (4 * octant)) & 7u);

        unsigned ny = yi ^ 1u;
        unsigned nz = zi ^ 1u;
        px ^= 0u - (xi & (ny | zi));
        py ^= 0u - ((xi & (yi | zi)) | (yi & nz));
        pz ^= 0u - ((xi & ny & nz) | (yi & nz));

        // permute: zi rotates (x, y, z) -> (y, z, x); otherwise !yi swaps x and z (selects, no divergent branch)
        unsigned t0 = px, t1 = py, t2 = pz;
        px          = zi ? t1 : (yi ? t0 : t2);
        py          = zi ? t2 : t1;
        pz          = zi ? t0 : (yi ? t2 : t0);
    }
    return key;
}

/*! Inverse of hilbertKey: integer coordinates of a key.
 *
 * Walks the digits from the finest level up. Before level l is visited, p holds the l finest coordinate bits
 * expressed in the frame that hilbertKey had reached at level l-1; each step undoes that level's permutation and
 * reflection on those bits (the reflection masks depend only on the level's Morton octant) and then inserts the
 * octant's own bits at position l.
 */
__host__ __device__ inline void hilbertDecode(uint64_t key, unsigned p[3])
{
    constexpr uint32_t digitToOctant = 0x45762310u; // nibble h holds the Morton octant of Hilbert digit h
    unsigned px = 0, py = 0, pz = 0;
    for (unsigned level = 0; level < kMaxLevel; ++level)
    {
        unsigned digit  = unsigned(key >> (3u * level)) & 7u;
        unsigned octant = (digitToOctant >> (4u * digit)) & 7u;
        unsigned xi     = octant >> 2;
        unsigned yi     = (octant >> 1) & 1u;
        unsigned zi     = octant & 1u;
        unsigned mask   = (1u << level) - 1u;

        if (zi)
        {
            unsigned t = pz; // undo (x,y,z) <- (y,z,x)
            pz         = py;
            py         = px;
            px         = t;
        }
        else if (!yi)
        {
            unsigned t = px;
            px         = pz;
            pz         = t;
        }
        unsigned ny = yi ^ 1u;
        unsigned nz = zi ^ 1u;
        px ^= mask & (0u - (xi & (ny | zi)));
        py ^= mask & (0u - ((xi & (yi | zi)) | (yi & nz)));
        pz ^= mask & (0u - ((xi & ny & nz) | (yi & nz)));

        px |= xi << level;
        py |= yi << level;
        pz |= zi << level;
    }
    p[0] = px;
    p[1] = py;
    p[2] = pz;
}

/*! Quantise one coordinate: int(floor(x*m) - lo*m), clamped above at 2^21-1 (cstone/sfc/sfc.hpp:141-159), with
 *  m = 2^21 / (hi - lo). Explicit round-to-nearest intrinsics keep the CPU's uncontracted rounding. */
__host__ __device__ inline unsigned quantiseCoord(double x, double lo, double ilen)
{
    constexpr int mcoord = (1 << kMaxLevel) - 1;
#ifdef __CUDA_ARCH__
    double m  = __dmul_rn(double(1u << kMaxLevel), ilen);
    double fx = floor(__dmul_rn(x, m));
    int ix    = int(__dsub_rn(fx, __dmul_rn(lo, m)));
#else
    double m  = double(1u << kMaxLevel) * ilen;
    double fx = floor(x * m);
    int ix    = int(fx - lo * m);
#endif
    return unsigned(ix < mcoord ? ix : mcoord);
}

__host__ __device__ inline uint64_t hilbertKeyOf(double x, double y, double z, const DevBox& box)
{
    return hilbertKey(quantiseCoord(x, box.lo[0], box.ilen[0]), quantiseCoord(y, box.lo[1], box.ilen[1]),
                      quantiseCoord(z, box.lo[2], box.ilen[2]));
}

//! octree level of a cornerstone node of key range `range` (range = 8^(21 - level)); cstone/sfc/common.hpp treeLevel
__host__ __device__ inline unsigned treeLevelOf(uint64_t range)
{
#ifdef __CUDA_ARCH__
    unsigned lz = __clzll(range);
#else
    unsigned lz = __builtin_clzll(range);
#endif
    // range = 2^(3*(21-level)), leading zeros = 63 - 3*(21-level) = 3*level
    return lz / 3;
}

//! key range of a node at `level`
__host__ __device__ inline uint64_t nodeRangeAt(unsigned level) { return uint64_t(1) << (3u * (kMaxLevel - level)); }

//! placeholder-bit prefix of the node (start key, level): key >> (63 - 3 level) | 1 << 3 level (cstone/sfc/common.hpp)
__host__ __device__ inline uint64_t encodePrefix(uint64_t start, unsigned level)
{
    unsigned len = 3u * level;
    return (len ? (start >> (63u - len)) : uint64_t(0)) | (uint64_t(1) << len);
}

__host__ __device__ inline unsigned prefixLevel(uint64_t prefix)
{
#ifdef __CUDA_ARCH__
    unsigned lz = __clzll(prefix);
#else
    unsigned lz = __builtin_clzll(prefix);
#endif
    return (63u - lz) / 3u;
}

__host__ __device__ inline uint64_t prefixStart(uint64_t prefix)
{
    unsigned level = prefixLevel(prefix);
    unsigned len   = 3u * level;
    uint64_t body  = prefix ^ (uint64_t(1) << len);
    return len ? (body << (63u - len)) : uint64_t(0);
}

int launchSfcKeys(const double* x, const double* y, const double* z, uint64_t* keys, size_t n, const DevBox& box,
                  cudaStream_t stream);

} // namespace sphb
