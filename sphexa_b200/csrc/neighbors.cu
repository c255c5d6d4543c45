// Neighbour search on sm_100a: one warp per target group of 32 consecutive (SFC-ordered) particles.
//
// Per group: (1) the search box = union over the group's still-active particles of [x - 2h, x + 2h];
// (2) a depth-first traversal of the focus octree in child (= SFC) order, warp-cooperative with 8 lanes testing the
// 8 children of a node against the box (periodic axes use the minimum image), collecting overlapping leaves in
// ascending order in shared memory; (3) each buffered leaf is cut into the 8-particle SFC blocks it covers, every
// block's bounding box (precomputed once per step) is tested against the search box 32 blocks at a time, and the
// particles of surviving blocks are streamed 32 at a time through shared memory; (4) every lane tests the staged
// candidates against its own particle, two candidates per packed FP32x2 instruction on coordinates relative to the
// group centre, and runs the exact FP64 test of the reference (cstone/findneighbors.hpp:33-51,77-147: squared
// minimum-image distance < (2h)^2, j != i) only for candidates within a narrow band around the radius.
// Candidates arrive in ascending particle order, so each list equals the reference CPU list, which is also ascending
// (depth-first octree traversal over SFC-ordered leaves), including which neighbours are kept when more than ngmax
// qualify. The smoothing-length iteration of sph/include/sph/find_neighbors.hpp:10-41 is fused: lanes whose count
// left [ng0/4, ngmax+1] update h and search again, at most maxIterations times; settled lanes keep their lists.
#include "neighbors.cuh"
#include "primitives.cuh"

namespace sphb
{

namespace
{

constexpr int kNbWarps   = 4;
constexpr int kNbThreads = kNbWarps * kWarp;
constexpr int kStackCap  = 176; // depth-first stack: <= 7 pending siblings per level + 8
constexpr int kLeafCap   = 256; // candidate leaves buffered before they are streamed

struct NbShared
{
    int stack[kNbWarps][kStackCap];
    int leafFirst[kNbWarps][kLeafCap]; // first particle of each buffered leaf
    int leafEnd[kNbWarps][kLeafCap];   // one past its last particle
    int blkPre[kNbWarps][kLeafCap + 1]; // exclusive prefix of the number of blocks per buffered leaf
    int pStart[kNbWarps][kWarp];       // surviving pieces (block and leaf intersections) of one round
    int pPre[kNbWarps][kWarp + 1];     // exclusive prefix of their lengths
    uint8_t pieceOf[kNbWarps][kWarp * kBlockSize]; // candidate of the round -> its piece
    // staged candidates: position relative to the group centre (FP32, pairs loaded as float2) and index
    alignas(16) float cx[kNbWarps][kWarp];
    alignas(16) float cy[kNbWarps][kWarp];
    alignas(16) float cz[kNbWarps][kWarp];
    int cj[kNbWarps][kWarp];
    // per lane: the neighbours of the list chunk being filled, written out as one 32-byte sector when full; lane
    // minor, so that the lanes' appends fall into distinct banks
    uint32_t nbuf[kNbWarps][kNbChunk][kWarp];
    uint16_t dbuf[kNbWarps][kNbChunk][kWarp]; // skin rows: the quantised build distance of each entry
};

/*! Half width of the band |d^2 - (2h)^2| < band * (2h)^2 in which the FP32 distance cannot decide and the exact FP64
 *  test runs. Relative coordinates are formed in FP64 and rounded once to FP32, so each has an error of at most
 *  2^-24 S, S = the largest distance from the group centre at which a neighbour of the group can lie. For a pair at
 *  distance ~2h that bounds the FP32 squared-distance error by about 2^-21 (S / 2h + 1) (2h)^2 including the FP32
 *  arithmetic; the band is four times that. */
__device__ inline float bandOf(float S, float twoH) { return 2.0e-6f * (S / twoH + 1.0f); }

__device__ inline double warpMin(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

__device__ inline double warpMax(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

//! warp-wide exclusive prefix of one value per lane; *total receives the sum
__device__ inline int warpExclusive(int v, int lane, int* total)
{
    int incl = v;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1)
    {
        int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) { incl += t; }
    }
    *total = __shfl_sync(0xffffffffu, incl, kWarp - 1);
    return incl - v;
}

//! largest r in [0, n) with pre[r] <= t (pre ascending, pre[0] = 0 <= t)
__device__ inline int findSlot(const int* pre, int n, int t)
{
    int lo = 0, hi = n;
    while (hi - lo > 1)
    {
        int mid = (lo + hi) >> 1;
        if (pre[mid] <= t) { lo = mid; }
        else { hi = mid; }
    }
    return lo;
}

//! 32-byte read-only load of a packed position (two 16-byte loads of one sector)
__device__ inline double4 ldPos(const double4* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 lo = __ldg(q), hi = __ldg(q + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

//! what one launch of the search computes
enum SearchKind : int
{
    kSearchAll,    // neighbour lists of every group, with the smoothing-length iteration
    kSearchListed, // the same for the groups of a device-side list
    kSearchSkin    // skin lists: every j within 2 h (1 + skin), no iteration, h read only
};

//! launch inputs of the listed and skin searches
struct SearchExtras
{
    const unsigned* groups;
    const unsigned* numListed;
    SkinLists sl;
    double onePlusSkin;
    const unsigned* gate; // if set: the launch runs only when bit *gate of gateMask is set (a device-side mode)
    unsigned gateMask;
};

template<bool kBatched, int kKind>
__global__ void __launch_bounds__(kNbThreads, 8) findNeighborsKernel(const double* __restrict__ x,
                                                                  const double* __restrict__ y,
                                                                  const double* __restrict__ z,
                                                                  const double4* __restrict__ pos, double* h, size_t n,
                                                                  TreeView tree, DevBox box, NeighborParams prm,
                                                                  uint32_t* __restrict__ nidx,
                                                                  unsigned* __restrict__ ncOut, unsigned* status,
                                                                  const TreeView* __restrict__ views,
                                                                  const uint8_t* __restrict__ inst, SearchExtras ex)
{
    __shared__ NbShared sh;
    if (ex.gate && !((ex.gateMask >> __ldg(ex.gate)) & 1u)) { return; }
    const int warp         = threadIdx.x / kWarp;
    const int lane         = threadIdx.x & (kWarp - 1);
    const size_t numGroups = (n + kWarp - 1) / kWarp;
    size_t group           = size_t(blockIdx.x) * kNbWarps + warp;
    if constexpr (kKind == kSearchListed)
    {
        if (group >= *ex.numListed) { return; }
        group = ex.groups[group];
    }
    if (group >= numGroups) { return; }
    constexpr bool kSkin = kKind == kSearchSkin;
    // the lists written: neighbour lists (ngmax entries) or skin rows (cap entries)
    uint32_t* const outList  = kSkin ? ex.sl.rows : nidx;
    const unsigned listCap   = kSkin ? ex.sl.cap : prm.ngmax;

    const size_t i = group * kWarp + lane;
    // an ensemble: the group's instance (its first slot is never padding) selects the tree; padding slots idle
    TreeView tv = tree;
    if constexpr (kBatched) { tv = views[inst[group * kWarp]]; }
    const bool valid = i < n && !(kBatched && inst[i] == kGhost);
    const double xi  = valid ? x[i] : 0.0;
    const double yi  = valid ? y[i] : 0.0;
    const double zi  = valid ? z[i] : 0.0;
    double hi        = valid ? h[i] : 0.0;

    const unsigned ngmin = prm.ng0 / 4;
    const unsigned ngPad = kSkin ? ex.sl.cap : paddedNgmax(prm.ngmax);
    bool active          = valid;
    int updates          = 0;
    unsigned count       = 0;
    bool overflow        = false;

    int* stack     = sh.stack[warp];
    int* leafFirst = sh.leafFirst[warp];
    int* leafEnd   = sh.leafEnd[warp];
    int* blkPre    = sh.blkPre[warp];
    int* pStart    = sh.pStart[warp];
    int* pPre      = sh.pPre[warp];

    while (__ballot_sync(0xffffffffu, active) != 0u && !overflow)
    {
        const double r        = kSkin ? __dmul_rn(2.0 * hi, ex.onePlusSkin) : 2.0 * hi;
        // the exact test: (2h)^2 as the reference computes it, or R^2 for skin rows
        const double radiusSq = kSkin ? __dmul_rn(r, r) : searchRadiusSq(hi);
        double blo[3], bhi[3];
        blo[0] = warpMin(active ? xi - r : INFINITY);
        blo[1] = warpMin(active ? yi - r : INFINITY);
        blo[2] = warpMin(active ? zi - r : INFINITY);
        bhi[0] = warpMax(active ? xi + r : -INFINITY);
        bhi[1] = warpMax(active ? yi + r : -INFINITY);
        bhi[2] = warpMax(active ? zi + r : -INFINITY);
        double gc[3], gs[3];
        float gcb[3], gsb[3], lenf[3], ilenf[3]; // group box in the block-box frame (relative to the box corner)
        for (int k = 0; k < 3; ++k)
        {
            gc[k]    = 0.5 * (blo[k] + bhi[k]);
            gs[k]    = 0.5 * (bhi[k] - blo[k]) * (1.0 + 1e-12) + 1e-14 * box.len[k];
            gcb[k]   = float(gc[k] - box.lo[k]);
            gsb[k]   = __double2float_ru(gs[k] + 4e-7 * box.len[k]);
            lenf[k]  = float(box.len[k]);
            ilenf[k] = float(box.ilen[k]);
        }
        // this particle relative to the group centre in FP32, and the FP32 acceptance band
        const float rix  = float(minImage(xi - gc[0], box.len[0], box.ilen[0], box.periodic[0]));
        const float riy  = float(minImage(yi - gc[1], box.len[1], box.ilen[1], box.periodic[1]));
        const float riz  = float(minImage(zi - gc[2], box.len[2], box.ilen[2], box.periodic[2]));
        const float twoH = float(r);
        const float r2f  = twoH * twoH;
        float reach      = active ? sqrtf(rix * rix + riy * riy + riz * riz) * 1.001f + twoH : 0.f;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            reach = fmaxf(reach, __shfl_xor_sync(0xffffffffu, reach, off));
        }
        // Differences of two coordinates that were each folded to the nearest image of the group centre are the
        // minimum image of the pair only while 2h + (offset from the centre) < L/2 on every periodic axis. Groups
        // whose reach exceeds that (search radii comparable to the box) test every candidate exactly instead.
        bool wrapTest = false;
        float maxSpan = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            if (box.periodic[k])
            {
                wrapTest = wrapTest || reach >= 0.5f * lenf[k];
                maxSpan  = fmaxf(maxSpan, 0.5f * lenf[k]);
            }
        }
        const float band = active ? bandOf(wrapTest ? fmaxf(reach, maxSpan) : reach, twoH) : 0.f;
        const float r2lo = r2f * (1.f - band);
        const float r2hi = r2f * (1.f + band);

        if (active) { count = 0; }
        int numLeaves = 0;

        // this lane's chunk buffer and its store to the chunked list layout (nidxAt)
        uint32_t* chunk     = &sh.nbuf[warp][0][lane];
        uint16_t* dchunk    = &sh.dbuf[warp][0][lane];
        const double qScale = kSkinDistUnits / r; // skin rows: distance -> units of R / kSkinDistUnits
        auto storeChunk = [&](unsigned c) {
            uint32_t* dst = outList + nidxAt(group, ngPad, c * kNbChunk, lane);
            if constexpr (kSkin)
            {
                uint4 d;
                d.x = unsigned(dchunk[0]) | (unsigned(dchunk[kWarp]) << 16);
                d.y = unsigned(dchunk[2 * kWarp]) | (unsigned(dchunk[3 * kWarp]) << 16);
                d.z = unsigned(dchunk[4 * kWarp]) | (unsigned(dchunk[5 * kWarp]) << 16);
                d.w = unsigned(dchunk[6 * kWarp]) | (unsigned(dchunk[7 * kWarp]) << 16);
                *reinterpret_cast<uint4*>(ex.sl.dist + nidxAt(group, ngPad, c * kNbChunk, lane)) = d;
            }
            // one 256-bit streaming store of the whole sector (the lists are next read once per J-loop)
            asm volatile("st.global.cs.v8.u32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(dst), "r"(chunk[0]),
                         "r"(chunk[kWarp]), "r"(chunk[2 * kWarp]), "r"(chunk[3 * kWarp]), "r"(chunk[4 * kWarp]),
                         "r"(chunk[5 * kWarp]), "r"(chunk[6 * kWarp]), "r"(chunk[7 * kWarp])
                         : "memory");
        };

        // test the staged 32 candidates against this lane's particle and append the neighbours in index order
        auto testStaged = [&](int numReal) {
            if (!active) { return; }
            // bit k of sure: candidate k lies inside the sphere by its FP32 distance (below the band); of maybe: it
            // may (below the upper edge of the band)
            unsigned maybe = 0u, sure = 0u;
            if (!wrapTest)
            {
                const float2 mx = make_float2(-rix, -rix), my = make_float2(-riy, -riy), mz = make_float2(-riz, -riz);
#pragma unroll
                for (int k = 0; k < kWarp; k += 2)
                {
                    float2 X  = *reinterpret_cast<const float2*>(&sh.cx[warp][k]);
                    float2 Y  = *reinterpret_cast<const float2*>(&sh.cy[warp][k]);
                    float2 Z  = *reinterpret_cast<const float2*>(&sh.cz[warp][k]);
                    float2 dx = __fadd2_rn(X, mx);
                    float2 dy = __fadd2_rn(Y, my);
                    float2 dz = __fadd2_rn(Z, mz);
                    float2 d2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                    maybe |= (unsigned(d2.x < r2hi) << k) | (unsigned(d2.y < r2hi) << (k + 1));
                    sure |= (unsigned(d2.x < r2lo) << k) | (unsigned(d2.y < r2lo) << (k + 1));
                }
            }
            else
            {
                // every real candidate of the chunk goes through the exact FP64 test below, which folds the pair
                // difference itself (padding sits at the end of the last chunk)
                maybe = numReal >= kWarp ? 0xffffffffu : ((1u << numReal) - 1u);
            }
            // candidates too close to the search radius for FP32: the exact test of the reference (rare)
            unsigned band = maybe & ~sure;
            while (band)
            {
                int k = __ffs(band) - 1;
                band &= band - 1u;
                int j      = sh.cj[warp][k];
                double4 pj = ldPos(pos + j);
                if (exactDistSq(pj.x, pj.y, pj.z, xi, yi, zi, box) < radiusSq) { sure |= 1u << k; }
            }
            // append the neighbours in candidate (= index) order
            while (sure)
            {
                int k = __ffs(sure) - 1;
                sure &= sure - 1u;
                int j = sh.cj[warp][k];
                if (size_t(j) == i) { continue; }
                if (count < listCap)
                {
                    if constexpr (kSkin)
                    {
                        // the build distance, from the reference's FP64 expression, for the refilter's bounds
                        double4 pj = ldPos(pos + j);
                        double q   = rint(sqrt(exactDistSq(pj.x, pj.y, pj.z, xi, yi, zi, box)) * qScale);
                        dchunk[(count % kNbChunk) * kWarp] = uint16_t(fmin(q, kSkinDistUnits));
                    }
                    chunk[(count % kNbChunk) * kWarp] = uint32_t(j);
                    if (count % kNbChunk == kNbChunk - 1) { storeChunk(count / kNbChunk); }
                }
                ++count;
            }
        };

        // stream the buffered candidate leaves, pruned to the 8-particle blocks that meet the search box
        auto flush = [&]() {
            int local[kLeafCap / kWarp];
            int sum = 0;
#pragma unroll
            for (int q = 0; q < kLeafCap / kWarp; ++q)
            {
                int t   = lane * (kLeafCap / kWarp) + q;
                int nbk = 0;
                if (t < numLeaves)
                {
                    int b = leafFirst[t], e = leafEnd[t];
                    nbk   = e > b ? (e - 1) / kBlockSize - b / kBlockSize + 1 : 0;
                }
                local[q] = nbk;
                sum += nbk;
            }
            int totalBlocks;
            int run = warpExclusive(sum, lane, &totalBlocks);
#pragma unroll
            for (int q = 0; q < kLeafCap / kWarp; ++q)
            {
                int t = lane * (kLeafCap / kWarp) + q;
                if (t < numLeaves) { blkPre[t] = run; }
                run += local[q];
            }
            __syncwarp();

            for (int base = 0; base < totalBlocks; base += kWarp)
            {
                int t     = base + lane;
                bool keep = false;
                int ps = 0, plen = 0;
                if (t < totalBlocks)
                {
                    int rr = findSlot(blkPre, numLeaves, t);
                    int b = leafFirst[rr], e = leafEnd[rr];
                    int c = b / kBlockSize + (t - blkPre[rr]);
                    ps    = max(c * kBlockSize, b);
                    plen  = min(c * kBlockSize + kBlockSize, e) - ps;
                    float4 lo = __ldg(tv.blockLo + c);
                    float4 hb = __ldg(tv.blockHi + c);
                    float bl[3] = {lo.x, lo.y, lo.z};
                    float bh[3] = {hb.x, hb.y, hb.z};
                    keep = plen > 0;
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                    {
                        float d = 0.5f * (bl[k] + bh[k]) - gcb[k];
                        if (box.periodic[k]) { d -= lenf[k] * rintf(d * ilenf[k]); }
                        keep = keep && fabsf(d) <= gsb[k] + 0.5f * (bh[k] - bl[k]) + 1e-6f * lenf[k];
                    }
                }
                unsigned m = __ballot_sync(0xffffffffu, keep);
                int totalCand;
                int ex = warpExclusive(keep ? plen : 0, lane, &totalCand);
                if (keep)
                {
                    int pos     = __popc(m & ((1u << lane) - 1u));
                    pStart[pos] = ps;
                    pPre[pos]   = ex;
                    for (int q = 0; q < plen; ++q)
                    {
                        sh.pieceOf[warp][ex + q] = uint8_t(pos);
                    }
                }
                __syncwarp();
                for (int cbase = 0; cbase < totalCand; cbase += kWarp)
                {
                    int tc = cbase + lane;
                    if (tc < totalCand)
                    {
                        int rr = sh.pieceOf[warp][tc];
                        int j  = pStart[rr] + (tc - pPre[rr]);
                        if (j < 0 || size_t(j) >= n)
                        {
                            // a layout that points outside the particle arrays: report, stage a far-away point
                            atomicOr(status, 2u);
                            sh.cx[warp][lane] = INFINITY;
                            sh.cy[warp][lane] = INFINITY;
                            sh.cz[warp][lane] = INFINITY;
                            sh.cj[warp][lane] = -1;
                        }
                        else
                        {
                            sh.cx[warp][lane] =
                                float(minImage(x[j] - gc[0], box.len[0], box.ilen[0], box.periodic[0]));
                            sh.cy[warp][lane] =
                                float(minImage(y[j] - gc[1], box.len[1], box.ilen[1], box.periodic[1]));
                            sh.cz[warp][lane] =
                                float(minImage(z[j] - gc[2], box.len[2], box.ilen[2], box.periodic[2]));
                            sh.cj[warp][lane] = j;
                        }
                    }
                    else
                    {
                        // pad with points that no sphere reaches, so the test is branch-free
                        sh.cx[warp][lane] = INFINITY;
                        sh.cy[warp][lane] = INFINITY;
                        sh.cz[warp][lane] = INFINITY;
                        sh.cj[warp][lane] = -1;
                    }
                    __syncwarp();
                    testStaged(totalCand - cbase);
                    __syncwarp();
                }
            }
            numLeaves = 0;
        };

        // depth-first traversal in SFC order
        int sp = 0;
        if (lane == 0) { stack[0] = 0; }
        sp = 1;
        __syncwarp();
        while (sp > 0)
        {
            int node = stack[sp - 1];
            --sp;
            int child0 = tv.childOffsets[node];
            if (child0 == 0)
            {
                if (numLeaves == kLeafCap) { flush(); }
                if (lane == 0)
                {
                    int leaf             = tv.nodeToLeaf[node];
                    leafFirst[numLeaves] = tv.layout[leaf];
                    leafEnd[numLeaves]   = tv.layout[leaf + 1];
                }
                ++numLeaves;
                __syncwarp();
                continue;
            }
            bool ov = false;
            if (lane < 8)
            {
                int c = child0 + lane;
                ov    = true;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                {
                    double d = tv.centers[3 * c + k] - gc[k];
                    if (box.periodic[k]) { d -= box.len[k] * rint(d * box.ilen[k]); }
                    ov = ov && fabs(d) <= gs[k] + tv.sizes[3 * c + k] * (1.0 + 1e-12) + tv.ext;
                }
            }
            unsigned m = __ballot_sync(0xffffffffu, ov) & 0xffu;
            int pushes = __popc(m);
            if (sp + pushes > kStackCap)
            {
                overflow = true;
                break;
            }
            __syncwarp();
            if (ov)
            {
                // children are pushed in reverse so that the lowest key is popped first
                int pos         = __popc(m >> (lane + 1));
                stack[sp + pos] = child0 + lane;
            }
            sp += pushes;
            __syncwarp();
        }
        if (overflow) { break; }
        if (numLeaves > 0) { flush(); }
        // the last, partly filled chunk of the list (entries past the count, or past the capacity, are never read)
        if (active)
        {
            unsigned kept = min(count, listCap);
            if (kept % kNbChunk != 0) { storeChunk(kept / kNbChunk); }
        }

        // smoothing-length iteration (skin rows: one pass at the given h)
        if (kSkin) { active = false; }
        if (active)
        {
            unsigned ncSph = count + 1;
            bool failing   = ngmin > ncSph || (ncSph - 1) > prm.ngmax;
            if (failing && updates < prm.maxIterations)
            {
                hi = updateH(prm.ng0, ncSph, hi);
                ++updates;
            }
            else { active = false; }
        }
    }

    if (overflow)
    {
        if (lane == 0) { atomicOr(status, 1u); }
        return;
    }
    if (valid)
    {
        if constexpr (kSkin)
        {
            ex.sl.count[i]  = count;
            ex.sl.radius[i] = __dmul_rn(2.0 * hi, ex.onePlusSkin);
        }
        else
        {
            ncOut[i] = count + 1;
            h[i]     = hi;
        }
    }
}

//! bounding box of each run of kBlockSize consecutive particles, relative to the box corner, rounded outwards
__global__ void blockBoxesKernel(const double* __restrict__ x, const double* __restrict__ y,
                                 const double* __restrict__ z, size_t n, DevBox box, float4* lo, float4* hi)
{
    size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    size_t b = c * kBlockSize;
    if (b >= n) { return; }
    size_t e  = min(b + kBlockSize, n);
    double l[3] = {INFINITY, INFINITY, INFINITY}, u[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t j = b; j < e; ++j)
    {
        double p[3] = {x[j] - box.lo[0], y[j] - box.lo[1], z[j] - box.lo[2]};
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            l[k] = fmin(l[k], p[k]);
            u[k] = fmax(u[k], p[k]);
        }
    }
    lo[c] = make_float4(__double2float_rd(l[0]), __double2float_rd(l[1]), __double2float_rd(l[2]), 0.f);
    hi[c] = make_float4(__double2float_ru(u[0]), __double2float_ru(u[1]), __double2float_ru(u[2]), 0.f);
}

} // namespace

int computeBlockBoxes(const double* x, const double* y, const double* z, size_t n, const DevBox& box, float4* lo,
                      float4* hi, cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    size_t blocks = (n + kBlockSize - 1) / kBlockSize;
    blockBoxesKernel<<<ceilDiv(blocks, 256), 256, 0, stream>>>(x, y, z, n, box, lo, hi);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int findNeighbors(const double* x, const double* y, const double* z, const double4* pos, double* h, size_t n,
                  const TreeView& tree, const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc,
                  unsigned* status, cudaStream_t stream, const TreeView* views, const uint8_t* inst,
                  const unsigned* gate, unsigned gateMask)
{
    if (n == 0) { return kOk; }
    if ((views == nullptr) != (inst == nullptr)) { return kErrArg; }
    size_t numGroups = (n + kWarp - 1) / kWarp;
    unsigned blocks  = unsigned((numGroups + kNbWarps - 1) / kNbWarps);
    SearchExtras ex{};
    ex.gate     = gate;
    ex.gateMask = gateMask;
    if (views)
    {
        findNeighborsKernel<true, kSearchAll><<<blocks, kNbThreads, 0, stream>>>(x, y, z, pos, h, n, tree, box, prm,
                                                                                 nidx, nc, status, views, inst, ex);
    }
    else
    {
        findNeighborsKernel<false, kSearchAll><<<blocks, kNbThreads, 0, stream>>>(x, y, z, pos, h, n, tree, box, prm,
                                                                                  nidx, nc, status, nullptr, nullptr, ex);
    }
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int findNeighborsListed(const double* x, const double* y, const double* z, const double4* pos, double* h, size_t n,
                        const TreeView& tree, const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc,
                        unsigned* status, const unsigned* groups, const unsigned* numListed, cudaStream_t stream,
                        const TreeView* views, const uint8_t* inst)
{
    if (n == 0) { return kOk; }
    if (!groups || !numListed || (views == nullptr) != (inst == nullptr)) { return kErrArg; }
    size_t numGroups = (n + kWarp - 1) / kWarp;
    unsigned blocks  = unsigned((numGroups + kNbWarps - 1) / kNbWarps);
    SearchExtras ex{};
    ex.groups    = groups;
    ex.numListed = numListed;
    if (views)
    {
        findNeighborsKernel<true, kSearchListed><<<blocks, kNbThreads, 0, stream>>>(x, y, z, pos, h, n, tree, box,
                                                                                    prm, nidx, nc, status, views, inst,
                                                                                    ex);
    }
    else
    {
        findNeighborsKernel<false, kSearchListed><<<blocks, kNbThreads, 0, stream>>>(
            x, y, z, pos, h, n, tree, box, prm, nidx, nc, status, nullptr, nullptr, ex);
    }
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int buildSkinLists(const double* x, const double* y, const double* z, const double4* pos, const double* h, size_t n,
                   const TreeView& tree, const DevBox& box, NeighborParams prm, double skin, SkinLists sl,
                   unsigned* status, cudaStream_t stream, const TreeView* views, const uint8_t* inst,
                   const unsigned* gate, unsigned gateMask)
{
    if (n == 0) { return kOk; }
    if (!(skin > 0.0) || sl.cap == 0 || sl.cap % kNbChunk != 0 || (views == nullptr) != (inst == nullptr))
    {
        return kErrArg;
    }
    size_t numGroups = (n + kWarp - 1) / kWarp;
    unsigned blocks  = unsigned((numGroups + kNbWarps - 1) / kNbWarps);
    SearchExtras ex{};
    ex.sl          = sl;
    ex.onePlusSkin = 1.0 + skin;
    ex.gate        = gate;
    ex.gateMask    = gateMask;
    // the kernel writes h only in the iterating kinds, never in this one
    if (views)
    {
        findNeighborsKernel<true, kSearchSkin><<<blocks, kNbThreads, 0, stream>>>(
            x, y, z, pos, const_cast<double*>(h), n, tree, box, prm, nullptr, nullptr, status, views, inst, ex);
    }
    else
    {
        findNeighborsKernel<false, kSearchSkin><<<blocks, kNbThreads, 0, stream>>>(
            x, y, z, pos, const_cast<double*>(h), n, tree, box, prm, nullptr, nullptr, status, nullptr, nullptr, ex);
    }
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

} // namespace sphb
