// Neighbour search on sm_100a: one warp per target group of 32 consecutive (SFC-ordered) particles.
//
// Per group: (1) the search box = union over the group's still-active particles of [x - 2h, x + 2h];
// (2) a depth-first traversal of the focus octree in child (= SFC) order, warp-cooperative with 8 lanes testing the
// 8 children of a node against the box (periodic axes use the minimum image), collecting overlapping leaves in
// ascending order in shared memory; (3) the particles of those leaves are streamed 32 at a time through shared
// memory and every lane tests them against its own particle with the exact FP64 distance of the reference
// (cstone/findneighbors.hpp:33-51,77-147: squared minimum-image distance < (2h)^2, j != i).
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
    int leaf[kNbWarps][kLeafCap];
    int first[kNbWarps][kLeafCap];
    int prefix[kNbWarps][kLeafCap + 1];
    float4 cand[kNbWarps][kWarp]; // candidate position relative to the group centre (FP32) and its index
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

//! d folded to the nearest periodic image: d - L * rint(d / L), rounded like the reference's uncontracted CPU code
__device__ inline double minImage(double d, double len, double ilen, int periodic)
{
    if (!periodic) { return d; }
    return __dsub_rn(d, __dmul_rn(len, rint(__dmul_rn(d, ilen))));
}

//! smoothing-length update h * 0.5 * (1 + 1023 ng0 / nc)^(1/10) (sph/include/sph/kernels.hpp:27-33)
__device__ inline double updateH(unsigned ng0, unsigned nc, double h)
{
    double ratio = __ddiv_rn(__dmul_rn(1023.0, double(ng0)), double(nc));
    return __dmul_rn(__dmul_rn(h, 0.5), pow(__dadd_rn(1.0, ratio), 0.1));
}

__global__ void __launch_bounds__(kNbThreads) findNeighborsKernel(const double* __restrict__ x,
                                                                  const double* __restrict__ y,
                                                                  const double* __restrict__ z, double* h, size_t n,
                                                                  TreeView tree, DevBox box, NeighborParams prm,
                                                                  uint32_t* __restrict__ nidx,
                                                                  unsigned* __restrict__ ncOut, unsigned* status)
{
    __shared__ NbShared sh;
    const int warp        = threadIdx.x / kWarp;
    const int lane        = threadIdx.x & (kWarp - 1);
    const size_t numGroups = (n + kWarp - 1) / kWarp;
    const size_t group    = size_t(blockIdx.x) * kNbWarps + warp;
    if (group >= numGroups) { return; }

    const size_t i  = group * kWarp + lane;
    const bool valid = i < n;
    const double xi = valid ? x[i] : 0.0;
    const double yi = valid ? y[i] : 0.0;
    const double zi = valid ? z[i] : 0.0;
    double hi       = valid ? h[i] : 0.0;

    const unsigned ngmin = prm.ng0 / 4;
    bool active          = valid;
    int updates          = 0;
    unsigned count       = 0;
    bool overflow        = false;

    int* stack   = sh.stack[warp];
    int* leaves  = sh.leaf[warp];
    int* firsts  = sh.first[warp];
    int* prefix  = sh.prefix[warp];

    while (__ballot_sync(0xffffffffu, active) != 0u && !overflow)
    {
        const double radiusSq = __dmul_rn(__dmul_rn(4.0, hi), hi);
        const double r        = 2.0 * hi;
        double blo[3], bhi[3];
        blo[0] = warpMin(active ? xi - r : INFINITY);
        blo[1] = warpMin(active ? yi - r : INFINITY);
        blo[2] = warpMin(active ? zi - r : INFINITY);
        bhi[0] = warpMax(active ? xi + r : -INFINITY);
        bhi[1] = warpMax(active ? yi + r : -INFINITY);
        bhi[2] = warpMax(active ? zi + r : -INFINITY);
        double gc[3], gs[3];
        for (int k = 0; k < 3; ++k)
        {
            gc[k] = 0.5 * (blo[k] + bhi[k]);
            gs[k] = 0.5 * (bhi[k] - blo[k]) * (1.0 + 1e-12) + 1e-14 * box.len[k];
        }
        // this particle relative to the group centre in FP32, and the FP32 acceptance band
        const float rix = float(minImage(xi - gc[0], box.len[0], box.ilen[0], box.periodic[0]));
        const float riy = float(minImage(yi - gc[1], box.len[1], box.ilen[1], box.periodic[1]));
        const float riz = float(minImage(zi - gc[2], box.len[2], box.ilen[2], box.periodic[2]));
        const float twoH = float(r);
        const float r2f  = twoH * twoH;
        float reach      = active ? sqrtf(rix * rix + riy * riy + riz * riz) * 1.001f + twoH : 0.f;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            reach = fmaxf(reach, __shfl_xor_sync(0xffffffffu, reach, off));
        }
        const float band = active ? bandOf(reach, twoH) : 0.f;
        const float r2lo = r2f * (1.f - band);
        const float r2hi = r2f * (1.f + band);

        if (active) { count = 0; }
        int numLeaves = 0;

        // stream the buffered candidate leaves through the per-lane distance test
        auto flush = [&]() {
            // sizes and exclusive prefix of the buffered leaves (8 per lane at most)
            int local[kLeafCap / kWarp];
            int sum = 0;
#pragma unroll
            for (int q = 0; q < kLeafCap / kWarp; ++q)
            {
                int t    = lane * (kLeafCap / kWarp) + q;
                int size = 0;
                if (t < numLeaves)
                {
                    int leaf  = leaves[t];
                    int b     = tree.layout[leaf];
                    size      = tree.layout[leaf + 1] - b;
                    firsts[t] = b;
                }
                local[q] = size;
                sum += size;
            }
            int incl = sum;
#pragma unroll
            for (int off = 1; off < kWarp; off <<= 1)
            {
                int v = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) { incl += v; }
            }
            int run = incl - sum;
#pragma unroll
            for (int q = 0; q < kLeafCap / kWarp; ++q)
            {
                int t = lane * (kLeafCap / kWarp) + q;
                if (t < numLeaves) { prefix[t] = run; }
                run += local[q];
            }
            int total = __shfl_sync(0xffffffffu, incl, kWarp - 1);
            if (lane == 0) { prefix[numLeaves] = total; }
            __syncwarp();

            for (int base = 0; base < total; base += kWarp)
            {
                int t = base + lane;
                if (t < total)
                {
                    int lo = 0, hiIdx = numLeaves; // find the leaf r with prefix[r] <= t < prefix[r+1]
                    while (hiIdx - lo > 1)
                    {
                        int mid = (lo + hiIdx) >> 1;
                        if (prefix[mid] <= t) { lo = mid; }
                        else { hiIdx = mid; }
                    }
                    int j = firsts[lo] + (t - prefix[lo]);
                    float4 c;
                    if (j < 0 || size_t(j) >= n)
                    {
                        // a layout that points outside the particle arrays: report, stage a far-away point
                        atomicOr(status, 2u);
                        c = make_float4(INFINITY, INFINITY, INFINITY, __int_as_float(0));
                    }
                    else
                    {
                        c = make_float4(float(minImage(x[j] - gc[0], box.len[0], box.ilen[0], box.periodic[0])),
                                        float(minImage(y[j] - gc[1], box.len[1], box.ilen[1], box.periodic[1])),
                                        float(minImage(z[j] - gc[2], box.len[2], box.ilen[2], box.periodic[2])),
                                        __int_as_float(j));
                    }
                    sh.cand[warp][lane] = c;
                }
                __syncwarp();
                int cnt = min(kWarp, total - base);
                if (active)
                {
                    for (int k = 0; k < cnt; ++k)
                    {
                        float4 c  = sh.cand[warp][k];
                        float dx  = c.x - rix;
                        float dy  = c.y - riy;
                        float dz  = c.z - riz;
                        float d2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        if (d2f >= r2hi) { continue; }
                        int j   = __float_as_int(c.w);
                        bool in = d2f < r2lo;
                        if (!in)
                        {
                            // too close to the search radius for FP32: the exact test of the reference
                            double ex = minImage(x[j] - xi, box.len[0], box.ilen[0], box.periodic[0]);
                            double ey = minImage(y[j] - yi, box.len[1], box.ilen[1], box.periodic[1]);
                            double ez = minImage(z[j] - zi, box.len[2], box.ilen[2], box.periodic[2]);
                            double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
                            in        = d2 < radiusSq;
                        }
                        if (in && size_t(j) != i)
                        {
                            if (count < prm.ngmax) { nidx[nidxSlot(group, prm.ngmax, count, lane)] = uint32_t(j); }
                            ++count;
                        }
                    }
                }
                __syncwarp();
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
            int child0 = tree.childOffsets[node];
            if (child0 == 0)
            {
                if (numLeaves == kLeafCap) { flush(); }
                if (lane == 0) { leaves[numLeaves] = tree.nodeToLeaf[node]; }
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
                    double d = tree.centers[3 * c + k] - gc[k];
                    if (box.periodic[k]) { d -= box.len[k] * rint(d * box.ilen[k]); }
                    ov = ov && fabs(d) <= gs[k] + tree.sizes[3 * c + k] * (1.0 + 1e-12);
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
                int pos                        = __popc(m >> (lane + 1));
                stack[sp + pos]                = child0 + lane;
            }
            sp += pushes;
            __syncwarp();
        }
        if (overflow) { break; }
        if (numLeaves > 0) { flush(); }

        // smoothing-length iteration
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
        ncOut[i] = count + 1;
        h[i]     = hi;
    }
}

} // namespace

int findNeighbors(const double* x, const double* y, const double* z, double* h, size_t n, const TreeView& tree,
                  const DevBox& box, NeighborParams prm, uint32_t* nidx, unsigned* nc, unsigned* status,
                  cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    size_t numGroups = (n + kWarp - 1) / kWarp;
    unsigned blocks  = unsigned((numGroups + kNbWarps - 1) / kNbWarps);
    findNeighborsKernel<<<blocks, kNbThreads, 0, stream>>>(x, y, z, h, n, tree, box, prm, nidx, nc, status);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

} // namespace sphb
