// Reuse of candidate lists across steps ("skin" lists).
//
// The reference searches the octree for every particle in every step (sph/include/sph/find_neighbors.hpp:10-41).
// Most particles move a small fraction of h per step, so the candidates within a slightly larger radius
// R_i = 2 h_i (1 + skin), found once, still contain every neighbour for many steps. Each step then only refilters
// those rows with the exact pair test, which reads ~1.2 entries per neighbour instead of testing the ~15 candidates
// per neighbour that the tree search stages.
//
// Exactness. Let j be outside the row of i, so |x_i - x_j| >= R_i at the build. Now
// |x_i - x_j| >= R_i - d_i - d_j, with d the displacement since the build. If 2 h_i + d_i + D <= R_i, where D bounds
// d_j for every j that can now lie within 2 h_i <= R_i of i, no such j is a neighbour. D is the largest displacement
// over the cells of a uniform grid that overlap the group's boxes [x_i - R_i, x_i + R_i]; the grid is binned by
// current positions, so it sees every particle that can be near. A relative margin of 1e-9 covers the rounding of
// the FP64 displacement and distance arithmetic. Indices must not have changed either: a row stores build indices,
// so a group is served only when none of its particles and none of its rows' entries moved to another index since
// the build. The sort permutations are composed into a current-to-build index map; a particle at another index than
// at the build puts an infinite displacement into the grid cell of its build position, which lies within
// R_i + d_i of x_i for every row i that lists it, so every group whose rows can hold it is deferred. Every deferred
// group goes to a worklist for the tree search.
// Entries are tested with the reference's exact FP64 expression (FP64 chain) or in FP32 from the fixed-point
// coordinates with an uncertainty band around the radius inside which the exact FP64 test decides (mixed chain), so
// the lists, counts and smoothing lengths are those of the tree search bit for bit.
#include "neighbors.cuh"
#include "primitives.cuh"

#include <algorithm>

namespace sphb
{

namespace
{

constexpr int kFilterWarps   = 8;
constexpr int kFilterThreads = kFilterWarps * kWarp;

//! 1 + the relative margin of the completeness test
constexpr double kSkinMargin = 1.0 + 1e-9;

__device__ inline double warpMinD(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

__device__ inline double warpMaxD(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

__device__ inline unsigned warpMaxU(unsigned v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        v = max(v, __shfl_xor_sync(0xffffffffu, v, off));
    }
    return v;
}

__device__ inline bool bitSet(const uint32_t* bits, size_t i) { return (__ldg(bits + i / kWarp) >> (i % kWarp)) & 1u; }

//! 32-byte read-only load of a packed position
__device__ inline double4 loadPos(const double4* p)
{
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 lo = __ldg(q), hi = __ldg(q + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

//! displacement of a particle since the build (minimum image on periodic axes), FP64
__device__ inline double displacement(double x, double y, double z, double bx, double by, double bz,
                                      const DevBox& box)
{
    double dx = minImage(x - bx, box.len[0], box.ilen[0], box.periodic[0]);
    double dy = minImage(y - by, box.len[1], box.ilen[1], box.periodic[1]);
    double dz = minImage(z - bz, box.len[2], box.ilen[2], box.periodic[2]);
    return sqrt(dx * dx + dy * dy + dz * dz);
}

/*! grid cell of a coordinate on one axis: wrapped on a periodic axis, clamped on an open one, as checkGroup maps
 *  the search ranges (positions outside the box occur between domain syncs under block time steps) */
__device__ inline int cellOf(double v, double lo, double ilen, int periodic)
{
    double f = floor((v - lo) * ilen * kSkinGrid);
    if (periodic)
    {
        int c = int(f - double(kSkinGrid) * floor(f * (1.0 / kSkinGrid)));
        return min(max(c, 0), kSkinGrid - 1);
    }
    return int(fmin(fmax(f, 0.0), double(kSkinGrid - 1)));
}

__device__ inline int gridCell(double x, double y, double z, const DevBox& box)
{
    return (cellOf(x, box.lo[0], box.ilen[0], box.periodic[0]) * kSkinGrid +
            cellOf(y, box.lo[1], box.ilen[1], box.periodic[1])) *
               kSkinGrid +
           cellOf(z, box.lo[2], box.ilen[2], box.periodic[2]);
}

__global__ void skinDisplacementKernel(const double4* __restrict__ pos, const double* __restrict__ xb,
                                       const double* __restrict__ yb, const double* __restrict__ zb,
                                       const uint32_t* __restrict__ buildOf, size_t n, DevBox box,
                                       unsigned* __restrict__ grid, const uint8_t* __restrict__ inst,
                                       const unsigned* gate)
{
    if (gate && __ldg(gate) != kSkinModeFilter) { return; }
    size_t i   = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool valid = i < n && !(inst && inst[i] == kGhost);
    unsigned bits = 0u;
    int cell      = -1;
    if (valid)
    {
        double4 p = loadPos(pos + i);
        size_t b  = buildOf ? buildOf[i] : i;
        double d  = displacement(p.x, p.y, p.z, xb[b], yb[b], zb[b], box);
        // rounded up, so that the grid bounds the FP64 value
        bits = __float_as_uint(__double2float_ru(d));
        const int gridBase = inst ? int(inst[i]) * kSkinCells : 0;
        cell = gridBase + gridCell(p.x, p.y, p.z, box);
        // The displacement also goes to the cell of the build position, which every group whose rows list this
        // particle checks: the refilter decides most entries from their build distance and these bounds. A particle
        // at another index than at the build makes those rows stale: infinite there.
        int cb = gridBase + gridCell(xb[b], yb[b], zb[b], box);
        unsigned atBuild = b != i ? __float_as_uint(INFINITY) : bits;
        if (cb != cell && atBuild != 0u) { atomicMax(grid + cb, atBuild); }
        else if (cb == cell) { bits = max(bits, atBuild); }
    }
    // consecutive particles are close in space: a warp whose particles share one cell issues a single atomic
    int cell0 = __shfl_sync(0xffffffffu, cell, 0);
    if (__all_sync(0xffffffffu, cell == cell0 || !valid))
    {
        unsigned m = warpMaxU(bits);
        if ((threadIdx.x & (kWarp - 1)) == 0 && m != 0u && cell0 >= 0) { atomicMax(grid + cell0, m); }
    }
    else if (valid && bits != 0u) { atomicMax(grid + cell, bits); }
}

__global__ void skinRemapKernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ buildOld,
                                uint32_t* __restrict__ buildNew, uint32_t* __restrict__ moved, size_t n)
{
    size_t i   = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool valid = i < n;
    uint32_t b = 0;
    if (valid)
    {
        uint32_t o = order[i];
        b          = buildOld ? buildOld[o] : o;
        buildNew[i] = b;
    }
    unsigned m = __ballot_sync(0xffffffffu, valid && size_t(b) != i);
    if ((threadIdx.x & (kWarp - 1)) == 0 && i < n) { moved[i / kWarp] = m; }
}

//! groupD entry of a group deferred by the check
constexpr unsigned kDeferred = 0xffffffffu;

/*! Whether the group's rows can serve every particle of the group at its current h (and D, the largest displacement
 *  near the group, for the later checks of the smoothing-length iteration). One warp, one lane per particle. */
__device__ inline bool checkGroup(const SkinFilterArgs& a, int lane, bool valid, const double4& pi, double Ri, double di,
                                  unsigned rowCount, double hi, size_t i, float* Dout)
{
    bool ok = !valid || (rowCount <= a.sl.cap && !(a.moved && bitSet(a.moved, i)));
    // an ensemble: the grid of the group's instance (the group's first slot is never padding)
    const unsigned* grid = a.dispGrid + (a.inst ? size_t(a.inst[i - lane]) * kSkinCells : 0);

    // The largest displacement of any particle that can now be within R_i of a particle of the group. The region
    // also holds the build position of every particle in the group's rows (within R_i of the build position of i,
    // which is d_i away), so a particle of the rows that changed index marks it infinite.
    const double reach = valid ? (Ri + di) * kSkinMargin : 0.0;
    double lo[3], hb[3];
    lo[0] = warpMinD(valid ? pi.x - reach : INFINITY);
    lo[1] = warpMinD(valid ? pi.y - reach : INFINITY);
    lo[2] = warpMinD(valid ? pi.z - reach : INFINITY);
    hb[0] = warpMaxD(valid ? pi.x + reach : -INFINITY);
    hb[1] = warpMaxD(valid ? pi.y + reach : -INFINITY);
    hb[2] = warpMaxD(valid ? pi.z + reach : -INFINITY);
    int c0[3], span[3];
    int numCells = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double fl = floor((lo[k] - a.box.lo[k]) * a.box.ilen[k] * kSkinGrid);
        double fh = floor((hb[k] - a.box.lo[k]) * a.box.ilen[k] * kSkinGrid);
        int cl = 0, ch = kSkinGrid - 1;
        if (a.box.periodic[k])
        {
            // cells wrap below; a range of a whole period or more (or not a number) covers every cell
            if (fh - fl + 1.0 < double(kSkinGrid))
            {
                cl = int(fl);
                ch = int(fh);
            }
        }
        else if (fl <= fh)
        {
            cl = int(fmin(fmax(fl, 0.0), double(kSkinGrid - 1)));
            ch = int(fmin(fmax(fh, 0.0), double(kSkinGrid - 1)));
        }
        c0[k]   = cl;
        span[k] = ch - cl + 1;
        numCells *= span[k];
    }
    unsigned dmax = 0u;
    for (int t = lane; t < numCells; t += kWarp)
    {
        int q[3] = {t / (span[1] * span[2]), (t / span[2]) % span[1], t % span[2]};
        int c[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            c[k] = c0[k] + q[k];
            if (a.box.periodic[k]) { c[k] = ((c[k] % kSkinGrid) + kSkinGrid) % kSkinGrid; }
        }
        dmax = max(dmax, __ldg(grid + (c[0] * kSkinGrid + c[1]) * kSkinGrid + c[2]));
    }
    const float D = __uint_as_float(warpMaxU(dmax));
    *Dout         = D;
    ok            = ok && (!valid || (2.0 * hi + di + double(D)) * kSkinMargin <= Ri);
    return __all_sync(0xffffffffu, ok);
}

/*! The check of every group before the refilter: deferred groups go to the worklist at once, so that their tree
 *  search can run beside the refilter of the others. groupD receives D, or kDeferred. */
__global__ void __launch_bounds__(kFilterThreads) skinCheckKernel(SkinFilterArgs a)
{
    const int warp         = threadIdx.x / kWarp;
    const int lane         = threadIdx.x & (kWarp - 1);
    const size_t numGroups = (a.n + kWarp - 1) / kWarp;
    const size_t group     = size_t(blockIdx.x) * kFilterWarps + warp;
    if (group >= numGroups || (a.gate && __ldg(a.gate) != kSkinModeFilter)) { return; }
    const size_t i    = group * kWarp + lane;
    const bool valid  = i < a.n && !(a.inst && a.inst[i] == kGhost);
    double4 pi        = valid ? loadPos(a.pos + i) : make_double4(0, 0, 0, 0);
    double hi         = valid ? a.h[i] : 0.0;
    double Ri         = valid ? a.sl.radius[i] : 0.0;
    unsigned rowCount = valid ? a.sl.count[i] : 0u;
    double di         = valid ? displacement(pi.x, pi.y, pi.z, a.xb[i], a.yb[i], a.zb[i], a.box) : 0.0;
    float D;
    bool ok = checkGroup(a, lane, valid, pi, Ri, di, rowCount, hi, i, &D);
    if (lane == 0)
    {
        a.groupD[group] = ok ? __float_as_uint(D) : kDeferred;
        if (!ok) { a.worklist[atomicAdd(a.numWorklist, 1u)] = unsigned(group); }
    }
}

/*! One warp per group of 32 consecutive particles, one lane per particle: the neighbour lists come out in the same
 *  chunked layout, written as whole sectors, as from the tree search. Groups the check deferred are skipped; a group
 *  whose smoothing-length iteration leaves its rows goes to the second worklist. */
template<bool kFixed>
__global__ void __launch_bounds__(kFilterThreads) skinFilterKernel(SkinFilterArgs a)
{
    // per lane: a ring of two list chunks, the one being filled and the next (lane minor: the lanes' appends fall
    // into distinct banks); one row chunk adds at most eight neighbours, so it completes at most one list chunk
    __shared__ uint32_t nbuf[kFilterWarps][2 * kNbChunk][kWarp];
    const int warp         = threadIdx.x / kWarp;
    const int lane         = threadIdx.x & (kWarp - 1);
    const size_t numGroups = (a.n + kWarp - 1) / kWarp;
    const size_t group     = size_t(blockIdx.x) * kFilterWarps + warp;
    if (group >= numGroups || (a.gate && __ldg(a.gate) != kSkinModeFilter)) { return; }
    const unsigned gD = __ldg(a.groupD + group);
    if (gD == kDeferred) { return; }
    const double D   = double(__uint_as_float(gD));
    const size_t i   = group * kWarp + lane;
    const bool valid = i < a.n && !(a.inst && a.inst[i] == kGhost);

    double4 pi = valid ? loadPos(a.pos + i) : make_double4(0, 0, 0, 0);
    double hi  = valid ? a.h[i] : 0.0;
    double Ri  = valid ? a.sl.radius[i] : 0.0;
    unsigned rowCount = valid ? a.sl.count[i] : 0u;
    double di  = valid ? displacement(pi.x, pi.y, pi.z, a.xb[i], a.yb[i], a.zb[i], a.box) : 0.0;

    auto covered = [&](double h) { return (2.0 * h + di + D) * kSkinMargin <= Ri; };
    auto defer   = [&]() {
        if (lane == 0) { a.worklist2[atomicAdd(a.numWorklist2, 1u)] = unsigned(group); }
    };

    const unsigned ngmin  = a.prm.ng0 / 4;
    const unsigned ngPad  = paddedNgmax(a.prm.ngmax);
    const unsigned rowLen = min(rowCount, a.sl.cap);
    int4 qi               = make_int4(0, 0, 0, 0);
    if constexpr (kFixed)
    {
        if (valid) { qi = __ldg(a.posq + i); }
    }
    uint32_t* ring = &nbuf[warp][0][lane];
    auto storeChunk = [&](unsigned c) {
        uint32_t* dst       = a.nidx + nidxAt(group, ngPad, c * kNbChunk, lane);
        const uint32_t* src = ring + (c % 2) * kNbChunk * kWarp;
        asm volatile("st.global.cs.v8.u32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(dst), "r"(src[0]),
                     "r"(src[kWarp]), "r"(src[2 * kWarp]), "r"(src[3 * kWarp]), "r"(src[4 * kWarp]),
                     "r"(src[5 * kWarp]), "r"(src[6 * kWarp]), "r"(src[7 * kWarp])
                     : "memory");
    };

    bool active    = valid;
    bool bad       = false;
    int updates    = 0;
    unsigned count = 0;
    while (__ballot_sync(0xffffffffu, active) != 0u)
    {
        if (active)
        {
            const double radiusSq = searchRadiusSq(hi);
            // FP32 decision outside a band around (2h)^2 that bounds the error of the fixed-point separation (one
            // unit per coordinate difference) and of the FP32 arithmetic; the exact test inside it
            const float twoH = float(2.0 * hi);
            const float r2f  = twoH * twoH;
            const float u    = a.qunit / twoH;
            const float band = 2.0e-6f + 8.0f * u + 8.0f * u * u;
            const float r2lo = r2f * (1.f - band);
            const float r2hi = r2f * (1.f + band);
            // Most entries are decided from their quantised build distance q (units of Ri / kSkinDistUnits, the true
            // build distance within (q +- 0.5) units): now |x_i - x_j| lies within d_i + D of it, so entries with
            // q <= qIn are surely inside 2 h_i and entries with q >= qOut surely outside, by a relative margin of
            // 1e-9 that covers the FP64 rounding of the exact test. Only the rest are gathered and tested.
            const double unit = Ri / kSkinDistUnits;
            const double tIn  = (2.0 * hi * (1.0 - 1e-9) - di - D) / unit - 0.501;
            const double tOut = (2.0 * hi * (1.0 + 1e-9) + di + D) / unit + 0.501;
            const int qIn     = tIn > 0.0 ? int(ceil(tIn)) - 1 : -1;               // largest q < tIn
            const int qOut    = tOut < kSkinDistUnits ? int(floor(tOut)) + 1 : 65536; // smallest q > tOut
            count           = 0;
            unsigned stored = 0; // list chunks written
            for (unsigned c = 0; c < rowLen; c += kNbChunk)
            {
                const uint32_t* src = a.sl.rows + nidxAt(group, a.sl.cap, c, lane);
                uint4 e0 = __ldg(reinterpret_cast<const uint4*>(src));
                uint4 e1 = __ldg(reinterpret_cast<const uint4*>(src) + 1);
                uint4 dq = __ldg(reinterpret_cast<const uint4*>(a.sl.dist + nidxAt(group, a.sl.cap, c, lane)));
                uint32_t e[kNbChunk] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
                int q[kNbChunk] = {int(dq.x & 0xffffu), int(dq.x >> 16), int(dq.y & 0xffffu), int(dq.y >> 16),
                                   int(dq.z & 0xffffu), int(dq.z >> 16), int(dq.w & 0xffffu), int(dq.w >> 16)};
                // entries past the row's end (garbage in its last chunk) are masked out
                unsigned in = 0u, test = 0u;
#pragma unroll
                for (unsigned k = 0; k < kNbChunk; ++k)
                {
                    const bool real = c + k < rowLen;
                    in |= unsigned(real && q[k] <= qIn) << k;
                    test |= unsigned(real && q[k] > qIn && q[k] < qOut) << k;
                }
                if (test)
                {
#pragma unroll
                    for (unsigned k = 0; k < kNbChunk; ++k)
                    {
                        if (!((test >> k) & 1u)) { continue; }
                        bool inside;
                        if constexpr (kFixed)
                        {
                            // FP32 from the fixed-point coordinates, the exact FP64 test inside the band
                            int4 qj  = __ldg(a.posq + e[k]);
                            float dx = float(int(unsigned(qi.x) - unsigned(qj.x))) * a.qscale[0];
                            float dy = float(int(unsigned(qi.y) - unsigned(qj.y))) * a.qscale[1];
                            float dz = float(int(unsigned(qi.z) - unsigned(qj.z))) * a.qscale[2];
                            float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                            inside   = d2 < r2lo;
                            if (!inside && d2 < r2hi)
                            {
                                double4 pj = loadPos(a.pos + e[k]);
                                inside     = exactDistSq(pj.x, pj.y, pj.z, pi.x, pi.y, pi.z, a.box) < radiusSq;
                            }
                        }
                        else
                        {
                            double4 pj = loadPos(a.pos + e[k]);
                            inside     = exactDistSq(pj.x, pj.y, pj.z, pi.x, pi.y, pi.z, a.box) < radiusSq;
                        }
                        in |= unsigned(inside) << k;
                    }
                }
                // append the neighbours in row (= index) order
#pragma unroll
                for (unsigned k = 0; k < kNbChunk; ++k)
                {
                    if ((in >> k) & 1u)
                    {
                        if (count < a.prm.ngmax) { ring[(count % (2 * kNbChunk)) * kWarp] = e[k]; }
                        ++count;
                    }
                }
                if (min(count, a.prm.ngmax) / kNbChunk > stored) { storeChunk(stored++); }
            }
            // the last, partly filled chunk (entries past the count, or past ngmax, are never read)
            const unsigned kept = min(count, a.prm.ngmax);
            if (kept % kNbChunk != 0) { storeChunk(kept / kNbChunk); }

            // smoothing-length iteration, as in the tree search; a new h must stay covered by the row
            unsigned ncSph = count + 1;
            bool failing   = ngmin > ncSph || (ncSph - 1) > a.prm.ngmax;
            if (failing && updates < a.prm.maxIterations)
            {
                hi = updateH(a.prm.ng0, ncSph, hi);
                ++updates;
                if (!covered(hi)) { bad = true; }
            }
            else { active = false; }
        }
        if (__any_sync(0xffffffffu, bad))
        {
            // lists already written for this group are rewritten by the tree search; h and nc were not touched
            defer();
            return;
        }
    }
    if (valid)
    {
        a.nc[i] = count + 1;
        a.h[i]  = hi;
    }
}

/*! The row policy of a simulation stepped without host reads (an ensemble in a captured graph), on one thread: the
 *  same rules as the host policy of a single simulation (rebuild when more than a tenth of the groups were deferred
 *  in the previous step; rows rebuilt within three steps of the last build give way to 32 steps of tree searches). */
__global__ void skinDecideKernel(unsigned* ctl)
{
    unsigned deferred = ctl[kCtlDeferredA] + ctl[kCtlDeferredB];
    ctl[kCtlDeferredTotal] += deferred;
    ctl[kCtlDeferredA] = 0;
    ctl[kCtlDeferredB] = 0;
    unsigned mode;
    if (ctl[kCtlHoldoff] > 0)
    {
        --ctl[kCtlHoldoff];
        ctl[kCtlValid] = 0;
        mode           = kSkinModeTree;
    }
    else if (!ctl[kCtlValid]) { mode = kSkinModeBuild; }
    else if (size_t(deferred) * 10 > size_t(ctl[kCtlGroups]))
    {
        if (ctl[kCtlAge] <= 3)
        {
            ctl[kCtlHoldoff] = 32;
            ctl[kCtlValid]   = 0;
            mode             = kSkinModeTree;
        }
        else { mode = kSkinModeBuild; }
    }
    else { mode = kSkinModeFilter; }
    if (mode == kSkinModeFilter)
    {
        ++ctl[kCtlAge];
        ++ctl[kCtlFilterSteps];
    }
    else { ++ctl[kCtlTreeSearches]; }
    if (mode == kSkinModeBuild) { ++ctl[kCtlBuilds]; }
    ctl[kCtlMode] = mode;
}

//! after a build: build positions = current positions, build index = current index, rows valid
__global__ void skinCommitKernel(const double* __restrict__ x, const double* __restrict__ y,
                                 const double* __restrict__ z, size_t n, double* xb, double* yb, double* zb,
                                 uint32_t* buildOf, uint32_t* moved, unsigned* ctl)
{
    if (__ldg(ctl + kCtlMode) != kSkinModeBuild) { return; }
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i < n)
    {
        xb[i]      = x[i];
        yb[i]      = y[i];
        zb[i]      = z[i];
        buildOf[i] = uint32_t(i);
        if (i % kWarp == 0) { moved[i / kWarp] = 0u; }
    }
    if (i == 0)
    {
        ctl[kCtlValid] = 1;
        ctl[kCtlAge]   = 0;
    }
}

__global__ void idsDifferKernel(const uint64_t* __restrict__ a, const uint64_t* __restrict__ b, size_t n,
                                unsigned* flag)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool d   = i < n && a[i] != b[i];
    if (__any_sync(0xffffffffu, d) && (threadIdx.x & (kWarp - 1)) == 0) { atomicOr(flag, 1u); }
}

} // namespace

int idsDiffer(const uint64_t* a, const uint64_t* b, size_t n, unsigned* flag, cudaStream_t stream)
{
    SPHB_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(unsigned), stream));
    if (n == 0) { return kOk; }
    idsDifferKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(a, b, n, flag);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int skinDecide(unsigned* ctl, cudaStream_t stream)
{
    skinDecideKernel<<<1, 1, 0, stream>>>(ctl);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int skinCommit(const double* x, const double* y, const double* z, size_t n, double* xb, double* yb, double* zb,
               uint32_t* buildOf, uint32_t* moved, unsigned* ctl, cudaStream_t stream)
{
    skinCommitKernel<<<ceilDiv(std::max<size_t>(n, 1), 256), 256, 0, stream>>>(x, y, z, n, xb, yb, zb, buildOf, moved,
                                                                               ctl);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int skinDisplacement(const double4* pos, const double* xb, const double* yb, const double* zb,
                     const uint32_t* buildOf, size_t n, const DevBox& box, unsigned* dispGrid, cudaStream_t stream,
                     const uint8_t* inst, const unsigned* gate)
{
    if (n == 0) { return kOk; }
    skinDisplacementKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(pos, xb, yb, zb, buildOf, n, box, dispGrid, inst,
                                                                gate);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int skinRemap(const uint32_t* order, const uint32_t* buildOld, uint32_t* buildNew, uint32_t* moved, size_t n,
              cudaStream_t stream)
{
    if (n == 0) { return kOk; }
    skinRemapKernel<<<ceilDiv(n, 256), 256, 0, stream>>>(order, buildOld, buildNew, moved, n);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int checkSkinGroups(const SkinFilterArgs& a, cudaStream_t stream)
{
    if (a.n == 0) { return kOk; }
    if (a.sl.cap == 0 || a.sl.cap % kNbChunk != 0) { return kErrArg; }
    size_t numGroups = (a.n + kWarp - 1) / kWarp;
    unsigned blocks  = unsigned((numGroups + kFilterWarps - 1) / kFilterWarps);
    skinCheckKernel<<<blocks, kFilterThreads, 0, stream>>>(a);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int filterSkinLists(const SkinFilterArgs& a, cudaStream_t stream)
{
    if (a.n == 0) { return kOk; }
    if (a.sl.cap == 0 || a.sl.cap % kNbChunk != 0) { return kErrArg; }
    size_t numGroups = (a.n + kWarp - 1) / kWarp;
    unsigned blocks  = unsigned((numGroups + kFilterWarps - 1) / kFilterWarps);
    if (a.posq) { skinFilterKernel<true><<<blocks, kFilterThreads, 0, stream>>>(a); }
    else { skinFilterKernel<false><<<blocks, kFilterThreads, 0, stream>>>(a); }
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

} // namespace sphb
