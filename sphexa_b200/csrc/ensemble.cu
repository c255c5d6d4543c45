// Batched ensemble of independent VE hydro simulations stepped together: every stage of the step is one launch over
// all instances, the step has no host synchronisation, and it is captured once into a CUDA graph and replayed.
//
// Layout: instance k owns the slots [off_k, off_k + n_k) of every particle array, off_k a multiple of 32; the slots
// up to off_{k+1} are padding ("ghosts": instance byte kGhost, key 2^63, mass 0), so a warp group of 32 slots never
// spans two instances and per-instance reductions take one atomic per warp. Instances share the box and the kernel
// (sinc index, ng0, ngmax, AV constants); they differ in their particles, gamma, mui and time step.
//
// The step (sync, neighbour search with the h iteration, the SPH-VE chain, per-instance time step, integration,
// h update, per-instance conserved sums) computes for every instance exactly what one simulation of that instance
// computes (sim.cu): the sort orders each instance's particles by key as the single sort does, the per-particle
// arithmetic is the same code, and the time step is the same expression evaluated on the device. The focus trees
// are rebuilt on the host only outside the captured step: neighbour lists do not depend on the tree (every j with
// |x_i - x_j| < 2 h_i, in index order), so a tree that lags the particles changes the search cost, never its result;
// the layout of each tree is recomputed from the sorted keys inside the step.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "hydro.cuh"
#include "integrate.cuh"
#include "neighbors.cuh"
#include "octree.cuh"
#include "primitives.cuh"
#include "sfc.cuh"
#include "sort.cuh"
#include "tables.hpp"

namespace sphb
{
namespace
{

constexpr int kFields    = 14; // conserved fields, order x y z h m temp vx vy vz x_m1 y_m1 z_m1 du_m1 alpha
constexpr int kNumCons   = 9;  // per-instance conserved sums
constexpr int kJLoops    = 5;  // tunable J-loop launches
constexpr int kAvLoop    = 3;  // their index of the AV switches
constexpr int kMaxInst   = 254;
const char* const kFieldNames[kFields] = {"x",  "y",  "z",    "h",    "m",    "temp",  "vx",
                                          "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha"};

enum Derived : int
{
    dXm, dKx, dGradh, dPrho, dC, dC11, dC12, dC13, dC22, dC23, dC33, dDivv, dCurlv, dAx, dAy, dAz, kNumDerived
};
const char* const kDerivedNames[kNumDerived] = {"xm",  "kx",  "gradh", "prho", "c",     "c11", "c12", "c13",
                                                "c22", "c23", "c33",   "divv", "curlv", "ax",  "ay",  "az"};

//! leaves of one instance's focus tree and where its global layout goes
struct LeafDesc
{
    const uint64_t* leaves;
    int* layout;
    int numLeaves;
    uint32_t off;
    uint32_t n;
};

double idealGasCvE(double mui, double gamma) { return 8.317e7 / mui / (gamma - 1.0); }

} // namespace
} // namespace sphb

using namespace sphb;

struct sphb_ensemble
{
    int num{0};
    std::vector<size_t> n;      // particles per instance
    std::vector<size_t> off;    // first slot per instance
    size_t slots{0};
    std::vector<sphb_params> ip;
    sphb_params p{};
    sphb_box hbox{};
    DevBox box{};
    bool mixed{false};
    cudaStream_t stream{nullptr};

    DeviceBuffer<double> f[kFields], fAlt[kFields];
    DeviceBuffer<uint64_t> id, idAlt, keys, keysAlt, keysTmp, segKey, segOfSlot;
    DeviceBuffer<uint32_t> order;
    DeviceBuffer<uint8_t> inst;
    DeviceBuffer<char> sortScratch;
    DeviceBuffer<double4> pos;
    DeviceBuffer<int4> posq;
    DeviceBuffer<float4> blockLo, blockHi;
    DeviceBuffer<uint32_t> nidx;
    DeviceBuffer<unsigned> nc;
    DeviceBuffer<char> derived[kNumDerived];
    DeviceBuffer<double> du;
    DeviceBuffer<char> hrec, grec, avrec;
    DeviceBuffer<char> dvrec, dv; // AV cleaning only
    DeviceBuffer<double> whD, whdD;
    DeviceBuffer<float> whF, whdF;
    double K{0};
    int polyOk{0};
    float wpoly[kPolyTerms]{};
    float dwpoly[kPolyTerms]{};

    // per instance
    DeviceBuffer<double> gamma, cv, dt, dtm1, ttot, cons;
    DeviceBuffer<unsigned long long> reduce;
    DeviceBuffer<unsigned> status; // [0] search overflow, [1] h flag, [2] sort look-back timeout
    DeviceBuffer<uint32_t> sortFlags; // [0] pairs out of order before the tile repair, [1] after it

    // trees
    std::vector<std::unique_ptr<GlobalTree>> gtrees;
    std::vector<std::unique_ptr<FocusTree>> ftrees;
    std::vector<std::unique_ptr<DeviceBuffer<int>>> layouts;
    TreeScratch ts;
    DeviceBuffer<TreeView> views;
    DeviceBuffer<LeafDesc> leafDescs;
    int maxLeaves{0};
    DeviceBuffer<double> alphaBackup, hBackup;
    uint64_t launchesPerStep{0};

    // skin rows (neighbors.cuh): kept across steps and refiltered; the mode of each step is chosen on the device
    bool skin{false};
    unsigned skinCap{0};
    DeviceBuffer<uint32_t> skinRows;
    DeviceBuffer<uint16_t> skinDist;
    DeviceBuffer<unsigned> skinCount;
    DeviceBuffer<double> skinRadius, skinXb, skinYb, skinZb;
    DeviceBuffer<uint32_t> skinBuild, skinBuildTmp, skinMoved;
    DeviceBuffer<unsigned> skinGrid, skinWork, skinGroupD, skinCtl;

    // stage times of the last step (same stages as a single simulation's, sim.cu), recorded inside the graph
    static constexpr int kStages = 9;
    cudaEvent_t ev[kStages + 1]{};

    int threads[kJLoops]{128, 128, 128, 128, 128};
    // two captured steps: they gather the particle state between the two buffer sets in opposite directions, so the
    // state alternates between f and fAlt with no copy; graphs[parity] is the one whose input is the current set
    cudaGraphExec_t graphs[2]{};
    int parity{0};
    bool uploaded{false};
    bool synced{false};
    uint64_t steps{0};

    template<class T>
    T* dptr(int d) const
    {
        return reinterpret_cast<T*>(derived[d].data());
    }
    size_t elemBytes() const { return mixed ? sizeof(float) : sizeof(double); }
};

namespace sphb
{
namespace
{

// ------------------------------------------------------------------------------------------------------------------
// batched helper kernels
// ------------------------------------------------------------------------------------------------------------------

//! layout[l] = off + lower_bound(sorted keys of the instance, leaves[l]) for every leaf of every instance
__global__ void forestLayoutKernel(const LeafDesc* __restrict__ descs, const uint64_t* __restrict__ keys)
{
    LeafDesc d = descs[blockIdx.y];
    int l      = blockIdx.x * blockDim.x + threadIdx.x;
    if (l > d.numLeaves) { return; }
    uint64_t key    = d.leaves[l];
    const uint64_t* k = keys + d.off;
    uint32_t lo = 0, hi = d.n;
    while (lo < hi)
    {
        uint32_t mid = (lo + hi) >> 1;
        if (k[mid] < key) { lo = mid + 1; }
        else { hi = mid; }
    }
    d.layout[l] = int(d.off + lo);
}

//! the time step of every instance (ts_global.hpp:100-128): min(Courant, Krho / |max divv|, 1.1 dt), then reset
//! the per-instance reductions for the next step
__global__ void timestepKernel(int num, unsigned long long* reduce, double* dt, double* dtm1, double* ttot,
                               double Krho)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= num) { return; }
    double maxDivv  = fromOrderedBits(reduce[2 * k]);
    double courant  = fromOrderedBits(reduce[2 * k + 1]);
    double rho      = Krho / fabs(maxDivv);
    double prev     = dt[k];
    double dtNew    = fmin(fmin(courant, rho), 1.1 * prev);
    dtm1[k]         = prev;
    dt[k]           = dtNew;
    ttot[k]        += dtNew;
    reduce[2 * k]     = orderedBits(-INFINITY);
    reduce[2 * k + 1] = orderedBits(INFINITY);
}

__global__ void initReduceKernel(int num, unsigned long long* reduce, double* cons)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= num) { return; }
    reduce[2 * k]     = orderedBits(-INFINITY);
    reduce[2 * k + 1] = orderedBits(INFINITY);
#pragma unroll
    for (int q = 0; q < kNumCons; ++q)
    {
        cons[kNumCons * k + q] = 0.0;
    }
}

//! warps of the per-instance sums below: a few per SM, each over a contiguous run of 32-slot chunks
constexpr int kConsWarps = 148 * 16;

/*! Per-instance sums of eKin, eInt, P, L, nc (conserved_quantities.hpp:117-175). Each warp walks a contiguous run
 *  of 32-slot chunks (a chunk never spans two instances), keeps per-lane sums and adds them to the instance's slots
 *  with one atomic per component when the instance changes or the run ends: about (warps + instances) x 9 atomics
 *  per step instead of one set per warp of particles. */
__global__ void consBatchKernel(size_t n, const uint8_t* __restrict__ inst, const double* x, const double* y,
                                const double* z, const double* vx, const double* vy, const double* vz,
                                const double* m, const double* temp, const unsigned* nc, const double* cv,
                                double* cons)
{
    const int lane          = threadIdx.x & 31;
    const size_t numChunks  = (n + 31) / 32;
    const size_t warpId     = (blockIdx.x * size_t(blockDim.x) + threadIdx.x) / 32;
    const size_t numWarps   = size_t(gridDim.x) * blockDim.x / 32;
    const size_t perWarp    = (numChunks + numWarps - 1) / numWarps;
    const size_t c0         = warpId * perWarp;
    const size_t c1         = min(numChunks, c0 + perWarp);
    double acc[kNumCons]    = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint8_t cur             = kGhost;
    auto flush = [&]() {
#pragma unroll
        for (int c = 0; c < kNumCons; ++c)
        {
            double v = acc[c];
            for (int o = 16; o > 0; o >>= 1)
            {
                v += __shfl_xor_sync(0xffffffffu, v, o);
            }
            if (lane == 0 && cur != kGhost) { atomicAdd(cons + kNumCons * cur + c, v); }
            acc[c] = 0.0;
        }
    };
    for (size_t c = c0; c < c1; ++c)
    {
        // the chunk's instance: its first slot (never padding when the chunk holds any particle)
        uint8_t cq = inst[c * 32];
        if (cq != cur)
        {
            flush();
            cur = cq;
        }
        size_t i  = c * 32 + lane;
        uint8_t q = i < n ? inst[i] : kGhost;
        if (q == kGhost) { continue; }
        double mi   = m[i];
        double X[3] = {x[i], y[i], z[i]};
        double V[3] = {vx[i], vy[i], vz[i]};
        acc[0] += mi * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
        acc[1] += cv[q] * temp[i] * mi;
        acc[2] += mi * V[0];
        acc[3] += mi * V[1];
        acc[4] += mi * V[2];
        acc[5] += mi * (X[1] * V[2] - X[2] * V[1]);
        acc[6] += mi * (X[2] * V[0] - X[0] * V[2]);
        acc[7] += mi * (X[0] * V[1] - X[1] * V[0]);
        acc[8] += double(nc[i]);
    }
    flush();
}

__global__ void orFlagsKernel(const unsigned* src, unsigned* dst, int count)
{
    int k = threadIdx.x;
    if (k < count && src[k]) { atomicOr(dst + k, src[k]); }
}

// ------------------------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------------------------

int allocate(sphb_ensemble& e)
{
    size_t n = e.slots;
    for (int k = 0; k < kFields; ++k)
    {
        SPHB_TRY(e.f[k].reserve(n));
        SPHB_TRY(e.fAlt[k].reserve(n));
    }
    SPHB_TRY(e.id.reserve(n));
    SPHB_TRY(e.idAlt.reserve(n));
    SPHB_TRY(e.keys.reserve(n));
    SPHB_TRY(e.keysAlt.reserve(n));
    SPHB_TRY(e.keysTmp.reserve(n));
    SPHB_TRY(e.segKey.reserve(n));
    SPHB_TRY(e.segOfSlot.reserve(n));
    SPHB_TRY(e.order.reserve(n));
    SPHB_TRY(e.inst.reserve(n));
    SPHB_TRY(e.sortScratch.reserve(sortScratchBytes(n)));
    SPHB_TRY(e.pos.reserve(n));
    if (e.mixed) { SPHB_TRY(e.posq.reserve(n)); }
    SPHB_TRY(e.blockLo.reserve(n / kBlockSize + 1));
    SPHB_TRY(e.blockHi.reserve(n / kBlockSize + 1));
    SPHB_TRY(e.nidx.reserve((n / kWarp) * size_t(paddedNgmax(e.p.ngmax)) * kWarp));
    SPHB_TRY(e.nc.reserve(n));
    for (int d = 0; d < kNumDerived; ++d)
    {
        SPHB_TRY(e.derived[d].reserve(n * e.elemBytes()));
    }
    SPHB_TRY(e.du.reserve(n));
    SPHB_TRY(e.hrec.reserve(n * 8 * e.elemBytes()));
    SPHB_TRY(e.grec.reserve(n * 8 * e.elemBytes()));
    SPHB_TRY(e.avrec.reserve(n * 8 * e.elemBytes()));
    if (e.p.av_clean)
    {
        SPHB_TRY(e.dvrec.reserve(n * 8 * e.elemBytes()));
        SPHB_TRY(e.dv.reserve(n * 6 * e.elemBytes()));
    }
    SPHB_TRY(e.alphaBackup.reserve(n));
    SPHB_TRY(e.hBackup.reserve(n));
    int m = e.num;
    SPHB_TRY(e.gamma.reserve(m));
    SPHB_TRY(e.cv.reserve(m));
    SPHB_TRY(e.dt.reserve(m));
    SPHB_TRY(e.dtm1.reserve(m));
    SPHB_TRY(e.ttot.reserve(m));
    SPHB_TRY(e.cons.reserve(size_t(kNumCons) * m));
    SPHB_TRY(e.reduce.reserve(2 * size_t(m)));
    SPHB_TRY(e.status.reserve(4));
    SPHB_TRY(e.sortFlags.reserve(2));
    SPHB_TRY(e.views.reserve(m));
    SPHB_TRY(e.leafDescs.reserve(m));
    for (auto& ev : e.ev)
    {
        SPHB_CUDA_TRY(cudaEventCreate(&ev));
    }
    e.skin = e.p.nb_skin > 0.0;
    if (e.skin)
    {
        double grow = (1.0 + e.p.nb_skin) * (1.0 + e.p.nb_skin) * (1.0 + e.p.nb_skin);
        e.skinCap   = paddedNgmax(unsigned(std::ceil(e.p.ngmax * grow * 1.1)));
        size_t groups = n / kWarp;
        SPHB_TRY(e.skinRows.reserve(groups * size_t(e.skinCap) * kWarp));
        SPHB_TRY(e.skinDist.reserve(groups * size_t(e.skinCap) * kWarp));
        SPHB_TRY(e.skinCount.reserve(n));
        SPHB_TRY(e.skinRadius.reserve(n));
        SPHB_TRY(e.skinXb.reserve(n));
        SPHB_TRY(e.skinYb.reserve(n));
        SPHB_TRY(e.skinZb.reserve(n));
        SPHB_TRY(e.skinBuild.reserve(n));
        SPHB_TRY(e.skinBuildTmp.reserve(n));
        SPHB_TRY(e.skinMoved.reserve(groups));
        SPHB_TRY(e.skinGrid.reserve(size_t(kSkinCells) * size_t(m)));
        SPHB_TRY(e.skinWork.reserve(2 * groups));
        SPHB_TRY(e.skinGroupD.reserve(groups));
        SPHB_TRY(e.skinCtl.reserve(kCtlWords));
    }

    std::vector<double> wh(kTableSize), whd(kTableSize);
    e.K = sincKernelTables(e.p.sinc_index, wh.data(), whd.data(), kTableSize);
    double cw[kPolyTerms], cdw[kPolyTerms];
    double err = sincPolyCoeffs(e.p.sinc_index, kPolyTerms - 1, cw, cdw);
    e.polyOk   = err < 1e-6 ? 1 : 0;
    for (int q = 0; q < kPolyTerms; ++q)
    {
        e.wpoly[q]  = float(cw[q]);
        e.dwpoly[q] = float(cdw[q]);
    }
    SPHB_TRY(e.whD.reserve(kTableSize));
    SPHB_TRY(e.whdD.reserve(kTableSize));
    SPHB_TRY(e.whF.reserve(kTableSize));
    SPHB_TRY(e.whdF.reserve(kTableSize));
    std::vector<float> whf(wh.begin(), wh.end()), whdf(whd.begin(), whd.end());
    SPHB_CUDA_TRY(cudaMemcpy(e.whD.data(), wh.data(), kTableSize * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.whdD.data(), whd.data(), kTableSize * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.whF.data(), whf.data(), kTableSize * sizeof(float), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.whdF.data(), whdf.data(), kTableSize * sizeof(float), cudaMemcpyHostToDevice));

    // static slot maps: instance byte (kGhost for padding) and the segment index as a sort key
    std::vector<uint8_t> inst(n, kGhost);
    std::vector<uint64_t> seg(n);
    for (int k = 0; k < m; ++k)
    {
        size_t end = k + 1 < m ? e.off[k + 1] : n;
        for (size_t s = e.off[k]; s < end; ++s)
        {
            seg[s]  = uint64_t(k);
            inst[s] = s < e.off[k] + e.n[k] ? uint8_t(k) : kGhost;
        }
    }
    SPHB_CUDA_TRY(cudaMemcpy(e.inst.data(), inst.data(), n, cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.segOfSlot.data(), seg.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice));

    std::vector<double> g(m), c(m), d(m), d1(m), z(m, 0.0);
    for (int k = 0; k < m; ++k)
    {
        g[k]  = e.ip[k].gamma;
        c[k]  = idealGasCvE(e.ip[k].mui, e.ip[k].gamma);
        d[k]  = e.ip[k].minDt;
        d1[k] = e.ip[k].minDt_m1;
    }
    SPHB_CUDA_TRY(cudaMemcpy(e.gamma.data(), g.data(), m * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.cv.data(), c.data(), m * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.dt.data(), d.data(), m * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.dtm1.data(), d1.data(), m * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(e.ttot.data(), z.data(), m * sizeof(double), cudaMemcpyHostToDevice));

    for (int k = 0; k < m; ++k)
    {
        e.gtrees.emplace_back(new GlobalTree);
        e.ftrees.emplace_back(new FocusTree);
        e.layouts.emplace_back(new DeviceBuffer<int>);
    }
    return kOk;
}

//! the particle state (14 fields, ids, keys) now lives in the other buffer set
void swapState(sphb_ensemble& e)
{
    for (int k = 0; k < kFields; ++k)
    {
        e.f[k].swap(e.fAlt[k]);
    }
    e.id.swap(e.idAlt);
    e.keys.swap(e.keysAlt);
}

/*! keys, segmented sort, gather of 16 fields into the other buffer set, which then becomes the current one (a
 *  captured step records the buffers of its set; the two captured steps alternate). The sort is decided on the
 *  device, as the single simulation's nearly-sorted sort is on the host: the particles of the previous step are
 *  nearly in order within every instance, so the tiles holding out-of-order pairs are repaired in shared memory,
 *  and the full segmented radix sort (by key over all slots, then stably by instance) runs only if pairs remain out
 *  of order (every one of its kernels reads that count and returns at once when it is zero). The result is the same
 *  stable sort either way. */
int syncBatched(sphb_ensemble& e, bool withLayout)
{
    cudaStream_t st = e.stream;
    size_t n        = e.slots;
    SPHB_TRY(launchSfcKeys(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.keys.data(), n, e.box, st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(e.keysTmp.data(), e.keys.data(), n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    SPHB_TRY(repairSegmentedAsync(e.keysTmp.data(), e.order.data(), e.segOfSlot.data(), n, e.sortFlags.data(), st));
    const uint32_t* remaining = e.sortFlags.data() + 1;
    SPHB_TRY(sortByKeyAsync(e.keysTmp.data(), e.order.data(), n, false, e.sortScratch.data(),
                            e.sortScratch.capacity(), 0xffu, e.status.data() + 2, st, remaining));
    const void* segSrc[1] = {e.segOfSlot.data()};
    void* segDst[1]       = {e.segKey.data()};
    SPHB_TRY(gather8(e.order.data(), n, 1, segSrc, segDst, st));
    SPHB_TRY(sortByKeyAsync(e.segKey.data(), e.order.data(), n, false, e.sortScratch.data(),
                            e.sortScratch.capacity(), 0x1u, e.status.data() + 2, st, remaining));
    const void* src[16];
    void* dst[16];
    for (int k = 0; k < kFields; ++k)
    {
        src[k] = e.f[k].data();
        dst[k] = e.fAlt[k].data();
    }
    src[14] = e.id.data();
    dst[14] = e.idAlt.data();
    src[15] = e.keys.data();
    dst[15] = e.keysAlt.data();
    SPHB_TRY(gather8(e.order.data(), n, 16, src, dst, st));
    swapState(e);
    countLaunch(9);
    if (e.skin)
    {
        // the skin rows hold build indices: compose this sort into the current-to-build map
        SPHB_TRY(skinRemap(e.order.data(), e.skinBuild.data(), e.skinBuildTmp.data(), e.skinMoved.data(), n, st));
        SPHB_CUDA_TRY(cudaMemcpyAsync(e.skinBuild.data(), e.skinBuildTmp.data(), n * sizeof(uint32_t),
                                      cudaMemcpyDeviceToDevice, st));
    }
    if (withLayout)
    {
        dim3 grid(unsigned(ceilDiv(size_t(e.maxLeaves) + 1, 256)), unsigned(e.num));
        forestLayoutKernel<<<grid, 256, 0, st>>>(e.leafDescs.data(), e.keys.data());
        countLaunch();
        SPHB_CUDA_TRY(cudaGetLastError());
    }
    SPHB_TRY(packPositionsAndBoxes(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.f[4].data(), n, e.pos.data(),
                                   e.mixed ? e.posq.data() : nullptr, e.box, e.blockLo.data(), e.blockHi.data(), st));
    return kOk;
}

//! per-instance trees from the current sorted keys (host-driven, outside any capture)
int rebuildTrees(sphb_ensemble& e)
{
    cudaStream_t st = e.stream;
    std::vector<TreeView> views(e.num);
    std::vector<LeafDesc> descs(e.num);
    e.maxLeaves = 0;
    for (int k = 0; k < e.num; ++k)
    {
        GlobalTree& g = *e.gtrees[k];
        FocusTree& f  = *e.ftrees[k];
        const uint64_t* keys = e.keys.data() + e.off[k];
        size_t nk            = e.n[k];
        SPHB_TRY(updateGlobalTree(g, keys, nk, e.ts, st));
        bool converged = false;
        if (f.firstCall)
        {
            int guard = 0;
            while (!converged)
            {
                SPHB_TRY(focusUpdateTree(f, g, e.ts, st, &converged));
                SPHB_TRY(focusUpdateCounts(f, keys, nk, e.ts, st));
                if (++guard > 100) { return kErrNotConverged; }
            }
            f.firstCall = false;
        }
        SPHB_TRY(focusUpdateTree(f, g, e.ts, st, &converged));
        SPHB_TRY(focusUpdateCounts(f, keys, nk, e.ts, st));
        SPHB_TRY(computeGeoCenters(f.tree, e.box, st));
        SPHB_TRY(e.layouts[k]->reserve(size_t(f.numLeaves) + 1));
        TreeView tv;
        tv.childOffsets = f.tree.childOffsets.data();
        tv.nodeToLeaf   = f.tree.nodeToLeaf.data();
        tv.centers      = f.tree.centers.data();
        tv.sizes        = f.tree.sizes.data();
        tv.layout       = e.layouts[k]->data();
        tv.blockLo      = e.blockLo.data();
        tv.blockHi      = e.blockHi.data();
        tv.numNodes     = f.tree.numNodes;
        views[k]        = tv;
        descs[k]        = LeafDesc{f.leaves.data(), e.layouts[k]->data(), f.numLeaves, uint32_t(e.off[k]),
                            uint32_t(e.n[k])};
        e.maxLeaves     = std::max(e.maxLeaves, f.numLeaves);
    }
    SPHB_CUDA_TRY(cudaMemcpyAsync(e.views.data(), views.data(), e.num * sizeof(TreeView), cudaMemcpyHostToDevice, st));
    SPHB_CUDA_TRY(
        cudaMemcpyAsync(e.leafDescs.data(), descs.data(), e.num * sizeof(LeafDesc), cudaMemcpyHostToDevice, st));
    dim3 grid(unsigned(ceilDiv(size_t(e.maxLeaves) + 1, 256)), unsigned(e.num));
    forestLayoutKernel<<<grid, 256, 0, st>>>(e.leafDescs.data(), e.keys.data());
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    return kOk;
}

template<class T>
ChainArrays<T> chainOf(sphb_ensemble& e)
{
    ChainArrays<T> a;
    a.n     = e.slots;
    a.pos   = e.pos.data();
    a.posq  = e.posq.data();
    a.h     = e.f[3].data();
    a.vx    = e.f[6].data();
    a.vy    = e.f[7].data();
    a.vz    = e.f[8].data();
    a.temp  = e.f[5].data();
    a.alpha = e.f[13].data();
    a.nidx  = e.nidx.data();
    a.nc    = e.nc.data();
    if constexpr (sizeof(T) == 8)
    {
        a.wh  = reinterpret_cast<const T*>(e.whD.data());
        a.whd = reinterpret_cast<const T*>(e.whdD.data());
    }
    else
    {
        a.wh  = reinterpret_cast<const T*>(e.whF.data());
        a.whd = reinterpret_cast<const T*>(e.whdF.data());
    }
    a.xm    = e.dptr<T>(dXm);
    a.kx    = e.dptr<T>(dKx);
    a.gradh = e.dptr<T>(dGradh);
    a.prho  = e.dptr<T>(dPrho);
    a.c     = e.dptr<T>(dC);
    for (int q = 0; q < 6; ++q)
    {
        a.cij[q] = e.dptr<T>(dC11 + q);
    }
    a.divv         = e.dptr<T>(dDivv);
    a.curlv        = e.dptr<T>(dCurlv);
    a.ax           = e.dptr<T>(dAx);
    a.ay           = e.dptr<T>(dAy);
    a.az           = e.dptr<T>(dAz);
    a.du           = e.du.data();
    a.hrec         = reinterpret_cast<HydroRec<T>*>(e.hrec.data());
    a.grec         = reinterpret_cast<GradRec<T>*>(e.grec.data());
    a.reduce       = e.reduce.data();
    a.batch.inst   = e.inst.data();
    a.batch.gamma  = e.gamma.data();
    a.batch.cv     = e.cv.data();
    a.batch.dt     = e.dt.data();
    a.batch.dtm1   = e.dtm1.data();
    a.batch.reduce = e.reduce.data();
    a.avrec        = reinterpret_cast<AVRec<T>*>(e.avrec.data());
    if (e.p.av_clean)
    {
        a.dvrec = reinterpret_cast<DVRec<T>*>(e.dvrec.data());
        for (int q = 0; q < 6; ++q)
        {
            a.dv[q] = reinterpret_cast<T*>(e.dv.data()) + size_t(q) * e.slots;
        }
    }
    return a;
}

template<class T>
HydroConsts<T> constsOf(const sphb_ensemble& e)
{
    HydroConsts<T> k;
    k.K        = T(e.K);
    k.alphamin = T(e.p.alphamin);
    k.alphamax = T(e.p.alphamax);
    k.decay    = T(e.p.decay_constant);
    k.Atmin    = T(0.1);
    k.Atmax    = T(0.2);
    k.ramp     = T(1.0) / (k.Atmax - k.Atmin);
    k.Kcour    = double(float(e.p.Kcour));
    k.gamma    = e.p.gamma;
    k.cv       = idealGasCvE(e.p.mui, e.p.gamma);
    k.ngmax    = e.p.ngmax;
    k.usePoly  = 0;
    if constexpr (sizeof(T) == 4)
    {
        k.usePoly = e.polyOk;
        for (int q = 0; q < kPolyTerms; ++q)
        {
            k.wpoly[q]  = e.wpoly[q];
            k.dwpoly[q] = e.dwpoly[q];
        }
        FixedFrame fr = fixedFrameOf(e.box);
        for (int d = 0; d < 3; ++d)
        {
            k.qscale[d] = float(fr.unit[d]);
        }
    }
    return k;
}

//! the J-loops in chain order with the tuned block sizes; which < 0: all, else only that one
//! record the event that starts a stage time; inside a stream capture it becomes an event-record node of the graph
cudaError_t stageMark(sphb_ensemble& e, int k)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err            = cudaStreamIsCapturing(e.stream, &cs);
    if (err != cudaSuccess) { return err; }
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e.ev[k], e.stream, cudaEventRecordExternal)
                                               : cudaEventRecord(e.ev[k], e.stream);
}

template<class T>
int runChainBatched(sphb_ensemble& e, int which = -1)
{
    ChainArrays<T> a = chainOf<T>(e);
    HydroConsts<T> k = constsOf<T>(e);
    cudaStream_t st  = e.stream;
    auto with        = [&](int q) {
        ChainArrays<T> b = a;
        b.threads        = e.threads[q];
        return b;
    };
    auto mark = [&](int stage) { return which < 0 ? stageMark(e, stage) : cudaSuccess; };
    SPHB_CUDA_TRY(mark(2));
    if (which < 0 || which == 0) { SPHB_TRY(launchXMass(with(0), k, e.box, st)); }
    SPHB_CUDA_TRY(mark(3));
    if (which < 0 || which == 1) { SPHB_TRY(launchVeDefGradhEos(with(1), k, e.box, st)); }
    SPHB_CUDA_TRY(mark(4));
    if (which < 0 || which == 2) { SPHB_TRY(launchIadDivvCurlv(with(2), k, e.box, st)); }
    SPHB_CUDA_TRY(mark(5));
    if (which < 0 || which == 3) { SPHB_TRY(launchAVswitches(with(3), k, e.box, 0.0, st)); }
    SPHB_CUDA_TRY(mark(6));
    if (which < 0 || which == 4) { SPHB_TRY(launchMomentumEnergy(with(4), k, e.box, st)); }
    return kOk;
}

template<class T>
int integrateBatched(sphb_ensemble& e)
{
    cudaStream_t st = e.stream;
    size_t n        = e.slots;
    timestepKernel<<<ceilDiv(size_t(e.num), 64), 64, 0, st>>>(e.num, e.reduce.data(), e.dt.data(), e.dtm1.data(),
                                                             e.ttot.data(), e.p.Krho);
    countLaunch();
    IntegrateArrays<T> a;
    a.x          = e.f[0].data();
    a.y          = e.f[1].data();
    a.z          = e.f[2].data();
    a.vx         = e.f[6].data();
    a.vy         = e.f[7].data();
    a.vz         = e.f[8].data();
    a.xm1        = e.f[9].data();
    a.ym1        = e.f[10].data();
    a.zm1        = e.f[11].data();
    a.temp       = e.f[5].data();
    a.duM1       = e.f[12].data();
    a.du         = e.du.data();
    a.ax         = e.dptr<T>(dAx);
    a.ay         = e.dptr<T>(dAy);
    a.az         = e.dptr<T>(dAz);
    a.batch.inst = e.inst.data();
    a.batch.dt   = e.dt.data();
    a.batch.dtm1 = e.dtm1.data();
    a.batch.cv   = e.cv.data();
    SPHB_TRY(launchPositions(n, a, e.box, 0.0, 1.0, 1.0, st));
    SPHB_TRY(launchUpdateH(n, e.p.ng0, e.nc.data(), e.f[3].data(), e.keys.data(), e.status.data() + 1, st,
                           e.inst.data()));
    return kOk;
}

//! rows invalid, counters zero (a new state)
int resetSkin(sphb_ensemble& e)
{
    if (!e.skin) { return kOk; }
    unsigned ctl[kCtlWords] = {};
    ctl[kCtlGroups]         = unsigned(e.slots / kWarp);
    SPHB_CUDA_TRY(cudaMemcpyAsync(e.skinCtl.data(), ctl, sizeof(ctl), cudaMemcpyHostToDevice, e.stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(e.stream));
    return kOk;
}

/*! The neighbour stage with skin rows, every step the same launches (graph-replayable): skinDecide picks the mode on
 *  the device, and each launch returns at once unless the mode is its own. The lists are those of the tree search. */
int searchBatchedSkin(sphb_ensemble& e, const NeighborParams& np)
{
    cudaStream_t st      = e.stream;
    size_t n             = e.slots;
    size_t groups        = n / kWarp;
    unsigned* ctl        = e.skinCtl.data();
    const unsigned* mode = ctl + kCtlMode;
    TreeView dummy{};
    SPHB_TRY(skinDecide(ctl, st));
    SPHB_TRY(findNeighbors(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.pos.data(), e.f[3].data(), n, dummy, e.box,
                           np, e.nidx.data(), e.nc.data(), e.status.data(), st, e.views.data(), e.inst.data(), mode,
                           (1u << kSkinModeTree) | (1u << kSkinModeBuild)));
    SkinLists sl{e.skinRows.data(), e.skinCount.data(), e.skinRadius.data(), e.skinCap, e.skinDist.data()};
    SPHB_TRY(buildSkinLists(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.pos.data(), e.f[3].data(), n, dummy, e.box,
                            np, e.p.nb_skin, sl, e.status.data(), st, e.views.data(), e.inst.data(), mode,
                            1u << kSkinModeBuild));
    SPHB_TRY(skinCommit(e.f[0].data(), e.f[1].data(), e.f[2].data(), n, e.skinXb.data(), e.skinYb.data(),
                        e.skinZb.data(), e.skinBuild.data(), e.skinMoved.data(), ctl, st));
    SPHB_CUDA_TRY(cudaMemsetAsync(e.skinGrid.data(), 0, size_t(kSkinCells) * size_t(e.num) * sizeof(unsigned), st));
    SPHB_TRY(skinDisplacement(e.pos.data(), e.skinXb.data(), e.skinYb.data(), e.skinZb.data(), e.skinBuild.data(), n,
                              e.box, e.skinGrid.data(), st, e.inst.data(), mode));
    SkinFilterArgs a{};
    a.pos  = e.pos.data();
    a.posq = e.mixed ? e.posq.data() : nullptr;
    FixedFrame fr  = fixedFrameOf(e.box);
    double unitMax = 0;
    for (int k = 0; k < 3; ++k)
    {
        a.qscale[k] = float(fr.unit[k]);
        unitMax     = std::max(unitMax, fr.unit[k]);
    }
    a.qunit        = float(unitMax * (1.0 + 1e-6));
    a.h            = e.f[3].data();
    a.nc           = e.nc.data();
    a.nidx         = e.nidx.data();
    a.sl           = sl;
    a.xb           = e.skinXb.data();
    a.yb           = e.skinYb.data();
    a.zb           = e.skinZb.data();
    a.moved        = e.skinMoved.data();
    a.dispGrid     = e.skinGrid.data();
    a.groupD       = e.skinGroupD.data();
    a.numWorklist  = ctl + kCtlDeferredA;
    a.numWorklist2 = ctl + kCtlDeferredB;
    a.worklist     = e.skinWork.data();
    a.worklist2    = e.skinWork.data() + groups;
    a.n            = n;
    a.box          = e.box;
    a.prm          = np;
    a.inst         = e.inst.data();
    a.gate         = mode;
    SPHB_TRY(checkSkinGroups(a, st));
    // the deferred counts stay zero unless the mode is the refilter, and then the listed searches see them
    SPHB_TRY(findNeighborsListed(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.pos.data(), e.f[3].data(), n, dummy,
                                 e.box, np, e.nidx.data(), e.nc.data(), e.status.data(), a.worklist, a.numWorklist, st,
                                 e.views.data(), e.inst.data()));
    SPHB_TRY(filterSkinLists(a, st));
    return findNeighborsListed(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.pos.data(), e.f[3].data(), n, dummy,
                               e.box, np, e.nidx.data(), e.nc.data(), e.status.data(), a.worklist2, a.numWorklist2,
                               st, e.views.data(), e.inst.data());
}

//! one whole step for every instance, without host synchronisation (capturable)
int stepBatched(sphb_ensemble& e)
{
    cudaStream_t st = e.stream;
    size_t n        = e.slots;
    SPHB_CUDA_TRY(stageMark(e, 0));
    SPHB_TRY(syncBatched(e, true));
    SPHB_CUDA_TRY(stageMark(e, 1));
    initReduceKernel<<<ceilDiv(size_t(e.num), 64), 64, 0, st>>>(e.num, e.reduce.data(), e.cons.data());
    countLaunch();
    TreeView dummy{};
    NeighborParams np{e.p.ng0, e.p.ngmax, 10};
    if (e.skin) { SPHB_TRY(searchBatchedSkin(e, np)); }
    else
    {
        SPHB_TRY(findNeighbors(e.f[0].data(), e.f[1].data(), e.f[2].data(), e.pos.data(), e.f[3].data(), n, dummy,
                               e.box, np, e.nidx.data(), e.nc.data(), e.status.data(), st, e.views.data(),
                               e.inst.data()));
    }
    if (e.mixed) { SPHB_TRY(runChainBatched<float>(e)); }
    else { SPHB_TRY(runChainBatched<double>(e)); }
    SPHB_CUDA_TRY(stageMark(e, 7));
    consBatchKernel<<<kConsWarps / 8, 256, 0, st>>>(n, e.inst.data(), e.f[0].data(), e.f[1].data(), e.f[2].data(),
                                                     e.f[6].data(), e.f[7].data(), e.f[8].data(), e.f[4].data(),
                                                     e.f[5].data(), e.nc.data(), e.cv.data(), e.cons.data());
    countLaunch();
    SPHB_CUDA_TRY(stageMark(e, 8));
    if (e.mixed) { SPHB_TRY(integrateBatched<float>(e)); }
    else { SPHB_TRY(integrateBatched<double>(e)); }
    SPHB_CUDA_TRY(stageMark(e, 9));
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int dropGraph(sphb_ensemble& e)
{
    for (auto& g : e.graphs)
    {
        if (g)
        {
            SPHB_CUDA_TRY(cudaGraphExecDestroy(g));
            g = nullptr;
        }
    }
    e.parity = 0;
    return kOk;
}

/*! Capture two consecutive steps. Capturing runs nothing, but each captured step swaps the host's buffer sets, so
 *  after both the host's sets are as before and graphs[0] starts from the current state. */
int captureGraph(sphb_ensemble& e)
{
    SPHB_TRY(dropGraph(e));
    const double* current = e.f[0].data(); // where the state is: capturing moves nothing
    for (int q = 0; q < 2; ++q)
    {
        cudaGraph_t g = nullptr;
        SPHB_CUDA_TRY(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
        uint64_t l0       = launchCounter();
        int rc            = stepBatched(e);
        e.launchesPerStep = launchCounter() - l0;
        launchCounter()   = l0; // counted again on every replay
        cudaError_t ce    = cudaStreamEndCapture(e.stream, &g);
        if (rc != kOk)
        {
            if (g) { cudaGraphDestroy(g); }
            if (e.f[0].data() != current) { swapState(e); }
            dropGraph(e);
            return rc;
        }
        SPHB_CUDA_TRY(ce);
        cudaError_t ie = cudaGraphInstantiate(&e.graphs[q], g, 0);
        cudaGraphDestroy(g);
        SPHB_CUDA_TRY(ie);
    }
    return kOk;
}

int checkStatus(sphb_ensemble& e)
{
    unsigned st[4] = {0, 0, 0, 0};
    SPHB_CUDA_TRY(cudaMemcpyAsync(st, e.status.data(), sizeof(st), cudaMemcpyDeviceToHost, e.stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(e.stream));
    if (st[0] || st[2]) { return kErrCapacity; }
    if (st[1]) { return kErrNotConverged; }
    return kOk;
}

bool fieldPtr(sphb_ensemble* e, const char* name, void** ptr, int* kind)
{
    for (int k = 0; k < kFields; ++k)
    {
        if (std::strcmp(name, kFieldNames[k]) == 0)
        {
            *ptr  = e->f[k].data();
            *kind = 0;
            return true;
        }
    }
    for (int d = 0; d < kNumDerived; ++d)
    {
        if (std::strcmp(name, kDerivedNames[d]) == 0)
        {
            *ptr  = e->derived[d].data();
            *kind = 1;
            return true;
        }
    }
    if (std::strcmp(name, "du") == 0)
    {
        *ptr  = e->du.data();
        *kind = 0;
        return true;
    }
    if (std::strcmp(name, "nc") == 0)
    {
        *ptr  = e->nc.data();
        *kind = 2;
        return true;
    }
    if (std::strcmp(name, "id") == 0 || std::strcmp(name, "keys") == 0)
    {
        *ptr  = name[0] == 'i' ? e->id.data() : e->keys.data();
        *kind = 3;
        return true;
    }
    return false;
}

} // namespace
} // namespace sphb

// ------------------------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------------------------

extern "C" int sphb_ensemble_create(sphb_ensemble** out, int num, const size_t* sizes, const sphb_box* box,
                                    const sphb_params* params)
{
    if (!out || !sizes || !box || !params || num < 1 || num > kMaxInst) { return SPHB_ERR_ARG; }
    const sphb_params& p0 = params[0];
    if (p0.ng0 > p0.ngmax || p0.ngmax == 0 || p0.bucket_focus == 0) { return SPHB_ERR_ARG; }
    if (p0.precision != SPHB_FP64 && p0.precision != SPHB_MIXED) { return SPHB_ERR_ARG; }
    for (int k = 0; k < 3; ++k)
    {
        if (!(box->hi[k] > box->lo[k]) || !box->periodic[k]) { return SPHB_ERR_ARG; }
    }
    size_t total = 0;
    for (int k = 0; k < num; ++k)
    {
        const sphb_params& q = params[k];
        if (sizes[k] == 0 || q.ng0 != p0.ng0 || q.ngmax != p0.ngmax || q.precision != p0.precision ||
            q.sinc_index != p0.sinc_index || q.bucket_focus != p0.bucket_focus || q.alphamin != p0.alphamin ||
            q.alphamax != p0.alphamax || q.decay_constant != p0.decay_constant || q.Kcour != p0.Kcour ||
            q.Krho != p0.Krho || q.av_clean != p0.av_clean || !(q.gamma > 1.0))
        {
            return SPHB_ERR_ARG;
        }
        total += (sizes[k] + kWarp - 1) / kWarp * kWarp;
    }
    if (total >= (size_t(1) << 30)) { return SPHB_ERR_ARG; }
    auto* e  = new sphb_ensemble;
    e->num   = num;
    e->p     = p0;
    e->hbox  = *box;
    e->box   = makeDevBox(*box);
    e->mixed = p0.precision == SPHB_MIXED;
    e->ip.assign(params, params + num);
    size_t o = 0;
    for (int k = 0; k < num; ++k)
    {
        e->n.push_back(sizes[k]);
        e->off.push_back(o);
        o += (sizes[k] + kWarp - 1) / kWarp * kWarp;
    }
    e->slots = o;
    int rc   = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess ? kOk : kErrCuda;
    if (rc == kOk) { rc = allocate(*e); }
    if (rc != kOk)
    {
        if (e->stream) { cudaStreamDestroy(e->stream); }
        delete e;
        return rc;
    }
    *out = e;
    return SPHB_OK;
}

extern "C" int sphb_ensemble_destroy(sphb_ensemble* e)
{
    if (!e) { return SPHB_ERR_ARG; }
    if (e->stream) { cudaStreamSynchronize(e->stream); }
    dropGraph(*e);
    for (auto& ev : e->ev)
    {
        if (ev) { cudaEventDestroy(ev); }
    }
    if (e->stream) { cudaStreamDestroy(e->stream); }
    delete e;
    return SPHB_OK;
}

extern "C" int sphb_ensemble_upload(sphb_ensemble* e, int k, const double* const* fields, const uint64_t* id,
                                    int on_device)
{
    if (!e || !fields || !id || k < 0 || k >= e->num) { return SPHB_ERR_ARG; }
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    size_t o = e->off[k], nk = e->n[k];
    size_t end = k + 1 < e->num ? e->off[k + 1] : e->slots;
    for (int f = 0; f < kFields; ++f)
    {
        if (!fields[f]) { return SPHB_ERR_ARG; }
        SPHB_CUDA_TRY(cudaMemcpyAsync(e->f[f].data() + o, fields[f], nk * sizeof(double), kind, e->stream));
        // padding slots: at the box centre, zero everything else
        SPHB_CUDA_TRY(cudaMemsetAsync(e->f[f].data() + o + nk, 0, (end - o - nk) * sizeof(double), e->stream));
    }
    SPHB_CUDA_TRY(cudaMemcpyAsync(e->id.data() + o, id, nk * sizeof(uint64_t), kind, e->stream));
    SPHB_CUDA_TRY(cudaMemsetAsync(e->id.data() + o + nk, 0xff, (end - o - nk) * sizeof(uint64_t), e->stream));
    SPHB_CUDA_TRY(cudaMemsetAsync(e->keys.data() + o, 0, nk * sizeof(uint64_t), e->stream));
    std::vector<uint64_t> ghostKeys(end - o - nk, kRemoveKey);
    std::vector<double> centre(end - o - nk);
    if (!ghostKeys.empty())
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(e->keys.data() + o + nk, ghostKeys.data(), ghostKeys.size() * sizeof(uint64_t),
                                      cudaMemcpyHostToDevice, e->stream));
        for (int d = 0; d < 3; ++d)
        {
            std::fill(centre.begin(), centre.end(), 0.5 * (e->hbox.lo[d] + e->hbox.hi[d]));
            SPHB_CUDA_TRY(cudaMemcpyAsync(e->f[d].data() + o + nk, centre.data(), centre.size() * sizeof(double),
                                          cudaMemcpyHostToDevice, e->stream));
        }
    }
    SPHB_CUDA_TRY(cudaMemsetAsync(e->du.data() + o, 0, (end - o) * sizeof(double), e->stream));
    SPHB_TRY(initGlobalTree(*e->gtrees[k], std::max<unsigned>(e->p.bucket_focus, unsigned(nk / 100)), e->stream));
    SPHB_TRY(initFocusTree(*e->ftrees[k], e->p.bucket_focus, e->ts, e->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(e->stream));
    e->uploaded = true;
    e->synced   = false;
    return resetSkin(*e);
}

extern "C" int sphb_ensemble_initial_sync(sphb_ensemble* e)
{
    if (!e || !e->uploaded) { return e ? SPHB_ERR_STATE : SPHB_ERR_ARG; }
    SPHB_CUDA_TRY(cudaMemsetAsync(e->status.data(), 0, 4 * sizeof(unsigned), e->stream));
    initReduceKernel<<<ceilDiv(size_t(e->num), 64), 64, 0, e->stream>>>(e->num, e->reduce.data(), e->cons.data());
    SPHB_TRY(resetSkin(*e));
    SPHB_TRY(syncBatched(*e, false));
    SPHB_TRY(rebuildTrees(*e));
    SPHB_TRY(checkStatus(*e));
    SPHB_TRY(dropGraph(*e));
    e->synced = true;
    return SPHB_OK;
}

extern "C" int sphb_ensemble_rebuild_trees(sphb_ensemble* e)
{
    if (!e || !e->synced) { return e ? SPHB_ERR_STATE : SPHB_ERR_ARG; }
    SPHB_TRY(rebuildTrees(*e));
    // the captured step holds the tree views by device address, which stay valid unless a tree grew
    return dropGraph(*e);
}

extern "C" int sphb_ensemble_set_threads(sphb_ensemble* e, const int* threads)
{
    if (!e || !threads) { return SPHB_ERR_ARG; }
    for (int q = 0; q < kJLoops; ++q)
    {
        int t   = threads[q];
        int tmx = (q == kAvLoop && e->mixed) ? kAvMaxThreads : kChainMaxThreads;
        if (t < 32 || t > tmx || t % 32) { return SPHB_ERR_ARG; }
    }
    std::copy(threads, threads + kJLoops, e->threads);
    return dropGraph(*e);
}

extern "C" int sphb_ensemble_step(sphb_ensemble* e, int steps, int use_graph)
{
    if (!e || steps < 0) { return SPHB_ERR_ARG; }
    if (!e->synced) { return SPHB_ERR_STATE; }
    if (use_graph && !e->graphs[0]) { SPHB_TRY(captureGraph(*e)); }
    // an eager step moves the state to the other buffer set on its own, which the captured pair cannot follow
    if (!use_graph && steps > 0) { SPHB_TRY(dropGraph(*e)); }
    for (int s = 0; s < steps; ++s)
    {
        if (use_graph)
        {
            SPHB_CUDA_TRY(cudaGraphLaunch(e->graphs[e->parity], e->stream));
            countLaunch(e->launchesPerStep);
            swapState(*e);
            e->parity ^= 1;
        }
        else { SPHB_TRY(stepBatched(*e)); }
    }
    e->steps += uint64_t(steps);
    return checkStatus(*e);
}

/*! Autotuner of the J-loop launch shapes: with the forces of the current state computed once, each J-loop is timed
 *  (CUDA events, median of 3) at every candidate block size and the fastest is kept. The AV switches update alpha in
 *  place, so alpha is restored after each of their trials; the other J-loops only overwrite their outputs. */
extern "C" int sphb_ensemble_autotune(sphb_ensemble* e, int* threads_out)
{
    if (!e || !e->synced) { return e ? SPHB_ERR_STATE : SPHB_ERR_ARG; }
    cudaStream_t st = e->stream;
    size_t n        = e->slots;
    SPHB_TRY(syncBatched(*e, true));
    initReduceKernel<<<ceilDiv(size_t(e->num), 64), 64, 0, st>>>(e->num, e->reduce.data(), e->cons.data());
    // the search may change h (count iterations): the state is restored after tuning
    SPHB_CUDA_TRY(cudaMemcpyAsync(e->hBackup.data(), e->f[3].data(), n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TreeView dummy{};
    NeighborParams np{e->p.ng0, e->p.ngmax, 10};
    SPHB_TRY(findNeighbors(e->f[0].data(), e->f[1].data(), e->f[2].data(), e->pos.data(), e->f[3].data(), n, dummy, e->box, np,
                           e->nidx.data(), e->nc.data(), e->status.data(), st, e->views.data(), e->inst.data()));
    SPHB_CUDA_TRY(cudaMemcpyAsync(e->alphaBackup.data(), e->f[13].data(), n * sizeof(double),
                                  cudaMemcpyDeviceToDevice, st));
    if (e->mixed) { SPHB_TRY(runChainBatched<float>(*e)); }
    else { SPHB_TRY(runChainBatched<double>(*e)); }
    cudaEvent_t a, b;
    SPHB_CUDA_TRY(cudaEventCreate(&a));
    SPHB_CUDA_TRY(cudaEventCreate(&b));
    // 384 only for the FP32 AV switches, the one J-loop whose bound allows it
    const int cand[4] = {64, 128, 256, 384};
    int rc            = kOk;
    for (int q = 0; q < kJLoops && rc == kOk; ++q)
    {
        float best = INFINITY;
        int bestT  = e->threads[q];
        for (int c : cand)
        {
            if (c > kChainMaxThreads && !(q == kAvLoop && e->mixed)) { continue; }
            e->threads[q] = c;
            float times[3];
            for (int r = 0; r < 3 && rc == kOk; ++r)
            {
                if (q == kAvLoop)
                {
                    cudaMemcpyAsync(e->f[13].data(), e->alphaBackup.data(), n * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st);
                }
                cudaEventRecord(a, st);
                rc = e->mixed ? runChainBatched<float>(*e, q) : runChainBatched<double>(*e, q);
                cudaEventRecord(b, st);
                if (cudaEventSynchronize(b) != cudaSuccess) { rc = kErrCuda; }
                cudaEventElapsedTime(&times[r], a, b);
            }
            std::sort(times, times + 3);
            if (times[1] < best)
            {
                best  = times[1];
                bestT = c;
            }
        }
        e->threads[q] = bestT;
    }
    cudaMemcpyAsync(e->f[13].data(), e->alphaBackup.data(), n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(e->f[3].data(), e->hBackup.data(), n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    initReduceKernel<<<ceilDiv(size_t(e->num), 64), 64, 0, st>>>(e->num, e->reduce.data(), e->cons.data());
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    SPHB_TRY(rc);
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    if (threads_out) { std::copy(e->threads, e->threads + kJLoops, threads_out); }
    return dropGraph(*e);
}

extern "C" int sphb_ensemble_stage_times(sphb_ensemble* e, float* out)
{
    if (!e || !out) { return SPHB_ERR_ARG; }
    if (e->steps == 0) { return SPHB_ERR_STATE; }
    SPHB_CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int k = 0; k < sphb_ensemble::kStages; ++k)
    {
        SPHB_CUDA_TRY(cudaEventElapsedTime(&out[k], e->ev[k], e->ev[k + 1]));
    }
    return SPHB_OK;
}

extern "C" int sphb_ensemble_search_stats(sphb_ensemble* e, uint64_t* out)
{
    if (!e || !out) { return SPHB_ERR_ARG; }
    unsigned ctl[kCtlWords] = {};
    if (e->skin)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(ctl, e->skinCtl.data(), sizeof(ctl), cudaMemcpyDeviceToHost, e->stream));
        SPHB_CUDA_TRY(cudaStreamSynchronize(e->stream));
    }
    out[0] = ctl[kCtlTreeSearches];
    out[1] = ctl[kCtlBuilds];
    out[2] = ctl[kCtlFilterSteps];
    out[3] = ctl[kCtlDeferredTotal] + ctl[kCtlDeferredA] + ctl[kCtlDeferredB];
    return SPHB_OK;
}

extern "C" size_t sphb_ensemble_size(const sphb_ensemble* e, int k)
{
    if (!e || k < 0 || k >= e->num) { return 0; }
    return e->n[k];
}

extern "C" int sphb_ensemble_get_field(sphb_ensemble* e, int k, const char* name, double* out)
{
    if (!e || !name || !out || k < 0 || k >= e->num) { return SPHB_ERR_ARG; }
    void* ptr = nullptr;
    int kind  = 0;
    if (!fieldPtr(e, name, &ptr, &kind)) { return SPHB_ERR_ARG; }
    size_t nk   = e->n[k];
    size_t elem = kind == 0 || kind == 3 ? 8 : kind == 2 ? 4 : e->elemBytes();
    std::vector<char> host(nk * elem);
    const char* src = static_cast<const char*>(ptr) + e->off[k] * elem;
    SPHB_CUDA_TRY(cudaMemcpyAsync(host.data(), src, nk * elem, cudaMemcpyDeviceToHost, e->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (size_t i = 0; i < nk; ++i)
    {
        double v;
        if (kind == 0 || kind == 3 || (kind == 1 && elem == 8)) { std::memcpy(&v, host.data() + 8 * i, 8); }
        else if (kind == 1) { v = double(reinterpret_cast<const float*>(host.data())[i]); }
        else { v = double(reinterpret_cast<const uint32_t*>(host.data())[i]); }
        out[i] = v;
    }
    return SPHB_OK;
}

extern "C" int sphb_ensemble_scalars(sphb_ensemble* e, int k, double* out)
{
    if (!e || !out || k < 0 || k >= e->num) { return SPHB_ERR_ARG; }
    double d[3], c[kNumCons];
    SPHB_CUDA_TRY(cudaMemcpyAsync(&d[0], e->dt.data() + k, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    SPHB_CUDA_TRY(cudaMemcpyAsync(&d[1], e->dtm1.data() + k, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    SPHB_CUDA_TRY(cudaMemcpyAsync(&d[2], e->ttot.data() + k, sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    SPHB_CUDA_TRY(cudaMemcpyAsync(c, e->cons.data() + kNumCons * k, sizeof(c), cudaMemcpyDeviceToHost, e->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(e->stream));
    out[0] = d[0];
    out[1] = d[1];
    out[2] = d[2];
    out[3] = 0.5 * c[0] + c[1];
    out[4] = 0.5 * c[0];
    out[5] = c[1];
    out[6] = std::sqrt(c[2] * c[2] + c[3] * c[3] + c[4] * c[4]);
    out[7] = std::sqrt(c[5] * c[5] + c[6] * c[6] + c[7] * c[7]);
    out[8] = c[8];
    return SPHB_OK;
}

extern "C" void* sphb_ensemble_stream(sphb_ensemble* e) { return e ? static_cast<void*>(e->stream) : nullptr; }
