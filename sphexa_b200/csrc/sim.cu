// The simulation object: particle dataset in HBM and the whole HydroVeProp step
// (main/src/propagator/ve_hydro.hpp:126-220) at one rank, driven from the host.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "sim.cuh"
#include "tables.hpp"

namespace
{

int allocateSim(sphb_sim& s)
{
    size_t n = s.n;
    for (int k = 0; k < kNumConserved; ++k)
    {
        SPHB_TRY(s.f[k].reserve(n));
        SPHB_TRY(s.fAlt[k].reserve(n));
    }
    SPHB_TRY(s.id.reserve(n));
    SPHB_TRY(s.idAlt.reserve(n));
    SPHB_TRY(s.keys.reserve(n));
    SPHB_TRY(s.order.reserve(n));
    SPHB_TRY(s.sortScratch.reserve(sortScratchBytes(n)));
    SPHB_TRY(s.pos.reserve(n));
    if (s.mixed) { SPHB_TRY(s.posq.reserve(n)); }
    SPHB_TRY(s.blockLo.reserve(n / kBlockSize + 1));
    SPHB_TRY(s.blockHi.reserve(n / kBlockSize + 1));
    SPHB_TRY(s.nidx.reserve(s.numGroups() * size_t(paddedNgmax(s.p.ngmax)) * kWarp));
    SPHB_TRY(s.nc.reserve(n));
    for (int d = 0; d < kNumDerived; ++d)
    {
        SPHB_TRY(s.derived[d].reserve(n * s.elemBytes()));
    }
    SPHB_TRY(s.du.reserve(n));
    SPHB_TRY(s.hrec.reserve(n * 8 * s.elemBytes()));
    SPHB_TRY(s.grec.reserve(n * 8 * s.elemBytes()));
    SPHB_TRY(s.avrec.reserve(n * 8 * s.elemBytes()));
    if (s.p.av_clean)
    {
        SPHB_TRY(s.dvrec.reserve(n * 8 * s.elemBytes()));
        SPHB_TRY(s.dv.reserve(n * 6 * s.elemBytes()));
    }
    SPHB_TRY(s.reduce.reserve(4));
    SPHB_TRY(s.status.reserve(4));
    SPHB_CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&s.hostMsg), 32 * sizeof(unsigned long long)));
    SPHB_TRY(s.partial.reserve(9 * 1024));
    SPHB_TRY(s.cons.reserve(16));

    std::vector<double> wh(kTableSize), whd(kTableSize);
    s.K = sincKernelTables(s.p.sinc_index, wh.data(), whd.data(), kTableSize);
    {
        // the polynomial replaces the table only if it reproduces the kernel to well inside FP32 resolution
        double cw[kPolyTerms], cdw[kPolyTerms];
        double err = sincPolyCoeffs(s.p.sinc_index, kPolyTerms - 1, cw, cdw);
        s.polyOk   = err < 1e-6 ? 1 : 0;
        for (int q = 0; q < kPolyTerms; ++q)
        {
            s.wpoly[q]  = float(cw[q]);
            s.dwpoly[q] = float(cdw[q]);
        }
        s.polyReady = true;
    }
    SPHB_TRY(s.whD.reserve(kTableSize));
    SPHB_TRY(s.whdD.reserve(kTableSize));
    SPHB_CUDA_TRY(cudaMemcpy(s.whD.data(), wh.data(), kTableSize * sizeof(double), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(s.whdD.data(), whd.data(), kTableSize * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<float> whf(wh.begin(), wh.end()), whdf(whd.begin(), whd.end());
    SPHB_TRY(s.whF.reserve(kTableSize));
    SPHB_TRY(s.whdF.reserve(kTableSize));
    SPHB_CUDA_TRY(cudaMemcpy(s.whF.data(), whf.data(), kTableSize * sizeof(float), cudaMemcpyHostToDevice));
    SPHB_CUDA_TRY(cudaMemcpy(s.whdF.data(), whdf.data(), kTableSize * sizeof(float), cudaMemcpyHostToDevice));
    for (auto& e : s.ev)
    {
        SPHB_CUDA_TRY(cudaEventCreate(&e));
    }
    return kOk;
}

double idealGasCv(double mui, double gamma) { return 8.317e7 / mui / (gamma - 1.0); }

//! limitBoxShrinking (cstone/sfc/box.hpp:398-414) and makeGlobalBox (cstone/sfc/box_mpi.hpp:69-107) for open axes
int updateBox(sphb_sim& s)
{
    bool anyOpen = !s.hbox.periodic[0] || !s.hbox.periodic[1] || !s.hbox.periodic[2];
    if (!anyOpen || s.boxFromCaller) { return kOk; }
    double fit[6];
    // the extrema of all three axes in one pass and one read back
    SPHB_TRY(s.boxExtrema.reserve(6));
    SPHB_TRY(minMax3(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.n, s.boxExtrema.data(), s.stream));
    unsigned long long mm[6];
    SPHB_TRY(readBack(s.stream, {{mm, s.boxExtrema.data(), sizeof(mm)}}));
    for (int k = 0; k < 3; ++k)
    {
        fit[2 * k]     = s.hbox.lo[k];
        fit[2 * k + 1] = s.hbox.hi[k];
        if (!s.hbox.periodic[k])
        {
            fit[2 * k]     = fromOrderedBits(mm[2 * k]);
            fit[2 * k + 1] = fromOrderedBits(mm[2 * k + 1]);
        }
    }
    if (!s.boxFirstCall)
    {
        for (int k = 0; k < 3; ++k)
        {
            if (s.hbox.periodic[k]) { continue; }
            double len = s.hbox.hi[k] - s.hbox.lo[k];
            fit[2 * k]     = std::min(fit[2 * k], s.hbox.lo[k] + 0.05 * len);
            fit[2 * k + 1] = std::max(fit[2 * k + 1], s.hbox.hi[k] - 0.05 * len);
        }
    }
    for (int k = 0; k < 3; ++k)
    {
        s.hbox.lo[k] = fit[2 * k];
        s.hbox.hi[k] = fit[2 * k + 1];
    }
    s.box = makeDevBox(s.hbox);
    return kOk;
}

//! Domain::sync at one rank (cstone/domain/domain.hpp:165-213 with assign, assignment.hpp:91-142)
int syncDomain(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    // late fields a previous reordering sync left ungathered are put in its order before this one reorders again
    if (s.midGatherPending) { SPHB_TRY(simimpl::waitMidFields(s)); }
    for (int g = 0; g < sphb_sim::kLateGroups; ++g)
    {
        if (s.lateGatherPending[g]) { SPHB_TRY(simimpl::waitLateGroup(s, g)); }
    }
    SPHB_TRY(updateBox(s));
    s.boxFirstCall = false;
    SPHB_TRY(launchSfcKeys(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.keys.data(), s.n, s.box, st));
    // particles move a fraction of h per step, so the previous order is nearly sorted (often exactly)
    bool identity = false;
    SPHB_TRY(sortNearlySorted(s.keys.data(), s.order.data(), s.n, s.sortScratch.data(), s.sortScratch.capacity(),
                              &identity, st));
    s.lastSyncIdentity = identity;
    if (s.skinValid && !identity)
    {
        // the skin rows hold build indices: track which particle now sits at each index
        SPHB_TRY(skinRemap(s.order.data(), s.skinAnyMoved ? s.skinBuild.data() : nullptr, s.skinBuildAlt.data(),
                           s.skinMoved.data(), s.n, st));
        s.skinBuild.swap(s.skinBuildAlt);
        s.skinAnyMoved = true;
        s.syncRemapped = true;
    }
    SPHB_TRY(updateGlobalTree(s.gtree, s.keys.data(), s.n, s.ts, st));

    if (!identity)
    {
        // reorder every conserved field and the ids into SFC order. Fields of a typed host load still in flight are
        // gathered with the same order once they arrive (waitMidFields: h and the ids, before the search;
        // waitLateGroup): the rest of the sync reads only x, y, z and m
        const void* src[kNumConserved + 2];
        void* dst[kNumConserved + 2];
        bool now[kNumConserved];
        int numFields = 0;
        for (int k = 0; k < kNumConserved; ++k)
        {
            int g  = simimpl::lateGroupOf(k);
            now[k] = k == fH ? !s.midPending : (g < 0 || !s.latePending[g]);
            if (g >= 0 && s.latePending[g]) { s.lateGatherPending[g] = true; }
            if (!now[k]) { continue; }
            src[numFields] = s.f[k].data();
            dst[numFields] = s.fAlt[k].data();
            ++numFields;
        }
        s.midGatherPending = s.midPending;
        if (!s.midPending)
        {
            src[numFields] = s.id.data();
            dst[numFields] = s.idAlt.data();
            ++numFields;
        }
        if (s.bdt)
        {
            src[numFields] = s.rung.data();
            dst[numFields] = s.rungAlt.data();
            ++numFields;
        }
        SPHB_TRY(gather8(s.order.data(), s.n, numFields, src, dst, st));
        for (int k = 0; k < kNumConserved; ++k)
        {
            if (now[k]) { s.f[k].swap(s.fAlt[k]); }
        }
        if (!s.midGatherPending) { s.id.swap(s.idAlt); }
        if (s.bdt) { s.rung.swap(s.rungAlt); }
    }

    bool converged = false;
    if (s.ftree.firstCall)
    {
        int guard = 0;
        while (!converged)
        {
            SPHB_TRY(focusUpdateTree(s.ftree, s.gtree, s.ts, st, &converged));
            SPHB_TRY(focusUpdateCounts(s.ftree, s.keys.data(), s.n, s.ts, st));
            if (++guard > 100) { return kErrNotConverged; }
        }
        s.ftree.firstCall = false;
    }
    SPHB_TRY(focusUpdateTree(s.ftree, s.gtree, s.ts, st, &converged));
    SPHB_TRY(focusUpdateCounts(s.ftree, s.keys.data(), s.n, s.ts, st));
    SPHB_TRY(computeGeoCenters(s.ftree.tree, s.box, st));
    SPHB_TRY(packPositionsAndBoxes(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.f[fM].data(), s.n,
                                   s.pos.data(), s.mixed ? s.posq.data() : nullptr, s.box, s.blockLo.data(),
                                   s.blockHi.data(), st));
    return kOk;
}

template<class T>
ChainArrays<T> chainArrays(sphb_sim& s)
{
    ChainArrays<T> a;
    a.n     = s.n;
    a.pos   = s.pos.data();
    a.posq  = s.posq.data();
    a.h     = s.f[fH].data();
    a.vx    = s.f[fVx].data();
    a.vy    = s.f[fVy].data();
    a.vz    = s.f[fVz].data();
    a.temp  = s.f[fTemp].data();
    a.alpha = s.f[fAlpha].data();
    a.nidx  = s.nidx.data();
    a.nc    = s.nc.data();
    if constexpr (sizeof(T) == 8)
    {
        a.wh  = reinterpret_cast<const T*>(s.whD.data());
        a.whd = reinterpret_cast<const T*>(s.whdD.data());
    }
    else
    {
        a.wh  = reinterpret_cast<const T*>(s.whF.data());
        a.whd = reinterpret_cast<const T*>(s.whdF.data());
    }
    a.xm    = s.dptr<T>(dXm);
    a.kx    = s.dptr<T>(dKx);
    a.gradh = s.dptr<T>(dGradh);
    a.prho  = s.dptr<T>(dPrho);
    a.c     = s.dptr<T>(dC);
    for (int q = 0; q < 6; ++q)
    {
        a.cij[q] = s.dptr<T>(dC11 + q);
    }
    a.divv   = s.dptr<T>(dDivv);
    a.curlv  = s.dptr<T>(dCurlv);
    a.ax     = s.dptr<T>(dAx);
    a.ay     = s.dptr<T>(dAy);
    a.az     = s.dptr<T>(dAz);
    a.du     = s.du.data();
    a.hrec   = reinterpret_cast<HydroRec<T>*>(s.hrec.data());
    a.grec   = reinterpret_cast<GradRec<T>*>(s.grec.data());
    a.reduce = s.reduce.data();
    a.avrec  = reinterpret_cast<AVRec<T>*>(s.avrec.data());
    if (s.p.av_clean)
    {
        a.dvrec = reinterpret_cast<DVRec<T>*>(s.dvrec.data());
        for (int q = 0; q < 6; ++q)
        {
            a.dv[q] = reinterpret_cast<T*>(s.dv.data()) + size_t(q) * s.n;
        }
    }
    if (s.taping)
    {
        T* t          = reinterpret_cast<T*>(s.tapeT.data());
        a.tape.whomega = t;
        a.tape.wrho0   = t + s.n;
        a.tape.gx      = t + 2 * s.n;
        a.tape.gy      = t + 3 * s.n;
        a.tape.gz      = t + 4 * s.n;
        a.tape.vsig    = t + 5 * s.n;
        a.tape.energy  = t + 6 * s.n;
        a.tape.avisc   = t + 7 * s.n;
        a.tape.vsigJ   = s.tapeJ.data();
    }
    return a;
}

template<class T>
HydroConsts<T> hydroConsts(const sphb_sim& s)
{
    HydroConsts<T> k;
    k.K        = T(s.K);
    k.alphamin = T(s.p.alphamin);
    k.alphamax = T(s.p.alphamax);
    k.decay    = T(s.p.decay_constant);
    // Atwood ramp of the crossed/uncrossed momentum weights (sph/include/sph/particles_data.hpp:128-133)
    k.Atmin = T(0.1);
    k.Atmax = T(0.2);
    k.ramp  = T(1.0) / (k.Atmax - k.Atmin);
    k.Kcour = double(float(s.p.Kcour));
    k.gamma = s.p.gamma;
    k.cv    = idealGasCv(s.p.mui, s.p.gamma);
    k.ngmax = s.p.ngmax;
    k.usePoly = 0;
    if constexpr (sizeof(T) == 4)
    {
        k.usePoly = s.polyOk;
        for (int q = 0; q < kPolyTerms; ++q)
        {
            k.wpoly[q]  = s.wpoly[q];
            k.dwpoly[q] = s.dwpoly[q];
        }
        FixedFrame fr = fixedFrameOf(s.box);
        for (int d = 0; d < 3; ++d)
        {
            k.qscale[d] = float(fr.unit[d]);
        }
    }
    return k;
}

/*! Block size of a J-loop launch. 256 threads (8 consecutive groups per block share their neighbours in L1), the FP32
 *  AV switches 384, and 128 for the FP64 AV switches and MomentumEnergy, whose register counts leave more warps
 *  resident that way. Measured at 128^3 against 128 everywhere: FP32 step 6.09 -> 6.04 ms; FP64 XMass, VeDefGradh, IAD
 *  7.07 -> 6.86 ms, while FP64 MomentumEnergy went 5.33 -> 6.61 ms at 256. */
int chainThreads(bool mixed, int stage)
{
    if (mixed) { return stage == sAV ? 384 : 256; }
    return stage == sAV || stage == sMomentum ? 128 : 256;
}

template<class T>
int runChainStage(sphb_sim& s, int stage)
{
    cudaStream_t st  = s.stream;
    ChainArrays<T> a = chainArrays<T>(s);
    HydroConsts<T> k = hydroConsts<T>(s);
    a.threads        = chainThreads(s.mixed, stage);
    switch (stage)
    {
    case sXMass: return launchXMass(a, k, s.box, st);
    case sVeDefGradh:
        // the velocities of a typed host load still in flight: their part of the hydro record follows before IAD
        a.recordNoVelocity    = s.latePending[1];
        s.velocityPackPending = a.recordNoVelocity;
        return launchVeDefGradhEos(a, k, s.box, st);
    case sIad: return launchIadDivvCurlv(a, k, s.box, st);
    case sAV:
        if (s.taping)
        {
            SPHB_CUDA_TRY(cudaMemcpyAsync(s.alphaPre.data(), s.f[fAlpha].data(), s.n * sizeof(double),
                                          cudaMemcpyDeviceToDevice, st));
        }
        return launchAVswitches(a, k, s.box, s.minDt, st);
    case sMomentum: return launchMomentumEnergy(a, k, s.box, st);
    default: return kErrArg;
    }
}

TreeView treeView(sphb_sim& s)
{
    TreeView tv;
    tv.childOffsets = s.ftree.tree.childOffsets.data();
    tv.nodeToLeaf   = s.ftree.tree.nodeToLeaf.data();
    tv.centers      = s.ftree.tree.centers.data();
    tv.sizes        = s.ftree.tree.sizes.data();
    tv.layout       = s.ftree.layout.data();
    tv.blockLo      = s.blockLo.data();
    tv.blockHi      = s.blockHi.data();
    tv.numNodes     = s.ftree.tree.numNodes;
    tv.ext          = s.treeExt;
    return tv;
}

int allocateSkin(sphb_sim& s)
{
    if (s.skinRows.data()) { return kOk; }
    double grow = (1.0 + s.p.nb_skin) * (1.0 + s.p.nb_skin) * (1.0 + s.p.nb_skin);
    s.skinCap   = paddedNgmax(unsigned(std::ceil(s.p.ngmax * grow * 1.1)));
    size_t n = s.n;
    SPHB_TRY(s.skinRows.reserve(s.numGroups() * size_t(s.skinCap) * kWarp));
    SPHB_TRY(s.skinDist.reserve(s.numGroups() * size_t(s.skinCap) * kWarp));
    SPHB_TRY(s.skinCount.reserve(n));
    SPHB_TRY(s.skinRadius.reserve(n));
    SPHB_TRY(s.skinXb.reserve(n));
    SPHB_TRY(s.skinYb.reserve(n));
    SPHB_TRY(s.skinZb.reserve(n));
    SPHB_TRY(s.skinBuild.reserve(n));
    SPHB_TRY(s.skinBuildAlt.reserve(n));
    SPHB_TRY(s.skinMoved.reserve(s.numGroups()));
    SPHB_TRY(s.skinGrid.reserve(size_t(kSkinGrid) * kSkinGrid * kSkinGrid));
    SPHB_TRY(s.skinWork.reserve(2 * s.numGroups() + 2));
    SPHB_TRY(s.skinGroupD.reserve(s.numGroups()));
    // highest priority, so that the few long tree searches start before the refilter fills the GPU
    int leastPriority = 0, greatestPriority = 0;
    SPHB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority));
    SPHB_CUDA_TRY(cudaStreamCreateWithPriority(&s.sideStream, cudaStreamNonBlocking, greatestPriority));
    SPHB_CUDA_TRY(cudaEventCreateWithFlags(&s.skinFork, cudaEventDisableTiming));
    SPHB_CUDA_TRY(cudaEventCreateWithFlags(&s.skinJoin, cudaEventDisableTiming));
    return kOk;
}

/*! The neighbour stage: the tree search of every group (sph/include/sph/find_neighbors.hpp:10-41), or the exact
 *  refilter of the skin rows plus the tree search of the groups the rows cannot serve. Rows are rebuilt when more
 *  than a tenth of the groups were deferred in the previous step; rows that needed a rebuild within three steps
 *  (particles moving fast everywhere) are dropped for 32 steps of plain tree searches. Every path gives the same
 *  lists, counts and smoothing lengths. */
int searchNeighbors(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    TreeView tv     = treeView(s);
    NeighborParams np{s.p.ng0, s.p.ngmax, 10};
    s.skinFiltered = false;
    auto treeSearch = [&]() {
        ++s.searchStats[0];
        return findNeighbors(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.pos.data(), s.f[fH].data(), s.n, tv,
                             s.box, np, s.nidx.data(), s.nc.data(), s.status.data(), st);
    };

    SPHB_TRY(simimpl::resolveIdCheck(s));
    // a remap counts once the rows are known to be kept (a pending id comparison may drop them)
    if (s.syncRemapped && s.skinValid) { ++s.searchStats[4]; }
    s.syncRemapped = false;
    bool useSkin = s.p.nb_skin > 0.0 && !s.taping;
    if (!useSkin || s.skinHoldoff > 0)
    {
        if (s.skinHoldoff > 0) { --s.skinHoldoff; }
        s.skinValid = false;
        return treeSearch();
    }
    bool rebuild = !s.skinValid;
    if (!rebuild && size_t(s.skinDeferredLast) * 10 > s.numGroups())
    {
        if (s.skinAge <= 3)
        {
            s.skinHoldoff = 32;
            s.skinValid   = false;
            return treeSearch();
        }
        rebuild = true;
    }
    if (rebuild)
    {
        SPHB_TRY(allocateSkin(s));
        SPHB_TRY(treeSearch());
        SkinLists sl{s.skinRows.data(), s.skinCount.data(), s.skinRadius.data(), s.skinCap, s.skinDist.data()};
        SPHB_TRY(buildSkinLists(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.pos.data(), s.f[fH].data(), s.n, tv,
                                s.box, np, s.p.nb_skin, sl, s.status.data(), st));
        size_t bytes = s.n * sizeof(double);
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.skinXb.data(), s.f[fX].data(), bytes, cudaMemcpyDeviceToDevice, st));
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.skinYb.data(), s.f[fY].data(), bytes, cudaMemcpyDeviceToDevice, st));
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.skinZb.data(), s.f[fZ].data(), bytes, cudaMemcpyDeviceToDevice, st));
        s.skinValid        = true;
        s.skinAnyMoved     = false;
        s.skinAge          = 0;
        s.skinDeferredLast = 0;
        ++s.searchStats[1];
        return kOk;
    }

    ++s.skinAge;
    ++s.searchStats[2];
    s.skinFiltered = true;
    SPHB_CUDA_TRY(cudaMemsetAsync(s.skinGrid.data(), 0, size_t(kSkinGrid) * kSkinGrid * kSkinGrid * sizeof(unsigned),
                                  st));
    SPHB_CUDA_TRY(cudaMemsetAsync(s.skinWork.data(), 0, 2 * sizeof(unsigned), st));
    const uint32_t* buildOf = s.skinAnyMoved ? s.skinBuild.data() : nullptr;
    SPHB_TRY(skinDisplacement(s.pos.data(), s.skinXb.data(), s.skinYb.data(), s.skinZb.data(), buildOf, s.n, s.box,
                              s.skinGrid.data(), st));
    SkinFilterArgs a{};
    a.pos  = s.pos.data();
    a.posq = s.mixed ? s.posq.data() : nullptr;
    FixedFrame fr = fixedFrameOf(s.box);
    double unitMax = 0;
    for (int k = 0; k < 3; ++k)
    {
        a.qscale[k] = float(fr.unit[k]);
        unitMax     = std::max(unitMax, fr.unit[k]);
    }
    a.qunit        = float(unitMax * (1.0 + 1e-6));
    a.h            = s.f[fH].data();
    a.nc           = s.nc.data();
    a.nidx         = s.nidx.data();
    a.sl           = SkinLists{s.skinRows.data(), s.skinCount.data(), s.skinRadius.data(), s.skinCap,
                               s.skinDist.data()};
    a.xb           = s.skinXb.data();
    a.yb           = s.skinYb.data();
    a.zb           = s.skinZb.data();
    a.moved        = s.skinAnyMoved ? s.skinMoved.data() : nullptr;
    a.dispGrid     = s.skinGrid.data();
    a.groupD       = s.skinGroupD.data();
    a.numWorklist  = s.skinWork.data();
    a.numWorklist2 = s.skinWork.data() + 1;
    a.worklist     = s.skinWork.data() + 2;
    a.worklist2    = s.skinWork.data() + 2 + s.numGroups();
    a.n            = s.n;
    a.box          = s.box;
    a.prm          = np;
    SPHB_TRY(checkSkinGroups(a, st));
    // the tree search of the deferred groups runs on the side stream while the refilter serves the others (the two
    // write disjoint groups)
    SPHB_CUDA_TRY(cudaEventRecord(s.skinFork, st));
    SPHB_CUDA_TRY(cudaStreamWaitEvent(s.sideStream, s.skinFork, 0));
    SPHB_TRY(findNeighborsListed(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.pos.data(), s.f[fH].data(), s.n,
                                 tv, s.box, np, s.nidx.data(), s.nc.data(), s.status.data(), a.worklist,
                                 a.numWorklist, s.sideStream));
    SPHB_CUDA_TRY(cudaEventRecord(s.skinJoin, s.sideStream));
    SPHB_TRY(filterSkinLists(a, st));
    SPHB_CUDA_TRY(cudaStreamWaitEvent(st, s.skinJoin, 0));
    return findNeighborsListed(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.pos.data(), s.f[fH].data(), s.n, tv,
                               s.box, np, s.nidx.data(), s.nc.data(), s.status.data(), a.worklist2, a.numWorklist2,
                               st);
}

/*! One stage of HydroVeProp::computeForces (ve_hydro.hpp:126-203), in the reference's order: the domain sync, the
 *  neighbour search with the h iteration, XMass, VeDefGradh + EOS, IAD + divv/curlv, AV switches, MomentumEnergy, and
 *  the conserved sums with the time-step reductions (which complete the force computation). Each stage records the
 *  CUDA event that starts its stage time. */
int runStage(sphb_sim& s, int stage)
{
    cudaStream_t st = s.stream;
    // the sync (unless it reorders), the search and XMass read only x, y, z, h and m, VeDefGradh also temp, IAD and
    // the later J-loops also v and alpha; the force stages no x_m1, y_m1, z_m1 or du_m1
    if (stage > sXMass) { SPHB_TRY(simimpl::waitLateGroup(s, 0)); }
    if (stage > sVeDefGradh) { SPHB_TRY(simimpl::waitLateGroup(s, 1)); }
    if (stage >= sConserved) { SPHB_TRY(simimpl::waitLateFields(s)); }
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[stage], st));
    switch (stage)
    {
    case sSync: return syncDomain(s);
    case sNeighbors:
    {
        // h and the ids of a typed host load
        SPHB_TRY(simimpl::waitMidFields(s));
        if (s.taping)
        {
            SPHB_CUDA_TRY(cudaMemcpyAsync(s.hPre.data(), s.f[fH].data(), s.n * sizeof(double),
                                          cudaMemcpyDeviceToDevice, st));
        }
        SPHB_TRY(setWords(s.reduce.data(), 2, orderedBits(-INFINITY), orderedBits(INFINITY), st));
        SPHB_CUDA_TRY(cudaMemsetAsync(s.status.data(), 0, sizeof(unsigned), st));
        return searchNeighbors(s);
    }
    case sXMass:
    case sVeDefGradh:
    case sIad:
    case sAV:
    case sMomentum: return s.mixed ? runChainStage<float>(s, stage) : runChainStage<double>(s, stage);
    case sConserved: break;
    default: return kErrArg;
    }

    double cv = idealGasCv(s.p.mui, s.p.gamma);
    SPHB_TRY(conservedSums(s.n, s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.f[fVx].data(), s.f[fVy].data(),
                           s.f[fVz].data(), s.f[fM].data(), s.f[fTemp].data(), s.nc.data(), cv, s.partial.data(), 1024,
                           s.cons.data(), st));
    // hostMsg: [0, 9) the sums, [9, 11) the two reductions, [11] status, [12] the two deferred counts, [13] the h
    // update's flag under block time steps
    unsigned long long* msg = s.hostMsg;
    std::memset(msg + 11, 0, 2 * sizeof(unsigned long long));
    SPHB_CUDA_TRY(cudaMemcpyAsync(msg, s.cons.data(), 9 * sizeof(double), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(msg + 9, s.reduce.data(), 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                  st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(msg + 11, s.status.data(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    if (s.skinFiltered)
    {
        SPHB_CUDA_TRY(cudaMemcpyAsync(msg + 12, s.skinWork.data(), 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    }
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sIntegrate], st));
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    double cons[9];
    unsigned long long red[2];
    unsigned status, deferred[2];
    std::memcpy(cons, msg, sizeof(cons));
    std::memcpy(red, msg + 9, sizeof(red));
    std::memcpy(&status, msg + 11, sizeof(status));
    std::memcpy(deferred, msg + 12, sizeof(deferred));
    s.skinDeferredLast = deferred[0] + deferred[1];
    s.searchStats[3] += s.skinDeferredLast;
    if (status) { return kErrCapacity; }

    double maxDivv = fromOrderedBits(red[0]);
    s.minDtRho     = s.p.Krho / std::abs(maxDivv);
    s.minDtCourant = fromOrderedBits(red[1]);
    s.ecin         = 0.5 * cons[0];
    s.eint         = cons[1];
    s.etot         = s.ecin + s.eint;
    s.linmom       = std::sqrt(cons[2] * cons[2] + cons[3] * cons[3] + cons[4] * cons[4]);
    s.angmom       = std::sqrt(cons[5] * cons[5] + cons[6] * cons[6] + cons[7] * cons[7]);
    s.totalNeighbors = cons[8];
    s.forcesDone     = true;
    return kOk;
}

/*! The stage ABI's ordering rule: stage k runs only after stage k-1 of the same force computation (the sync after
 *  the previous integration, or at any time to start over). A failed stage leaves the computation to restart. */
int runStageChecked(sphb_sim& s, int stage)
{
    if (stage != sSync && stage != s.nextStage) { return kErrState; }
    s.forcesDone = false;
    s.nextStage  = sSync;
    int rc       = runStage(s, stage);
    if (rc != kOk) { return rc; }
    s.nextStage = stage == sConserved ? int(sSync) : stage + 1;
    return kOk;
}

int computeForces(sphb_sim& s)
{
    for (int stage = sSync; stage <= sConserved; ++stage)
    {
        SPHB_TRY(runStageChecked(s, stage));
    }
    return kOk;
}

template<class T>
int runPositions(sphb_sim& s, double cv)
{
    IntegrateArrays<T> a;
    a.x    = s.f[fX].data();
    a.y    = s.f[fY].data();
    a.z    = s.f[fZ].data();
    a.vx   = s.f[fVx].data();
    a.vy   = s.f[fVy].data();
    a.vz   = s.f[fVz].data();
    a.xm1  = s.f[fXm1].data();
    a.ym1  = s.f[fYm1].data();
    a.zm1  = s.f[fZm1].data();
    a.temp = s.f[fTemp].data();
    a.duM1 = s.f[fDuM1].data();
    a.du   = s.du.data();
    a.ax   = s.dptr<T>(dAx);
    a.ay   = s.dptr<T>(dAy);
    a.az   = s.dptr<T>(dAz);
    return launchPositions(s.n, a, s.box, s.minDt, s.minDt_m1, cv, s.stream);
}

//! HydroVeProp::integrate (ve_hydro.hpp:205-220): computeTimestep (ts_global.hpp:100-128), positions, h update
int integrateStep(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    double dtNew    = s.fixedDt > 0 ? s.fixedDt : std::min({s.minDtCourant, s.minDtRho, 1.1 * s.minDt});
    s.ttot += dtNew;
    s.minDt_m1 = s.minDt;
    s.minDt    = dtNew;

    double cv = idealGasCv(s.p.mui, s.p.gamma);
    if (s.mixed) { SPHB_TRY(runPositions<float>(s, cv)); }
    else { SPHB_TRY(runPositions<double>(s, cv)); }
    SPHB_CUDA_TRY(cudaMemsetAsync(s.status.data() + 1, 0, sizeof(unsigned), st));
    SPHB_TRY(launchUpdateH(s.n, s.p.ng0, s.nc.data(), s.f[fH].data(), s.keys.data(), s.status.data() + 1, st));
    unsigned flag = 0;
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[kNumStages], st));
    SPHB_TRY(readBack(st, {{&flag, s.status.data() + 1, sizeof(unsigned)}}));
    for (int k = 0; k < kNumStages; ++k)
    {
        cudaEventElapsedTime(&s.stageMs[k], s.ev[k], s.ev[k + 1]);
    }
    s.iteration++;
    s.forcesDone = false;
    return flag ? kErrNotConverged : kOk;
}

// ---------------------------------------------------------------------------------------------------------------
// Block time steps: HydroVeBdtProp (main/src/propagator/ve_hydro_bdt.hpp:165-380) over fixed groups of 32
// SFC-consecutive particles, with the rung logic of sph/include/sph/ts_rungs.hpp.
// ---------------------------------------------------------------------------------------------------------------

//! cstone::butterfly (cstone/primitives/math.hpp:35-40): 0, then 1 + trailing zeros
int butterflyOf(uint32_t i) { return i == 0 ? 0 : 1 + __builtin_ctz(i); }

//! HydroVeBdtProp::activeRung (ve_hydro_bdt.hpp:109-113): the rungs below it are active at this substep
int activeRungOf(int substep, int numRungs)
{
    if (substep == 0 || substep >= (1 << (numRungs - 1))) { return 0; }
    return butterflyOf(uint32_t(substep));
}

int allocateBdt(sphb_sim& s)
{
    size_t G = s.numGroups();
    SPHB_TRY(s.rung.reserve(s.n));
    SPHB_TRY(s.rungAlt.reserve(s.n));
    SPHB_TRY(s.groupDt.reserve(G));
    SPHB_TRY(s.groupIdx.reserve(G));
    SPHB_TRY(s.grpSfc.reserve(G));
    SPHB_TRY(s.grpTs.reserve(G));
    SPHB_TRY(s.dtKeys.reserve(G));
    SPHB_TRY(s.rungInfo.reserve(8));
    SPHB_TRY(s.xs.reserve(s.n));
    SPHB_TRY(s.ys.reserve(s.n));
    SPHB_TRY(s.zs.reserve(s.n));
    SPHB_TRY(s.dispMax.reserve(1));
    return kOk;
}

//! the propagator's state after construction: one rung, dt_m1[0] = minDt (ve_hydro_bdt.hpp:116-130), rungs 0
int resetBdt(sphb_sim& s)
{
    s.bts       = sphb_sim::BdtTimestep{};
    s.bts.dtm1[0] = float(s.minDt);
    s.bprevTs   = s.bts;
    s.treeExt   = 0.0;
    s.activeList = nullptr;
    s.numActive  = 0;
    SPHB_CUDA_TRY(cudaMemsetAsync(s.rung.data(), 0, s.n * sizeof(uint64_t), s.stream));
    return kOk;
}

//! fullSync / partialSync (ve_hydro_bdt.hpp:165-215)
int bdtSync(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    if (activeRungOf(s.bts.substep, s.bts.numRungs) == 0)
    {
        SPHB_TRY(syncDomain(s));
        // computeGroups -> computeSpatialGroups (sph/include/sph/groups.hpp:41-74; ve_hydro_bdt.hpp:185): the spatial
        // target groups of 32 from the focus tree of this sync, tolFactor 2
        unsigned G = 0;
        SPHB_TRY(computeGroupSplits(0, s.n, s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.f[fH].data(), SPHB_F64,
                                    s.ftree.leaves.data(), s.ftree.numLeaves,
                                    reinterpret_cast<const uint32_t*>(s.ftree.layout.data()), s.box, kWarp, 2.0f,
                                    s.grpScratch, s.grpBounds, &G, st));
        s.numBdtGroups = G;
        SPHB_TRY(s.groupDt.reserve(G));
        SPHB_TRY(s.groupIdx.reserve(G));
        SPHB_TRY(s.grpSfc.reserve(G));
        SPHB_TRY(s.grpTs.reserve(G));
        SPHB_TRY(s.dtKeys.reserve(G));
        SPHB_TRY(launchSequence(s.grpSfc.data(), G, 0, st));
        s.activeList = s.grpSfc.data();
        s.numActive  = G;
        std::vector<float> big(G, std::numeric_limits<float>::max());
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.groupDt.data(), big.data(), G * sizeof(float), cudaMemcpyHostToDevice, st));
        size_t bytes = s.n * sizeof(double);
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.xs.data(), s.f[fX].data(), bytes, cudaMemcpyDeviceToDevice, st));
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.ys.data(), s.f[fY].data(), bytes, cudaMemcpyDeviceToDevice, st));
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.zs.data(), s.f[fZ].data(), bytes, cudaMemcpyDeviceToDevice, st));
        SPHB_CUDA_TRY(cudaStreamSynchronize(st)); // the host vector above
        s.treeExt = 0.0;
        return kOk;
    }
    // partial sync: no resort, so the groups keep their particles; the packed positions and the block boxes follow
    // the drifted particles, and the tree's node boxes are widened by the largest drift since the full sync (the
    // reference widens its search by 1.2 % per substep instead, ve_hydro_bdt.hpp:201-203)
    SPHB_TRY(packPositionsAndBoxes(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.f[fM].data(), s.n,
                                   s.pos.data(), s.mixed ? s.posq.data() : nullptr, s.box, s.blockLo.data(),
                                   s.blockHi.data(), st));
    unsigned long long dmax = 0;
    SPHB_TRY(setWords(s.dispMax.data(), 1, orderedBits(0.0), 0, st));
    SPHB_TRY(launchMaxDisplacement(s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.xs.data(), s.ys.data(),
                                   s.zs.data(), s.n, s.box, s.dispMax.data(), st));
    SPHB_TRY(readBack(st, {{&dmax, s.dispMax.data(), sizeof(dmax)}}));
    double lenMax = std::max({s.box.len[0], s.box.len[1], s.box.len[2]});
    s.treeExt     = fromOrderedBits(dmax) * (1.0 + 1e-9) + 1e-14 * lenMax;
    int highest   = butterflyOf(uint32_t(s.bts.substep));
    s.activeList  = s.grpTs.data() + s.bts.rungRanges[0];
    s.numActive   = s.bts.rungRanges[highest] - s.bts.rungRanges[0];
    return kOk;
}

//! computeForces of the block time-step propagator on the active groups (ve_hydro_bdt.hpp:224-296)
template<class T>
int bdtChain(sphb_sim& s)
{
    cudaStream_t st  = s.stream;
    ChainArrays<T> a = chainArrays<T>(s);
    HydroConsts<T> k = hydroConsts<T>(s);
    ChainArrays<T> l = a;
    l.groupList      = s.activeList;
    l.groupBounds    = s.grpBounds.data();
    l.numListed      = s.numActive;
    l.groupDt        = s.groupDt.data();
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sXMass], st));
    l.threads = chainThreads(s.mixed, sXMass);
    SPHB_TRY(launchXMass(l, k, s.box, st));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sVeDefGradh], st));
    l.threads = chainThreads(s.mixed, sVeDefGradh);
    SPHB_TRY(launchVeDefGradhEos(l, k, s.box, st));
    SPHB_TRY(launchEosRefresh(a, k, st));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sIad], st));
    l.threads = chainThreads(s.mixed, sIad);
    SPHB_TRY(launchIadDivvCurlv(l, k, s.box, st));
    SPHB_TRY(launchGroupDivv(s.activeList, s.numActive, s.grpBounds.data(), a.divv, float(s.p.Krho),
                             s.groupDt.data(), st));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sAV], st));
    l.threads = chainThreads(s.mixed, sAV);
    SPHB_TRY(launchAVswitches(l, k, s.box, s.minDt, st));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sMomentum], st));
    l.threads = chainThreads(s.mixed, sMomentum);
    SPHB_TRY(launchMomentumEnergy(l, k, s.box, st));
    return launchGroupAcc(s.activeList, s.numActive, s.grpBounds.data(), a.ax, a.ay, a.az, s.f[fH].data(), s.etaAcc,
                          s.groupDt.data(), st);
}

/*! Stage events as the global step records them (sphb_sim_stage_times): sync, neighbours, the five J-loops (with
 *  the EOS of every particle in VeDefGradh and the group time steps in IAD and MomentumEnergy), conserved sums, and
 *  the integration with the rung sort. */
int bdtComputeForces(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sSync], st));
    SPHB_TRY(bdtSync(s));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sNeighbors], st));
    SPHB_TRY(setWords(s.reduce.data(), 2, orderedBits(-INFINITY), orderedBits(INFINITY), st));
    SPHB_CUDA_TRY(cudaMemsetAsync(s.status.data(), 0, sizeof(unsigned), st));
    SPHB_TRY(searchNeighbors(s));
    SPHB_TRY(s.mixed ? bdtChain<float>(s) : bdtChain<double>(s));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sConserved], st));
    double cv = idealGasCv(s.p.mui, s.p.gamma);
    SPHB_TRY(conservedSums(s.n, s.f[fX].data(), s.f[fY].data(), s.f[fZ].data(), s.f[fVx].data(), s.f[fVy].data(),
                           s.f[fVz].data(), s.f[fM].data(), s.f[fTemp].data(), s.nc.data(), cv, s.partial.data(), 1024,
                           s.cons.data(), st));
    // the sums and the status word through the pinned block, one wait
    unsigned long long* msg = s.hostMsg;
    msg[11]                 = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(msg, s.cons.data(), 9 * sizeof(double), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaMemcpyAsync(msg + 11, s.status.data(), sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[sIntegrate], st));
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    double cons[9];
    unsigned status;
    std::memcpy(cons, msg, sizeof(cons));
    std::memcpy(&status, msg + 11, sizeof(status));
    if (status) { return kErrCapacity; }
    s.ecin           = 0.5 * cons[0];
    s.eint           = cons[1];
    s.etot           = s.ecin + s.eint;
    s.linmom         = std::sqrt(cons[2] * cons[2] + cons[3] * cons[3] + cons[4] * cons[4]);
    s.angmom         = std::sqrt(cons[5] * cons[5] + cons[6] * cons[6] + cons[7] * cons[7]);
    s.totalNeighbors = cons[8];
    return kOk;
}

/*! computeMinTimestep + findRungRanges (ts_rungs.hpp:84-146) on groupDt[0, num): sorts it (and groupIdx[0, num),
 *  the permutation) and returns the smallest dt, the dt at index 0.4 num, and the lower bounds of 2^r min dt */
int sortGroupDt(sphb_sim& s, unsigned num, float* minDt, float* fastDt, uint32_t lb[kMaxRungs])
{
    cudaStream_t st = s.stream;
    SPHB_TRY(launchDtKeys(s.groupDt.data(), num, s.dtKeys.data(), s.groupIdx.data(), st));
    SPHB_TRY(sortByKeyAsync(s.dtKeys.data(), s.groupIdx.data(), num, false, s.sortScratch.data(),
                            s.sortScratch.capacity(), 0x0fu, s.status.data() + 2, st));
    unsigned fastIdx = unsigned(0.4f * float(num)); // LocalIndex(fastFraction * numGroups), ts_rungs.hpp:86,102
    SPHB_TRY(launchSortedDt(s.dtKeys.data(), num, fastIdx, s.groupDt.data(), s.rungInfo.data(), st));
    uint32_t info[1 + kMaxRungs];
    unsigned err = 0;
    SPHB_TRY(readBack(st, {{info, s.rungInfo.data(), sizeof(info)}, {&err, s.status.data() + 2, sizeof(err)}}));
    if (err) { return kErrCuda; }
    std::memcpy(minDt, &info[0], sizeof(float));
    std::memcpy(fastDt, &info[1], sizeof(float));
    lb[0] = 0;
    for (int r = 1; r < kMaxRungs; ++r)
    {
        lb[r] = info[1 + r];
    }
    return kOk;
}

//! computeRungs (ve_hydro_bdt.hpp:299-334) with rungTimestep / minimumGroupDt (ts_rungs.hpp:148-166)
int bdtComputeRungs(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    unsigned G      = s.numBdtGroups;
    int highRung    = activeRungOf(s.bts.substep, s.bts.numRungs);
    SPHB_CUDA_TRY(cudaMemsetAsync(s.status.data() + 2, 0, sizeof(unsigned), st));
    if (highRung == 0)
    {
        s.bprevTs   = s.bts;
        float maxDt = float(double(s.bts.dtm1[0]) * 1.1); // maxDtIncrease (particles_data.hpp:138)
        float minDt, fastDt;
        uint32_t lb[kMaxRungs];
        SPHB_TRY(sortGroupDt(s, G, &minDt, &fastDt, lb));
        int numRungs = std::min(int(std::log2(fastDt / minDt)) + 1, kMaxRungs);
        sphb_sim::BdtTimestep t{};
        t.rungRanges[0] = 0;
        for (int r = 1; r <= kMaxRungs; ++r)
        {
            t.rungRanges[r] = r < numRungs ? lb[r] : G;
        }
        minDt      = std::min(maxDt, minDt);
        t.nextDt   = minDt;
        t.totDt    = minDt * float(1 << numRungs);
        t.numRungs = numRungs;
        s.bts      = t;
    }
    else
    {
        unsigned numActive = s.bts.rungRanges[highRung];
        unsigned numTot    = s.bts.rungRanges[kMaxRungs];
        float minDt, fastDt;
        uint32_t lb[kMaxRungs];
        SPHB_TRY(sortGroupDt(s, numActive, &minDt, &fastDt, lb));
        SPHB_TRY(launchSequence(s.groupIdx.data() + numActive, numTot - numActive, numActive, st));
        float timeLeft   = s.bts.totDt - s.bts.elapsedDt;
        int substepsLeft = (1 << s.bts.numRungs) - s.bts.substep;
        s.bts.nextDt      = std::min(minDt, timeLeft / float(substepsLeft));
        for (int r = 1; r < highRung; ++r)
        {
            s.bts.rungRanges[r] = lb[r];
        }
        s.bts.rungRanges[0] = 0;
    }
    if (highRung == 0 || highRung > 1)
    {
        if (highRung > 1) { s.grpSfc.swap(s.grpTs); }
        SPHB_TRY(launchGatherGroups(s.grpSfc.data(), s.groupIdx.data(), s.bts.rungRanges[kMaxRungs], s.grpTs.data(),
                                    st));
    }
    return kOk;
}

template<class T>
IntegrateArrays<T> integrateArrays(sphb_sim& s)
{
    IntegrateArrays<T> a;
    a.x    = s.f[fX].data();
    a.y    = s.f[fY].data();
    a.z    = s.f[fZ].data();
    a.vx   = s.f[fVx].data();
    a.vy   = s.f[fVy].data();
    a.vz   = s.f[fVz].data();
    a.xm1  = s.f[fXm1].data();
    a.ym1  = s.f[fYm1].data();
    a.zm1  = s.f[fZm1].data();
    a.temp = s.f[fTemp].data();
    a.duM1 = s.f[fDuM1].data();
    a.du   = s.du.data();
    a.ax   = s.dptr<T>(dAx);
    a.ay   = s.dptr<T>(dAy);
    a.az   = s.dptr<T>(dAz);
    return a;
}

//! integrate of the block time-step propagator (ve_hydro_bdt.hpp:336-380)
template<class T>
int bdtIntegrateRungs(sphb_sim& s)
{
    cudaStream_t st          = s.stream;
    IntegrateArrays<T> a     = integrateArrays<T>(s);
    double cv                = idealGasCv(s.p.mui, s.p.gamma);
    int lowestDriftRung      = butterflyOf(uint32_t(s.bts.substep + 1));
    bool isLastSubstep       = activeRungOf(s.bts.substep + 1, s.bts.numRungs) == 0;
    DevBox box               = s.box;
    if (!isLastSubstep) { box.periodic[0] = box.periodic[1] = box.periodic[2] = 0; }
    for (int i = 0; i < s.bts.numRungs; ++i)
    {
        bool useRung = s.bts.substep == s.bts.substep % (1 << i); // drift back to the start of the hierarchy
        bool advance = i < lowestDriftRung;
        float dt     = s.bts.nextDt;
        RungSteps steps;
        std::memcpy(steps.dtm1, useRung ? s.bprevTs.dtm1 : s.bts.dtm1, sizeof(steps.dtm1));
        const uint32_t* list = s.grpTs.data() + s.bts.rungRanges[i];
        unsigned num         = s.bts.rungRanges[i + 1] - s.bts.rungRanges[i];
        if (advance)
        {
            if (s.bts.dtDrift[i] > 0)
            {
                SPHB_TRY(launchDrift(list, num, s.grpBounds.data(), 0.f, s.bts.dtDrift[i], steps, s.rung.data(), a, cv, st));
            }
            SPHB_TRY(launchRungPositions(list, num, s.grpBounds.data(), s.bts.dtDrift[i] + dt, steps, s.rung.data(), a, box, cv,
                                         st));
            s.bts.dtm1[i]    = s.bts.dtDrift[i] + dt;
            s.bts.dtDrift[i] = 0;
            SPHB_TRY(launchStoreRung(list, num, s.grpBounds.data(), uint64_t(i), s.rung.data(), st));
        }
        else
        {
            SPHB_TRY(launchDrift(list, num, s.grpBounds.data(), s.bts.dtDrift[i] + dt, s.bts.dtDrift[i], steps, s.rung.data(), a, cv,
                                 st));
            s.bts.dtDrift[i] += dt;
        }
    }
    return kOk;
}

int bdtIntegrate(sphb_sim& s)
{
    cudaStream_t st = s.stream;
    SPHB_TRY(bdtComputeRungs(s));
    SPHB_TRY(s.mixed ? bdtIntegrateRungs<float>(s) : bdtIntegrateRungs<double>(s));
    SPHB_CUDA_TRY(cudaMemsetAsync(s.status.data() + 1, 0, sizeof(unsigned), st));
    SPHB_TRY(launchListUpdateH(s.activeList, s.numActive, s.grpBounds.data(), s.p.ng0, s.nc.data(), s.f[fH].data(), s.keys.data(),
                               s.status.data() + 1, st));
    s.hostMsg[13] = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(s.hostMsg + 13, s.status.data() + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    SPHB_CUDA_TRY(cudaEventRecord(s.ev[kNumStages], st));
    SPHB_CUDA_TRY(cudaStreamSynchronize(st));
    unsigned flag;
    std::memcpy(&flag, s.hostMsg + 13, sizeof(flag));
    for (int k = 0; k < kNumStages; ++k)
    {
        cudaEventElapsedTime(&s.stageMs[k], s.ev[k], s.ev[k + 1]);
    }
    s.bts.substep++;
    s.bts.elapsedDt += s.bts.nextDt;
    s.ttot += double(s.bts.nextDt);
    s.minDt_m1 = s.minDt;
    s.minDt    = double(s.bts.nextDt);
    s.iteration++;
    return flag ? kErrNotConverged : kOk;
}

int allocateAdjoint(sphb_sim& s)
{
    size_t n = s.n;
    SPHB_TRY(s.hPre.reserve(n));
    SPHB_TRY(s.alphaPre.reserve(n));
    SPHB_TRY(s.tapeT.reserve(8 * n * s.elemBytes()));
    SPHB_TRY(s.tapeJ.reserve(n));
    SPHB_TRY(s.adjT.reserve(size_t(kNumAdjFields) * n * s.elemBytes()));
    if (s.mixed) { SPHB_TRY(s.adjJacc.reserve(5 * n)); }
    SPHB_TRY(s.adjWork.reserve(14 * n));
    SPHB_TRY(s.adjScalar.reserve(1));
    return kOk;
}

//! the device buffers a step adjoint reads after the taped force computation (pointer, bytes)
std::vector<std::pair<void*, size_t>> tapedBuffers(sphb_sim& s)
{
    size_t n = s.n, e = s.elemBytes();
    std::vector<std::pair<void*, size_t>> b;
    for (int k = 0; k < kNumConserved; ++k)
    {
        b.push_back({s.f[k].data(), n * sizeof(double)});
    }
    b.push_back({s.order.data(), n * sizeof(uint32_t)});
    b.push_back({s.pos.data(), n * sizeof(double4)});
    if (s.mixed) { b.push_back({s.posq.data(), n * sizeof(int4)}); }
    b.push_back({s.nidx.data(), s.numGroups() * size_t(paddedNgmax(s.p.ngmax)) * kWarp * sizeof(uint32_t)});
    b.push_back({s.nc.data(), n * sizeof(unsigned)});
    for (int d = 0; d < kNumDerived; ++d)
    {
        b.push_back({s.derived[d].data(), n * e});
    }
    b.push_back({s.du.data(), n * sizeof(double)});
    b.push_back({s.hrec.data(), n * 8 * e});
    b.push_back({s.grec.data(), n * 8 * e});
    b.push_back({s.avrec.data(), n * 8 * e});
    b.push_back({s.tapeT.data(), 8 * n * e});
    b.push_back({s.tapeJ.data(), n * sizeof(int)});
    b.push_back({s.hPre.data(), n * sizeof(double)});
    b.push_back({s.alphaPre.data(), n * sizeof(double)});
    return b;
}

size_t alignTape(size_t x) { return (x + 255) / 256 * 256; }

//! copy the taped buffers into slot (save) or back from it
int copyTape(sphb_sim& s, int slot, bool save)
{
    char* base = s.tapeSlots.data() + size_t(slot) * s.tapeSlotBytes;
    size_t off = 0;
    for (auto [ptr, bytes] : tapedBuffers(s))
    {
        void* dst = save ? static_cast<void*>(base + off) : ptr;
        void* src = save ? ptr : static_cast<void*>(base + off);
        SPHB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s.stream));
        off += alignTape(bytes);
    }
    return kOk;
}

template<class T>
int runStepVjp(sphb_sim& s, const double* const* post, double* const* pre, double* alphamaxBar)
{
    ChainArrays<T> a = chainArrays<T>(s);
    HydroConsts<T> k = hydroConsts<T>(s);
    if (!a.tape.whomega || !a.tape.energy || !a.tape.vsigJ) { return SPHB_ERR_STATE; }
    AdjointStepArgs args;
    args.n           = s.n;
    args.dt          = s.fixedDt;
    args.dtm1        = s.fixedDt;
    args.cv          = idealGasCv(s.p.mui, s.p.gamma);
    args.gamma       = s.p.gamma;
    args.ng0         = s.p.ng0;
    args.order       = s.order.data();
    args.hPre        = s.hPre.data();
    args.alphaPre    = s.alphaPre.data();
    args.temp        = s.f[fTemp].data();
    args.xm1         = s.f[fXm1].data();
    args.ym1         = s.f[fYm1].data();
    args.zm1         = s.f[fZm1].data();
    args.duM1        = s.f[fDuM1].data();
    args.du          = s.du.data();
    args.dtAV        = s.minDt;
    args.alphamaxBar = s.adjScalar.data();

    StateAdj postA, preA, work;
    for (int f = 0; f < kNumConserved; ++f)
    {
        postA.f[f] = const_cast<double*>(post[f]);
        preA.f[f]  = pre[f];
        work.f[f]  = s.adjWork.data() + size_t(f) * s.n;
    }
    AdjArrays<T> g;
    T* base = reinterpret_cast<T*>(s.adjT.data());
    T** slots[kNumAdjFields] = {&g.x,      &g.y,      &g.z,      &g.vx,     &g.vy,     &g.vz,      &g.h,
                                &g.c,      &g.prho,   &g.alpha,  &g.cij[0], &g.cij[1], &g.cij[2],  &g.cij[3],
                                &g.cij[4], &g.cij[5], &g.divv,   &g.xm,     &g.vol,    &g.kx,      &g.gradh,
                                &g.ax,     &g.ay,     &g.az,     &g.du};
    for (int q = 0; q < kNumAdjFields; ++q)
    {
        *slots[q] = base + size_t(q) * s.n;
    }
    if constexpr (sizeof(T) == 4) { g.jacc = s.adjJacc.data(); }
    SPHB_CUDA_TRY(cudaMemsetAsync(s.adjScalar.data(), 0, sizeof(double), s.stream));
    SPHB_TRY(stepVjp<T>(a, k, s.box, args, postA, preA, g, work, s.stream));
    double amB = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&amB, s.adjScalar.data(), sizeof(double), cudaMemcpyDeviceToHost, s.stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s.stream));
    if (alphamaxBar) { *alphamaxBar += amB; }
    return kOk;
}

} // namespace

// -------------------------------------------------------------------------------------------------------------------
// C ABI
// -------------------------------------------------------------------------------------------------------------------

extern "C" void sphb_default_params(sphb_params* p)
{
    if (!p) { return; }
    p->ng0            = 100;
    p->ngmax          = 150;
    p->gamma          = 5.0 / 3.0;
    p->mui            = 10.0;
    p->Kcour          = 0.2;
    p->Krho           = 0.06;
    p->alphamin       = 0.05;
    p->alphamax       = 1.0;
    p->decay_constant = 0.2;
    p->sinc_index     = 6.0;
    p->minDt          = 1e-12;
    p->minDt_m1       = 1e-12;
    p->precision      = SPHB_FP64;
    p->bucket_focus   = 64;
    p->av_clean       = 0;
    p->nb_skin        = 0.05;
}

extern "C" const char* sphb_version(void) { return "sphb200 0.1 (sm_100a)"; }

extern "C" int sphb_sim_create(sphb_sim** out, size_t n, const sphb_box* box, const sphb_params* params)
{
    if (!out || !box || !params || n == 0 || n >= (size_t(1) << 30)) { return SPHB_ERR_ARG; }
    if (params->ng0 > params->ngmax || params->ngmax == 0 || params->bucket_focus == 0) { return SPHB_ERR_ARG; }
    if (params->precision != SPHB_FP64 && params->precision != SPHB_MIXED) { return SPHB_ERR_ARG; }
    if (!(params->nb_skin >= 0.0 && params->nb_skin <= 1.0)) { return SPHB_ERR_ARG; }
    for (int k = 0; k < 3; ++k)
    {
        if (!(box->hi[k] > box->lo[k])) { return SPHB_ERR_ARG; }
    }
    auto* s     = new sphb_sim;
    s->n        = n;
    s->p        = *params;
    s->hbox     = *box;
    s->box      = makeDevBox(*box);
    s->mixed    = params->precision == SPHB_MIXED;
    s->minDt    = params->minDt;
    s->minDt_m1 = params->minDt_m1;
    int rc      = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess ? kOk : kErrCuda;
    // the copy stream and its events of the typed host loads and sphb_sim_step_fields
    int leastPriority = 0, greatestPriority = 0;
    if (rc == kOk && cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority) != cudaSuccess)
    {
        rc = kErrCuda;
    }
    if (rc == kOk &&
        cudaStreamCreateWithPriority(&s->copyStream, cudaStreamNonBlocking, greatestPriority) != cudaSuccess)
    {
        rc = kErrCuda;
    }
    if (rc == kOk && cudaEventCreateWithFlags(&s->copyFork, cudaEventDisableTiming) != cudaSuccess) { rc = kErrCuda; }
    for (auto& e : s->lateReady)
    {
        if (rc == kOk && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) { rc = kErrCuda; }
    }
    if (rc == kOk && cudaEventCreateWithFlags(&s->midReady, cudaEventDisableTiming) != cudaSuccess) { rc = kErrCuda; }
    if (rc == kOk && cudaEventCreateWithFlags(&s->idCheckDone, cudaEventDisableTiming) != cudaSuccess)
    {
        rc = kErrCuda;
    }
    if (rc == kOk) { rc = allocateSim(*s); }
    if (rc != kOk)
    {
        sphb_sim_destroy(s);
        return rc;
    }
    *out = s;
    return SPHB_OK;
}

extern "C" int sphb_sim_destroy(sphb_sim* s)
{
    if (!s) { return SPHB_ERR_ARG; }
    if (s->stream) { cudaStreamSynchronize(s->stream); }
    for (auto& e : s->ev)
    {
        if (e) { cudaEventDestroy(e); }
    }
    if (s->stream) { cudaStreamDestroy(s->stream); }
    if (s->sideStream)
    {
        cudaStreamSynchronize(s->sideStream);
        cudaStreamDestroy(s->sideStream);
    }
    if (s->copyStream)
    {
        cudaStreamSynchronize(s->copyStream);
        cudaStreamDestroy(s->copyStream);
    }
    if (s->copyFork) { cudaEventDestroy(s->copyFork); }
    for (auto& e : s->lateReady)
    {
        if (e) { cudaEventDestroy(e); }
    }
    if (s->midReady) { cudaEventDestroy(s->midReady); }
    if (s->idCheckDone) { cudaEventDestroy(s->idCheckDone); }
    if (s->skinFork) { cudaEventDestroy(s->skinFork); }
    if (s->skinJoin) { cudaEventDestroy(s->skinJoin); }
    if (s->hostMsg) { cudaFreeHost(s->hostMsg); }
    delete s;
    return SPHB_OK;
}

extern "C" int sphb_sim_upload(sphb_sim* s, const double* const* fields, const uint64_t* id, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !fields || !id) { return SPHB_ERR_ARG; }
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int k = 0; k < kNumConserved; ++k)
    {
        if (!fields[k]) { return SPHB_ERR_ARG; }
        SPHB_CUDA_TRY(cudaMemcpyAsync(s->f[k].data(), fields[k], s->n * sizeof(double), kind, s->stream));
    }
    SPHB_CUDA_TRY(cudaMemcpyAsync(s->id.data(), id, s->n * sizeof(uint64_t), kind, s->stream));
    return simimpl::finishUpload(*s);
}

extern "C" int sphb_sim_initial_sync(sphb_sim* s)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s) { return SPHB_ERR_ARG; }
    if (!s->uploaded) { return SPHB_ERR_STATE; }
    s->skinValid = false;
    SPHB_TRY(syncDomain(*s));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_sim_compute_forces(sphb_sim* s)
{
    // no wait here: the stages wait for a typed load's late fields where they first read them, and the conserved
    // stage returns to the host after that
    if (!s) { return SPHB_ERR_ARG; }
    if (!s->uploaded || s->bdt) { return SPHB_ERR_STATE; }
    return computeForces(*s);
}

extern "C" int sphb_sim_integrate(sphb_sim* s)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s) { return SPHB_ERR_ARG; }
    if (!s->forcesDone) { return SPHB_ERR_STATE; }
    return integrateStep(*s);
}

extern "C" int sphb_sim_step(sphb_sim* s)
{
    int rc = sphb_sim_compute_forces(s);
    if (rc != SPHB_OK) { return rc; }
    return sphb_sim_integrate(s);
}

extern "C" int sphb_sim_bdt_enable(sphb_sim* s, double eta_acc)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !(eta_acc > 0.0)) { return SPHB_ERR_ARG; }
    if (s->taping) { return SPHB_ERR_ARG; } // the adjoint has no block time-step variant
    SPHB_TRY(allocateBdt(*s));
    s->bdt    = true;
    s->etaAcc = float(eta_acc);
    s->skinValid = false;
    SPHB_TRY(resetBdt(*s));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_sim_bdt_step(sphb_sim* s)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s) { return SPHB_ERR_ARG; }
    if (!s->uploaded || !s->bdt) { return SPHB_ERR_STATE; }
    SPHB_TRY(bdtComputeForces(*s));
    return bdtIntegrate(*s);
}

extern "C" int sphb_sim_bdt_timestep(const sphb_sim* s, sphb_bdt_timestep* out)
{
    if (!s || !out) { return SPHB_ERR_ARG; }
    if (!s->bdt) { return SPHB_ERR_STATE; }
    out->next_dt    = s->bts.nextDt;
    out->elapsed_dt = s->bts.elapsedDt;
    out->total_dt   = s->bts.totDt;
    out->num_rungs  = s->bts.numRungs;
    out->substep    = s->bts.substep;
    for (int r = 0; r <= kMaxRungs; ++r)
    {
        out->rung_ranges[r] = s->bts.rungRanges[r];
    }
    for (int r = 0; r < kMaxRungs; ++r)
    {
        out->dt_m1[r]    = s->bts.dtm1[r];
        out->dt_drift[r] = s->bts.dtDrift[r];
    }
    out->num_active = s->numActive;
    return SPHB_OK;
}

namespace
{

int stageEntry(sphb_sim* s, int stage)
{
    if (!s) { return SPHB_ERR_ARG; }
    if (s->bdt) { return SPHB_ERR_STATE; }
    if (!s->uploaded) { return SPHB_ERR_STATE; }
    return runStageChecked(*s, stage);
}

} // namespace

extern "C" int sphb_sim_sync(sphb_sim* s) { return stageEntry(s, sSync); }
extern "C" int sphb_sim_find_neighbors(sphb_sim* s) { return stageEntry(s, sNeighbors); }
extern "C" int sphb_sim_xmass(sphb_sim* s) { return stageEntry(s, sXMass); }
extern "C" int sphb_sim_ve_def_gradh_eos(sphb_sim* s) { return stageEntry(s, sVeDefGradh); }
extern "C" int sphb_sim_iad_divv_curlv(sphb_sim* s) { return stageEntry(s, sIad); }
extern "C" int sphb_sim_av_switches(sphb_sim* s) { return stageEntry(s, sAV); }

extern "C" int sphb_sim_momentum_energy(sphb_sim* s, double* min_dt_courant)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    int rc = stageEntry(s, sMomentum);
    if (rc != SPHB_OK || !min_dt_courant) { return rc; }
    unsigned long long bits = 0;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&bits, s->reduce.data() + 1, sizeof(bits), cudaMemcpyDeviceToHost, s->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    *min_dt_courant = fromOrderedBits(bits);
    return SPHB_OK;
}

extern "C" int sphb_sim_conserved(sphb_sim* s, double* out)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    int rc = stageEntry(s, sConserved);
    if (rc != SPHB_OK || !out) { return rc; }
    double v[5] = {s->ecin, s->eint, s->etot, s->linmom, s->angmom};
    std::memcpy(out, v, sizeof(v));
    return SPHB_OK;
}

extern "C" size_t sphb_sim_size(const sphb_sim* s) { return s ? s->n : 0; }

namespace
{

//! locate a field by name: returns device pointer and element kind (0 double, 1 T, 2 uint32, 3 uint64)
bool findField(sphb_sim* s, const char* name, void** ptr, int* kind)
{
    for (int k = 0; k < kNumConserved; ++k)
    {
        if (std::strcmp(name, kConservedNames[k]) == 0)
        {
            *ptr  = s->f[k].data();
            *kind = 0;
            return true;
        }
    }
    for (int d = 0; d < kNumDerived; ++d)
    {
        if (std::strcmp(name, kDerivedNames[d]) == 0)
        {
            *ptr  = s->derived[d].data();
            *kind = 1;
            return true;
        }
    }
    if (std::strcmp(name, "du") == 0)
    {
        *ptr  = s->du.data();
        *kind = 0;
        return true;
    }
    static const char* const dvNames[6] = {"dV11", "dV12", "dV13", "dV22", "dV23", "dV33"};
    for (int q = 0; q < 6 && s->p.av_clean; ++q)
    {
        if (std::strcmp(name, dvNames[q]) == 0)
        {
            *ptr  = s->dv.data() + size_t(q) * s->n * s->elemBytes();
            *kind = 1;
            return true;
        }
    }
    if (std::strcmp(name, "nc") == 0)
    {
        *ptr  = s->nc.data();
        *kind = 2;
        return true;
    }
    if (std::strcmp(name, "keys") == 0)
    {
        *ptr  = s->keys.data();
        *kind = 3;
        return true;
    }
    if (std::strcmp(name, "id") == 0)
    {
        *ptr  = s->id.data();
        *kind = 3;
        return true;
    }
    if (s->bdt && std::strcmp(name, "rung") == 0)
    {
        *ptr  = s->rung.data();
        *kind = 3;
        return true;
    }
    return false;
}

} // namespace

extern "C" int sphb_sim_get_field(sphb_sim* s, const char* name, double* out, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !name || !out) { return SPHB_ERR_ARG; }
    void* ptr = nullptr;
    int kind  = 0;
    if (!findField(s, name, &ptr, &kind)) { return SPHB_ERR_ARG; }
    size_t n = s->n;
    size_t elem = kind == 0 || kind == 3 ? 8 : kind == 2 ? 4 : s->elemBytes();
    std::vector<char> host(n * elem);
    SPHB_CUDA_TRY(cudaMemcpyAsync(host.data(), ptr, n * elem, cudaMemcpyDeviceToHost, s->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    std::vector<double> conv;
    double* dst = out;
    if (on_device)
    {
        conv.resize(n);
        dst = conv.data();
    }
    for (size_t i = 0; i < n; ++i)
    {
        double v;
        if (kind == 0 || (kind == 1 && elem == 8)) { std::memcpy(&v, host.data() + 8 * i, 8); }
        else if (kind == 1) { v = double(reinterpret_cast<const float*>(host.data())[i]); }
        else if (kind == 2) { v = double(reinterpret_cast<const uint32_t*>(host.data())[i]); }
        else { std::memcpy(&v, host.data() + 8 * i, 8); } // uint64 bits
        dst[i] = v;
    }
    if (on_device) { SPHB_CUDA_TRY(cudaMemcpy(out, conv.data(), n * sizeof(double), cudaMemcpyHostToDevice)); }
    return SPHB_OK;
}

extern "C" int sphb_sim_set_field(sphb_sim* s, const char* name, const double* in, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !name || !in) { return SPHB_ERR_ARG; }
    void* ptr = nullptr;
    int kind  = 0;
    if (!findField(s, name, &ptr, &kind)) { return SPHB_ERR_ARG; }
    s->skinValid = false;
    size_t n = s->n;
    std::vector<double> src(n);
    SPHB_CUDA_TRY(cudaMemcpy(src.data(), in, n * sizeof(double),
                             on_device ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost));
    if (kind == 0 || kind == 3 || (kind == 1 && s->elemBytes() == 8))
    {
        SPHB_CUDA_TRY(cudaMemcpy(ptr, src.data(), n * 8, cudaMemcpyHostToDevice));
    }
    else if (kind == 1)
    {
        std::vector<float> f(src.begin(), src.end());
        SPHB_CUDA_TRY(cudaMemcpy(ptr, f.data(), n * 4, cudaMemcpyHostToDevice));
    }
    else
    {
        std::vector<uint32_t> u(n);
        for (size_t i = 0; i < n; ++i)
        {
            u[i] = uint32_t(src[i]);
        }
        SPHB_CUDA_TRY(cudaMemcpy(ptr, u.data(), n * 4, cudaMemcpyHostToDevice));
    }
    if (std::strcmp(name, "x") == 0 || std::strcmp(name, "y") == 0 || std::strcmp(name, "z") == 0 ||
        std::strcmp(name, "m") == 0)
    {
        SPHB_TRY(packPositions(s->f[fX].data(), s->f[fY].data(), s->f[fZ].data(), s->f[fM].data(), s->n,
                               s->pos.data(), s->mixed ? s->posq.data() : nullptr, s->box, s->stream));
        SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    return SPHB_OK;
}

extern "C" int sphb_sim_scalars(sphb_sim* s, double* out)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !out) { return SPHB_ERR_ARG; }
    double v[18] = {s->minDt,  s->minDt_m1,          s->minDtCourant,     s->minDtRho,  s->ttot,     s->etot,
                    s->ecin,   s->eint,              s->linmom,           s->angmom,    s->totalNeighbors,
                    double(s->iteration), s->hbox.lo[0], s->hbox.hi[0], s->hbox.lo[1], s->hbox.hi[1], s->hbox.lo[2],
                    s->hbox.hi[2]};
    std::memcpy(out, v, sizeof(v));
    return SPHB_OK;
}

extern "C" int sphb_sim_tree(sphb_sim* s, size_t* num_leaves, uint64_t* leaves, uint32_t* counts, uint32_t* layout)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !num_leaves) { return SPHB_ERR_ARG; }
    int L       = s->ftree.numLeaves;
    *num_leaves = size_t(L);
    if (leaves)
    {
        SPHB_CUDA_TRY(cudaMemcpy(leaves, s->ftree.leaves.data(), (L + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    }
    if (counts)
    {
        SPHB_CUDA_TRY(cudaMemcpy(counts, s->ftree.leafCounts.data(), L * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    if (layout)
    {
        SPHB_CUDA_TRY(cudaMemcpy(layout, s->ftree.layout.data(), (L + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    return SPHB_OK;
}

extern "C" int sphb_sim_neighbors(sphb_sim* s, uint32_t* out)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !out) { return SPHB_ERR_ARG; }
    size_t ng    = s->p.ngmax;
    unsigned pad = paddedNgmax(s->p.ngmax);
    std::vector<uint32_t> raw(s->numGroups() * pad * kWarp);
    SPHB_CUDA_TRY(cudaMemcpy(raw.data(), s->nidx.data(), raw.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < s->n; ++i)
    {
        size_t g = i / kWarp, lane = i % kWarp;
        for (size_t k = 0; k < ng; ++k)
        {
            out[i * ng + k] = raw[nidxAt(g, pad, unsigned(k), unsigned(lane))];
        }
    }
    return SPHB_OK;
}

extern "C" int sphb_sim_stage_times(sphb_sim* s, float* out)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !out) { return SPHB_ERR_ARG; }
    std::memcpy(out, s->stageMs, sizeof(s->stageMs));
    return SPHB_OK;
}

extern "C" uint64_t sphb_sim_kernel_launches(const sphb_sim*) { return launchCounter(); }

extern "C" int sphb_sim_search_stats(const sphb_sim* s, uint64_t* out)
{
    if (!s || !out) { return SPHB_ERR_ARG; }
    std::memcpy(out, s->searchStats, sizeof(s->searchStats));
    return SPHB_OK;
}

extern "C" void* sphb_sim_stream(sphb_sim* s) { return s ? static_cast<void*>(s->stream) : nullptr; }

extern "C" int sphb_sim_load_state(sphb_sim* s, const double* const* fields, const uint64_t* id, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !fields || !id) { return SPHB_ERR_ARG; }
    if (!s->uploaded) { return SPHB_ERR_STATE; }
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int k = 0; k < kNumConserved; ++k)
    {
        if (!fields[k]) { return SPHB_ERR_ARG; }
        SPHB_CUDA_TRY(cudaMemcpyAsync(s->f[k].data(), fields[k], s->n * sizeof(double), kind, s->stream));
    }
    SPHB_CUDA_TRY(cudaMemcpyAsync(s->idAlt.data(), id, s->n * sizeof(uint64_t), kind, s->stream));
    return simimpl::finishLoad(*s);
}

extern "C" int sphb_sim_store_state(sphb_sim* s, double* const* fields, uint64_t* id, int on_device)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !fields || !id) { return SPHB_ERR_ARG; }
    cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (int k = 0; k < kNumConserved; ++k)
    {
        if (!fields[k]) { return SPHB_ERR_ARG; }
        SPHB_CUDA_TRY(cudaMemcpyAsync(fields[k], s->f[k].data(), s->n * sizeof(double), kind, s->stream));
    }
    SPHB_CUDA_TRY(cudaMemcpyAsync(id, s->id.data(), s->n * sizeof(uint64_t), kind, s->stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SPHB_OK;
}

extern "C" int sphb_sim_set_fixed_dt(sphb_sim* s, double dt)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !(dt >= 0.0)) { return SPHB_ERR_ARG; }
    s->fixedDt = dt;
    if (dt > 0)
    {
        s->minDt    = dt;
        s->minDt_m1 = dt;
    }
    return SPHB_OK;
}

extern "C" int sphb_sim_set_params(sphb_sim* s, const sphb_params* p)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !p) { return SPHB_ERR_ARG; }
    if (p->ng0 != s->p.ng0 || p->ngmax != s->p.ngmax || p->precision != s->p.precision ||
        p->sinc_index != s->p.sinc_index || p->bucket_focus != s->p.bucket_focus || p->av_clean != s->p.av_clean ||
        !(p->gamma > 1.0))
    {
        return SPHB_ERR_ARG;
    }
    if (!(p->nb_skin >= 0.0) || (s->skinRows.data() && p->nb_skin != s->p.nb_skin)) { return SPHB_ERR_ARG; }
    double minDt = s->p.minDt, minDtM1 = s->p.minDt_m1;
    s->skinValid  = false;
    s->p          = *p;
    s->p.minDt    = minDt;
    s->p.minDt_m1 = minDtM1;
    return SPHB_OK;
}

extern "C" int sphb_sim_step_vjp(sphb_sim* s, const double* const* adj_post, double* const* adj_pre,
                                 double* alphamax_bar)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !adj_post || !adj_pre) { return SPHB_ERR_ARG; }
    for (int f = 0; f < kNumConserved; ++f)
    {
        if (!adj_post[f] || !adj_pre[f] || adj_post[f] == adj_pre[f]) { return SPHB_ERR_ARG; }
    }
    if (!s->uploaded || !(s->fixedDt > 0) || s->p.av_clean) { return SPHB_ERR_STATE; }
    if (!s->hPre.data()) { SPHB_TRY(allocateAdjoint(*s)); }
    s->skinValid = false;
    // the chain arrays of the recomputed step and of its adjoint both carry the tape pointers
    s->taping = true;
    int rc    = computeForces(*s);
    if (rc == SPHB_OK)
    {
        rc = s->mixed ? runStepVjp<float>(*s, adj_post, adj_pre, alphamax_bar)
                      : runStepVjp<double>(*s, adj_post, adj_pre, alphamax_bar);
    }
    s->taping = false;
    return rc;
}

extern "C" int sphb_sim_tape_reserve(sphb_sim* s, int slots)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || slots < 1) { return SPHB_ERR_ARG; }
    if (!s->uploaded || s->p.av_clean) { return SPHB_ERR_STATE; }
    if (!s->hPre.data()) { SPHB_TRY(allocateAdjoint(*s)); }
    size_t bytes = 0;
    for (auto pb : tapedBuffers(*s))
    {
        bytes += alignTape(pb.second);
    }
    SPHB_TRY(s->tapeSlots.reserve(bytes * size_t(slots)));
    s->tapeSlotBytes = bytes;
    s->numTapeSlots  = slots;
    return SPHB_OK;
}

extern "C" int sphb_sim_step_record(sphb_sim* s, int slot)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || slot < 0) { return SPHB_ERR_ARG; }
    if (!s->uploaded || !(s->fixedDt > 0) || slot >= s->numTapeSlots) { return SPHB_ERR_STATE; }
    s->taping = true;
    int rc    = computeForces(*s);
    s->taping = false;
    if (rc != SPHB_OK) { return rc; }
    SPHB_TRY(copyTape(*s, slot, true));
    return integrateStep(*s);
}

extern "C" int sphb_sim_step_vjp_recorded(sphb_sim* s, int slot, const double* const* adj_post,
                                          double* const* adj_pre, double* alphamax_bar)
{
    if (s) { SPHB_TRY(simimpl::waitLateFields(*s, true)); }
    if (!s || !adj_post || !adj_pre || slot < 0) { return SPHB_ERR_ARG; }
    for (int f = 0; f < kNumConserved; ++f)
    {
        if (!adj_post[f] || !adj_pre[f] || adj_post[f] == adj_pre[f]) { return SPHB_ERR_ARG; }
    }
    if (!s->uploaded || !(s->fixedDt > 0) || slot >= s->numTapeSlots) { return SPHB_ERR_STATE; }
    s->skinValid = false;
    SPHB_TRY(copyTape(*s, slot, false));
    s->taping = true;
    int rc = s->mixed ? runStepVjp<float>(*s, adj_post, adj_pre, alphamax_bar)
                      : runStepVjp<double>(*s, adj_post, adj_pre, alphamax_bar);
    s->taping = false;
    return rc;
}

namespace sphb
{
namespace simimpl
{
int runStage(sphb_sim& s, int stage) { return runStageChecked(s, stage); }
int waitMidFields(sphb_sim& s)
{
    if (s.midPending)
    {
        SPHB_CUDA_TRY(cudaStreamWaitEvent(s.stream, s.midReady, 0));
        s.midPending = false;
    }
    if (s.idCheckPending && !s.idCheckIssued)
    {
        // the loaded ids (now s.id) against the previous ones (s.idAlt), before a reordering sync reuses idAlt; the
        // host reads the flag where it decides between the rows and the tree search
        SPHB_TRY(idsDiffer(s.id.data(), s.idAlt.data(), s.n, s.skinWork.data(), s.stream));
        s.hostMsg[14] = 1;
        SPHB_CUDA_TRY(cudaMemcpyAsync(s.hostMsg + 14, s.skinWork.data(), sizeof(unsigned), cudaMemcpyDeviceToHost,
                                      s.stream));
        SPHB_CUDA_TRY(cudaEventRecord(s.idCheckDone, s.stream));
        s.idCheckIssued = true;
    }
    if (s.midGatherPending)
    {
        // h and the ids into the order of the last sync (which gathered the fields it reads itself)
        const void* src[2] = {s.f[fH].data(), s.id.data()};
        void* dst[2]       = {s.fAlt[fH].data(), s.idAlt.data()};
        SPHB_TRY(gather8(s.order.data(), s.n, 2, src, dst, s.stream));
        s.f[fH].swap(s.fAlt[fH]);
        s.id.swap(s.idAlt);
        s.midGatherPending = false;
    }
    return kOk;
}

int resolveIdCheck(sphb_sim& s)
{
    if (!s.idCheckPending) { return kOk; }
    SPHB_TRY(waitMidFields(s));
    SPHB_CUDA_TRY(cudaEventSynchronize(s.idCheckDone));
    unsigned differ = 1;
    std::memcpy(&differ, s.hostMsg + 14, sizeof(differ));
    if (differ) { s.skinValid = false; }
    s.idCheckPending = false;
    s.idCheckIssued  = false;
    return kOk;
}

int lateGroupOf(int field)
{
    switch (field)
    {
    case fTemp: return 0;
    case fVx:
    case fVy:
    case fVz:
    case fAlpha: return 1;
    case fXm1:
    case fYm1:
    case fZm1:
    case fDuM1: return 2;
    default: return -1;
    }
}

int packVelocity(sphb_sim& s)
{
    return s.mixed ? launchPackVelocity(chainArrays<float>(s), s.stream)
                   : launchPackVelocity(chainArrays<double>(s), s.stream);
}

int waitLateGroup(sphb_sim& s, int group)
{
    SPHB_TRY(waitMidFields(s));
    if (s.latePending[group])
    {
        SPHB_CUDA_TRY(cudaStreamWaitEvent(s.stream, s.lateReady[group], 0));
        s.latePending[group] = false;
    }
    if (s.lateGatherPending[group])
    {
        // the group's fields into the order of the last sync (which gathered the others)
        const void* src[kNumConserved];
        void* dst[kNumConserved];
        int numFields = 0;
        for (int k = 0; k < kNumConserved; ++k)
        {
            if (lateGroupOf(k) != group) { continue; }
            src[numFields] = s.f[k].data();
            dst[numFields] = s.fAlt[k].data();
            ++numFields;
        }
        SPHB_TRY(gather8(s.order.data(), s.n, numFields, src, dst, s.stream));
        for (int k = 0; k < kNumConserved; ++k)
        {
            if (lateGroupOf(k) == group) { s.f[k].swap(s.fAlt[k]); }
        }
        s.lateGatherPending[group] = false;
    }
    if (group == 1 && s.velocityPackPending)
    {
        SPHB_TRY(packVelocity(s));
        s.velocityPackPending = false;
    }
    return kOk;
}

int waitLateFields(sphb_sim& s, bool host)
{
    for (int g = 0; g < sphb_sim::kLateGroups; ++g)
    {
        bool pending = s.latePending[g];
        SPHB_TRY(waitLateGroup(s, g));
        if (host && pending) { SPHB_CUDA_TRY(cudaEventSynchronize(s.lateReady[g])); }
    }
    if (host) { SPHB_TRY(resolveIdCheck(s)); }
    return kOk;
}
bool findField(sphb_sim& s, const char* name, void** ptr, int* kind) { return ::findField(&s, name, ptr, kind); }
double cv(const sphb_sim& s) { return idealGasCv(s.p.mui, s.p.gamma); }

int finishUpload(sphb_sim& s)
{
    SPHB_CUDA_TRY(cudaMemsetAsync(s.keys.data(), 0, s.n * sizeof(uint64_t), s.stream));
    SPHB_CUDA_TRY(cudaMemsetAsync(s.du.data(), 0, s.n * sizeof(double), s.stream));
    SPHB_TRY(initGlobalTree(s.gtree, std::max<unsigned>(s.p.bucket_focus, unsigned(s.n / 100)), s.stream));
    SPHB_TRY(initFocusTree(s.ftree, s.p.bucket_focus, s.ts, s.stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s.stream));
    s.boxFirstCall = true;
    s.skinValid    = false;
    s.nextStage    = sSync;
    s.minDt        = s.p.minDt;
    s.minDt_m1     = s.p.minDt_m1;
    s.ttot         = 0;
    s.iteration    = 1;
    s.uploaded     = true;
    s.forcesDone   = false;
    if (s.bdt) { SPHB_TRY(resetBdt(s)); }
    return kOk;
}

int finishLoad(sphb_sim& s)
{
    if (!s.skinValid)
    {
        s.id.swap(s.idAlt);
        return kOk;
    }
    // the skin rows stay usable when every index holds the same particle as before (positions and h may differ
    // arbitrarily: the next refilter checks them against the build)
    if (s.midPending)
    {
        // the ids are still in flight on the copy stream: compared once they arrive (waitMidFields), read by the
        // host before the neighbour search
        s.id.swap(s.idAlt);
        s.idCheckPending = true;
        s.idCheckIssued  = false;
        return kOk;
    }
    SPHB_TRY(idsDiffer(s.id.data(), s.idAlt.data(), s.n, s.skinWork.data(), s.stream));
    unsigned differ = 1;
    SPHB_CUDA_TRY(cudaMemcpyAsync(&differ, s.skinWork.data(), sizeof(unsigned), cudaMemcpyDeviceToHost, s.stream));
    SPHB_CUDA_TRY(cudaStreamSynchronize(s.stream));
    s.id.swap(s.idAlt);
    if (differ) { s.skinValid = false; }
    return kOk;
}

int positions(sphb_sim& s, double dt, double dtM1)
{
    SPHB_TRY(waitLateFields(s));
    s.minDt    = dt;
    s.minDt_m1 = dtM1;
    double c   = idealGasCv(s.p.mui, s.p.gamma);
    return s.mixed ? runPositions<float>(s, c) : runPositions<double>(s, c);
}
} // namespace simimpl
} // namespace sphb
