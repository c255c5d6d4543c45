// Internal header of the simulation object (sim.cu): the particle dataset in HBM and the state of the step. Shared
// with the typed-boundary entry points (bound.cu), which run the same stages on caller-owned arrays.
#pragma once

#include <cstring>
#include <string>
#include <vector>

#include "adjoint.cuh"
#include "bdt.cuh"
#include "groups.cuh"
#include "hydro.cuh"
#include "integrate.cuh"
#include "neighbors.cuh"
#include "octree.cuh"
#include "primitives.cuh"
#include "sfc.cuh"
#include "sort.cuh"

namespace sphb
{

//! conserved fields, in the order of the upload ABI
enum Field : int
{
    fX, fY, fZ, fH, fM, fTemp, fVx, fVy, fVz, fXm1, fYm1, fZm1, fDuM1, fAlpha, kNumConserved
};
inline const char* const kConservedNames[kNumConserved] = {"x",  "y",    "z",    "h",    "m",     "temp", "vx",
                                                           "vy", "vz",   "x_m1", "y_m1", "z_m1", "du_m1", "alpha"};

//! derived fields stored in the J-loop type
enum Derived : int
{
    dXm, dKx, dGradh, dPrho, dC, dC11, dC12, dC13, dC22, dC23, dC33, dDivv, dCurlv, dAx, dAy, dAz, kNumDerived
};
inline const char* const kDerivedNames[kNumDerived] = {"xm",  "kx",  "gradh", "prho", "c",     "c11", "c12", "c13",
                                                       "c22", "c23", "c33",   "divv", "curlv", "ax",  "ay",  "az"};

enum Stage : int
{
    sSync, sNeighbors, sXMass, sVeDefGradh, sIad, sAV, sMomentum, sConserved, sIntegrate, kNumStages
};

} // namespace sphb

using namespace sphb;

struct sphb_sim
{
    size_t n{0};
    sphb_params p{};
    sphb_box hbox{};
    DevBox box{};
    bool mixed{false};
    cudaStream_t stream{nullptr};

    DeviceBuffer<double> f[kNumConserved];
    DeviceBuffer<double> fAlt[kNumConserved];
    DeviceBuffer<uint64_t> id, idAlt, keys;
    DeviceBuffer<uint32_t> order;
    DeviceBuffer<char> sortScratch;
    DeviceBuffer<double4> pos;
    DeviceBuffer<int4> posq;
    DeviceBuffer<float4> blockLo, blockHi;
    DeviceBuffer<uint32_t> nidx;
    DeviceBuffer<unsigned> nc;
    DeviceBuffer<char> derived[kNumDerived];
    DeviceBuffer<double> du;
    DeviceBuffer<char> hrec, grec, avrec;
    DeviceBuffer<char> dvrec, dv; // AV cleaning only: symmetrised velocity gradients (record + 6 arrays)
    DeviceBuffer<double> whD, whdD;
    DeviceBuffer<float> whF, whdF;
    DeviceBuffer<unsigned long long> reduce;
    DeviceBuffer<unsigned> status;
    DeviceBuffer<double> partial, cons;
    double K{0};
    // FP32 polynomial kernel: fitted once per simulation (it depends only on the sinc index)
    bool polyReady{false};
    int polyOk{0};
    float wpoly[kPolyTerms]{};
    float dwpoly[kPolyTerms]{};

    GlobalTree gtree;
    FocusTree ftree;
    TreeScratch ts;
    bool boxFirstCall{true};

    double minDt{0}, minDt_m1{0}, minDtCourant{INFINITY}, minDtRho{INFINITY}, ttot{0};
    double etot{0}, ecin{0}, eint{0}, linmom{0}, angmom{0};
    double totalNeighbors{0};
    uint64_t iteration{1};
    bool uploaded{false};
    bool forcesDone{false};
    int nextStage{0}; // the stage of the force computation that may run next (StageOrder), 0 = the domain sync

    // fixed time step (> 0) instead of computeTimestep; required by the step adjoint
    double fixedDt{0};
    // adjoint support: when taping, the forward also records what its adjoint needs
    bool taping{false};
    DeviceBuffer<double> hPre, alphaPre;
    DeviceBuffer<char> tapeT;
    DeviceBuffer<int> tapeJ;
    DeviceBuffer<char> adjT;
    DeviceBuffer<double> adjWork, adjScalar;
    DeviceBuffer<float4> adjJacc; // FP32 adjoint: vector-atomic neighbour sums of the MomentumEnergy adjoint
    // recorded steps: copies of everything the step adjoint reads, one slot per step of a checkpoint segment
    DeviceBuffer<char> tapeSlots;
    size_t tapeSlotBytes{0};
    int numTapeSlots{0};

    // skin lists (neighbors.cuh): candidate rows kept across steps and refiltered exactly every step
    DeviceBuffer<uint32_t> skinRows;
    DeviceBuffer<uint16_t> skinDist;
    DeviceBuffer<unsigned> skinCount;
    DeviceBuffer<double> skinRadius, skinXb, skinYb, skinZb;
    DeviceBuffer<uint32_t> skinBuild, skinBuildAlt, skinMoved;
    DeviceBuffer<unsigned> skinGrid;
    DeviceBuffer<unsigned> skinWork; // [0], [1]: deferred by the check / by the iteration, then the two lists
    DeviceBuffer<unsigned> skinGroupD;
    cudaStream_t sideStream{nullptr}; // the tree search of deferred groups, beside the refilter
    // typed loads from host memory: x, y, z and m come first on the compute stream; the rest follows on copyStream in
    // the order the step reads it: h and the ids while the sync runs (midReady: read by a reordering sync's gather,
    // else by the search); then the late groups, temp (first read by VeDefGradh, group 0), v and alpha (IAD and the
    // velocity part of the hydro record, group 1), x_m1, y_m1, z_m1 and du_m1 (the integration, group 2).
    // midPending / latePending say that the compute stream has not waited for them yet; lateGatherPending, that a
    // reordering sync left the group to be gathered once it arrives; velocityPackPending, that VeDefGradh left the
    // velocities of the hydro record to the arrival of group 1; idCheckPending, that the comparison of the loaded ids
    // with the previous ones (whether the skin rows stay usable) is on its way to hostMsg[14] (idCheckDone)
    static constexpr int kLateGroups = 3;
    cudaStream_t copyStream{nullptr};
    cudaEvent_t copyFork{nullptr}, midReady{nullptr}, idCheckDone{nullptr};
    cudaEvent_t lateReady[kLateGroups]{};
    bool midPending{false};
    bool latePending[kLateGroups]{};
    bool lateGatherPending[kLateGroups]{};
    bool idCheckPending{false};
    bool idCheckIssued{false}; // the comparison is on the compute stream (idCheckDone recorded)
    bool velocityPackPending{false};
    bool midGatherPending{false}; // a reordering sync left h and the ids to be gathered once they arrive
    cudaEvent_t skinFork{nullptr}, skinJoin{nullptr};
    unsigned skinCap{0};
    bool skinValid{false};    // rows match the particles' current indices (up to the tracked permutation)
    bool skinAnyMoved{false}; // some index holds another particle than at the build (skinBuild, skinMoved valid)
    bool skinFiltered{false}; // this step's lists came from the rows
    bool syncRemapped{false}; // the last sync composed its order into the rows' index map (counted at the search)
    int skinAge{0};           // steps since the build
    int skinHoldoff{0};       // steps left of plain tree searches after rows proved short-lived
    unsigned skinDeferredLast{0};
    // tree searches of every group, row builds, refiltered steps, deferred groups, syncs that remapped the rows
    uint64_t searchStats[5]{};

    // block time steps (main/src/propagator/ve_hydro_bdt.hpp), after sphb_sim_bdt_enable
    struct BdtTimestep // sph::Timestep (sph/include/sph/timestep.h:17-31)
    {
        float nextDt{0}, elapsedDt{0}, totDt{0};
        int numRungs{1};
        int substep{0};
        uint32_t rungRanges[kMaxRungs + 1]{};
        float dtm1[kMaxRungs]{};
        float dtDrift[kMaxRungs]{};
    };
    bool bdt{false};
    float etaAcc{0.2f};
    BdtTimestep bts, bprevTs;
    DeviceBuffer<uint64_t> rung, rungAlt;   // rung each particle was last advanced on (a conserved field)
    DeviceBuffer<float> groupDt;            // per group of the current group order
    DeviceBuffer<uint32_t> groupIdx;        // sort permutation of groupDt
    DeviceBuffer<uint32_t> grpSfc, grpTs;   // groups_ (SFC order after a full sync) and tsGroups_ (by time step)
    DeviceBuffer<uint32_t> grpBounds;       // the spatial target groups of the last full sync: group g holds the
                                            // particles [grpBounds[g], grpBounds[g + 1])
    DeviceBuffer<int> grpScratch;
    unsigned numBdtGroups{0};
    DeviceBuffer<uint64_t> dtKeys;
    DeviceBuffer<uint32_t> rungInfo;
    DeviceBuffer<double> xs, ys, zs;        // positions at the last full sync (drift bound of the tree search)
    DeviceBuffer<unsigned long long> dispMax;
    const uint32_t* activeList{nullptr};    // activeRungs_: groups whose forces this substep computes
    unsigned numActive{0};
    double treeExt{0.0};                    // widening of the tree's node boxes (TreeView::ext)

    // typed boundary (bound.cu): the caller's device arrays by reference field name, and staging of typed copies
    struct Binding
    {
        std::string name;
        void* data;
        int dtype;
    };
    std::vector<Binding> bound;
    bool boxFromCaller{false};   // the bound dataset's box is the caller's: the sync does not refit open axes
    bool lastSyncIdentity{true}; // the last domain sync found the particles already in SFC order
    DeviceBuffer<char> typedStage;
    DeviceBuffer<unsigned long long> boxExtrema; // open axes: min/max of x, y, z as ordered bits
    DeviceBuffer<char> earlyStage; // sphb_sim_step_fields: converted outputs copied out before the step ends

    cudaEvent_t ev[kNumStages + 1]{};
    float stageMs[kNumStages]{};
    // pinned landing place of the small per-step reads (sums, reductions, status), so that they queue behind the
    // kernels and the host waits once
    unsigned long long* hostMsg{nullptr};

    size_t elemBytes() const { return mixed ? sizeof(float) : sizeof(double); }
    size_t numGroups() const { return (n + kWarp - 1) / kWarp; }

    template<class T>
    T* dptr(int d) const
    {
        return reinterpret_cast<T*>(derived[d].data());
    }
};

namespace sphb
{
namespace simimpl
{
//! one stage of the force computation under the stage ABI's ordering rule (sim.cu runStageChecked)
int runStage(sphb_sim& s, int stage);
//! device pointer and element kind (0 double, 1 J-loop type, 2 uint32, 3 uint64) of a field by reference name
bool findField(sphb_sim& s, const char* name, void** ptr, int* kind);
//! the ideal-gas heat capacity of the simulation's parameters
double cv(const sphb_sim& s);
//! after the conserved fields and ids were written: reset the step state as sphb_sim_upload does
int finishUpload(sphb_sim& s);
//! after the conserved fields were written and the new ids placed in s.idAlt: take the ids as sphb_sim_load_state
//! does (the skin rows survive if every index holds the same particle)
int finishLoad(sphb_sim& s);
//! computePositions of the global step with time steps dt, dt_m1 (kick-drift and energy update, FP64)
int positions(sphb_sim& s, double dt, double dtM1);
//! the compute stream waits for h and the ids of a typed host load, if they are still in flight, and compares the
//! ids with the previous ones when skin rows exist
int waitMidFields(sphb_sim& s);
//! late group of a conserved field of a typed host load (temp: 0; v, alpha: 1; x_m1, y_m1, z_m1, du_m1: 2; -1 for
//! the fields copied before them)
int lateGroupOf(int field);
//! the compute stream waits for one late group of a typed host load if it is still in flight, and gathers it if a
//! reordering sync left it
int waitLateGroup(sphb_sim& s, int group);
//! the compute stream waits for every field of a typed host load still in flight and gathers the late ones a
//! reordering sync left; with host, the calling thread waits for them too and learns the id comparison (entry points
//! other than the step: their caller may reuse the host arrays)
int waitLateFields(sphb_sim& s, bool host = false);
//! the host learns the result of a pending id comparison; rows whose indices now hold other particles are dropped
int resolveIdCheck(sphb_sim& s);
} // namespace simimpl
} // namespace sphb
