/*
 * TEST ORACLE ONLY — not product code.
 *
 * C-ABI driver around the reference's own OpenMP CPU implementation of the SPH-VE hydro step, compiled from the
 * reference sources where they lie (headers only; nothing is copied) by oracle/Makefile into oracle/_ref/libsphref.so.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it.
 *
 * The step mirrors HydroVeProp::computeForces + integrate (main/src/propagator/ve_hydro.hpp:126-220) with avClean=false
 * and no gravity, with the main loop's first propagator->sync before step 1 (main/src/sphexa/sphexa.cpp:141) and the
 * observables call between the two halves (sphexa.cpp:150-156).
 *
 * Two builds exist: the FP64 one (every field double, via the type override in oracle/ref/stub/sph/types.hpp) and the
 * reference-default mixed one (f64 coordinates, f32 hydro fields). Field access by name copies to/from double host
 * arrays so one C ABI serves both builds.
 */
#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>

#include "cstone/domain/domain.hpp"
#include "cstone/traversal/collisions.hpp"
#include "cstone/fields/field_get.hpp"
#include "sph/particles_data.hpp"
#include "sph/sph.hpp"
#include "sph/hydro_ve/av_switches_kern.hpp"
#include "sph/hydro_ve/divv_curlv_kern.hpp"
#include "sph/hydro_ve/iad_kern.hpp"
#include "sph/hydro_ve/momentum_energy_kern.hpp"
#include "sph/hydro_ve/ve_def_gradh_kern.hpp"
#include "sph/hydro_ve/xmass_kern.hpp"
#include "sph/sph_kernel_tables.hpp"

#include "../../main/src/observables/conserved_quantities.hpp"

using namespace sph;
using cstone::CpuTag;
using util::FieldList;

using Dataset = sphexa::ParticlesData<CpuTag>;
using Domain  = cstone::Domain<uint64_t, double, CpuTag>;

using ConservedFields = FieldList<"temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha", "id">;
using DependentFields =
    FieldList<"ax", "ay", "az", "prho", "c", "du", "c11", "c12", "c13", "c22", "c23", "c33", "xm", "kx", "nc">;

struct RefSim
{
    Dataset d;
    std::unique_ptr<Domain> domain;
    cstone::Box<double> box{0, 1};
    double timeSync{0}, timeNeighbors{0}, timeChain{0}, timeIntegrate{0};
    bool synced{false};
    bool avClean{false};
};

namespace
{

template<class V>
int copyOut(const V& v, size_t first, size_t n, double* out)
{
    if (v.size() < first + n) { return -1; }
    for (size_t i = 0; i < n; ++i)
    {
        out[i] = double(v[first + i]);
    }
    return 0;
}

template<class V>
int copyIn(V& v, size_t first, size_t n, const double* in)
{
    if (v.size() < first + n) { return -1; }
    using E = typename V::value_type;
    for (size_t i = 0; i < n; ++i)
    {
        v[first + i] = E(in[i]);
    }
    return 0;
}

using Clock = std::chrono::steady_clock;
double since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

void syncOnce(RefSim& s)
{
    auto& d = s.d;
    s.domain->sync(cstone::get<"keys">(d), cstone::get<"x">(d), cstone::get<"y">(d), cstone::get<"z">(d),
                   cstone::get<"h">(d), std::tuple_cat(std::tie(cstone::get<"m">(d)), cstone::get<ConservedFields>(d)),
                   cstone::get<DependentFields>(d));
    d.treeView = s.domain->octreeProperties();
    s.box      = s.domain->box();
}

} // namespace

extern "C"
{

    //! @brief return 64 for the FP64 oracle build, 32 for the reference-default (f32 hydro fields) build
    int ref_hydro_bits() { return int(sizeof(Dataset::HydroType) * 8); }

    /*! @brief create a simulation from host arrays (double), in any particle order
     *
     * fields: x,y,z,h,m,temp,vx,vy,vz,x_m1,y_m1,z_m1,du_m1,alpha (14 arrays of n doubles), id (n uint64)
     * boxLimits: xmin,xmax,ymin,ymax,zmin,zmax; periodic: 1 = periodic in all 3 dimensions, 0 = open
     * params: ng0, ngmax, gamma, muiConst, minDt, minDt_m1, Kcour, Krho, alphamin, alphamax, decay_constant
     */
    void* ref_sim_create(size_t n, const double* const* fields, const uint64_t* id, const double* boxLimits,
                         int periodic, const double* params)
    {
        auto s  = new RefSim;
        auto& d = s->d;
        d.setConserved("x", "y", "z", "h", "m");
        d.setDependent("keys");
        std::apply([&d](auto... f) { d.setConserved(f.value...); }, make_tuple(ConservedFields{}));
        std::apply([&d](auto... f) { d.setDependent(f.value...); }, make_tuple(DependentFields{}));
        d.setDependent("gradh", "divv", "curlv");

        d.ng0            = unsigned(params[0]);
        d.ngmax          = unsigned(params[1]);
        d.gamma          = params[2];
        d.muiConst       = params[3];
        d.minDt          = params[4];
        d.minDt_m1       = params[5];
        d.Kcour          = params[6];
        d.Krho           = params[7];
        d.alphamin       = params[8];
        d.alphamax       = params[9];
        d.decay_constant = params[10];
        d.numParticlesGlobal = n;
        d.resize(n);

        copyIn(d.x, 0, n, fields[0]);
        copyIn(d.y, 0, n, fields[1]);
        copyIn(d.z, 0, n, fields[2]);
        copyIn(d.h, 0, n, fields[3]);
        copyIn(d.m, 0, n, fields[4]);
        copyIn(d.temp, 0, n, fields[5]);
        copyIn(d.vx, 0, n, fields[6]);
        copyIn(d.vy, 0, n, fields[7]);
        copyIn(d.vz, 0, n, fields[8]);
        copyIn(d.x_m1, 0, n, fields[9]);
        copyIn(d.y_m1, 0, n, fields[10]);
        copyIn(d.z_m1, 0, n, fields[11]);
        copyIn(d.du_m1, 0, n, fields[12]);
        copyIn(d.alpha, 0, n, fields[13]);
        for (size_t i = 0; i < n; ++i)
        {
            d.id[i] = id[i];
        }

        auto bt = periodic ? cstone::BoundaryType::periodic : cstone::BoundaryType::open;
        s->box  = cstone::Box<double>(boxLimits[0], boxLimits[1], boxLimits[2], boxLimits[3], boxLimits[4],
                                      boxLimits[5], bt, bt, bt);

        uint64_t bucketSizeFocus = 64;
        uint64_t bucketSize      = std::max(bucketSizeFocus, d.numParticlesGlobal / 100);
        float theta              = 1.0f;
        s->domain = std::make_unique<Domain>(0, 1, bucketSize, bucketSizeFocus, theta, s->box);
        return s;
    }

    void ref_sim_destroy(void* p) { delete static_cast<RefSim*>(p); }

    //! @brief HydroVeProp<avClean = true> (ve_hydro.hpp:48-90,175-185): the symmetric velocity gradients are kept
    //! (iad_divv_curlv.hpp:62-69 computes them when the fields exist) and MomentumEnergy applies the AV cleaning
    void ref_sim_set_av_clean(void* p, int on)
    {
        auto& s   = *static_cast<RefSim*>(p);
        s.avClean = on != 0;
        if (s.avClean)
        {
            s.d.setDependent("dV11", "dV12", "dV13", "dV22", "dV23", "dV33");
            s.d.resize(s.d.x.size());
        }
    }

    //! @brief the sync that the main program performs once before the first step (sphexa.cpp:141)
    int ref_sim_initial_sync(void* p)
    {
        auto& s = *static_cast<RefSim*>(p);
        try
        {
            syncOnce(s);
        }
        catch (std::exception& e)
        {
            std::fprintf(stderr, "ref_sim_initial_sync: %s\n", e.what());
            return -1;
        }
        s.synced = true;
        return 0;
    }

    //! @brief first half of a step: HydroVeProp::computeForces (ve_hydro.hpp:126-203) + conserved quantities
    int ref_sim_compute_forces(void* p)
    {
        auto& s = *static_cast<RefSim*>(p);
        auto& d = s.d;
        try
        {
            auto t0 = Clock::now();
            syncOnce(s);
            s.timeSync += since(t0);

            d.resize(s.domain->nParticlesWithHalos());
            resizeNeighbors(d, s.domain->nParticles() * d.ngmax);
            size_t first = s.domain->startIndex();
            size_t last  = s.domain->endIndex();

            t0 = Clock::now();
            findNeighborsSfc(first, last, d, s.box);
            s.timeNeighbors += since(t0);

            t0 = Clock::now();
            GroupView grp{first, last, 0, nullptr, nullptr};
            computeXMass(grp, d, s.box);
            computeVeDefGradh(grp, d, s.box);
            computeEOS(first, last, d);
            computeIadDivvCurlv(grp, d, s.box);
            d.minDtRho = rhoTimestep(first, last, d);
            computeAVswitches(grp, d, s.box);
            if (s.avClean) { computeMomentumEnergy<true>(grp, nullptr, d, s.box); }
            else { computeMomentumEnergy<false>(grp, nullptr, d, s.box); }
            s.timeChain += since(t0);

            sphexa::computeConservedQuantities(first, last, d, MPI_COMM_WORLD);
        }
        catch (std::exception& e)
        {
            std::fprintf(stderr, "ref_sim_compute_forces: %s\n", e.what());
            return -1;
        }
        return 0;
    }

    //! @brief second half of a step: HydroVeProp::integrate (ve_hydro.hpp:205-220); returns 1 if particles failed
    int ref_sim_integrate(void* p)
    {
        auto& s = *static_cast<RefSim*>(p);
        auto& d = s.d;
        auto t0 = Clock::now();
        size_t first = s.domain->startIndex();
        size_t last  = s.domain->endIndex();
        GroupView grp{first, last, 0, nullptr, nullptr};
        computeTimestep(first, last, d);
        computePositions(grp, d, s.box, d.minDt, {float(d.minDt_m1)});
        bool unconverged = updateSmoothingLength(grp, d);
        d.iteration++;
        s.timeIntegrate += since(t0);
        return unconverged ? 1 : 0;
    }

    int ref_sim_step(void* p)
    {
        int rc = ref_sim_compute_forces(p);
        if (rc) { return rc; }
        return ref_sim_integrate(p);
    }

    //! @brief index range [first, last) of the locally owned particles inside the field buffers
    void ref_sim_range(void* p, size_t* first, size_t* last)
    {
        auto& s = *static_cast<RefSim*>(p);
        *first  = s.domain->startIndex();
        *last   = s.domain->endIndex();
    }

    //! @brief copy the owned part of a named field (ParticlesData::fieldNames) into a double array
    int ref_sim_get(void* p, const char* name, double* out)
    {
        auto& s      = *static_cast<RefSim*>(p);
        auto& d      = s.d;
        size_t first = s.domain->startIndex();
        size_t n     = s.domain->endIndex() - first;
        auto ptrs    = d.data();
        for (size_t f = 0; f < Dataset::fieldNames.size(); ++f)
        {
            if (std::strcmp(Dataset::fieldNames[f], name) == 0)
            {
                return std::visit([&](auto* vec) { return copyOut(*vec, first, n, out); }, ptrs[f]);
            }
        }
        return -2;
    }

    //! @brief overwrite the owned part of a named field
    int ref_sim_set(void* p, const char* name, const double* in)
    {
        auto& s      = *static_cast<RefSim*>(p);
        auto& d      = s.d;
        size_t first = s.domain->startIndex();
        size_t n     = s.domain->endIndex() - first;
        auto ptrs    = d.data();
        for (size_t f = 0; f < Dataset::fieldNames.size(); ++f)
        {
            if (std::strcmp(Dataset::fieldNames[f], name) == 0)
            {
                return std::visit([&](auto* vec) { return copyIn(*vec, first, n, in); }, ptrs[f]);
            }
        }
        return -2;
    }

    //! @brief SFC keys of the owned particles
    int ref_sim_keys(void* p, uint64_t* out)
    {
        auto& s      = *static_cast<RefSim*>(p);
        size_t first = s.domain->startIndex();
        size_t n     = s.domain->endIndex() - first;
        std::memcpy(out, s.d.keys.data() + first, n * sizeof(uint64_t));
        return 0;
    }

    //! @brief scalars: minDt, minDt_m1, minDtCourant, minDtRho, ttot, etot, ecin, eint, linmom, angmom,
    //!        totalNeighbors, iteration, box xmin..zmax (6)
    void ref_sim_scalars(void* p, double* out)
    {
        auto& s = *static_cast<RefSim*>(p);
        auto& d = s.d;
        double v[18] = {d.minDt, d.minDt_m1, d.minDtCourant, d.minDtRho, d.ttot, d.etot, d.ecin, d.eint, d.linmom,
                        d.angmom, double(d.totalNeighbors), double(d.iteration), s.box.xmin(), s.box.xmax(),
                        s.box.ymin(), s.box.ymax(), s.box.zmin(), s.box.zmax()};
        std::memcpy(out, v, sizeof(v));
    }

    //! @brief accumulated wall seconds of sync, neighbour search, SPH chain, integration
    void ref_sim_timings(void* p, double* out)
    {
        auto& s = *static_cast<RefSim*>(p);
        out[0]  = s.timeSync;
        out[1]  = s.timeNeighbors;
        out[2]  = s.timeChain;
        out[3]  = s.timeIntegrate;
    }

    //! @brief number of leaf cells of the focus tree used for the neighbour search
    size_t ref_sim_num_leaves(void* p)
    {
        auto& s = *static_cast<RefSim*>(p);
        return s.domain->focusTree().treeLeaves().size() - 1;
    }

    //! @brief focus-tree leaves (numLeaves+1 keys), leaf counts (numLeaves) and particle layout (numLeaves+1)
    int ref_sim_tree(void* p, uint64_t* leaves, unsigned* counts, unsigned* layout)
    {
        auto& s     = *static_cast<RefSim*>(p);
        auto lv     = s.domain->focusTree().treeLeaves();
        auto lay    = s.domain->layout();
        size_t numL = lv.size() - 1;
        std::memcpy(leaves, lv.data(), (numL + 1) * sizeof(uint64_t));
        // the focus tree keeps its leaf counts private; at one rank they equal the layout differences
        for (size_t i = 0; i < numL; ++i)
        {
            counts[i] = lay[i + 1] - lay[i];
        }
        for (size_t i = 0; i <= numL; ++i)
        {
            layout[i] = lay[i];
        }
        return 0;
    }

    //! @brief number of leaves of the global (assignment) tree
    size_t ref_sim_num_global_leaves(void* p)
    {
        auto& s = *static_cast<RefSim*>(p);
        return s.domain->globalTree().numLeafNodes;
    }

    //! @brief neighbour lists of the last force computation, [n][ngmax] with list order as stored
    int ref_sim_neighbors(void* p, uint32_t* out)
    {
        auto& s      = *static_cast<RefSim*>(p);
        size_t first = s.domain->startIndex();
        size_t n     = s.domain->endIndex() - first;
        if (s.d.neighbors.size() < n * s.d.ngmax) { return -1; }
        std::memcpy(out, s.d.neighbors.data(), n * s.d.ngmax * sizeof(uint32_t));
        return 0;
    }

    //! @brief the normalisation constant K and the wh/whd tables (20000 entries each) of the dataset
    void ref_sim_tables(void* p, double* K, double* wh, double* whd)
    {
        auto& s = *static_cast<RefSim*>(p);
        *K      = s.d.K;
        for (int i = 0; i < lt::kTableSize; ++i)
        {
            wh[i]  = s.d.wh[i];
            whd[i] = s.d.whd[i];
        }
    }

    // ---------------------------------------------------------------------------------------------------------------
    // Standalone J-loop calls on caller arrays (all double), used to pin the kernels against the reference's own
    // known-answer fixture (sph/test/ve.cpp) and to feed identical inputs to CUDA kernels. The box is given as
    // limits[6] + periodic flag. Neighbour lists: nbr[i*ngmax + k], count[i] neighbours (self excluded).
    // ---------------------------------------------------------------------------------------------------------------

    static cstone::Box<double> mkBox(const double* lim, int periodic)
    {
        auto bt = periodic ? cstone::BoundaryType::periodic : cstone::BoundaryType::open;
        return cstone::Box<double>(lim[0], lim[1], lim[2], lim[3], lim[4], lim[5], bt, bt, bt);
    }

    //! @brief fill the FP64 sinc^n tables and K exactly as ParticlesData::createTables (particles_data.hpp:377-387)
    void ref_tables_fp64(double sincIndex, double* K, double* wh, double* whd)
    {
        *K      = sph::kernel_3D_k(getSphKernel(SphKernelType::sinc_n, sincIndex), 2.0);
        auto a  = tabulateFunction<double, lt::kTableSize>(getSphKernel(SphKernelType::sinc_n, sincIndex), 0, 2);
        auto b  = tabulateFunction<double, lt::kTableSize>(getSphKernelDerivative(SphKernelType::sinc_n, sincIndex), 0, 2);
        std::memcpy(wh, a.data(), sizeof(double) * lt::kTableSize);
        std::memcpy(whd, b.data(), sizeof(double) * lt::kTableSize);
    }

    double ref_sphynx_3d_k(double n) { return sphynx_3D_k(n); }

    void ref_jloop_xmass(size_t numTargets, const uint32_t* targets, double K, const double* lim, int periodic,
                         const uint32_t* nbr, const unsigned* count, unsigned ngmax, const double* x, const double* y,
                         const double* z, const double* h, const double* m, const double* wh, const double* whd,
                         double* xmOut)
    {
        auto box = mkBox(lim, periodic);
        for (size_t t = 0; t < numTargets; ++t)
        {
            unsigned i = targets[t];
            xmOut[t]   = xmassJLoop(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, h, m, wh, whd);
        }
    }

    void ref_jloop_ve_def_gradh(size_t numTargets, const uint32_t* targets, double K, const double* lim, int periodic,
                                const uint32_t* nbr, const unsigned* count, unsigned ngmax, const double* x,
                                const double* y, const double* z, const double* h, const double* m, const double* wh,
                                const double* whd, const double* xm, double* kxOut, double* gradhOut)
    {
        auto box = mkBox(lim, periodic);
        for (size_t t = 0; t < numTargets; ++t)
        {
            unsigned i       = targets[t];
            auto [kx, gradh] = veDefGradhJLoop(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, h, m, wh, whd, xm);
            kxOut[t]         = kx;
            gradhOut[t]      = gradh;
        }
    }

    //! out: 6 IAD components per target, then divv, curlv, dV11..dV33 (8) -> 14 doubles per target
    void ref_jloop_iad_divv_curlv(size_t numTargets, const uint32_t* targets, double K, const double* lim, int periodic,
                                  const uint32_t* nbr, const unsigned* count, unsigned ngmax, const double* x,
                                  const double* y, const double* z, const double* vx, const double* vy,
                                  const double* vz, const double* h, const double* wh, const double* whd,
                                  const double* xm, const double* kx, const double* c11, const double* c12,
                                  const double* c13, const double* c22, const double* c23, const double* c33,
                                  double* out)
    {
        auto box = mkBox(lim, periodic);
        for (size_t t = 0; t < numTargets; ++t)
        {
            unsigned i = targets[t];
            double* o  = out + 14 * t;
            // IAD writes c_ij at index i of its output arrays: route them to local scalars
            std::vector<double> tmp(6 * (size_t(i) + 1));
            IADJLoop(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, h, wh, whd, xm, kx, tmp.data(),
                     tmp.data() + (i + 1), tmp.data() + 2 * (i + 1), tmp.data() + 3 * (i + 1),
                     tmp.data() + 4 * (i + 1), tmp.data() + 5 * (i + 1));
            for (int c = 0; c < 6; ++c)
            {
                o[c] = tmp[c * (size_t(i) + 1) + i];
            }
            std::vector<double> dv(8 * (size_t(i) + 1));
            size_t st = size_t(i) + 1;
            divV_curlVJLoop(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, vx, vy, vz, h, c11, c12, c13, c22,
                            c23, c33, wh, whd, kx, xm, dv.data(), dv.data() + st, dv.data() + 2 * st,
                            dv.data() + 3 * st, dv.data() + 4 * st, dv.data() + 5 * st, dv.data() + 6 * st,
                            dv.data() + 7 * st, true);
            for (int c = 0; c < 8; ++c)
            {
                o[6 + c] = dv[c * st + i];
            }
        }
    }

    void ref_jloop_av_switches(size_t numTargets, const uint32_t* targets, double K, const double* lim, int periodic,
                               const uint32_t* nbr, const unsigned* count, unsigned ngmax, const double* x,
                               const double* y, const double* z, const double* vx, const double* vy, const double* vz,
                               const double* h, const double* c, const double* c11, const double* c12,
                               const double* c13, const double* c22, const double* c23, const double* c33,
                               const double* wh, const double* whd, const double* kx, const double* xm,
                               const double* divv, double dt, double alphamin, double alphamax, double decay,
                               const double* alphaIn, double* alphaOut)
    {
        auto box = mkBox(lim, periodic);
        for (size_t t = 0; t < numTargets; ++t)
        {
            unsigned i  = targets[t];
            alphaOut[t] = AVswitchesJLoop(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, vx, vy, vz, h, c, c11,
                                          c12, c13, c22, c23, c33, wh, whd, kx, xm, divv, dt, alphamin, alphamax, decay,
                                          alphaIn[i]);
        }
    }

    //! out per target: ax, ay, az, du, maxvsignal (5 doubles); avClean selects the AV-cleaning variant
    void ref_jloop_momentum_energy(size_t numTargets, const uint32_t* targets, int avClean, double K,
                                   const double* lim, int periodic, const uint32_t* nbr, const unsigned* count,
                                   unsigned ngmax, const double* x, const double* y, const double* z,
                                   const double* vx, const double* vy, const double* vz, const double* h,
                                   const double* m, const double* prho, const double* c, const double* c11,
                                   const double* c12, const double* c13, const double* c22, const double* c23,
                                   const double* c33, double Atmin, double Atmax, double ramp, const double* wh,
                                   const double* kx, const double* xm, const double* alpha, const double* dV11,
                                   const double* dV12, const double* dV13, const double* dV22, const double* dV23,
                                   const double* dV33, double* out)
    {
        auto box = mkBox(lim, periodic);
        for (size_t t = 0; t < numTargets; ++t)
        {
            unsigned i = targets[t];
            size_t st  = size_t(i) + 1;
            std::vector<double> buf(4 * st);
            double mvs = 0;
            if (avClean)
            {
                momentumAndEnergyJLoop<true>(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, vx, vy, vz, h, m,
                                             prho, (const double*)nullptr, c, c11, c12, c13, c22, c23, c33, Atmin,
                                             Atmax, ramp, wh, kx, xm, alpha, dV11, dV12, dV13, dV22, dV23, dV33,
                                             buf.data(), buf.data() + st, buf.data() + 2 * st, buf.data() + 3 * st,
                                             &mvs);
            }
            else
            {
                momentumAndEnergyJLoop<false>(i, K, box, nbr + size_t(t) * ngmax, count[t], x, y, z, vx, vy, vz, h,
                                              m, prho, (const double*)nullptr, c, c11, c12, c13, c22, c23, c33, Atmin,
                                              Atmax, ramp, wh, kx, xm, alpha, dV11, dV12, dV13, dV22, dV23, dV33,
                                              buf.data(), buf.data() + st, buf.data() + 2 * st, buf.data() + 3 * st,
                                              &mvs);
            }
            double* o = out + 5 * t;
            o[0]      = buf[i];
            o[1]      = buf[st + i];
            o[2]      = buf[2 * st + i];
            o[3]      = buf[3 * st + i];
            o[4]      = mvs;
        }
    }

    //! @brief reference Hilbert keys for a coordinate array (sfc.hpp:267-275), removeKey entries preserved
    void ref_sfc_keys(size_t n, const double* x, const double* y, const double* z, const double* lim, int periodic,
                      uint64_t* keys)
    {
        auto box = mkBox(lim, periodic);
        cstone::computeSfcKeys(x, y, z, cstone::sfcKindPointer(keys), n, box);
    }

    //! @brief reference fully converged cornerstone tree (csarray.hpp:432-440) for sorted keys
    size_t ref_compute_octree(size_t n, const uint64_t* keys, unsigned bucketSize, uint64_t* leavesOut,
                              unsigned* countsOut, size_t cap)
    {
        auto [tree, counts] = cstone::computeOctree<uint64_t>({keys, n}, bucketSize);
        size_t numL         = tree.size() - 1;
        if (numL + 1 <= cap)
        {
            std::memcpy(leavesOut, tree.data(), (numL + 1) * sizeof(uint64_t));
            std::memcpy(countsOut, counts.data(), numL * sizeof(unsigned));
        }
        return numL;
    }

    /*! @brief the reference's internal octree of a cornerstone leaf array (buildOctreeCpu via updateInternalTree,
     *  cstone/tree/octree.hpp:170-196,358-364) in its OctreeData layout: prefixes, childOffsets, parents,
     *  levelRange (maxTreeLevel + 2), internalToLeaf, leafToInternal; returns numNodes */
    int ref_build_octree(const uint64_t* leaves, size_t numLeaves, uint64_t* prefixes, int* childOffsets,
                         int* parents, int* levelRange, int* internalToLeaf, int* leafToInternal)
    {
        std::vector<uint64_t> tree(leaves, leaves + numLeaves + 1);
        cstone::OctreeData<uint64_t, CpuTag> octree;
        octree.resize(cstone::nNodes(tree));
        cstone::updateInternalTree<uint64_t>(tree, octree.data());
        int nn = octree.numNodes;
        std::copy(octree.prefixes.begin(), octree.prefixes.begin() + nn, prefixes);
        std::copy(octree.childOffsets.begin(), octree.childOffsets.begin() + nn, childOffsets);
        std::copy(octree.parents.begin(), octree.parents.end(), parents);
        std::copy(octree.levelRange.begin(), octree.levelRange.end(), levelRange);
        std::copy(octree.internalToLeaf.begin(), octree.internalToLeaf.begin() + nn, internalToLeaf);
        std::copy(octree.leafToInternal.begin(), octree.leafToInternal.begin() + nn, leafToInternal);
        return nn;
    }

    //! @brief reference neighbour search (findneighbors.hpp:77-170) on a fully converged bucket tree of sorted keys
    int ref_find_neighbors(size_t n, const uint64_t* keys, const double* x, const double* y, const double* z,
                           const double* h, const double* lim, int periodic, unsigned bucketSize, unsigned ngmax,
                           uint32_t* nbr, unsigned* count)
    {
        auto box            = mkBox(lim, periodic);
        auto [tree, counts] = cstone::computeOctree<uint64_t>({keys, n}, bucketSize);
        cstone::OctreeData<uint64_t, CpuTag> octree;
        octree.resize(cstone::nNodes(tree));
        cstone::updateInternalTree<uint64_t>(tree, octree.data());
        std::vector<cstone::LocalIndex> layout(counts.size() + 1, 0);
        std::inclusive_scan(counts.begin(), counts.end(), layout.begin() + 1);
        std::vector<cstone::Vec3<double>> centers(octree.numNodes), sizes(octree.numNodes);
        cstone::nodeFpCenters<uint64_t>(octree.prefixes, centers.data(), sizes.data(), box);
        cstone::OctreeNsView<double, uint64_t> view{octree.numLeafNodes,
                                                    octree.prefixes.data(),
                                                    octree.childOffsets.data(),
                                                    octree.parents.data(),
                                                    octree.internalToLeaf.data(),
                                                    octree.levelRange.data(),
                                                    tree.data(),
                                                    layout.data(),
                                                    centers.data(),
                                                    sizes.data()};
        cstone::findNeighbors(x, y, z, h, 0, cstone::LocalIndex(n), box, view, ngmax, nbr, count);
        return 0;
    }

    //! @brief leaf counts of sorted keys in a cornerstone tree (computeNodeCounts, csarray.hpp:181-235)
    void ref_leaf_counts(const uint64_t* leaves, size_t numLeaves, const uint64_t* keys, size_t n, unsigned* counts)
    {
        cstone::computeNodeCounts(leaves, counts, cstone::TreeNodeIndex(numLeaves), std::span<const uint64_t>(keys, n),
                                  std::numeric_limits<unsigned>::max(), false);
    }

    /*! @brief one rebalance step on given counts (rebalanceDecision + rebalanceTree, csarray.hpp:309-389);
     *  returns the new leaf count (newLeaves receives it + 1 keys if it fits), *converged = rebalanceDecision's result */
    size_t ref_rebalance_tree(const uint64_t* leaves, size_t numLeaves, const unsigned* counts, unsigned bucket,
                              uint64_t* newLeaves, size_t capacity, int* converged)
    {
        std::vector<uint64_t> tree(leaves, leaves + numLeaves + 1), newTree;
        std::vector<cstone::TreeNodeIndex> ops(numLeaves + 1);
        *converged = cstone::rebalanceDecision(tree.data(), counts, cstone::TreeNodeIndex(numLeaves), bucket,
                                               ops.data());
        cstone::rebalanceTree(tree, newTree, ops.data());
        size_t nl = newTree.size() - 1;
        if (nl + 1 <= capacity) { std::copy(newTree.begin(), newTree.end(), newLeaves); }
        return nl;
    }

    /*! @brief halo flags per leaf of the rank owning leaves [firstNode, lastNode) of a cornerstone tree, as
     *  FocusedOctree::discoverHalos computes them on the CPU (octree_focus_mpi.hpp:556-569): leaf search boxes by
     *  computeBoundingBox started at the leaf centres, then findHalos over the linked octree; the node flags are read
     *  per leaf through leafToInternal as computeNodeLayout does (layout.hpp:151-177). h is double, or float when hf
     *  is given. layout: numAssigned + 1 particle offsets. */
    void ref_find_halos(const uint64_t* leaves, size_t numLeaves, const double* x, const double* y, const double* z,
                        const double* h, const float* hf, const unsigned* layout, int firstNode, int lastNode,
                        const double* lim, int periodic, float searchExt, uint8_t* leafFlags)
    {
        auto box = mkBox(lim, periodic);
        std::vector<uint64_t> tree(leaves, leaves + numLeaves + 1);
        cstone::OctreeData<uint64_t, CpuTag> octree;
        octree.resize(cstone::nNodes(tree));
        cstone::updateInternalTree<uint64_t>(tree, octree.data());
        int nn = octree.numNodes;
        std::vector<cstone::Vec3<double>> centers(nn), sizes(nn);
        cstone::nodeFpCenters<uint64_t>(octree.prefixes, centers.data(), sizes.data(), box);
        const int* l2i = octree.leafToInternal.data() + octree.numInternalNodes;
        std::vector<cstone::Vec3<double>> searchCenters(numLeaves), searchSizes(numLeaves);
        for (size_t l = 0; l < numLeaves; ++l)
        {
            searchCenters[l] = centers[l2i[l]];
        }
        for (int leaf = firstNode; leaf < lastNode; ++leaf)
        {
            int i = leaf - firstNode;
            if (hf)
            {
                std::tie(searchCenters[leaf], searchSizes[leaf]) = cstone::computeBoundingBox(
                    x, y, z, hf, layout[i], layout[i + 1], float(2 * searchExt), searchCenters[leaf]);
            }
            else
            {
                std::tie(searchCenters[leaf], searchSizes[leaf]) = cstone::computeBoundingBox(
                    x, y, z, h, layout[i], layout[i + 1], double(2 * searchExt), searchCenters[leaf]);
            }
        }
        std::vector<uint8_t> flags(nn, 0);
        cstone::findHalos(octree.prefixes.data(), octree.childOffsets.data(), octree.parents.data(), centers.data(),
                          sizes.data(), tree.data(), searchCenters.data(), searchSizes.data(), box, firstNode,
                          lastNode, flags.data());
        for (size_t l = 0; l < numLeaves; ++l)
        {
            leafFlags[l] = flags[l2i[l]];
        }
    }

    /*! @brief the SFC assignment of numRanks ranks on a global tree (makeSfcAssignment, domaindecomp.hpp:112-127):
     *  rank boundary keys (numRanks + 1), first leaf of every rank (numRanks + 1) and particles per rank */
    void ref_sfc_assignment(int numRanks, const unsigned* counts, size_t numLeaves, const uint64_t* leaves,
                            uint64_t* boundaries, int* treeOffsets, unsigned* rankCounts)
    {
        std::vector<unsigned> c(counts, counts + numLeaves);
        auto a = cstone::makeSfcAssignment(numRanks, c, leaves);
        for (int r = 0; r <= numRanks; ++r)
        {
            boundaries[r]  = a[r];
            treeOffsets[r] = a.treeOffsetsConst()[r];
            if (r < numRanks) { rankCounts[r] = a.totalCount(r); }
        }
    }
}
