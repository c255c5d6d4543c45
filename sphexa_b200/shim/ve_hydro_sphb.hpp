/* A propagator of the reference (main/src/propagator/ipropagator.hpp) whose whole VE step runs on sphb200: the
 * drop-in at the level of HydroVeProp (main/src/propagator/ve_hydro.hpp:48-220). A maintainer registers it next to
 * HydroVeProp in the propagator factory, adds include/ of this repository to the include path and links
 * libsphb200.so.
 *
 * The sphb_sim object owns the particle state in HBM from the first sync on and runs computeForces and integrate
 * itself (domain sync, neighbour search, the VE chain, time step, positions, h update). The Dataset keeps its own
 * fields for output and observables: integrate copies the conserved fields and the chain's outputs back into it, in
 * the Dataset's own element types (SphTypes, sph/types.hpp:39-46), through the typed store. Host or device arrays are
 * handled alike: on_device follows the Dataset's accelerator.
 *
 * Scope: one rank, the global time step, gravity off (g = 0); avClean = true selects HydroVeProp<avClean = true>.
 */
#pragma once

#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "cstone/primitives/primitives_acc.hpp"
#include "propagator/ipropagator.hpp"
#include "sphb200.h"

namespace sphexa
{

template<bool avClean, class DomainType, class DataType>
class HydroVeSphbProp final : public Propagator<DomainType, DataType>
{
    using Base = Propagator<DomainType, DataType>;
    using Acc  = typename DataType::AcceleratorType;

    static constexpr int kOnDevice = cstone::HaveGpu<Acc>{} ? 1 : 0;

    sphb_sim* sim_ = nullptr;

    static void check(int rc, const char* what)
    {
        if (rc != SPHB_OK)
        {
            throw std::runtime_error(std::string("sphb200: ") + what + " returned status " + std::to_string(rc));
        }
    }

    template<class T>
    static constexpr int dtypeOf()
    {
        if constexpr (std::is_same_v<T, float>) { return SPHB_F32; }
        else if constexpr (std::is_same_v<T, double>) { return SPHB_F64; }
        else if constexpr (std::is_same_v<T, unsigned>) { return SPHB_U32; }
        else
        {
            static_assert(std::is_same_v<T, uint64_t>, "field type without an sphb element type");
            return SPHB_U64;
        }
    }

    template<class Vec>
    static void add(std::vector<sphb_field>& f, const char* name, Vec& v)
    {
        using T = typename Vec::value_type;
        f.push_back({name, static_cast<void*>(v.data()), dtypeOf<T>()});
    }

    //! the 14 conserved fields of the VE step and the ids, in the Dataset's own types
    template<class Dataset>
    static std::vector<sphb_field> conserved(Dataset& d)
    {
        std::vector<sphb_field> f;
        add(f, "x", d.x);
        add(f, "y", d.y);
        add(f, "z", d.z);
        add(f, "h", d.h);
        add(f, "m", d.m);
        add(f, "temp", d.temp);
        add(f, "vx", d.vx);
        add(f, "vy", d.vy);
        add(f, "vz", d.vz);
        add(f, "x_m1", d.x_m1);
        add(f, "y_m1", d.y_m1);
        add(f, "z_m1", d.z_m1);
        add(f, "du_m1", d.du_m1);
        add(f, "alpha", d.alpha);
        add(f, "id", d.id);
        return f;
    }

public:
    HydroVeSphbProp(std::ostream& output, size_t rank)
        : Base(output, rank)
    {
    }

    ~HydroVeSphbProp() override
    {
        if (sim_) { sphb_sim_destroy(sim_); }
    }

    std::vector<std::string> conservedFields() const override
    {
        return {"x", "y", "z", "h", "m", "temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha", "id"};
    }

    void activateFields(DataType& simData) override
    {
        auto& d = simData.hydro;
        d.setConserved("x", "y", "z", "h", "m", "temp", "vx", "vy", "vz", "x_m1", "y_m1", "z_m1", "du_m1", "alpha",
                       "id");
        d.setDependent("keys", "ax", "ay", "az", "prho", "c", "du", "c11", "c12", "c13", "c22", "c23", "c33", "xm",
                       "kx", "nc", "gradh", "divv", "curlv");
    }

    //! the first call creates the simulation from the Dataset (the reference's initial Domain::sync); the
    //! simulation runs its own domain sync inside computeForces from then on
    void sync(DomainType& domain, DataType& simData) override
    {
        if (sim_) { return; }
        auto& d         = simData.hydro;
        const auto& box = domain.box();
        sphb_box b;
        b.lo[0]       = box.xmin();
        b.hi[0]       = box.xmax();
        b.lo[1]       = box.ymin();
        b.hi[1]       = box.ymax();
        b.lo[2]       = box.zmin();
        b.hi[2]       = box.zmax();
        b.periodic[0] = box.boundaryX() == cstone::BoundaryType::periodic;
        b.periodic[1] = box.boundaryY() == cstone::BoundaryType::periodic;
        b.periodic[2] = box.boundaryZ() == cstone::BoundaryType::periodic;
        sphb_params p;
        sphb_default_params(&p);
        p.ng0            = d.ng0;
        p.ngmax          = d.ngmax;
        p.gamma          = d.gamma;
        p.mui            = d.muiConst;
        p.Kcour          = d.Kcour;
        p.Krho           = d.Krho;
        p.alphamin       = d.alphamin;
        p.alphamax       = d.alphamax;
        p.decay_constant = d.decay_constant;
        p.sinc_index     = d.sincIndex;
        p.minDt          = d.minDt;
        p.minDt_m1       = d.minDt_m1;
        p.precision      = std::is_same_v<typename DataType::HydroData::HydroType, float> ? SPHB_MIXED : SPHB_FP64;
        p.av_clean       = avClean ? 1 : 0;
        check(sphb_sim_create(&sim_, d.x.size(), &b, &p), "sphb_sim_create");
        auto f = conserved(d);
        check(sphb_sim_upload_fields(sim_, f.data(), int(f.size()), kOnDevice), "sphb_sim_upload_fields");
        check(sphb_sim_initial_sync(sim_), "sphb_sim_initial_sync");
    }

    void computeForces(DomainType&, DataType&) override { check(sphb_sim_compute_forces(sim_), "computeForces"); }

    void integrate(DomainType&, DataType& simData) override
    {
        int rc = sphb_sim_integrate(sim_);
        if (rc != SPHB_OK && rc != SPHB_ERR_NOT_CONVERGED) { check(rc, "integrate"); }
        auto& d = simData.hydro;
        double s[18];
        check(sphb_sim_scalars(sim_, s), "sphb_sim_scalars");
        d.minDt        = s[0];
        d.minDt_m1     = s[1];
        d.minDtCourant = s[2];
        d.minDtRho     = s[3];
        d.ttot         = s[4];
        d.etot         = s[5];
        d.ecin         = s[6];
        d.eint         = s[7];
        d.linmom       = s[8];
        d.angmom       = s[9];
        auto f         = conserved(d);
        add(f, "keys", d.keys);
        add(f, "nc", d.nc);
        add(f, "du", d.du);
        add(f, "xm", d.xm);
        add(f, "kx", d.kx);
        add(f, "divv", d.divv);
        check(sphb_sim_store_fields(sim_, f.data(), int(f.size()), kOnDevice), "sphb_sim_store_fields");
    }
};

} // namespace sphexa
