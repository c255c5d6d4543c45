/* The GPU stage functions of SPH-EXA's VE propagator (sph/include/sph/sph_gpu.hpp:24-87) implemented on sphb200.
 *
 * A maintainer of the reference builds this file into the reference in place of the definitions in
 * sph/include/sph/hydro_ve/{xmass,ve_def_gradh,eos,iad_divv_curlv,av_switches,momentum_energy}_gpu.cu and of the
 * global-step kernels of sph/include/sph/{positions,update_h}_gpu.cu, adds include/ of this repository to the include
 * path and links libsphb200.so. Nothing else in the reference changes: HydroVeProp (main/src/propagator/ve_hydro.hpp)
 * keeps calling sph::gpu::computeXMass(grp, d, box) and its siblings.
 *
 * The Dataset's device arrays (DeviceVector fields of ParticlesData, sph/include/sph/particles_data.hpp:218-246) are
 * bound by field name, in their own element types (SphTypes, sph/types.hpp:39-46), to one sphb_sim; the binding is
 * renewed whenever a field's array moves (a DeviceVector reallocated) or the particle count changes. The stages then
 * run in place on those arrays. Errors throw std::runtime_error, as the reference's traversal-stack check does
 * (sph/include/sph/hydro_ve/xmass_gpu.cu:123).
 *
 * Scope: one rank without halos (GroupView = all particles), the global time step, avClean = false. Block time
 * steps (a non-null groupDt or rung array) and AV cleaning throw.
 *
 * SPHB_SHIM_PRECISION selects the neighbour sums: SPHB_MIXED (FP32 sums, the default, matching the reference's float
 * hydro types) or SPHB_FP64.
 */
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "cstone/cuda/device_vector.h"
#include "sph/particles_data.hpp"
#include "sph/sph_gpu.hpp"
#include "sphb200.h"

#ifndef SPHB_SHIM_PRECISION
#define SPHB_SHIM_PRECISION SPHB_MIXED
#endif

namespace sphb_shim
{

template<class T>
constexpr int dtypeOf()
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

inline void check(int rc, const char* what)
{
    if (rc != SPHB_OK)
    {
        throw std::runtime_error(std::string("sphb200: ") + what + " returned status " + std::to_string(rc));
    }
}

struct Binding
{
    sphb_sim* sim{nullptr};
    std::vector<sphb_field> fields;
};

inline Binding& binding()
{
    static Binding b;
    return b;
}

template<class Vec>
void addField(std::vector<sphb_field>& f, const char* name, Vec& v, size_t n)
{
    using T = typename Vec::value_type;
    if (v.size() == n) { f.push_back({name, static_cast<void*>(rawPtr(v)), dtypeOf<T>()}); }
}

//! every field of the Dataset that the VE stages read or write, by the reference's names
template<class Dataset>
std::vector<sphb_field> datasetFields(Dataset& d)
{
    size_t n = d.x.size();
    std::vector<sphb_field> f;
    addField(f, "x", d.x, n);
    addField(f, "y", d.y, n);
    addField(f, "z", d.z, n);
    addField(f, "h", d.h, n);
    addField(f, "m", d.m, n);
    addField(f, "temp", d.temp, n);
    addField(f, "vx", d.vx, n);
    addField(f, "vy", d.vy, n);
    addField(f, "vz", d.vz, n);
    addField(f, "x_m1", d.x_m1, n);
    addField(f, "y_m1", d.y_m1, n);
    addField(f, "z_m1", d.z_m1, n);
    addField(f, "du_m1", d.du_m1, n);
    addField(f, "alpha", d.alpha, n);
    addField(f, "xm", d.xm, n);
    addField(f, "kx", d.kx, n);
    addField(f, "gradh", d.gradh, n);
    addField(f, "prho", d.prho, n);
    addField(f, "c", d.c, n);
    addField(f, "c11", d.c11, n);
    addField(f, "c12", d.c12, n);
    addField(f, "c13", d.c13, n);
    addField(f, "c22", d.c22, n);
    addField(f, "c23", d.c23, n);
    addField(f, "c33", d.c33, n);
    addField(f, "divv", d.divv, n);
    addField(f, "curlv", d.curlv, n);
    addField(f, "ax", d.ax, n);
    addField(f, "ay", d.ay, n);
    addField(f, "az", d.az, n);
    addField(f, "du", d.du, n);
    addField(f, "nc", d.nc, n);
    addField(f, "keys", d.keys, n);
    addField(f, "id", d.id, n);
    return f;
}

inline bool sameFields(const std::vector<sphb_field>& a, const std::vector<sphb_field>& b)
{
    if (a.size() != b.size()) { return false; }
    for (size_t q = 0; q < a.size(); ++q)
    {
        if (std::string(a[q].name) != b[q].name || a[q].data != b[q].data || a[q].dtype != b[q].dtype) { return false; }
    }
    return true;
}

template<class T>
sphb_box toBox(const cstone::Box<T>& box)
{
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
    return b;
}

//! the simulation object bound to the Dataset's current arrays (created on the first call)
template<class Dataset>
sphb_sim* simFor(Dataset& d, const sphb_box& box)
{
    Binding& b = binding();
    auto f     = datasetFields(d);
    size_t n   = d.x.size();
    if (b.sim && sphb_sim_size(b.sim) == n && sameFields(f, b.fields)) { return b.sim; }
    if (b.sim && sphb_sim_size(b.sim) != n)
    {
        sphb_sim_destroy(b.sim);
        b.sim = nullptr;
    }
    if (!b.sim)
    {
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
        p.precision      = SPHB_SHIM_PRECISION;
        check(sphb_sim_create(&b.sim, n, &box, &p), "sphb_sim_create");
    }
    check(sphb_sim_bind_fields(b.sim, f.data(), int(f.size())), "sphb_sim_bind_fields");
    b.fields = std::move(f);
    return b.sim;
}

//! the bound simulation, for the raw-pointer functions: ptr must be the bound array of the named field
inline sphb_sim* boundSim(const char* name, const void* ptr)
{
    Binding& b = binding();
    if (!b.sim) { throw std::runtime_error("sphb200: no Dataset bound (computeXMass runs first)"); }
    for (const auto& f : b.fields)
    {
        if (std::string(f.name) == name && f.data == ptr) { return b.sim; }
    }
    throw std::runtime_error(std::string("sphb200: the array of ") + name + " is not the bound Dataset's");
}

} // namespace sphb_shim

namespace sph
{
namespace gpu
{

template<class Dataset>
void computeXMass(const GroupView& grp, Dataset& d, const cstone::Box<typename Dataset::RealType>& box)
{
    sphb_box b  = sphb_shim::toBox(box);
    sphb_sim* s = sphb_shim::simFor(d, b);
    sphb_shim::check(sphb_dataset_xmass(s, grp.firstBody, grp.lastBody, &b), "computeXMass");
}

template<class Dataset>
void computeVeDefGradh(const GroupView& grp, Dataset& d, const cstone::Box<typename Dataset::RealType>& box)
{
    sphb_box b  = sphb_shim::toBox(box);
    sphb_sim* s = sphb_shim::simFor(d, b);
    sphb_shim::check(sphb_dataset_ve_def_gradh(s, grp.firstBody, grp.lastBody, &b), "computeVeDefGradh");
}

template<class Dataset>
void computeIadDivvCurlv(const GroupView& grp, Dataset& d, const cstone::Box<typename Dataset::RealType>& box)
{
    sphb_box b  = sphb_shim::toBox(box);
    sphb_sim* s = sphb_shim::simFor(d, b);
    sphb_shim::check(sphb_dataset_iad_divv_curlv(s, grp.firstBody, grp.lastBody, &b), "computeIadDivvCurlv");
}

template<class Dataset>
void computeAVswitches(const GroupView& grp, Dataset& d, const cstone::Box<typename Dataset::RealType>& box)
{
    sphb_box b  = sphb_shim::toBox(box);
    sphb_sim* s = sphb_shim::simFor(d, b);
    sphb_shim::check(sphb_dataset_av_switches(s, grp.firstBody, grp.lastBody, &b, d.minDt), "computeAVswitches");
}

template<bool avClean, class Dataset>
void computeMomentumEnergy(const GroupView& grp, float* groupDt, Dataset& d,
                           const cstone::Box<typename Dataset::RealType>& box)
{
    if (avClean || groupDt) { throw std::runtime_error("sphb200: AV cleaning and block time steps are not bound"); }
    sphb_box b  = sphb_shim::toBox(box);
    sphb_sim* s = sphb_shim::simFor(d, b);
    float minDt = 0.f;
    sphb_shim::check(sphb_dataset_momentum_energy(s, grp.firstBody, grp.lastBody, &b, &minDt),
                     "computeMomentumEnergy");
    d.minDtCourant = minDt;
}

template<class Tt, class Tm, class Thydro>
void computeIdealGasEOS(size_t firstParticle, size_t lastParticle, Tm mui, Tt gamma, const Tt* temp, const Tt* u,
                        const Tm* m, const Thydro* kx, const Thydro* xm, const Thydro* gradh, Thydro* prho, Thydro* c,
                        Thydro* rho, Thydro* p)
{
    using sphb_shim::dtypeOf;
    std::vector<sphb_field> f;
    auto add = [&](const char* name, const void* ptr, int dtype) {
        if (ptr) { f.push_back({name, const_cast<void*>(ptr), dtype}); }
    };
    add(u ? "u" : "temp", u ? static_cast<const void*>(u) : static_cast<const void*>(temp), dtypeOf<Tt>());
    add("m", m, dtypeOf<Tm>());
    add("kx", kx, dtypeOf<Thydro>());
    add("xm", xm, dtypeOf<Thydro>());
    add("gradh", gradh, dtypeOf<Thydro>());
    add("prho", prho, dtypeOf<Thydro>());
    add("c", c, dtypeOf<Thydro>());
    add("rho", rho, dtypeOf<Thydro>());
    add("p", p, dtypeOf<Thydro>());
    sphb_shim::check(sphb_ideal_gas_eos(firstParticle, lastParticle, double(mui), double(gamma), f.data(),
                                        int(f.size()), nullptr),
                     "computeIdealGasEOS");
    sphb_shim::check(cudaDeviceSynchronize() == cudaSuccess ? SPHB_OK : SPHB_ERR_CUDA, "computeIdealGasEOS");
}

template void computeXMass(const GroupView&, sphexa::ParticlesData<cstone::GpuTag>&,
                           const cstone::Box<SphTypes::CoordinateType>&);
template void computeVeDefGradh(const GroupView&, sphexa::ParticlesData<cstone::GpuTag>&,
                                const cstone::Box<SphTypes::CoordinateType>&);
template void computeIadDivvCurlv(const GroupView&, sphexa::ParticlesData<cstone::GpuTag>&,
                                  const cstone::Box<SphTypes::CoordinateType>&);
template void computeAVswitches(const GroupView&, sphexa::ParticlesData<cstone::GpuTag>&,
                                const cstone::Box<SphTypes::CoordinateType>&);
template void computeMomentumEnergy<false>(const GroupView&, float*, sphexa::ParticlesData<cstone::GpuTag>&,
                                           const cstone::Box<SphTypes::CoordinateType>&);
template void computeMomentumEnergy<true>(const GroupView&, float*, sphexa::ParticlesData<cstone::GpuTag>&,
                                          const cstone::Box<SphTypes::CoordinateType>&);
template void computeIdealGasEOS(size_t, size_t, SphTypes::Tmass, SphTypes::CoordinateType,
                                 const SphTypes::CoordinateType*, const SphTypes::CoordinateType*,
                                 const SphTypes::Tmass*, const SphTypes::HydroType*, const SphTypes::HydroType*,
                                 const SphTypes::HydroType*, SphTypes::HydroType*, SphTypes::HydroType*,
                                 SphTypes::HydroType*, SphTypes::HydroType*);

} // namespace gpu

template<class Tc, class Tv, class Ta, class Tdu, class Tm1, class Tu, class Thydro>
void computePositionsGpu(const GroupView& grp, float dt, util::array<float, Timestep::maxNumRungs> dt_m1, Tc* x,
                         Tc* /*y*/, Tc* /*z*/, Tv* /*vx*/, Tv* /*vy*/, Tv* /*vz*/, Tm1* /*x_m1*/, Tm1* /*y_m1*/,
                         Tm1* /*z_m1*/, Ta* /*ax*/, Ta* /*ay*/, Ta* /*az*/, const uint8_t* rung, Tu* /*temp*/,
                         Tu* /*u*/, Tdu* /*du*/, Tm1* /*du_m1*/, Thydro* /*h*/, Thydro* /*mui*/, Tc /*gamma*/,
                         Tc /*constCv*/, const cstone::Box<Tc>& box)
{
    if (rung) { throw std::runtime_error("sphb200: block time steps are not bound"); }
    sphb_sim* s = sphb_shim::boundSim("x", x);
    sphb_box b  = sphb_shim::toBox(box);
    sphb_shim::check(sphb_dataset_positions(s, grp.firstBody, grp.lastBody, dt, dt_m1[0], &b),
                     "computePositionsGpu");
}

template<class Th, class KeyType>
bool updateSmoothingLengthGpu(const GroupView& grp, unsigned ng0, const unsigned* nc, Th* /*h*/, KeyType* /*keys*/)
{
    sphb_sim* s = sphb_shim::boundSim("nc", nc);
    int rc      = sphb_dataset_update_h(s, grp.firstBody, grp.lastBody, ng0);
    if (rc == SPHB_ERR_NOT_CONVERGED) { return true; } // keys of particles with nc <= 1 were set to the removal key
    sphb_shim::check(rc, "updateSmoothingLengthGpu");
    return false;
}

template void computePositionsGpu(const GroupView&, float, util::array<float, Timestep::maxNumRungs>,
                                  SphTypes::CoordinateType*, SphTypes::CoordinateType*, SphTypes::CoordinateType*,
                                  SphTypes::HydroType*, SphTypes::HydroType*, SphTypes::HydroType*,
                                  SphTypes::XM1Type*, SphTypes::XM1Type*, SphTypes::XM1Type*, SphTypes::HydroType*,
                                  SphTypes::HydroType*, SphTypes::HydroType*, const uint8_t*,
                                  SphTypes::CoordinateType*, SphTypes::CoordinateType*, SphTypes::CoordinateType*,
                                  SphTypes::XM1Type*, SphTypes::HydroType*, SphTypes::HydroType*,
                                  SphTypes::CoordinateType, SphTypes::CoordinateType,
                                  const cstone::Box<SphTypes::CoordinateType>&);
template bool updateSmoothingLengthGpu(const GroupView&, unsigned, const unsigned*, SphTypes::HydroType*,
                                       SphTypes::KeyType*);

} // namespace sph
