// Device side of the block time-step propagator (main/src/propagator/ve_hydro_bdt.hpp): per-group time steps,
// their sort into rungs, the EOS over every particle, and drift / kick-drift of the particles of each rung.
#pragma once

#include "common.cuh"
#include "hydro.cuh"
#include "integrate.cuh"

namespace sphb
{

//! Timestep::maxNumRungs (sph/include/sph/timestep.h:19)
constexpr int kMaxRungs = 4;

//! the previous full step per rung, indexed by the rung a particle was last advanced on
struct RungSteps
{
    float dtm1[kMaxRungs];
};

/*! computeEOS over every particle (ve_hydro_bdt.hpp:244-245): prho and c from the stored kx, xm, gradh and temp,
 *  and the neighbour-side records of every particle refreshed from its current velocity, h, c and prho (the J-loops
 *  of the active groups read them for inactive neighbours too). */
template<class T>
int launchEosRefresh(const ChainArrays<T>& a, const HydroConsts<T>& k, cudaStream_t s);

//! groupDivvTimestepGpu (sph/include/sph/ts_groups.cu:17-45): groupDt[w] = min(groupDt[w], Krho / |max divv|)
template<class T>
int launchGroupDivv(const uint32_t* groups, unsigned num, const uint32_t* bounds, const T* divv, float Krho, float* groupDt,
                    cudaStream_t s);

//! groupAccTimestepGpu (ts_groups.cu:47-80): groupDt[w] = min(groupDt[w], etaAcc (min h^2 / |a|^2)^(1/4))
template<class T>
int launchGroupAcc(const uint32_t* groups, unsigned num, const uint32_t* bounds, const T* ax, const T* ay, const T* az,
                   const double* h, float etaAcc, float* groupDt, cudaStream_t s);

/*! driftPositionsGpu (sph/include/sph/positions_gpu.cu:45-90): recover the state at the start of the rung's step by
 *  going back dtBack, then go forward dt from there, with the acceleration and x_m1 of that start; no periodic
 *  folding. Updates x, v and temp. */
template<class T>
int launchDrift(const uint32_t* groups, unsigned num, const uint32_t* bounds, float dt, float dtBack, RungSteps steps,
                const uint64_t* rung, const IntegrateArrays<T>& a, double cv, cudaStream_t s);

/*! computePositionsGpu (positions_gpu.cu:117-166) over the groups of one rung: kick-drift by dt with the previous
 *  step of each particle's last rung, energy update, du_m1 = du. box.periodic all zero: no folding. */
template<class T>
int launchRungPositions(const uint32_t* groups, unsigned num, const uint32_t* bounds, float dt, RungSteps steps,
                        const uint64_t* rung, const IntegrateArrays<T>& a, const DevBox& box, double cv,
                        cudaStream_t s);

//! storeRungGpu (ts_groups.cu:82-104): rung of every particle of the listed groups
int launchStoreRung(const uint32_t* groups, unsigned num, const uint32_t* bounds, uint64_t value, uint64_t* rung, cudaStream_t s);

//! updateSmoothingLength over the listed groups (sph/include/sph/update_h.hpp:33-47)
int launchListUpdateH(const uint32_t* groups, unsigned num, const uint32_t* bounds, unsigned ng0, const unsigned* nc, double* h,
                      uint64_t* keys, unsigned* flag, cudaStream_t s);

//! out = ordered bits of max_i max_k |x_k,i - xs_k,i| (minimum image on periodic axes); out must hold the bits of 0
int launchMaxDisplacement(const double* x, const double* y, const double* z, const double* xs, const double* ys,
                          const double* zs, size_t n, const DevBox& box, unsigned long long* out, cudaStream_t s);

//! keys[w] = bit pattern of groupDt[w] (non-negative floats sort like their bits), values[w] = w
int launchDtKeys(const float* groupDt, unsigned num, uint64_t* keys, uint32_t* values, cudaStream_t s);

/*! After the sort: groupDt[w] = float of keys[w]; out[0] = smallest dt, out[1] = dt at index fastIdx,
 *  out[1 + r] = lower bound of 2^r * smallest dt in the sorted dt (r = 1..3) (ts_rungs.hpp:92-146) */
int launchSortedDt(const uint64_t* keys, unsigned num, unsigned fastIdx, float* groupDt, uint32_t* out,
                   cudaStream_t s);

//! dst[w] = src[idx[w]] for w < num (extractGroupGpu, sph/include/sph/groups.hpp:77-93)
int launchGatherGroups(const uint32_t* src, const uint32_t* idx, unsigned num, uint32_t* dst, cudaStream_t s);

//! list[w] = w + first for w < num
int launchSequence(uint32_t* list, unsigned num, uint32_t first, cudaStream_t s);

} // namespace sphb
