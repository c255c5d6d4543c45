// Adjoint (vector-Jacobian product) of one VE hydro step with the discrete structure of the step held fixed: the
// sort permutation, the neighbour lists and counts, and the smoothing-length factors chosen by the neighbour-count
// iterations. See adjoint.cu.
#pragma once

#include "hydro.cuh"
#include "integrate.cuh"

namespace sphb
{

//! adjoints of the chain's intermediate fields (J-loop type T), accumulated by scatter from the pair loops
template<class T>
struct AdjArrays
{
    T *x, *y, *z;
    T *vx, *vy, *vz;
    T* h;
    T* c;
    T* prho;
    T* alpha; // of the AV coefficient after the switches
    T* cij[6];
    T* divv;
    T* xm;
    T* vol; // of xm / kx
    T* kx;
    T* gradh;
    T *ax, *ay, *az;
    T* du;
    /*! FP32 only (may be null): the MomentumEnergy adjoint's neighbour-side sums, 5 float4 per particle
     *  {x, y, z, h} {vx, vy, vz, c} {c11, c12, c13, c22} {c23, c33, alpha, prho} {xm, vol, -, -}, added with vector
     *  atomics (5 per pair instead of 18 scalar ones) and folded into the arrays above after that kernel */
    float4* jacc{nullptr};
};

//! number of T arrays in AdjArrays
constexpr int kNumAdjFields = 25;

/*! Adjoint of the conserved state, one double array per field in the order x, y, z, h, m, temp, vx, vy, vz, x_m1,
 *  y_m1, z_m1, du_m1, alpha. */
struct StateAdj
{
    double* f[14];
};

struct AdjointStepArgs
{
    size_t n;
    double dt, dtm1, cv, gamma;
    unsigned ng0;
    const uint32_t* order;   // the step's sort permutation: post-sync i <- pre-sync order[i]
    const double* hPre;      // h after the sync, before the neighbour-count iterations
    const double* alphaPre;  // alpha after the sync, before the AV switches
    const double* temp;      // temp after the sync (the step's input)
    const double* xm1;       // x_m1, y_m1, z_m1, du_m1 after the sync
    const double* ym1;
    const double* zm1;
    const double* duM1;
    const double* du;        // du/dt of the step
    double dtAV;             // the time step the AV switches used
    double* alphamaxBar;     // device scalar, accumulated
};

/*! Given the adjoint of the state after the step (in the step's post-sync particle order) compute the adjoint of the
 *  state before the step (in the pre-sync order). The chain arrays must hold the recomputed forward step with its
 *  tape; work holds kNumAdjFields arrays of n T and scratch 14 arrays of n doubles. */
template<class T>
int stepVjp(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, const AdjointStepArgs& s,
            const StateAdj& post, const StateAdj& pre, AdjArrays<T> g, StateAdj work, cudaStream_t stream);

} // namespace sphb
