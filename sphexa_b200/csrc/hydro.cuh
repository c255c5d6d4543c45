// Device helpers and launch interface of the SPH-VE chain (see hydro_ve.cu).
#pragma once

#include "common.cuh"

namespace sphb
{

//! number of coefficients of the FP32 polynomial kernel (degree 12 in t)
constexpr int kPolyTerms = 13;

//! largest block size a J-loop launch may use (ChainArrays::threads; the ensemble autotuner picks 64, 128 or 256)
constexpr int kChainMaxThreads = 256;
constexpr int kAvMaxThreads    = 384; // the AV switches, which need no block reduction

//! physics constants of one simulation, in the J-loop type T
template<class T>
struct HydroConsts
{
    T K;           // kernel normalisation
    T alphamin, alphamax, decay;
    T Atmin, Atmax, ramp;
    double Kcour;  // stored as the float the reference passes to tsKCourant (sph/include/sph/kernels.hpp:10-17)
    double gamma, cv;
    unsigned ngmax;
    // FP32 path only: polynomial kernel W(v) = P(t), dW/dv = v Q(t), t = v^2/2 - 1 (instead of table lookups)
    int usePoly;
    float wpoly[kPolyTerms];
    float dwpoly[kPolyTerms];
    // FP32 path only: length of one unit of the 32-bit fixed-point coordinates, per axis (box length / 2^32)
    float qscale[3];
};

/*! Per-particle neighbour-side records, written by the stage that produces the values and gathered once per
 *  neighbour by the next stages (one 16-byte-aligned record instead of one scattered load per field).
 *  pos:   x, y, z, m            (double; FP64 path)
 *  posq:  qx, qy, qz, m         (FP32 path: coordinates as 32-bit fixed point over the box, q = (x - lo) 2^32 / L,
 *                                m as float bits; the int32 difference of two q is the pair separation in units of
 *                                L / 2^32, wrapped to the nearest periodic image by integer overflow)
 *  hydro: vx, vy, vz, 1/h, xm, xm/kx, c, prho   (T; written by VeDefGradh+EOS)
 *  grad:  c11, c12, c13, c22, c23, c33, divv, alpha   (T; c_ij and divv by IAD, alpha by the AV switches) */
template<class T>
struct alignas(8 * sizeof(T)) HydroRec
{
    T vx, vy, vz, hInv, xm, vol, c, prho; // hInv = 1/h, vol = xm/kx
};

template<class T>
struct alignas(8 * sizeof(T)) GradRec
{
    T c11, c12, c13, c22, c23, c33, divv, alpha;
};

/*! Neighbour-side record of the AV switches, written by IAD: velocity, sound speed, xm/kx and divv (one 32-byte
 *  gather per neighbour instead of three records). */
template<class T>
struct alignas(8 * sizeof(T)) AVRec
{
    T vx, vy, vz, c, vol, divv;
    T pad0, pad1;
};

/*! AV cleaning only: the symmetrised velocity gradient of a particle (dV11, dV12 = dVxy + dVyx, dV13, dV22, dV23,
 *  dV33, each times K / (h^3 kx); divv_curlv_kern.hpp:114-122), written by IAD, read per neighbour by
 *  MomentumEnergy. */
template<class T>
struct alignas(8 * sizeof(T)) DVRec
{
    T dv[6];
    T pad0, pad1;
};

/*! Intermediate values the adjoint of the chain needs and the outputs do not determine; written only when the
 *  pointers are set (a step recomputed for its adjoint). whomega, wrho0: the two kernel-derivative sums of VeDefGradh
 *  after normalisation; gx, gy, gz, vsig, vsigJ: the divv gradient, the signal velocity of the AV switches and the
 *  neighbour that set it (-1: none); energy, avisc: the energy and viscous-energy sums of MomentumEnergy. */
template<class T>
struct ChainTape
{
    T* whomega{nullptr};
    T* wrho0{nullptr};
    T* gx{nullptr};
    T* gy{nullptr};
    T* gz{nullptr};
    T* vsig{nullptr};
    int* vsigJ{nullptr};
    T* energy{nullptr};
    T* avisc{nullptr};
};

//! device arrays of one simulation used by the chain; derived fields are stored in T
template<class T>
struct ChainArrays
{
    size_t n;
    const double4* pos;       // x, y, z, m (FP64 path)
    const int4* posq;         // fixed-point x, y, z and float m (FP32 path)
    const double* h;          // smoothing length (FP64 state)
    const double* vx;
    const double* vy;
    const double* vz;
    const double* temp;
    double* alpha;            // AV coefficient (FP64 state)
    const uint32_t* nidx;
    const unsigned* nc;
    const T* wh;
    const T* whd;
    T* xm;
    T* kx;
    T* gradh;
    T* prho;
    T* c;
    T* cij[6];
    T* divv;
    T* curlv;
    T* ax;
    T* ay;
    T* az;
    double* du;
    HydroRec<T>* hrec;
    GradRec<T>* grec;
    // reduction outputs: [0] max divv (ordered bits), [1] min Courant dt (ordered bits)
    unsigned long long* reduce;
    ChainTape<T> tape;
    BatchView batch;
    AVRec<T>* avrec{nullptr};
    // VeDefGradh leaves the velocity of the hydro record to launchPackVelocity (the velocities of a typed host load
    // still in flight)
    bool recordNoVelocity{false};
    DVRec<T>* dvrec{nullptr}; // set: AV cleaning (HydroVeProp<avClean = true>)
    T* dv[6]{};              // the same six fields as arrays (dV11 .. dV33)
    int threads{128}; // block size of the J-loop launches
    // block time steps: the launch covers only the groups groupList[0, numListed) (one warp each); group g holds
    // the particles [groupBounds[g], groupBounds[g + 1]) (at most 32, the spatial target groups); MomentumEnergy
    // then lowers groupDt[w] of listed group w to the Courant step of its particles
    const uint32_t* groupList{nullptr};
    const uint32_t* groupBounds{nullptr};
    unsigned numListed{0};
    float* groupDt{nullptr};
};

template<class T>
int launchXMass(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s);
template<class T>
int launchVeDefGradhEos(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s);
//! the velocity of every particle into its hydro record (after a VeDefGradh with recordNoVelocity)
template<class T>
int launchPackVelocity(const ChainArrays<T>& a, cudaStream_t s);
template<class T>
int launchIadDivvCurlv(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s);
template<class T>
int launchAVswitches(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, double dt,
                     cudaStream_t s);
template<class T>
int launchMomentumEnergy(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s);

//! order-preserving bit patterns of doubles for atomic min/max
__host__ __device__ inline unsigned long long orderedBits(double v)
{
#ifdef __CUDA_ARCH__
    long long b = __double_as_longlong(v);
#else
    long long b;
    static_assert(sizeof(b) == sizeof(v));
    __builtin_memcpy(&b, &v, sizeof(b));
#endif
    return b >= 0 ? (unsigned long long)(b) ^ 0x8000000000000000ull : ~(unsigned long long)(b);
}

__host__ __device__ inline double fromOrderedBits(unsigned long long u)
{
    unsigned long long b = (u & 0x8000000000000000ull) ? (u ^ 0x8000000000000000ull) : ~u;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double v;
    __builtin_memcpy(&v, &b, sizeof(v));
    return v;
#endif
}

} // namespace sphb
