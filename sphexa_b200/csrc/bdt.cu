// Kernels of the block time-step propagator (main/src/propagator/ve_hydro_bdt.hpp). Each listed group is one warp:
// group g holds the particles [bounds[g], bounds[g + 1]) (the spatial target groups, at most 32 particles); the lists
// are the dt-sorted group ids of one rung or of the active rungs.
#include <algorithm>

#include "bdt.cuh"
#include "neighbors.cuh"
#include "primitives.cuh"

namespace sphb
{

namespace
{

constexpr int kBdtThreads = 256;

//! particle of this thread in list mode (-1: none): lane of group groups[slot], slot = warp of the launch
__device__ inline long long listedParticle(const uint32_t* groups, unsigned num, const uint32_t* bounds,
                                           unsigned* slotOut)
{
    size_t slot = (blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5;
    *slotOut    = unsigned(slot);
    if (slot >= num) { return -1; }
    uint32_t g = groups[slot];
    size_t i   = size_t(bounds[g]) + (threadIdx.x & 31);
    return i < bounds[g + 1] ? (long long)i : -1;
}

template<class T>
__global__ void eosRefreshKernel(ChainArrays<T> a, HydroConsts<T> k)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= a.n) { return; }
    T mi;
    if constexpr (sizeof(T) == 8) { mi = T(a.pos[i].w); }
    else { mi = __int_as_float(a.posq[i].w); }
    T kxi    = a.kx[i];
    T xmassi = a.xm[i];
    T gradhi = a.gradh[i];
    T hi     = T(a.h[i]);
    // the expressions of veDefGradhEosKernel, so that an active particle gets the same values as there
    double rho  = double(kxi) * double(mi) / double(xmassi);
    double u    = k.cv * a.temp[i];
    double tmp  = u * (k.gamma - 1.0);
    double p    = rho * tmp;
    double c    = sqrt(k.gamma * tmp);
    double prho = p / (double(kxi) * double(mi) * double(mi) * double(gradhi));
    a.prho[i]   = T(prho);
    a.c[i]      = T(c);
    T vx = T(a.vx[i]), vy = T(a.vy[i]), vz = T(a.vz[i]);
    a.hrec[i] = HydroRec<T>{vx, vy, vz, T(1) / hi, xmassi, xmassi / kxi, T(c), T(prho)};
    if (a.avrec) { a.avrec[i] = AVRec<T>{vx, vy, vz, T(c), xmassi / kxi, a.divv[i], T(0), T(0)}; }
}

template<class T>
__global__ void groupDivvKernel(const uint32_t* groups, unsigned num, const uint32_t* bounds, const T* divv, float Krho,
                                float* groupDt)
{
    unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= num) { return; }
    size_t first = bounds[groups[w]];
    size_t last  = bounds[groups[w] + 1];
    // float localMax = max(localMax, divv[i]) per particle: the max of the values rounded once (rounding is monotonic)
    T m = T(-INFINITY);
    for (size_t i = first; i < last; ++i)
    {
        m = divv[i] > m ? divv[i] : m;
    }
    float localMax = float(m);
    groupDt[w]     = fminf(groupDt[w], Krho / fabsf(localMax));
}

template<class T>
__global__ void groupAccKernel(const uint32_t* groups, unsigned num, const uint32_t* bounds, const T* ax, const T* ay, const T* az,
                               const double* h, float etaAcc, float* groupDt)
{
    unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= num) { return; }
    size_t first = bounds[groups[w]];
    size_t last  = bounds[groups[w] + 1];
    double m     = INFINITY;
    for (size_t i = first; i < last; ++i)
    {
        double a2 = double(ax[i]) * double(ax[i]) + double(ay[i]) * double(ay[i]) + double(az[i]) * double(az[i]);
        double q  = h[i] * h[i] / a2;
        m         = q < m ? q : m;
    }
    float minH2A2 = float(m);
    groupDt[w]    = fminf(groupDt[w], etaAcc * sqrtf(sqrtf(minH2A2)));
}

//! positionUpdate (sph/include/sph/positions.hpp:100-111) of one axis: returns X_n+1, writes V_n+1 and dX_n+1
__device__ inline double pressAxis(double X, double A, double dX, double dt, double dtm1, double* V, double* dXn1)
{
    double vHalf = dX * (1.0 / dtm1);
    double vn    = vHalf + (0.5 * dtm1) * A;
    *V           = vn + A * dt;
    *dXn1        = (vn + (0.5 * A) * fabs(dt)) * dt;
    return X + *dXn1;
}

//! energyUpdate (positions.hpp:77-84)
__device__ inline double energyUpdate(double uOld, double dt, double dtm1, double du, double duM1)
{
    double uNew = uOld + du * dt + 0.5 * (du - duM1) / dtm1 * fabs(dt) * dt;
    if (uNew < 0.0) { uNew = uOld * exp(uNew * dt / uOld); }
    return uNew;
}

template<class T>
__global__ void driftKernel(const uint32_t* groups, unsigned num, const uint32_t* bounds, float dt, float dtBack, RungSteps steps,
                            const uint64_t* rung, IntegrateArrays<T> a, double cv)
{
    unsigned slot;
    long long ii = listedParticle(groups, num, bounds, &slot);
    if (ii < 0) { return; }
    size_t i      = size_t(ii);
    double dtm1   = double(steps.dtm1[min(rung[i], uint64_t(kMaxRungs - 1))]);
    double back   = -double(dtBack);
    double fwd    = double(dt);
    double A[3]   = {double(a.ax[i]), double(a.ay[i]), double(a.az[i])};
    double dX[3]  = {a.xm1[i], a.ym1[i], a.zm1[i]};
    double* P[3]  = {a.x, a.y, a.z};
    double* Vv[3] = {a.vx, a.vy, a.vz};
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double v, d;
        double Xn = pressAxis(P[k][i], A[k], dX[k], back, dtm1, &v, &d); // recover X_n
        P[k][i]   = pressAxis(Xn, A[k], dX[k], fwd, dtm1, &v, &d);
        Vv[k][i]  = v;
    }
    double du = a.du[i], duM1 = a.duM1[i];
    double u  = energyUpdate(a.temp[i] * cv, back, dtm1, du, duM1);
    a.temp[i] = energyUpdate(u, fwd, dtm1, du, duM1) / cv;
}

//! putInBox (cstone/sfc/box.hpp) on the periodic axes of box
__device__ inline double foldPeriodic(double v, int k, const DevBox& box)
{
    if (!box.periodic[k]) { return v; }
    if (v > box.hi[k]) { return v - box.len[k]; }
    if (v < box.lo[k]) { return v + box.len[k]; }
    return v;
}

template<class T>
__global__ void rungPositionsKernel(const uint32_t* groups, unsigned num, const uint32_t* bounds, float dt, RungSteps steps,
                                    const uint64_t* rung, IntegrateArrays<T> a, DevBox box, double cv)
{
    unsigned slot;
    long long ii = listedParticle(groups, num, bounds, &slot);
    if (ii < 0) { return; }
    size_t i      = size_t(ii);
    double dtm1   = double(steps.dtm1[min(rung[i], uint64_t(kMaxRungs - 1))]);
    double dtD    = double(dt);
    double A[3]   = {double(a.ax[i]), double(a.ay[i]), double(a.az[i])};
    double dX[3]  = {a.xm1[i], a.ym1[i], a.zm1[i]};
    double* P[3]  = {a.x, a.y, a.z};
    double* Vv[3] = {a.vx, a.vy, a.vz};
    double* M[3]  = {a.xm1, a.ym1, a.zm1};
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double v, d;
        double X = pressAxis(P[k][i], A[k], dX[k], dtD, dtm1, &v, &d);
        P[k][i]  = foldPeriodic(X, k, box);
        M[k][i]  = d;
        Vv[k][i] = v;
    }
    double du = a.du[i];
    a.temp[i] = energyUpdate(cv * a.temp[i], dtD, dtm1, du, a.duM1[i]) / cv;
    a.duM1[i] = du;
}

__global__ void storeRungKernel(const uint32_t* groups, unsigned num, const uint32_t* bounds, uint64_t value, uint64_t* rung)
{
    unsigned slot;
    long long i = listedParticle(groups, num, bounds, &slot);
    if (i >= 0) { rung[i] = value; }
}

__global__ void listUpdateHKernel(const uint32_t* groups, unsigned num, const uint32_t* bounds, unsigned ng0, const unsigned* nc,
                                  double* h, uint64_t* keys, unsigned* flag)
{
    unsigned slot;
    long long ii = listedParticle(groups, num, bounds, &slot);
    if (ii < 0) { return; }
    size_t i   = size_t(ii);
    unsigned c = nc[i];
    if (c <= 1)
    {
        keys[i] = kRemoveKey;
        atomicOr(flag, 1u);
    }
    double ratio = __ddiv_rn(__dmul_rn(1023.0, double(ng0)), double(c));
    h[i]         = __dmul_rn(__dmul_rn(h[i], 0.5), pow(__dadd_rn(1.0, ratio), 0.1));
}

//! grid-stride maximum with one atomic per block: one per warp on the single word serialised ~65 k atomics at 128^3
__global__ void __launch_bounds__(kBdtThreads) maxDisplacementKernel(const double* x, const double* y,
                                                                     const double* z, const double* xs,
                                                                     const double* ys, const double* zs, size_t n,
                                                                     DevBox box, unsigned long long* out)
{
    double d = 0.0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        double di = fmax(fabs(minImage(x[i] - xs[i], box.len[0], box.ilen[0], box.periodic[0])),
                         fabs(minImage(y[i] - ys[i], box.len[1], box.ilen[1], box.periodic[1])));
        d         = fmax(d, fmax(di, fabs(minImage(z[i] - zs[i], box.len[2], box.ilen[2], box.periodic[2]))));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        d = fmax(d, __shfl_xor_sync(0xffffffffu, d, off));
    }
    __shared__ double warpMax[kBdtThreads / 32];
    if ((threadIdx.x & 31) == 0) { warpMax[threadIdx.x >> 5] = d; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int w = 1; w < int(blockDim.x >> 5); ++w)
        {
            d = fmax(d, warpMax[w]);
        }
        atomicMax(out, orderedBits(d));
    }
}

__global__ void dtKeysKernel(const float* groupDt, unsigned num, uint64_t* keys, uint32_t* values)
{
    unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= num) { return; }
    keys[w]   = uint64_t(__float_as_uint(groupDt[w]));
    values[w] = w;
}

__global__ void sortedDtKernel(const uint64_t* keys, unsigned num, float* groupDt)
{
    unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < num) { groupDt[w] = __uint_as_float(unsigned(keys[w])); }
}

//! first index of sorted[0, num) with sorted[idx] >= v (std::lower_bound)
__device__ inline unsigned lowerBound(const uint64_t* sortedKeys, unsigned num, float v)
{
    unsigned lo = 0, hi = num;
    while (lo < hi)
    {
        unsigned mid = (lo + hi) >> 1;
        if (__uint_as_float(unsigned(sortedKeys[mid])) < v) { lo = mid + 1; }
        else { hi = mid; }
    }
    return lo;
}

__global__ void rungInfoKernel(const uint64_t* keys, unsigned num, unsigned fastIdx, uint32_t* out)
{
    float minDt = __uint_as_float(unsigned(keys[0]));
    out[0]      = unsigned(keys[0]);
    out[1]      = unsigned(keys[min(fastIdx, num - 1)]);
    for (int r = 1; r < kMaxRungs; ++r)
    {
        float maxDtRung = float(1 << r) * minDt;
        out[1 + r]      = lowerBound(keys, num, maxDtRung);
    }
}

__global__ void gatherGroupsKernel(const uint32_t* src, const uint32_t* idx, unsigned num, uint32_t* dst)
{
    unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < num) { dst[w] = src[idx[w]]; }
}

__global__ void sequenceKernel(uint32_t* list, unsigned num, uint32_t first)
{
    unsigned w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < num) { list[w] = w + first; }
}

unsigned warpBlocks(unsigned numGroups) { return ceilDiv(size_t(numGroups) * 32, kBdtThreads); }

} // namespace

template<class T>
int launchEosRefresh(const ChainArrays<T>& a, const HydroConsts<T>& k, cudaStream_t s)
{
    if (a.n == 0) { return kOk; }
    eosRefreshKernel<T><<<ceilDiv(a.n, kBdtThreads), kBdtThreads, 0, s>>>(a, k);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchGroupDivv(const uint32_t* groups, unsigned num, const uint32_t* bounds, const T* divv, float Krho, float* groupDt,
                    cudaStream_t s)
{
    if (num == 0) { return kOk; }
    groupDivvKernel<T><<<ceilDiv(num, kBdtThreads), kBdtThreads, 0, s>>>(groups, num, bounds, divv, Krho, groupDt);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchGroupAcc(const uint32_t* groups, unsigned num, const uint32_t* bounds, const T* ax, const T* ay, const T* az,
                   const double* h, float etaAcc, float* groupDt, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    groupAccKernel<T><<<ceilDiv(num, kBdtThreads), kBdtThreads, 0, s>>>(groups, num, bounds, ax, ay, az, h, etaAcc,
                                                                         groupDt);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchDrift(const uint32_t* groups, unsigned num, const uint32_t* bounds, float dt, float dtBack, RungSteps steps,
                const uint64_t* rung, const IntegrateArrays<T>& a, double cv, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    driftKernel<T><<<warpBlocks(num), kBdtThreads, 0, s>>>(groups, num, bounds, dt, dtBack, steps, rung, a, cv);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchRungPositions(const uint32_t* groups, unsigned num, const uint32_t* bounds, float dt, RungSteps steps,
                        const uint64_t* rung, const IntegrateArrays<T>& a, const DevBox& box, double cv,
                        cudaStream_t s)
{
    if (num == 0) { return kOk; }
    rungPositionsKernel<T><<<warpBlocks(num), kBdtThreads, 0, s>>>(groups, num, bounds, dt, steps, rung, a, box, cv);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchStoreRung(const uint32_t* groups, unsigned num, const uint32_t* bounds, uint64_t value, uint64_t* rung, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    storeRungKernel<<<warpBlocks(num), kBdtThreads, 0, s>>>(groups, num, bounds, value, rung);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchListUpdateH(const uint32_t* groups, unsigned num, const uint32_t* bounds, unsigned ng0, const unsigned* nc, double* h,
                      uint64_t* keys, unsigned* flag, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    listUpdateHKernel<<<warpBlocks(num), kBdtThreads, 0, s>>>(groups, num, bounds, ng0, nc, h, keys, flag);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchMaxDisplacement(const double* x, const double* y, const double* z, const double* xs, const double* ys,
                          const double* zs, size_t n, const DevBox& box, unsigned long long* out, cudaStream_t s)
{
    if (n == 0) { return kOk; }
    unsigned blocks = unsigned(std::min<size_t>(ceilDiv(n, kBdtThreads), size_t(smCount()) * 8));
    maxDisplacementKernel<<<blocks, kBdtThreads, 0, s>>>(x, y, z, xs, ys, zs, n, box, out);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchDtKeys(const float* groupDt, unsigned num, uint64_t* keys, uint32_t* values, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    dtKeysKernel<<<ceilDiv(num, kBdtThreads), kBdtThreads, 0, s>>>(groupDt, num, keys, values);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchSortedDt(const uint64_t* keys, unsigned num, unsigned fastIdx, float* groupDt, uint32_t* out,
                   cudaStream_t s)
{
    if (num == 0) { return kErrArg; }
    sortedDtKernel<<<ceilDiv(num, kBdtThreads), kBdtThreads, 0, s>>>(keys, num, groupDt);
    rungInfoKernel<<<1, 1, 0, s>>>(keys, num, fastIdx, out);
    countLaunch();
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchGatherGroups(const uint32_t* src, const uint32_t* idx, unsigned num, uint32_t* dst, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    gatherGroupsKernel<<<ceilDiv(num, kBdtThreads), kBdtThreads, 0, s>>>(src, idx, num, dst);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchSequence(uint32_t* list, unsigned num, uint32_t first, cudaStream_t s)
{
    if (num == 0) { return kOk; }
    sequenceKernel<<<ceilDiv(num, kBdtThreads), kBdtThreads, 0, s>>>(list, num, first);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

#define SPHB_BDT_INSTANTIATE(T)                                                                                        \
    template int launchEosRefresh<T>(const ChainArrays<T>&, const HydroConsts<T>&, cudaStream_t);                    \
    template int launchGroupDivv<T>(const uint32_t*, unsigned, const uint32_t*, const T*, float, float*, cudaStream_t);       \
    template int launchGroupAcc<T>(const uint32_t*, unsigned, const uint32_t*, const T*, const T*, const T*, const double*,   \
                                   float, float*, cudaStream_t);                                                     \
    template int launchDrift<T>(const uint32_t*, unsigned, const uint32_t*, float, float, RungSteps, const uint64_t*,         \
                                const IntegrateArrays<T>&, double, cudaStream_t);                                    \
    template int launchRungPositions<T>(const uint32_t*, unsigned, const uint32_t*, float, RungSteps, const uint64_t*,        \
                                        const IntegrateArrays<T>&, const DevBox&, double, cudaStream_t);

SPHB_BDT_INSTANTIATE(double)
SPHB_BDT_INSTANTIATE(float)

} // namespace sphb
