// Device helpers shared by the SPH-VE J-loops (hydro_ve.cu) and their adjoints (adjoint.cu): neighbour-sum
// accumulators, kernel evaluation, pair separations per precision, packed record loads and the chunked list reads.
#pragma once

#include "hydro.cuh"
#include "neighbors.cuh"

namespace sphb
{
namespace chain
{

constexpr int kChainThreads = 128;

//! compile-time variants of the J-loop kernels: write the adjoint's tape, or run over a batched ensemble
constexpr int kModeTape    = 1;
constexpr int kModeBatch   = 2;
constexpr int kModeAvClean = 4;
constexpr int kModeList    = 8; // block time steps: only the groups of a device-side list

/*! Neighbour-sum accumulator. FP64: every term is added as it comes, in list order (the reference's order).
 *  FP32: terms are summed plainly within one list chunk of 8 neighbours and each chunk sum is added to a
 *  Kahan-compensated accumulator; explicit round-to-nearest intrinsics keep the compiler from fusing or reordering
 *  the compensation. */
template<class T>
struct BlockSum;

template<>
struct BlockSum<double>
{
    double s;
    __device__ explicit BlockSum(double v = 0.0)
        : s(v)
    {
    }
    __device__ void add(double v) { s += v; }
    __device__ void flush() {}
    __device__ double get() const { return s; }
};

template<>
struct BlockSum<float>
{
    float s, comp, part;
    __device__ explicit BlockSum(float v = 0.f)
        : s(v)
        , comp(0.f)
        , part(0.f)
    {
    }
    __device__ void add(float v) { part += v; }
    __device__ void flush()
    {
        float y = __fsub_rn(part, comp);
        float t = __fadd_rn(s, y);
        comp    = __fsub_rn(__fsub_rn(t, s), y);
        s       = t;
        part    = 0.f;
    }
    __device__ float get() const { return s; }
};

//! a / b: IEEE division in FP64 (the reference's rounding), the fast 2-ulp reciprocal-multiply in FP32
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

//! linear interpolation in a 20000-entry table on [0, 2] (sph/include/sph/table_lookup.hpp:14-26)
template<class T>
__device__ __forceinline__ T tableLookup(const T* __restrict__ table, T v)
{
    constexpr int numIntervals = kTableSize - 1;
    constexpr T dx             = T(2.0) / numIntervals;
    constexpr T invDx          = T(1) / dx;
    int idx                    = int(v * invDx);
    if (idx >= numIntervals) { return T(0); }
    T t0 = __ldg(table + idx);
    T t1 = __ldg(table + idx + 1);
    T derivative = (t1 - t0) * invDx;
    return t0 + derivative * (v - T(idx) * dx);
}

//! Horner evaluation of the FP32 kernel polynomial at t = v^2/2 - 1
__device__ __forceinline__ float polyEvalT(const float (&c)[kPolyTerms], float t)
{
    float acc = c[kPolyTerms - 1];
#pragma unroll
    for (int p = kPolyTerms - 2; p >= 0; --p)
    {
        acc = fmaf(acc, t, c[p]);
    }
    return acc;
}

//! Horner evaluation of the FP32 kernel polynomial in t = v^2/2 - 1
__device__ __forceinline__ float polyEval(const float (&c)[kPolyTerms], float v)
{
    float t   = fmaf(0.5f * v, v, -1.0f);
    float acc = c[kPolyTerms - 1];
#pragma unroll
    for (int p = kPolyTerms - 2; p >= 0; --p)
    {
        acc = fmaf(acc, t, c[p]);
    }
    return acc;
}

//! the smoothing kernel W(v), zero from v = 2 on: FP64 by table lookup (as the reference), FP32 by polynomial
template<class T>
__device__ __forceinline__ T kernelW(const T* __restrict__ table, const HydroConsts<T>& k, T v)
{
    if constexpr (sizeof(T) == 4)
    {
        if (k.usePoly) { return v < T(2) ? polyEval(k.wpoly, v) : T(0); }
    }
    return tableLookup(table, v);
}

/*! W of a pair from its squared separation r2, for a target with hInv = 1/h and hh = hInv^2 / 2. FP32 with the
 *  polynomial: t = v^2/2 - 1 = r2 hh - 1 directly, zero from t = 1 (v = 2) on, without the square root. Otherwise
 *  (FP64, or an FP32 simulation whose polynomial fit failed) the table at v = sqrt(r2) hInv, the expression of the
 *  reference's order. */
template<class T>
__device__ __forceinline__ T kernelWr2(const T* __restrict__ table, const HydroConsts<T>& k, T r2, T hInv, T hh)
{
    if constexpr (sizeof(T) == 4)
    {
        if (k.usePoly)
        {
            float t = fmaf(r2, hh, -1.0f);
            return t < 1.0f ? polyEvalT(k.wpoly, t) : 0.0f;
        }
    }
    return tableLookup(table, T(sqrt(r2)) * hInv);
}

//! dW/dv, zero from v = 2 on
template<class T>
__device__ __forceinline__ T kernelDW(const T* __restrict__ table, const HydroConsts<T>& k, T v)
{
    if constexpr (sizeof(T) == 4)
    {
        if (k.usePoly) { return v < T(2) ? v * polyEval(k.dwpoly, v) : T(0); }
    }
    return tableLookup(table, v);
}

//! periodic shift of a pair separation by one box length if it exceeds r (cstone/sfc/box.hpp applyPBC, legacy form)
__device__ __forceinline__ void shiftPbc(double& rx, double& ry, double& rz, double r, const DevBox& box)
{
    if (box.periodic[0])
    {
        if (rx > r) { rx -= box.len[0]; }
        else if (rx < -r) { rx += box.len[0]; }
    }
    if (box.periodic[1])
    {
        if (ry > r) { ry -= box.len[1]; }
        else if (ry < -r) { ry += box.len[1]; }
    }
    if (box.periodic[2])
    {
        if (rz > r) { rz -= box.len[2]; }
        else if (rz < -r) { rz += box.len[2]; }
    }
}

//! one 32-byte (256-bit) read-only vector load of 8 floats; p must be 32-byte aligned
__device__ __forceinline__ void ldg256(const void* p, float (&v)[8])
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(p));
}

//! 32-byte read-only load as two 16-byte vector loads (one sector)
__device__ __forceinline__ double4 ldg4(const double4* p)
{
    double4 v;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w) : "l"(p));
    return v;
}

// ---------------------------------------------------------------------------------------------------------------
// positions and pair separations per precision
// ---------------------------------------------------------------------------------------------------------------

template<class T>
struct Pos;

template<>
struct Pos<double>
{
    double x, y, z, m;
};

template<>
struct Pos<float>
{
    int x, y, z;
    float m;
};

__device__ __forceinline__ Pos<double> posOf(const ChainArrays<double>& a, size_t j)
{
    double4 v = ldg4(a.pos + j);
    return {v.x, v.y, v.z, v.w};
}

__device__ __forceinline__ Pos<float> posOf(const ChainArrays<float>& a, size_t j)
{
    int4 v = __ldg(a.posq + j);
    return {v.x, v.y, v.z, __int_as_float(v.w)};
}

template<class T>
struct Sep
{
    T rx, ry, rz;
};

//! x_i - x_j with the reference's periodic shift (threshold r = 2 h_i), FP64
__device__ __forceinline__ Sep<double> separation(const Pos<double>& pi, const Pos<double>& pj, double r,
                                                  const DevBox& box, const HydroConsts<double>&)
{
    double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
    shiftPbc(rx, ry, rz, r, box);
    return {rx, ry, rz};
}

//! x_i - x_j from fixed-point coordinates: an exact integer difference, wrapped to the nearest image on periodic
//! axes, rounded once to FP32
__device__ __forceinline__ Sep<float> separation(const Pos<float>& pi, const Pos<float>& pj, double,
                                                 const DevBox&, const HydroConsts<float>& k)
{
    int dx = int(unsigned(pi.x) - unsigned(pj.x));
    int dy = int(unsigned(pi.y) - unsigned(pj.y));
    int dz = int(unsigned(pi.z) - unsigned(pj.z));
    return {float(dx) * k.qscale[0], float(dy) * k.qscale[1], float(dz) * k.qscale[2]};
}

template<class T>
__device__ __forceinline__ HydroRec<T> loadHydro(const HydroRec<T>* p)
{
    HydroRec<T> r;
    if constexpr (sizeof(T) == 8)
    {
        const double4* q = reinterpret_cast<const double4*>(p);
        double4 a = ldg4(q), b = ldg4(q + 1);
        r = {T(a.x), T(a.y), T(a.z), T(a.w), T(b.x), T(b.y), T(b.z), T(b.w)};
    }
    else
    {
        float v[8];
        ldg256(p, v);
        r = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
    }
    return r;
}

template<class T>
__device__ __forceinline__ GradRec<T> loadGrad(const GradRec<T>* p)
{
    GradRec<T> r;
    if constexpr (sizeof(T) == 8)
    {
        const double4* q = reinterpret_cast<const double4*>(p);
        double4 a = ldg4(q), b = ldg4(q + 1);
        r = {T(a.x), T(a.y), T(a.z), T(a.w), T(b.x), T(b.y), T(b.z), T(b.w)};
    }
    else
    {
        float v[8];
        ldg256(p, v);
        r = {v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
    }
    return r;
}

struct Target
{
    size_t i;
    size_t group;
    unsigned lane;
    unsigned count;
    unsigned ngPad;
};

__device__ __forceinline__ bool targetOf(size_t n, const unsigned* nc, unsigned ngmax, Target& t,
                                         const uint8_t* inst = nullptr)
{
    t.i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (t.i >= n) { return false; }
    if (inst && inst[t.i] == kGhost) { return false; }
    t.group = t.i >> 5;
    t.lane  = unsigned(t.i & 31);
    t.count = min(nc[t.i] - 1u, ngmax);
    t.ngPad = paddedNgmax(ngmax);
    return true;
}

/*! The target of this thread: thread i of the launch, or in list mode lane i % 32 of group groupList[i / 32], whose
 *  particles are [groupBounds[g], groupBounds[g + 1]) (GroupView slices of sph/include/sph/groups.hpp:96-103; a warp
 *  is one group of at most 32). *w receives the list slot. */
template<int kMode, class T>
__device__ __forceinline__ bool chainTarget(const ChainArrays<T>& a, unsigned ngmax, Target& t, unsigned* w = nullptr)
{
    if constexpr (kMode & kModeList)
    {
        size_t slot = (blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5;
        if (w) { *w = unsigned(slot); }
        if (slot >= a.numListed) { return false; }
        uint32_t g = __ldg(a.groupList + slot);
        t.i        = size_t(__ldg(a.groupBounds + g)) + (threadIdx.x & 31);
        if (t.i >= __ldg(a.groupBounds + g + 1)) { return false; }
        t.group = t.i >> 5;
        t.lane  = unsigned(t.i & 31);
        t.count = min(a.nc[t.i] - 1u, ngmax);
        t.ngPad = paddedNgmax(ngmax);
        return true;
    }
    else { return targetOf(a.n, a.nc, ngmax, t, (kMode & kModeBatch) ? a.batch.inst : nullptr); }
}

template<class T>
__device__ __forceinline__ AVRec<T> loadAV(const AVRec<T>* p)
{
    AVRec<T> r;
    if constexpr (sizeof(T) == 8)
    {
        const double4* q = reinterpret_cast<const double4*>(p);
        double4 a = ldg4(q), b = ldg4(q + 1);
        r = {a.x, a.y, a.z, a.w, b.x, b.y, T(0), T(0)};
    }
    else
    {
        float v[8];
        ldg256(p, v);
        r = {v[0], v[1], v[2], v[3], v[4], v[5], 0.f, 0.f};
    }
    return r;
}

template<class T>
__device__ __forceinline__ void loadDV(const DVRec<T>* p, T (&g)[6])
{
    if constexpr (sizeof(T) == 8)
    {
        const double2* q = reinterpret_cast<const double2*>(p);
        double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
        g[0] = a.x, g[1] = a.y, g[2] = b.x, g[3] = b.y, g[4] = c.x, g[5] = c.y;
    }
    else
    {
        const float4* q = reinterpret_cast<const float4*>(p);
        float4 a = __ldg(q);
        float2 b = __ldg(reinterpret_cast<const float2*>(q + 1));
        g[0] = a.x, g[1] = a.y, g[2] = a.z, g[3] = a.w, g[4] = b.x, g[5] = b.y;
    }
}

/*! Additive AV-cleaning correction of rv = r . v_ij (momentum_energy_kern.hpp:43-63): the quadratic forms of both
 *  particles' symmetrised velocity gradients along r, damped by how far min(v_i, v_j) falls below eta_crit. */
template<class T>
__device__ __forceinline__ T avRvCorrection(T rx, T ry, T rz, T etaAb, T etaCrit, const T (&gi)[6], const T (&gj)[6])
{
    T dmy1 = rx * (gi[0] * rx + gi[1] * ry + gi[2] * rz) + ry * (gi[3] * ry + gi[4] * rz) + rz * (gi[5] * rz);
    T dmy2 = rx * (gj[0] * rx + gj[1] * ry + gj[2] * rz) + ry * (gj[3] * ry + gj[4] * rz) + rz * (gj[5] * rz);
    T dmy3 = T(1);
    if (etaAb < etaCrit)
    {
        T etaDiff = T(5) * (etaAb - etaCrit);
        dmy3      = exp(-etaDiff * etaDiff);
    }
    T aAb   = (dmy2 != T(0)) ? dmy1 / dmy2 : T(0);
    T aAbp1 = T(1) + aAb;
    T q     = T(4) * aAb / (aAbp1 * aAbp1);
    q       = q < T(1) ? q : T(1);
    q       = q > T(0) ? q : T(0);
    T phiAb = T(0.5) * dmy3 * q;
    return -phiAb * (dmy1 + dmy2);
}

//! the 8 neighbour indices of list chunk q0 / 8 of the target (two 16-byte loads of one sector)
__device__ __forceinline__ void loadChunk(const uint32_t* nidx, const Target& t, unsigned ngPad, unsigned q0,
                                          uint32_t (&js)[kNbChunk])
{
    const uint32_t* p = nidx + nidxAt(t.group, ngPad, q0, t.lane);
    // one 256-bit load of the chunk's sector; the lists are read once per kernel, so the streaming (evict-first)
    // hint keeps them from evicting the neighbour records in L2
    asm("ld.global.cs.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(js[0]), "=r"(js[1]), "=r"(js[2]), "=r"(js[3]), "=r"(js[4]), "=r"(js[5]), "=r"(js[6]), "=r"(js[7])
        : "l"(p));
}

/*! The next neighbour index of a list chunk: returns js[0] and shifts the rest down. Every index stays static, so
 *  the chunk stays in registers while a pair loop runs one pair per iteration instead of fully unrolled (the largest
 *  FP32 J-loop's unrolled 8-pair body overflowed the instruction cache). */
__device__ __forceinline__ uint32_t popChunk(uint32_t (&js)[kNbChunk])
{
    uint32_t j = js[0];
#pragma unroll
    for (unsigned r = 0; r + 1 < kNbChunk; ++r)
    {
        js[r] = js[r + 1];
    }
    return j;
}

/*! Maximum (kMax) or minimum of one double per thread, published as ordered bits with one atomic per block on
 *  *single (one simulation), or one atomic per warp on the warp's instance slot batch.reduce[2 q + slot] (an ensemble:
 *  a warp never spans two instances). Every thread of the block must call it. */
template<bool kMax, bool kBatched>
__device__ __forceinline__ void reduceOrdered(double v, size_t n, unsigned long long* single, const BatchView& batch,
                                              int slot)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        double o = __shfl_xor_sync(0xffffffffu, v, off);
        v        = kMax ? fmax(v, o) : fmin(v, o);
    }
    if constexpr (kBatched)
    {
        size_t first = blockIdx.x * size_t(blockDim.x) + (threadIdx.x & ~31u);
        if ((threadIdx.x & 31) == 0 && first < n)
        {
            uint8_t q = batch.inst[first];
            if (q != kGhost)
            {
                if (kMax) { atomicMax(batch.reduce + 2 * q + slot, orderedBits(v)); }
                else { atomicMin(batch.reduce + 2 * q + slot, orderedBits(v)); }
            }
        }
        return;
    }
    __shared__ double warpVal[kChainMaxThreads / 32];
    if ((threadIdx.x & 31) == 0) { warpVal[threadIdx.x >> 5] = v; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double m = warpVal[0];
        for (int w = 1; w < int(blockDim.x >> 5); ++w)
        {
            m = kMax ? fmax(m, warpVal[w]) : fmin(m, warpVal[w]);
        }
        if (kMax) { atomicMax(single, orderedBits(m)); }
        else { atomicMin(single, orderedBits(m)); }
    }
}

} // namespace chain
} // namespace sphb
