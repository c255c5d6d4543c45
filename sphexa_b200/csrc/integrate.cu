// Per-particle FP64 kernels around the neighbour sums: position packing, kick-drift + energy integration,
// smoothing-length update, coordinate min/max and the conservation reductions.
#include "hydro.cuh"
#include "integrate.cuh"
#include "neighbors.cuh"
#include "primitives.cuh"

namespace sphb
{

namespace
{

//! one coordinate as 32-bit fixed point over [lo, lo + 2^32 unit), unit = span / 2^32 (periodic: span = L, the value
//! L wraps to 0; open: span = 2 L so that differences of up to L stay below half the range and never wrap)
//! Coordinates below lo (drifted out of the box between two domain syncs under block time steps) wrap modulo 2^32:
//! on a periodic axis that is the periodic image, on an open axis differences below L still come out right.
__device__ inline int quantiseFixed(double v, double lo, double invUnit)
{
    double q = (v - lo) * invUnit;
    unsigned long long u = q >= 0.0 ? (unsigned long long)(q + 0.5) : 0ull - (unsigned long long)(0.5 - q);
    return int(unsigned(u & 0xffffffffull));
}

__global__ void packPosKernel(const double* x, const double* y, const double* z, const double* m, size_t n,
                              double4* pos, int4* posq, FixedFrame fr)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    if (pos) { pos[i] = make_double4(x[i], y[i], z[i], m[i]); }
    if (posq)
    {
        posq[i] = make_int4(quantiseFixed(x[i], fr.lo[0], fr.invUnit[0]), quantiseFixed(y[i], fr.lo[1], fr.invUnit[1]),
                            quantiseFixed(z[i], fr.lo[2], fr.invUnit[2]), __float_as_int(float(m[i])));
    }
}

/*! packPosKernel and the bounding boxes of the runs of kBlockSize consecutive particles (computeBlockBoxes) in one
 *  pass over the coordinates: the lanes of a run reduce their box with shuffles (runs start at multiples of
 *  kBlockSize, and so do lane groups of kBlockSize in a block of a multiple of 32 threads). */
__global__ void packPosBoxesKernel(const double* x, const double* y, const double* z, const double* m, size_t n,
                                   double4* pos, int4* posq, FixedFrame fr, DevBox box, float4* boxLo, float4* boxHi)
{
    size_t i   = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    bool valid = i < n;
    double p[3] = {0.0, 0.0, 0.0};
    if (valid)
    {
        p[0] = x[i];
        p[1] = y[i];
        p[2] = z[i];
        double mi = m[i];
        if (pos) { pos[i] = make_double4(p[0], p[1], p[2], mi); }
        if (posq)
        {
            posq[i] = make_int4(quantiseFixed(p[0], fr.lo[0], fr.invUnit[0]), quantiseFixed(p[1], fr.lo[1], fr.invUnit[1]),
                                quantiseFixed(p[2], fr.lo[2], fr.invUnit[2]), __float_as_int(float(mi)));
        }
    }
    double l[3], u[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        l[k] = valid ? p[k] - box.lo[k] : INFINITY;
        u[k] = valid ? p[k] - box.lo[k] : -INFINITY;
#pragma unroll
        for (int off = 1; off < kBlockSize; off <<= 1)
        {
            l[k] = fmin(l[k], __shfl_xor_sync(0xffffffffu, l[k], off));
            u[k] = fmax(u[k], __shfl_xor_sync(0xffffffffu, u[k], off));
        }
    }
    if (valid && i % kBlockSize == 0)
    {
        size_t c = i / kBlockSize;
        boxLo[c] = make_float4(__double2float_rd(l[0]), __double2float_rd(l[1]), __double2float_rd(l[2]), 0.f);
        boxHi[c] = make_float4(__double2float_ru(u[0]), __double2float_ru(u[1]), __double2float_ru(u[2]), 0.f);
    }
}

//! fold a coordinate back into a periodic box once (cstone/sfc/box.hpp putInBox)
__device__ inline double putInBox(double v, int k, const DevBox& box)
{
    if (!box.periodic[k]) { return v; }
    if (v > box.hi[k]) { return v - box.len[k]; }
    if (v < box.lo[k]) { return v + box.len[k]; }
    return v;
}

/*! Press kick-drift (sph/include/sph/positions.hpp:100-111) and the Adams-Bashforth energy update of temp
 *  (positions.hpp:77-84,139-160), in FP64, with the operation order of the reference expressions. */
template<class T>
__global__ void positionsKernel(size_t n, IntegrateArrays<T> a, DevBox box, double dt, double dtm1, double cv)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    if (a.batch.inst)
    {
        uint8_t q = a.batch.inst[i];
        if (q == kGhost) { return; }
        dt   = a.batch.dt[q];
        dtm1 = a.batch.dtm1[q];
        cv   = a.batch.cv[q];
    }
    double X[3]  = {a.x[i], a.y[i], a.z[i]};
    double A[3]  = {double(a.ax[i]), double(a.ay[i]), double(a.az[i])};
    double dX[3] = {a.xm1[i], a.ym1[i], a.zm1[i]};
    double* V[3] = {a.vx, a.vy, a.vz};
    double* P[3] = {a.x, a.y, a.z};
    double* M[3] = {a.xm1, a.ym1, a.zm1};
    double invDtm1 = 1.0 / dtm1;
    double adt     = fabs(dt);
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        double vHalf = dX[k] * invDtm1;
        double vn    = vHalf + (0.5 * dtm1) * A[k];
        double vnp1  = vn + A[k] * dt;
        double dXn1  = (vn + (0.5 * A[k]) * adt) * dt;
        P[k][i]      = putInBox(X[k] + dXn1, k, box);
        M[k][i]      = dXn1;
        V[k][i]      = vnp1;
    }
    double uOld = cv * a.temp[i];
    double du   = a.du[i];
    double duM1 = a.duM1[i];
    double uNew = uOld + du * dt + 0.5 * (du - duM1) / dtm1 * adt * dt;
    if (uNew < 0.0) { uNew = uOld * exp(uNew * dt / uOld); }
    a.temp[i] = uNew / cv;
    a.duM1[i] = du;
}

/*! end-of-step smoothing length: h * 0.5 (1 + 1023 ng0/nc)^(1/10); nc <= 1 flags the particle for removal
 *  (sph/include/sph/update_h.hpp:12-33) */
__global__ void updateHKernel(size_t n, unsigned ng0, const unsigned* nc, double* h, uint64_t* keys, unsigned* flag,
                              const uint8_t* inst)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    if (inst && inst[i] == kGhost) { return; }
    unsigned c = nc[i];
    if (c <= 1)
    {
        keys[i] = kRemoveKey;
        atomicOr(flag, 1u);
    }
    double ratio = __ddiv_rn(__dmul_rn(1023.0, double(ng0)), double(c));
    h[i]         = __dmul_rn(__dmul_rn(h[i], 0.5), pow(__dadd_rn(1.0, ratio), 0.1));
}

//! the smoothing length updateHKernel will write, in FP32 or FP64 (SPHB_F32 / SPHB_F64), without its side effects
__global__ void predictHKernel(size_t n, unsigned ng0, const unsigned* nc, const double* h, void* out, int outType)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    double ratio = __ddiv_rn(__dmul_rn(1023.0, double(ng0)), double(nc[i]));
    double hNew  = __dmul_rn(__dmul_rn(h[i], 0.5), pow(__dadd_rn(1.0, ratio), 0.1));
    if (outType == SPHB_F32) { static_cast<float*>(out)[i] = float(hNew); }
    else { static_cast<double*>(out)[i] = hNew; }
}

constexpr int kRedThreads = 256;

//! per-block partial sums of the conserved quantities: eKin, eInt, P(3), L(3), sum nc (9 doubles)
__global__ void __launch_bounds__(kRedThreads) conservedPartialKernel(size_t n, const double* x, const double* y,
                                                                      const double* z, const double* vx,
                                                                      const double* vy, const double* vz,
                                                                      const double* m, const double* temp,
                                                                      const unsigned* nc, double cv, double* partial)
{
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        double mi = m[i];
        double X[3] = {x[i], y[i], z[i]};
        double V[3] = {vx[i], vy[i], vz[i]};
        acc[0] += mi * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
        acc[1] += cv * temp[i] * mi;
        acc[2] += mi * V[0];
        acc[3] += mi * V[1];
        acc[4] += mi * V[2];
        acc[5] += mi * (X[1] * V[2] - X[2] * V[1]);
        acc[6] += mi * (X[2] * V[0] - X[0] * V[2]);
        acc[7] += mi * (X[0] * V[1] - X[1] * V[0]);
        acc[8] += double(nc[i]);
    }
    __shared__ double sh[kRedThreads / 32][9];
#pragma unroll
    for (int q = 0; q < 9; ++q)
    {
        double v = acc[q];
        for (int off = 16; off > 0; off >>= 1)
        {
            v += __shfl_xor_sync(0xffffffffu, v, off);
        }
        if ((threadIdx.x & 31) == 0) { sh[threadIdx.x >> 5][q] = v; }
    }
    __syncthreads();
    if (threadIdx.x < 9)
    {
        double s = 0;
        for (int w = 0; w < kRedThreads / 32; ++w)
        {
            s += sh[w][threadIdx.x];
        }
        partial[blockIdx.x * 9 + threadIdx.x] = s;
    }
}

//! the 9 block partials reduced in a fixed order (deterministic): warp q sums quantity q, lane l the blocks
//! l, l + 32, ... in turn, then a fixed shuffle tree over the lanes
__global__ void conservedFinalKernel(const double* partial, int numBlocks, double* out)
{
    int q    = threadIdx.x >> 5;
    int lane = threadIdx.x & 31;
    if (q >= 9) { return; }
    double s = 0;
    for (int b = lane; b < numBlocks; b += 32)
    {
        s += partial[b * 9 + q];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        s += __shfl_xor_sync(0xffffffffu, s, off);
    }
    if (lane == 0) { out[q] = s; }
}

__global__ void setWordsKernel(unsigned long long* dst, int count, unsigned long long v0, unsigned long long v1)
{
    if (threadIdx.x < unsigned(count)) { dst[threadIdx.x] = threadIdx.x == 0 ? v0 : v1; }
}

//! out[0..6) = ordered bits of the running min/max of x, y and z (after minMax3InitKernel)
__global__ void minMax3InitKernel(unsigned long long* out)
{
    int k = threadIdx.x;
    if (k < 6) { out[k] = (k & 1) ? orderedBits(-INFINITY) : orderedBits(INFINITY); }
}

//! the three axes' extrema in one pass: min and max of x, y and z, a per-warp reduction and one atomic per value
__global__ void minMax3Kernel(const double* x, const double* y, const double* z, size_t n, unsigned long long* out)
{
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    {
        double v[3] = {x[i], y[i], z[i]};
        for (int k = 0; k < 3; ++k)
        {
            lo[k] = fmin(lo[k], v[k]);
            hi[k] = fmax(hi[k], v[k]);
        }
    }
    for (int k = 0; k < 3; ++k)
    {
        for (int off = 16; off > 0; off >>= 1)
        {
            lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0)
    {
        for (int k = 0; k < 3; ++k)
        {
            atomicMin(out + 2 * k, orderedBits(lo[k]));
            atomicMax(out + 2 * k + 1, orderedBits(hi[k]));
        }
    }
}

} // namespace

int predictH(size_t n, unsigned ng0, const unsigned* nc, const double* h, void* out, int outType, cudaStream_t s)
{
    if (outType != SPHB_F32 && outType != SPHB_F64) { return kErrArg; }
    if (n == 0) { return kOk; }
    predictHKernel<<<ceilDiv(n, 256), 256, 0, s>>>(n, ng0, nc, h, out, outType);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int setWords(unsigned long long* dst, int count, unsigned long long v0, unsigned long long v1, cudaStream_t s)
{
    if (count < 1 || count > 2) { return kErrArg; }
    setWordsKernel<<<1, 32, 0, s>>>(dst, count, v0, v1);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int minMax3(const double* x, const double* y, const double* z, size_t n, unsigned long long* out6, cudaStream_t s)
{
    minMax3InitKernel<<<1, 32, 0, s>>>(out6);
    int blocks = int(std::min<size_t>(std::max<size_t>(ceilDiv(n, 256), 1), size_t(smCount()) * 4));
    minMax3Kernel<<<blocks, 256, 0, s>>>(x, y, z, n, out6);
    countLaunch(2);
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

FixedFrame fixedFrameOf(const DevBox& box)
{
    FixedFrame fr;
    for (int k = 0; k < 3; ++k)
    {
        double span   = box.periodic[k] ? box.len[k] : 2.0 * box.len[k];
        fr.lo[k]      = box.lo[k];
        fr.invUnit[k] = 4294967296.0 / span;
        fr.unit[k]    = span / 4294967296.0;
    }
    return fr;
}

int packPositionsAndBoxes(const double* x, const double* y, const double* z, const double* m, size_t n, double4* pos,
                          int4* posq, const DevBox& box, float4* boxLo, float4* boxHi, cudaStream_t s)
{
    if (n == 0) { return kOk; }
    static_assert(256 % kBlockSize == 0 && kWarp % kBlockSize == 0, "runs must not straddle warps");
    packPosBoxesKernel<<<ceilDiv(n, 256), 256, 0, s>>>(x, y, z, m, n, pos, posq, fixedFrameOf(box), box, boxLo,
                                                       boxHi);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int packPositions(const double* x, const double* y, const double* z, const double* m, size_t n, double4* pos,
                  int4* posq, const DevBox& box, cudaStream_t s)
{
    if (n == 0) { return kOk; }
    packPosKernel<<<ceilDiv(n, 256), 256, 0, s>>>(x, y, z, m, n, pos, posq, fixedFrameOf(box));
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchPositions(size_t n, const IntegrateArrays<T>& a, const DevBox& box, double dt, double dtm1, double cv,
                    cudaStream_t s)
{
    if (n == 0) { return kOk; }
    positionsKernel<T><<<ceilDiv(n, 256), 256, 0, s>>>(n, a, box, dt, dtm1, cv);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int launchUpdateH(size_t n, unsigned ng0, const unsigned* nc, double* h, uint64_t* keys, unsigned* flag,
                  cudaStream_t s, const uint8_t* inst)
{
    if (n == 0) { return kOk; }
    updateHKernel<<<ceilDiv(n, 256), 256, 0, s>>>(n, ng0, nc, h, keys, flag, inst);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

int conservedSums(size_t n, const double* x, const double* y, const double* z, const double* vx, const double* vy,
                  const double* vz, const double* m, const double* temp, const unsigned* nc, double cv,
                  double* partial, int maxBlocks, double* out9, cudaStream_t s)
{
    int blocks = int(std::min<size_t>(std::max<size_t>(ceilDiv(n, kRedThreads), 1), size_t(maxBlocks)));
    conservedPartialKernel<<<blocks, kRedThreads, 0, s>>>(n, x, y, z, vx, vy, vz, m, temp, nc, cv, partial);
    conservedFinalKernel<<<1, 9 * 32, 0, s>>>(partial, blocks, out9);
    countLaunch(2);
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}


template int launchPositions<double>(size_t, const IntegrateArrays<double>&, const DevBox&, double, double, double,
                                     cudaStream_t);
template int launchPositions<float>(size_t, const IntegrateArrays<float>&, const DevBox&, double, double, double,
                                    cudaStream_t);

} // namespace sphb
