// Hand-written adjoint of the VE hydro step (sph/include/sph/hydro_ve/*_kern.hpp, sph/include/sph/positions.hpp,
// sph/include/sph/update_h.hpp) for a fixed time step, with the step's discrete structure held fixed: sort
// permutation, neighbour lists and counts, the smoothing-length factors of the neighbour-count iterations, and every
// branch (signal-velocity maximum, viscosity sign, Atwood ramp, AV-switch cases) as the forward took it.
//
// The kernels run in the reverse order of the forward chain. Each J-loop adjoint is one thread per target particle
// that recomputes its pair terms exactly as the forward kernel does (same separations, same kernel evaluation) and
// differentiates them: adjoints of the target's own inputs are summed in registers, adjoints of a neighbour's inputs
// are scattered with atomics. The derivative of the kernel W is that of what the forward evaluates: the slope of the
// interpolated table in FP64, the derivative of the fitted polynomial in FP32. A J-loop adjoint reads only adjoint
// fields that earlier launches have completed.
#include "adjoint.cuh"
#include "chain_detail.cuh"
#include "primitives.cuh"

namespace sphb
{

namespace
{

using namespace chain;

//! f and df/dv of the forward's linear table interpolation (the slope of the interval v falls in)
template<class T>
__device__ __forceinline__ void tableLookupD(const T* __restrict__ table, T v, T& f, T& df)
{
    constexpr int numIntervals = kTableSize - 1;
    constexpr T dx             = T(2.0) / numIntervals;
    constexpr T invDx          = T(1) / dx;
    int idx                    = int(v * invDx);
    if (idx >= numIntervals)
    {
        f  = T(0);
        df = T(0);
        return;
    }
    T t0         = __ldg(table + idx);
    T t1         = __ldg(table + idx + 1);
    T derivative = (t1 - t0) * invDx;
    f            = t0 + derivative * (v - T(idx) * dx);
    df           = derivative;
}

//! the forward's Horner polynomial in t = v^2/2 - 1 and its t-derivative, evaluated together
__device__ __forceinline__ void polyEvalD(const float (&c)[kPolyTerms], float v, float& p, float& dpdt)
{
    float t   = fmaf(0.5f * v, v, -1.0f);
    float acc = c[kPolyTerms - 1];
    float dac = 0.f;
#pragma unroll
    for (int q = kPolyTerms - 2; q >= 0; --q)
    {
        dac = fmaf(dac, t, acc);
        acc = fmaf(acc, t, c[q]);
    }
    p    = acc;
    dpdt = dac;
}

//! W(v) and dW/dv of the forward's kernelW
template<class T>
__device__ __forceinline__ void kernelWD(const T* __restrict__ table, const HydroConsts<T>& k, T v, T& w, T& dw)
{
    if constexpr (sizeof(T) == 4)
    {
        if (k.usePoly)
        {
            if (v < T(2))
            {
                float p, dp;
                polyEvalD(k.wpoly, v, p, dp);
                w  = p;
                dw = v * dp;
            }
            else
            {
                w  = T(0);
                dw = T(0);
            }
            return;
        }
    }
    tableLookupD(table, v, w, dw);
}

//! DW(v) and dDW/dv of the forward's kernelDW (FP32: DW = v Q(t))
template<class T>
__device__ __forceinline__ void kernelDWD(const T* __restrict__ table, const HydroConsts<T>& k, T v, T& d, T& dd)
{
    if constexpr (sizeof(T) == 4)
    {
        if (k.usePoly)
        {
            if (v < T(2))
            {
                float q, dq;
                polyEvalD(k.dwpoly, v, q, dq);
                d  = v * q;
                dd = q + v * v * dq;
            }
            else
            {
                d  = T(0);
                dd = T(0);
            }
            return;
        }
    }
    tableLookupD(table, v, d, dd);
}

template<class T>
struct V3
{
    T x, y, z;
};

template<class T>
__device__ __forceinline__ T dot3(const V3<T>& a, const V3<T>& b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

//! C r for the symmetric 3x3 matrix stored as (c11, c12, c13, c22, c23, c33)
template<class T>
__device__ __forceinline__ V3<T> symMul(const T (&c)[6], const V3<T>& r)
{
    return {c[0] * r.x + c[1] * r.y + c[2] * r.z, c[1] * r.x + c[3] * r.y + c[4] * r.z,
            c[2] * r.x + c[4] * r.y + c[5] * r.z};
}

/*! For tA = -(C r) W: accumulate s * d(tA . tAbar)/dC into cb (adjoint of the stored six entries, each off-diagonal
 *  entry used twice) with s = -W. */
template<class T>
__device__ __forceinline__ void symOuterAdd(T (&cb)[6], const V3<T>& tb, const V3<T>& r, T s)
{
    cb[0] += s * tb.x * r.x;
    cb[1] += s * (tb.x * r.y + tb.y * r.x);
    cb[2] += s * (tb.x * r.z + tb.z * r.x);
    cb[3] += s * tb.y * r.y;
    cb[4] += s * (tb.y * r.z + tb.z * r.y);
    cb[5] += s * tb.z * r.z;
}

template<class T>
__device__ __forceinline__ void loadC(const ChainArrays<T>& a, size_t i, T (&c)[6])
{
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        c[q] = a.cij[q][i];
    }
}

/*! the distance of a pair from its squared separation: FP64 by the square root, FP32 by one rsqrt, which also gives
 *  rinv = 1 / dist for the divisions by the distance (0 for coincident particles, whose terms the kernels skip) */
__device__ __forceinline__ void distOf(double r2, double& dist, double& rinv)
{
    dist = sqrt(r2);
    rinv = 0.0;
}
__device__ __forceinline__ void distOf(float r2, float& dist, float& rinv)
{
    rinv = r2 > 0.0f ? rsqrtf(r2) : 0.0f;
    dist = r2 * rinv;
}
//! x / dist: IEEE in FP64, by the reciprocal from distOf in FP32
__device__ __forceinline__ double overDist(double x, double dist, double) { return x / dist; }
__device__ __forceinline__ float overDist(float x, float, float rinv) { return x * rinv; }

//! 1 / x: IEEE in FP64, the fast approximate division in FP32
__device__ __forceinline__ double recipT(double x) { return 1.0 / x; }
__device__ __forceinline__ float recipT(float x) { return __fdividef(1.0f, x); }

//! scatter the adjoint of a neighbour's position (the pair separation is x_i - x_j)
template<class T>
__device__ __forceinline__ void scatterPos(const AdjArrays<T>& g, uint32_t j, const V3<T>& rb)
{
    atomicAdd(g.x + j, -rb.x);
    atomicAdd(g.y + j, -rb.y);
    atomicAdd(g.z + j, -rb.z);
}

template<class T>
__device__ __forceinline__ V3<T> sepV(const Sep<T>& r)
{
    return {r.rx, r.ry, r.rz};
}

// -------------------------------------------------------------------------------------------------------------------
// integration (positions.hpp:77-111) and end-of-step h update (update_h.hpp:12-33)
// -------------------------------------------------------------------------------------------------------------------
//! add the MomentumEnergy adjoint's vector-atomic neighbour sums (AdjArrays::jacc) into the per-field adjoints
template<class T>
__global__ void foldNeighbourSumsKernel(size_t n, AdjArrays<T> g)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    const float4* q = g.jacc + i * 5;
    float4 a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
    g.x[i] += a.x;
    g.y[i] += a.y;
    g.z[i] += a.z;
    g.h[i] += a.w;
    g.vx[i] += b.x;
    g.vy[i] += b.y;
    g.vz[i] += b.z;
    g.c[i] += b.w;
    g.cij[0][i] += c.x;
    g.cij[1][i] += c.y;
    g.cij[2][i] += c.z;
    g.cij[3][i] += c.w;
    g.cij[4][i] += d.x;
    g.cij[5][i] += d.y;
    g.alpha[i] += d.z;
    g.prho[i] += d.w;
    g.xm[i] += e.x;
    g.vol[i] += e.y;
}

template<class T>
__global__ void integrationVjpKernel(AdjointStepArgs s, const unsigned* nc, StateAdj post, StateAdj work,
                                     AdjArrays<T> g)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) { return; }
    const double dt = s.dt, dtm1 = s.dtm1, adt = fabs(dt);
    // kick-drift: x' = x + dX, x_m1' = dX, v' = vn + a dt with vn = x_m1 / dtm1 + dtm1 a / 2, dX = (vn + a |dt| / 2) dt
    const int P[3] = {0, 1, 2}, M1[3] = {9, 10, 11}, Vv[3] = {6, 7, 8};
    T* A[3] = {g.ax, g.ay, g.az};
#pragma unroll
    for (int q = 0; q < 3; ++q)
    {
        double xb   = post.f[P[q]][i];
        double dXb  = xb + post.f[M1[q]][i];
        double vnp1 = post.f[Vv[q]][i];
        double vnb  = vnp1 + dXb * dt;
        double ab   = vnp1 * dt + dXb * (0.5 * adt * dt) + vnb * (0.5 * dtm1);
        work.f[P[q]][i]  = xb;
        work.f[M1[q]][i] = vnb / dtm1;
        work.f[Vv[q]][i] = 0.0; // the step overwrites v: only the force terms depend on it
        A[q][i]          = T(ab);
    }
    // u' = u + du dt + (du - du_m1) |dt| dt / (2 dtm1), or u exp(u' dt / u) when that is negative; temp = u / cv
    double uOld  = s.cv * s.temp[i];
    double du    = s.du[i];
    double duM1  = s.duM1[i];
    double uLin  = uOld + du * dt + 0.5 * (du - duM1) / dtm1 * adt * dt;
    double uFinB = post.f[5][i] / s.cv;
    double uLinB, uOldB;
    if (uLin < 0.0)
    {
        double q = uLin * dt / uOld;
        double e = exp(q);
        uLinB    = uFinB * e * dt;
        uOldB    = uFinB * e * (1.0 - q) + uLinB;
    }
    else
    {
        uLinB = uFinB;
        uOldB = uFinB;
    }
    g.du[i]      = T(uLinB * (dt + 0.5 * adt * dt / dtm1) + post.f[12][i]);
    work.f[12][i] = -uLinB * 0.5 * adt * dt / dtm1;
    work.f[5][i]  = uOldB * s.cv;
    // h_end = h 0.5 (1 + 1023 ng0 / nc)^(1/10)
    unsigned c   = nc[i];
    double ratio = double(1023.0) * double(s.ng0) / double(c);
    work.f[3][i] = post.f[3][i] * 0.5 * pow(1.0 + ratio, 0.1);
    work.f[4][i] = post.f[4][i];
    work.f[13][i] = 0.0;
    g.alpha[i]   = T(post.f[13][i]);
}

// -------------------------------------------------------------------------------------------------------------------
// MomentumEnergy (momentum_energy_kern.hpp:65-222, avClean = false)
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void __launch_bounds__(kChainThreads) momentumEnergyVjpKernel(ChainArrays<T> a, HydroConsts<T> k,
                                                                         DevBox box, AdjArrays<T> g)
{
    Target t;
    if (!targetOf(a.n, a.nc, k.ngmax, t)) { return; }
    Pos<T> pi      = posOf(a, t.i);
    double hiD     = a.h[t.i];
    HydroRec<T> hr = a.hrec[t.i];
    GradRec<T> gr  = a.grec[t.i];
    T ci[6];
    loadC(a, t.i, ci);
    const T hi = T(hiD), mi = T(pi.m), cI = hr.c, kxi = a.kx[t.i], alphaI = gr.alpha, xmassi = hr.xm;
    const T rhoi = kxi * mi / xmassi, prhoi = hr.prho;
    const T hiInv = T(1) / hi, hiInv3 = hiInv * hiInv * hiInv;
    // reciprocals and logarithms reused by every pair (FP32: fast division, no IEEE slow path in the pair loop)
    const T invRhoi = recipT(rhoi), invXmi = recipT(xmassi);

    const V3<T> momB = {-k.K * g.ax[t.i], -k.K * g.ay[t.i], -k.K * g.az[t.i]};
    const T duB      = g.du[t.i];
    const T energyB  = k.K * prhoi * duB;
    const T aViscEB  = a.tape.avisc[t.i] > T(0) ? k.K * T(0.5) * duB : T(0);

    T prhoiB = k.K * a.tape.energy[t.i] * duB;
    T rhoiB = T(0), xmiB = T(0), hiB = T(0), ciB = T(0), alphaiB = T(0);
    V3<T> xiB = {0, 0, 0}, viB = {0, 0, 0};
    T ciCB[6] = {0, 0, 0, 0, 0, 0};

    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
        // one pair per iteration: unrolled over the chunk, the pair body overflowed the instruction cache
#pragma unroll 1
        for (unsigned q = 0; q < qn; ++q)
        {
            uint32_t j     = popChunk(js);
            Pos<T> pj      = posOf(a, j);
            HydroRec<T> hj = loadHydro(a.hrec + j);
            GradRec<T> gj  = loadGrad(a.grec + j);
            const T cj6[6] = {gj.c11, gj.c12, gj.c13, gj.c22, gj.c23, gj.c33};
            V3<T> r        = sepV(separation(pi, pj, 2.0 * hiD, box, k));
            T r2           = r.x * r.x + r.y * r.y + r.z * r.z;
            T rinv, dist;
            if constexpr (sizeof(T) == 4)
            {
                rinv = rsqrtf(r2);
                dist = r2 * rinv;
            }
            else
            {
                dist = sqrt(r2);
                rinv = T(1) / dist;
            }
            V3<T> vij      = {hr.vx - hj.vx, hr.vy - hj.vy, hr.vz - hj.vz};
            T v1 = dist * hiInv, v2 = dist * hj.hInv;
            T hjInv3 = hj.hInv * hj.hInv * hj.hInv;
            T wk1, dwk1, wk2, dwk2;
            kernelWD(a.wh, k, v1, wk1, dwk1);
            kernelWD(a.wh, k, v2, wk2, dwk2);
            T Wi = hiInv3 * wk1, Wj = hjInv3 * wk2;
            V3<T> cri = symMul(ci, r), crj = symMul(cj6, r);
            V3<T> tAi = {-cri.x * Wi, -cri.y * Wi, -cri.z * Wi};
            V3<T> tAj = {-crj.x * Wj, -crj.y * Wj, -crj.z * Wj};

            T mj = T(pj.m), cj = hj.c, xmassj = hj.xm;
            T rhoj    = fdiv(mj, hj.vol);
            T invRhoj = fdiv(hj.vol, mj);
            T rv      = dot3(r, vij);
            T wij     = rv * rinv;
            T visc = T(0), vijSignal = T(0);
            if (wij < T(0))
            {
                vijSignal = (alphaI + gj.alpha) * T(0.25) * (cI + cj) - T(2) * wij;
                visc      = -vijSignal * wij;
            }
            T aMom, bMom, sigma = T(0);
            int branch;
            // FP32 decides the branch without the division and needs the Atwood number only on the ramp
            T atwood = sizeof(T) == 4 ? T(0) : fdiv(fabs(rhoi - rhoj), rhoi + rhoj);
            // the forward's branch decision: FP32 compares the thresholds without the division
            bool belowMin = sizeof(T) == 4 ? fabs(rhoi - rhoj) < k.Atmin * (rhoi + rhoj) : atwood < k.Atmin;
            bool aboveMax = sizeof(T) == 4 ? fabs(rhoi - rhoj) > k.Atmax * (rhoi + rhoj) : atwood > k.Atmax;
            if (belowMin)
            {
                aMom   = xmassi * xmassi;
                bMom   = xmassj * xmassj;
                branch = 0;
            }
            else if (aboveMax)
            {
                aMom   = xmassi * xmassj;
                bMom   = aMom;
                branch = 1;
            }
            else
            {
                if constexpr (sizeof(T) == 4) { atwood = fdiv(fabs(rhoi - rhoj), rhoi + rhoj); }
                sigma = k.ramp * (atwood - k.Atmin);
                if constexpr (sizeof(T) == 4)
                {
                    T li = log2f(xmassi), lj = log2f(xmassj);
                    aMom = exp2f((T(2) - sigma) * li + sigma * lj);
                    bMom = exp2f((T(2) - sigma) * lj + sigma * li);
                }
                else
                {
                    aMom = pow(xmassi, T(2) - sigma) * pow(xmassj, sigma);
                    bMom = pow(xmassj, T(2) - sigma) * pow(xmassi, sigma);
                }
                branch = 2;
            }
            T aVisc = mj * invRhoi * visc;
            T bVisc = mj * invRhoj * visc;
            V3<T> aViscV = {T(0.5) * (aVisc * tAi.x + bVisc * tAj.x), T(0.5) * (aVisc * tAi.y + bVisc * tAj.y),
                            T(0.5) * (aVisc * tAi.z + bVisc * tAj.z)};
            T momI = mj * prhoi * aMom;
            T momJ = mj * hj.prho * bMom;

            // adjoints of the pair terms
            V3<T> avB = {momB.x + aViscEB * vij.x, momB.y + aViscEB * vij.y, momB.z + aViscEB * vij.z};
            T eFac    = energyB * mj * aMom;
            V3<T> tAiB = {momI * momB.x + eFac * vij.x + T(0.5) * aVisc * avB.x,
                          momI * momB.y + eFac * vij.y + T(0.5) * aVisc * avB.y,
                          momI * momB.z + eFac * vij.z + T(0.5) * aVisc * avB.z};
            V3<T> tAjB = {momJ * momB.x + T(0.5) * bVisc * avB.x, momJ * momB.y + T(0.5) * bVisc * avB.y,
                          momJ * momB.z + T(0.5) * bVisc * avB.z};
            T momIB  = dot3(momB, tAi);
            T momJB  = dot3(momB, tAj);
            T aViscB = T(0.5) * dot3(avB, tAi);
            T bViscB = T(0.5) * dot3(avB, tAj);
            V3<T> vijB = {eFac * tAi.x + aViscEB * aViscV.x, eFac * tAi.y + aViscEB * aViscV.y,
                          eFac * tAi.z + aViscEB * aViscV.z};
            T aMomB = energyB * mj * dot3(vij, tAi) + momIB * mj * prhoi;
            T bMomB = momJB * mj * hj.prho;
            prhoiB += momIB * mj * aMom;
            T prhojB = momJB * mj * bMom;
            T viscB  = aViscB * mj * invRhoi + bViscB * mj * invRhoj;
            rhoiB -= aViscB * aVisc * invRhoi;
            T rhojB = -bViscB * bVisc * invRhoj;
            T wijB = T(0), alphajB = T(0), cjB = T(0);
            if (wij < T(0))
            {
                T sigB = -viscB * wij;
                wijB   = -viscB * vijSignal - T(2) * sigB;
                T aB   = sigB * T(0.25) * (cI + cj);
                T cB   = sigB * T(0.25) * (alphaI + gj.alpha);
                alphaiB += aB;
                alphajB = aB;
                ciB += cB;
                cjB = cB;
            }
            T xmjB;
            if (branch == 0)
            {
                xmiB += T(2) * xmassi * aMomB;
                xmjB = T(2) * xmassj * bMomB;
            }
            else if (branch == 1)
            {
                T sB = aMomB + bMomB;
                xmiB += sB * xmassj;
                xmjB = sB * xmassi;
            }
            else
            {
                T invXmj  = recipT(xmassj);
                xmiB += (aMomB * (T(2) - sigma) * aMom + bMomB * sigma * bMom) * invXmi;
                xmjB      = (aMomB * sigma * aMom + bMomB * (T(2) - sigma) * bMom) * invXmj;
                T lnr     = log(xmassj) - log(xmassi);
                T sigmaB  = (aMomB * aMom - bMomB * bMom) * lnr;
                T atB     = sigmaB * k.ramp;
                T D       = rhoi + rhoj;
                T sgn     = rhoi > rhoj ? T(1) : T(-1);
                T invD = recipT(D);
                rhoiB += atB * (sgn - atwood) * invD;
                rhojB += atB * (-sgn - atwood) * invD;
            }
            // wij = rv / dist, rv = r . vij
            T rvB   = wijB * rinv;
            T distB = -wijB * wij * rinv;
            V3<T> rB = {rvB * vij.x, rvB * vij.y, rvB * vij.z};
            vijB.x += rvB * r.x;
            vijB.y += rvB * r.y;
            vijB.z += rvB * r.z;
            // tA = -(C r) W for i and j
            T WiB = -dot3(cri, tAiB);
            T WjB = -dot3(crj, tAjB);
            V3<T> ctb = symMul(ci, tAiB);
            rB.x -= Wi * ctb.x;
            rB.y -= Wi * ctb.y;
            rB.z -= Wi * ctb.z;
            symOuterAdd(ciCB, tAiB, r, -Wi);
            ctb = symMul(cj6, tAjB);
            rB.x -= Wj * ctb.x;
            rB.y -= Wj * ctb.y;
            rB.z -= Wj * ctb.z;
            T cjCB[6] = {0, 0, 0, 0, 0, 0};
            symOuterAdd(cjCB, tAjB, r, -Wj);
            // Wi = h_i^-3 W(dist / h_i), Wj likewise with h_j
            T v1B = WiB * hiInv3 * dwk1;
            hiB += WiB * (-T(3) * Wi * hiInv) - v1B * v1 * hiInv;
            distB += v1B * hiInv;
            T v2B = WjB * hjInv3 * dwk2;
            T hjB = WjB * (-T(3) * Wj * hj.hInv) - v2B * v2 * hj.hInv;
            distB += v2B * hj.hInv;
            if (dist > T(0))
            {
                T f = distB * rinv;
                rB.x += f * r.x;
                rB.y += f * r.y;
                rB.z += f * r.z;
            }
            xiB.x += rB.x;
            xiB.y += rB.y;
            xiB.z += rB.z;
            viB.x += vijB.x;
            viB.y += vijB.y;
            viB.z += vijB.z;
            // neighbour side
            if constexpr (sizeof(T) == 4)
            {
                if (g.jacc)
                {
                    float4* q = g.jacc + size_t(j) * 5;
                    atomicAdd(q + 0, make_float4(-rB.x, -rB.y, -rB.z, hjB));
                    atomicAdd(q + 1, make_float4(-vijB.x, -vijB.y, -vijB.z, cjB));
                    atomicAdd(q + 2, make_float4(cjCB[0], cjCB[1], cjCB[2], cjCB[3]));
                    atomicAdd(q + 3, make_float4(cjCB[4], cjCB[5], alphajB, prhojB));
                    atomicAdd(reinterpret_cast<float2*>(q + 4), make_float2(xmjB, -rhojB * rhoj / hj.vol));
                    continue;
                }
            }
            scatterPos(g, j, rB);
            atomicAdd(g.vx + j, -vijB.x);
            atomicAdd(g.vy + j, -vijB.y);
            atomicAdd(g.vz + j, -vijB.z);
            atomicAdd(g.h + j, hjB);
#pragma unroll
            for (int c = 0; c < 6; ++c)
            {
                atomicAdd(g.cij[c] + j, cjCB[c]);
            }
            atomicAdd(g.c + j, cjB);
            atomicAdd(g.prho + j, prhojB);
            atomicAdd(g.alpha + j, alphajB);
            atomicAdd(g.xm + j, xmjB);
            atomicAdd(g.vol + j, -rhojB * rhoj / hj.vol);
        }
    }
    // rho_i = kx_i m_i / xm_i
    xmiB -= rhoiB * rhoi / xmassi;
    atomicAdd(g.kx + t.i, rhoiB * mi / xmassi);
    atomicAdd(g.x + t.i, xiB.x);
    atomicAdd(g.y + t.i, xiB.y);
    atomicAdd(g.z + t.i, xiB.z);
    atomicAdd(g.vx + t.i, viB.x);
    atomicAdd(g.vy + t.i, viB.y);
    atomicAdd(g.vz + t.i, viB.z);
    atomicAdd(g.h + t.i, hiB);
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        atomicAdd(g.cij[c] + t.i, ciCB[c]);
    }
    atomicAdd(g.c + t.i, ciB);
    atomicAdd(g.prho + t.i, prhoiB);
    atomicAdd(g.alpha + t.i, alphaiB);
    atomicAdd(g.xm + t.i, xmiB);
}

// -------------------------------------------------------------------------------------------------------------------
// AV switches (av_switches_kern.hpp:43-137)
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void __launch_bounds__(kChainThreads) avSwitchesVjpKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box,
                                                                     double dt, const double* alphaPre,
                                                                     AdjArrays<T> g, double* alphaPreBar,
                                                                     double* alphamaxBar)
{
    Target t;
    bool valid        = targetOf(a.n, a.nc, k.ngmax, t);
    double alphamaxB  = 0.0;
    if (valid)
    {
        Pos<T> pi      = posOf(a, t.i);
        double hiD     = a.h[t.i];
        HydroRec<T> hr = a.hrec[t.i];
        GradRec<T> gr  = a.grec[t.i];
        T ci6[6];
        loadC(a, t.i, ci6);
        const T hi = T(hiD), cI = hr.c, divvI = gr.divv;
        const T hiInv = T(1) / hi, KhiInv3 = k.K * hiInv * hiInv * hiInv;
        const V3<T> gv = {a.tape.gx[t.i], a.tape.gy[t.i], a.tape.gz[t.i]};
        const T vsig   = a.tape.vsig[t.i];
        const T gnorm  = sqrt(gv.x * gv.x + gv.y * gv.y + gv.z * gv.z);
        const T alphaOld = T(alphaPre[t.i]);
        const T alphaNewB = g.alpha[t.i];

        // forward of the switch
        T alphaloc = T(0), aConst = T(0), den = T(1);
        if (divvI < T(0))
        {
            aConst   = hi * hi * gnorm;
            den      = aConst + hi * fabs(divvI) + T(0.05) * cI;
            alphaloc = k.alphamax * aConst / den;
        }
        T alphalocB = T(0), alphaOldB = T(0), vsigB = T(0), hiB = T(0), ciB = T(0), divviB = T(0);
        if (alphaloc >= alphaOld) { alphalocB = alphaNewB; }
        else
        {
            T decay    = hi / (k.decay * vsig);
            T target   = alphaloc >= k.alphamin ? alphaloc : k.alphamin;
            T alphadot = (target - alphaOld) / decay;
            T fdt      = T(dt) / decay;
            alphaOldB  = alphaNewB * (T(1) - fdt);
            T targetB  = alphaNewB * fdt;
            T decayB   = -alphaNewB * alphadot * T(dt) / decay;
            hiB += decayB / (k.decay * vsig);
            vsigB = -decayB * decay / vsig;
            if (alphaloc >= k.alphamin) { alphalocB = targetB; }
        }
        V3<T> gB = {0, 0, 0};
        if (divvI < T(0) && alphalocB != T(0))
        {
            alphamaxB = double(alphalocB * aConst / den);
            T aB   = alphalocB * k.alphamax * (den - aConst) / (den * den);
            T denB = -alphalocB * alphaloc / den;
            hiB += denB * fabs(divvI);
            divviB -= denB * hi; // |divv| = -divv here
            ciB += denB * T(0.05);
            hiB += aB * T(2) * hi * gnorm;
            T gnB = aB * hi * hi;
            if (gnorm > T(0))
            {
                T f = gnB / gnorm;
                gB  = {f * gv.x, f * gv.y, f * gv.z};
            }
        }
        V3<T> xiB = {0, 0, 0}, viB = {0, 0, 0};
        T ciCB[6] = {0, 0, 0, 0, 0, 0};
        // the signal velocity came from one neighbour: c_i + c_j - 3 rv / dist
        int js = a.tape.vsigJ[t.i];
        if (vsigB != T(0) && js >= 0)
        {
            uint32_t j     = uint32_t(js);
            Pos<T> pj      = posOf(a, j);
            HydroRec<T> hj = loadHydro(a.hrec + j);
            V3<T> r        = sepV(separation(pi, pj, 2.0 * hiD, box, k));
            T dist         = sqrt(r.x * r.x + r.y * r.y + r.z * r.z);
            V3<T> vij      = {hr.vx - hj.vx, hr.vy - hj.vy, hr.vz - hj.vz};
            T rv           = dot3(r, vij);
            if (rv < T(0))
            {
                ciB += vsigB;
                atomicAdd(g.c + j, vsigB);
                T rvB   = -T(3) * vsigB / dist;
                T distB = T(3) * vsigB * rv / (dist * dist);
                V3<T> rB = {rvB * vij.x + distB * r.x / dist, rvB * vij.y + distB * r.y / dist,
                            rvB * vij.z + distB * r.z / dist};
                V3<T> vB = {rvB * r.x, rvB * r.y, rvB * r.z};
                xiB = rB;
                viB = vB;
                scatterPos(g, j, rB);
                atomicAdd(g.vx + j, -vB.x);
                atomicAdd(g.vy + j, -vB.y);
                atomicAdd(g.vz + j, -vB.z);
            }
        }
        // gradient of divv: g = sum_j vol_j (divv_i - divv_j) tA, tA = -(C_i r) K h^-3 W
        if (gB.x != T(0) || gB.y != T(0) || gB.z != T(0))
        {
            for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
            {
                uint32_t jl[kNbChunk];
                loadChunk(a.nidx, t, t.ngPad, q0, jl);
                unsigned qn = min(kNbChunk, t.count - q0);
                // one pair per iteration, as the other adjoint pair loops
#pragma unroll 1
                for (unsigned q = 0; q < qn; ++q)
                {
                    uint32_t j     = popChunk(jl);
                    Pos<T> pj      = posOf(a, j);
                    HydroRec<T> hj = loadHydro(a.hrec + j);
                    T divvJ        = __ldg(reinterpret_cast<const T*>(a.grec + j) + 6);
                    V3<T> r        = sepV(separation(pi, pj, 2.0 * hiD, box, k));
                    T dist, rinv;
                    distOf(r.x * r.x + r.y * r.y + r.z * r.z, dist, rinv);
                    T v            = dist * hiInv;
                    T wk, dwk;
                    kernelWD(a.wh, k, v, wk, dwk);
                    T Wi      = KhiInv3 * wk;
                    V3<T> cr  = symMul(ci6, r);
                    V3<T> tA  = {-cr.x * Wi, -cr.y * Wi, -cr.z * Wi};
                    T f       = hj.vol * (divvI - divvJ);
                    T fB      = dot3(gB, tA);
                    V3<T> tAB = {f * gB.x, f * gB.y, f * gB.z};
                    atomicAdd(g.vol + j, fB * (divvI - divvJ));
                    divviB += fB * hj.vol;
                    atomicAdd(g.divv + j, -fB * hj.vol);
                    T WiB     = -dot3(cr, tAB);
                    V3<T> ctb = symMul(ci6, tAB);
                    V3<T> rB  = {-Wi * ctb.x, -Wi * ctb.y, -Wi * ctb.z};
                    symOuterAdd(ciCB, tAB, r, -Wi);
                    T vB = WiB * KhiInv3 * dwk;
                    hiB += WiB * (-T(3) * Wi * hiInv) - vB * v * hiInv;
                    if (dist > T(0))
                    {
                        T fd = overDist(vB * hiInv, dist, rinv);
                        rB.x += fd * r.x;
                        rB.y += fd * r.y;
                        rB.z += fd * r.z;
                    }
                    xiB.x += rB.x;
                    xiB.y += rB.y;
                    xiB.z += rB.z;
                    scatterPos(g, j, rB);
                }
            }
        }
        alphaPreBar[t.i] = double(alphaOldB);
        atomicAdd(g.x + t.i, xiB.x);
        atomicAdd(g.y + t.i, xiB.y);
        atomicAdd(g.z + t.i, xiB.z);
        atomicAdd(g.vx + t.i, viB.x);
        atomicAdd(g.vy + t.i, viB.y);
        atomicAdd(g.vz + t.i, viB.z);
        atomicAdd(g.h + t.i, hiB);
        atomicAdd(g.c + t.i, ciB);
        atomicAdd(g.divv + t.i, divviB);
#pragma unroll
        for (int c = 0; c < 6; ++c)
        {
            atomicAdd(g.cij[c] + t.i, ciCB[c]);
        }
    }
    // block sum of the alphamax adjoint -> one atomic per block
    double v = alphamaxB;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    __shared__ double warpSum[kChainThreads / 32];
    if ((threadIdx.x & 31) == 0) { warpSum[threadIdx.x >> 5] = v; }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double sum = 0.0;
        for (int w = 0; w < kChainThreads / 32; ++w)
        {
            sum += warpSum[w];
        }
        if (sum != 0.0) { atomicAdd(alphamaxBar, sum); }
    }
}

// -------------------------------------------------------------------------------------------------------------------
// divv (divv_curlv_kern.hpp:43-123; curlv feeds nothing downstream in the VE step)
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void __launch_bounds__(kChainThreads) divvVjpKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box,
                                                               AdjArrays<T> g)
{
    Target t;
    if (!targetOf(a.n, a.nc, k.ngmax, t)) { return; }
    const T divvB = g.divv[t.i];
    if (divvB == T(0)) { return; }
    Pos<T> pi      = posOf(a, t.i);
    double hiD     = a.h[t.i];
    HydroRec<T> hr = a.hrec[t.i];
    T ci6[6];
    loadC(a, t.i, ci6);
    const T hi = T(hiD), hiInv = T(1) / hi, kxi = a.kx[t.i], divv = a.divv[t.i];
    const T N  = k.K * hiInv * hiInv * hiInv / kxi;
    T hiB      = -T(3) * divvB * divv * hiInv;
    T kxiB     = -divvB * divv / kxi;
    const T DB = divvB * N;
    V3<T> xiB = {0, 0, 0}, viB = {0, 0, 0};
    T ciCB[6] = {0, 0, 0, 0, 0, 0};
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
        // one pair per iteration: the chunk stays in registers and the loop body is not replicated
#pragma unroll 1
        for (unsigned q = 0; q < qn; ++q)
        {
            uint32_t j     = popChunk(js);
            Pos<T> pj      = posOf(a, j);
            HydroRec<T> hj = loadHydro(a.hrec + j);
            V3<T> r        = sepV(separation(pi, pj, 2.0 * hiD, box, k));
            T dist, rinv;
            distOf(r.x * r.x + r.y * r.y + r.z * r.z, dist, rinv);
            T v            = dist * hiInv;
            T wk, dwk;
            kernelWD(a.wh, k, v, wk, dwk);
            V3<T> cr  = symMul(ci6, r);
            V3<T> tA  = {-cr.x * wk, -cr.y * wk, -cr.z * wk};
            V3<T> dv  = {hj.vx - hr.vx, hj.vy - hr.vy, hj.vz - hr.vz};
            // term = xm_j dv . tA
            V3<T> fB  = {DB * tA.x, DB * tA.y, DB * tA.z};
            V3<T> tAB = {DB * dv.x * hj.xm, DB * dv.y * hj.xm, DB * dv.z * hj.xm};
            atomicAdd(g.vx + j, fB.x * hj.xm);
            atomicAdd(g.vy + j, fB.y * hj.xm);
            atomicAdd(g.vz + j, fB.z * hj.xm);
            viB.x -= fB.x * hj.xm;
            viB.y -= fB.y * hj.xm;
            viB.z -= fB.z * hj.xm;
            atomicAdd(g.xm + j, DB * dot3(dv, tA));
            T wB      = -dot3(cr, tAB);
            V3<T> ctb = symMul(ci6, tAB);
            V3<T> rB  = {-wk * ctb.x, -wk * ctb.y, -wk * ctb.z};
            symOuterAdd(ciCB, tAB, r, -wk);
            T vB = wB * dwk;
            hiB -= vB * v * hiInv;
            if (dist > T(0))
            {
                T fd = overDist(vB * hiInv, dist, rinv);
                rB.x += fd * r.x;
                rB.y += fd * r.y;
                rB.z += fd * r.z;
            }
            xiB.x += rB.x;
            xiB.y += rB.y;
            xiB.z += rB.z;
            scatterPos(g, j, rB);
        }
    }
    atomicAdd(g.x + t.i, xiB.x);
    atomicAdd(g.y + t.i, xiB.y);
    atomicAdd(g.z + t.i, xiB.z);
    atomicAdd(g.vx + t.i, viB.x);
    atomicAdd(g.vy + t.i, viB.y);
    atomicAdd(g.vz + t.i, viB.z);
    atomicAdd(g.h + t.i, hiB);
    atomicAdd(g.kx + t.i, kxiB);
#pragma unroll
    for (int c = 0; c < 6; ++c)
    {
        atomicAdd(g.cij[c] + t.i, ciCB[c]);
    }
}

// -------------------------------------------------------------------------------------------------------------------
// IAD (iad_kern.hpp:43-110): C = (h^3 / K) tau^-1, tau = sum_j vol_j W(dist / h) r r^T
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void __launch_bounds__(kChainThreads) iadVjpKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box,
                                                              AdjArrays<T> g)
{
    Target t;
    if (!targetOf(a.n, a.nc, k.ngmax, t)) { return; }
    if (t.count == 0) { return; }
    T c[6], cb[6];
    loadC(a, t.i, c);
#pragma unroll
    for (int q = 0; q < 6; ++q)
    {
        cb[q] = g.cij[q][t.i];
    }
    Pos<T> pi  = posOf(a, t.i);
    double hiD = a.h[t.i];
    const T hi = T(hiD), hiInv = T(1) / hi;
    // dL/dh through the h^3 factor
    T hiB = T(3) * hiInv *
            (cb[0] * c[0] + cb[1] * c[1] + cb[2] * c[2] + cb[3] * c[3] + cb[4] * c[4] + cb[5] * c[5]);
    // full symmetric adjoint G of C (off-diagonal stored adjoints split over both entries), tauB = -(K/h^3) C G C
    const T G[3][3] = {{cb[0], T(0.5) * cb[1], T(0.5) * cb[2]},
                       {T(0.5) * cb[1], cb[3], T(0.5) * cb[4]},
                       {T(0.5) * cb[2], T(0.5) * cb[4], cb[5]}};
    const T C[3][3] = {{c[0], c[1], c[2]}, {c[1], c[3], c[4]}, {c[2], c[4], c[5]}};
    T CG[3][3];
#pragma unroll
    for (int p = 0; p < 3; ++p)
    {
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            CG[p][q] = C[p][0] * G[0][q] + C[p][1] * G[1][q] + C[p][2] * G[2][q];
        }
    }
    const T scale = -k.K * hiInv * hiInv * hiInv;
    T tb[3][3];
#pragma unroll
    for (int p = 0; p < 3; ++p)
    {
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            tb[p][q] = scale * (CG[p][0] * C[0][q] + CG[p][1] * C[1][q] + CG[p][2] * C[2][q]);
        }
    }
    V3<T> xiB = {0, 0, 0};
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
        // one pair per iteration: the chunk stays in registers and the loop body is not replicated
#pragma unroll 1
        for (unsigned q = 0; q < qn; ++q)
        {
            uint32_t j     = popChunk(js);
            Pos<T> pj      = posOf(a, j);
            HydroRec<T> hj = loadHydro(a.hrec + j);
            V3<T> r        = sepV(separation(pi, pj, 2.0 * hiD, box, k));
            T dist, rinv;
            distOf(r.x * r.x + r.y * r.y + r.z * r.z, dist, rinv);
            T v            = dist * hiInv;
            T wk, dwk;
            kernelWD(a.wh, k, v, wk, dwk);
            T w      = hj.vol * wk;
            V3<T> tr = {tb[0][0] * r.x + tb[0][1] * r.y + tb[0][2] * r.z,
                        tb[1][0] * r.x + tb[1][1] * r.y + tb[1][2] * r.z,
                        tb[2][0] * r.x + tb[2][1] * r.y + tb[2][2] * r.z};
            T wB     = dot3(r, tr);
            V3<T> rB = {T(2) * w * tr.x, T(2) * w * tr.y, T(2) * w * tr.z};
            atomicAdd(g.vol + j, wB * wk);
            T vB = wB * hj.vol * dwk;
            hiB -= vB * v * hiInv;
            if (dist > T(0))
            {
                T fd = overDist(vB * hiInv, dist, rinv);
                rB.x += fd * r.x;
                rB.y += fd * r.y;
                rB.z += fd * r.z;
            }
            xiB.x += rB.x;
            xiB.y += rB.y;
            xiB.z += rB.z;
            scatterPos(g, j, rB);
        }
    }
    atomicAdd(g.x + t.i, xiB.x);
    atomicAdd(g.y + t.i, xiB.y);
    atomicAdd(g.z + t.i, xiB.z);
    atomicAdd(g.h + t.i, hiB);
}

// -------------------------------------------------------------------------------------------------------------------
// per particle: vol = xm / kx, and the ideal-gas EOS prho = (gamma - 1) u / (m xm gradh), c = sqrt(gamma (gamma-1) u)
// (hydro_ve/eos.hpp:52-94 with rho = kx m / xm, p = rho u (gamma - 1))
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void volEosVjpKernel(ChainArrays<T> a, AdjointStepArgs s, AdjArrays<T> g, StateAdj work)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) { return; }
    T kx = a.kx[i], xm = a.xm[i];
    T vol  = a.hrec[i].vol;
    T volB = g.vol[i];
    T xmB  = g.xm[i] + volB / kx;
    T kxB  = g.kx[i] - volB * vol / kx;
    double u     = s.cv * s.temp[i];
    double prho  = double(a.prho[i]);
    double c     = double(a.c[i]);
    double prhoB = double(g.prho[i]);
    double cB    = double(g.c[i]);
    double uB    = 0.0;
    if (u > 0.0) { uB = prhoB * prho / u + cB * c / (2.0 * u); }
    xmB -= T(prhoB * prho / double(xm));
    g.gradh[i] = T(-prhoB * prho / double(a.gradh[i]));
    g.xm[i]    = xmB;
    g.kx[i]    = kxB;
    work.f[5][i] += s.cv * uB;
}

// -------------------------------------------------------------------------------------------------------------------
// VeDefGradh (ve_def_gradh_kern.hpp:43-90)
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void __launch_bounds__(kChainThreads) veDefGradhVjpKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box,
                                                                     AdjArrays<T> g)
{
    Target t;
    if (!targetOf(a.n, a.nc, k.ngmax, t)) { return; }
    Pos<T> pi  = posOf(a, t.i);
    double hiD = a.h[t.i];
    const T hi = T(hiD), mi = T(pi.m), xmi = a.xm[t.i], kxi = a.kx[t.i];
    const T hInv = T(1) / hi, h3Inv = hInv * hInv * hInv;
    const T whomega = a.tape.whomega[t.i], wrho0 = a.tape.wrho0[t.i];
    const T Omega   = whomega * mi / xmi + (kxi - k.K * xmi * h3Inv) * wrho0;
    const T rho     = kxi * mi / xmi;
    const T gradhB  = g.gradh[t.i];

    T OmegaB   = gradhB * hi / (T(3) * rho);
    T dhdrhoB  = -gradhB * Omega;
    T hiB      = -dhdrhoB / (T(3) * rho);
    T rhoB     = dhdrhoB * hi / (T(3) * rho * rho);
    T kxTotB   = g.kx[t.i] + rhoB * mi / xmi + OmegaB * wrho0;
    T xmiB     = -rhoB * rho / xmi - OmegaB * whomega * mi / (xmi * xmi) - OmegaB * k.K * h3Inv * wrho0;
    T whomegaB = OmegaB * mi / xmi;
    T wrho0B   = OmegaB * (kxi - k.K * xmi * h3Inv);
    hiB += OmegaB * wrho0 * T(3) * k.K * xmi * h3Inv * hInv;
    const T kxSB = kxTotB * k.K * h3Inv;
    hiB -= kxTotB * T(3) * kxi * hInv;
    const T whSB = whomegaB * k.K * h3Inv * hInv;
    hiB -= whomegaB * T(4) * whomega * hInv;
    const T wrSB = wrho0B * k.K * h3Inv * hInv;
    hiB -= wrho0B * T(4) * wrho0 * hInv;
    xmiB += kxSB - T(3) * whSB;

    V3<T> xiB = {0, 0, 0};
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
        // one pair per iteration: the chunk stays in registers and the loop body is not replicated
#pragma unroll 1
        for (unsigned q = 0; q < qn; ++q)
        {
            uint32_t j = popChunk(js);
            Pos<T> pj  = posOf(a, j);
            V3<T> r    = sepV(separation(pi, pj, 2.0 * hiD, box, k));
            T dist, rinv;
            distOf(r.x * r.x + r.y * r.y + r.z * r.z, dist, rinv);
            T v        = dist * hInv;
            T w, dw, d, dd;
            kernelWD(a.wh, k, v, w, dw);
            kernelDWD(a.whd, k, v, d, dd);
            T dterh  = -(T(3) * w + v * d);
            T xmassj = __ldg(a.xm + j);
            T mj     = T(pj.m);
            atomicAdd(g.xm + j, kxSB * w + whSB * dterh);
            T wB     = kxSB * xmassj;
            T dterhB = whSB * xmassj + wrSB * mj;
            T vB     = wB * dw - dterhB * (T(3) * dw + d + v * dd);
            hiB -= vB * v * hInv;
            if (dist > T(0))
            {
                T fd     = overDist(vB * hInv, dist, rinv);
                V3<T> rB = {fd * r.x, fd * r.y, fd * r.z};
                xiB.x += rB.x;
                xiB.y += rB.y;
                xiB.z += rB.z;
                scatterPos(g, j, rB);
            }
        }
    }
    atomicAdd(g.x + t.i, xiB.x);
    atomicAdd(g.y + t.i, xiB.y);
    atomicAdd(g.z + t.i, xiB.z);
    atomicAdd(g.h + t.i, hiB);
    atomicAdd(g.xm + t.i, xmiB);
}

// -------------------------------------------------------------------------------------------------------------------
// XMass (xmass_kern.hpp:50-79): xm = m h^3 / (K S), S = m_i + sum_j W(dist / h) m_j
// -------------------------------------------------------------------------------------------------------------------
template<class T>
__global__ void __launch_bounds__(kChainThreads) xmassVjpKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box,
                                                                AdjArrays<T> g)
{
    Target t;
    if (!targetOf(a.n, a.nc, k.ngmax, t)) { return; }
    const T xmB = g.xm[t.i];
    if (xmB == T(0)) { return; }
    Pos<T> pi  = posOf(a, t.i);
    double hiD = a.h[t.i];
    const T hi = T(hiD), mi = T(pi.m), xm = a.xm[t.i];
    const T hInv = T(1) / hi, h3Inv = hInv * hInv * hInv;
    const T S    = mi / (xm * k.K * h3Inv);
    const T SB   = -xmB * xm / S;
    T hiB        = T(3) * xmB * xm * hInv;
    V3<T> xiB    = {0, 0, 0};
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
        // one pair per iteration: the chunk stays in registers and the loop body is not replicated
#pragma unroll 1
        for (unsigned q = 0; q < qn; ++q)
        {
            uint32_t j = popChunk(js);
            Pos<T> pj  = posOf(a, j);
            V3<T> r    = sepV(separation(pi, pj, 2.0 * hiD, box, k));
            T dist, rinv;
            distOf(r.x * r.x + r.y * r.y + r.z * r.z, dist, rinv);
            T v        = dist * hInv;
            T w, dw;
            kernelWD(a.wh, k, v, w, dw);
            T vB = SB * T(pj.m) * dw;
            hiB -= vB * v * hInv;
            if (dist > T(0))
            {
                T fd     = overDist(vB * hInv, dist, rinv);
                V3<T> rB = {fd * r.x, fd * r.y, fd * r.z};
                xiB.x += rB.x;
                xiB.y += rB.y;
                xiB.z += rB.z;
                scatterPos(g, j, rB);
            }
        }
    }
    atomicAdd(g.x + t.i, xiB.x);
    atomicAdd(g.y + t.i, xiB.y);
    atomicAdd(g.z + t.i, xiB.z);
    atomicAdd(g.h + t.i, hiB);
}

/*! Sum the chain adjoints into the state adjoint, carry h back through the neighbour-count iterations
 *  (h_searched = h_pre * (h_searched / h_pre), a constant factor with the counts fixed) and scatter every field to the
 *  pre-sync particle order. */
template<class T>
__global__ void finalizeVjpKernel(ChainArrays<T> a, AdjointStepArgs s, AdjArrays<T> g, StateAdj work, StateAdj pre)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) { return; }
    double hPost = a.h[i];
    double hPre  = s.hPre[i];
    double vals[14];
#pragma unroll
    for (int f = 0; f < 14; ++f)
    {
        vals[f] = work.f[f][i];
    }
    vals[0] += double(g.x[i]);
    vals[1] += double(g.y[i]);
    vals[2] += double(g.z[i]);
    vals[3] = (vals[3] + double(g.h[i])) * (hPost / hPre);
    vals[6] += double(g.vx[i]);
    vals[7] += double(g.vy[i]);
    vals[8] += double(g.vz[i]);
    uint32_t dst = s.order[i];
#pragma unroll
    for (int f = 0; f < 14; ++f)
    {
        pre.f[f][dst] = vals[f];
    }
}

template<class T>
unsigned blocksFor(size_t n)
{
    return unsigned((n + kChainThreads - 1) / kChainThreads);
}

} // namespace

template<class T>
int stepVjp(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, const AdjointStepArgs& s,
            const StateAdj& post, const StateAdj& pre, AdjArrays<T> g, StateAdj work, cudaStream_t stream)
{
    if (s.n == 0) { return kOk; }
    unsigned nb = blocksFor<T>(s.n);
    // zero the chain adjoints (they are accumulated by scatter)
    T* fields[kNumAdjFields] = {g.x,      g.y,      g.z,      g.vx,     g.vy,     g.vz,    g.h,    g.c,  g.prho,
                                g.alpha,  g.cij[0], g.cij[1], g.cij[2], g.cij[3], g.cij[4], g.cij[5], g.divv, g.xm,
                                g.vol,    g.kx,     g.gradh,  g.ax,     g.ay,     g.az,     g.du};
    for (T* f : fields)
    {
        SPHB_CUDA_TRY(cudaMemsetAsync(f, 0, s.n * sizeof(T), stream));
    }
    integrationVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(s, a.nc, post, work, g);
    if (sizeof(T) == 4 && g.jacc)
    {
        SPHB_CUDA_TRY(cudaMemsetAsync(g.jacc, 0, a.n * 5 * sizeof(float4), stream));
    }
    momentumEnergyVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, k, box, g);
    if (sizeof(T) == 4 && g.jacc)
    {
        foldNeighbourSumsKernel<T><<<ceilDiv(a.n, 256), 256, 0, stream>>>(a.n, g);
        countLaunch();
    }
    avSwitchesVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, k, box, s.dtAV, s.alphaPre, g, work.f[13],
                                                              s.alphamaxBar);
    divvVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, k, box, g);
    iadVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, k, box, g);
    volEosVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, s, g, work);
    veDefGradhVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, k, box, g);
    xmassVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, k, box, g);
    finalizeVjpKernel<T><<<nb, kChainThreads, 0, stream>>>(a, s, g, work, pre);
    for (int q = 0; q < 9; ++q)
    {
        countLaunch();
    }
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template int stepVjp<double>(const ChainArrays<double>&, const HydroConsts<double>&, const DevBox&,
                             const AdjointStepArgs&, const StateAdj&, const StateAdj&, AdjArrays<double>, StateAdj,
                             cudaStream_t);
template int stepVjp<float>(const ChainArrays<float>&, const HydroConsts<float>&, const DevBox&,
                            const AdjointStepArgs&, const StateAdj&, const StateAdj&, AdjArrays<float>, StateAdj,
                            cudaStream_t);

} // namespace sphb
