// SPH-VE kernel chain on sm_100a: XMass, VeDefGradh (+ ideal-gas EOS), IAD + divv/curlv, AV switches,
// momentum-energy. One thread per target particle; a warp is a group of 32 consecutive SFC-ordered particles whose
// neighbour lists are read slot-major (one coalesced line per slot). Each J-loop walks the list in stored (ascending)
// order, like the reference CPU loops, and reads neighbour data through the packed records of hydro.cuh.
//
// T = double: the plain FP64 drop-in. Positions are FP64, the periodic shift is the reference's, sums run in list
// order with the reference's expression order, so results differ from the reference CPU only by FMA contraction.
//
// T = float: the mixed form. Pair separations come from 32-bit fixed-point coordinates (exact integer differences,
// periodic wrap by overflow; one unit = L / 2^32), all pair arithmetic is FP32, the kernel W is a degree-12
// polynomial instead of a table, and every neighbour sum is block-compensated: plain FP32 partial sums over blocks of
// 8 neighbours, each added to a Kahan-compensated FP32 accumulator.
#include "chain_detail.cuh"
#include "hydro.cuh"
#include "neighbors.cuh"
#include "primitives.cuh"

namespace sphb
{

namespace
{

using namespace chain;

// ---------------------------------------------------------------------------------------------------------------
// XMass: rho0_i = (m_i + sum_j W_ij m_j) K / h_i^3, xm_i = m_i / rho0_i (sph/include/sph/hydro_ve/xmass_kern.hpp:50-79)
// ---------------------------------------------------------------------------------------------------------------
// FP32: at most 32 registers, eight 256-thread blocks per SM: more gathers in flight (0.348 -> 0.325 ms at 128^3)
template<class T, int kMode>
__global__ void __launch_bounds__(kChainMaxThreads, sizeof(T) == 4 ? 8 : 0)
    xmassKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box)
{
    Target t;
    if (!chainTarget<kMode>(a, k.ngmax, t)) { return; }
    Pos<T> pi  = posOf(a, t.i);
    double hiD = a.h[t.i];
    T hi       = T(hiD);
    T mi       = T(pi.m);
    T hInv     = T(1.0) / hi;
    T h3Inv    = hInv * hInv * hInv;
    T hh       = T(0.5) * hInv * hInv;

    BlockSum<T> rho0(mi);
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
#pragma unroll
        for (unsigned q = 0; q < kNbChunk; ++q)
        {
            if (q >= qn) { break; }
            uint32_t j = js[q];
            Pos<T> pj  = posOf(a, j);
            Sep<T> r   = separation(pi, pj, 2.0 * hiD, box, k);
            T r2       = r.rx * r.rx + r.ry * r.ry + r.rz * r.rz;
            rho0.add(kernelWr2(a.wh, k, r2, hInv, hh) * T(pj.m));
        }
        rho0.flush();
    }
    a.xm[t.i] = mi / (rho0.get() * k.K * h3Inv);
}

// ---------------------------------------------------------------------------------------------------------------
// VeDefGradh (sph/include/sph/hydro_ve/ve_def_gradh_kern.hpp:43-90) + ideal-gas EOS (hydro_ve/eos.hpp:52-94,
// sph/include/sph/eos.hpp:19-50); writes kx, gradh, prho, c and the hydro record of the particle.
// ---------------------------------------------------------------------------------------------------------------
// FP32: at most 40 registers, six 256-thread blocks per SM, for the gathers' latency (0.625 -> 0.566 ms at 128^3,
// though it spills a little; 48 registers gave 0.588, 32 gave 0.582)
template<class T, int kMode>
__global__ void __launch_bounds__(kChainMaxThreads, sizeof(T) == 4 ? 6 : 0)
    veDefGradhEosKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box)
{
    Target t;
    if (!chainTarget<kMode>(a, k.ngmax, t)) { return; }
    Pos<T> pi  = posOf(a, t.i);
    double hiD = a.h[t.i];
    T hi       = T(hiD);
    T mi       = T(pi.m);
    T xmassi   = a.xm[t.i];
    T hInv     = T(1) / hi;
    T h3Inv    = hInv * hInv * hInv;
    [[maybe_unused]] float hhV = 0.5f * float(hInv) * float(hInv);

    BlockSum<T> kxS(xmassi), whomegaS(-T(3) * xmassi), wrho0S(-T(3) * mi);
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
#pragma unroll
        for (unsigned q = 0; q < kNbChunk; ++q)
        {
            if (q >= qn) { break; }
            uint32_t j = js[q];
            Pos<T> pj  = posOf(a, j);
            Sep<T> r   = separation(pi, pj, 2.0 * hiD, box, k);
            T r2       = r.rx * r.rx + r.ry * r.ry + r.rz * r.rz;
            T w, dterh;
            if constexpr (sizeof(T) == 4)
            {
                if (k.usePoly)
                {
                    // t = v^2/2 - 1 from r2 (no square root); W and dW's polynomial side by side in packed FP32
                    // (sm_100 FFMA2); v dW = v^2 P'(t) = 2 (t + 1) P'(t) (0.638 -> 0.624 ms at 128^3)
                    float tt   = fmaf(r2, hhV, -1.0f);
                    float2 acc = make_float2(k.wpoly[kPolyTerms - 1], k.dwpoly[kPolyTerms - 1]);
#pragma unroll
                    for (int p = kPolyTerms - 2; p >= 0; --p)
                    {
                        acc = __ffma2_rn(acc, make_float2(tt, tt), make_float2(k.wpoly[p], k.dwpoly[p]));
                    }
                    bool in = tt < 1.0f;
                    w       = in ? acc.x : 0.0f;
                    dterh   = in ? -(3.0f * acc.x + 2.0f * (tt + 1.0f) * acc.y) : 0.0f;
                }
                else
                {
                    T vloc = T(r2 * rsqrtf(float(r2))) * hInv;
                    w      = kernelW(a.wh, k, vloc);
                    dterh  = -(T(3) * w + vloc * kernelDW(a.whd, k, vloc));
                }
            }
            else
            {
                T vloc = T(sqrt(r2)) * hInv;
                w      = kernelW(a.wh, k, vloc);
                T dw   = kernelDW(a.whd, k, vloc);
                dterh  = -(T(3) * w + vloc * dw);
            }
            T xmassj   = __ldg(a.xm + j);
            kxS.add(w * xmassj);
            whomegaS.add(dterh * xmassj);
            wrho0S.add(dterh * T(pj.m));
        }
        kxS.flush();
        whomegaS.flush();
        wrho0S.flush();
    }
    T kxi      = kxS.get() * (k.K * h3Inv);
    T whomegai = whomegaS.get() * (k.K * h3Inv * hInv);
    T wrho0i   = wrho0S.get() * (k.K * h3Inv * hInv);
    if constexpr (kMode & kModeTape)
    {
        a.tape.whomega[t.i] = whomegai;
        a.tape.wrho0[t.i]   = wrho0i;
    }
    whomegai   = whomegai * mi / xmassi + (kxi - k.K * xmassi * h3Inv) * wrho0i;
    T rhoi     = kxi * mi / xmassi;
    T dhdrho   = -hi / (rhoi * T(3));
    T gradhi   = T(1) - dhdrho * whomegai;

    // EOS in FP64 (per particle): rho = kx m / xm, p = rho u (gamma - 1), c = sqrt(gamma u (gamma - 1))
    double gamma = k.gamma, cv = k.cv;
    if constexpr (kMode & kModeBatch)
    {
        uint8_t q = a.batch.inst[t.i];
        gamma     = a.batch.gamma[q];
        cv        = a.batch.cv[q];
    }
    double rho  = double(kxi) * double(mi) / double(xmassi);
    double u    = cv * a.temp[t.i];
    double tmp  = u * (gamma - 1.0);
    double p    = rho * tmp;
    double c    = sqrt(gamma * tmp);
    double prho = p / (double(kxi) * double(mi) * double(mi) * double(gradhi));

    a.kx[t.i]    = kxi;
    a.gradh[t.i] = gradhi;
    a.prho[t.i]  = T(prho);
    a.c[t.i]     = T(c);
    if (a.recordNoVelocity)
    {
        a.hrec[t.i] = HydroRec<T>{T(0), T(0), T(0), T(1) / hi, xmassi, xmassi / kxi, T(c), T(prho)};
    }
    else
    {
        a.hrec[t.i] = HydroRec<T>{T(a.vx[t.i]), T(a.vy[t.i]), T(a.vz[t.i]), T(1) / hi, xmassi, xmassi / kxi, T(c),
                                  T(prho)};
    }
}

//! the velocity part of the hydro record, the same values VeDefGradh writes there otherwise
template<class T>
__global__ void packVelocityKernel(size_t n, const double* __restrict__ vx, const double* __restrict__ vy,
                                   const double* __restrict__ vz, HydroRec<T>* __restrict__ hrec)
{
    size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) { return; }
    hrec[i].vx = T(vx[i]);
    hrec[i].vy = T(vy[i]);
    hrec[i].vz = T(vz[i]);
}

// ---------------------------------------------------------------------------------------------------------------
// IAD (sph/include/sph/hydro_ve/iad_kern.hpp:43-110) then divv/curlv with the particle's own c_ij
// (sph/include/sph/hydro_ve/divv_curlv_kern.hpp:43-123); also the running max of divv for the rho time step.
// ---------------------------------------------------------------------------------------------------------------
template<class T>
__device__ __forceinline__ int expOf(T v)
{
    return v == T(0) ? 0 : ilogb(v);
}

template<class T, int kMode>
__global__ void __launch_bounds__(kChainMaxThreads) iadDivvCurlvKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box)
{
    Target t;
    bool valid     = chainTarget<kMode>(a, k.ngmax, t);
    double divvOut = -INFINITY;
    if (valid)
    {
        Pos<T> pi  = posOf(a, t.i);
        double hiD = a.h[t.i];
        T hi       = T(hiD);
        T hiInv    = T(1) / hi;

        BlockSum<T> s11, s12, s13, s22, s23, s33;
        for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
        {
            uint32_t js[kNbChunk];
            loadChunk(a.nidx, t, t.ngPad, q0, js);
            unsigned qn = min(kNbChunk, t.count - q0);
#pragma unroll
            for (unsigned q = 0; q < kNbChunk; ++q)
            {
                if (q >= qn) { break; }
                uint32_t j = js[q];
                Pos<T> pj      = posOf(a, j);
                HydroRec<T> hj = loadHydro(a.hrec + j);
                Sep<T> r       = separation(pi, pj, 2.0 * hiD, box, k);
                T dist         = sqrt(r.rx * r.rx + r.ry * r.ry + r.rz * r.rz);
                T w            = kernelW(a.wh, k, dist * hiInv);
                T voljW        = hj.vol * w;
                s11.add(r.rx * r.rx * voljW);
                s12.add(r.rx * r.ry * voljW);
                s13.add(r.rx * r.rz * voljW);
                s22.add(r.ry * r.ry * voljW);
                s23.add(r.ry * r.rz * voljW);
                s33.add(r.rz * r.rz * voljW);
            }
            s11.flush();
            s12.flush();
            s13.flush();
            s22.flush();
            s23.flush();
            s33.flush();
        }
        T tau11 = s11.get(), tau12 = s12.get(), tau13 = s13.get();
        T tau22 = s22.get(), tau23 = s23.get(), tau33 = s33.get();
        int expSum = expOf(tau11) + expOf(tau12) + expOf(tau13) + expOf(tau22) + expOf(tau23) + expOf(tau33);
        T norm     = ldexp(T(1), -expSum / 6);
        tau11 *= norm;
        tau12 *= norm;
        tau13 *= norm;
        tau22 *= norm;
        tau23 *= norm;
        tau33 *= norm;
        T det = tau11 * tau22 * tau33 + T(2) * tau12 * tau23 * tau13 - tau11 * tau23 * tau23 - tau22 * tau13 * tau13 -
                tau33 * tau12 * tau12;
        T factor = norm * (hi * hi * hi) / (det * k.K);
        if (isnan(factor) && t.count == 0) { factor = T(0); }
        T c11i = (tau22 * tau33 - tau23 * tau23) * factor;
        T c12i = (tau13 * tau23 - tau33 * tau12) * factor;
        T c13i = (tau12 * tau23 - tau22 * tau13) * factor;
        T c22i = (tau11 * tau33 - tau13 * tau13) * factor;
        T c23i = (tau13 * tau12 - tau11 * tau23) * factor;
        T c33i = (tau11 * tau22 - tau12 * tau12) * factor;

        HydroRec<T> hrI = a.hrec[t.i];
        T vxi = hrI.vx, vyi = hrI.vy, vzi = hrI.vz;
        T kxi = a.kx[t.i];
        BlockSum<T> dVxx, dVxy, dVxz, dVyx, dVyy, dVyz, dVzx, dVzy, dVzz;
        for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
        {
            uint32_t js[kNbChunk];
            loadChunk(a.nidx, t, t.ngPad, q0, js);
            unsigned qn = min(kNbChunk, t.count - q0);
#pragma unroll
            for (unsigned q = 0; q < kNbChunk; ++q)
            {
                if (q >= qn) { break; }
                uint32_t j = js[q];
                Pos<T> pj      = posOf(a, j);
                HydroRec<T> hj = loadHydro(a.hrec + j);
                Sep<T> r       = separation(pi, pj, 2.0 * hiD, box, k);
                T dist         = sqrt(r.rx * r.rx + r.ry * r.ry + r.rz * r.rz);
                T Wi           = kernelW(a.wh, k, dist * hiInv);
                T tA0          = -(c11i * r.rx + c12i * r.ry + c13i * r.rz) * Wi;
                T tA1          = -(c12i * r.rx + c22i * r.ry + c23i * r.rz) * Wi;
                T tA2          = -(c13i * r.rx + c23i * r.ry + c33i * r.rz) * Wi;
                T fx           = (hj.vx - vxi) * hj.xm;
                T fy           = (hj.vy - vyi) * hj.xm;
                T fz           = (hj.vz - vzi) * hj.xm;
                dVxx.add(fx * tA0);
                dVxy.add(fx * tA1);
                dVxz.add(fx * tA2);
                dVyx.add(fy * tA0);
                dVyy.add(fy * tA1);
                dVyz.add(fy * tA2);
                dVzx.add(fz * tA0);
                dVzy.add(fz * tA1);
                dVzz.add(fz * tA2);
            }
            dVxx.flush();
            dVxy.flush();
            dVxz.flush();
            dVyx.flush();
            dVyy.flush();
            dVyz.flush();
            dVzx.flush();
            dVzy.flush();
            dVzz.flush();
        }
        T hiInv3 = hiInv * hiInv * hiInv;
        T normKx = k.K * hiInv3 / kxi;
        T divv   = normKx * (dVxx.get() + dVyy.get() + dVzz.get());
        T cx     = dVzy.get() - dVyz.get();
        T cy     = dVxz.get() - dVzx.get();
        T cz     = dVyx.get() - dVxy.get();
        T curlv  = normKx * sqrt(cx * cx + cy * cy + cz * cz);
        if constexpr (kMode & kModeAvClean)
        {
            DVRec<T> g{{normKx * dVxx.get(), normKx * (dVxy.get() + dVyx.get()), normKx * (dVxz.get() + dVzx.get()),
                        normKx * dVyy.get(), normKx * (dVyz.get() + dVzy.get()), normKx * dVzz.get()},
                       T(0),
                       T(0)};
            a.dvrec[t.i] = g;
#pragma unroll
            for (int q = 0; q < 6; ++q)
            {
                a.dv[q][t.i] = g.dv[q];
            }
        }

        a.cij[0][t.i] = c11i;
        a.cij[1][t.i] = c12i;
        a.cij[2][t.i] = c13i;
        a.cij[3][t.i] = c22i;
        a.cij[4][t.i] = c23i;
        a.cij[5][t.i] = c33i;
        a.divv[t.i]   = divv;
        a.curlv[t.i]  = curlv;
        a.grec[t.i]   = GradRec<T>{c11i, c12i, c13i, c22i, c23i, c33i, divv, T(a.alpha[t.i])};
        a.avrec[t.i]  = AVRec<T>{hrI.vx, hrI.vy, hrI.vz, hrI.c, hrI.vol, divv, T(0), T(0)};
        divvOut       = double(divv);
    }
    reduceOrdered<true, (kMode & kModeBatch) != 0>(divvOut, a.n, a.reduce + 0, a.batch, 0);
}

/*! FP32 IAD + divv/curlv in one pass over the list. The divv/curlv loop of the reference sums, per pair,
 *  f_a tA_b with f = (v_j - v_i) xm_j and tA = -(C_i r) W, i.e. dV_ab = -sum_c C_bc M_ac with
 *  M_ac = sum_j f_a r_c W: M is accumulated in the same pass as tau, and C_i, known only after the pass, is applied
 *  to the nine sums at the end. Same quantities, one gather of each neighbour instead of two. */
// at most 80 registers (three 256-thread blocks per SM), as MomentumEnergy: measured 1.04 -> 0.95 ms at 128^3 against
// 87 registers
template<int kMode>
__global__ void __launch_bounds__(kChainMaxThreads, 3) iadDivvCurlvFusedKernel(ChainArrays<float> a,
                                                                              HydroConsts<float> k, DevBox box)
{
    using T = float;
    Target t;
    bool valid     = chainTarget<kMode>(a, k.ngmax, t);
    double divvOut = -INFINITY;
    if (valid)
    {
        Pos<T> pi      = posOf(a, t.i);
        double hiD     = a.h[t.i];
        T hi           = T(hiD);
        T hiInv        = T(1) / hi;
        T hh           = T(0.5) * hiInv * hiInv;
        HydroRec<T> hr = a.hrec[t.i];

        BlockSum<T> s11, s12, s13, s22, s23, s33;
        BlockSum<T> mxx, mxy, mxz, myx, myy, myz, mzx, mzy, mzz;
        for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
        {
            uint32_t js[kNbChunk];
            loadChunk(a.nidx, t, t.ngPad, q0, js);
            unsigned qn = min(kNbChunk, t.count - q0);
#pragma unroll
            for (unsigned q = 0; q < kNbChunk; ++q)
            {
                if (q >= qn) { break; }
                uint32_t j     = js[q];
                Pos<T> pj      = posOf(a, j);
                HydroRec<T> hj = loadHydro(a.hrec + j);
                Sep<T> r       = separation(pi, pj, 2.0 * hiD, box, k);
                T r2           = r.rx * r.rx + r.ry * r.ry + r.rz * r.rz;
                T w            = kernelWr2(a.wh, k, r2, hiInv, hh);
                T voljW        = hj.vol * w;
                s11.add(r.rx * r.rx * voljW);
                s12.add(r.rx * r.ry * voljW);
                s13.add(r.rx * r.rz * voljW);
                s22.add(r.ry * r.ry * voljW);
                s23.add(r.ry * r.rz * voljW);
                s33.add(r.rz * r.rz * voljW);
                T xw = hj.xm * w;
                T fx = (hj.vx - hr.vx) * xw;
                T fy = (hj.vy - hr.vy) * xw;
                T fz = (hj.vz - hr.vz) * xw;
                mxx.add(fx * r.rx);
                mxy.add(fx * r.ry);
                mxz.add(fx * r.rz);
                myx.add(fy * r.rx);
                myy.add(fy * r.ry);
                myz.add(fy * r.rz);
                mzx.add(fz * r.rx);
                mzy.add(fz * r.ry);
                mzz.add(fz * r.rz);
            }
            s11.flush();
            s12.flush();
            s13.flush();
            s22.flush();
            s23.flush();
            s33.flush();
            mxx.flush();
            mxy.flush();
            mxz.flush();
            myx.flush();
            myy.flush();
            myz.flush();
            mzx.flush();
            mzy.flush();
            mzz.flush();
        }
        T tau11 = s11.get(), tau12 = s12.get(), tau13 = s13.get();
        T tau22 = s22.get(), tau23 = s23.get(), tau33 = s33.get();
        int expSum = expOf(tau11) + expOf(tau12) + expOf(tau13) + expOf(tau22) + expOf(tau23) + expOf(tau33);
        T norm     = ldexp(T(1), -expSum / 6);
        tau11 *= norm;
        tau12 *= norm;
        tau13 *= norm;
        tau22 *= norm;
        tau23 *= norm;
        tau33 *= norm;
        T det = tau11 * tau22 * tau33 + T(2) * tau12 * tau23 * tau13 - tau11 * tau23 * tau23 - tau22 * tau13 * tau13 -
                tau33 * tau12 * tau12;
        T factor = norm * (hi * hi * hi) / (det * k.K);
        if (isnan(factor) && t.count == 0) { factor = T(0); }
        T c11i = (tau22 * tau33 - tau23 * tau23) * factor;
        T c12i = (tau13 * tau23 - tau33 * tau12) * factor;
        T c13i = (tau12 * tau23 - tau22 * tau13) * factor;
        T c22i = (tau11 * tau33 - tau13 * tau13) * factor;
        T c23i = (tau13 * tau12 - tau11 * tau23) * factor;
        T c33i = (tau11 * tau22 - tau12 * tau12) * factor;

        // dV_ab = -sum_c C_bc M_ac
        T M[3][3] = {{mxx.get(), mxy.get(), mxz.get()}, {myx.get(), myy.get(), myz.get()},
                     {mzx.get(), mzy.get(), mzz.get()}};
        T C[3][3] = {{c11i, c12i, c13i}, {c12i, c22i, c23i}, {c13i, c23i, c33i}};
        T dV[3][3];
#pragma unroll
        for (int p = 0; p < 3; ++p)
        {
#pragma unroll
            for (int q = 0; q < 3; ++q)
            {
                dV[p][q] = -(C[q][0] * M[p][0] + C[q][1] * M[p][1] + C[q][2] * M[p][2]);
            }
        }
        T hiInv3 = hiInv * hiInv * hiInv;
        T normKx = k.K * hiInv3 / a.kx[t.i];
        T divv   = normKx * (dV[0][0] + dV[1][1] + dV[2][2]);
        T cx     = dV[2][1] - dV[1][2];
        T cy     = dV[0][2] - dV[2][0];
        T cz     = dV[1][0] - dV[0][1];
        T curlv  = normKx * sqrt(cx * cx + cy * cy + cz * cz);
        if constexpr (kMode & kModeAvClean)
        {
            DVRec<T> g{{normKx * dV[0][0], normKx * (dV[0][1] + dV[1][0]), normKx * (dV[0][2] + dV[2][0]),
                        normKx * dV[1][1], normKx * (dV[1][2] + dV[2][1]), normKx * dV[2][2]},
                       T(0),
                       T(0)};
            a.dvrec[t.i] = g;
#pragma unroll
            for (int q = 0; q < 6; ++q)
            {
                a.dv[q][t.i] = g.dv[q];
            }
        }

        a.cij[0][t.i] = c11i;
        a.cij[1][t.i] = c12i;
        a.cij[2][t.i] = c13i;
        a.cij[3][t.i] = c22i;
        a.cij[4][t.i] = c23i;
        a.cij[5][t.i] = c33i;
        a.divv[t.i]   = divv;
        a.curlv[t.i]  = curlv;
        a.grec[t.i]   = GradRec<T>{c11i, c12i, c13i, c22i, c23i, c33i, divv, T(a.alpha[t.i])};
        a.avrec[t.i]  = AVRec<T>{hr.vx, hr.vy, hr.vz, hr.c, hr.vol, divv, T(0), T(0)};
        divvOut       = double(divv);
    }
    reduceOrdered<true, (kMode & kModeBatch) != 0>(divvOut, a.n, a.reduce + 0, a.batch, 0);
}

// ---------------------------------------------------------------------------------------------------------------
// AV switches (sph/include/sph/hydro_ve/av_switches_kern.hpp:43-137)
// ---------------------------------------------------------------------------------------------------------------
// FP32: up to 384 threads, run in 384-thread blocks (12 consecutive groups sharing their neighbours in L1), measured
// 0.817 -> 0.795 ms at 128^3 against 256; at most 56 registers for three such blocks per SM. FP64 keeps the common
// bound with no block minimum (0): an explicit minimum of 1 raised it from 96 to 108 registers and slowed it from
// 2.45 to 2.64 ms at 128 threads.
template<class T, int kMode>
__global__ void __launch_bounds__(sizeof(T) == 4 ? kAvMaxThreads : kChainMaxThreads, sizeof(T) == 4 ? 3 : 0)
    avSwitchesKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box, double dt)
{
    Target t;
    if (!chainTarget<kMode>(a, k.ngmax, t)) { return; }
    Pos<T> pi      = posOf(a, t.i);
    double hiD     = a.h[t.i];
    HydroRec<T> hr = a.hrec[t.i];
    GradRec<T> gr  = a.grec[t.i];
    T hi           = T(hiD);
    T ci           = hr.c;
    T vijsignalI   = T(1.e-40) * ci;
    T hiInv        = T(1) / hi;
    T hiInv3       = hiInv * hiInv * hiInv;
    T KhiInv3      = k.K * hiInv3;
    T hh           = T(0.5) * hiInv * hiInv;
    T divvI        = gr.divv;

    BlockSum<T> gx, gy, gz;
    int vsigJ = -1;
    for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
    {
        uint32_t js[kNbChunk];
        loadChunk(a.nidx, t, t.ngPad, q0, js);
        unsigned qn = min(kNbChunk, t.count - q0);
#pragma unroll
        for (unsigned q = 0; q < kNbChunk; ++q)
        {
            if (q >= qn) { break; }
            uint32_t j = js[q];
            Pos<T> pj      = posOf(a, j);
            AVRec<T> hj    = loadAV(a.avrec + j);
            T divvJ        = hj.divv;
            Sep<T> r       = separation(pi, pj, 2.0 * hiD, box, k);
            T r2           = r.rx * r.rx + r.ry * r.ry + r.rz * r.rz;
            T rv           = r.rx * (hr.vx - hj.vx) + r.ry * (hr.vy - hj.vy) + r.rz * (hr.vz - hj.vz);
            T vsig         = T(0);
            if (rv < T(0))
            {
                // FP32: 3 r.v / r with one rsqrt; FP64: the reference's division
                if constexpr (sizeof(T) == 4) { vsig = ci + hj.c - T(3) * rv * rsqrtf(r2); }
                else { vsig = ci + hj.c - fdiv(T(3) * rv, T(sqrt(r2))); }
            }
            if constexpr (kMode & kModeTape)
            {
                if (!(vijsignalI > vsig)) { vsigJ = int(j); }
            }
            vijsignalI = vijsignalI > vsig ? vijsignalI : vsig;
            T Wi       = KhiInv3 * kernelWr2(a.wh, k, r2, hiInv, hh);
            T fac      = hj.vol * (divvI - divvJ);
            if constexpr (sizeof(T) == 4)
            {
                // FP32: sum fac W r and apply -C_i once after the loop (the same vector, 9 FMAs less per pair)
                T sw = fac * Wi;
                gx.add(sw * r.rx);
                gy.add(sw * r.ry);
                gz.add(sw * r.rz);
            }
            else
            {
                T tA1 = -(gr.c11 * r.rx + gr.c12 * r.ry + gr.c13 * r.rz) * Wi;
                T tA2 = -(gr.c12 * r.rx + gr.c22 * r.ry + gr.c23 * r.rz) * Wi;
                T tA3 = -(gr.c13 * r.rx + gr.c23 * r.ry + gr.c33 * r.rz) * Wi;
                gx.add(fac * tA1);
                gy.add(fac * tA2);
                gz.add(fac * tA3);
            }
        }
        gx.flush();
        gy.flush();
        gz.flush();
    }
    T gdx = gx.get(), gdy = gy.get(), gdz = gz.get();
    if constexpr (sizeof(T) == 4)
    {
        T sx = gdx, sy = gdy, sz = gdz;
        gdx  = -(gr.c11 * sx + gr.c12 * sy + gr.c13 * sz);
        gdy  = -(gr.c12 * sx + gr.c22 * sy + gr.c23 * sz);
        gdz  = -(gr.c13 * sx + gr.c23 * sy + gr.c33 * sz);
    }
    T graddivv = sqrt(gdx * gdx + gdy * gdy + gdz * gdz);
    if constexpr (kMode & kModeTape)
    {
        a.tape.gx[t.i]    = gdx;
        a.tape.gy[t.i]    = gdy;
        a.tape.gz[t.i]    = gdz;
        a.tape.vsig[t.i]  = vijsignalI;
        a.tape.vsigJ[t.i] = vsigJ;
    }
    T alphaI   = T(a.alpha[t.i]);
    T alphaloc = T(0);
    if (divvI < T(0))
    {
        T aConst = hi * hi * graddivv;
        alphaloc = k.alphamax * aConst / (aConst + hi * fabs(divvI) + T(0.05) * ci);
    }
    if (alphaloc >= alphaI) { alphaI = alphaloc; }
    else
    {
        T decay    = hi / (k.decay * vijsignalI);
        T alphadot = alphaloc >= k.alphamin ? (alphaloc - alphaI) / decay : (k.alphamin - alphaI) / decay;
        double dtq = dt;
        if constexpr (kMode & kModeBatch) { dtq = a.batch.dt[a.batch.inst[t.i]]; }
        alphaI += alphadot * T(dtq);
    }
    a.alpha[t.i]      = double(alphaI);
    a.grec[t.i].alpha = alphaI; // the alpha slot of the record is not read by this kernel
}

// ---------------------------------------------------------------------------------------------------------------
// Momentum and energy (sph/include/sph/hydro_ve/momentum_energy_kern.hpp:65-222, avClean = false;
// artificial_viscosity sph/include/sph/kernels.hpp:71-85) with the Courant time step per particle
// (tsKCourant, kernels.hpp:10-17) reduced to the minimum.
// ---------------------------------------------------------------------------------------------------------------
// FP32 without AV cleaning: at most 80 registers (three 256-thread blocks per SM) keeps more warps resident for the
// gathers; measured 2.11 -> 2.05 ms at 128^3 against 96 registers (the AV-cleaning form would spill)
template<class T, int kMode>
__global__ void __launch_bounds__(kChainMaxThreads, (sizeof(T) == 4 && !(kMode & kModeAvClean)) ? 3 : 1)
    momentumEnergyKernel(ChainArrays<T> a, HydroConsts<T> k, DevBox box)
{
    Target t;
    bool valid   = chainTarget<kMode>(a, k.ngmax, t);
    double dtMin = INFINITY;
    if (valid)
    {
        Pos<T> pi      = posOf(a, t.i);
        double hiD     = a.h[t.i];
        HydroRec<T> hr = a.hrec[t.i];
        GradRec<T> gr  = a.grec[t.i];
        T hi          = T(hiD);
        T mi          = T(pi.m);
        T ci          = hr.c;
        T kxi         = a.kx[t.i];
        T alphaI      = gr.alpha;
        T xmassi      = hr.xm;
        // FP32: log2 xm_i for the Atwood ramp's xm_i^(2-s) xm_j^s = exp2((2-s) log2 xm_i + s log2 xm_j)
        T lxi         = sizeof(T) == 4 ? T(log2f(float(xmassi))) : T(0);
        T rhoi        = kxi * mi / xmassi;
        T invRhoi     = T(1) / rhoi;
        T prhoi       = hr.prho;
        T hiInv       = T(1) / hi;
        T hiInv3      = hiInv * hiInv * hiInv;
        T maxvsignalI = T(0);
        BlockSum<T> momX, momY, momZ, energyS, aViscE;
        [[maybe_unused]] T gradVi[6];
        [[maybe_unused]] T etaCrit = T(0);
        if constexpr (kMode & kModeAvClean)
        {
            loadDV(a.dvrec + t.i, gradVi);
            etaCrit = T(cbrt(32.0 * M_PI / 3.0 / double(t.count + 1)));
        }

        // the term of one neighbour j, added to the five sums
        auto pairTerm = [&](uint32_t j) {
            if constexpr (sizeof(T) == 4 && !(kMode & kModeAvClean))
            {
                // FP32: the i and j halves of the pair side by side in packed FP32 (sm_100 FFMA2/FMUL2): the IAD
                // gradients tA = -(C r) W, their products with v_ij and the momentum coefficients. The viscous
                // term joins the momentum sums as (m_j prho_i a_mom + aVisc/2) tA_i + (m_j prho_j b_mom + bVisc/2)
                // tA_j (1.54 -> 1.48 ms at 128^3; the errors against FP64 unchanged). The ensemble's batch form
                // takes the same body, so that its members stay bit-identical to single simulations (it spills a
                // little there: 4.97 ms per step for 64 members, against 4.84 with the scalar body)
                Pos<T> pj      = posOf(a, j);
                HydroRec<T> hj = loadHydro(a.hrec + j);
                GradRec<T> gj  = loadGrad(a.grec + j);
                Sep<T> r       = separation(pi, pj, 2.0 * hiD, box, k);
                float r2       = r.rx * r.rx + r.ry * r.ry + r.rz * r.rz;
                float rinv     = rsqrtf(r2);
                float dist     = r2 * rinv;
                float vxij     = hr.vx - hj.vx;
                float vyij     = hr.vy - hj.vy;
                float vzij     = hr.vz - hj.vz;

                float v1 = dist * hiInv, v2 = dist * hj.hInv;
                float hjInv3 = hj.hInv * hj.hInv * hj.hInv;
                float2 W = make_float2(-hiInv3 * kernelW(a.wh, k, v1), -hjInv3 * kernelW(a.wh, k, v2));

                // tA = -(C r) W of i and j side by side
                float2 RX  = make_float2(r.rx, r.rx), RY = make_float2(r.ry, r.ry), RZ = make_float2(r.rz, r.rz);
                float2 tA1 = __ffma2_rn(make_float2(gr.c13, gj.c13), RZ,
                                        __ffma2_rn(make_float2(gr.c12, gj.c12), RY,
                                                   __fmul2_rn(make_float2(gr.c11, gj.c11), RX)));
                float2 tA2 = __ffma2_rn(make_float2(gr.c23, gj.c23), RZ,
                                        __ffma2_rn(make_float2(gr.c22, gj.c22), RY,
                                                   __fmul2_rn(make_float2(gr.c12, gj.c12), RX)));
                float2 tA3 = __ffma2_rn(make_float2(gr.c33, gj.c33), RZ,
                                        __ffma2_rn(make_float2(gr.c23, gj.c23), RY,
                                                   __fmul2_rn(make_float2(gr.c13, gj.c13), RX)));
                tA1 = __fmul2_rn(tA1, W);
                tA2 = __fmul2_rn(tA2, W);
                tA3 = __fmul2_rn(tA3, W);

                float mj     = float(pj.m);
                float cj     = hj.c;
                float xmassj = hj.xm;
                float rhoj   = fdiv(mj, hj.vol);
                float rv     = r.rx * vxij + r.ry * vyij + r.rz * vzij;
                float wij    = rv * rinv;
                float visc   = 0.0f;
                if (wij < 0.0f)
                {
                    float vijSignal = (alphaI + gj.alpha) * 0.25f * (ci + cj) - 2.0f * wij;
                    visc            = -vijSignal * wij;
                }
                float vijsignal = 0.5f * (ci + cj) - 2.0f * wij;
                maxvsignalI     = vijsignal > maxvsignalI ? vijsignal : maxvsignalI;

                float aMom, bMom;
                float dRho = fabsf(rhoi - rhoj), sRho = rhoi + rhoj;
                if (dRho < k.Atmin * sRho)
                {
                    aMom = xmassi * xmassi;
                    bMom = xmassj * xmassj;
                }
                else if (dRho > k.Atmax * sRho)
                {
                    aMom = xmassi * xmassj;
                    bMom = aMom;
                }
                else
                {
                    float sigma = k.ramp * (fdiv(dRho, sRho) - k.Atmin);
                    float lxj   = log2f(xmassj);
                    aMom        = exp2f((2.0f - sigma) * lxi + sigma * lxj);
                    bMom        = exp2f((2.0f - sigma) * lxj + sigma * lxi);
                }
                float aVisc = mj * invRhoi * visc;
                float bVisc = hj.vol * visc;
                // (tA_i . v_ij, tA_j . v_ij)
                float2 dv = __ffma2_rn(tA3, make_float2(vzij, vzij),
                                       __ffma2_rn(tA2, make_float2(vyij, vyij),
                                                  __fmul2_rn(tA1, make_float2(vxij, vxij))));
                aViscE.add(0.5f * (aVisc * dv.x + bVisc * dv.y));
                energyS.add(mj * aMom * dv.x);
                float cI = mj * prhoi * aMom + 0.5f * aVisc;
                float cJ = mj * hj.prho * bMom + 0.5f * bVisc;
                momX.add(cI * tA1.x + cJ * tA1.y);
                momY.add(cI * tA2.x + cJ * tA2.y);
                momZ.add(cI * tA3.x + cJ * tA3.y);
            }
            else
            {
                Pos<T> pj      = posOf(a, j);
                HydroRec<T> hj = loadHydro(a.hrec + j);
                GradRec<T> gj  = loadGrad(a.grec + j);
                Sep<T> r       = separation(pi, pj, 2.0 * hiD, box, k);
                T r2           = r.rx * r.rx + r.ry * r.ry + r.rz * r.rz;
                // FP32: 1/r from one rsqrt (r and w_ij = r.v / r without a square root or a division), m_j / rho_j as
                // vol_j, and the Atwood thresholds compared without a division (1.68 -> 1.58 ms at 128^3; the errors
                // against FP64 unchanged)
                T rinv, dist;
                if constexpr (sizeof(T) == 4)
                {
                    rinv = rsqrtf(r2);
                    dist = r2 * rinv;
                }
                else { dist = sqrt(r2); }
                T vxij         = hr.vx - hj.vx;
                T vyij         = hr.vy - hj.vy;
                T vzij         = hr.vz - hj.vz;
                T v1           = dist * hiInv;
                T v2           = dist * hj.hInv;
                T hjInv3       = hj.hInv * hj.hInv * hj.hInv;
                T Wi           = hiInv3 * kernelW(a.wh, k, v1);
                T Wj           = hjInv3 * kernelW(a.wh, k, v2);

                T tA1i = -(gr.c11 * r.rx + gr.c12 * r.ry + gr.c13 * r.rz) * Wi;
                T tA2i = -(gr.c12 * r.rx + gr.c22 * r.ry + gr.c23 * r.rz) * Wi;
                T tA3i = -(gr.c13 * r.rx + gr.c23 * r.ry + gr.c33 * r.rz) * Wi;
                T tA1j = -(gj.c11 * r.rx + gj.c12 * r.ry + gj.c13 * r.rz) * Wj;
                T tA2j = -(gj.c12 * r.rx + gj.c22 * r.ry + gj.c23 * r.rz) * Wj;
                T tA3j = -(gj.c13 * r.rx + gj.c23 * r.ry + gj.c33 * r.rz) * Wj;

                T mj     = T(pj.m);
                T cj     = hj.c;
                T xmassj = hj.xm;
                T rhoj   = fdiv(mj, hj.vol);

                T rv   = r.rx * vxij + r.ry * vyij + r.rz * vzij;
                if constexpr (kMode & kModeAvClean)
                {
                    T gradVj[6];
                    loadDV(a.dvrec + j, gradVj);
                    rv += avRvCorrection(r.rx, r.ry, r.rz, v1 < v2 ? v1 : v2, etaCrit, gradVi, gradVj);
                }
                T wij;
                if constexpr (sizeof(T) == 4) { wij = rv * rinv; }
                else { wij = fdiv(rv, dist); }
                T visc = T(0);
                if (wij < T(0))
                {
                    T vijSignal = (alphaI + gj.alpha) * T(0.25) * (ci + cj) - T(2) * wij;
                    visc        = -vijSignal * wij;
                }
                T vijsignal = T(0.5) * (ci + cj) - T(2) * wij;
                maxvsignalI = vijsignal > maxvsignalI ? vijsignal : maxvsignalI;

                T aMom, bMom;
                T dRho = fabs(rhoi - rhoj), sRho = rhoi + rhoj;
                if (sizeof(T) == 4 ? dRho < k.Atmin * sRho : fdiv(dRho, sRho) < k.Atmin)
                {
                    aMom = xmassi * xmassi;
                    bMom = xmassj * xmassj;
                }
                else if (sizeof(T) == 4 ? dRho > k.Atmax * sRho : fdiv(dRho, sRho) > k.Atmax)
                {
                    aMom = xmassi * xmassj;
                    bMom = aMom;
                }
                else
                {
                    T sigma = k.ramp * (fdiv(dRho, sRho) - k.Atmin);
                    if constexpr (sizeof(T) == 4)
                    {
                        T lxj = log2f(xmassj);
                        aMom  = exp2f((T(2) - sigma) * lxi + sigma * lxj);
                        bMom  = exp2f((T(2) - sigma) * lxj + sigma * lxi);
                    }
                    else
                    {
                        aMom = pow(xmassi, T(2) - sigma) * pow(xmassj, sigma);
                        bMom = pow(xmassj, T(2) - sigma) * pow(xmassi, sigma);
                    }
                }

                T aVisc, bVisc;
                if constexpr (sizeof(T) == 4)
                {
                    aVisc = mj * invRhoi * visc;
                    bVisc = hj.vol * visc;
                }
                else
                {
                    aVisc = fdiv(mj, rhoi) * visc;
                    bVisc = fdiv(mj, rhoj) * visc;
                }
                T aViscX = T(0.5) * (aVisc * tA1i + bVisc * tA1j);
                T aViscY = T(0.5) * (aVisc * tA2i + bVisc * tA2j);
                T aViscZ = T(0.5) * (aVisc * tA3i + bVisc * tA3j);
                aViscE.add(aViscX * vxij + aViscY * vyij + aViscZ * vzij);
                energyS.add(mj * aMom * (vxij * tA1i + vyij * tA2i + vzij * tA3i));
                T momI = mj * prhoi * aMom;
                T momJ = mj * hj.prho * bMom;
                momX.add(momI * tA1i + momJ * tA1j + aViscX);
                momY.add(momI * tA2i + momJ * tA2j + aViscY);
                momZ.add(momI * tA3i + momJ * tA3j + aViscZ);
            }
        };
        for (unsigned q0 = 0; q0 < t.count; q0 += kNbChunk)
        {
            uint32_t js[kNbChunk];
            loadChunk(a.nidx, t, t.ngPad, q0, js);
            unsigned qn = min(kNbChunk, t.count - q0);
            if constexpr (sizeof(T) == 4)
            {
                // one pair per iteration: the unrolled 8-pair body overflowed the instruction cache (2.04 -> 1.71 ms
                // at 128^3); unrolled by 2 or 4 it ran slower too (1.59 against 1.48 ms)
#pragma unroll 1
                for (unsigned q = 0; q < qn; ++q)
                {
                    pairTerm(popChunk(js));
                }
            }
            else
            {
                // bound by the FP64 pipe, the unrolled body is faster here (5.31 ms against 6.02 rolled)
#pragma unroll
                for (unsigned q = 0; q < kNbChunk; ++q)
                {
                    if (q >= qn) { break; }
                    pairTerm(js[q]);
                }
            }
            momX.flush();
            momY.flush();
            momZ.flush();
            energyS.flush();
            aViscE.flush();
        }
        if constexpr (kMode & kModeTape)
        {
            a.tape.energy[t.i] = energyS.get();
            a.tape.avisc[t.i]  = aViscE.get();
        }
        T aViscEnergy = aViscE.get() > T(0) ? aViscE.get() : T(0);
        a.du[t.i] = double(k.K * (prhoi * energyS.get() + T(0.5) * aViscEnergy));
        a.ax[t.i] = -k.K * momX.get();
        a.ay[t.i] = -k.K * momY.get();
        a.az[t.i] = -k.K * momZ.get();

        double v = maxvsignalI > T(0) ? double(maxvsignalI) : double(ci);
        // FP32: h read again here rather than kept in two registers across the pair loop (1.478 -> 1.465 ms)
        double hEnd = sizeof(T) == 4 ? a.h[t.i] : hiD;
        dtMin       = hEnd > 0.0 ? k.Kcour * hEnd / v : INFINITY;
    }
    if constexpr (kMode & kModeList)
    {
        // the group's Courant step lowers its block time step (momentum_energy_gpu.cu:96-103); rounding to float is
        // monotonic, so min(float, double) stored as float equals the min of the float values
        unsigned w  = unsigned((blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5);
        double gmin = dtMin;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            gmin = fmin(gmin, __shfl_xor_sync(0xffffffffu, gmin, off));
        }
        if ((threadIdx.x & 31) == 0 && w < a.numListed) { a.groupDt[w] = fminf(a.groupDt[w], float(gmin)); }
    }
    reduceOrdered<false, (kMode & kModeBatch) != 0>(dtMin, a.n, a.reduce + 1, a.batch, 1);
}

template<class T>
unsigned chainBlocks(const ChainArrays<T>& a)
{
    if (a.groupList) { return ceilDiv(size_t(a.numListed) * 32, unsigned(a.threads)); }
    return ceilDiv(a.n, size_t(a.threads));
}

} // namespace

//! kernel variant: kModeTape when the adjoint's tape pointers are set, kModeBatch for an ensemble
template<class T>
int chainMode(const ChainArrays<T>& a)
{
    int mode = (a.tape.energy ? kModeTape : 0) | (a.batch.inst ? kModeBatch : 0);
    if (a.groupList) { return mode == 0 ? kModeList : -1; } // block time steps: no tape, no ensemble
    return mode == (kModeTape | kModeBatch) ? -1 : mode;
}

//! the mode of the two kernels that AV cleaning changes (IAD writes the gradients, MomentumEnergy reads them)
template<class T>
int chainModeAv(const ChainArrays<T>& a)
{
    int mode = chainMode(a);
    if (mode < 0 || !a.dvrec) { return mode; }
    return (mode & kModeTape) ? -1 : (mode | kModeAvClean); // the adjoint has no AV-cleaning variant
}

#define SPHB_DISPATCH_AV(KERNEL, ...)                                                                                   \
    switch (chainModeAv(a))                                                                                             \
    {                                                                                                                   \
    case 0: KERNEL<T, 0><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                                    \
    case kModeTape: KERNEL<T, kModeTape><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                    \
    case kModeBatch: KERNEL<T, kModeBatch><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                  \
    case kModeAvClean: KERNEL<T, kModeAvClean><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;              \
    case kModeList: KERNEL<T, kModeList><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                    \
    case kModeAvClean | kModeList:                                                                                      \
        KERNEL<T, kModeAvClean | kModeList><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__);                          \
        break;                                                                                                          \
    case kModeAvClean | kModeBatch:                                                                                     \
        KERNEL<T, kModeAvClean | kModeBatch><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__);                         \
        break;                                                                                                          \
    default: return kErrArg;                                                                                            \
    }

#define SPHB_DISPATCH(KERNEL, ...)                                                                                      \
    switch (chainMode(a))                                                                                               \
    {                                                                                                                   \
    case 0: KERNEL<T, 0><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                                    \
    case kModeTape: KERNEL<T, kModeTape><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                    \
    case kModeBatch: KERNEL<T, kModeBatch><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                  \
    case kModeList: KERNEL<T, kModeList><<<chainBlocks(a), a.threads, 0, s>>>(__VA_ARGS__); break;                    \
    default: return kErrArg;                                                                                            \
    }

template<class T>
int launchXMass(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s)
{
    if (a.n == 0 || (a.groupList && a.numListed == 0)) { return kOk; }
    SPHB_DISPATCH(xmassKernel, a, k, box)
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchVeDefGradhEos(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s)
{
    if (a.n == 0 || (a.groupList && a.numListed == 0)) { return kOk; }
    SPHB_DISPATCH(veDefGradhEosKernel, a, k, box)
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchPackVelocity(const ChainArrays<T>& a, cudaStream_t s)
{
    if (a.n == 0) { return kOk; }
    packVelocityKernel<T><<<ceilDiv(a.n, 256), 256, 0, s>>>(a.n, a.vx, a.vy, a.vz, a.hrec);
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchIadDivvCurlv(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s)
{
    if (a.n == 0 || (a.groupList && a.numListed == 0)) { return kOk; }
    if constexpr (sizeof(T) == 4)
    {
        switch (chainModeAv(a))
        {
        case 0: iadDivvCurlvFusedKernel<0><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box); break;
        case kModeTape: iadDivvCurlvFusedKernel<kModeTape><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box); break;
        case kModeBatch: iadDivvCurlvFusedKernel<kModeBatch><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box); break;
        case kModeList: iadDivvCurlvFusedKernel<kModeList><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box); break;
        case kModeAvClean:
            iadDivvCurlvFusedKernel<kModeAvClean><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box);
            break;
        case kModeAvClean | kModeBatch:
            iadDivvCurlvFusedKernel<kModeAvClean | kModeBatch><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box);
            break;
        case kModeAvClean | kModeList:
            iadDivvCurlvFusedKernel<kModeAvClean | kModeList><<<chainBlocks(a), a.threads, 0, s>>>(a, k, box);
            break;
        default: return kErrArg;
        }
    }
    else { SPHB_DISPATCH_AV(iadDivvCurlvKernel, a, k, box) }
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchAVswitches(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, double dt, cudaStream_t s)
{
    if (a.n == 0 || (a.groupList && a.numListed == 0)) { return kOk; }
    SPHB_DISPATCH(avSwitchesKernel, a, k, box, dt)
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

template<class T>
int launchMomentumEnergy(const ChainArrays<T>& a, const HydroConsts<T>& k, const DevBox& box, cudaStream_t s)
{
    if (a.n == 0 || (a.groupList && a.numListed == 0)) { return kOk; }
    SPHB_DISPATCH_AV(momentumEnergyKernel, a, k, box)
    countLaunch();
    SPHB_CUDA_TRY(cudaGetLastError());
    return kOk;
}

#define SPHB_INSTANTIATE(T)                                                                                            \
    template int launchXMass<T>(const ChainArrays<T>&, const HydroConsts<T>&, const DevBox&, cudaStream_t);          \
    template int launchVeDefGradhEos<T>(const ChainArrays<T>&, const HydroConsts<T>&, const DevBox&, cudaStream_t);  \
    template int launchPackVelocity<T>(const ChainArrays<T>&, cudaStream_t);                                           \
    template int launchIadDivvCurlv<T>(const ChainArrays<T>&, const HydroConsts<T>&, const DevBox&, cudaStream_t);   \
    template int launchAVswitches<T>(const ChainArrays<T>&, const HydroConsts<T>&, const DevBox&, double,            \
                                     cudaStream_t);                                                                  \
    template int launchMomentumEnergy<T>(const ChainArrays<T>&, const HydroConsts<T>&, const DevBox&, cudaStream_t);

SPHB_INSTANTIATE(double)
SPHB_INSTANTIATE(float)

} // namespace sphb
