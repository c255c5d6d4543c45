// Host-side SPH kernel tables: the sinc^n kernel, its derivative and its 3D normalisation constant.
#pragma once

#include <algorithm>
#include <cmath>
#include <vector>

namespace sphb
{

//! sinc(pi/2 v) and its derivative with respect to v (sph/include/sph/kernels.hpp:36-59)
inline double sincHalfPi(double v)
{
    if (v == 0.0) { return 1.0; }
    double a = 0.5 * M_PI * v;
    return std::sin(a) / a;
}

inline double sincHalfPiDerivative(double v)
{
    if (v == 0.0) { return 0.0; }
    double a = 0.5 * M_PI * v;
    double s = std::sin(a) / a;
    return s * (0.5 * M_PI) * (std::cos(a) / std::sin(a) - 1.0 / a);
}

/*! Composite Simpson rule on [a, b] with n intervals; odd- and even-index samples are each summed in ascending order
 *  of value, the way the reference integrates the kernel volume (sph/include/sph/sph_kernel_tables.hpp:28-59). */
template<class F>
double simpsonSorted(double a, double b, int n, F&& f)
{
    double h = (b - a) / double(n);
    std::vector<double> odd, even;
    for (int i = 1; i < n; ++i)
    {
        double v = f(a + double(i) * h);
        if (i % 2) { odd.push_back(v); }
        else { even.push_back(v); }
    }
    std::sort(odd.begin(), odd.end());
    std::sort(even.begin(), even.end());
    double so = 0, se = 0;
    for (double v : odd)
    {
        so += v;
    }
    for (double v : even)
    {
        se += v;
    }
    return h / 3.0 * (f(a) + f(b) + 4.0 * so + 2.0 * se);
}

/*! Fill wh, whd (size entries on [0, 2]) with sinc^n and its derivative and return the normalisation constant
 *  K = 1 / integral_0^2 4 pi x^2 sinc^n(x) dx (2000 Simpson intervals), as ParticlesData::createTables does
 *  (sph/include/sph/particles_data.hpp:377-387, sph_kernel_tables.hpp:62-102). */
inline double sincKernelTables(double n, double* wh, double* whd, int size)
{
    auto kernel = [n](double x) { return std::pow(sincHalfPi(x), n); };
    auto deriv  = [n](double x) { return n * std::pow(sincHalfPi(x), n - 1.0) * sincHalfPiDerivative(x); };
    double K    = 1.0 / simpsonSorted(0.0, 2.0, 2000, [&](double x) { return 4.0 * M_PI * x * x * kernel(x); });
    double dx   = 2.0 / double(size - 1);
    for (int i = 0; i < size; ++i)
    {
        double x = 0.0 + double(i) * dx;
        wh[i]    = kernel(x);
        whd[i]   = deriv(x);
    }
    return K;
}

/*! Polynomial form of the kernel for FP32 evaluation without table lookups: with u = v^2 and t = u/2 - 1 on
 *  v in [0, 2], W(v) ~ sum_k cw[k] t^k and dW/dv ~ v sum_k cdw[k] t^k (W is even and dW/dv odd in v). Coefficients
 *  come from Chebyshev interpolation of degree `degree` in t, converted to powers of t. Returns the largest absolute
 *  error of the two fits (evaluated in double) on a fine grid, so the caller can reject a poor fit. */
inline double sincPolyCoeffs(double n, int degree, double* cw, double* cdw)
{
    const int N = degree + 1;
    auto W      = [n](double v) { return std::pow(sincHalfPi(v), n); };
    auto dWv    = [n](double v) {
        if (v == 0.0)
        {
            // limit of n sinc^(n-1) sinc' / v at 0: n * d^2 sinc / dv^2 (0) = -n (pi/2)^2 / 3
            return -n * (0.5 * M_PI) * (0.5 * M_PI) / 3.0;
        }
        return n * std::pow(sincHalfPi(v), n - 1.0) * sincHalfPiDerivative(v) / v;
    };
    std::vector<double> fw(N), fd(N), tn(N);
    for (int j = 0; j < N; ++j)
    {
        tn[j]    = std::cos(M_PI * (j + 0.5) / N);
        double v = std::sqrt(2.0 * (tn[j] + 1.0));
        fw[j]    = W(v);
        fd[j]    = dWv(v);
    }
    // Chebyshev coefficients a_k = 2/N sum_j f(t_j) T_k(t_j), a_0 halved
    std::vector<double> aw(N, 0.0), ad(N, 0.0);
    for (int k = 0; k < N; ++k)
    {
        for (int j = 0; j < N; ++j)
        {
            double Tk = std::cos(k * std::acos(tn[j]));
            aw[k] += fw[j] * Tk;
            ad[k] += fd[j] * Tk;
        }
        aw[k] *= 2.0 / N;
        ad[k] *= 2.0 / N;
    }
    aw[0] *= 0.5;
    ad[0] *= 0.5;
    // powers of t: T_0 = 1, T_1 = t, T_{k+1} = 2 t T_k - T_{k-1}
    std::vector<std::vector<double>> T(N, std::vector<double>(N, 0.0));
    T[0][0] = 1.0;
    if (N > 1) { T[1][1] = 1.0; }
    for (int k = 1; k + 1 < N; ++k)
    {
        for (int p = 0; p < N; ++p)
        {
            double v = -T[k - 1][p];
            if (p > 0) { v += 2.0 * T[k][p - 1]; }
            T[k + 1][p] = v;
        }
    }
    for (int p = 0; p < N; ++p)
    {
        cw[p]  = 0.0;
        cdw[p] = 0.0;
        for (int k = 0; k < N; ++k)
        {
            cw[p] += aw[k] * T[k][p];
            cdw[p] += ad[k] * T[k][p];
        }
    }
    double err = 0.0;
    for (int s = 0; s <= 20000; ++s)
    {
        double v  = 2.0 * s / 20000.0;
        double t  = 0.5 * v * v - 1.0;
        double pw = 0.0, pd = 0.0;
        for (int p = N - 1; p >= 0; --p)
        {
            pw = pw * t + cw[p];
            pd = pd * t + cdw[p];
        }
        double dW = v == 0.0 ? 0.0 : dWv(v) * v;
        err       = std::max(err, std::max(std::abs(pw - W(v)), std::abs(pd * v - dW)));
    }
    return err;
}

} // namespace sphb
