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

} // namespace sphb
