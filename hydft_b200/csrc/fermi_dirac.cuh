// Fermi-Dirac integrals I_p(alpha), their alpha-derivatives and the inverse
// of I_{1/2}, in FP64 on the device.  Same table (alpha in [-30, 300],
// h = 0.05, 6601 nodes; columns I_{-1/2}, I_{1/2}, I_{3/2}, I'_{-1/2},
// I''_{-1/2}, I'''_{-1/2}), cubic Hermite interpolation with exact-derivative
// columns, Sommerfeld / classical expansions outside the table, and
// safeguarded Newton inverse as src/special/fermi_dirac.f90:20-267.
#pragma once

#include <cfloat>
#include "common.cuh"

namespace hydft {
namespace fd {

constexpr double AMIN = -30.0;
constexpr double AMAX = 300.0;
constexpr double H = 0.05;
constexpr int NTAB = 6601;   // nint((AMAX - AMIN)/H) + 1
constexpr int NGL = 20;

__host__ __device__ __forceinline__ int node(double a)
{
    int i = (int)((a - AMIN) / H) + 1;   // Fortran int(): truncation toward zero
    i = i < 1 ? 1 : i;
    i = i > NTAB - 1 ? NTAB - 1 : i;
    return i;
}

// tab[6*(i-1) + (col-1)]
__host__ __device__ __forceinline__ double T(const double *tab, int col, int i)
{
    return tab[6 * (i - 1) + (col - 1)];
}

__host__ __device__ __forceinline__ double hermite(const double *tab, int col, double a, double d0, double d1)
{
    const int i = node(a);
    const double t = (a - (AMIN + (i - 1) * H)) / H;
    const double t2 = t * t, t3 = t2 * t;
    const double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t, h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
    return h00 * T(tab, col, i) + h10 * H * d0 + h01 * T(tab, col, i + 1) + h11 * H * d1;
}

// Sommerfeld expansion, m-th derivative of I_p (fermi_dirac.f90:116-133)
__host__ __device__ inline double sommerfeld(double p, double a, int m)
{
    const double pi = 3.14159265358979323846264338327950288;
    double c[3];
    c[0] = 1.0;
    c[1] = (pi * pi / 6.0) * p * (p + 1.0);
    c[2] = (7.0 * pi * pi * pi * pi / 360.0) * (p + 1.0) * p * (p - 1.0) * (p - 2.0);
    double v = 0.0;
    for (int j = 0; j <= 2; ++j) {
        const double ex = p + 1.0 - 2 * j;
        double coef = c[j] / (p + 1.0);
        for (int l = 0; l <= m - 1; ++l) coef *= (ex - l);
        v += coef * pow(a, ex - m);
    }
    return v;
}

// Gamma(p+1) for the three orders used (p = -1/2, 1/2, 3/2)
__host__ __device__ __forceinline__ double gamma_p1(double p)
{
    // Gamma(1/2) = sqrt(pi), Gamma(3/2) = sqrt(pi)/2, Gamma(5/2) = 3 sqrt(pi)/4
    const double sp = 1.77245385090551602729816748334114518;
    return p < 0.0 ? sp : (p < 1.0 ? 0.5 * sp : 0.75 * sp);
}

// classical expansion, m-th derivative of I_p (fermi_dirac.f90:136-147)
__host__ __device__ inline double classical(double p, double a, int m)
{
    double v = 0.0, sgn = 1.0;
    for (int j = 1; j <= 12; ++j) {
        v += sgn * exp(j * a) * pow((double)j, m - p - 1.0);
        sgn = -sgn;
    }
    return v * gamma_p1(p);
}

__host__ __device__ inline double im12(const double *tab, double a)
{
    if (a > AMAX) return sommerfeld(-0.5, a, 0);
    if (a < AMIN) return classical(-0.5, a, 0);
    const int i = node(a);
    return hermite(tab, 1, a, T(tab, 4, i), T(tab, 4, i + 1));
}

__host__ __device__ inline double ip12(const double *tab, double a)
{
    if (a > AMAX) return sommerfeld(0.5, a, 0);
    if (a < AMIN) return classical(0.5, a, 0);
    const int i = node(a);
    return hermite(tab, 2, a, 0.5 * T(tab, 1, i), 0.5 * T(tab, 1, i + 1));
}

__host__ __device__ inline double ip32(const double *tab, double a)
{
    if (a > AMAX) return sommerfeld(1.5, a, 0);
    if (a < AMIN) return classical(1.5, a, 0);
    const int i = node(a);
    return hermite(tab, 3, a, 1.5 * T(tab, 2, i), 1.5 * T(tab, 2, i + 1));
}

__host__ __device__ inline double dim12(const double *tab, double a)
{
    if (a > AMAX) return sommerfeld(-0.5, a, 1);
    if (a < AMIN) return classical(-0.5, a, 1);
    const int i = node(a);
    return hermite(tab, 4, a, T(tab, 5, i), T(tab, 5, i + 1));
}

__host__ __device__ inline double d2im12(const double *tab, double a)
{
    if (a > AMAX) return sommerfeld(-0.5, a, 2);
    if (a < AMIN) return classical(-0.5, a, 2);
    const int i = node(a);
    return hermite(tab, 5, a, T(tab, 6, i), T(tab, 6, i + 1));
}

__host__ __device__ inline double xi(const double *tab, double a)
{
    const double im = im12(tab, a);
    return dim12(tab, a) / (im * im);
}

__host__ __device__ inline double dxi(const double *tab, double a)
{
    const double im = im12(tab, a), d1 = dim12(tab, a), d2 = d2im12(tab, a);
    return (d2 * im - 2.0 * d1 * d1) / (im * im * im);
}

// Safeguarded Newton inverse of I_{1/2} (fermi_dirac.f90:241-267).  Sets
// *ok = false when y <= 0 or the 100 iterations end without meeting the
// step tolerance.
__host__ __device__ inline double alpha_from_ip12(const double *tab, double y, bool *ok)
{
    const double sqrtpi = 1.77245385090551602729816748334114518;
    if (!(y > 0.0)) {
        *ok = false;
        return 0.0;
    }
    const double a1 = log(2.0 * y / sqrtpi);
    const double a2 = pow(1.5 * y, 2.0 / 3.0) - 1.0;
    double alpha = a1 > a2 ? a1 : a2;
    if (y < 1.0) alpha = a1;
    double lo = -DBL_MAX, hi = DBL_MAX;
    bool conv = false;
    for (int it = 1; it <= 100; ++it) {
        const double f = ip12(tab, alpha) - y;
        if (f > 0.0) hi = hi < alpha ? hi : alpha;
        else lo = lo > alpha ? lo : alpha;
        const double df = 0.5 * im12(tab, alpha);
        const double step = f / df;
        const double am = fabs(alpha) > 1.0 ? fabs(alpha) : 1.0;
        if (fabs(step) < 1.0e-14 * am) { conv = true; break; }
        alpha = alpha - step;
        if (alpha <= lo || alpha >= hi) {
            if (lo > -DBL_MAX && hi < DBL_MAX) alpha = 0.5 * (lo + hi);
        }
    }
    *ok = conv;
    return alpha;
}

}  // namespace fd
}  // namespace hydft
