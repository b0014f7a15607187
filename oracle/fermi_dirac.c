/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 * Fermi-Dirac integrals and their inverse: src/special/fermi_dirac.f90:30-267
 * and src/special/quadrature.f90:17-38, restated statement by statement.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>

static const double PI = 3.14159265358979323846264338327950288;
static const double SQRTPI = 1.77245385090551602729816748334114518;

#define AMIN (-30.0)
#define AMAX 300.0
#define HH 0.05
#define NGL 20

static int ntab = 0;
static double *tab = NULL;   /* tab[6*i + c] for node i (0-based), column c (0-based) */

/* quadrature.f90:17-38 */
void orc_gauss_legendre(int n, double *x, double *w)
{
    for (int i = 1; i <= (n + 1) / 2; ++i) {
        double z = cos(PI * (i - 0.25) / (n + 0.5));
        double z1, p1, p2, p3, pp = 0.0;
        for (int it = 1; it <= 100; ++it) {
            p1 = 1.0; p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                p3 = p2; p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) < 1.0e-15) break;
        }
        x[i - 1] = -z; x[n - i] = z;
        w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp); w[n - i] = w[i - 1];
    }
}

/* fermi_dirac.f90:78-90 */
static void fermi_derivs(double y, double *f, double *p1, double *p2, double *p3)
{
    double g;
    if (y > 0.0) { g = exp(-y); *f = g / (1.0 + g); }
    else { g = exp(y); *f = 1.0 / (1.0 + g); }
    *p1 = *f * (1.0 - *f);
    *p2 = *p1 * (1.0 - 2.0 * *f);
    *p3 = *p1 * (1.0 - 6.0 * *f + 6.0 * *f * *f);
}

/* fermi_dirac.f90:30-74 */
void orc_fd_init(void)
{
    if (tab) return;
    int n = (int)lround((AMAX - AMIN) / HH) + 1;
    double *t6 = (double *)malloc(sizeof(double) * 6 * n);
    double xg[NGL], wg[NGL];
    orc_gauss_legendre(NGL, xg, wg);
    for (int i = 1; i <= n; ++i) {
        double alpha = AMIN + (i - 1) * HH;
        double xmax = (alpha > 0.0 ? alpha : 0.0) + 45.0;
        double s[6] = {0, 0, 0, 0, 0, 0};
        double f, p1, p2, p3;
        for (int q = 0; q < NGL; ++q) {
            double t = 0.5 * (xg[q] + 1.0);
            double x = t * t;
            fermi_derivs(x - alpha, &f, &p1, &p2, &p3);
            double e = wg[q] * 0.5 * 2.0;
            s[0] += e * f;
            s[1] += e * t * t * f;
            s[2] += e * pow(t, 4) * f;
            s[3] += e * p1;
            s[4] += e * p2;
            s[5] += e * p3;
        }
        int npan = (int)ceil(xmax - 1.0);
        for (int ip = 1; ip <= npan; ++ip) {
            double a = 1.0 + (ip - 1);
            double b = a + 1.0 < xmax ? a + 1.0 : xmax;
            double xm = 0.5 * (a + b), xr = 0.5 * (b - a);
            for (int q = 0; q < NGL; ++q) {
                double x = xm + xr * xg[q];
                fermi_derivs(x - alpha, &f, &p1, &p2, &p3);
                double e = wg[q] * xr;
                double t = 1.0 / sqrt(x);
                s[0] += e * t * f;
                s[1] += e * sqrt(x) * f;
                s[2] += e * x * sqrt(x) * f;
                s[3] += e * t * p1;
                s[4] += e * t * p2;
                s[5] += e * t * p3;
            }
        }
        for (int c = 0; c < 6; ++c) t6[6 * (i - 1) + c] = s[c];
    }
    ntab = n;
    tab = t6;
}

const double *orc_fd_table(int *n)
{
    orc_fd_init();
    if (n) *n = ntab;
    return tab;
}

#define TAB(col, i) tab[6 * ((i) - 1) + ((col) - 1)]

/* fermi_dirac.f90:109-113 (1-based node) */
static int node(double alpha)
{
    int i = (int)((alpha - AMIN) / HH) + 1;   /* Fortran int() truncates toward zero */
    if (i < 1) i = 1;
    if (i > ntab - 1) i = ntab - 1;
    return i;
}

/* fermi_dirac.f90:94-107 */
static double hermite(int col, double alpha, double d0, double d1)
{
    int i = node(alpha);
    double t = (alpha - (AMIN + (i - 1) * HH)) / HH;
    double t2 = t * t, t3 = t2 * t;
    double h00 = 2 * t3 - 3 * t2 + 1, h10 = t3 - 2 * t2 + t, h01 = -2 * t3 + 3 * t2, h11 = t3 - t2;
    double y0 = TAB(col, i), y1 = TAB(col, i + 1);
    return h00 * y0 + h10 * HH * d0 + h01 * y1 + h11 * HH * d1;
}

/* fermi_dirac.f90:116-133 */
static double sommerfeld(double p, double alpha, int m)
{
    double c[3];
    c[0] = 1.0;
    c[1] = (PI * PI / 6.0) * p * (p + 1.0);
    c[2] = (7.0 * pow(PI, 4) / 360.0) * (p + 1.0) * p * (p - 1.0) * (p - 2.0);
    double v = 0.0;
    for (int j = 0; j <= 2; ++j) {
        double ex = p + 1.0 - 2 * j;
        double coef = c[j] / (p + 1.0);
        for (int l = 0; l <= m - 1; ++l) coef = coef * (ex - l);
        v = v + coef * pow(alpha, ex - m);
    }
    return v;
}

/* fermi_dirac.f90:136-147 */
static double classical(double p, double alpha, int m)
{
    double v = 0.0, sgn = 1.0;
    for (int j = 1; j <= 12; ++j) {
        v = v + sgn * exp(j * alpha) * pow((double)j, m - p - 1.0);
        sgn = -sgn;
    }
    return v * tgamma(p + 1.0);
}

/* fermi_dirac.f90:150-162 */
double orc_fd_im12(double a)
{
    orc_fd_init();
    if (a > AMAX) return sommerfeld(-0.5, a, 0);
    if (a < AMIN) return classical(-0.5, a, 0);
    int i = node(a);
    return hermite(1, a, TAB(4, i), TAB(4, i + 1));
}

/* fermi_dirac.f90:165-177 */
double orc_fd_ip12(double a)
{
    orc_fd_init();
    if (a > AMAX) return sommerfeld(0.5, a, 0);
    if (a < AMIN) return classical(0.5, a, 0);
    int i = node(a);
    return hermite(2, a, 0.5 * TAB(1, i), 0.5 * TAB(1, i + 1));
}

/* fermi_dirac.f90:180-192 */
double orc_fd_ip32(double a)
{
    orc_fd_init();
    if (a > AMAX) return sommerfeld(1.5, a, 0);
    if (a < AMIN) return classical(1.5, a, 0);
    int i = node(a);
    return hermite(3, a, 1.5 * TAB(2, i), 1.5 * TAB(2, i + 1));
}

/* fermi_dirac.f90:195-207 */
double orc_fd_dim12(double a)
{
    orc_fd_init();
    if (a > AMAX) return sommerfeld(-0.5, a, 1);
    if (a < AMIN) return classical(-0.5, a, 1);
    int i = node(a);
    return hermite(4, a, TAB(5, i), TAB(5, i + 1));
}

/* fermi_dirac.f90:210-222 */
double orc_fd_d2im12(double a)
{
    orc_fd_init();
    if (a > AMAX) return sommerfeld(-0.5, a, 2);
    if (a < AMIN) return classical(-0.5, a, 2);
    int i = node(a);
    return hermite(5, a, TAB(6, i), TAB(6, i + 1));
}

/* fermi_dirac.f90:225-230 */
double orc_fd_xi(double a)
{
    double im = orc_fd_im12(a);
    return orc_fd_dim12(a) / (im * im);
}

/* fermi_dirac.f90:233-238 */
double orc_fd_dxi(double a)
{
    double im = orc_fd_im12(a), d1 = orc_fd_dim12(a), d2 = orc_fd_d2im12(a);
    return (d2 * im - 2.0 * d1 * d1) / (im * im * im);
}

/* fermi_dirac.f90:241-267.  status = 1 for y <= 0 (the reference's fatal). */
double orc_fd_alpha_from_ip12(double y, int *status)
{
    if (status) *status = 0;
    if (y <= 0.0) {
        if (status) *status = 1;
        return NAN;
    }
    double a1 = log(2.0 * y / SQRTPI);
    double a2 = pow(1.5 * y, 2.0 / 3.0) - 1.0;
    double alpha = a1 > a2 ? a1 : a2;
    if (y < 1.0) alpha = log(2.0 * y / SQRTPI);
    double lo = -DBL_MAX, hi = DBL_MAX;
    for (int it = 1; it <= 100; ++it) {
        double f = orc_fd_ip12(alpha) - y;
        if (f > 0.0) hi = hi < alpha ? hi : alpha;
        else lo = lo > alpha ? lo : alpha;
        double df = 0.5 * orc_fd_im12(alpha);
        double step = f / df;
        double am = fabs(alpha) > 1.0 ? fabs(alpha) : 1.0;
        if (fabs(step) < 1.0e-14 * am) break;
        alpha = alpha - step;
        if (alpha <= lo || alpha >= hi) {
            if (lo > -DBL_MAX && hi < DBL_MAX) alpha = 0.5 * (lo + hi);
        }
    }
    return alpha;
}
