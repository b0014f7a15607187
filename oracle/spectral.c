/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 * Grid and spectral operators, restating src/core/grid.f90:34-123 and
 * src/core/spectral.f90:40-188 operation by operation (each operator does
 * its own forward/backward transform round trip, as the reference does).
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double TWOPI = 2.0 * 3.14159265358979323846264338327950288;

/* grid.f90:116-123 */
static int wrap(int m, int n) { return m <= n / 2 ? m : m - n; }

/* grid.f90:34-113 */
static int grid_init(orc_grid *g, int nx, int ny, int nz, double lx, double ly, double lz,
                     int dealias)
{
    if (nx < 2) return 1;
    if (nx % 2 != 0) return 1;
    if (ny > 1 && ny % 2 != 0) return 1;
    if (nz > 1 && nz % 2 != 0) return 1;
    g->nx = nx; g->ny = ny; g->nz = nz;
    g->nkx = nx / 2 + 1;
    g->ndim = 1;
    if (ny > 1) g->ndim = 2;
    if (nz > 1) g->ndim = 3;
    g->lx = lx; g->ly = ly; g->lz = lz;
    g->dx = lx / nx; g->dy = ly / ny; g->dz = lz / nz;
    g->volume = lx;
    if (ny > 1) g->volume *= ly;
    if (nz > 1) g->volume *= lz;
    g->x = (double *)malloc(sizeof(double) * nx);
    g->y = (double *)malloc(sizeof(double) * ny);
    g->z = (double *)malloc(sizeof(double) * nz);
    for (int i = 0; i < nx; ++i) g->x[i] = i * g->dx;
    for (int j = 0; j < ny; ++j) g->y[j] = j * g->dy;
    for (int k = 0; k < nz; ++k) g->z[k] = k * g->dz;
    g->kx = (double *)malloc(sizeof(double) * g->nkx);
    g->ky = (double *)calloc(ny, sizeof(double));
    g->kz = (double *)calloc(nz, sizeof(double));
    for (int i = 0; i < g->nkx; ++i) g->kx[i] = TWOPI * i / lx;
    if (ny > 1)
        for (int j = 0; j < ny; ++j) g->ky[j] = TWOPI * wrap(j, ny) / ly;
    if (nz > 1)
        for (int k = 0; k < nz; ++k) g->kz[k] = TWOPI * wrap(k, nz) / lz;
    const long nh = (long)g->nkx * ny * nz;
    g->k2 = (double *)malloc(sizeof(double) * nh);
    g->kabs = (double *)malloc(sizeof(double) * nh);
    g->mask = (double *)malloc(sizeof(double) * nh);
    const double kxc = TWOPI * (nx / 2) / lx * (2.0 / 3.0);
    const double kyc = ny > 1 ? TWOPI * (ny / 2) / ly * (2.0 / 3.0) : DBL_MAX;
    const double kzc = nz > 1 ? TWOPI * (nz / 2) / lz * (2.0 / 3.0) : DBL_MAX;
    g->kmax_dealiased = 0.0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < g->nkx; ++i) {
                long q = i + (long)g->nkx * (j + (long)ny * k);
                g->k2[q] = g->kx[i] * g->kx[i] + g->ky[j] * g->ky[j] + g->kz[k] * g->kz[k];
                g->kabs[q] = sqrt(g->k2[q]);
                g->mask[q] = 1.0;
                if (dealias) {
                    if (fabs(g->kx[i]) >= kxc || fabs(g->ky[j]) >= kyc || fabs(g->kz[k]) >= kzc)
                        g->mask[q] = 0.0;
                } else {
                    if (i == g->nkx - 1) g->mask[q] = 0.0;
                    if (ny > 1 && j == ny / 2) g->mask[q] = 0.0;
                    if (nz > 1 && k == nz / 2) g->mask[q] = 0.0;
                }
                if (g->mask[q] > 0.0 && g->kabs[q] > g->kmax_dealiased) g->kmax_dealiased = g->kabs[q];
            }
    return 0;
}

static void grid_free(orc_grid *g)
{
    free(g->x); free(g->y); free(g->z);
    free(g->kx); free(g->ky); free(g->kz);
    free(g->k2); free(g->kabs); free(g->mask);
    memset(g, 0, sizeof(*g));
}

/* spectral.f90:40-50 */
int orc_spec_init(orc_spec *s, int nx, int ny, int nz, double lx, double ly, double lz,
                  int dealias)
{
    memset(s, 0, sizeof(*s));
    if (grid_init(&s->g, nx, ny, nz, lx, ly, lz, dealias)) return 1;
    s->fft = orc_fft3_create(nx, ny, nz);
    const long nh = (long)s->g.nkx * ny * nz;
    s->w1 = (orc_cplx *)malloc(sizeof(orc_cplx) * nh);
    s->w2 = (orc_cplx *)malloc(sizeof(orc_cplx) * nh);
    return 0;
}

void orc_spec_free(orc_spec *s)
{
    grid_free(&s->g);
    orc_fft3_destroy(s->fft);
    free(s->w1);
    free(s->w2);
    memset(s, 0, sizeof(*s));
}

static long nhalf(const orc_spec *s) { return (long)s->g.nkx * s->g.ny * s->g.nz; }
static long ncell(const orc_spec *s) { return (long)s->g.nx * s->g.ny * s->g.nz; }

void orc_spec_fwd(orc_spec *s, const double *u, orc_cplx *uhat) { orc_fft3_fwd(s->fft, u, uhat); }
void orc_spec_bwd(orc_spec *s, const orc_cplx *uhat, double *u) { orc_fft3_bwd(s->fft, uhat, u); }

/* spectral.f90:67-90 */
void orc_spec_grad_hat(orc_spec *s, const orc_cplx *uhat, int idir, double *du)
{
    const orc_grid *g = &s->g;
#pragma omp parallel for schedule(static) collapse(2)
    for (int k = 0; k < g->nz; ++k)
        for (int j = 0; j < g->ny; ++j)
            for (int i = 0; i < g->nkx; ++i) {
                long q = i + (long)g->nkx * (j + (long)g->ny * k);
                double kd = idir == 1 ? g->kx[i] : (idir == 2 ? g->ky[j] : g->kz[k]);
                s->w1[q] = I * kd * uhat[q] * g->mask[q];
            }
    orc_fft3_bwd(s->fft, s->w1, du);
}

/* spectral.f90:93-106 */
void orc_spec_grad(orc_spec *s, const double *u, double *du)
{
    const long nc = ncell(s);
    orc_fft3_fwd(s->fft, u, s->w2);
    for (int d = 1; d <= 3; ++d) {
        if (d > s->g.ndim)
            memset(du + (d - 1) * nc, 0, sizeof(double) * nc);
        else
            orc_spec_grad_hat(s, s->w2, d, du + (d - 1) * nc);
    }
}

/* spectral.f90:109-116 */
void orc_spec_lap(orc_spec *s, const double *u, double *lu)
{
    orc_fft3_fwd(s->fft, u, s->w2);
    const long nh = nhalf(s);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) s->w2[q] = -s->g.k2[q] * s->w2[q] * s->g.mask[q];
    orc_fft3_bwd(s->fft, s->w2, lu);
}

/* spectral.f90:119-144 */
void orc_spec_div(orc_spec *s, const double *v, double *dv)
{
    const orc_grid *g = &s->g;
    const long nh = nhalf(s), nc = ncell(s);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) s->w1[q] = 0;
    for (int d = 1; d <= g->ndim; ++d) {
        orc_fft3_fwd(s->fft, v + (d - 1) * nc, s->w2);
#pragma omp parallel for schedule(static) collapse(2)
        for (int k = 0; k < g->nz; ++k)
            for (int j = 0; j < g->ny; ++j)
                for (int i = 0; i < g->nkx; ++i) {
                    long q = i + (long)g->nkx * (j + (long)g->ny * k);
                    double kd = d == 1 ? g->kx[i] : (d == 2 ? g->ky[j] : g->kz[k]);
                    s->w1[q] = s->w1[q] + I * kd * s->w2[q];
                }
    }
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) s->w1[q] *= g->mask[q];
    orc_fft3_bwd(s->fft, s->w1, dv);
}

/* spectral.f90:147-154 */
void orc_spec_convolve(orc_spec *s, const double *kern, const orc_cplx *uhat, double *cu)
{
    const long nh = nhalf(s);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) s->w1[q] = kern[q] * uhat[q] * s->g.mask[q];
    orc_fft3_bwd(s->fft, s->w1, cu);
}

/* spectral.f90:157-163 */
void orc_spec_dealias(orc_spec *s, double *u)
{
    orc_fft3_fwd(s->fft, u, s->w2);
    const long nh = nhalf(s);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) s->w2[q] *= s->g.mask[q];
    orc_fft3_bwd(s->fft, s->w2, u);
}

/* spectral.f90:172-176 */
double orc_spec_mean(const orc_spec *s, const double *u)
{
    const long nc = ncell(s);
    double acc = 0.0;
    for (long q = 0; q < nc; ++q) acc += u[q];
    return acc / (double)nc;
}

/* spectral.f90:179-188 */
orc_cplx orc_spec_mode(orc_spec *s, const double *u, int mx, int my, int mz)
{
    orc_fft3_fwd(s->fft, u, s->w2);
    int jy = ((my % s->g.ny) + s->g.ny) % s->g.ny;
    int kz = ((mz % s->g.nz) + s->g.nz) % s->g.nz;
    return s->w2[mx + (long)s->g.nkx * (jy + (long)s->g.ny * kz)];
}
