/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Replacement for the reference's FFTW3
 * dependency (unpinned; cmake/FindFFTW.cmake:1-23; call sites
 * src/core/fft.f90:46-47,57,67 and src/structure/oz_hnc.f90:75,85,94).
 *
 * 1-D complex DFT X_k = sum_j x_j exp(sign 2 pi i jk/n) by the Stockham
 * autosort algorithm (mixed radix: 4, 2, 3, 5 and a direct butterfly for any
 * other prime factor), written from the textbook formulation.  The 3-D
 * real transforms restate FFTW's r2c/c2r semantics on the (nx/2+1, ny, nz)
 * half spectrum: c2r uses the Hermitian extension along x and keeps the real
 * part (FFTW ignores the imaginary parts of the kx = 0 and kx = nx/2 planes).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double ORC_PI = 3.14159265358979323846264338327950288;

struct orc_fft1 {
    int n, nf;
    int f[64];
    orc_cplx *w;      /* w[t] = exp(-2 pi i t/n), t < n */
    /* Bluestein (chirp-z) for lengths with a prime factor above 64 */
    struct orc_fft1 *sub;   /* power-of-two plan of length mb >= 2n-1 */
    int mb;
    orc_cplx *chirp;        /* exp(-i pi j^2/n), j < n */
    orc_cplx *bf[2];        /* FFT of the conjugate-chirp filter, [0] forward, [1] backward */
};

static orc_fft1 *create_plain(int n);

static int largest_prime(int n)
{
    int m = n, lp = 1;
    for (int q = 2; (long)q * q <= m; ++q)
        while (m % q == 0) { lp = q; m /= q; }
    return m > lp ? m : lp;
}

static void exec_buf(orc_fft1 *p, orc_cplx *data, orc_cplx *work, int sign);

orc_fft1 *orc_fft1_create(int n)
{
    if (n <= 64 || largest_prime(n) <= 64) return create_plain(n);
    /* Bluestein: w^{jk} = c_j c_k conj(c_{k-j}), c_j = exp(sign i pi j^2/n) */
    orc_fft1 *p = (orc_fft1 *)calloc(1, sizeof(*p));
    p->n = n;
    int mb = 1;
    while (mb < 2 * n - 1) mb *= 2;
    p->mb = mb;
    p->sub = create_plain(mb);
    p->chirp = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
    for (int j = 0; j < n; ++j) {
        long jj = ((long)j * j) % (2L * n);
        double a = -ORC_PI * (double)jj / (double)n;
        p->chirp[j] = cos(a) + I * sin(a);
    }
    orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * mb);
    for (int s = 0; s < 2; ++s) {
        /* s = 0: forward (sign -1) uses c = chirp; filter b_m = conj(c_m) */
        orc_cplx *b = (orc_cplx *)calloc(mb, sizeof(orc_cplx));
        for (int m = 0; m < n; ++m) {
            orc_cplx c = s == 0 ? p->chirp[m] : conj(p->chirp[m]);
            b[m] = conj(c);
            if (m > 0) b[mb - m] = conj(c);
        }
        exec_buf(p->sub, b, work, -1);
        p->bf[s] = b;
    }
    free(work);
    return p;
}

static orc_fft1 *create_plain(int n)
{
    orc_fft1 *p = (orc_fft1 *)calloc(1, sizeof(*p));
    p->n = n;
    int m = n;
    while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
    while (m % 5 == 0) { p->f[p->nf++] = 5; m /= 5; }
    for (int q = 7; m > 1; q += 2) {
        while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
        if ((long)q * q > m && m > 1) { p->f[p->nf++] = m; m = 1; }
    }
    p->w = (orc_cplx *)malloc(sizeof(orc_cplx) * (n > 0 ? n : 1));
    for (int t = 0; t < n; ++t) {
        double a = -2.0 * ORC_PI * (double)t / (double)n;
        p->w[t] = cos(a) + I * sin(a);
    }
    return p;
}

void orc_fft1_destroy(orc_fft1 *p)
{
    if (!p) return;
    free(p->w);
    if (p->sub) {
        orc_fft1_destroy(p->sub);
        free(p->chirp);
        free(p->bf[0]);
        free(p->bf[1]);
    }
    free(p);
}

/* one Stockham pass of radix R: Ns = span already combined */
static void pass(const orc_fft1 *p, int R, int Ns, const orc_cplx *in, orc_cplx *out, int sign)
{
    const int n = p->n;
    const int m = n / R;
    const int tw_step = n / (Ns * R);
    orc_cplx v[64], ob[64];
    orc_cplx *vv = v, *o = ob;
    orc_cplx *heap = NULL;
    if (R > 64) {
        heap = (orc_cplx *)malloc(sizeof(orc_cplx) * 2 * R);
        vv = heap;
        o = heap + R;
    }
    for (int j = 0; j < m; ++j) {
        const int k = j % Ns;
        for (int r = 0; r < R; ++r) {
            orc_cplx x = in[j + r * m];
            long t = ((long)k * r * tw_step) % n;
            orc_cplx w = p->w[t];
            if (sign > 0) w = conj(w);
            vv[r] = x * w;
        }
        const int idxD = (j / Ns) * Ns * R + k;
        if (R == 2) {
            out[idxD] = vv[0] + vv[1];
            out[idxD + Ns] = vv[0] - vv[1];
        } else if (R == 4) {
            orc_cplx a0 = vv[0] + vv[2], a1 = vv[0] - vv[2];
            orc_cplx b0 = vv[1] + vv[3], b1 = vv[1] - vv[3];
            /* forward: -i * b1 ; backward: +i * b1 */
            orc_cplx jb1 = (sign < 0) ? (cimag(b1) - I * creal(b1)) : (-cimag(b1) + I * creal(b1));
            out[idxD] = a0 + b0;
            out[idxD + Ns] = a1 + jb1;
            out[idxD + 2 * Ns] = a0 - b0;
            out[idxD + 3 * Ns] = a1 - jb1;
        } else {
            /* direct R-point DFT, R prime (3, 5 or larger) */
            const int step = n / R;
            for (int q = 0; q < R; ++q) {
                orc_cplx s = 0;
                for (int r = 0; r < R; ++r) {
                    long t = ((long)r * q % R) * step;
                    orc_cplx w = p->w[t];
                    if (sign > 0) w = conj(w);
                    s += vv[r] * w;
                }
                o[q] = s;
            }
            for (int q = 0; q < R; ++q) out[idxD + q * Ns] = o[q];
        }
    }
    free(heap);
}

static void exec_bluestein(orc_fft1 *p, orc_cplx *data, int sign)
{
    const int n = p->n, mb = p->mb;
    orc_cplx *a = (orc_cplx *)calloc(mb, sizeof(orc_cplx));
    orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * mb);
    const int s = sign < 0 ? 0 : 1;
    for (int j = 0; j < n; ++j) a[j] = data[j] * (s == 0 ? p->chirp[j] : conj(p->chirp[j]));
    exec_buf(p->sub, a, work, -1);
    for (int m = 0; m < mb; ++m) a[m] *= p->bf[s][m];
    exec_buf(p->sub, a, work, +1);
    for (int k = 0; k < n; ++k)
        data[k] = a[k] / (double)mb * (s == 0 ? p->chirp[k] : conj(p->chirp[k]));
    free(a);
    free(work);
}

static void exec_buf(orc_fft1 *p, orc_cplx *data, orc_cplx *work, int sign)
{
    if (p->sub) { exec_bluestein(p, data, sign); return; }
    orc_cplx *a = data, *b = work;
    int Ns = 1;
    for (int s = 0; s < p->nf; ++s) {
        pass(p, p->f[s], Ns, a, b, sign);
        Ns *= p->f[s];
        orc_cplx *t = a; a = b; b = t;
    }
    if (a != data) memcpy(data, a, sizeof(orc_cplx) * p->n);
}

void orc_fft1_exec(orc_fft1 *p, orc_cplx *data, int sign)
{
    if (p->n <= 1) return;
    orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * p->n);
    exec_buf(p, data, work, sign);
    free(work);
}

void orc_fft1_c(int n, orc_cplx *data, int sign)
{
    orc_fft1 *p = orc_fft1_create(n);
    orc_fft1_exec(p, data, sign);
    orc_fft1_destroy(p);
}

/* ---------------------------------------------------------------- 3-D */
struct orc_fft3 {
    int nx, ny, nz, nkx;
    orc_fft1 *px, *py, *pz;
    double norm;
    long count;
};

orc_fft3 *orc_fft3_create(int nx, int ny, int nz)
{
    orc_fft3 *f = (orc_fft3 *)calloc(1, sizeof(*f));
    f->nx = nx; f->ny = ny; f->nz = nz; f->nkx = nx / 2 + 1;
    f->px = orc_fft1_create(nx);
    f->py = orc_fft1_create(ny);
    f->pz = orc_fft1_create(nz);
    f->norm = 1.0 / ((double)nx * (double)ny * (double)nz);
    return f;
}

void orc_fft3_destroy(orc_fft3 *f)
{
    if (!f) return;
    orc_fft1_destroy(f->px);
    orc_fft1_destroy(f->py);
    orc_fft1_destroy(f->pz);
    free(f);
}

long orc_fft3_count(const orc_fft3 *f) { return f->count; }

/* transform along y (axis 1) or z (axis 2) of a (nkx,ny,nz) complex array */
static void lines_yz(orc_fft3 *f, orc_cplx *a, int axis, int sign)
{
    const int nkx = f->nkx, ny = f->ny, nz = f->nz;
    if ((axis == 1 && ny == 1) || (axis == 2 && nz == 1)) return;
    const int len = axis == 1 ? ny : nz;
    const int nlines = axis == 1 ? nkx * nz : nkx * ny;
    orc_fft1 *p = axis == 1 ? f->py : f->pz;
#pragma omp parallel
    {
        orc_cplx *buf = (orc_cplx *)malloc(sizeof(orc_cplx) * len);
        orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * len);
#pragma omp for schedule(static)
        for (int l = 0; l < nlines; ++l) {
            long base, stride;
            if (axis == 1) {
                int i = l % nkx, k = l / nkx;
                base = i + (long)nkx * ny * k;
                stride = nkx;
            } else {
                int i = l % nkx, j = l / nkx;
                base = i + (long)nkx * j;
                stride = (long)nkx * ny;
            }
            for (int e = 0; e < len; ++e) buf[e] = a[base + e * stride];
            exec_buf(p, buf, work, sign);
            for (int e = 0; e < len; ++e) a[base + e * stride] = buf[e];
        }
        free(buf);
        free(work);
    }
}

void orc_fft3_fwd(orc_fft3 *f, const double *u, orc_cplx *uhat)
{
    const int nx = f->nx, ny = f->ny, nz = f->nz, nkx = f->nkx;
    const int nrows = ny * nz;
#pragma omp parallel
    {
        orc_cplx *buf = (orc_cplx *)malloc(sizeof(orc_cplx) * nx);
        orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * nx);
#pragma omp for schedule(static)
        for (int r = 0; r < nrows; ++r) {
            const double *row = u + (long)nx * r;
            for (int i = 0; i < nx; ++i) buf[i] = row[i];
            exec_buf(f->px, buf, work, -1);
            for (int i = 0; i < nkx; ++i) uhat[(long)nkx * r + i] = buf[i];
        }
        free(buf);
        free(work);
    }
    lines_yz(f, uhat, 1, -1);
    lines_yz(f, uhat, 2, -1);
    const long nh = (long)nkx * ny * nz;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) uhat[q] *= f->norm;
    f->count++;
}

void orc_fft3_bwd(orc_fft3 *f, const orc_cplx *uhat, double *u)
{
    const int nx = f->nx, ny = f->ny, nz = f->nz, nkx = f->nkx;
    const long nh = (long)nkx * ny * nz;
    orc_cplx *a = (orc_cplx *)malloc(sizeof(orc_cplx) * nh);
    memcpy(a, uhat, sizeof(orc_cplx) * nh);
    lines_yz(f, a, 2, +1);
    lines_yz(f, a, 1, +1);
    const int nrows = ny * nz;
#pragma omp parallel
    {
        orc_cplx *buf = (orc_cplx *)malloc(sizeof(orc_cplx) * nx);
        orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * nx);
#pragma omp for schedule(static)
        for (int r = 0; r < nrows; ++r) {
            const orc_cplx *h = a + (long)nkx * r;
            /* Hermitian extension along x; the imaginary parts of the
             * self-conjugate bins contribute only to the discarded
             * imaginary part of the result. */
            for (int i = 0; i < nkx; ++i) buf[i] = h[i];
            for (int i = nkx; i < nx; ++i) buf[i] = conj(h[nx - i]);
            exec_buf(f->px, buf, work, +1);
            double *row = u + (long)nx * r;
            for (int i = 0; i < nx; ++i) row[i] = creal(buf[i]);
        }
        free(buf);
        free(work);
    }
    free(a);
    f->count++;
}

/* ---------------------------------------------------------------- DST-I */
struct orc_dst1 {
    int n;
    orc_fft1 *p;   /* length 2(n+1) */
};

orc_dst1 *orc_dst1_create(int n)
{
    orc_dst1 *d = (orc_dst1 *)calloc(1, sizeof(*d));
    d->n = n;
    d->p = orc_fft1_create(2 * (n + 1));
    return d;
}

void orc_dst1_destroy(orc_dst1 *d)
{
    if (!d) return;
    orc_fft1_destroy(d->p);
    free(d);
}

/* odd extension of length M = 2(n+1): DFT_k = -2i sum_j x_j sin(pi (j+1) k/(n+1)) */
void orc_dst1_exec(orc_dst1 *d, const double *x, double *y)
{
    const int n = d->n, M = 2 * (n + 1);
    orc_cplx *b = (orc_cplx *)calloc(M, sizeof(orc_cplx));
    for (int j = 0; j < n; ++j) {
        b[j + 1] = x[j];
        b[M - j - 1] = -x[j];
    }
    orc_fft1_exec(d->p, b, -1);
    for (int k = 0; k < n; ++k) y[k] = -cimag(b[k + 1]);
    free(b);
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
