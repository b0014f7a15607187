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
/*
 * The 3-D transforms run the same Stockham passes (same factor order, same
 * twiddle values, same butterflies) on OB lines at once: a batch holds
 * element e of lane b at [e*OB + b], real and imaginary parts in separate
 * arrays, so every butterfly is a short loop over the lanes.  Lengths with
 * a prime factor above 64 (Bluestein) go line by line through exec_buf.
 */
#define OB 8

typedef struct {
    int n, nf, batched;
    int f[64], ns[64];
    double *twr[64], *twi[64];   /* pass s: W_n^{k r tw_step} at [k*(R-1) + r-1] */
    double *wr, *wi;             /* W_n^t = exp(-2 pi i t/n) */
    orc_fft1 *line;
} bplan;

static bplan *bplan_create(int n)
{
    bplan *p = (bplan *)calloc(1, sizeof(*p));
    p->n = n;
    p->line = orc_fft1_create(n);
    if (n <= 1 || p->line->sub) return p;
    p->batched = 1;
    p->nf = p->line->nf;
    p->wr = (double *)malloc(sizeof(double) * n);
    p->wi = (double *)malloc(sizeof(double) * n);
    for (int t = 0; t < n; ++t) {
        p->wr[t] = creal(p->line->w[t]);
        p->wi[t] = cimag(p->line->w[t]);
    }
    int Ns = 1;
    for (int s = 0; s < p->nf; ++s) {
        const int R = p->line->f[s];
        p->f[s] = R;
        p->ns[s] = Ns;
        const int tw_step = n / (Ns * R);
        p->twr[s] = (double *)malloc(sizeof(double) * (size_t)Ns * (R - 1) + 8);
        p->twi[s] = (double *)malloc(sizeof(double) * (size_t)Ns * (R - 1) + 8);
        for (int k = 0; k < Ns; ++k)
            for (int r = 1; r < R; ++r) {
                const long t = ((long)k * r * tw_step) % n;
                p->twr[s][(long)k * (R - 1) + r - 1] = p->wr[t];
                p->twi[s][(long)k * (R - 1) + r - 1] = p->wi[t];
            }
        Ns *= R;
    }
    return p;
}

static void bplan_destroy(bplan *p)
{
    if (!p) return;
    for (int s = 0; s < p->nf; ++s) { free(p->twr[s]); free(p->twi[s]); }
    free(p->wr);
    free(p->wi);
    orc_fft1_destroy(p->line);
    free(p);
}

/* one batched pass of radix R; the arithmetic of each lane is that of pass():
 * input element j + r m (j = jj Ns + k) times W^{k r tw_step}, an R-point
 * butterfly, output element jj Ns R + k + q Ns */
static void bpass(const bplan *p, int s, const double *restrict ar, const double *restrict ai,
                  double *restrict br, double *restrict bi, int sign)
{
    const int n = p->n, R = p->f[s], Ns = p->ns[s], m = n / R;
    const double *twr = p->twr[s], *twi = p->twi[s];
    const double sg = sign < 0 ? 1.0 : -1.0;      /* backward: conjugate twiddles */
    const int nj = m / Ns;
    if (R == 4) {
        for (int jj = 0; jj < nj; ++jj)
            for (int k = 0; k < Ns; ++k) {
                const long j = (long)jj * Ns + k;
                const long d = (long)jj * Ns * 4 + k;
                const double c1 = twr[3 * k], s1 = sg * twi[3 * k];
                const double c2 = twr[3 * k + 1], s2 = sg * twi[3 * k + 1];
                const double c3 = twr[3 * k + 2], s3 = sg * twi[3 * k + 2];
                const double *x0r = ar + j * OB, *x0i = ai + j * OB;
                const double *x1r = ar + (j + m) * OB, *x1i = ai + (j + m) * OB;
                const double *x2r = ar + (j + 2 * m) * OB, *x2i = ai + (j + 2 * m) * OB;
                const double *x3r = ar + (j + 3 * m) * OB, *x3i = ai + (j + 3 * m) * OB;
                double *o0r = br + d * OB, *o0i = bi + d * OB;
                double *o1r = br + (d + Ns) * OB, *o1i = bi + (d + Ns) * OB;
                double *o2r = br + (d + 2 * Ns) * OB, *o2i = bi + (d + 2 * Ns) * OB;
                double *o3r = br + (d + 3 * Ns) * OB, *o3i = bi + (d + 3 * Ns) * OB;
                for (int b = 0; b < OB; ++b) {
                    const double v0r = x0r[b], v0i = x0i[b];
                    const double v1r = x1r[b] * c1 - x1i[b] * s1, v1i = x1r[b] * s1 + x1i[b] * c1;
                    const double v2r = x2r[b] * c2 - x2i[b] * s2, v2i = x2r[b] * s2 + x2i[b] * c2;
                    const double v3r = x3r[b] * c3 - x3i[b] * s3, v3i = x3r[b] * s3 + x3i[b] * c3;
                    const double a0r = v0r + v2r, a0i = v0i + v2i;
                    const double a1r = v0r - v2r, a1i = v0i - v2i;
                    const double b0r = v1r + v3r, b0i = v1i + v3i;
                    const double b1r = v1r - v3r, b1i = v1i - v3i;
                    /* forward: -i b1; backward: +i b1 */
                    const double jr = sign < 0 ? b1i : -b1i, ji = sign < 0 ? -b1r : b1r;
                    o0r[b] = a0r + b0r; o0i[b] = a0i + b0i;
                    o1r[b] = a1r + jr;  o1i[b] = a1i + ji;
                    o2r[b] = a0r - b0r; o2i[b] = a0i - b0i;
                    o3r[b] = a1r - jr;  o3i[b] = a1i - ji;
                }
            }
        return;
    }
    if (R == 2) {
        for (int jj = 0; jj < nj; ++jj)
            for (int k = 0; k < Ns; ++k) {
                const long j = (long)jj * Ns + k;
                const long d = (long)jj * Ns * 2 + k;
                const double c1 = twr[k], s1 = sg * twi[k];
                const double *x0r = ar + j * OB, *x0i = ai + j * OB;
                const double *x1r = ar + (j + m) * OB, *x1i = ai + (j + m) * OB;
                double *o0r = br + d * OB, *o0i = bi + d * OB;
                double *o1r = br + (d + Ns) * OB, *o1i = bi + (d + Ns) * OB;
                for (int b = 0; b < OB; ++b) {
                    const double v1r = x1r[b] * c1 - x1i[b] * s1, v1i = x1r[b] * s1 + x1i[b] * c1;
                    o0r[b] = x0r[b] + v1r; o0i[b] = x0i[b] + v1i;
                    o1r[b] = x0r[b] - v1r; o1i[b] = x0i[b] - v1i;
                }
            }
        return;
    }
    /* direct R-point DFT, R prime (3, 5 or larger) */
    double vr[64][OB], vi[64][OB];
    const int step = n / R;
    for (int jj = 0; jj < nj; ++jj)
        for (int k = 0; k < Ns; ++k) {
            const long j = (long)jj * Ns + k;
            const long d = (long)jj * Ns * R + k;
            for (int r = 0; r < R; ++r) {
                const double *xr = ar + (j + (long)r * m) * OB, *xi = ai + (j + (long)r * m) * OB;
                if (r == 0) {
                    for (int b = 0; b < OB; ++b) { vr[0][b] = xr[b]; vi[0][b] = xi[b]; }
                } else {
                    const double c = twr[(long)k * (R - 1) + r - 1], sn = sg * twi[(long)k * (R - 1) + r - 1];
                    for (int b = 0; b < OB; ++b) {
                        vr[r][b] = xr[b] * c - xi[b] * sn;
                        vi[r][b] = xr[b] * sn + xi[b] * c;
                    }
                }
            }
            for (int q = 0; q < R; ++q) {
                double sr[OB], si[OB];
                for (int b = 0; b < OB; ++b) { sr[b] = 0.0; si[b] = 0.0; }
                for (int r = 0; r < R; ++r) {
                    const long t = ((long)r * q % R) * step;
                    const double c = p->wr[t], sn = sg * p->wi[t];
                    for (int b = 0; b < OB; ++b) {
                        sr[b] = sr[b] + (vr[r][b] * c - vi[r][b] * sn);
                        si[b] = si[b] + (vr[r][b] * sn + vi[r][b] * c);
                    }
                }
                double *or_ = br + (d + (long)q * Ns) * OB, *oi = bi + (d + (long)q * Ns) * OB;
                for (int b = 0; b < OB; ++b) { or_[b] = sr[b]; oi[b] = si[b]; }
            }
        }
}

/* transform OB lanes held in (re, im); (wr, wi) is scratch of the same size */
static void bexec(const bplan *p, double *re, double *im, double *wr, double *wi, int sign)
{
    const int n = p->n;
    if (n <= 1) return;
    if (!p->batched) {
        orc_cplx *buf = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
        orc_cplx *work = (orc_cplx *)malloc(sizeof(orc_cplx) * n);
        for (int b = 0; b < OB; ++b) {
            for (int e = 0; e < n; ++e) buf[e] = re[e * OB + b] + I * im[e * OB + b];
            exec_buf(p->line, buf, work, sign);
            for (int e = 0; e < n; ++e) { re[e * OB + b] = creal(buf[e]); im[e * OB + b] = cimag(buf[e]); }
        }
        free(buf);
        free(work);
        return;
    }
    double *ar = re, *ai = im, *br = wr, *bi = wi;
    for (int s = 0; s < p->nf; ++s) {
        bpass(p, s, ar, ai, br, bi, sign);
        double *t = ar; ar = br; br = t;
        t = ai; ai = bi; bi = t;
    }
    if (ar != re) {
        memcpy(re, ar, sizeof(double) * (size_t)n * OB);
        memcpy(im, ai, sizeof(double) * (size_t)n * OB);
    }
}

struct orc_fft3 {
    int nx, ny, nz, nkx;
    bplan *px, *py, *pz;
    double norm;
    long count;
    orc_cplx *tmp;    /* (nkx,ny,nz) work array of the backward transform */
};

orc_fft3 *orc_fft3_create(int nx, int ny, int nz)
{
    orc_fft3 *f = (orc_fft3 *)calloc(1, sizeof(*f));
    f->nx = nx; f->ny = ny; f->nz = nz; f->nkx = nx / 2 + 1;
    f->px = bplan_create(nx);
    f->py = bplan_create(ny);
    f->pz = bplan_create(nz);
    f->norm = 1.0 / ((double)nx * (double)ny * (double)nz);
    f->tmp = (orc_cplx *)malloc(sizeof(orc_cplx) * (size_t)f->nkx * ny * nz);
    return f;
}

void orc_fft3_destroy(orc_fft3 *f)
{
    if (!f) return;
    bplan_destroy(f->px);
    bplan_destroy(f->py);
    bplan_destroy(f->pz);
    free(f->tmp);
    free(f);
}

long orc_fft3_count(const orc_fft3 *f) { return f->count; }

/* transform along y (axis 1) or z (axis 2) of a (nkx,ny,nz) complex array,
 * reading src and writing dst (which may be src), OB consecutive kx at once */
static void lines_yz(orc_fft3 *f, const orc_cplx *src, orc_cplx *dst, int axis, int sign)
{
    const int nkx = f->nkx, ny = f->ny, nz = f->nz;
    const int len = axis == 1 ? ny : nz;
    const int nblk = (nkx + OB - 1) / OB;
    const int nother = axis == 1 ? nz : ny;
    const long stride = axis == 1 ? nkx : (long)nkx * ny;
    const bplan *p = axis == 1 ? f->py : f->pz;
#pragma omp parallel
    {
        double *re = (double *)malloc(sizeof(double) * 4 * (size_t)len * OB);
        double *im = re + (size_t)len * OB, *wr = im + (size_t)len * OB, *wi = wr + (size_t)len * OB;
#pragma omp for schedule(static)
        for (long t = 0; t < (long)nblk * nother; ++t) {
            const int blk = (int)(t % nblk), o = (int)(t / nblk);
            const int i0 = blk * OB, lanes = nkx - i0 < OB ? nkx - i0 : OB;
            const long base = i0 + (axis == 1 ? (long)nkx * ny * o : (long)nkx * o);
            for (int e = 0; e < len; ++e) {
                const orc_cplx *a = src + base + e * stride;
                for (int b = 0; b < OB; ++b) {
                    re[e * OB + b] = b < lanes ? creal(a[b]) : 0.0;
                    im[e * OB + b] = b < lanes ? cimag(a[b]) : 0.0;
                }
            }
            bexec(p, re, im, wr, wi, sign);
            for (int e = 0; e < len; ++e) {
                orc_cplx *a = dst + base + e * stride;
                for (int b = 0; b < lanes; ++b) a[b] = re[e * OB + b] + I * im[e * OB + b];
            }
        }
        free(re);
    }
}

void orc_fft3_fwd(orc_fft3 *f, const double *u, orc_cplx *uhat)
{
    const int nx = f->nx, ny = f->ny, nz = f->nz, nkx = f->nkx;
    const long nrows = (long)ny * nz;
    /* two real rows per lane: z = x_a + i x_b, Z = DFT(z);
     * X_a[k] = (Z[k] + conj Z[-k])/2, X_b[k] = (Z[k] - conj Z[-k])/(2i) */
    const long nblk = (nrows + 2 * OB - 1) / (2 * OB);
#pragma omp parallel
    {
        double *re = (double *)malloc(sizeof(double) * 4 * (size_t)nx * OB);
        double *im = re + (size_t)nx * OB, *wr = im + (size_t)nx * OB, *wi = wr + (size_t)nx * OB;
#pragma omp for schedule(static)
        for (long blk = 0; blk < nblk; ++blk) {
            const long r0 = blk * 2 * OB;
            for (int b = 0; b < OB; ++b) {
                const long ra = r0 + b, rb = r0 + OB + b;
                const double *rowa = u + nx * ra, *rowb = u + nx * rb;
                for (int i = 0; i < nx; ++i) {
                    re[i * OB + b] = ra < nrows ? rowa[i] : 0.0;
                    im[i * OB + b] = rb < nrows ? rowb[i] : 0.0;
                }
            }
            bexec(f->px, re, im, wr, wi, -1);
            for (int b = 0; b < OB; ++b) {
                const long ra = r0 + b, rb = r0 + OB + b;
                for (int i = 0; i < nkx; ++i) {
                    const int ni = i == 0 ? 0 : nx - i;
                    const double zr = re[i * OB + b], zi = im[i * OB + b];
                    const double vr = re[ni * OB + b], vi = im[ni * OB + b];
                    if (ra < nrows) uhat[(long)nkx * ra + i] = 0.5 * (zr + vr) + I * (0.5 * (zi - vi));
                    if (rb < nrows) uhat[(long)nkx * rb + i] = 0.5 * (zi + vi) - I * (0.5 * (zr - vr));
                }
            }
        }
        free(re);
    }
    if (ny > 1) lines_yz(f, uhat, uhat, 1, -1);
    if (nz > 1) lines_yz(f, uhat, uhat, 2, -1);
    const long nh = (long)nkx * ny * nz;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nh; ++q) uhat[q] *= f->norm;
    f->count++;
}

void orc_fft3_bwd(orc_fft3 *f, const orc_cplx *uhat, double *u)
{
    const int nx = f->nx, ny = f->ny, nz = f->nz, nkx = f->nkx;
    const orc_cplx *src = uhat;
    if (nz > 1) { lines_yz(f, src, f->tmp, 2, +1); src = f->tmp; }
    if (ny > 1) { lines_yz(f, src, f->tmp, 1, +1); src = f->tmp; }
    const long nrows = (long)ny * nz;
    /* two half-spectrum rows per lane: Z = A + i B with A, B the Hermitian
     * extensions of rows a and b; z = IDFT(Z) gives x_a = Re z, x_b = Im z.
     * The imaginary parts of the self-conjugate bins (kx = 0 and kx = nx/2)
     * are dropped, as a c2r transform ignores them. */
    const long nblk = (nrows + 2 * OB - 1) / (2 * OB);
#pragma omp parallel
    {
        double *re = (double *)malloc(sizeof(double) * 4 * (size_t)nx * OB);
        double *im = re + (size_t)nx * OB, *wr = im + (size_t)nx * OB, *wi = wr + (size_t)nx * OB;
#pragma omp for schedule(static)
        for (long blk = 0; blk < nblk; ++blk) {
            const long r0 = blk * 2 * OB;
            for (int b = 0; b < OB; ++b) {
                const long ra = r0 + b, rb = r0 + OB + b;
                const orc_cplx *ha = src + (long)nkx * (ra < nrows ? ra : 0);
                const orc_cplx *hb = src + (long)nkx * (rb < nrows ? rb : 0);
                const double ma = ra < nrows ? 1.0 : 0.0, mb = rb < nrows ? 1.0 : 0.0;
                for (int i = 0; i < nx; ++i) {
                    const int h = i < nkx ? i : nx - i;
                    const int self = (i == 0) || (2 * i == nx);
                    double ar = ma * creal(ha[h]), ai = self ? 0.0 : ma * cimag(ha[h]);
                    double br = mb * creal(hb[h]), bi = self ? 0.0 : mb * cimag(hb[h]);
                    if (i >= nkx) { ai = -ai; bi = -bi; }
                    re[i * OB + b] = ar - bi;
                    im[i * OB + b] = ai + br;
                }
            }
            bexec(f->px, re, im, wr, wi, +1);
            for (int b = 0; b < OB; ++b) {
                const long ra = r0 + b, rb = r0 + OB + b;
                if (ra < nrows) {
                    double *row = u + (long)nx * ra;
                    for (int i = 0; i < nx; ++i) row[i] = re[i * OB + b];
                }
                if (rb < nrows) {
                    double *row = u + (long)nx * rb;
                    for (int i = 0; i < nx; ++i) row[i] = im[i * OB + b];
                }
            }
        }
        free(re);
    }
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
