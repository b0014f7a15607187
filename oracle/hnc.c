/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 * Pair potentials (src/structure/pair_potential.f90:62-143), the
 * Fourier-Bessel transform pair and the Ornstein-Zernike/HNC solver
 * (src/structure/oz_hnc.f90:57-296), and the structure source
 * (src/structure/structure_source.f90:37-83), plus linear interpolation
 * (src/core/utils.f90:30-55).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double PI = 3.14159265358979323846264338327950288;
static const double TWOPI = 2.0 * 3.14159265358979323846264338327950288;

/* ------------------------------------------------------------ potentials */
double orc_pot_beta_v(const orc_pot *p, double r)
{
    switch (p->kind) {
    case ORC_POT_YUKAWA:   /* pair_potential.f90:62-66 */
        return p->gamma * exp(-p->kappa * r) / r;
    case ORC_POT_COULOMB:  /* :68-72 */
        return p->gamma / r;
    default: {             /* hm_beta_v :74-84 */
        const double ln2 = 0.693147180559945309417232121458;
        double v;
        if (r > 0.0) v = p->gamma * (1.0 - exp(-TWOPI * r / p->lambda)) / r;
        else v = p->gamma * TWOPI / p->lambda;
        if (p->pauli) v = v + ln2 * exp(-4.0 * PI * r * r / (p->lambda * p->lambda * ln2));
        return v;
    }
    }
}

/* pair_potential.f90:86-96 */
double orc_pot_beta_v_long_r(const orc_pot *p, double r)
{
    double kp = p->kappa + p->ksplit;
    if (r > 1.0e-12) return p->gamma * (exp(-p->kappa * r) - exp(-kp * r)) / r;
    return p->gamma * (kp - p->kappa);
}

/* pair_potential.f90:99-105 */
double orc_pot_beta_v_long_k(const orc_pot *p, double k)
{
    double kp = p->kappa + p->ksplit;
    return 4.0 * PI * p->gamma * (1.0 / (k * k + p->kappa * p->kappa) - 1.0 / (k * k + kp * kp));
}

/* pair_potential.f90:107-111 */
double orc_pot_beta_v_short(const orc_pot *p, double r)
{
    return orc_pot_beta_v(p, r) - orc_pot_beta_v_long_r(p, r);
}

/* pair_potential.f90:114-118 */
double orc_pot_beta_v_k(const orc_pot *p, double k)
{
    return 4.0 * PI * p->gamma / (k * k + p->kappa * p->kappa);
}

/* ------------------------------------------------------- Fourier-Bessel */
typedef struct {
    int n;
    double dr, dk;
    double *r, *k, *win, *wout;
    orc_dst1 *dst;
} fb_t;

/* oz_hnc.f90:57-76 */
static void fb_init(fb_t *fb, int n, double rmax)
{
    fb->n = n;
    fb->dr = rmax / (n + 1);
    fb->dk = PI / ((n + 1) * fb->dr);
    fb->r = (double *)malloc(sizeof(double) * n);
    fb->k = (double *)malloc(sizeof(double) * n);
    fb->win = (double *)malloc(sizeof(double) * n);
    fb->wout = (double *)malloc(sizeof(double) * n);
    for (int j = 1; j <= n; ++j) {
        fb->r[j - 1] = j * fb->dr;
        fb->k[j - 1] = j * fb->dk;
    }
    fb->dst = orc_dst1_create(n);
}

static void fb_free(fb_t *fb)
{
    free(fb->r); free(fb->k); free(fb->win); free(fb->wout);
    orc_dst1_destroy(fb->dst);
    memset(fb, 0, sizeof(*fb));
}

/* oz_hnc.f90:79-86 */
static void fb_r2k(fb_t *fb, const double *fr, double *fk)
{
    for (int j = 0; j < fb->n; ++j) fb->win[j] = fb->r[j] * fr[j];
    orc_dst1_exec(fb->dst, fb->win, fb->wout);
    for (int j = 0; j < fb->n; ++j) fk[j] = TWOPI * fb->dr * fb->wout[j] / fb->k[j];
}

/* oz_hnc.f90:89-96 */
static void fb_k2r(fb_t *fb, const double *fk, double *fr)
{
    for (int j = 0; j < fb->n; ++j) fb->win[j] = fb->k[j] * fk[j];
    orc_dst1_exec(fb->dst, fb->win, fb->wout);
    for (int j = 0; j < fb->n; ++j) fr[j] = fb->dk * fb->wout[j] / (4.0 * PI * PI * fb->r[j]);
}

void orc_fb_r2k(int n, double rmax, const double *fr, double *fk)
{
    fb_t fb; fb_init(&fb, n, rmax); fb_r2k(&fb, fr, fk); fb_free(&fb);
}

void orc_fb_k2r(int n, double rmax, const double *fk, double *fr)
{
    fb_t fb; fb_init(&fb, n, rmax); fb_k2r(&fb, fk, fr); fb_free(&fb);
}

static double dot(int n, const double *a, const double *b)
{
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += a[j] * b[j];
    return s;
}

/* oz_hnc.f90:142-296.  Returns 0 on success; *unstable_out as in the reference. */
static void hnc_solve_direct(const orc_pot *pot, double n0, int nr, double rmax, double tol,
                             double mix, int maxiter, orc_hnc_result *res, int *unstable_out,
                             double *gs_out, const double *gamma_s_init)
{
    const double expcap = 40.0;
    const int npicard = 5;
    fb_t fb;
    fb_init(&fb, nr, rmax);
    double *bvs = malloc(sizeof(double) * nr), *bvl_r = malloc(sizeof(double) * nr);
    double *bvl_k = malloc(sizeof(double) * nr), *gs = malloc(sizeof(double) * nr);
    double *gnew = malloc(sizeof(double) * nr), *cs = malloc(sizeof(double) * nr);
    double *csk = malloc(sizeof(double) * nr), *ck = malloc(sizeof(double) * nr);
    double *gk = malloc(sizeof(double) * nr);
    double *hin = calloc(3 * (size_t)nr, sizeof(double)), *hout = calloc(3 * (size_t)nr, sizeof(double));
    double *d0 = malloc(sizeof(double) * nr), *d01 = malloc(sizeof(double) * nr);
    double *d02 = malloc(sizeof(double) * nr), *gtry = malloc(sizeof(double) * nr);
    double *gk_mf = malloc(sizeof(double) * nr);
    for (int j = 0; j < nr; ++j) {
        bvs[j] = orc_pot_beta_v_short(pot, fb.r[j]);
        bvl_r[j] = orc_pot_beta_v_long_r(pot, fb.r[j]);
        bvl_k[j] = orc_pot_beta_v_long_k(pot, fb.k[j]);
    }
    for (int j = 0; j < nr; ++j) {
        ck[j] = -orc_pot_beta_v_k(pot, fb.k[j]);
        gk[j] = n0 * ck[j] * ck[j] / (1.0 - n0 * ck[j]) - bvl_k[j];
    }
    fb_k2r(&fb, gk, gs);
    if (gamma_s_init) memcpy(gs, gamma_s_init, sizeof(double) * nr);
    double mixc = mix;
    res->converged = 0;
    for (int j = 0; j < nr; ++j) {
        ck[j] = -orc_pot_beta_v_k(pot, fb.k[j]);
        gk_mf[j] = n0 * ck[j] * ck[j] / (1.0 - n0 * ck[j]) - bvl_k[j];
    }
    double resid = 0.0;
    int unstable = 0, it_total = 0;
    for (int irestart = 1; irestart <= 4; ++irestart) {
        memset(hin, 0, sizeof(double) * 3 * nr);
        memset(hout, 0, sizeof(double) * 3 * nr);
        int nhist = 0, ng_cooldown = 0;
        double resid_prev = 1.0e100;
        unstable = 0;
        it_total = 0;
        for (int it = 1; it <= maxiter; ++it) {
            it_total = it;
            for (int j = 0; j < nr; ++j) {
                double ex = -bvs[j] + gs[j];
                cs[j] = exp(ex < expcap ? ex : expcap) - 1.0 - gs[j];
            }
            fb_r2k(&fb, cs, csk);
            int bad = 0;
            for (int j = 0; j < nr; ++j) {
                ck[j] = csk[j] - bvl_k[j];
                if (n0 * ck[j] >= 1.0) bad = 1;
            }
            if (bad) { unstable = 1; break; }
            for (int j = 0; j < nr; ++j) gk[j] = n0 * ck[j] * ck[j] / (1.0 - n0 * ck[j]) - bvl_k[j];
            fb_k2r(&fb, gk, gnew);
            resid = 0.0;
            for (int j = 0; j < nr; ++j) {
                double d = fabs(gnew[j] - gs[j]);
                if (d > resid) resid = d;
            }
            if (resid < tol) {
                memcpy(gs, gnew, sizeof(double) * nr);
                res->converged = 1;
                break;
            }
            if (resid > 1.0e6) { unstable = 1; break; }
            /* history shift: column 3 <- 2 <- 1 <- current */
            memcpy(hin + 2 * nr, hin + nr, sizeof(double) * nr);
            memcpy(hin + nr, hin, sizeof(double) * nr);
            memcpy(hin, gs, sizeof(double) * nr);
            memcpy(hout + 2 * nr, hout + nr, sizeof(double) * nr);
            memcpy(hout + nr, hout, sizeof(double) * nr);
            memcpy(hout, gnew, sizeof(double) * nr);
            nhist = nhist + 1 < 3 ? nhist + 1 : 3;
            if (resid > 10.0 * resid_prev) ng_cooldown = 10;
            if (nhist == 3 && it > npicard && ng_cooldown == 0) {
                for (int j = 0; j < nr; ++j) {
                    d0[j] = hout[j] - hin[j];
                    d01[j] = d0[j] - (hout[nr + j] - hin[nr + j]);
                    d02[j] = d0[j] - (hout[2 * nr + j] - hin[2 * nr + j]);
                }
                double a11 = dot(nr, d01, d01), a12 = dot(nr, d01, d02), a22 = dot(nr, d02, d02);
                double b1 = dot(nr, d0, d01), b2 = dot(nr, d0, d02);
                double det = a11 * a22 - a12 * a12;
                int accepted = 0;
                if (fabs(det) > 1.0e-14 * a11 * a22 && a11 > 0.0 && a22 > 0.0) {
                    double c1 = (b1 * a22 - b2 * a12) / det;
                    double c2 = (a11 * b2 - a12 * b1) / det;
                    if (fabs(c1) < 20.0 && fabs(c2) < 20.0) {
                        double mx = -INFINITY;
                        for (int j = 0; j < nr; ++j) {
                            gtry[j] = (1.0 - c1 - c2) * hout[j] + c1 * hout[nr + j] + c2 * hout[2 * nr + j];
                            double d = gtry[j] - bvs[j];
                            if (d > mx) mx = d;
                        }
                        if (mx < expcap) {
                            memcpy(gs, gtry, sizeof(double) * nr);
                            accepted = 1;
                        }
                    }
                }
                if (!accepted)
                    for (int j = 0; j < nr; ++j) gs[j] = (1.0 - mixc) * gs[j] + mixc * gnew[j];
            } else {
                for (int j = 0; j < nr; ++j) gs[j] = (1.0 - mixc) * gs[j] + mixc * gnew[j];
                if (ng_cooldown > 0) ng_cooldown = ng_cooldown - 1;
            }
            resid_prev = resid;
        }
        if (res->converged || !unstable) break;
        mixc = 0.5 * mixc;
        fb_k2r(&fb, gk_mf, gs);
        if (gamma_s_init) memcpy(gs, gamma_s_init, sizeof(double) * nr);
    }
    res->niter = it_total < maxiter ? it_total : maxiter;
    res->residual = resid;
    *unstable_out = unstable;
    memcpy(gs_out, gs, sizeof(double) * nr);
    if (!unstable) {
        res->nr = nr; res->n0 = n0; res->dr = fb.dr; res->dk = fb.dk;
        res->r = malloc(sizeof(double) * nr); res->k = malloc(sizeof(double) * nr);
        res->g = malloc(sizeof(double) * nr); res->cr = malloc(sizeof(double) * nr);
        res->ck = malloc(sizeof(double) * nr); res->hk = malloc(sizeof(double) * nr);
        res->sk = malloc(sizeof(double) * nr);
        memcpy(res->r, fb.r, sizeof(double) * nr);
        memcpy(res->k, fb.k, sizeof(double) * nr);
        for (int j = 0; j < nr; ++j) {
            double ex = -bvs[j] + gs[j];
            res->g[j] = exp(ex < expcap ? ex : expcap);
            cs[j] = res->g[j] - 1.0 - gs[j];
        }
        fb_r2k(&fb, cs, csk);
        for (int j = 0; j < nr; ++j) {
            res->ck[j] = csk[j] - bvl_k[j];
            res->hk[j] = res->ck[j] / (1.0 - n0 * res->ck[j]);
            res->sk[j] = 1.0 + n0 * res->hk[j];
            res->cr[j] = cs[j] - bvl_r[j];
        }
        double s = 0.0;
        for (int j = 0; j < nr; ++j)
            s += fb.r[j] * fb.r[j] * (res->g[j] - 1.0) * orc_pot_beta_v(pot, fb.r[j]);
        res->u_ex = 2.0 * PI * n0 * (fb.dr * s);
    }
    free(bvs); free(bvl_r); free(bvl_k); free(gs); free(gnew); free(cs); free(csk); free(ck);
    free(gk); free(hin); free(hout); free(d0); free(d01); free(d02); free(gtry); free(gk_mf);
    fb_free(&fb);
}

void orc_hnc_result_free(orc_hnc_result *res)
{
    free(res->r); free(res->k); free(res->g); free(res->cr); free(res->ck);
    free(res->hk); free(res->sk);
    memset(res, 0, sizeof(*res));
}

/* oz_hnc.f90:111-140.  Returns 1 where the reference calls fatal. */
int orc_hnc_solve(const orc_pot *pot, double n0, int nr, double rmax, double tol, double mix,
                  int maxiter, orc_hnc_result *res)
{
    memset(res, 0, sizeof(*res));
    double *gs = malloc(sizeof(double) * nr), *gs_init = calloc(nr, sizeof(double));
    int unstable = 0;
    hnc_solve_direct(pot, n0, nr, rmax, tol, mix, maxiter, res, &unstable, gs, NULL);
    int rc = 0;
    if (unstable) {
        orc_pot p = *pot;
        double gtarget = pot->gamma;
        double g = gtarget < 2.0 ? gtarget : 2.0;
        for (int istep = 1; istep <= 200; ++istep) {
            p.gamma = g;
            orc_hnc_result_free(res);
            hnc_solve_direct(&p, n0, nr, rmax, tol, mix, maxiter, res, &unstable, gs, gs_init);
            if (unstable) { rc = 1; break; }
            memcpy(gs_init, gs, sizeof(double) * nr);
            if (g >= gtarget) break;
            g = gtarget < g * 1.3 ? gtarget : g * 1.3;
        }
    }
    free(gs);
    free(gs_init);
    return rc;
}

/* ----------------------------------------------------------- structure */
/* utils.f90:30-55 */
double orc_interp_linear(int n, const double *x, const double *y, double xq)
{
    if (n == 1) return y[0];
    int lo;
    if (xq <= x[0]) lo = 1;
    else if (xq >= x[n - 1]) lo = n - 1;
    else {
        lo = 1;
        int hi = n;
        while (hi - lo > 1) {
            int mid = (lo + hi) / 2;
            if (x[mid - 1] <= xq) lo = mid; else hi = mid;
        }
    }
    double w = (xq - x[lo - 1]) / (x[lo] - x[lo - 1]);
    return (1.0 - w) * y[lo - 1] + w * y[lo];
}

/* structure_source.f90:37-41 */
double orc_structure_c_of_k(const orc_structure *st, double k)
{
    double kk = k < st->k[st->n - 1] ? k : st->k[st->n - 1];
    return orc_interp_linear(st->n, st->k, st->c, kk);
}

void orc_structure_set(orc_structure *st, int n, const double *k, const double *c, double n0,
                       double u_ex, double du_dgamma, int has_energy)
{
    memset(st, 0, sizeof(*st));
    st->n = n;
    st->n0 = n0;
    st->k = malloc(sizeof(double) * n);
    st->c = malloc(sizeof(double) * n);
    st->s = malloc(sizeof(double) * n);
    memcpy(st->k, k, sizeof(double) * n);
    memcpy(st->c, c, sizeof(double) * n);
    for (int j = 0; j < n; ++j) st->s[j] = 1.0 / (1.0 - n0 * c[j]);
    st->u_ex = u_ex;
    st->du_dgamma = du_dgamma;
    st->has_energy = has_energy;
}

void orc_structure_free(orc_structure *st)
{
    free(st->k); free(st->c); free(st->s);
    memset(st, 0, sizeof(*st));
}

/* structure_source.f90:50-83.  Returns nonzero where the reference is fatal. */
int orc_structure_from_hnc(orc_pot *pot, double n0, int nr, double rmax, double tol, double mix,
                           int maxiter, int with_derivative, orc_structure *st)
{
    orc_hnc_result res, rp1, rm1;
    if (orc_hnc_solve(pot, n0, nr, rmax, tol, mix, maxiter, &res)) return 1;
    if (!res.converged) { orc_hnc_result_free(&res); return 2; }
    memset(st, 0, sizeof(*st));
    st->n = nr;
    st->n0 = n0;
    st->k = res.k; st->c = res.ck; st->s = res.sk;
    res.k = res.ck = res.sk = NULL;
    st->u_ex = res.u_ex;
    st->has_energy = 1;
    orc_hnc_result_free(&res);
    if (with_derivative) {
        double g0 = pot->gamma, dg = 0.02 * g0;
        pot->gamma = g0 + dg;
        int e1 = orc_hnc_solve(pot, n0, nr, rmax, tol, mix, maxiter, &rp1);
        pot->gamma = g0 - dg;
        int e2 = orc_hnc_solve(pot, n0, nr, rmax, tol, mix, maxiter, &rm1);
        pot->gamma = g0;
        if (e1 || e2 || !(rp1.converged && rm1.converged)) {
            orc_hnc_result_free(&rp1); orc_hnc_result_free(&rm1);
            return 3;
        }
        st->du_dgamma = (rp1.u_ex - rm1.u_ex) / (2.0 * dg);
        orc_hnc_result_free(&rp1); orc_hnc_result_free(&rm1);
    }
    return 0;
}
