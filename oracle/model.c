/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 * Species factory, free-energy terms, stress closure, external potential,
 * initial conditions, the time-dependent model, diagnostics, linear response
 * and analysis fits, restating (file:line in the reference):
 *   src/core/units.f90:41-70           units_init
 *   src/transport/transport.f90:61-111 transport_setup
 *   src/transport/stanton_murillo.f90:63-154
 *   src/model/species.f90:49-169       species_build / allocate_state
 *   src/functional/functional.f90:56-102, fe_ideal_classical.f90:33-55,
 *   fe_kinetic_tfk.f90:63-166, fe_hartree.f90:34-80, fe_correlation_ry.f90:39-98
 *   src/closure/stress.f90:37-105
 *   src/model/external_potential.f90:39-93
 *   src/model/initial.f90:23-75        (uniform, mode, gaussian)
 *   src/model/model.f90:56-227         init, velocity, rhs, compute_dt, advance
 *   src/model/diagnostics.f90:41-60    budgets
 *   src/linear/linear_response.f90:45-171
 *   src/model/analysis.f90:21-98
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double PI = 3.14159265358979323846264338327950288;
static const double TWOPI = 2.0 * 3.14159265358979323846264338327950288;
static const double SQRT2 = 1.41421356237309504880168872420969808;

/* ------------------------------------------------------------- params */
/* params.f90:17-78 defaults */
void orc_params_default(orc_params *p)
{
    memset(p, 0, sizeof(*p));
    p->nx = 64; p->ny = 1; p->nz = 1;
    p->lx = 20.0; p->ly = 1.0; p->lz = 1.0;
    p->dealias = 1;
    p->electron = 0;
    p->gamma = 2.0; p->kappa = 0.1; p->rs = 1.86; p->theta = -1.0; p->mass = 1.0;
    p->nterms = 0;
    p->tfk_gamma = 1.0 / 9.0;
    p->maxwell = 0;
    p->transport = ORC_TR_CONSTANT;
    p->eta = 0.0; p->xi = 0.0; p->tau = 0.0;
    p->tau_ichimaru = 1;
    p->adiabatic_index = 5.0 / 3.0;
    p->hnc_nr = 8192; p->hnc_maxiter = 20000;
    p->hnc_rmax = 80.0; p->hnc_tol = 1.0e-9; p->hnc_mix = 0.2;
    p->dt = 0.0; p->cfl = 0.4;
    p->vext = ORC_VEXT_NONE;
    p->vext_amplitude = 0.0; p->vext_omega = 0.0; p->vext_width = 1.0; p->vext_ramp = 0.0;
    p->vext_mode[0] = 1; p->vext_mode[1] = 0; p->vext_mode[2] = 0;
}

/* ------------------------------------------------------ stanton-murillo */
static const double SM_A[4][5] = {
    {1.4660, -1.7836, 1.4313, -0.55833, 0.061162},
    {0.52094, 0.25153, -1.1337, 1.2155, -0.43784},
    {0.30346, 0.23739, -0.62167, 0.56110, -0.18046},
    {0.85401, -0.22898, -0.60059, 0.80591, -0.30555}};
static const double SM_B[4][5] = {
    {0.081033, -0.091336, 0.051760, -0.50026, 0.17044},
    {0.20572, -0.16536, 0.061572, -0.12770, 0.066993},
    {0.68375, -0.38459, 0.10711, 0.10649, 0.028760},
    {0.43475, -0.21147, 0.11116, 0.19665, 0.15195}};
static const int SM_N[4] = {1, 1, 1, 2}, SM_M[4] = {1, 2, 3, 2};
static const double SQRT3PI = 3.0699801238394655;

/* stanton_murillo.f90:63-82 (idx 1..4) */
double orc_sm_knm(int idx, double g)
{
    const int ii = idx - 1;
    double fact = 1.0;
    for (int i = 2; i <= SM_M[ii] - 1; ++i) fact *= i;
    if (g < 1.0) {
        double s = 0.0, gg = g > DBL_MIN ? g : DBL_MIN;
        for (int i = 5; i >= 1; --i) s = (s + SM_A[ii][i - 1]) * gg;
        return -0.25 * SM_N[ii] * fact * log(s);
    }
    double lg = log(g);
    return (SM_B[ii][0] + SM_B[ii][1] * lg + SM_B[ii][2] * lg * lg) /
           (1.0 + SM_B[ii][3] * g + SM_B[ii][4] * g * g);
}

/* stanton_murillo.f90:105-108, 130-133 */
double orc_sm_viscosity(double gamma, double kappa)
{
    double g = gamma * sqrt(kappa * kappa + 3.0 * gamma / (1.0 + 3.0 * gamma));
    return 5.0 * SQRT3PI / (36.0 * pow(gamma, 2.5) * orc_sm_knm(4, g));
}

/* stanton_murillo.f90:105-108 (sm_g), 124-127: D* = sqrt(3 pi)/(12 Gamma^{5/2} K_11(g)) */
double orc_sm_diffusion(double gamma, double kappa)
{
    double g = gamma * sqrt(kappa * kappa + 3.0 * gamma / (1.0 + 3.0 * gamma));
    return SQRT3PI / (12.0 * pow(gamma, 2.5) * orc_sm_knm(1, g));
}

/* stanton_murillo.f90:136-139: K* = 25 sqrt(3 pi)/(48 Gamma^{5/2} K_22(g)) */
double orc_sm_conductivity(double gamma, double kappa)
{
    double g = gamma * sqrt(kappa * kappa + 3.0 * gamma / (1.0 + 3.0 * gamma));
    return 25.0 * SQRT3PI / (48.0 * pow(gamma, 2.5) * orc_sm_knm(4, g));
}

/* stanton_murillo.f90:143-154 */
void orc_sm_electron_viscosity(double rs, double gamma, double theta, double lambda_tf,
                               double *eta_l, double *eta_cv, double *eta_sm)
{
    double cv = 1.0 / sqrt(3.0 * rs) /
                (60.0 * pow(rs, -1.5) + 80.0 / rs - 40.0 * pow(rs, -2.0 / 3.0) +
                 62.0 * pow(rs, -1.0 / 3.0));
    double sm = 5.0 * SQRT3PI / (36.0 * pow(gamma, 2.5) * orc_sm_knm(4, gamma / lambda_tf));
    *eta_l = 4.0 / 3.0 * (cv + theta * sm) / (1.0 + theta);
    if (eta_cv) *eta_cv = cv;
    if (eta_sm) *eta_sm = sm;
}

/* -------------------------------------------------------------- model */
typedef struct {
    int id;
    double n0, beta;
    double cn, alpha0, cg;          /* tf, gradient */
    double e2, kappa;               /* hartree, ry */
    int subtract_mean_field;        /* ry */
    double *vk, *ck, *w;            /* (nkx,ny,nz) kernels; w real work */
    double *alpha, *lapn, *gn;      /* work */
} term_t;

struct orc_model {
    orc_params p;
    orc_spec spc;
    /* units */
    int quantum;
    double n0, e2, gamma, kappa, beta, kT, mass, rs, hbar, theta, alpha0, cn, lambda_qsp, lambda_tf;
    orc_structure st;
    int has_st;
    int nterms;
    term_t terms[8];
    /* transport */
    double tr_eta, tr_xi, tr_tau, eta_l, elastic_modulus;
    /* stress */
    int evolve;
    double s_tau, s_eta, s_xi;
    double *gu;      /* (nx,ny,nz,3,3): gu[c + nc*(i + 3*j)] */
    /* vext */
    int ext_kind, ext_active, ext_time_dependent;
    double ext_amp, ext_omega, ext_width, ext_ramp, ext_kvec[3];
    double *ext_v, *ext_f;
    /* state and work */
    double t, dt;
    double ts;      /* stage time of the step in progress */
    int step;
    double *n, *mom, *pi;
    double *u, *mu, *gmu, *flux, *divf;
    double *wpi, *pi0, *pi0_old, *fpi, *gpi;
    double *dn, *dmom, *dpi, *dn_o, *dmom_o, *dpi_o;
    orc_cplx *nhat;
    double *tmpv;    /* 3 fields work for stress divergence */
    double *gtmp;    /* 3 fields work for stress_pi0 */
    orc_cplx *chat;  /* half-spectrum work of the RY convolution */
};

static long NC(const orc_model *m) { return (long)m->p.nx * m->p.ny * m->p.nz; }
static long NH(const orc_model *m) { return (long)m->spc.g.nkx * m->p.ny * m->p.nz; }
static double *dalloc(long n) { return (double *)calloc(n > 0 ? n : 1, sizeof(double)); }

/* memcpy of n doubles split over the OpenMP threads */
static void pcopy(double *dst, const double *src, long n)
{
#pragma omp parallel for schedule(static)
    for (long q = 0; q < n; ++q) dst[q] = src[q];
}

/* fe_hartree.f90:56-64 */
static double hartree_kernel(const term_t *t, double k)
{
    if (k * k + t->kappa * t->kappa > 0.0) return 4.0 * PI * t->e2 / (k * k + t->kappa * t->kappa);
    return 0.0;
}

/* fe_correlation_ry.f90:39-49 */
static double ry_c_cor(const orc_model *m, const term_t *t, double k)
{
    double k1 = k > m->st.k[0] ? k : m->st.k[0];
    double c = orc_structure_c_of_k(&m->st, k1);
    if (t->subtract_mean_field) c = c + t->beta * 4.0 * PI * t->e2 / (k1 * k1 + t->kappa * t->kappa);
    return c;
}

double orc_model_term_kernel(const orc_model *m, int i, double k)
{
    const term_t *t = &m->terms[i];
    switch (t->id) {
    case ORC_TERM_IDEAL: return 1.0 / (t->beta * t->n0);                          /* :49-53 */
    case ORC_TERM_TF: return 2.0 / (t->beta * t->cn * orc_fd_im12(t->alpha0));    /* tfk :84-88 */
    case ORC_TERM_GRADIENT: return 2.0 * t->cg * orc_fd_xi(t->alpha0) * k * k;    /* tfk :140-144 */
    case ORC_TERM_HARTREE: return hartree_kernel(t, k);
    case ORC_TERM_RY: return -ry_c_cor(m, t, k) / t->beta;                        /* ry :81-85 */
    }
    return 0.0;
}

/* functional.f90:72-80 */
double orc_model_kernel(const orc_model *m, double k)
{
    double kk = 0.0;
    for (int i = 0; i < m->nterms; ++i) kk += orc_model_term_kernel(m, i, k);
    return kk;
}

static int min_nonpositive(const double *a, long n)
{
    double mn = DBL_MAX;
    for (long q = 0; q < n; ++q) if (a[q] < mn) mn = a[q];
    return mn <= 0.0;
}

/* tf_alpha_of_n fe_kinetic_tfk.f90:63-72 */
static int tf_alpha_of_n(const term_t *t, const double *n, double *alpha, long nc)
{
    if (min_nonpositive(n, nc)) return 10;
    orc_fd_init();
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nc; ++q) alpha[q] = orc_fd_alpha_from_ip12(n[q] / t->cn, NULL);
    return 0;
}

/* the add_mu of each term; returns nonzero where the reference is fatal */
int orc_model_term_add_mu(orc_model *m, int i, const double *n, const orc_cplx *nhat, double *mu)
{
    term_t *t = &m->terms[i];
    orc_spec *spc = &m->spc;
    const long nc = NC(m), nh = NH(m);
    switch (t->id) {
    case ORC_TERM_IDEAL:   /* fe_ideal_classical.f90:33-41 */
        if (min_nonpositive(n, nc)) return 11;
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) mu[q] = mu[q] + log(n[q]) / t->beta;
        return 0;
    case ORC_TERM_TF: {    /* fe_kinetic_tfk.f90:74-82 */
        int rc = tf_alpha_of_n(t, n, t->alpha, nc);
        if (rc) return rc;
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) mu[q] = mu[q] + t->alpha[q] / t->beta;
        return 0;
    }
    case ORC_TERM_GRADIENT: {   /* fe_kinetic_tfk.f90:114-138 */
        if (min_nonpositive(n, nc)) return 12;
        for (int d = 1; d <= 3; ++d) {
            if (d <= spc->g.ndim) orc_spec_grad_hat(spc, nhat, d, t->gn + (d - 1) * nc);
            else memset(t->gn + (d - 1) * nc, 0, sizeof(double) * nc);
        }
        double *negk2 = dalloc(nh);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nh; ++q) negk2[q] = -spc->g.k2[q];
        orc_spec_convolve(spc, negk2, nhat, t->lapn);
        free(negk2);
        orc_fd_init();
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) {
            double a = orc_fd_alpha_from_ip12(n[q] / t->cn, NULL);
            double xi = orc_fd_xi(a);
            double dxidn = orc_fd_dxi(a) / (0.5 * t->cn * orc_fd_im12(a));
            double g2 = t->gn[q] * t->gn[q] + t->gn[nc + q] * t->gn[nc + q] +
                        t->gn[2 * nc + q] * t->gn[2 * nc + q];
            mu[q] = mu[q] - t->cg * (dxidn * g2 + 2.0 * xi * t->lapn[q]);
        }
        return 0;
    }
    case ORC_TERM_HARTREE:  /* fe_hartree.f90:46-54 */
        orc_spec_convolve(spc, t->vk, nhat, t->w);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) mu[q] = mu[q] + t->w[q];
        return 0;
    case ORC_TERM_RY: {     /* fe_correlation_ry.f90:64-80 */
        orc_cplx *b = m->chat;
        pcopy((double *)b, (const double *)nhat, 2 * nh);
        b[0] = nhat[0] - t->n0;
        orc_spec_convolve(spc, t->ck, b, t->w);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) mu[q] = mu[q] - t->w[q] / t->beta;
        return 0;
    }
    }
    return 99;
}

/* functional.f90:56-67 */
int orc_model_mu_total(orc_model *m, const double *n, const orc_cplx *nhat, double *mu)
{
    const long nc = NC(m);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nc; ++q) mu[q] = 0.0;
    for (int i = 0; i < m->nterms; ++i) {
        int rc = orc_model_term_add_mu(m, i, n, nhat, mu);
        if (rc) return rc;
    }
    return 0;
}

/* energies: fe_ideal :49-55, tf :90-103, gradient :146-166, hartree :73-80, ry :88-98 */
double orc_model_energy(orc_model *m, const double *n, const orc_cplx *nhat)
{
    orc_spec *spc = &m->spc;
    const long nc = NC(m), nh = NH(m);
    const double vol = spc->g.volume;
    double e = 0.0;
    for (int i = 0; i < m->nterms; ++i) {
        term_t *t = &m->terms[i];
        double f = 0.0, s = 0.0;
        switch (t->id) {
        case ORC_TERM_IDEAL:
            for (long q = 0; q < nc; ++q) s += n[q] * (log(n[q]) - 1.0);
            f = s / nc * vol / t->beta;
            break;
        case ORC_TERM_TF:
            tf_alpha_of_n(t, n, t->alpha, nc);
            for (long q = 0; q < nc; ++q)
                s += n[q] * t->alpha[q] - (2.0 / 3.0) * t->cn * orc_fd_ip32(t->alpha[q]);
            f = s / nc * vol / t->beta;
            break;
        case ORC_TERM_GRADIENT:
            for (int d = 1; d <= 3; ++d) {
                if (d <= spc->g.ndim) orc_spec_grad_hat(spc, nhat, d, t->gn + (d - 1) * nc);
                else memset(t->gn + (d - 1) * nc, 0, sizeof(double) * nc);
            }
            for (long q = 0; q < nc; ++q) {
                double a = orc_fd_alpha_from_ip12(n[q] / t->cn, NULL);
                s += orc_fd_xi(a) * (t->gn[q] * t->gn[q] + t->gn[nc + q] * t->gn[nc + q] +
                                     t->gn[2 * nc + q] * t->gn[2 * nc + q]);
            }
            f = t->cg * s / nc * vol;
            break;
        case ORC_TERM_HARTREE:
            orc_spec_convolve(spc, t->vk, nhat, t->w);
            for (long q = 0; q < nc; ++q) s += n[q] * t->w[q];
            f = 0.5 * (s / nc) * vol;
            break;
        case ORC_TERM_RY: {
            orc_cplx *b = (orc_cplx *)malloc(sizeof(orc_cplx) * nh);
            memcpy(b, nhat, sizeof(orc_cplx) * nh);
            b[0] = nhat[0] - t->n0;
            orc_spec_convolve(spc, t->ck, b, t->w);
            free(b);
            for (long q = 0; q < nc; ++q) s += (n[q] - t->n0) * t->w[q];
            f = -0.5 * (s / nc) * vol / t->beta;
            break;
        }
        }
        e += f;
    }
    return e;
}

/* external_potential.f90:65-93 */
static void vext_eval(orc_model *m, double t)
{
    if (!m->ext_active) return;
    orc_grid *g = &m->spc.g;
    const long nc = NC(m);
    double a = m->ext_amp;
    if (m->ext_time_dependent && m->ext_ramp > 0.0) a = a * (1.0 < t / m->ext_ramp ? 1.0 : t / m->ext_ramp);
    if (m->ext_kind == ORC_VEXT_MODE || m->ext_kind == ORC_VEXT_DRIVEN) {
        for (int k = 0; k < g->nz; ++k)
            for (int j = 0; j < g->ny; ++j)
                for (int i = 0; i < g->nx; ++i) {
                    long q = i + (long)g->nx * (j + (long)g->ny * k);
                    double ph = m->ext_kvec[0] * g->x[i] + m->ext_kvec[1] * g->y[j] +
                                m->ext_kvec[2] * g->z[k] - m->ext_omega * t;
                    m->ext_v[q] = a * cos(ph);
                    double s = a * sin(ph);
                    m->ext_f[q] = s * m->ext_kvec[0];
                    m->ext_f[nc + q] = s * m->ext_kvec[1];
                    m->ext_f[2 * nc + q] = s * m->ext_kvec[2];
                }
    } else if (m->ext_kind == ORC_VEXT_GAUSSIAN) {
        for (int k = 0; k < g->nz; ++k)
            for (int j = 0; j < g->ny; ++j)
                for (int i = 0; i < g->nx; ++i) {
                    long q = i + (long)g->nx * (j + (long)g->ny * k);
                    double x = g->x[i] - 0.5 * g->lx, y = 0.0, z = 0.0;
                    if (g->ny > 1) y = g->y[j] - 0.5 * g->ly;
                    if (g->nz > 1) z = g->z[k] - 0.5 * g->lz;
                    double r2 = x * x + y * y + z * z;
                    m->ext_v[q] = -a * exp(-0.5 * r2 / (m->ext_width * m->ext_width));
                }
        orc_spec_grad(&m->spc, m->ext_v, m->ext_f);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < 3 * nc; ++q) m->ext_f[q] = -m->ext_f[q];
    }
}

/* stress.f90:60-83 */
static void stress_pi0(orc_model *m, const double *u, double *pi)
{
    orc_spec *spc = &m->spc;
    const long nc = NC(m);
    double *gtmp = m->gtmp;
    for (int i = 1; i <= 3; ++i) {
        if (i <= spc->g.ndim) {
            orc_spec_grad(spc, u + (i - 1) * nc, gtmp);
            for (int j = 1; j <= 3; ++j)
                pcopy(m->gu + nc * ((i - 1) + 3 * (j - 1)), gtmp + (j - 1) * nc, nc);
        } else {
            for (int j = 1; j <= 3; ++j) memset(m->gu + nc * ((i - 1) + 3 * (j - 1)), 0, sizeof(double) * nc);
        }
    }
#define GU(c, i, j) m->gu[(c) + nc * (((i) - 1) + 3 * ((j) - 1))]
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; ++c) {
        double divu = GU(c, 1, 1) + GU(c, 2, 2) + GU(c, 3, 3);
        for (int i = 1; i <= 3; ++i)
            pi[(i - 1) * nc + c] = m->s_eta * (2.0 * GU(c, i, i) - (2.0 / 3.0) * divu) + m->s_xi * divu;
        pi[3 * nc + c] = m->s_eta * (GU(c, 1, 2) + GU(c, 2, 1));
        pi[4 * nc + c] = m->s_eta * (GU(c, 1, 3) + GU(c, 3, 1));
        pi[5 * nc + c] = m->s_eta * (GU(c, 2, 3) + GU(c, 3, 2));
    }
#undef GU
}

/* stress.f90:86-105 */
static void stress_divergence(orc_model *m, const double *pi, double *f)
{
    static const int idx[3][3] = {{1, 4, 5}, {4, 2, 6}, {5, 6, 3}};
    orc_spec *spc = &m->spc;
    const long nc = NC(m);
    for (int i = 1; i <= 3; ++i) {
        if (i > spc->g.ndim) {
            memset(f + (i - 1) * nc, 0, sizeof(double) * nc);
            continue;
        }
        for (int j = 1; j <= 3; ++j)
            pcopy(m->tmpv + (j - 1) * nc, pi + (idx[i - 1][j - 1] - 1) * nc, nc);
        orc_spec_div(spc, m->tmpv, f + (i - 1) * nc);
    }
}

static void setup_term(orc_model *m, term_t *t)
{
    orc_spec *spc = &m->spc;
    const long nh = NH(m), nc = NC(m);
    switch (t->id) {
    case ORC_TERM_TF:
        t->alpha = dalloc(nc);
        break;
    case ORC_TERM_GRADIENT:
        t->lapn = dalloc(nc);
        t->gn = dalloc(3 * nc);
        break;
    case ORC_TERM_HARTREE:   /* fe_hartree.f90:34-44 */
        t->vk = dalloc(nh);
        t->w = dalloc(nc);
        for (long q = 0; q < nh; ++q) t->vk[q] = hartree_kernel(t, spc->g.kabs[q]);
        break;
    case ORC_TERM_RY:        /* fe_correlation_ry.f90:51-62 */
        t->ck = dalloc(nh);
        t->w = dalloc(nc);
        for (long q = 0; q < nh; ++q) t->ck[q] = ry_c_cor(m, t, spc->g.kabs[q]);
        break;
    }
}

/* model.f90:56-74 with species.f90:49-169 and external_potential.f90:39-63 */
orc_model *orc_model_create(const orc_params *pin, const orc_structure *st_in, int *status)
{
    orc_model *m = (orc_model *)calloc(1, sizeof(*m));
    m->p = *pin;
    orc_params *p = &m->p;
    int rc = 0;
    /* derived defaults of params_read (params.f90:161-172) */
    if (p->nterms == 0) {
        if (p->electron) {
            p->nterms = 4;
            p->terms[0] = ORC_TERM_TF; p->terms[1] = ORC_TERM_GRADIENT;
            p->terms[2] = ORC_TERM_HARTREE; p->terms[3] = ORC_TERM_RY;
        } else {
            p->nterms = 3;
            p->terms[0] = ORC_TERM_IDEAL; p->terms[1] = ORC_TERM_HARTREE; p->terms[2] = ORC_TERM_RY;
        }
    }
    if (p->electron && p->theta > 0.0) p->gamma = 2.0 * p->rs / (p->theta * pow(9.0 * PI / 4.0, 2.0 / 3.0));
    if (p->electron) p->kappa = 0.0;

    if (orc_spec_init(&m->spc, p->nx, p->ny, p->nz, p->lx, p->ly, p->lz, p->dealias)) { rc = 1; goto fail; }
    /* units.f90:41-70 */
    m->n0 = 3.0 / (4.0 * PI);
    m->e2 = 1.0 / 3.0;
    m->gamma = p->gamma; m->kappa = p->kappa; m->mass = p->mass;
    m->beta = 3.0 * p->gamma;
    m->kT = 1.0 / m->beta;
    m->rs = p->rs;
    if (p->electron) {
        m->quantum = 1;
        m->kappa = 0.0;
        m->hbar = 1.0 / sqrt(3.0 * p->rs);
        m->cn = SQRT2 / (PI * PI * pow(m->hbar, 3) * pow(m->beta, 1.5)) * pow(m->mass, 1.5);
        m->alpha0 = orc_fd_alpha_from_ip12(m->n0 / m->cn, NULL);
        double tf = m->hbar * m->hbar * pow(3.0 * PI * PI * m->n0, 2.0 / 3.0) / (2.0 * m->mass);
        m->theta = m->kT / tf;
        m->lambda_qsp = 2.0 * sqrt(PI * p->gamma / p->rs);
        m->lambda_tf = 1.0 / sqrt(4.0 * PI * m->e2 * m->beta * m->cn * 0.5 * orc_fd_im12(m->alpha0));
    } else {
        m->quantum = 0;
        m->hbar = 0.0;
        m->theta = DBL_MAX;
        m->lambda_tf = 1.0 / sqrt(3.0 * p->gamma);
    }
    /* structure (species.f90:80-101) */
    int need_deriv = p->maxwell && p->tau_ichimaru;
    int need_st = 0;
    for (int i = 0; i < p->nterms; ++i) if (p->terms[i] == ORC_TERM_RY) need_st = 1;
    if (need_deriv) need_st = 1;
    if (st_in) {
        orc_structure_set(&m->st, st_in->n, st_in->k, st_in->c, st_in->n0, st_in->u_ex,
                          st_in->du_dgamma, st_in->has_energy);
        m->has_st = 1;
    } else if (need_st) {
        orc_pot pot;
        memset(&pot, 0, sizeof(pot));
        pot.ksplit = 1.0;
        if (m->quantum) {
            pot.kind = ORC_POT_HM; pot.gamma = m->gamma; pot.kappa = 0.0;
            pot.lambda = m->lambda_qsp; pot.pauli = 1;
        } else {
            pot.kind = ORC_POT_YUKAWA; pot.gamma = m->gamma; pot.kappa = m->kappa; pot.lambda = 1.0;
        }
        if (orc_structure_from_hnc(&pot, m->n0, p->hnc_nr, p->hnc_rmax, p->hnc_tol, p->hnc_mix,
                                   p->hnc_maxiter, need_deriv, &m->st)) { rc = 2; goto fail; }
        m->has_st = 1;
    }
    /* functional terms (species.f90:104-151) */
    int has_hartree = 0;
    for (int i = 0; i < p->nterms; ++i) if (p->terms[i] == ORC_TERM_HARTREE) has_hartree = 1;
    m->nterms = p->nterms;
    for (int i = 0; i < p->nterms; ++i) {
        term_t *t = &m->terms[i];
        memset(t, 0, sizeof(*t));
        t->id = p->terms[i];
        t->n0 = m->n0; t->beta = m->beta;
        switch (t->id) {
        case ORC_TERM_TF:
            if (!m->quantum) { rc = 3; goto fail; }
            t->cn = m->cn; t->alpha0 = m->alpha0;
            break;
        case ORC_TERM_GRADIENT:
            if (!m->quantum) { rc = 3; goto fail; }
            t->cn = m->cn; t->alpha0 = m->alpha0;
            t->cg = p->tfk_gamma * (3.0 * SQRT2 * PI * PI / 8.0) * pow(m->hbar, 5) *
                    pow(m->beta, 1.5) / pow(m->mass, 2.5);
            break;
        case ORC_TERM_HARTREE:
            t->e2 = m->e2; t->kappa = m->kappa;
            break;
        case ORC_TERM_RY:
            if (!m->has_st) { rc = 3; goto fail; }
            t->e2 = m->e2; t->kappa = m->kappa;
            t->subtract_mean_field = has_hartree;
            break;
        }
        setup_term(m, t);
    }
    /* transport.f90:61-111 */
    switch (p->transport) {
    case ORC_TR_CONSTANT:
        m->tr_eta = p->eta; m->tr_xi = p->xi;
        break;
    case ORC_TR_YUKAWA_FIT: {
        double geff = m->gamma * (1.0 + m->kappa + 0.5 * m->kappa * m->kappa) * exp(-m->kappa);
        m->tr_eta = 0.482 / (geff * geff) + 0.629 / pow(geff, 0.878) + 1.88e-3 * geff;
        m->tr_xi = p->xi;
        break;
    }
    case ORC_TR_STANTON_MURILLO:
        if (m->quantum) { rc = 4; goto fail; }
        m->tr_eta = orc_sm_viscosity(m->gamma, m->kappa);
        m->tr_xi = p->xi;
        break;
    case ORC_TR_ELECTRON_FIT: {
        if (!m->quantum) { rc = 4; goto fail; }
        double el;
        orc_sm_electron_viscosity(m->rs, m->gamma, m->theta, m->lambda_tf, &el, NULL, NULL);
        m->tr_eta = 0.75 * el;
        m->tr_xi = 0.0;
        break;
    }
    }
    m->eta_l = 4.0 * m->tr_eta / 3.0 + m->tr_xi;
    m->tr_tau = 0.0;
    if (p->maxwell) {
        if (!p->tau_ichimaru) {
            m->tr_tau = p->tau;
        } else {
            if (!m->st.has_energy) { rc = 5; goto fail; }
            double u = m->st.u_ex, du = m->st.du_dgamma;
            double muc = u / 3.0 + m->gamma * du / 9.0;
            m->elastic_modulus = 1.0 - p->adiabatic_index * muc + 4.0 * u / 15.0;
            if (m->elastic_modulus <= 0.0) { rc = 5; goto fail; }
            m->tr_tau = 3.0 * m->gamma * m->eta_l / m->elastic_modulus;
        }
    }
    /* stress.f90:37-57 */
    if (p->maxwell) {
        m->evolve = m->tr_tau > 0.0;
        m->s_tau = m->tr_tau;
    } else {
        m->evolve = 0;
        m->s_tau = 0.0;
    }
    m->s_eta = m->tr_eta * m->n0;
    m->s_xi = m->tr_xi * m->n0;
    const long nc = NC(m);
    m->gu = dalloc(9 * nc);
    /* allocate_state (species.f90:155-169) */
    m->n = dalloc(nc);
    m->mom = dalloc(3 * nc);
    for (long q = 0; q < nc; ++q) m->n[q] = m->n0;
    if (m->evolve) m->pi = dalloc(6 * nc);
    /* vext_setup (external_potential.f90:39-63) */
    m->ext_kind = p->vext;
    m->ext_amp = p->vext_amplitude; m->ext_omega = p->vext_omega;
    m->ext_width = p->vext_width; m->ext_ramp = p->vext_ramp;
    m->ext_kvec[0] = TWOPI * p->vext_mode[0] / p->lx;
    m->ext_kvec[1] = TWOPI * p->vext_mode[1] / p->ly;
    m->ext_kvec[2] = TWOPI * p->vext_mode[2] / p->lz;
    if (p->ny == 1) m->ext_kvec[1] = 0.0;
    if (p->nz == 1) m->ext_kvec[2] = 0.0;
    m->ext_active = p->vext != ORC_VEXT_NONE;
    m->ext_time_dependent = p->vext == ORC_VEXT_DRIVEN;
    m->ext_v = dalloc(nc);
    m->ext_f = dalloc(3 * nc);
    if (m->ext_active) vext_eval(m, 0.0);
    /* work arrays (model.f90:66-71) */
    m->u = dalloc(3 * nc); m->mu = dalloc(nc); m->gmu = dalloc(3 * nc);
    m->flux = dalloc(3 * nc); m->divf = dalloc(nc);
    m->wpi = dalloc(6 * nc); m->pi0 = dalloc(6 * nc); m->pi0_old = dalloc(6 * nc);
    m->fpi = dalloc(3 * nc); m->gpi = dalloc(3 * nc);
    m->dn = dalloc(nc); m->dmom = dalloc(3 * nc); m->dpi = dalloc(6 * nc);
    m->dn_o = dalloc(nc); m->dmom_o = dalloc(3 * nc); m->dpi_o = dalloc(6 * nc);
    m->nhat = (orc_cplx *)calloc(NH(m), sizeof(orc_cplx));
    m->tmpv = dalloc(3 * nc);
    m->gtmp = dalloc(3 * nc);
    m->chat = (orc_cplx *)calloc(NH(m), sizeof(orc_cplx));
    m->t = 0.0; m->step = 0;
    m->dt = p->dt;
    if (status) *status = 0;
    return m;
fail:
    if (status) *status = rc;
    orc_model_destroy(m);
    return NULL;
}

void orc_model_destroy(orc_model *m)
{
    if (!m) return;
    for (int i = 0; i < m->nterms; ++i) {
        term_t *t = &m->terms[i];
        free(t->vk); free(t->ck); free(t->w); free(t->alpha); free(t->lapn); free(t->gn);
    }
    if (m->spc.fft) orc_spec_free(&m->spc);
    orc_structure_free(&m->st);
    free(m->gu); free(m->n); free(m->mom); free(m->pi); free(m->ext_v); free(m->ext_f);
    free(m->u); free(m->mu); free(m->gmu); free(m->flux); free(m->divf);
    free(m->wpi); free(m->pi0); free(m->pi0_old); free(m->fpi); free(m->gpi);
    free(m->dn); free(m->dmom); free(m->dpi); free(m->dn_o); free(m->dmom_o); free(m->dpi_o);
    free(m->nhat); free(m->tmpv); free(m->gtmp); free(m->chat);
    free(m);
}

/* model.f90:76-82 */
void orc_model_velocity(orc_model *m)
{
    const long nc = NC(m);
    for (int d = 0; d < 3; ++d)
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) m->u[d * nc + q] = m->mom[d * nc + q] / (m->mass * m->n[q]);
}

/* model.f90:85-146.  Returns nonzero where the reference is fatal. */
int orc_model_rhs(orc_model *m, double t, double *dn, double *dmom, double *dpi)
{
    orc_spec *spc = &m->spc;
    const long nc = NC(m);
    const int ndim = spc->g.ndim;
    if (min_nonpositive(m->n, nc)) return 20;
    orc_model_velocity(m);
    orc_spec_fwd(spc, m->n, m->nhat);
    /* continuity */
    orc_spec_div(spc, m->mom, dn);
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nc; ++q) dn[q] = -dn[q] / m->mass;
    /* chemical potential and its gradient */
    int rc = orc_model_mu_total(m, m->n, m->nhat, m->mu);
    if (rc) return rc;
    orc_spec_grad(spc, m->mu, m->gmu);
    /* external force */
    if (m->ext_active && m->ext_time_dependent) vext_eval(m, t);
    /* dissipative stress */
    if (m->evolve) pcopy(m->wpi, m->pi, 6 * nc);
    else stress_pi0(m, m->u, m->wpi);
    stress_divergence(m, m->wpi, m->fpi);
    /* momentum */
    for (int i = 1; i <= 3; ++i) {
        double *dm = dmom + (i - 1) * nc;
        if (i > ndim) {
            memset(dm, 0, sizeof(double) * nc);
            continue;
        }
        for (int j = 1; j <= 3; ++j)
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nc; ++q)
                m->flux[(j - 1) * nc + q] = m->mom[(i - 1) * nc + q] * m->u[(j - 1) * nc + q];
        orc_spec_div(spc, m->flux, m->divf);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) m->divf[q] = m->divf[q] + m->n[q] * m->gmu[(i - 1) * nc + q];
        double mean = orc_spec_mean(spc, m->divf);
#pragma omp parallel for schedule(static)
        for (long q = 0; q < nc; ++q) dm[q] = -(m->divf[q] - mean) + m->fpi[(i - 1) * nc + q];
        if (m->ext_active)
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nc; ++q) dm[q] = dm[q] + m->n[q] * m->ext_f[(i - 1) * nc + q];
    }
    /* stress advection */
    if (m->evolve) {
        for (int c = 0; c < 6; ++c) {
            orc_spec_grad(spc, m->pi + c * nc, m->gpi);
            double *dp = dpi + c * nc;
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nc; ++q) dp[q] = 0.0;
            for (int d = 0; d < ndim; ++d)
#pragma omp parallel for schedule(static)
                for (long q = 0; q < nc; ++q) dp[q] = dp[q] - m->u[d * nc + q] * m->gpi[d * nc + q];
        }
    }
    /* dealias */
    orc_spec_dealias(spc, dn);
    for (int i = 0; i < ndim; ++i) orc_spec_dealias(spc, dmom + i * nc);
    if (m->evolve)
        for (int c = 0; c < 6; ++c) orc_spec_dealias(spc, dpi + c * nc);
    return 0;
}

/* model.f90:150-183.  Returns nonzero where the reference is fatal. */
int orc_model_compute_dt(orc_model *m)
{
    orc_spec *spc = &m->spc;
    orc_grid *g = &spc->g;
    if (m->p.dt > 0.0) { m->dt = m->p.dt; return 0; }
    double wmax = 0.0;
    for (int l = 0; l < g->nz; ++l)
        for (int j = 0; j < g->ny; ++j)
            for (int i = 0; i < g->nkx; ++i) {
                long q = i + (long)g->nkx * (j + (long)g->ny * l);
                if (g->mask[q] == 0.0) continue;
                double k = g->kabs[q];
                if (k == 0.0) continue;
                double c2 = m->n0 * orc_model_kernel(m, k) / m->mass;
                if (m->evolve) c2 = c2 + m->eta_l / (m->mass * m->s_tau);
                double kk = k * k * (c2 > 0.0 ? c2 : 0.0);
                double w = sqrt(kk);
                if (w > wmax) wmax = w;
            }
    double numax = 0.0;
    if (!m->evolve) numax = m->eta_l / m->mass * g->kmax_dealiased * g->kmax_dealiased;
    orc_model_velocity(m);
    double umax = 0.0;
    for (long q = 0; q < 3 * NC(m); ++q) if (fabs(m->u[q]) > umax) umax = fabs(m->u[q]);
    double dxmin = g->dx;
    if (g->ny > 1 && g->dy < dxmin) dxmin = g->dy;
    if (g->nz > 1 && g->dz < dxmin) dxmin = g->dz;
    double dtm = DBL_MAX;
    if (wmax > 0.0 && 1.7 / wmax < dtm) dtm = 1.7 / wmax;
    if (numax > 0.0 && 2.5 / numax < dtm) dtm = 2.5 / numax;
    if (umax > 0.0 && dxmin / umax < dtm) dtm = dxmin / umax;
    if (dtm == DBL_MAX) return 30;
    m->dt = m->p.cfl * dtm;
    return 0;
}

static const double RK_A[3] = {32.0 / 60.0, 25.0 / 60.0, 45.0 / 60.0};
static const double RK_B[3] = {0.0, -17.0 / 60.0, -25.0 / 60.0};

/* one pass of the stage loop of model.f90:186-227 (s = 0, 1, 2); stage 0
 * starts the step at t, stage 2 finishes it */
int orc_model_stage(orc_model *m, int s)
{
    orc_spec *spc = &m->spc;
    const long nc = NC(m);
    const int ndim = spc->g.ndim;
    if (s < 0 || s > 2) return 99;
    if (s == 0) m->ts = m->t;
    double ts = m->ts;
    {
        int rc = orc_model_rhs(m, ts, m->dn, m->dmom, m->dpi);
        if (rc) return rc;
        if (m->evolve) stress_pi0(m, m->u, m->pi0_old);
        const double dt = m->dt;
        if (s == 0) {
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nc; ++q) m->n[q] = m->n[q] + dt * RK_A[0] * m->dn[q];
#pragma omp parallel for schedule(static)
            for (long q = 0; q < 3 * nc; ++q) m->mom[q] = m->mom[q] + dt * RK_A[0] * m->dmom[q];
            if (m->evolve)
#pragma omp parallel for schedule(static)
                for (long q = 0; q < 6 * nc; ++q) m->pi[q] = m->pi[q] + dt * RK_A[0] * m->dpi[q];
        } else {
#pragma omp parallel for schedule(static)
            for (long q = 0; q < nc; ++q) m->n[q] = m->n[q] + dt * (RK_A[s] * m->dn[q] + RK_B[s] * m->dn_o[q]);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < 3 * nc; ++q)
                m->mom[q] = m->mom[q] + dt * (RK_A[s] * m->dmom[q] + RK_B[s] * m->dmom_o[q]);
            if (m->evolve)
#pragma omp parallel for schedule(static)
                for (long q = 0; q < 6 * nc; ++q)
                    m->pi[q] = m->pi[q] + dt * (RK_A[s] * m->dpi[q] + RK_B[s] * m->dpi_o[q]);
        }
        pcopy(m->dn_o, m->dn, nc);
        pcopy(m->dmom_o, m->dmom, 3 * nc);
        if (m->evolve) pcopy(m->dpi_o, m->dpi, 6 * nc);
        double dts = (RK_A[s] + RK_B[s]) * dt;
        ts = ts + dts;
        if (m->evolve) {
            orc_model_velocity(m);
            stress_pi0(m, m->u, m->pi0);
            double fac = exp(-dts / m->s_tau);
            double phi = (m->s_tau / dts) * (1.0 - fac);
#pragma omp parallel for schedule(static)
            for (long q = 0; q < 6 * nc; ++q)
                m->pi[q] = m->pi0[q] - (m->pi0[q] - m->pi0_old[q]) * phi + (m->pi[q] - m->pi0_old[q]) * fac;
            for (int c = 0; c < 6; ++c) orc_spec_dealias(spc, m->pi + c * nc);
        }
        orc_spec_dealias(spc, m->n);
        for (int i = 0; i < ndim; ++i) orc_spec_dealias(spc, m->mom + i * nc);
    }
    m->ts = ts;
    if (s == 2) {
        m->t = m->t + m->dt;
        m->step = m->step + 1;
    }
    return 0;
}

/* model.f90:186-227 */
int orc_model_advance(orc_model *m)
{
    for (int s = 0; s < 3; ++s) {
        int rc = orc_model_stage(m, s);
        if (rc) return rc;
    }
    return 0;
}

/* initial.f90:23-75 for 'uniform' (kind 0), 'mode' (1) and 'gaussian' (3).
 * 'random' (2) depends on gfortran's intrinsic generator and is not
 * restated; tests inject seeded arrays instead. */
int orc_model_set_ic(orc_model *m, int kind, double amp, const int mode[3], double width)
{
    orc_spec *spc = &m->spc;
    orc_grid *g = &spc->g;
    const long nc = NC(m);
    double *d = dalloc(nc);
    memset(m->mom, 0, sizeof(double) * 3 * nc);
    if (m->pi) memset(m->pi, 0, sizeof(double) * 6 * nc);
    if (kind == 1) {
        double kv[3] = {TWOPI * mode[0] / g->lx, TWOPI * mode[1] / g->ly, TWOPI * mode[2] / g->lz};
        if (g->ny == 1) kv[1] = 0.0;
        if (g->nz == 1) kv[2] = 0.0;
        for (int k = 0; k < g->nz; ++k)
            for (int j = 0; j < g->ny; ++j)
                for (int i = 0; i < g->nx; ++i) {
                    double ph = kv[0] * g->x[i] + kv[1] * g->y[j] + kv[2] * g->z[k];
                    d[i + (long)g->nx * (j + (long)g->ny * k)] = cos(ph);
                }
    } else if (kind == 3) {
        for (int k = 0; k < g->nz; ++k)
            for (int j = 0; j < g->ny; ++j)
                for (int i = 0; i < g->nx; ++i) {
                    double x = g->x[i] - 0.5 * g->lx, y = 0.0, z = 0.0;
                    if (g->ny > 1) y = g->y[j] - 0.5 * g->ly;
                    if (g->nz > 1) z = g->z[k] - 0.5 * g->lz;
                    d[i + (long)g->nx * (j + (long)g->ny * k)] = exp(-0.5 * (x * x + y * y + z * z) / (width * width));
                }
        orc_spec_dealias(spc, d);
        double mean = orc_spec_mean(spc, d);
        for (long q = 0; q < nc; ++q) d[q] -= mean;
    } else if (kind != 0) {
        free(d);
        return 40;
    }
    for (long q = 0; q < nc; ++q) m->n[q] = m->n0 * (1.0 + amp * d[q]);
    free(d);
    if (min_nonpositive(m->n, nc)) return 41;
    return 0;
}

/* diagnostics.f90:41-60 */
void orc_model_budgets(orc_model *m, double *mass, double mom[3], double *ekin, double *fe)
{
    orc_spec *spc = &m->spc;
    const long nc = NC(m);
    const double v = spc->g.volume;
    *mass = orc_spec_mean(spc, m->n) * v;
    for (int i = 0; i < 3; ++i) mom[i] = orc_spec_mean(spc, m->mom + i * nc) * v;
    double ek = 0.0;
    double *tmp = dalloc(nc);
    for (int i = 0; i < spc->g.ndim; ++i) {
        for (long q = 0; q < nc; ++q) tmp[q] = m->mom[i * nc + q] * m->mom[i * nc + q] / m->n[q];
        ek += orc_spec_mean(spc, tmp);
    }
    *ekin = 0.5 * ek * v / m->mass;
    orc_spec_fwd(spc, m->n, m->nhat);
    *fe = orc_model_energy(m, m->n, m->nhat);
    if (m->ext_active) {
        for (long q = 0; q < nc; ++q) tmp[q] = m->n[q] * m->ext_v[q];
        *fe += orc_spec_mean(spc, tmp) * v;
    }
    free(tmp);
}

/* ---------------------------------------------------- accessors */
int orc_model_ncells(const orc_model *m) { return (int)NC(m); }
int orc_model_has_pi(const orc_model *m) { return m->evolve; }
double *orc_model_n(orc_model *m) { return m->n; }
double *orc_model_mom(orc_model *m) { return m->mom; }
double *orc_model_pi(orc_model *m) { return m->pi; }
double *orc_model_mu(orc_model *m) { return m->mu; }
double *orc_model_vext_v(orc_model *m) { return m->ext_v; }
orc_spec *orc_model_spec(orc_model *m) { return &m->spc; }
long orc_model_fft_count(const orc_model *m) { return orc_fft3_count(m->spc.fft); }
int orc_model_nterms(const orc_model *m) { return m->nterms; }
int orc_model_term_id(const orc_model *m, int i) { return m->terms[i].id; }

double orc_model_get(const orc_model *m, const char *k)
{
    if (!strcmp(k, "t")) return m->t;
    if (!strcmp(k, "dt")) return m->dt;
    if (!strcmp(k, "step")) return m->step;
    if (!strcmp(k, "n0")) return m->n0;
    if (!strcmp(k, "beta")) return m->beta;
    if (!strcmp(k, "gamma")) return m->gamma;
    if (!strcmp(k, "kappa")) return m->kappa;
    if (!strcmp(k, "mass")) return m->mass;
    if (!strcmp(k, "hbar")) return m->hbar;
    if (!strcmp(k, "theta")) return m->theta;
    if (!strcmp(k, "alpha0")) return m->alpha0;
    if (!strcmp(k, "cn")) return m->cn;
    if (!strcmp(k, "lambda_qsp")) return m->lambda_qsp;
    if (!strcmp(k, "lambda_tf")) return m->lambda_tf;
    if (!strcmp(k, "eta")) return m->tr_eta;
    if (!strcmp(k, "xi")) return m->tr_xi;
    if (!strcmp(k, "tau")) return m->s_tau;
    if (!strcmp(k, "eta_l")) return m->eta_l;
    if (!strcmp(k, "stress_eta")) return m->s_eta;
    if (!strcmp(k, "stress_xi")) return m->s_xi;
    if (!strcmp(k, "evolve")) return m->evolve;
    if (!strcmp(k, "u_ex")) return m->st.u_ex;
    if (!strcmp(k, "du_dgamma")) return m->st.du_dgamma;
    if (!strcmp(k, "kmax_dealiased")) return m->spc.g.kmax_dealiased;
    if (!strcmp(k, "volume")) return m->spc.g.volume;
    if (!strcmp(k, "ext_omega")) return m->ext_omega;
    if (!strcmp(k, "cg")) {
        for (int i = 0; i < m->nterms; ++i) if (m->terms[i].id == ORC_TERM_GRADIENT) return m->terms[i].cg;
        return 0.0;
    }
    if (!strcmp(k, "st_n")) return m->st.n;
    return NAN;
}

void orc_model_set(orc_model *m, const char *k, double v)
{
    if (!strcmp(k, "t")) m->t = v;
    else if (!strcmp(k, "dt")) m->dt = v;
    else if (!strcmp(k, "ext_omega")) m->ext_omega = v;
    else if (!strcmp(k, "step")) m->step = (int)v;
}

/* -------------------------------------------------- linear response */
/* linear_response.f90:59-63 */
double orc_linear_c2(const orc_model *m, double k) { return m->n0 * orc_model_kernel(m, k) / m->mass; }

static orc_cplx lin_den(const orc_model *m, double k, orc_cplx w)
{
    return -w * w + k * k * orc_linear_c2(m, k) -
           I * k * k * (m->eta_l / m->mass) * w / (1.0 - I * w * m->s_tau);
}

/* :72-76 */
orc_cplx orc_linear_chi(const orc_model *m, double k, double w)
{
    return -k * k * m->n0 / lin_den(m, k, w + 0.0 * I);
}

static orc_cplx poly(const orc_cplx *a, int deg, orc_cplx x)
{
    orc_cplx p = a[deg];
    for (int q = deg - 1; q >= 0; --q) p = p * x + a[q];
    return p;
}

static orc_cplx dpoly(const orc_cplx *a, int deg, orc_cplx x)
{
    orc_cplx p = deg * a[deg];
    for (int q = deg - 1; q >= 1; --q) p = p * x + q * a[q];
    return p;
}

/* :82-147 */
orc_cplx orc_linear_dispersion(const orc_model *m, double k)
{
    orc_cplx a[4], z[3], zn[3];
    int deg;
    double c2k2 = k * k * orc_linear_c2(m, k);
    double nu = k * k * m->eta_l / m->mass;
    double tau = m->s_tau;
    if (tau > 0.0) {
        deg = 3;
        a[3] = -I * tau; a[2] = 1.0; a[1] = I * (nu + c2k2 * tau); a[0] = -c2k2;
    } else {
        deg = 2;
        a[2] = 1.0; a[1] = I * nu; a[0] = -c2k2;
        a[3] = 0.0;
    }
    z[0] = 0.4 + 0.9 * I; z[1] = z[0] * z[0]; z[2] = z[0] * z[0] * z[0];
    for (int it = 1; it <= 500; ++it) {
        for (int i = 0; i < deg; ++i) {
            orc_cplx num = poly(a, deg, z[i]);
            orc_cplx den = a[deg];
            for (int j = 0; j < deg; ++j) if (j != i) den = den * (z[i] - z[j]);
            zn[i] = z[i] - num / den;
        }
        double dmax = 0.0, zmax = 0.0;
        for (int i = 0; i < deg; ++i) {
            if (cabs(zn[i] - z[i]) > dmax) dmax = cabs(zn[i] - z[i]);
            if (cabs(zn[i]) > zmax) zmax = cabs(zn[i]);
        }
        for (int i = 0; i < deg; ++i) z[i] = zn[i];
        if (dmax < 1.0e-15 * (zmax > 1.0 ? zmax : 1.0)) break;
    }
    for (int i = 0; i < deg; ++i)
        for (int it = 0; it < 5; ++it) z[i] = z[i] - poly(a, deg, z[i]) / dpoly(a, deg, z[i]);
    orc_cplx w = z[0];
    for (int i = 1; i < deg; ++i) if (creal(z[i]) > creal(w)) w = z[i];
    return w;
}

/* :152-171 */
double orc_linear_dsf(const orc_model *m, double k, double w)
{
    double ratio;
    if (fabs(w) < 1.0e-6) {
        double c2 = orc_linear_c2(m, k);
        ratio = m->n0 * m->eta_l / (m->mass * c2 * c2);
    } else {
        ratio = -cimag(orc_linear_chi(m, k, w)) / w;
    }
    if (m->quantum) {
        double x = m->beta * m->hbar * w;
        if (fabs(x) < 1.0e-6) return ratio / (PI * m->n0 * m->beta * m->hbar) * (1.0 + 0.5 * x);
        return ratio / (PI * m->n0 * m->beta * m->hbar) * x / (1.0 - exp(-x));
    }
    return ratio / (PI * m->n0 * m->beta);
}

/* ------------------------------------------------------------ analysis */
/* analysis.f90:21-74 */
void orc_fit_damped_mode(int n, const double *t, const double *y, double t_start, double *omega,
                         double *gamma, int *nzeros)
{
    double *tz = dalloc(n), *tp = dalloc(n), *lp = dalloc(n);
    int i0 = 1;
    while (i0 < n && t[i0 - 1] < t_start) i0++;
    int nz = 0;
    for (int i = i0; i <= n - 1; ++i) {
        if (y[i - 1] == 0.0) continue;
        if (y[i - 1] * y[i] < 0.0) {
            double w = y[i - 1] / (y[i - 1] - y[i]);
            tz[nz++] = t[i - 1] + w * (t[i] - t[i - 1]);
        }
    }
    *nzeros = nz;
    *omega = 0.0; *gamma = 0.0;
    if (nz >= 3) {
        *omega = PI * (nz - 1) / (tz[nz - 1] - tz[0]);
        int np = 0;
        for (int i = 0; i < nz - 1; ++i) {
            double ta = tz[i], tb = tz[i + 1], ymax = 0.0, tmax = 0.5 * (ta + tb);
            for (int j = 0; j < n; ++j)
                if (t[j] > ta && t[j] < tb && fabs(y[j]) > ymax) { ymax = fabs(y[j]); tmax = t[j]; }
            if (ymax > 0.0) { tp[np] = tmax; lp[np] = log(ymax); np++; }
        }
        if (np >= 2) {
            double sx = 0, sy = 0, sxx = 0, sxy = 0;
            for (int i = 0; i < np; ++i) { sx += tp[i]; sy += lp[i]; sxx += tp[i] * tp[i]; sxy += tp[i] * lp[i]; }
            *gamma = (np * sxy - sx * sy) / (np * sxx - sx * sx);
        }
    }
    free(tz); free(tp); free(lp);
}

/* analysis.f90:78-98 */
void orc_fit_driven_response(int n, const double *t, const orc_cplx *z, double w, double t_start,
                             orc_cplx *a, double *scatter)
{
    orc_cplx s = 0.0;
    int cnt = 0;
    for (int i = 0; i < n; ++i)
        if (t[i] >= t_start) { s += z[i] * cexp(I * w * t[i]); cnt++; }
    *a = s / (cnt > 1 ? cnt : 1);
    double dev = 0.0;
    for (int i = 0; i < n; ++i)
        if (t[i] >= t_start) {
            double d = cabs(z[i] * cexp(I * w * t[i]) - *a);
            if (d > dev) dev = d;
        }
    double den = cabs(*a) > DBL_MIN ? cabs(*a) : DBL_MIN;
    *scatter = dev / den;
}
