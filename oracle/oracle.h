/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, single-process restatement of the HyDFT nonlinear
 * pseudo-spectral solver step (abdoudiaw/HyDFT, Fortran 2018) and of the setup
 * pieces it depends on.  It exists to check the CUDA product path: only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * it, and only as the reference the device results are compared with.
 * Nothing in the product links or calls it.
 *
 * It follows the reference's operator sequence literally (every spectral
 * operator does its own FFT round trip, exactly as src/core/spectral.f90 does),
 * so it reproduces the reference's 189/201/369 transforms per step.  The only
 * external dependency of the reference, FFTW3 (unpinned, found by
 * cmake/FindFFTW.cmake), is replaced by fft.c: a mixed-radix Stockham complex
 * FFT written from the textbook algorithm, wrapped with FFTW's r2c/c2r
 * half-spectrum semantics and RODFT00 (DST-I) definition.
 *
 * Parity pins: the reference's own known-answer tests (test/test_fft.f90,
 * test_ops.f90, test_kernels.f90, test_fermi_dirac.f90, test_hnc.f90,
 * test_conservation.f90, test_mode_*.f90, test_driven_mode.f90,
 * test_ground_state.f90) are restated against this oracle in tests/ with the
 * reference's thresholds.  The reference itself cannot be compiled here (no
 * Fortran compiler, no FFTW), so there are no reference-run trajectories.
 *
 * Array layout is the reference's Fortran order: a real field u(nx,ny,nz) is
 * u[i + nx*(j + ny*k)], a half spectrum uhat(nkx,ny,nz) is
 * uhat[i + nkx*(j + ny*k)], a vector field v(nx,ny,nz,3) is 3 fields back to
 * back.
 */
#ifndef HYDFT_ORACLE_H
#define HYDFT_ORACLE_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex orc_cplx;

/* ------------------------------------------------------------------ FFT */
/* 1-D complex transform plan (any length; radices 4,2,3,5 and a generic
 * prime butterfly).  sign = -1 forward, +1 backward, unnormalised. */
typedef struct orc_fft1 orc_fft1;
orc_fft1 *orc_fft1_create(int n);
void orc_fft1_destroy(orc_fft1 *p);
void orc_fft1_exec(orc_fft1 *p, orc_cplx *data, int sign);
void orc_fft1_c(int n, orc_cplx *data, int sign);       /* one-shot */

/* 3-D r2c / c2r with FFTW's conventions as used by src/core/fft.f90:
 * forward normalised by 1/(nx ny nz) (fft.f90:56-58), backward
 * unnormalised (fft.f90:62-69).  Input of c2r is preserved. */
typedef struct orc_fft3 orc_fft3;
orc_fft3 *orc_fft3_create(int nx, int ny, int nz);
void orc_fft3_destroy(orc_fft3 *f);
void orc_fft3_fwd(orc_fft3 *f, const double *u, orc_cplx *uhat);
void orc_fft3_bwd(orc_fft3 *f, const orc_cplx *uhat, double *u);
long orc_fft3_count(const orc_fft3 *f);   /* transforms executed */

/* FFTW_RODFT00 (DST-I): y_k = 2 sum_j x_j sin(pi (j+1)(k+1)/(n+1)). */
typedef struct orc_dst1 orc_dst1;
orc_dst1 *orc_dst1_create(int n);
void orc_dst1_destroy(orc_dst1 *d);
void orc_dst1_exec(orc_dst1 *d, const double *x, double *y);

/* ------------------------------------------------------------ grid/spec */
typedef struct {
    int nx, ny, nz, nkx, ndim;
    double lx, ly, lz, dx, dy, dz, volume;
    double *x, *y, *z, *kx, *ky, *kz;
    double *k2, *kabs, *mask;          /* (nkx,ny,nz) */
    double kmax_dealiased;
} orc_grid;

typedef struct {
    orc_grid g;
    orc_fft3 *fft;
    orc_cplx *w1, *w2;
} orc_spec;

int orc_spec_init(orc_spec *s, int nx, int ny, int nz, double lx, double ly,
                  double lz, int dealias);
void orc_spec_free(orc_spec *s);
void orc_spec_fwd(orc_spec *s, const double *u, orc_cplx *uhat);
void orc_spec_bwd(orc_spec *s, const orc_cplx *uhat, double *u);
void orc_spec_grad_hat(orc_spec *s, const orc_cplx *uhat, int idir, double *du);
void orc_spec_grad(orc_spec *s, const double *u, double *du);   /* du: 3 fields */
void orc_spec_lap(orc_spec *s, const double *u, double *lu);
void orc_spec_div(orc_spec *s, const double *v, double *dv);    /* v: 3 fields */
void orc_spec_convolve(orc_spec *s, const double *kern, const orc_cplx *uhat, double *cu);
void orc_spec_dealias(orc_spec *s, double *u);
double orc_spec_mean(const orc_spec *s, const double *u);
orc_cplx orc_spec_mode(orc_spec *s, const double *u, int mx, int my, int mz);

/* ---------------------------------------------------------- Fermi-Dirac */
void orc_gauss_legendre(int n, double *x, double *w);
void orc_fd_init(void);
const double *orc_fd_table(int *ntab);   /* tab[6*i + c], c = column-1 */
double orc_fd_im12(double a);
double orc_fd_ip12(double a);
double orc_fd_ip32(double a);
double orc_fd_dim12(double a);
double orc_fd_d2im12(double a);
double orc_fd_xi(double a);
double orc_fd_dxi(double a);
double orc_fd_alpha_from_ip12(double y, int *status);

/* ------------------------------------------------------ pair potentials */
enum { ORC_POT_YUKAWA = 0, ORC_POT_COULOMB = 1, ORC_POT_HM = 2 };
typedef struct {
    int kind;
    double gamma, kappa, ksplit, lambda;
    int pauli;
} orc_pot;
double orc_pot_beta_v(const orc_pot *p, double r);
double orc_pot_beta_v_long_r(const orc_pot *p, double r);
double orc_pot_beta_v_long_k(const orc_pot *p, double k);
double orc_pot_beta_v_short(const orc_pot *p, double r);
double orc_pot_beta_v_k(const orc_pot *p, double k);

/* ------------------------------------------------------------ OZ-HNC */
typedef struct {
    int nr;
    double n0, dr, dk;
    double *r, *k, *g, *cr, *ck, *hk, *sk;
    double u_ex;
    int converged, niter;
    double residual;
} orc_hnc_result;

void orc_fb_r2k(int n, double rmax, const double *fr, double *fk);
void orc_fb_k2r(int n, double rmax, const double *fk, double *fr);
/* returns 0 on success; nonzero mirrors the reference's fatal paths */
int orc_hnc_solve(const orc_pot *pot, double n0, int nr, double rmax, double tol,
                  double mix, int maxiter, orc_hnc_result *res);
void orc_hnc_result_free(orc_hnc_result *res);

typedef struct {
    int n;                 /* table length; 0 = no structure */
    double n0;
    double *k, *c, *s;
    double u_ex, du_dgamma;
    int has_energy;
} orc_structure;
int orc_structure_from_hnc(orc_pot *pot, double n0, int nr, double rmax, double tol,
                           double mix, int maxiter, int with_derivative,
                           orc_structure *st);
void orc_structure_set(orc_structure *st, int n, const double *k, const double *c,
                       double n0, double u_ex, double du_dgamma, int has_energy);
double orc_structure_c_of_k(const orc_structure *st, double k);
void orc_structure_free(orc_structure *st);
double orc_interp_linear(int n, const double *x, const double *y, double xq);

/* ------------------------------------------------------------ params */
enum { ORC_TERM_IDEAL = 1, ORC_TERM_TF = 2, ORC_TERM_GRADIENT = 3,
       ORC_TERM_HARTREE = 4, ORC_TERM_RY = 5 };
enum { ORC_VEXT_NONE = 0, ORC_VEXT_MODE = 1, ORC_VEXT_DRIVEN = 2, ORC_VEXT_GAUSSIAN = 3 };
enum { ORC_TR_CONSTANT = 0, ORC_TR_YUKAWA_FIT = 1, ORC_TR_STANTON_MURILLO = 2,
       ORC_TR_ELECTRON_FIT = 3 };

typedef struct {
    int nx, ny, nz;
    double lx, ly, lz;
    int dealias;
    int electron;                 /* kind: 0 ion, 1 electron */
    double gamma, kappa, rs, theta, mass;
    int nterms, terms[8];         /* ordered term list */
    double tfk_gamma;
    int maxwell;                  /* closure */
    int transport;                /* ORC_TR_* */
    double eta, xi, tau;
    int tau_ichimaru;             /* tau_model: 1 ichimaru, 0 constant */
    double adiabatic_index;
    int hnc_nr, hnc_maxiter;
    double hnc_rmax, hnc_tol, hnc_mix;
    double dt, cfl;
    int vext;
    double vext_amplitude, vext_omega, vext_width, vext_ramp;
    int vext_mode[3];
} orc_params;

void orc_params_default(orc_params *p);

/* ------------------------------------------------------------ model */
typedef struct orc_model orc_model;
/* st may be NULL: then the structure comes from HNC as in species_build. */
orc_model *orc_model_create(const orc_params *p, const orc_structure *st, int *status);
void orc_model_destroy(orc_model *m);
int orc_model_rhs(orc_model *m, double t, double *dn, double *dmom, double *dpi);
int orc_model_compute_dt(orc_model *m);
int orc_model_advance(orc_model *m);
/* stage s (0, 1, 2) of one RK3 step alone: three calls in order = advance */
int orc_model_stage(orc_model *m, int s);
void orc_model_velocity(orc_model *m);
int orc_model_set_ic(orc_model *m, int kind, double amp, const int mode[3], double width);

/* state and scalars */
int orc_model_ncells(const orc_model *m);
int orc_model_has_pi(const orc_model *m);
double *orc_model_n(orc_model *m);
double *orc_model_mom(orc_model *m);
double *orc_model_pi(orc_model *m);     /* NULL unless maxwell with tau > 0 */
double *orc_model_mu(orc_model *m);     /* work: mu of the last rhs */
double *orc_model_vext_v(orc_model *m);
double orc_model_get(const orc_model *m, const char *name);
void orc_model_set(orc_model *m, const char *name, double v);
orc_spec *orc_model_spec(orc_model *m);
long orc_model_fft_count(const orc_model *m);

/* functional on an arbitrary density (test_kernels / test_ground_state) */
int orc_model_nterms(const orc_model *m);
int orc_model_term_id(const orc_model *m, int i);
int orc_model_term_add_mu(orc_model *m, int i, const double *n, const orc_cplx *nhat, double *mu);
double orc_model_term_kernel(const orc_model *m, int i, double k);
double orc_model_kernel(const orc_model *m, double k);
int orc_model_mu_total(orc_model *m, const double *n, const orc_cplx *nhat, double *mu);
double orc_model_energy(orc_model *m, const double *n, const orc_cplx *nhat);

/* diagnostics (diagnostics.f90:41-60) */
void orc_model_budgets(orc_model *m, double *mass, double mom[3], double *ekin, double *fe);

/* linear response (linear_response.f90) */
double orc_linear_c2(const orc_model *m, double k);
orc_cplx orc_linear_chi(const orc_model *m, double k, double w);
orc_cplx orc_linear_dispersion(const orc_model *m, double k);
double orc_linear_dsf(const orc_model *m, double k, double w);

/* analysis (analysis.f90) */
void orc_fit_damped_mode(int n, const double *t, const double *y, double t_start,
                         double *omega, double *gamma, int *nzeros);
void orc_fit_driven_response(int n, const double *t, const orc_cplx *z, double w,
                             double t_start, orc_cplx *a, double *scatter);

/* transport fits (stanton_murillo.f90) */
double orc_sm_knm(int idx, double g);
double orc_sm_viscosity(double gamma, double kappa);
double orc_sm_diffusion(double gamma, double kappa);
double orc_sm_conductivity(double gamma, double kappa);
void orc_sm_electron_viscosity(double rs, double gamma, double theta, double lambda_tf,
                               double *eta_l, double *eta_cv, double *eta_sm);

/* OpenMP threads used by the oracle (1 = the reference's serial path) */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
