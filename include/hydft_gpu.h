/*
 * hydft_gpu.h -- C ABI of the B200 (sm_100a) implementation of HyDFT's
 * nonlinear pseudo-spectral solver step.
 *
 * The library replaces `model_t%advance` / `model_t%rhs` of HyDFT
 * (src/model/model.f90:85-227) and the setup it depends on (species build,
 * OZ-HNC c(k), Fermi-Dirac tables).  Every entry point is `extern "C"`,
 * takes plain pointers and sizes, returns an int status (HYDFT_OK = 0) and
 * never aborts: where the reference calls `fatal` (src/core/kinds.f90:26-30)
 * the library returns a non-zero code and hydft_gpu_last_error() gives the
 * message, so a Fortran shim can keep the reference's behaviour by calling
 * `fatal` itself.
 *
 * Field arrays on the host use the reference's Fortran order: n(nx,ny,nz)
 * with x fastest; mom(nx,ny,nz,3) and pi(nx,ny,nz,6) with the component index
 * slowest (Pi components xx,yy,zz,xy,xz,yz as in src/closure/stress.f90:7).
 *
 * One handle belongs to one host thread; calls on it are not re-entrant.
 */
#ifndef HYDFT_GPU_H
#define HYDFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    HYDFT_OK = 0,
    HYDFT_ERR_BAD_ARG = 1,             /* invalid parameter or size */
    HYDFT_ERR_OOM = 2,                 /* device allocation failed */
    HYDFT_ERR_NONPOSITIVE_DENSITY = 3, /* model.f90:91, fe_*.f90 positivity checks */
    HYDFT_ERR_NONFINITE = 4,           /* NaN/Inf in the state */
    HYDFT_ERR_NEWTON = 5,              /* Fermi-Dirac inverse did not converge */
    HYDFT_ERR_TIMEOUT = 6,             /* a bounded device wait ran out */
    HYDFT_ERR_CUDA = 7,                /* CUDA runtime error */
    HYDFT_ERR_UNSUPPORTED = 8,         /* option the GPU path does not implement */
    HYDFT_ERR_HNC = 9,                 /* structure: HNC failed (structure_source.f90:63) */
    HYDFT_ERR_IO = 10,                 /* cannot read an input file */
    HYDFT_ERR_CFL = 11                 /* compute_dt cannot determine a step (model.f90:180) */
};

/*
 * Run-time parameters: the reference's params_t (src/core/params.f90:17-78)
 * as a POD struct.  Strings are NUL-terminated, lower case.  Fields of the
 * namelists the solver step does not use (&linear, &output) are kept so the
 * struct round-trips an input file.  `gpu_precision` is new ("fp64" or
 * "fp32"), read from an optional &gpu namelist that the reference ignores.
 */
typedef struct hydft_params {
    /* &grid */
    int nx, ny, nz;
    double lx, ly, lz;
    int dealias;
    /* &species */
    char kind[16];            /* "ion" | "electron" */
    double gamma, kappa, rs, theta, mass;
    char terms[64];           /* comma list of ideal, tf, gradient, hartree, ry */
    double tfk_gamma;
    char closure[16];         /* "newtonian" | "maxwell" */
    char transport[16];       /* "constant" | "yukawa_fit" | "stanton_murillo" | "electron_fit" */
    double eta, xi, tau;
    char tau_model[16];       /* "ichimaru" | "constant" */
    double adiabatic_index;
    char structure[16];       /* "hnc" | "file" | "none" */
    char structure_file[256];
    char structure_kind[4];   /* "s" | "c" */
    /* &hnc */
    int hnc_nr, hnc_maxiter;
    double hnc_rmax, hnc_tol, hnc_mix;
    /* &time */
    double dt, cfl, tend;
    int nsteps_max, iout, iprobe, idiag;
    /* &initial */
    char ic[16];
    double ic_amplitude;
    int ic_mode[3];
    double ic_width;
    int ic_seed;
    /* &external */
    char vext[16];            /* "none" | "mode" | "driven" | "gaussian" */
    double vext_amplitude;
    int vext_mode[3];
    double vext_omega, vext_width, vext_ramp;
    /* &probe */
    int probe_mode[3];
    /* &output */
    char prefix[256];
    /* &gpu (new) */
    char gpu_precision[8];    /* "fp64" | "fp32" */
} hydft_params;

/* Defaults of params_t (src/core/params.f90:17-78) and "fp64". */
int hydft_params_default(hydft_params *p);

/* params_t%read (src/core/params.f90:82-180): read the namelists from
 * `path` over the values already in *p, then apply the derived defaults
 * (terms per kind, Gamma from rs and theta, kappa = 0 for electrons). */
int hydft_params_read(const char *path, hydft_params *p);

/* The derived defaults of params_read (params.f90:161-172) alone, for
 * callers that fill the struct in code as the reference's tests do. */
int hydft_params_finalize(hydft_params *p);

/* An optional structure table c(k) on increasing k > 0 that replaces the
 * HNC solve (the 'file' source, structure_source.f90:87-138, or a table
 * computed elsewhere).  u_ex / du_dgamma feed tau_model = 'ichimaru'. */
typedef struct hydft_structure {
    int n;
    const double *k;
    const double *c;
    double u_ex, du_dgamma;
    int has_energy;
} hydft_structure;

typedef struct hydft_gpu hydft_gpu;

/*
 * model_t%init (src/model/model.f90:56-74): grid, species build (units,
 * structure, functional terms, transport, stress closure), state allocation
 * (n = n0, mom = 0, Pi = 0) and the external potential.  With st == NULL
 * and p->structure == "hnc" the OZ-HNC equation is solved on the GPU in
 * FP64.  `device` selects the CUDA device.
 */
int hydft_gpu_create(const hydft_params *p, const hydft_structure *st, int device,
                     hydft_gpu **out);
void hydft_gpu_destroy(hydft_gpu *h);
const char *hydft_gpu_last_error(const hydft_gpu *h);
/* message of the last failed hydft_gpu_create on this thread */
const char *hydft_gpu_create_error(void);

/* Copy the state in / out (host arrays, Fortran order).  pi may be NULL
 * unless the Maxwell closure evolves Pi.  set_state projects the fields onto
 * the dealiased band, as the reference's state is after every stage. */
int hydft_gpu_set_state(hydft_gpu *h, const double *n, const double *mom, const double *pi);
int hydft_gpu_get_state(hydft_gpu *h, double *n, double *mom, double *pi);

/* set_initial_condition (src/model/initial.f90:23-75): kind "uniform",
 * "mode", "gaussian", or "random" (seeded counter-based stream in place of
 * gfortran's generator).  Resets mom and Pi to zero. */
int hydft_gpu_set_initial_condition(hydft_gpu *h, const char *kind, double amplitude,
                                    const int mode[3], double width, int seed);

/* nsteps calls of model_t%advance (model.f90:186-227) at the current dt. */
int hydft_gpu_advance(hydft_gpu *h, int nsteps);

/* model_t%rhs (model.f90:85-146) of the current state at time t; outputs
 * are host arrays (dpi may be NULL unless Pi evolves). */
int hydft_gpu_rhs(hydft_gpu *h, double t, double *dn, double *dmom, double *dpi);

/* model_t%compute_dt (model.f90:150-183); the result is also the dt that
 * the next advance uses. */
int hydft_gpu_compute_dt(hydft_gpu *h, double *dt);

/* Scalars of model_t: t, dt, step. */
int hydft_gpu_get_time(const hydft_gpu *h, double *t, double *dt, int64_t *step);
int hydft_gpu_set_time(hydft_gpu *h, double t, double dt);

/* diag_t%budgets (src/model/diagnostics.f90:41-60): mass, momentum and
 * kinetic energy from FP64 compensated sums over the grid; free energy of
 * the functional (+ external potential).  nmin/nmax as in diag_write. */
int hydft_gpu_budgets(hydft_gpu *h, double *mass, double mom[3], double *ekin, double *fe,
                      double *nmin, double *nmax);

/* spec_t%mode (spectral.f90:179-188) of n (field 0) or mom_1..3 (1..3). */
int hydft_gpu_mode(hydft_gpu *h, int field, int mx, int my, int mz, double *re, double *im);

/* Setup scalars (units, transport, stress): name in
 * n0 beta gamma kappa mass hbar theta alpha0 cn lambda_qsp lambda_tf eta xi
 * tau eta_l u_ex du_dgamma kmax_dealiased volume cg ndim evolve precision. */
int hydft_gpu_get_scalar(const hydft_gpu *h, const char *name, double *value);
int hydft_gpu_set_scalar(hydft_gpu *h, const char *name, double value);

/* The structure table in use (k, c(k)); n is the table length. */
int hydft_gpu_get_structure(const hydft_gpu *h, int *n, double *k, double *c);

/* Total linear kernel K(k) = sum of the terms' kernels (functional.f90:72-80). */
int hydft_gpu_kernel(const hydft_gpu *h, double k, double *kk);

/* The device stream the handle launches on (cudaStream_t as void*). */
void *hydft_gpu_stream(const hydft_gpu *h);

/* Kernel launches made by the library since creation (for accounting). */
int64_t hydft_gpu_launch_count(const hydft_gpu *h);

/*
 * Timing of the step's kernels: runs nsteps uncaptured RK3 steps with a
 * CUDA event pair on the launching stream around every kernel, and reports
 * per kernel class (names comma-separated into `names`): total device time
 * in ms, algorithmic bytes per launch (each input read once, each output
 * written once) and the number of launches.  The state advances by nsteps.
 * No counterpart in the reference (it only times the run loop with
 * cpu_time, src/hydft.f90:39-55).
 */
int hydft_gpu_profile(hydft_gpu *h, int nsteps, int max_kernels, char *names, int names_len,
                      double *total_ms, double *bytes_per_launch, int64_t *launches, int *nkernels);

/* ------------------------------------------------- setup on the device */

/*
 * OZ-HNC solve (src/structure/oz_hnc.f90:111-296, hnc_solve with its
 * Gamma continuation) in FP64 on the GPU.  potential: "yukawa", "coulomb",
 * "hansen_mcdonald".  Outputs (length nr, any may be NULL): r, k, g(r),
 * c(k), S(k); scalars u_ex, converged, niter, residual.
 */
int hydft_gpu_hnc_solve(const char *potential, double gamma, double kappa, double lambda,
                        double n0, int nr, double rmax, double tol, double mix, int maxiter,
                        int device, double *r, double *k, double *g, double *ck, double *sk,
                        double *u_ex, int *converged, int *niter, double *residual);

/* Fourier-Bessel transform pair of the HNC solver (fourier_bessel_t%r2k /
 * %k2r, src/structure/oz_hnc.f90:79-96) on the GPU in FP64, host arrays of
 * length n: direction 0 is r2k, f(k) = (4 pi/k) int r f(r) sin(kr) dr;
 * direction 1 is k2r, f(r) = (1/(2 pi^2 r)) int k f(k) sin(kr) dk; on the
 * grids r_j = j dr, k_m = m dk, dr = rmax/(n+1), dk = pi/((n+1) dr).
 * n <= 9600. */
int hydft_gpu_fourier_bessel(const double *f_in, double *f_out, int n, double rmax, int direction,
                             int device);

/*
 * hydft_gpu_fourier_bessel without device allocation.  No counterpart in
 * the reference: it exists for callers that cannot allocate device memory
 * where they need the transform (inside a loop that must not synchronise
 * the device, or under a host framework that owns all device allocations).
 * d_in and d_out are device arrays of n doubles provided by the caller; the
 * sine table and weights live in a fixed scratch array inside the library
 * (2(n+1) + 2n doubles for n <= HYDFT_FB_NOALLOC_MAX_N, 262 160 bytes,
 * resident on every GPU that loads the library until the process exits).
 * n above the maximum is rejected with HYDFT_ERR_BAD_ARG, and so are d_in
 * and d_out ranges that overlap (the transform reads all of d_in while it
 * writes d_out).  The kernels run on `stream` (a cudaStream_t; NULL is the
 * calling thread's per-thread default stream, since the library is built
 * with --default-stream per-thread) and the call returns without waiting
 * for them.  Every call rebuilds the tables for its own n and rmax; calls
 * whose work overlaps on the GPU share the scratch array and race.  Every
 * call looks up the scratch array's address in the current context; the
 * first call on a device also loads the library's kernels there, so make
 * it before any stream capture.  Errors: hydft_gpu_create_error().
 */
#define HYDFT_FB_NOALLOC_MAX_N 8192
int hydft_gpu_fourier_bessel_noalloc(const double *d_in, double *d_out, int n, double rmax,
                                     int direction, void *stream);

/* Fermi-Dirac table tab(6, 6601) (fermi_dirac.f90:30-74) built on the GPU;
 * out has 6*6601 doubles, column index fastest. */
int hydft_gpu_fd_table(int device, double *out, int *ntab);

/* Batched Fermi-Dirac inverse alpha = I_{1/2}^{-1}(y) (fermi_dirac.f90:241-267)
 * on the GPU for n host values. */
int hydft_gpu_fd_alpha(int device, const double *y, double *alpha, int n);

/*
 * Ensembles.  The reference runs one model_t per process and steps it in
 * the driver loop of src/hydft.f90:41-51; an ensemble holds many such
 * models (each with its own grid, species, Gamma, kappa and closure) on one
 * GPU and advances all of them by one RK3 step per launch of a single
 * captured CUDA graph.  Members below 128^3 cells whose steps have the same
 * launches (same grid, closure, precision and term kinds) form a group:
 * each kernel of the step runs once for the whole group, every member's
 * arguments read from a device table, so a group of 59 members of 48^3
 * makes as many launches per step as one member.  Groups, members of 128^3
 * cells or more (whose launches fill the GPU alone) and members whose step
 * has no ensemble form (grids without register FFT plans) are independent
 * branches of the graph.  A member's fields are bit-identical to the same
 * model advanced alone.
 *
 * hydft_batch_create builds n members from params[i] (and structures[i]
 * when structures != NULL and structures[i].n > 0; members whose HNC
 * inputs agree share one OZ-HNC solve).  Errors: hydft_gpu_create_error().
 * hydft_batch_member gives member i as a hydft_gpu handle for every
 * single-model call (set_state, set_initial_condition, compute_dt,
 * get_state, budgets, mode, ...); the handle belongs to the ensemble and
 * hydft_gpu_destroy ignores it.  hydft_batch_advance runs nsteps ensemble
 * steps (every member at its own dt, which must be set) and then checks
 * every member's status; on an error hydft_batch_failed_member names the
 * first failing member and hydft_batch_last_error gives its message.
 */
typedef struct hydft_batch hydft_batch;
int hydft_batch_create(int n, const hydft_params *params, const hydft_structure *structures, int device,
                       hydft_batch **out);
void hydft_batch_destroy(hydft_batch *b);
int hydft_batch_size(const hydft_batch *b);
int hydft_batch_member(hydft_batch *b, int i, hydft_gpu **member);
int hydft_batch_advance(hydft_batch *b, int nsteps);
const char *hydft_batch_last_error(const hydft_batch *b);
int hydft_batch_failed_member(const hydft_batch *b);
/* kernels the ensemble's graph launched so far (a group launch counts
 * once), and the stream the ensemble graph runs on (a cudaStream_t) */
int64_t hydft_batch_launch_count(const hydft_batch *b);
void *hydft_batch_stream(const hydft_batch *b);
/* groups of members stepped by shared launches, and the members in them,
 * as of the last captured step (0 and 0 before the first advance) */
int hydft_batch_grouped(const hydft_batch *b, int *groups, int *members);

/* write_fields (src/model/io.f90:19-35): <prefix>_fld_NNNNNN.bin (NNNNNN =
 * step), raw little-endian: int32 nx, ny, nz, ndim, npi; float64 t, lx,
 * ly, lz; then n, mom(3), Pi(npi) in Fortran order. */
int hydft_gpu_write_fields(hydft_gpu *h, const char *prefix);
/* Resume from a field file of that format (no counterpart in the
 * reference, whose python/hydft_io.py:45-56 only reads them): the state and
 * t are set from the file, the step from its name; dt is kept. */
int hydft_gpu_read_fields(hydft_gpu *h, const char *path);
/* hydft_run's loop (src/hydft.f90:30-60) from the current state: dt from
 * compute_dt every 20 steps, the last step ending at tend, probes every
 * iprobe steps into <prefix>_probe.dat, budgets every idiag steps into
 * <prefix>_diag.dat, fields every iout steps (diagnostics.f90:32-77). */
int hydft_gpu_run(hydft_gpu *h);

/* Device bytes a model of these parameters allocates (the admission size
 * the server uses; Pi is assumed to evolve whenever the closure is Maxwell). */
int hydft_gpu_footprint(const hydft_params *p, double *bytes);

/*
 * Serving: solve requests on one GPU with continuous batching.  No
 * counterpart in the reference (each request runs the driver loop of
 * src/hydft.f90:41-51 for its model).
 *
 * hydft_serve_create starts a server on `device` with an HBM budget in
 * bytes (0: 80 % of the free memory), at most max_slots requests holding
 * device memory at once, and chunk_steps RK3 steps launched per scheduling
 * round of a request.  hydft_serve_submit queues a request: a model of *p,
 * its initial state (n, mom, pi host arrays as for hydft_gpu_set_state, or
 * n == NULL for p's initial condition), nsteps steps at p->dt (or the CFL
 * dt of hydft_gpu_compute_dt when p->dt is 0), keep_state != 0 to keep the
 * final fields.  Requests are admitted in arrival order as their footprint
 * (hydft_gpu_footprint) fits the budget; the models of admitted requests
 * stay resident and their steps overlap on the device.  A request larger
 * than the whole budget is refused (HYDFT_ERR_OOM).
 * hydft_serve_wait blocks until request `id` is done or failed (timeout_s <
 * 0: no limit) and reports its HYDFT_REQ_* state.  hydft_serve_result
 * copies the final fields (when kept) and HYDFT_SERVE_INFO_LEN scalars into
 * info: t, dt, step, mass, mom[3], ekin, nmin, nmax, then the submit,
 * admit, first-launch and completion times in seconds since the server
 * started, the footprint in bytes and the kernels launched; it returns the
 * request's status and releases it (message: hydft_gpu_create_error()).
 * hydft_serve_stats fills 6 values: queued, holding memory, completed,
 * most held at once, bytes in use, budget.
 */
#define HYDFT_REQ_QUEUED 0
#define HYDFT_REQ_SETUP 1
#define HYDFT_REQ_RUNNING 2
#define HYDFT_REQ_DONE 3
#define HYDFT_REQ_FAILED 4
#define HYDFT_SERVE_INFO_LEN 16
typedef struct hydft_server hydft_server;
int hydft_serve_create(int device, double hbm_budget_bytes, int max_slots, int chunk_steps, hydft_server **out);
int hydft_serve_submit(hydft_server *s, const hydft_params *p, const double *n, const double *mom,
                       const double *pi, int nsteps, int keep_state, int64_t *id);
int hydft_serve_wait(hydft_server *s, int64_t id, double timeout_s, int *state);
int hydft_serve_result(hydft_server *s, int64_t id, double *n, double *mom, double *pi, double *info);
int hydft_serve_stats(hydft_server *s, double *stats);
void hydft_serve_destroy(hydft_server *s);

#ifdef __cplusplus
}
#endif
#endif /* HYDFT_GPU_H */
