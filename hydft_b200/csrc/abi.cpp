// C ABI of the library (include/hydft_gpu.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <complex>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/hydft_gpu.h"
#include "handle.hpp"
#include "setup_gpu.hpp"

using namespace hydft;

static thread_local std::string g_create_err;

namespace hydft {
// message of a failed handle-less call, returned by hydft_gpu_create_error()
void set_thread_error(const std::string &msg) { g_create_err = msg; }
}  // namespace hydft

static int fail(hydft_gpu *h, int rc, const std::string &msg)
{
    if (h) h->err = msg;
    return rc;
}

extern "C" {

int hydft_params_default(hydft_params *p)
{
    if (!p) return HYDFT_ERR_BAD_ARG;
    params_default(p);
    return HYDFT_OK;
}

int hydft_params_finalize(hydft_params *p)
{
    if (!p) return HYDFT_ERR_BAD_ARG;
    params_finalize(p);
    return HYDFT_OK;
}

int hydft_params_read(const char *path, hydft_params *p)
{
    if (!p || !path) return HYDFT_ERR_BAD_ARG;
    std::string err;
    int rc = params_read(path, p, err);
    if (rc) g_create_err = err;
    return rc;
}

const char *hydft_gpu_create_error(void) { return g_create_err.c_str(); }

int hydft_gpu_create(const hydft_params *p, const hydft_structure *st, int device, hydft_gpu **out)
{
    if (!p || !out) return HYDFT_ERR_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
        g_create_err = "no CUDA device available (the solver has no CPU path)";
        return HYDFT_ERR_CUDA;
    }
    auto h = std::make_unique<hydft_gpu>();
    h->device = device;
    std::string err;
    int rc = build_setup(p, st, device, h->mh, err);
    if (rc) {
        g_create_err = err;
        return rc;
    }
    h->s = make_solver(h->mh.S, h->mh.precision, device, err);
    if (!h->s) {
        g_create_err = err;
        return HYDFT_ERR_CUDA;
    }
    h->s->set_time(0.0, h->mh.p.dt);
    *out = h.release();
    return HYDFT_OK;
}

int hydft_gpu_footprint(const hydft_params *p, double *bytes)
{
    if (!p || !bytes) return HYDFT_ERR_BAD_ARG;
    *bytes = footprint_bytes(p);
    return *bytes < 0 ? HYDFT_ERR_BAD_ARG : HYDFT_OK;
}

void hydft_gpu_destroy(hydft_gpu *h)
{
    if (!h || h->owned_by_batch) return;
    if (h->s) {
        cudaSetDevice(h->device);
        delete h->s;
    }
    delete h;
}

const char *hydft_gpu_last_error(const hydft_gpu *h) { return h ? h->err.c_str() : g_create_err.c_str(); }

static int wrap(hydft_gpu *h, int rc)
{
    if (rc && h->s) h->err = h->s->err;
    return rc;
}

int hydft_gpu_set_state(hydft_gpu *h, const double *n, const double *mom, const double *pi)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    // positivity of n is checked on the device by the solver
    return wrap(h, h->s->set_state(n, mom, pi));
}

int hydft_gpu_get_state(hydft_gpu *h, double *n, double *mom, double *pi)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    return wrap(h, h->s->get_state(n, mom, pi));
}

// set_initial_condition (initial.f90:23-75); 'random' uses the splitmix64
// counter stream documented in hydft_b200/ic.py
static double splitmix_u(uint64_t seed, uint64_t q)
{
    uint64_t z = (seed << 32) + (q + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int hydft_gpu_set_initial_condition(hydft_gpu *h, const char *kind, double amp, const int mode[3], double width,
                                    int seed)
{
    if (!h || !kind) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    const hydft_params &p = h->mh.p;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const size_t nc = (size_t)nx * ny * nz;
    const double twopi = 2.0 * 3.14159265358979323846264338327950288;
    std::vector<double> d(nc, 0.0), zero(3 * nc, 0.0), pz(6 * nc, 0.0);
    const std::string k = kind;
    const double dx = p.lx / nx, dy = p.ly / ny, dz = p.lz / nz;
    bool project = false, normalise = false, demean = false;
    if (k == "uniform") {
    } else if (k == "mode") {
        double kv[3] = {twopi * mode[0] / p.lx, twopi * mode[1] / p.ly, twopi * mode[2] / p.lz};
        if (ny == 1) kv[1] = 0.0;
        if (nz == 1) kv[2] = 0.0;
        for (int c = 0; c < nz; ++c)
            for (int b = 0; b < ny; ++b)
                for (int a = 0; a < nx; ++a)
                    d[a + (size_t)nx * (b + (size_t)ny * c)] = std::cos(kv[0] * (a * dx) + kv[1] * (b * dy) + kv[2] * (c * dz));
    } else if (k == "random") {
        for (size_t q = 0; q < nc; ++q) d[q] = splitmix_u((uint64_t)seed, q) - 0.5;
        project = normalise = demean = true;
    } else if (k == "gaussian") {
        for (int c = 0; c < nz; ++c)
            for (int b = 0; b < ny; ++b)
                for (int a = 0; a < nx; ++a) {
                    const double x = a * dx - 0.5 * p.lx;
                    const double y = ny > 1 ? b * dy - 0.5 * p.ly : 0.0;
                    const double z = nz > 1 ? c * dz - 0.5 * p.lz : 0.0;
                    d[a + (size_t)nx * (b + (size_t)ny * c)] = std::exp(-0.5 * (x * x + y * y + z * z) / (width * width));
                }
        project = demean = true;
    } else {
        return fail(h, HYDFT_ERR_UNSUPPORTED, "unknown initial condition: " + k);
    }
    const double n0 = h->mh.n0;
    if (project) {
        // dealias d on the device: the state projection keeps the band only.
        // d is carried as n = 1 + d so the density stays positive.
        std::vector<double> tmp(nc);
        for (size_t q = 0; q < nc; ++q) tmp[q] = 2.0 + d[q];
        int rc = h->s->set_state(tmp.data(), zero.data(), pz.data());
        if (rc) return wrap(h, rc);
        rc = h->s->get_state(tmp.data(), nullptr, nullptr);
        if (rc) return wrap(h, rc);
        for (size_t q = 0; q < nc; ++q) d[q] = tmp[q] - 2.0;
    }
    if (demean) {
        double s = 0.0;
        for (size_t q = 0; q < nc; ++q) s += d[q];
        s /= (double)nc;
        for (size_t q = 0; q < nc; ++q) d[q] -= s;
    }
    if (normalise) {
        double s = 0.0;
        for (size_t q = 0; q < nc; ++q) s += d[q] * d[q];
        const double rms = std::sqrt(s / (double)nc);
        if (rms > 0.0)
            for (size_t q = 0; q < nc; ++q) d[q] /= rms;
    }
    for (size_t q = 0; q < nc; ++q) {
        d[q] = n0 * (1.0 + amp * d[q]);
        if (!(d[q] > 0.0))
            return fail(h, HYDFT_ERR_NONPOSITIVE_DENSITY, "initial density is not positive; reduce the amplitude");
    }
    return wrap(h, h->s->set_state(d.data(), zero.data(), pz.data()));
}

int hydft_gpu_advance(hydft_gpu *h, int nsteps)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    if (nsteps < 0) return fail(h, HYDFT_ERR_BAD_ARG, "nsteps must be >= 0");
    cudaSetDevice(h->device);
    double t, dt;
    int64_t st;
    h->s->get_time(&t, &dt, &st);
    if (!(dt > 0.0)) return fail(h, HYDFT_ERR_BAD_ARG, "dt is not set; call compute_dt or set dt in &time");
    return wrap(h, h->s->advance(nsteps));
}

int hydft_gpu_rhs(hydft_gpu *h, double t, double *dn, double *dmom, double *dpi)
{
    if (!h || !dn || !dmom) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    return wrap(h, h->s->rhs(t, dn, dmom, dpi));
}

// model.f90:150-183
int hydft_gpu_compute_dt(hydft_gpu *h, double *dt_out)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    double t, dt;
    int64_t st;
    h->s->get_time(&t, &dt, &st);
    if (h->mh.p.dt > 0.0) {
        dt = h->mh.p.dt;
    } else {
        double sn, sm[3], sk, nmin, nmax, umax;
        int rc = h->s->reductions(&sn, sm, &sk, &nmin, &nmax, &umax);
        if (rc) return wrap(h, rc);
        double dtm = HUGE_VAL;
        if (h->mh.wmax > 0.0) dtm = std::min(dtm, 1.7 / h->mh.wmax);
        if (h->mh.numax > 0.0) dtm = std::min(dtm, 2.5 / h->mh.numax);
        if (umax > 0.0) dtm = std::min(dtm, h->mh.dxmin / umax);
        if (dtm == HUGE_VAL) return fail(h, HYDFT_ERR_CFL, "cannot determine a time step; set dt in &time");
        dt = h->mh.p.cfl * dtm;
    }
    h->s->set_time(t, dt);
    if (dt_out) *dt_out = dt;
    return HYDFT_OK;
}

int hydft_gpu_get_time(const hydft_gpu *h, double *t, double *dt, int64_t *step)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    h->s->get_time(t, dt, step);
    return HYDFT_OK;
}

int hydft_gpu_set_time(hydft_gpu *h, double t, double dt)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    h->s->set_time(t, dt);
    return HYDFT_OK;
}

int hydft_gpu_budgets(hydft_gpu *h, double *mass, double mom[3], double *ekin, double *fe, double *nmin,
                      double *nmax)
{
    if (!h) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    double sn, sm[3], sk, mn, mx, umax;
    int rc = h->s->reductions(&sn, sm, &sk, &mn, &mx, &umax);
    if (rc) return wrap(h, rc);
    const double nc = (double)h->mh.p.nx * h->mh.p.ny * h->mh.p.nz;
    const double v = h->mh.S.volume;
    if (mass) *mass = sn / nc * v;
    if (mom)
        for (int d = 0; d < 3; ++d) mom[d] = sm[d] / nc * v;
    if (ekin) *ekin = 0.5 * (sk / nc) * v / h->mh.mass;
    if (fe) {
        rc = h->s->energy(fe);
        if (rc) return wrap(h, rc);
    }
    if (nmin) *nmin = mn;
    if (nmax) *nmax = mx;
    return HYDFT_OK;
}

int hydft_gpu_mode(hydft_gpu *h, int field, int mx, int my, int mz, double *re, double *im)
{
    if (!h || field < 0 || field > 3 || !re || !im) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    return wrap(h, h->s->mode(field, mx, my, mz, re, im));
}

int hydft_gpu_get_scalar(const hydft_gpu *h, const char *name, double *v)
{
    if (!h || !name || !v) return HYDFT_ERR_BAD_ARG;
    const ModelHost &m = h->mh;
    const std::string k = name;
    if (k == "n0") *v = m.n0;
    else if (k == "beta") *v = m.beta;
    else if (k == "gamma") *v = m.gamma;
    else if (k == "kappa") *v = m.kappa;
    else if (k == "mass") *v = m.mass;
    else if (k == "hbar") *v = m.hbar;
    else if (k == "theta") *v = m.theta;
    else if (k == "alpha0") *v = m.alpha0;
    else if (k == "cn") *v = m.cn;
    else if (k == "lambda_qsp") *v = m.lambda_qsp;
    else if (k == "lambda_tf") *v = m.lambda_tf;
    else if (k == "eta") *v = m.eta;
    else if (k == "xi") *v = m.xi;
    else if (k == "tau") *v = m.s_tau;
    else if (k == "eta_l") *v = m.eta_l;
    else if (k == "u_ex") *v = m.u_ex;
    else if (k == "du_dgamma") *v = m.du_dgamma;
    else if (k == "kmax_dealiased") *v = m.kmax_dealiased;
    else if (k == "volume") *v = m.S.volume;
    else if (k == "cg") *v = m.cg;
    else if (k == "ndim") *v = m.S.g.ndim;
    else if (k == "evolve") *v = m.evolve ? 1.0 : 0.0;
    else if (k == "precision") *v = m.precision;
    else if (k == "device_bytes") *v = (double)h->s->device_bytes();
    else if (k == "yz_tile" || k == "yz_threads" || k == "yz_tile_fwd" || k == "yz_threads_fwd" ||
             k == "x_threads") {
        int t[5] = {0, 0, 0, 0, 0};
        h->s->tiles(t);
        const int i = k == "yz_tile" ? 0 : k == "yz_threads" ? 1 : k == "yz_tile_fwd" ? 2 : k == "yz_threads_fwd" ? 3 : 4;
        *v = t[i];
    }
    else if (k == "radix_x" || k == "radix_y" || k == "radix_z")
        *v = h->s->radix_code(k == "radix_x" ? 0 : (k == "radix_y" ? 1 : 2));
    else if (k == "band_axes") *v = h->s->band_axes();
    else if (k == "ext_omega") *v = m.ext_omega;
    else if (k == "hnc_niter") *v = m.hnc_niter;
    else if (k == "wmax") *v = m.wmax;
    else return HYDFT_ERR_BAD_ARG;
    return HYDFT_OK;
}

int hydft_gpu_set_scalar(hydft_gpu *h, const char *name, double v)
{
    if (!h || !name) return HYDFT_ERR_BAD_ARG;
    const std::string k = name;
    if (k == "ext_omega") {
        h->mh.ext_omega = v;
        h->mh.S.ext_omega = v;
        h->s->set_ext_omega(v);
        return HYDFT_OK;
    }
    return fail(h, HYDFT_ERR_BAD_ARG, "unknown or read-only scalar: " + k);
}

int hydft_gpu_get_structure(const hydft_gpu *h, int *n, double *k, double *c)
{
    if (!h || !n) return HYDFT_ERR_BAD_ARG;
    *n = (int)h->mh.st_k.size();
    if (k) std::memcpy(k, h->mh.st_k.data(), sizeof(double) * h->mh.st_k.size());
    if (c) std::memcpy(c, h->mh.st_c.data(), sizeof(double) * h->mh.st_c.size());
    return HYDFT_OK;
}

int hydft_gpu_kernel(const hydft_gpu *h, double k, double *kk)
{
    if (!h || !kk) return HYDFT_ERR_BAD_ARG;
    *kk = h->mh.kernel(k);
    return HYDFT_OK;
}

int hydft_gpu_profile(hydft_gpu *h, int nsteps, int max_kernels, char *names, int names_len, double *total_ms,
                      double *bytes_per_launch, int64_t *launches, int *nkernels)
{
    if (!h || nsteps < 1 || max_kernels < 1 || !names || names_len < 1) return HYDFT_ERR_BAD_ARG;
    cudaSetDevice(h->device);
    double t, dt;
    int64_t stp;
    h->s->get_time(&t, &dt, &stp);
    if (!(dt > 0.0)) return fail(h, HYDFT_ERR_BAD_ARG, "dt is not set");
    std::vector<KernelStat> ks;
    int rc = h->s->profile(nsteps, ks);
    if (rc) return wrap(h, rc);
    std::string nm;
    int k = 0;
    for (auto &s : ks) {
        if (k >= max_kernels) break;
        if (k) nm += ",";
        nm += s.name;
        if (total_ms) total_ms[k] = s.ms;
        if (bytes_per_launch) bytes_per_launch[k] = s.n ? s.bytes / (double)s.n : 0.0;
        if (launches) launches[k] = s.n;
        ++k;
    }
    std::snprintf(names, names_len, "%s", nm.c_str());
    if (nkernels) *nkernels = k;
    return HYDFT_OK;
}

void *hydft_gpu_stream(const hydft_gpu *h) { return h && h->s ? h->s->stream() : nullptr; }

int64_t hydft_gpu_launch_count(const hydft_gpu *h) { return h && h->s ? h->s->launches : 0; }

int hydft_gpu_hnc_solve(const char *potential, double gamma, double kappa, double lambda, double n0, int nr,
                        double rmax, double tol, double mix, int maxiter, int device, double *r, double *k,
                        double *g, double *ck, double *sk, double *u_ex, int *converged, int *niter,
                        double *residual)
{
    if (!potential) return HYDFT_ERR_BAD_ARG;
    Potential pot;
    const std::string pn = potential;
    if (pn == "yukawa") pot.kind = 0;
    else if (pn == "coulomb") pot.kind = 1;
    else if (pn == "hansen_mcdonald" || pn == "hm" || pn == "qsp") pot.kind = 2;
    else { g_create_err = "unknown pair potential: " + pn; return HYDFT_ERR_BAD_ARG; }
    pot.gamma = gamma;
    pot.kappa = kappa;
    pot.lambda = lambda;
    HncOut res;
    std::string err;
    int rc = gpu_hnc_solve(device, pot, n0, nr, rmax, tol, mix, maxiter, res, err);
    if (rc) { g_create_err = err; return rc; }
    auto put = [&](double *dst, const std::vector<double> &v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(double) * v.size());
    };
    put(r, res.r); put(k, res.k); put(g, res.g); put(ck, res.ck); put(sk, res.sk);
    if (u_ex) *u_ex = res.u_ex;
    if (converged) *converged = res.converged ? 1 : 0;
    if (niter) *niter = res.niter;
    if (residual) *residual = res.residual;
    return HYDFT_OK;
}

int hydft_gpu_fourier_bessel(const double *f_in, double *f_out, int n, double rmax, int direction, int device)
{
    if (!f_in || !f_out || n < 1 || !(rmax > 0.0) || (direction != 0 && direction != 1)) {
        g_create_err = "fourier_bessel: bad arguments";
        return HYDFT_ERR_BAD_ARG;
    }
    std::string err;
    int rc = gpu_fourier_bessel(device, f_in, f_out, n, rmax, direction, err);
    if (rc) g_create_err = err;
    return rc;
}

int hydft_gpu_fd_table(int device, double *out, int *ntab)
{
    std::vector<double> t;
    std::string err;
    int rc = gpu_fd_table(device, t, err);
    if (rc) { g_create_err = err; return rc; }
    if (out) std::memcpy(out, t.data(), sizeof(double) * t.size());
    if (ntab) *ntab = (int)(t.size() / 6);
    return HYDFT_OK;
}

int hydft_gpu_fd_alpha(int device, const double *y, double *alpha, int n)
{
    if (!y || !alpha || n < 0) return HYDFT_ERR_BAD_ARG;
    std::vector<double> t;
    std::string err;
    int rc = gpu_fd_table(device, t, err);
    if (rc) { g_create_err = err; return rc; }
    rc = gpu_fd_alpha(device, t, y, alpha, n, err);
    if (rc) { g_create_err = err; return rc; }
    return HYDFT_OK;
}

}  // extern "C"
