// FP64 setup on the GPU: the Fermi-Dirac table (fermi_dirac.f90:30-74), a
// batched Fermi-Dirac inverse, and the Ornstein-Zernike / HNC solver with
// Ng acceleration, restarts and Gamma continuation (oz_hnc.f90:111-296).
//
// The HNC's Fourier-Bessel transforms are DST-I's of length nr
// (y_k = 2 sum_j x_j sin(pi (j+1)(k+1)/(nr+1)), FFTW's RODFT00).  Their
// length 2(nr+1) has large prime factors for the usual nr (8194 = 2 17 241),
// so each output is summed directly: the sine of pi*m/(nr+1) is tabulated
// once for m < 2(nr+1) in shared memory and the integer phase (j+1)(k+1)
// mod 2(nr+1) advances by k+1 per term.  The iteration's control flow
// (convergence, instability, Ng acceptance, restarts, continuation) is
// driven from the host with the reductions read back each iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fermi_dirac.cuh"
#include "setup_gpu.hpp"

namespace hydft {

static const double PI = 3.14159265358979323846264338327950288;

#define CKS(call)                                                                \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return 7;                                                            \
        }                                                                        \
    } while (0)

// Gauss-Legendre nodes on (-1,1) by Newton on the Legendre recurrence
// (the method of quadrature.f90:17-38).
void gauss_legendre(int n, double *x, double *w)
{
    for (int i = 1; i <= (n + 1) / 2; ++i) {
        double z = std::cos(PI * (i - 0.25) / (n + 0.5));
        double pp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p1 = 1.0, p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            const double z1 = z;
            z = z1 - p1 / pp;
            if (std::fabs(z - z1) < 1.0e-15) break;
        }
        x[i - 1] = -z;
        x[n - i] = z;
        w[i - 1] = 2.0 / ((1.0 - z * z) * pp * pp);
        w[n - i] = w[i - 1];
    }
}

struct GL20 {
    double x[fd::NGL], w[fd::NGL];
};

__device__ __forceinline__ void fermi_derivs(double y, double &f, double &p1, double &p2, double &p3)
{
    if (y > 0.0) {
        const double g = exp(-y);
        f = g / (1.0 + g);
    } else {
        const double g = exp(y);
        f = 1.0 / (1.0 + g);
    }
    p1 = f * (1.0 - f);
    p2 = p1 * (1.0 - 2.0 * f);
    p3 = p1 * (1.0 - 6.0 * f + 6.0 * f * f);
}

// one thread per table node; the panel sums run in the same order as the
// serial reference loop
__global__ void fd_table_kernel(double *tab, GL20 q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= fd::NTAB) return;
    const double alpha = fd::AMIN + i * fd::H;
    const double xmax = fmax(alpha, 0.0) + 45.0;
    double s[6] = {0, 0, 0, 0, 0, 0};
    double f, p1, p2, p3;
    for (int k = 0; k < fd::NGL; ++k) {
        const double t = 0.5 * (q.x[k] + 1.0);
        const double x = t * t;
        fermi_derivs(x - alpha, f, p1, p2, p3);
        const double e = q.w[k] * 0.5 * 2.0;
        s[0] += e * f;
        s[1] += e * t * t * f;
        s[2] += e * (t * t) * (t * t) * f;
        s[3] += e * p1;
        s[4] += e * p2;
        s[5] += e * p3;
    }
    const int npan = (int)ceil(xmax - 1.0);
    for (int ip = 1; ip <= npan; ++ip) {
        const double a = 1.0 + (ip - 1);
        const double b = fmin(a + 1.0, xmax);
        const double xm = 0.5 * (a + b), xr = 0.5 * (b - a);
        for (int k = 0; k < fd::NGL; ++k) {
            const double x = xm + xr * q.x[k];
            fermi_derivs(x - alpha, f, p1, p2, p3);
            const double e = q.w[k] * xr;
            const double sx = sqrt(x);
            const double t = 1.0 / sx;
            s[0] += e * t * f;
            s[1] += e * sx * f;
            s[2] += e * x * sx * f;
            s[3] += e * t * p1;
            s[4] += e * t * p2;
            s[5] += e * t * p3;
        }
    }
    for (int c = 0; c < 6; ++c) tab[6 * i + c] = s[c];
}

int gpu_fd_table(int device, std::vector<double> &out, std::string &err)
{
    CKS(cudaSetDevice(device));
    GL20 q;
    gauss_legendre(fd::NGL, q.x, q.w);
    double *d = nullptr;
    CKS(cudaMalloc(&d, sizeof(double) * 6 * fd::NTAB));
    fd_table_kernel<<<(fd::NTAB + 127) / 128, 128>>>(d, q);
    out.resize(6 * fd::NTAB);
    cudaError_t e = cudaMemcpy(out.data(), d, sizeof(double) * 6 * fd::NTAB, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        err = std::string("fd table: ") + cudaGetErrorString(e);
        return 7;
    }
    return 0;
}

__global__ void fd_alpha_kernel(const double *tab, const double *y, double *alpha, int n, unsigned *bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool ok = true;
    alpha[i] = fd::alpha_from_ip12(tab, y[i], &ok);
    if (!(y[i] > 0.0)) atomicOr(bad, 1u);
}

int gpu_fd_alpha(int device, const std::vector<double> &tab, const double *y, double *alpha, int n,
                 std::string &err)
{
    CKS(cudaSetDevice(device));
    double *dt = nullptr, *dy = nullptr, *da = nullptr;
    unsigned *bad = nullptr;
    CKS(cudaMalloc(&dt, sizeof(double) * tab.size()));
    CKS(cudaMalloc(&dy, sizeof(double) * std::max(n, 1)));
    CKS(cudaMalloc(&da, sizeof(double) * std::max(n, 1)));
    CKS(cudaMalloc(&bad, sizeof(unsigned)));
    CKS(cudaMemset(bad, 0, sizeof(unsigned)));
    CKS(cudaMemcpy(dt, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    CKS(cudaMemcpy(dy, y, sizeof(double) * n, cudaMemcpyHostToDevice));
    if (n > 0) fd_alpha_kernel<<<(n + 127) / 128, 128>>>(dt, dy, da, n, bad);
    unsigned hb = 0;
    CKS(cudaMemcpy(alpha, da, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(&hb, bad, sizeof(unsigned), cudaMemcpyDeviceToHost));
    cudaFree(dt); cudaFree(dy); cudaFree(da); cudaFree(bad);
    if (hb) {
        err = "fermi_dirac: I_{1/2} inverse needs y > 0";
        return 1;
    }
    return 0;
}

// ------------------------------------------------------------------ HNC
// pair potentials (pair_potential.f90:62-118)
static double pot_beta_v(const Potential &p, double r)
{
    switch (p.kind) {
    case 0: return p.gamma * std::exp(-p.kappa * r) / r;
    case 1: return p.gamma / r;
    default: {
        const double ln2 = 0.693147180559945309417232121458;
        double v = r > 0.0 ? p.gamma * (1.0 - std::exp(-2.0 * PI * r / p.lambda)) / r : p.gamma * 2.0 * PI / p.lambda;
        if (p.pauli) v += ln2 * std::exp(-4.0 * PI * r * r / (p.lambda * p.lambda * ln2));
        return v;
    }
    }
}

static double pot_long_r(const Potential &p, double r)
{
    const double kp = p.kappa + p.ksplit;
    if (r > 1.0e-12) return p.gamma * (std::exp(-p.kappa * r) - std::exp(-kp * r)) / r;
    return p.gamma * (kp - p.kappa);
}

static double pot_long_k(const Potential &p, double k)
{
    const double kp = p.kappa + p.ksplit;
    return 4.0 * PI * p.gamma * (1.0 / (k * k + p.kappa * p.kappa) - 1.0 / (k * k + kp * kp));
}

static double pot_beta_v_k(const Potential &p, double k) { return 4.0 * PI * p.gamma / (k * k + p.kappa * p.kappa); }

// DST-I by direct summation with an integer phase; pre and post scale the
// input and output (the Fourier-Bessel weights): out_k = post_k * 2 sum_j
// pre_j x_j sin(pi (j+1)(k+1)/(n+1))
__global__ void dst_kernel(const double *x, const double *pre, const double *post, double *out, int n,
                           const double *sintab)
{
    extern __shared__ double sm[];
    const int M = 2 * (n + 1);
    double *st = sm;          // sin(pi m/(n+1)), m < M
    double *xs = sm + M;      // pre * x
    for (int m = threadIdx.x; m < M; m += blockDim.x) st[m] = sintab[m];
    for (int j = threadIdx.x; j < n; j += blockDim.x) xs[j] = pre[j] * x[j];
    __syncthreads();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int step = k + 1;
    int ph = step;            // (j+1)(k+1) mod M for j = 0
    double acc0 = 0.0, acc1 = 0.0;
    int j = 0;
    for (; j + 1 < n; j += 2) {
        acc0 += xs[j] * st[ph];
        ph += step; if (ph >= M) ph -= M;
        acc1 += xs[j + 1] * st[ph];
        ph += step; if (ph >= M) ph -= M;
    }
    if (j < n) acc0 += xs[j] * st[ph];
    out[k] = post[k] * 2.0 * (acc0 + acc1);
}

// closure of the short-range indirect correlation: cs = exp(min(ex, cap)) - 1 - gs
__global__ void hnc_closure_kernel(const double *bvs, const double *gs, double *cs, int n)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double ex = -bvs[j] + gs[j];
    cs[j] = exp(fmin(ex, 40.0)) - 1.0 - gs[j];
}

// ck = csk - bvl_k; unstable if n0 ck >= 1; gk = n0 ck^2/(1 - n0 ck) - bvl_k
__global__ void hnc_oz_kernel(const double *csk, const double *bvl_k, double n0, double *ck, double *gk, int n,
                              unsigned *unstable)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double c = csk[j] - bvl_k[j];
    ck[j] = c;
    if (n0 * c >= 1.0) atomicOr(unstable, 1u);
    gk[j] = n0 * c * c / (1.0 - n0 * c) - bvl_k[j];
}

// block maxima of |a - b| (non-negative doubles order like their bit patterns)
__global__ void maxabsdiff_kernel(const double *a, const double *b, int n, unsigned long long *out)
{
    double m = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[j] - b[j]));
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Ng: d0 = o1 - i1, d01 = d0 - (o2 - i2), d02 = d0 - (o3 - i3); block partial
// dot products a11, a12, a22, b1, b2 (fixed-order final sum on the host)
__global__ void ng_dots_kernel(const double *i1, const double *o1, const double *i2, const double *o2,
                               const double *i3, const double *o3, int n, double *part)
{
    __shared__ double sh[5][32];
    double a11 = 0, a12 = 0, a22 = 0, b1 = 0, b2 = 0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double d0 = o1[j] - i1[j];
        const double d01 = d0 - (o2[j] - i2[j]);
        const double d02 = d0 - (o3[j] - i3[j]);
        a11 += d01 * d01; a12 += d01 * d02; a22 += d02 * d02; b1 += d0 * d01; b2 += d0 * d02;
    }
    double v[5] = {a11, a12, a22, b1, b2};
    for (int off = 16; off > 0; off >>= 1)
        for (int i = 0; i < 5; ++i) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0)
        for (int i = 0; i < 5; ++i) sh[i][w] = v[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x / 32;
        for (int i = 0; i < 5; ++i) {
            double s = 0.0;
            for (int q = 0; q < nw; ++q) s += sh[i][q];
            part[blockIdx.x * 5 + i] = s;
        }
    }
}

// gtry = (1-c1-c2) o1 + c1 o2 + c2 o3; block maxima of gtry - bvs
__global__ void ng_try_kernel(const double *o1, const double *o2, const double *o3, double c1, double c2,
                              const double *bvs, double *gtry, int n, unsigned long long *mx)
{
    double m = -1e300;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const double gtj = (1.0 - c1 - c2) * o1[j] + c1 * o2[j] + c2 * o3[j];
        gtry[j] = gtj;
        m = fmax(m, gtj - bvs[j]);
    }
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    // map the double to an order-preserving unsigned key
    if ((threadIdx.x & 31) == 0) {
        unsigned long long b = (unsigned long long)__double_as_longlong(m);
        b = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
        atomicMax(mx, b);
    }
}

__global__ void mix_kernel(double *gs, const double *gnew, double mix, int n)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) gs[j] = (1.0 - mix) * gs[j] + mix * gnew[j];
}

// final quantities of hnc_solve_direct (oz_hnc.f90:276-294)
__global__ void hnc_final_kernel(const double *bvs, const double *gs, double *g, double *cs, int n)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double ex = -bvs[j] + gs[j];
    g[j] = exp(fmin(ex, 40.0));
    cs[j] = g[j] - 1.0 - gs[j];
}

struct HncDev {
    int n = 0, nb = 0;
    double *r, *k, *bvs, *bvl_k, *bvl_r, *pre_r2k, *post_r2k, *pre_k2r, *post_k2r, *sintab;
    double *gs, *gnew, *cs, *csk, *ck, *gk, *gtry, *gk_mf, *hin[3], *hout[3], *part, *gdev;
    unsigned *flag;
    unsigned long long *umax;
    std::vector<void *> mem;
    ~HncDev()
    {
        for (void *p : mem) cudaFree(p);
    }
};

static int hnc_alloc(HncDev &d, int n, std::string &err)
{
    d.n = n;
    d.nb = std::min(256, (n + 255) / 256);
    auto A = [&](double *&p, size_t m) -> int {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, sizeof(double) * std::max<size_t>(m, 1));
        if (e != cudaSuccess) { err = std::string("hnc alloc: ") + cudaGetErrorString(e); return 2; }
        d.mem.push_back(q);
        p = (double *)q;
        return 0;
    };
    double **one[] = {&d.r, &d.k, &d.bvs, &d.bvl_k, &d.bvl_r, &d.pre_r2k, &d.post_r2k, &d.pre_k2r, &d.post_k2r,
                      &d.gs, &d.gnew, &d.cs, &d.csk, &d.ck, &d.gk, &d.gtry, &d.gk_mf, &d.gdev};
    for (double **p : one)
        if (int rc = A(*p, n)) return rc;
    for (int i = 0; i < 3; ++i) {
        if (int rc = A(d.hin[i], n)) return rc;
        if (int rc = A(d.hout[i], n)) return rc;
    }
    if (int rc = A(d.sintab, 2 * (n + 1))) return rc;
    if (int rc = A(d.part, 5 * 256)) return rc;
    void *q = nullptr;
    if (cudaMalloc(&q, 16) != cudaSuccess) { err = "hnc alloc flags"; return 2; }
    d.mem.push_back(q);
    d.flag = (unsigned *)q;
    if (cudaMalloc(&q, 16) != cudaSuccess) { err = "hnc alloc flags"; return 2; }
    d.mem.push_back(q);
    d.umax = (unsigned long long *)q;
    return 0;
}

// y = DST(pre .* x) .* post
static void dst(HncDev &d, const double *x, const double *pre, const double *post, double *y)
{
    const int n = d.n;
    const size_t sm = sizeof(double) * (2 * (n + 1) + n);
    dst_kernel<<<(n + 127) / 128, 128, sm>>>(x, pre, post, y, n, d.sintab);
}

// Fourier-Bessel transform pair of fourier_bessel_t (oz_hnc.f90:79-96) on
// host arrays: direction 0 is r2k, f(k) = 2 pi dr DST(r f)/k; direction 1
// is k2r, f(r) = dk DST(k f)/(4 pi^2 r); r_j = j dr, k_m = m dk,
// dr = rmax/(n+1), dk = pi/((n+1) dr).
int gpu_fourier_bessel(int device, const double *fin, double *fout, int n, double rmax, int direction,
                       std::string &err)
{
    CKS(cudaSetDevice(device));
    if (n < 1) { err = "fourier_bessel: n must be >= 1"; return 1; }
    const size_t smd = sizeof(double) * (2 * ((size_t)n + 1) + n);
    if (smd > 227 * 1024) { err = "fourier_bessel: n too large for the on-chip sine table (n <= 9600)"; return 8; }
    const double dr = rmax / (n + 1), dk = PI / ((n + 1) * dr);
    std::vector<double> pre(n), post(n), sn(2 * (size_t)(n + 1));
    for (int j = 0; j < n; ++j) {
        const double r = (j + 1) * dr, k = (j + 1) * dk;
        pre[j] = direction == 0 ? r : k;
        post[j] = direction == 0 ? 2.0 * PI * dr / k : dk / (4.0 * PI * PI * r);
    }
    for (size_t m = 0; m < sn.size(); ++m) sn[m] = std::sin(PI * (double)m / (double)(n + 1));
    double *dx = nullptr, *dpre = nullptr, *dpost = nullptr, *dout = nullptr, *dsn = nullptr;
    int rc = 0;
    do {
        if (cudaMalloc(&dx, sizeof(double) * n) != cudaSuccess || cudaMalloc(&dpre, sizeof(double) * n) != cudaSuccess ||
            cudaMalloc(&dpost, sizeof(double) * n) != cudaSuccess || cudaMalloc(&dout, sizeof(double) * n) != cudaSuccess ||
            cudaMalloc(&dsn, sizeof(double) * sn.size()) != cudaSuccess) {
            err = "fourier_bessel: device allocation failed";
            rc = 2;
            break;
        }
        cudaError_t e = cudaMemcpy(dx, fin, sizeof(double) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dpre, pre.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dpost, post.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dsn, sn.data(), sizeof(double) * sn.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(dst_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)std::max<size_t>(smd, 48 * 1024));
        if (e == cudaSuccess) {
            dst_kernel<<<(n + 127) / 128, 128, smd>>>(dx, dpre, dpost, dout, n, dsn);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(fout, dout, sizeof(double) * n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            err = std::string("fourier_bessel: ") + cudaGetErrorString(e);
            rc = 7;
        }
    } while (0);
    cudaFree(dx); cudaFree(dpre); cudaFree(dpost); cudaFree(dout); cudaFree(dsn);
    return rc;
}

static int run_direct(HncDev &d, const Potential &pot, double n0, double rmax, double tol, double mix,
                      int maxiter, const double *gamma_s_init, HncOut &res, bool &unstable_out,
                      std::string &err)
{
    const int n = d.n;
    const int tb = 256, gb = (n + tb - 1) / tb;
    const double dr = rmax / (n + 1), dk = PI / ((n + 1) * dr);
    std::vector<double> r(n), k(n), bvs(n), bvlk(n), bvlr(n), prer(n), postr(n), prek(n), postk(n), gkmf(n);
    for (int j = 0; j < n; ++j) {
        r[j] = (j + 1) * dr;
        k[j] = (j + 1) * dk;
        bvs[j] = pot_beta_v(pot, r[j]) - pot_long_r(pot, r[j]);
        bvlr[j] = pot_long_r(pot, r[j]);
        bvlk[j] = pot_long_k(pot, k[j]);
        prer[j] = r[j];                        // fb_r2k: f(k) = 2 pi dr DST(r f)/k
        postr[j] = 2.0 * PI * dr / k[j];
        prek[j] = k[j];                        // fb_k2r: f(r) = dk DST(k f)/(4 pi^2 r)
        postk[j] = dk / (4.0 * PI * PI * r[j]);
        const double ck0 = -pot_beta_v_k(pot, k[j]);
        gkmf[j] = n0 * ck0 * ck0 / (1.0 - n0 * ck0) - bvlk[j];
    }
    std::vector<double> sn(2 * (n + 1));
    for (int m = 0; m < 2 * (n + 1); ++m) sn[m] = std::sin(PI * (double)m / (double)(n + 1));
    auto H2D = [&](double *dst_, const std::vector<double> &v) {
        return cudaMemcpy(dst_, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice);
    };
    CKS(H2D(d.r, r)); CKS(H2D(d.k, k)); CKS(H2D(d.bvs, bvs)); CKS(H2D(d.bvl_k, bvlk)); CKS(H2D(d.bvl_r, bvlr));
    CKS(H2D(d.pre_r2k, prer)); CKS(H2D(d.post_r2k, postr)); CKS(H2D(d.pre_k2r, prek));
    CKS(H2D(d.post_k2r, postk)); CKS(H2D(d.sintab, sn)); CKS(H2D(d.gk_mf, gkmf));
    const size_t smd = sizeof(double) * (2 * (n + 1) + n);
    CKS(cudaFuncSetAttribute(dst_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smd, 48 * 1024)));
    // initial guess: mean-field gamma_s = k2r(gk_mf) (oz_hnc.f90:175-183)
    dst(d, d.gk_mf, d.pre_k2r, d.post_k2r, d.gs);
    if (gamma_s_init) CKS(cudaMemcpy(d.gs, gamma_s_init, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    double mixc = mix;
    res.converged = false;
    double resid = 0.0;
    bool unstable = false;
    int it_total = 0;
    const int npicard = 5;
    for (int irestart = 1; irestart <= 4; ++irestart) {
        for (int i = 0; i < 3; ++i) {
            CKS(cudaMemset(d.hin[i], 0, sizeof(double) * n));
            CKS(cudaMemset(d.hout[i], 0, sizeof(double) * n));
        }
        int nhist = 0, ng_cooldown = 0;
        double resid_prev = 1.0e100;
        unstable = false;
        it_total = 0;
        for (int it = 1; it <= maxiter; ++it) {
            it_total = it;
            hnc_closure_kernel<<<gb, tb>>>(d.bvs, d.gs, d.cs, n);
            dst(d, d.cs, d.pre_r2k, d.post_r2k, d.csk);
            CKS(cudaMemsetAsync(d.flag, 0, sizeof(unsigned)));
            hnc_oz_kernel<<<gb, tb>>>(d.csk, d.bvl_k, n0, d.ck, d.gk, n, d.flag);
            dst(d, d.gk, d.pre_k2r, d.post_k2r, d.gnew);
            CKS(cudaMemsetAsync(d.umax, 0, sizeof(unsigned long long)));
            maxabsdiff_kernel<<<d.nb, tb>>>(d.gnew, d.gs, n, d.umax);
            unsigned fl = 0;
            unsigned long long um = 0;
            CKS(cudaMemcpy(&fl, d.flag, sizeof(unsigned), cudaMemcpyDeviceToHost));
            CKS(cudaMemcpy(&um, d.umax, sizeof(um), cudaMemcpyDeviceToHost));
            if (fl) { unstable = true; break; }
            std::memcpy(&resid, &um, sizeof(double));
            if (resid < tol) {
                CKS(cudaMemcpy(d.gs, d.gnew, sizeof(double) * n, cudaMemcpyDeviceToDevice));
                res.converged = true;
                break;
            }
            if (resid > 1.0e6) { unstable = true; break; }
            // history: rotate (3 <- 2 <- 1), then 1 <- current
            double *ti = d.hin[2], *to = d.hout[2];
            d.hin[2] = d.hin[1]; d.hin[1] = d.hin[0]; d.hin[0] = ti;
            d.hout[2] = d.hout[1]; d.hout[1] = d.hout[0]; d.hout[0] = to;
            CKS(cudaMemcpy(d.hin[0], d.gs, sizeof(double) * n, cudaMemcpyDeviceToDevice));
            CKS(cudaMemcpy(d.hout[0], d.gnew, sizeof(double) * n, cudaMemcpyDeviceToDevice));
            nhist = std::min(nhist + 1, 3);
            if (resid > 10.0 * resid_prev) ng_cooldown = 10;
            if (nhist == 3 && it > npicard && ng_cooldown == 0) {
                ng_dots_kernel<<<d.nb, tb>>>(d.hin[0], d.hout[0], d.hin[1], d.hout[1], d.hin[2], d.hout[2], n, d.part);
                std::vector<double> pt(5 * d.nb);
                CKS(cudaMemcpy(pt.data(), d.part, sizeof(double) * 5 * d.nb, cudaMemcpyDeviceToHost));
                double a[5] = {0, 0, 0, 0, 0};
                for (int b = 0; b < d.nb; ++b)
                    for (int i = 0; i < 5; ++i) a[i] += pt[5 * b + i];
                const double a11 = a[0], a12 = a[1], a22 = a[2], b1 = a[3], b2 = a[4];
                const double det = a11 * a22 - a12 * a12;
                bool accepted = false;
                if (std::fabs(det) > 1.0e-14 * a11 * a22 && a11 > 0.0 && a22 > 0.0) {
                    const double c1 = (b1 * a22 - b2 * a12) / det;
                    const double c2 = (a11 * b2 - a12 * b1) / det;
                    if (std::fabs(c1) < 20.0 && std::fabs(c2) < 20.0) {
                        CKS(cudaMemsetAsync(d.umax, 0, sizeof(unsigned long long)));
                        ng_try_kernel<<<d.nb, tb>>>(d.hout[0], d.hout[1], d.hout[2], c1, c2, d.bvs, d.gtry, n, d.umax);
                        unsigned long long key = 0;
                        CKS(cudaMemcpy(&key, d.umax, sizeof(key), cudaMemcpyDeviceToHost));
                        key = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
                        double mx;
                        std::memcpy(&mx, &key, sizeof(double));
                        if (mx < 40.0) {
                            CKS(cudaMemcpy(d.gs, d.gtry, sizeof(double) * n, cudaMemcpyDeviceToDevice));
                            accepted = true;
                        }
                    }
                }
                if (!accepted) mix_kernel<<<gb, tb>>>(d.gs, d.gnew, mixc, n);
            } else {
                mix_kernel<<<gb, tb>>>(d.gs, d.gnew, mixc, n);
                if (ng_cooldown > 0) ng_cooldown--;
            }
            resid_prev = resid;
        }
        if (res.converged || !unstable) break;
        mixc = 0.5 * mixc;
        dst(d, d.gk_mf, d.pre_k2r, d.post_k2r, d.gs);
        if (gamma_s_init) CKS(cudaMemcpy(d.gs, gamma_s_init, sizeof(double) * n, cudaMemcpyDeviceToDevice));
    }
    CKS(cudaGetLastError());
    res.niter = std::min(it_total, maxiter);
    res.residual = resid;
    unstable_out = unstable;
    if (unstable) return 0;
    res.nr = n;
    res.r = r;
    res.k = k;
    res.g.resize(n);
    res.ck.resize(n);
    res.sk.resize(n);
    hnc_final_kernel<<<gb, tb>>>(d.bvs, d.gs, d.gdev, d.cs, n);
    dst(d, d.cs, d.pre_r2k, d.post_r2k, d.csk);
    std::vector<double> csk(n), cs(n);
    CKS(cudaMemcpy(res.g.data(), d.gdev, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CKS(cudaMemcpy(csk.data(), d.csk, sizeof(double) * n, cudaMemcpyDeviceToHost));
    double s = 0.0;
    for (int j = 0; j < n; ++j) {
        res.ck[j] = csk[j] - bvlk[j];
        const double hk = res.ck[j] / (1.0 - n0 * res.ck[j]);
        res.sk[j] = 1.0 + n0 * hk;
        s += r[j] * r[j] * (res.g[j] - 1.0) * pot_beta_v(pot, r[j]);
    }
    res.u_ex = 2.0 * PI * n0 * (dr * s);
    return 0;
}

// hnc_solve (oz_hnc.f90:111-140): direct solve, else Gamma continuation.
int gpu_hnc_solve(int device, const Potential &pot, double n0, int nr, double rmax, double tol, double mix,
                  int maxiter, HncOut &res, std::string &err)
{
    CKS(cudaSetDevice(device));
    if (nr < 2) { err = "hnc: nr must be >= 2"; return 1; }
    const size_t smd = sizeof(double) * (2 * (nr + 1) + nr);
    if (smd > 227 * 1024) { err = "hnc: nr too large for the on-chip sine table (nr <= 9600)"; return 8; }
    HncDev d;
    if (int rc = hnc_alloc(d, nr, err)) return rc;
    bool unstable = false;
    res = HncOut();
    if (int rc = run_direct(d, pot, n0, rmax, tol, mix, maxiter, nullptr, res, unstable, err)) return rc;
    if (!unstable) return 0;
    Potential p = pot;
    const double gtarget = pot.gamma;
    double g = std::min(gtarget, 2.0);
    double *init = nullptr;
    if (cudaMalloc(&init, sizeof(double) * nr) != cudaSuccess) { err = "hnc alloc"; return 2; }
    cudaMemset(init, 0, sizeof(double) * nr);
    int rc = 0;
    for (int istep = 1; istep <= 200; ++istep) {
        p.gamma = g;
        res = HncOut();
        rc = run_direct(d, p, n0, rmax, tol, mix, maxiter, init, res, unstable, err);
        if (rc) break;
        if (unstable) {
            err = "hnc: continuation in Gamma failed";
            rc = 9;
            break;
        }
        cudaMemcpy(init, d.gs, sizeof(double) * nr, cudaMemcpyDeviceToDevice);
        if (g >= gtarget) break;
        g = std::min(gtarget, g * 1.3);
    }
    cudaFree(init);
    return rc;
}

}  // namespace hydft
