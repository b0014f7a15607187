// Device solver for one simulation (included once per precision): buffers, transform pipelines and the
// per-stage kernel sequence of the RK3 step.
//
// Per RK stage (model.f90:192-223 restated on a spectral-resident state):
//   phase A  inverse: dn, m_d [, grad n, lap n]   pointwise: u, m_i u_j, mu_local
//            forward: u_d, m_i u_j (i<=j), mu_local
//            combine A: mu-hat, -div(m u) + div Pi (partial dmom), Pi0 and
//                       the previous stage's Maxwell relaxation
//   phase B  inverse: d mu/dx_d [, d Pi_c/dx_d]   pointwise: n (dmu - F_ext),
//            -u.grad Pi_c   forward: those
//            combine B: dn, dmom, dPi and the low-storage RK update
// Linear operators (divergences, Pi0 and its divergence, hartree and RY
// convolutions, dealiasing, the RK update and the relaxation) act on the
// spectral state; only the nonlinear products are transformed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "passes_fast.cuh"
#include "solver.hpp"

#include <type_traits>

namespace hydft {

#define CK(call)                                                                 \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return HYDFT_E_CUDA;                                                 \
        }                                                                        \
    } while (0)

enum { HYDFT_E_OK = 0, HYDFT_E_BAD = 1, HYDFT_E_OOM = 2, HYDFT_E_NONPOS = 3, HYDFT_E_NONFINITE = 4,
       HYDFT_E_NEWTON = 5, HYDFT_E_CUDA = 7, HYDFT_E_UNSUPPORTED = 8 };

// reduction partials of the diagnostics kernel
struct RedPart {
    double sn, cn_, sm[3], cm[3], sk, ck, nmin, nmax, umax;
};

template <typename R>
__device__ __forceinline__ void neumaier(double &s, double &c, double v)
{
    const double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v;
    else c += (v - t) + s;
    s = t;
}

// FP64 compensated sums of n, m_d, m_d^2/n and extrema over the real-space
// fields; one partial per block, combined in a fixed order by reduce_final.
template <typename R>
__global__ void reduce_fields_kernel(const R *dn, const R *m, size_t ncell, int nm, const double *nmean,
                                     double inv_mass, RedPart *part)
{
    __shared__ RedPart sh[8];
    const double nref = *nmean;
    RedPart p;
    p.sn = p.cn_ = p.sk = p.ck = 0.0;
    for (int d = 0; d < 3; ++d) p.sm[d] = p.cm[d] = 0.0;
    p.nmin = 1e300; p.nmax = -1e300; p.umax = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ncell; q += (size_t)gridDim.x * blockDim.x) {
        const double n = nref + (double)dn[q];
        neumaier<R>(p.sn, p.cn_, n);
        p.nmin = fmin(p.nmin, n);
        p.nmax = fmax(p.nmax, n);
        for (int d = 0; d < nm; ++d) {
            const double md = (double)m[d * ncell + q];
            neumaier<R>(p.sm[d], p.cm[d], md);
            neumaier<R>(p.sk, p.ck, md * md / n);
            p.umax = fmax(p.umax, fabs(md * inv_mass / n));
        }
    }
    // warp reduction (compensation terms folded into the sums)
    double v[9] = {p.sn + p.cn_, p.sm[0] + p.cm[0], p.sm[1] + p.cm[1], p.sm[2] + p.cm[2], p.sk + p.ck,
                   p.nmin, p.nmax, p.umax, 0.0};
    for (int off = 16; off > 0; off >>= 1) {
        for (int i = 0; i < 5; ++i) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
        v[5] = fmin(v[5], __shfl_down_sync(0xffffffffu, v[5], off));
        v[6] = fmax(v[6], __shfl_down_sync(0xffffffffu, v[6], off));
        v[7] = fmax(v[7], __shfl_down_sync(0xffffffffu, v[7], off));
    }
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) {
        sh[w].sn = v[0]; sh[w].sm[0] = v[1]; sh[w].sm[1] = v[2]; sh[w].sm[2] = v[3]; sh[w].sk = v[4];
        sh[w].nmin = v[5]; sh[w].nmax = v[6]; sh[w].umax = v[7];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        RedPart o = sh[0];
        o.cn_ = o.ck = 0.0;
        for (int d = 0; d < 3; ++d) o.cm[d] = 0.0;
        const int nw = blockDim.x / 32;
        for (int i = 1; i < nw; ++i) {
            neumaier<R>(o.sn, o.cn_, sh[i].sn);
            for (int d = 0; d < 3; ++d) neumaier<R>(o.sm[d], o.cm[d], sh[i].sm[d]);
            neumaier<R>(o.sk, o.ck, sh[i].sk);
            o.nmin = fmin(o.nmin, sh[i].nmin);
            o.nmax = fmax(o.nmax, sh[i].nmax);
            o.umax = fmax(o.umax, sh[i].umax);
        }
        part[blockIdx.x] = o;
    }
}

template <typename R>
__global__ void reduce_final_kernel(const RedPart *part, int nb, RedPart *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    RedPart o;
    o.sn = o.cn_ = o.sk = o.ck = 0.0;
    for (int d = 0; d < 3; ++d) o.sm[d] = o.cm[d] = 0.0;
    o.nmin = 1e300; o.nmax = -1e300; o.umax = 0.0;
    for (int b = 0; b < nb; ++b) {
        neumaier<R>(o.sn, o.cn_, part[b].sn);
        neumaier<R>(o.sn, o.cn_, part[b].cn_);
        for (int d = 0; d < 3; ++d) {
            neumaier<R>(o.sm[d], o.cm[d], part[b].sm[d]);
            neumaier<R>(o.sm[d], o.cm[d], part[b].cm[d]);
        }
        neumaier<R>(o.sk, o.ck, part[b].sk);
        neumaier<R>(o.sk, o.ck, part[b].ck);
        o.nmin = fmin(o.nmin, part[b].nmin);
        o.nmax = fmax(o.nmax, part[b].nmax);
        o.umax = fmax(o.umax, part[b].umax);
    }
    o.sn += o.cn_;
    for (int d = 0; d < 3; ++d) o.sm[d] += o.cm[d];
    o.sk += o.ck;
    *out = o;
}


// ------------------------------------------------ energies and force means
// Up to 6 FP64 sums per block, each compensated (Neumaier) over the block's
// grid-stride share, the lanes then combined in a fixed order: the result
// does not depend on timing.
constexpr int NSUM = 6;

__device__ __forceinline__ void block_sums(double (&v)[NSUM], double *part)
{
    __shared__ double sh[NSUM][8];
    for (int off = 16; off > 0; off >>= 1)
        for (int i = 0; i < NSUM; ++i) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0)
        for (int i = 0; i < NSUM; ++i) sh[i][w] = v[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x / 32;
        for (int i = 0; i < NSUM; ++i) {
            double a = 0.0, c = 0.0;
            for (int j = 0; j < nw; ++j) neumaier<double>(a, c, sh[i][j]);
            part[blockIdx.x * NSUM + i] = a + c;
        }
    }
}

static __global__ void sums_final_kernel(const double *part, int nb, double *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < NSUM; ++i) {
        double a = 0.0, c = 0.0;
        for (int b = 0; b < nb; ++b) neumaier<double>(a, c, part[b * NSUM + i]);
        out[i] = a + c;
    }
}

// Hartree and RY energies by Parseval on the band, k != 0:
// sums of w |n_k|^2 v(k) and w |n_k|^2 c_cor(k), w = 1 at kx = 0, else 2
template <typename R>
__global__ void energy_spec_kernel(Grid g, const cplx<R> *N, const R *Kh, const R *Kr, double *part)
{
    const size_t total = (size_t)g.nkzc * g.nkyc * g.pkx;
    double a[2] = {0.0, 0.0}, c[2] = {0.0, 0.0};
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        int kxc, kyc, kzc;
        kvec(g, idx, kxc, kyc, kzc);
        if (kxc >= g.nkxc || (kxc == 0 && kyc == 0 && kzc == 0)) continue;
        const double w = kxc == 0 ? 1.0 : 2.0;
        const double re = (double)N[idx].x, im = (double)N[idx].y;
        const double a2 = w * (re * re + im * im);
        if (Kh) neumaier<double>(a[0], c[0], a2 * (double)Kh[idx]);
        if (Kr) neumaier<double>(a[1], c[1], a2 * (double)Kr[idx]);
    }
    double v[NSUM] = {a[0] + c[0], a[1] + c[1], 0.0, 0.0, 0.0, 0.0};
    block_sums(v, part);
}

// Real-space sums over the grid: 2 ideal n(ln n - 1), 3 TF n alpha -
// (2/3) c_n I_{3/2}(alpha), 4 gradient xi(alpha) |grad n|^2, 5 external n v
struct EnergyReal {
    double nref;
    const double *fdtab;
    double cn;
    int ideal, tf, grad, ext;      // ext: 0 none, 1 plane wave, 2 gaussian
    const cplx<double> *ex, *ey, *ez;
    const Ctrl *ctrl;
};

template <typename R>
__global__ void energy_real_kernel(Grid g, const R *dn, const R *gn, const R *gv, size_t ncell, EnergyReal e,
                                   double *part)
{
    double a[4] = {0.0, 0.0, 0.0, 0.0}, c[4] = {0.0, 0.0, 0.0, 0.0};
    double vamp = 0.0, vr = 1.0, vi = 0.0;
    if (e.ext == 1) {
        vamp = e.ctrl->v_amp;
        vr = e.ctrl->v_ewr;
        vi = e.ctrl->v_ewi;
    }
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ncell; q += (size_t)gridDim.x * blockDim.x) {
        const double n = e.nref + (double)dn[q];
        if (e.ideal) neumaier<double>(a[0], c[0], n * (log(n) - 1.0));
        if (e.tf || e.grad) {
            bool ok = true;
            const double al = fd::alpha_from_ip12(e.fdtab, n / e.cn, &ok);
            if (e.tf) neumaier<double>(a[1], c[1], n * al - (2.0 / 3.0) * e.cn * fd::ip32(e.fdtab, al));
            if (e.grad) {
                double g2 = 0.0;
                for (int d = 0; d < 3; ++d) {
                    const double gd = (double)gn[d * ncell + q];
                    g2 += gd * gd;
                }
                neumaier<double>(a[2], c[2], fd::xi(e.fdtab, al) * g2);
            }
        }
        if (e.ext == 1) {
            const int x = (int)(q % g.nx), y = (int)((q / g.nx) % g.ny), z = (int)(q / ((size_t)g.nx * g.ny));
            cplx<double> ph = e.ex[x] * e.ey[y];
            ph = ph * e.ez[z];
            const double v = vamp * (ph.x * vr - ph.y * vi);
            neumaier<double>(a[3], c[3], n * v);
        } else if (e.ext == 2) {
            neumaier<double>(a[3], c[3], n * (double)gv[q]);
        }
    }
    double v[NSUM] = {0.0, 0.0, a[0] + c[0], a[1] + c[1], a[2] + c[2], a[3] + c[3]};
    block_sums(v, part);
}

// mean of n F for the gaussian potential, F = -grad v:
// sum over the band of w k_i Im(conj(n_k) v_k)
template <typename R>
__global__ void gauss_force_mean_kernel(Grid g, const cplx<R> *N, const cplx<R> *V, double *part)
{
    const size_t total = (size_t)g.nkzc * g.nkyc * g.pkx;
    double a[3] = {0.0, 0.0, 0.0}, c[3] = {0.0, 0.0, 0.0};
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        int kxc, kyc, kzc;
        kvec(g, idx, kxc, kyc, kzc);
        if (kxc >= g.nkxc) continue;
        const double w = kxc == 0 ? 1.0 : 2.0;
        const double nr = (double)N[idx].x, ni = (double)N[idx].y;
        const double vr = (double)V[idx].x, vi = (double)V[idx].y;
        const double im = nr * vi - ni * vr;   // Im(conj(n) v)
        const double k[3] = {kxc * g.kx0, signed_idx(kyc, g.My) * g.ky0, signed_idx(kzc, g.Mz) * g.kz0};
        for (int d = 0; d < 3; ++d) neumaier<double>(a[d], c[d], w * k[d] * im);
    }
    double v[NSUM] = {a[0] + c[0], a[1] + c[1], a[2] + c[2], 0.0, 0.0, 0.0};
    block_sums(v, part);
}

static __global__ void gauss_force_final_kernel(const double *part, int nb, Ctrl *ctrl)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < 3; ++i) {
        double a = 0.0, c = 0.0;
        for (int b = 0; b < nb; ++b) neumaier<double>(a, c, part[b * NSUM + i]);
        ctrl->gf[i] = a + c;
    }
}

// FP64 compensated sum, minimum and count of non-finite values of x[0..n)
// per block, into part[block * NSUM + 0 / 1 / 2]
static __global__ void density_stats_kernel(const double *x, size_t n, double *part)
{
    double a = 0.0, c = 0.0, mn = 1e300, bad = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const double v = x[q];
        if (!isfinite(v)) bad += 1.0;
        neumaier<double>(a, c, v);
        mn = fmin(mn, v);
    }
    __shared__ double sh[3][8];
    double s = a + c;
    for (int off = 16; off > 0; off >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, off);
        mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, off));
        bad += __shfl_down_sync(0xffffffffu, bad, off);
    }
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) { sh[0][w] = s; sh[1][w] = mn; sh[2][w] = bad; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0, tc = 0.0, m = 1e300, b = 0.0;
        for (int j = 0; j < (int)(blockDim.x / 32); ++j) {
            neumaier<double>(t, tc, sh[0][j]);
            m = fmin(m, sh[1][j]);
            b += sh[2][j];
        }
        part[blockIdx.x * NSUM + 0] = t + tc;
        part[blockIdx.x * NSUM + 1] = m;
        part[blockIdx.x * NSUM + 2] = b;
    }
}

template <typename R>
__global__ void fill_real_kernel(R *dst, const double *src, double sub, size_t n)
{
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        dst[q] = R(src[q] - sub);
}

template <typename R>
__global__ void real_to_double_kernel(double *dst, const R *src, double add, size_t n)
{
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
        dst[q] = (double)src[q] + add;
}

template <typename R>
__global__ void set_k0_kernel(cplx<R> *a, double re)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) a[0] = cplx<R>{R(re), R(0)};
}

template <typename R>
static void make_twiddles(int L, std::vector<cplx<R>> &tw)
{
    tw.resize(std::max(L, 1));
    const double pi = 3.14159265358979323846264338327950288;
    for (int t = 0; t < L; ++t) {
        const double a = -2.0 * pi * (double)t / (double)L;
        tw[t] = cplx<R>{R(std::cos(a)), R(std::sin(a))};
    }
    if (L >= 4 && L % 4 == 0) {     // exact values at the quarter points
        tw[0] = cplx<R>{R(1), R(0)};
        tw[L / 4] = cplx<R>{R(0), R(-1)};
        tw[L / 2] = cplx<R>{R(-1), R(0)};
        tw[3 * L / 4] = cplx<R>{R(0), R(1)};
    }
}

// Calls f(integral_constant<T>, integral_constant<E>) for an axis length
// with a register FFT plan; returns false otherwise.
template <class F>
static bool with_plan(int L, F &&f)
{
    using std::integral_constant;
    switch (L) {
    case 32: f(integral_constant<int, 4>{}, integral_constant<int, 8>{}); return true;
    case 48: f(integral_constant<int, 4>{}, integral_constant<int, 12>{}); return true;
    case 64: f(integral_constant<int, 8>{}, integral_constant<int, 8>{}); return true;
    case 96: f(integral_constant<int, 4>{}, integral_constant<int, 24>{}); return true;
    case 128: f(integral_constant<int, 8>{}, integral_constant<int, 16>{}); return true;
    case 256: f(integral_constant<int, 16>{}, integral_constant<int, 16>{}); return true;
    default: return false;
    }
}

static bool has_plan(int L)
{
    return L == 32 || L == 48 || L == 64 || L == 96 || L == 128 || L == 256;
}

// The ensemble form of pack P's kernel for n simulations whose packs lie
// back to back at `packs` (host memory; LaunchRec::launch): one launch per
// PackSet<P>::N simulations, each carrying its packs as its parameter
template <class P>
void ensemble_launch(const void *packs, unsigned n, dim3 grid, dim3 block, size_t smem, cudaStream_t st)
{
    static_assert(std::is_trivially_copyable<P>::value, "a pack is copied as bytes");
    const unsigned char *src = static_cast<const unsigned char *>(packs);
    for (unsigned c = 0; c < n; c += PackSet<P>::N) {
        const unsigned k = std::min<unsigned>(PackSet<P>::N, n - c);
        PackSet<P> set;
        std::memset(static_cast<void *>(&set), 0, sizeof(set));
        std::memcpy(static_cast<void *>(set.p), src + (size_t)c * sizeof(P), (size_t)k * sizeof(P));
        ensemble_kernel<P><<<dim3(grid.x, grid.y, grid.z * k), block, smem, st>>>(set, grid.z);
    }
}

// Raises a kernel's dynamic shared-memory limit to all that the current
// device allows beside the kernel's static shared memory.  The limit only
// caps what a launch may ask for (occupancy follows each launch's own
// size), and it is never set lower: one kernel serves simulations whose
// blocks differ in size (the tuner picks the threads per block for each
// grid), and a limit fitted to one of them would make another's launch, or
// a graph captured with it, invalid.  Fails when `need` does not fit.
inline cudaError_t raise_smem_limit(const void *func, size_t need)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, func);
    if (e != cudaSuccess) return e;
    if ((size_t)optin < fa.sharedSizeBytes || need > (size_t)optin - fa.sharedSizeBytes) return cudaErrorInvalidValue;
    if ((size_t)fa.maxDynamicSharedSizeBytes >= (size_t)optin - fa.sharedSizeBytes) return cudaSuccess;
    return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

// the dynamic shared-memory limit of the ensemble form, set for every
// launch shape (the default limit is 48 KB)
template <class P>
cudaError_t ensemble_prepare(size_t smem)
{
    return raise_smem_limit(reinterpret_cast<const void *>(&ensemble_kernel<P>), smem);
}

template <typename R>
class Solver : public SolverBase {
public:
    static constexpr int TX = sizeof(R) == 4 ? 16 : 8;
    SolverSetup S;
    Grid g;
    Phys ph;
    int nm;
    int device;
    size_t csize, zsize, ysize, ncell;
    int nin_max, nout_max;
    cudaStream_t st = nullptr;
    std::vector<void *> allocs;
    // compact fields
    cplx<R> *N, *M[3], *P[6], *RN, *RM[3], *RP[6], *P0[6], *MU, *Q[3];
    cplx<R> *OA[16], *OB[12];       // phase outputs (compact)
    cplx<R> *HN, *HM[3], *HP[6];    // rhs-only outputs
    cplx<R> *zi, *yi, *xo;          // pass buffers
    R *dn_real, *u_real, *io_real;  // real-space fields
    R *Klin;
    double *fdtab = nullptr;
    cplx<double> *ex, *ey, *ez;
    cplx<R> *twx, *twy, *twz;
    cplx<R> *tpx = nullptr, *tpy = nullptr, *tpz = nullptr;   // planned tables of the register passes
    R *Kh = nullptr, *Kr = nullptr;        // hartree v(k), RY c_cor(k) on the band (energy)
    R *gV = nullptr, *gG = nullptr;        // gaussian potential and its gradient (3 fields), real space
    cplx<R> *Vg = nullptr;                 // gaussian potential on the band
    double *spart = nullptr, *sout = nullptr;   // block partials and results of the 6-sum reductions
    double *stage = nullptr;                    // one FP64 field: host copies pass through it
    double *pring = nullptr;                    // probe records (5 doubles each)
    int *pcount = nullptr;
    long long pidx = -1;
    int pconj = 0;
    static constexpr int PROBE_CAP = 4096;
    Ctrl *ctrl;
    RedPart *rpart, *rout;
    int red_blocks = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int xrb_a = 1, xrb_b = 1, xrb_io = 1;
    int smem_optin = 0;
    bool host_pending = false;   // a Maxwell relaxation waits for u of the new state
    bool fast_x = false;         // x passes on the register FFT (3-D grids, planned nx)
    bool staged_x = true;        // xa_regs / xb_rows (HYDFT_XPASS=v1 selects xa_fast / xb_fast)
    // the axis's band limit is the two-thirds rule's (L - 1) / 3, so the
    // register-FFT passes classify band elements at compile time
    // (HYDFT_BAND=0 selects the runtime test everywhere)
    bool band_x = false, band_y = false, band_z = false;
    // ky rows per thread in the inverse z pass (HYDFT_ZNB) and the forward
    // one (HYDFT_ZNB_FWD=2 for two; at 256^3 two rows made the forward 4 %
    // slower, same-box A/B).  Inverse: one on the plain path (its
    // output tile then goes out by one tensor store), two in the ensemble
    // forms (all loads in flight at once); HYDFT_ZNB = 1 | 2 sets both
    int z_nb = 1, z_nb_ens = 2, z_nbf = 1;
    // the y inverse, y forward and z forward passes of the plain path read
    // each block's input tile with one TMA tensor load (HYDFT_TMA=0: every
    // thread loads its own elements, as the ensemble forms always do; the
    // fields are the same to the bit either way)
    bool use_tma = true;
    // the z inverse pass's tensor load (HYDFT_TMA_ZINV=0 switches it off):
    // with one row per thread its tile goes into the exchange space; with two
    // (HYDFT_ZNB=2) it does not fit there, and the extra shared memory cost
    // blocks per SM (256^3 step 6.17 against 6.06 ms without the load)
    bool tma_zinv = true;
    // tensor stores of the output tiles on the plain path: y inverse, y
    // forward, z forward, z inverse with one row per thread
    // (HYDFT_TMA_YST / _YFST / _ZFST / _ZIST = 0 switch them off)
    bool tma_yst = true, tma_yfst = true, tma_zfst = true, tma_zist = true;

    // field coordinates of the pass inputs in[0..nf-1] within the buffer
    // base (fields `stride` complex values apart), for a TMA tensor map
    TmaFields tma_fields(const cplx<R> *const *in, int nf, const cplx<R> *base, size_t stride)
    {
        TmaFields tf;
        for (int f = 0; f < MAXF; ++f) {
            tf.src[f] = f < nf ? (int)((in[f] - base) / (ptrdiff_t)stride) : 0;
            tf.dst[f] = 0;
        }
        tf.status = &ctrl->status;
        return tf;
    }
    // tile shapes picked by tune(): kx columns per y/z block, threads per x block
    int yz_tx = sizeof(R) == 4 ? 16 : 8;      // inverse y/z passes
    int yz_nt = sizeof(R) == 4 ? 256 : 128;
    int yz_txf = sizeof(R) == 4 ? 16 : 8;     // forward y/z passes
    int yz_ntf = sizeof(R) == 4 ? 256 : 128;
    int x_ntmax = 256;
    bool tuned = false;
    size_t alloc_bytes = 0;      // device memory allocated by this solver
    int num_sms = 148;

    // per-kernel CUDA-event timing (profile mode, uncaptured steps only)
    struct KStat {
        std::string name;
        double ms = 0.0, bytes = 0.0;
        int64_t n = 0;
    };
    std::vector<KStat> kstats;
    struct EvRec {
        int k;
        cudaEvent_t a, b;
    };
    std::vector<EvRec> evrecs;
    bool profiling = false;

    // set while record_step runs: launches are recorded, not run
    std::vector<LaunchRec> *rec = nullptr;
    bool rec_ok = true;
    // this solver's step packs (the ensemble-of-one form of its step)

    template <class F>
    void launch(const char *name, double bytes, F &&f)
    {
        if (rec) {   // a launch without an ensemble form
            rec_ok = false;
            return;
        }
        cudaEvent_t a = nullptr, b = nullptr;
        if (profiling) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, st);
        }
        f();
        launches++;
        if (profiling) {
            cudaEventRecord(b, st);
            int k = -1;
            for (size_t i = 0; i < kstats.size(); ++i)
                if (kstats[i].name == name) k = (int)i;
            if (k < 0) {
                kstats.push_back(KStat());
                kstats.back().name = name;
                k = (int)kstats.size() - 1;
            }
            kstats[k].bytes += bytes;
            kstats[k].n += 1;
            evrecs.push_back({k, a, b});
        }
    }

    // a launch with an ensemble form: pack P holds its arguments, f runs the
    // plain kernel
    template <class P, class F>
    void launch_p(const char *name, double bytes, dim3 grid, dim3 block, size_t smem, const P &pack, F &&f)
    {
        if (rec) {
            LaunchRec r;
            r.kind = reinterpret_cast<const void *>(&ensemble_launch<P>);
            r.name = name;
            r.bytes = bytes;
            r.grid = grid;
            r.block = block;
            r.smem = smem;
            r.pack.resize(sizeof(P));
            std::memcpy(r.pack.data(), &pack, sizeof(P));
            r.per_launch = PackSet<P>::N;
            r.launch = &ensemble_launch<P>;
            r.prepare = &ensemble_prepare<P>;
            rec->push_back(std::move(r));
            return;
        }
        launch(name, bytes, f);
    }

    double cb() const { return 2.0 * sizeof(R); }   // bytes of one complex value

    int precision_bits() const override { return sizeof(R) * 8; }
    void set_ext_omega(double w) override
    {
        S.ext_omega = w;
        ph.ext_omega = w;
        ++graph_gen;
        if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
        if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
    }
    const SolverSetup &setup() const override { return S; }
    void *stream() override { return (void *)st; }

    ~Solver() override
    {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (void *p : allocs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }

    template <typename T>
    int alloc(T *&p, size_t n)
    {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) {
            err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
            return HYDFT_E_OOM;
        }
        allocs.push_back(q);
        alloc_bytes += std::max<size_t>(n, 1) * sizeof(T);
        p = static_cast<T *>(q);
        return 0;
    }

    int init(const SolverSetup &s, int dev)
    {
        S = s;
        g = s.g;
        nm = s.nm;
        device = dev;
        CK(cudaSetDevice(dev));
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        int optin = 0;
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        smem_optin = optin;
        std::memset(&ph, 0, sizeof(ph));
        ph.beta = s.beta; ph.inv_beta = 1.0 / s.beta; ph.mass = s.mass; ph.inv_mass = 1.0 / s.mass;
        ph.n0 = s.n0;
        ph.nterms_local = s.nterms_local;
        for (int i = 0; i < 8; ++i) ph.term_order[i] = s.term_order[i];
        for (int i = 0; i < s.nterms_local; ++i) {
            if (s.term_order[i] == 1) ph.has_ideal = 1;
            if (s.term_order[i] == 2) ph.has_tf = 1;
            if (s.term_order[i] == 3) ph.has_grad = 1;
        }
        ph.cn = s.cn; ph.cg = s.cg; ph.alpha_ref = s.alpha_ref;
        ph.evolve = s.evolve; ph.newtonian = s.newtonian;
        ph.eta = s.eta; ph.xi = s.xi; ph.tau = s.tau;
        ph.ext_active = s.ext_active; ph.ext_kind = s.ext_kind;
        for (int d = 0; d < 3; ++d) ph.ext_k[d] = s.ext_k[d];
        ph.ext_amp = s.ext_amp; ph.ext_omega = s.ext_omega; ph.ext_ramp = s.ext_ramp;
        ph.drive_in_band = s.drive_in_band; ph.drive_idx = s.drive_idx; ph.drive_conj = s.drive_conj;

        csize = (size_t)g.nkzc * g.nkyc * g.pkx;
        if (csize >= ((size_t)1 << 31)) { err = "grid too large: 2^31 or more band modes"; return HYDFT_E_BAD; }
        zsize = (size_t)g.nz * g.nkyc * g.pkx;
        ysize = (size_t)g.nz * g.ny * g.pkx;
        ncell = (size_t)g.nx * g.ny * g.nz;
        const int ngrad = (ph.has_tf || ph.has_grad) && ph.has_grad ? nm + 1 : 0;
        const int ninA = 1 + nm + ngrad;
        const int noutA = nm + nm * (nm + 1) / 2 + 1;
        const int ninB = nm + (ph.evolve ? 6 * nm : 0);
        const int noutB = nm + (ph.evolve ? 6 : 0);
        nin_max = std::max({ninA, ninB, 10});
        nout_max = std::max({noutA, noutB, 10});
        // compact fields: N M3 P6 RN RM3 RP6 P0_6 MU Q3 OA16 OB12 HN HM3 HP6
        const int ncf = 1 + 3 + 6 + 1 + 3 + 6 + 6 + 1 + 3 + 16 + 12 + 1 + 3 + 6;
        cplx<R> *cb;
        if (int rc = alloc(cb, ncf * csize)) return rc;
        CK(cudaMemset(cb, 0, ncf * csize * sizeof(cplx<R>)));
        cplx<R> *p = cb;
        auto take = [&]() { cplx<R> *r = p; p += csize; return r; };
        N = take();
        for (auto &x : M) x = take();
        for (auto &x : P) x = take();
        RN = take();
        for (auto &x : RM) x = take();
        for (auto &x : RP) x = take();
        for (auto &x : P0) x = take();
        MU = take();
        for (auto &x : Q) x = take();
        for (auto &x : OA) x = take();
        for (auto &x : OB) x = take();
        HN = take();
        for (auto &x : HM) x = take();
        for (auto &x : HP) x = take();
        if (int rc = alloc(zi, (size_t)nin_max * zsize)) return rc;
        if (g.ny > 1) {
            if (int rc = alloc(yi, (size_t)nin_max * ysize)) return rc;
        } else {
            yi = zi;   // y transform of length 1: ZI and YI layouts coincide
        }
        if (int rc = alloc(xo, (size_t)nout_max * ysize)) return rc;
        if (int rc = alloc(dn_real, ncell)) return rc;
        if (int rc = alloc(u_real, 3 * ncell)) return rc;
        if (int rc = alloc(io_real, 10 * ncell)) return rc;
        if (int rc = alloc(stage, ncell)) return rc;   // FP64 staging of host fields
        CK(cudaMemset(u_real, 0, 3 * ncell * sizeof(R)));
        if (int rc = alloc(Klin, csize)) return rc;
        {
            std::vector<R> kl(csize, R(0));
            for (size_t i = 0; i < csize && i < s.klin.size(); ++i) kl[i] = R(s.klin[i]);
            CK(cudaMemcpy(Klin, kl.data(), csize * sizeof(R), cudaMemcpyHostToDevice));
        }
        if (!s.fdtab.empty()) {
            if (int rc = alloc(fdtab, s.fdtab.size())) return rc;
            CK(cudaMemcpy(fdtab, s.fdtab.data(), s.fdtab.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
        auto up_c = [&](cplx<double> *&dst, const std::vector<std::complex<double>> &v, int n) -> int {
            if (int rc = alloc(dst, n)) return rc;
            std::vector<cplx<double>> h(n, cplx<double>{1.0, 0.0});
            for (int i = 0; i < n && i < (int)v.size(); ++i) h[i] = cplx<double>{v[i].real(), v[i].imag()};
            CK(cudaMemcpy(dst, h.data(), n * sizeof(cplx<double>), cudaMemcpyHostToDevice));
            return 0;
        };
        if (int rc = up_c(ex, s.ex, g.nx)) return rc;
        if (int rc = up_c(ey, s.ey, g.ny)) return rc;
        if (int rc = up_c(ez, s.ez, g.nz)) return rc;
        auto up_tw = [&](cplx<R> *&dst, int L) -> int {
            std::vector<cplx<R>> tw;
            make_twiddles<R>(L, tw);
            if (int rc = alloc(dst, tw.size())) return rc;
            CK(cudaMemcpy(dst, tw.data(), tw.size() * sizeof(cplx<R>), cudaMemcpyHostToDevice));
            return 0;
        };
        if (int rc = up_tw(twx, g.nx)) return rc;
        if (int rc = up_tw(twy, g.ny)) return rc;
        if (int rc = up_tw(twz, g.nz)) return rc;
        // register-pass tables: W_L^{t k2} at [k2 T + t], then W_L^{k2 m1} at
        // [L + m1 E + k2], entries of the W_L table above
        auto up_tp = [&](cplx<R> *&dst, int L) -> int {
            int rc = 0;
            with_plan(L, [&](auto Tc, auto Ec) {
                constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
                std::vector<cplx<R>> tw, tp(2 * (size_t)L);
                make_twiddles<R>(L, tw);
                for (int k2 = 0; k2 < E; ++k2)
                    for (int t = 0; t < T; ++t) tp[k2 * T + t] = tw[(t * k2) % L];
                for (int m1 = 0; m1 < T; ++m1)
                    for (int k2 = 0; k2 < E; ++k2) tp[L + m1 * E + k2] = tw[(k2 * m1) % L];
                if ((rc = alloc(dst, tp.size()))) return;
                const cudaError_t e = cudaMemcpy(dst, tp.data(), tp.size() * sizeof(cplx<R>), cudaMemcpyHostToDevice);
                if (e != cudaSuccess) {
                    err = std::string("cudaMemcpy (register-pass twiddles): ") + cudaGetErrorString(e);
                    rc = HYDFT_E_CUDA;
                }
            });
            return rc;
        };
        if (int rc = up_tp(tpx, g.nx)) return rc;
        if (int rc = up_tp(tpy, g.ny)) return rc;
        if (int rc = up_tp(tpz, g.nz)) return rc;
        if (int rc = alloc(ctrl, 1)) return rc;
        {
            Ctrl c;
            std::memset(&c, 0, sizeof(c));
            // vext_t%setup evaluates the potential at t = 0 (external_potential.f90:56)
            c.v_amp = (s.ext_td && s.ext_ramp > 0.0) ? 0.0 : s.ext_amp;
            c.v_ewr = 1.0;
            c.v_ewi = 0.0;
            c.nmean = s.n0;
            CK(cudaMemcpy(ctrl, &c, sizeof(c), cudaMemcpyHostToDevice));
        }
        red_blocks = 2 * 148;
        if (int rc = alloc(rpart, red_blocks)) return rc;
        if (int rc = alloc(rout, 1)) return rc;
        if (int rc = alloc(spart, (size_t)red_blocks * NSUM)) return rc;
        if (int rc = alloc(sout, NSUM)) return rc;
        auto up_band = [&](R *&dst, const std::vector<double> &v) -> int {
            if (v.empty()) return 0;
            if (int rc = alloc(dst, csize)) return rc;
            std::vector<R> h(csize, R(0));
            for (size_t i = 0; i < csize && i < v.size(); ++i) h[i] = R(v[i]);
            CK(cudaMemcpy(dst, h.data(), csize * sizeof(R), cudaMemcpyHostToDevice));
            return 0;
        };
        if (int rc = up_band(Kh, s.kh)) return rc;
        if (int rc = up_band(Kr, s.kr)) return rc;
        // x-pass rows per block
        xrb_a = pick_rb(ninA, noutA);
        xrb_b = pick_rb(ninB, noutB);
        xrb_io = pick_rb(10, 10);
        if (int rc = set_smem_attrs()) return rc;
        fast_x = has_plan(g.nx) && nm == 3;
        {
            const char *ev = std::getenv("HYDFT_XPASS");
            if (ev && std::string(ev) == "v1") staged_x = false;
            const char *zn = std::getenv("HYDFT_ZNB");
            if (zn && (std::string(zn) == "1" || std::string(zn) == "2")) z_nb = z_nb_ens = std::atoi(zn);
            const char *znf = std::getenv("HYDFT_ZNB_FWD");
            if (znf && std::string(znf) == "2") z_nbf = 2;
            const char *et = std::getenv("HYDFT_TMA");
            if (et && std::string(et) == "0") use_tma = false;
            const char *ez = std::getenv("HYDFT_TMA_ZINV");
            if (ez && *ez) tma_zinv = std::string(ez) == "1";
            auto flag = [](const char *name, bool &v) {
                const char *e = std::getenv(name);
                if (e && *e) v = std::string(e) == "1";
            };
            flag("HYDFT_TMA_YST", tma_yst);
            flag("HYDFT_TMA_YFST", tma_yfst);
            flag("HYDFT_TMA_ZFST", tma_zfst);
            flag("HYDFT_TMA_ZIST", tma_zist);
            const char *eb = std::getenv("HYDFT_BAND");
            const bool band_ok = !(eb && std::string(eb) == "0");
            band_x = band_ok && g.Mx == (g.nx - 1) / 3;
            band_y = band_ok && g.My == (g.ny - 1) / 3;
            band_z = band_ok && g.Mz == (g.nz - 1) / 3;
            CK(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
        }
        if (s.ext_active && s.ext_kind == 3) {
            // the gaussian potential, its band spectrum and its spectral gradient
            // (vext_eval: F = -grad v, external_potential.f90:81-91)
            if (int rc = alloc(gV, ncell)) return rc;
            if (int rc = alloc(gG, 3 * ncell)) return rc;
            if (int rc = alloc(Vg, csize)) return rc;
            if (int rc = up(gV, s.gauss_v.data(), 1, 0.0)) return rc;
            const R *src1[1] = {gV};
            cplx<R> *dst1[1] = {Vg};
            if (int rc = from_real(1, src1, dst1)) return rc;
            const cplx<R> *src3[3] = {Vg, Vg, Vg};
            int ops3[3] = {OP_IKX, OP_IKY, OP_IKZ};
            CK(cudaMemsetAsync(gG, 0, 3 * ncell * sizeof(R), st));
            inverse(nm, src3, ops3);
            PWToReal<R> pw;
            for (int f = 0; f < MAXF; ++f) pw.dst[f] = f < nm ? gG + (size_t)f * ncell : nullptr;
            pw.ncell = ncell;
            x_toreal(nm, pw);
            CK(cudaGetLastError());
        }
        // uniform initial state n = n0, mom = 0, Pi = 0 (species.f90:155-169)
        set_k0_kernel<R><<<1, 32, 0, st>>>(N, s.n0);
        launches++;
        CK(cudaStreamSynchronize(st));
        return 0;
    }

    int pick_rb(int nin, int nout)
    {
        int rb = std::max(1, 512 / g.nx);
        while (rb > 1 && xpass_smem<R>(g.nx, rb, nin, nout) > 100 * 1024) rb--;
        return rb;
    }

    int set_smem_attrs()
    {
        const int lim = smem_optin;
        CK(cudaFuncSetAttribute(zinv_kernel<R, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(yinv_kernel<R, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(yfwd_kernel<R, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(zfwd_kernel<R, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(xpass_kernel<R, PWA<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(xpass_kernel<R, PWB<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(xpass_kernel<R, PWU<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(xpass_kernel<R, PWToReal<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        CK(cudaFuncSetAttribute(xpass_kernel<R, PWFromReal<R>>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
        return 0;
    }

    // ------------------------------------------------------------ pipelines
    // inverse transform of nf spectral fields (with load-time operators) into
    // YI buffers 0..nf-1
    static constexpr int YZ_TX = sizeof(R) == 4 ? 16 : 8;

    // the y/z passes' block shape as compile-time constants: kx columns per
    // block (8, 16 or 32) and threads per block (YZ_NT, or 2 YZ_NT, which the
    // 256-point plan alone uses: a block then also spans two rows of the
    // other axis, or 32 columns)
    template <class F>
    void with_yz(bool fwd, F &&f) const
    {
        const int tx = fwd ? yz_txf : yz_tx, ntb = fwd ? yz_ntf : yz_nt;
        auto nt = [&](auto TXc) {
            if (ntb == 2 * YZ_NT) f(TXc, std::integral_constant<int, 2 * YZ_NT>{});
            else f(TXc, std::integral_constant<int, YZ_NT>{});
        };
        if (tx == 8) nt(std::integral_constant<int, 8>{});
        else if (tx == 16) nt(std::integral_constant<int, 16>{});
        else nt(std::integral_constant<int, 32>{});
    }
    // rows of the other axis per y/z block for T threads per column
    template <int T, int TX, int NTR>
    static constexpr int yz_rows()
    {
        constexpr int NT = T == 16 ? NTR : YZ_NT;
        return NT / (TX * T) > 0 ? NT / (TX * T) : 1;
    }
    static constexpr int YZ_NT = sizeof(R) == 4 ? 256 : 128;

    template <class K>
    void set_smem(K k, size_t bytes)
    {
        if (bytes > 48 * 1024) raise_smem_limit(reinterpret_cast<const void *>(k), bytes);
    }

    // inverse transform of nf spectral fields (with load-time operators) into
    // YI buffers 0..nf-1
    void inverse(int nf, const cplx<R> *const *src, const int *ops)
    {
        int ysrc[MAXF], yops[MAXF];
        for (int f = 0; f < nf; ++f) { ysrc[f] = f; yops[f] = OP_ID; }
        inverse_shared(nf, src, ops, nf, ysrc, yops);
    }

    // inverse transform with shared z transforms: nzf spectral fields (with
    // z-load operators) go to ZI buffers 0..nzf-1; YI buffer j is the y
    // transform of ZI buffer ysrc[j] with the y-load operator yops[j] (OP_ID,
    // or OP_IKY on axes with a register plan)
    void inverse_shared(int nzf, const cplx<R> *const *src, const int *ops, int nf, const int *ysrc,
                        const int *yops)
    {
        // the y transforms run in the order of their ZI sources, so that the
        // two reads of a shared ZI buffer follow each other (the second from
        // L2); each still writes YI buffer j
        int yord[MAXF];
        for (int j = 0; j < nf; ++j) yord[j] = j;
        std::stable_sort(yord, yord + nf, [&](int a, int b) { return ysrc[a] < ysrc[b]; });
        PassArgs<R> a;
        a.nf = nzf;
        for (int f = 0; f < nzf; ++f) {
            a.in[f] = src[f];
            a.out[f] = zi + (size_t)f * zsize;
            a.op[f] = ops[f];
        }
        const double zbytes = nzf * cb() * g.nkxc * g.nkyc * (double)(g.nkzc + g.nz);
        const bool zf = with_plan(g.nz, [&](auto Tc, auto Ec) {
            constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
            with_yz(false, [&](auto TXc, auto NTc) {
            constexpr int TX = decltype(TXc)::value;
            constexpr int G = yz_rows<T, TX, decltype(NTc)::value>();
            const size_t sm = yz_fast_smem<R>(T * E, T, TX, G);
            auto go = [&](auto k, auto pk, auto kt, auto kst, auto kl, int nb) {
                set_smem(k, sm);
                const dim3 grid((g.nkxc + TX - 1) / TX, (g.nkyc + G * nb - 1) / (G * nb), nzf);
                pk.g = g; pk.a = a; pk.tw = tpz;
                // one row per thread: the output tile by a tensor store (the
                // tile [nz][G][TX] fits in the exchange space)
                CUtensorMap otm;
                if (!rec && use_tma && tma_zist && nb == 1 && (size_t)g.nz * G * TX <= (size_t)G * (T * E + E) * TX &&
                    make_field_tmap<R>(&otm, zi, g.pkx, g.nkyc, g.nz, nin_max, TX, G, g.nz)) {
                    TmaFields tf = tma_fields(a.in, 0, zi, zsize);
                    for (int f = 0; f < nzf; ++f) tf.dst[f] = (int)((a.out[f] - zi) / (ptrdiff_t)zsize);
                    // with HYDFT_TMA_ZINV=1 the input tile by a tensor load into
                    // the exchange space as well
                    const size_t tl = sizeof(cplx<R>) * (size_t)TX * G * g.nkzc;
                    bool ld = tma_zinv && nzf <= 16 && tl + 8 <= sm - sizeof(cplx<R>) * 2 * T * E;
                    TmaMaps maps;
                    for (int f = 0; ld && f < nzf; ++f)
                        ld = make_field_tmap<R>(&maps.m[f], a.in[f], g.pkx, g.nkyc, g.nkzc, 1, TX, G, g.nkzc);
                    if (ld) {
                        set_smem(kl, sm);
                        launch("zinv", zbytes, [&] { kl<<<grid, TX * T * G, sm, st>>>(g, a, tpz, maps, otm, tf); });
                        return;
                    }
                    set_smem(kst, sm);
                    launch("zinv", zbytes, [&] { kst<<<grid, TX * T * G, sm, st>>>(g, a, tpz, otm, tf); });
                    return;
                }
                // TMA: one map per input field; the tile goes into the exchange
                // buffer where it fits (every column is read into registers
                // before the first exchange), else past the pass's own shared
                // memory (with two rows per thread it does not fit)
                const size_t tile = sizeof(cplx<R>) * (size_t)TX * G * nb * g.nkzc;
                const bool inbuf = tile + 8 <= sm - sizeof(cplx<R>) * 2 * T * E;
                const size_t smt = inbuf ? sm : (sm + tile + 8 + 127) / 128 * 128;
                bool tma = !rec && use_tma && tma_zinv && nzf <= 16 && (inbuf || sm % 128 == 0) &&
                           smt <= (size_t)smem_optin;
                TmaMaps maps;
                for (int f = 0; tma && f < nzf; ++f)
                    tma = make_field_tmap<R>(&maps.m[f], a.in[f], g.pkx, g.nkyc, g.nkzc, 1, TX, G * nb, g.nkzc);
                if (tma) {
                    set_smem(kt, smt);
                    const unsigned off = inbuf ? (unsigned)(2 * T * E) : (unsigned)(sm / sizeof(cplx<R>));
                    unsigned *stw = &ctrl->status;
                    launch("zinv", zbytes, [&] { kt<<<grid, TX * T * G, smt, st>>>(g, a, tpz, maps, off, stw); });
                    return;
                }
                launch_p("zinv", zbytes, grid, TX * T * G, sm, pk, [&] { k<<<grid, TX * T * G, sm, st>>>(g, a, tpz); });
            };
            if ((rec ? z_nb_ens : z_nb) == 2) {
                if (band_z) go(zinv_fast<R, T, E, TX, G, true, 2>, ZinvPack<R, T, E, TX, G, true, 2>{}, zinv_tma<R, T, E, TX, G, true, 2>, zinv_st<R, T, E, TX, G, true>, zinv_tma_st<R, T, E, TX, G, true>, 2);
                else go(zinv_fast<R, T, E, TX, G, false, 2>, ZinvPack<R, T, E, TX, G, false, 2>{}, zinv_tma<R, T, E, TX, G, false, 2>, zinv_st<R, T, E, TX, G, false>, zinv_tma_st<R, T, E, TX, G, false>, 2);
            } else {
                if (band_z) go(zinv_fast<R, T, E, TX, G, true, 1>, ZinvPack<R, T, E, TX, G, true, 1>{}, zinv_tma<R, T, E, TX, G, true, 1>, zinv_st<R, T, E, TX, G, true>, zinv_tma_st<R, T, E, TX, G, true>, 1);
                else go(zinv_fast<R, T, E, TX, G, false, 1>, ZinvPack<R, T, E, TX, G, false, 1>{}, zinv_tma<R, T, E, TX, G, false, 1>, zinv_st<R, T, E, TX, G, false>, zinv_tma_st<R, T, E, TX, G, false>, 1);
            }
            });
        });
        if (!zf) {
            const int ntx = (g.nkxc + TX - 1) / TX;
            const size_t smz = sizeof(cplx<R>) * (2 * (size_t)g.nz * TX + g.nz);
            launch("zinv", zbytes, [&] { zinv_kernel<R, TX><<<dim3(ntx, g.nkyc, nzf), 256, smz, st>>>(g, a, twz); });
        }
        if (g.ny > 1) {
            PassArgs<R> b;
            b.nf = nf;
            for (int f = 0; f < nf; ++f) {
                const int j = yord[f];
                b.in[f] = zi + (size_t)ysrc[j] * zsize;
                b.out[f] = yi + (size_t)j * ysize;
                b.op[f] = yops[j];
            }
            const double ybytes = nf * cb() * g.nkxc * g.nz * (double)(g.nkyc + g.ny);
            const bool yf = with_plan(g.ny, [&](auto Tc, auto Ec) {
                constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
                with_yz(false, [&](auto TXc, auto NTc) {
                constexpr int TX = decltype(TXc)::value;
                constexpr int G = yz_rows<T, TX, decltype(NTc)::value>();
                const size_t sm = yz_fast_smem<R>(T * E, T, TX, G);
                const dim3 grid((g.nkxc + TX - 1) / TX, (g.nz + G - 1) / G, nf);
                auto go = [&](auto k, auto pk, auto kt, auto pkt, auto kst) {
                    set_smem(k, sm);
                    pk.g = g; pk.a = b; pk.tw = tpy;
                    const size_t tile = sizeof(cplx<R>) * (size_t)TX * g.nkyc * G;
                    if (use_tma && tile + 8 <= sm - sizeof(cplx<R>) * 2 * T * E &&
                        make_field_tmap<R>(&pkt.tm, zi, g.pkx, g.nkyc, g.nz, nin_max, TX, g.nkyc, G)) {
                        pkt.g = g; pkt.a = b; pkt.tw = tpy; pkt.tf = tma_fields(b.in, nf, zi, zsize);
                        // the output tile by a tensor store as well (plain and ensemble forms)
                        pkt.store = 0;
                        std::memset(static_cast<void *>(&pkt.otm), 0, sizeof(pkt.otm));
                        if (tma_yst && make_field_tmap<R>(&pkt.otm, yi, g.pkx, g.ny, g.nz, nin_max, TX, g.ny, G)) {
                            for (int f = 0; f < nf; ++f) pkt.tf.dst[f] = (int)((b.out[f] - yi) / (ptrdiff_t)ysize);
                            pkt.store = 1;
                            set_smem(kst, sm);
                            launch_p("yinv", ybytes, grid, TX * T * G, sm, pkt,
                                     [&] { kst<<<grid, TX * T * G, sm, st>>>(g, b, tpy, pkt.tm, pkt.otm, pkt.tf); });
                            return;
                        }
                        set_smem(kt, sm);
                        launch_p("yinv", ybytes, grid, TX * T * G, sm, pkt,
                                 [&] { kt<<<grid, TX * T * G, sm, st>>>(g, b, tpy, pkt.tm, pkt.tf); });
                        return;
                    }
                    launch_p("yinv", ybytes, grid, TX * T * G, sm, pk, [&] { k<<<grid, TX * T * G, sm, st>>>(g, b, tpy); });
                };
                if (band_y) go(yinv_fast<R, T, E, TX, G, true>, YinvPack<R, T, E, TX, G, true>{}, yinv_tma<R, T, E, TX, G, true>, YinvTmaPack<R, T, E, TX, G, true>{}, yinv_tma_st<R, T, E, TX, G, true>);
                else go(yinv_fast<R, T, E, TX, G, false>, YinvPack<R, T, E, TX, G, false>{}, yinv_tma<R, T, E, TX, G, false>, YinvTmaPack<R, T, E, TX, G, false>{}, yinv_tma_st<R, T, E, TX, G, false>);
            });
            });
            if (!yf) {
                const int ntx = (g.nkxc + TX - 1) / TX;
                const size_t smy = sizeof(cplx<R>) * (2 * (size_t)g.ny * TX + g.ny);
                launch("yinv", ybytes, [&] { yinv_kernel<R, TX><<<dim3(ntx, g.nz, nf), 256, smy, st>>>(g, b, twy); });
            }
        }
    }

    // forward transform of the x-pass outputs 0..nf-1 into compact fields
    void forward(int nf, cplx<R> *const *dst)
    {
        const int ntx = (g.nkxc + TX - 1) / TX;
        const cplx<R> *src = xo;
        if (g.ny > 1) {
            PassArgs<R> b;
            b.nf = nf;
            for (int f = 0; f < nf; ++f) {
                b.in[f] = xo + (size_t)f * ysize;
                b.out[f] = zi + (size_t)f * zsize;
                b.op[f] = OP_ID;
            }
            const double ybytes = nf * cb() * g.nkxc * g.nz * (double)(g.nkyc + g.ny);
            const bool yf = with_plan(g.ny, [&](auto Tc, auto Ec) {
                constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
                with_yz(true, [&](auto TXc, auto NTc) {
                constexpr int TX = decltype(TXc)::value;
                constexpr int G = yz_rows<T, TX, decltype(NTc)::value>();
                const size_t sm = yz_fast_smem<R>(T * E, T, TX, G);
                const dim3 grid((g.nkxc + TX - 1) / TX, (g.nz + G - 1) / G, nf);
                auto go = [&](auto k, auto pk, auto kt, auto pkt, auto kst) {
                    set_smem(k, sm);
                    pk.g = g; pk.a = b; pk.tw = tpy;
                    const size_t tile = sizeof(cplx<R>) * (size_t)TX * g.ny * G;
                    if (use_tma && tile + 8 <= sm - sizeof(cplx<R>) * 2 * T * E &&
                        make_field_tmap<R>(&pkt.tm, xo, g.pkx, g.ny, g.nz, nout_max, TX, g.ny, G)) {
                        pkt.g = g; pkt.a = b; pkt.tw = tpy; pkt.tf = tma_fields(b.in, nf, xo, ysize);
                        // the output tile [G][nkyc][TX] by a tensor store as well
                        pkt.store = 0;
                        std::memset(static_cast<void *>(&pkt.otm), 0, sizeof(pkt.otm));
                        if (tma_yfst && make_field_tmap<R>(&pkt.otm, zi, g.pkx, g.nkyc, g.nz, nin_max, TX, g.nkyc, G)) {
                            for (int f = 0; f < nf; ++f) pkt.tf.dst[f] = (int)((b.out[f] - zi) / (ptrdiff_t)zsize);
                            pkt.store = 1;
                            set_smem(kst, sm);
                            launch_p("yfwd", ybytes, grid, TX * T * G, sm, pkt,
                                     [&] { kst<<<grid, TX * T * G, sm, st>>>(g, b, tpy, pkt.tm, pkt.otm, pkt.tf); });
                            return;
                        }
                        set_smem(kt, sm);
                        launch_p("yfwd", ybytes, grid, TX * T * G, sm, pkt,
                                 [&] { kt<<<grid, TX * T * G, sm, st>>>(g, b, tpy, pkt.tm, pkt.tf); });
                        return;
                    }
                    launch_p("yfwd", ybytes, grid, TX * T * G, sm, pk, [&] { k<<<grid, TX * T * G, sm, st>>>(g, b, tpy); });
                };
                if (band_y) go(yfwd_fast<R, T, E, TX, G, true>, YfwdPack<R, T, E, TX, G, true>{}, yfwd_tma<R, T, E, TX, G, true>, YfwdTmaPack<R, T, E, TX, G, true>{}, yfwd_tma_st<R, T, E, TX, G, true>);
                else go(yfwd_fast<R, T, E, TX, G, false>, YfwdPack<R, T, E, TX, G, false>{}, yfwd_tma<R, T, E, TX, G, false>, YfwdTmaPack<R, T, E, TX, G, false>{}, yfwd_tma_st<R, T, E, TX, G, false>);
            });
            });
            if (!yf) {
                const size_t smy = sizeof(cplx<R>) * (2 * (size_t)g.ny * TX + g.ny);
                launch("yfwd", ybytes, [&] { yfwd_kernel<R, TX><<<dim3(ntx, g.nz, nf), 256, smy, st>>>(g, b, twy); });
            }
            src = zi;
        }
        PassArgs<R> a;
        a.nf = nf;
        for (int f = 0; f < nf; ++f) {
            a.in[f] = src + (size_t)f * (g.ny > 1 ? zsize : ysize);
            a.out[f] = dst[f];
            a.op[f] = OP_ID;
        }
        const R norm = R(1.0 / ((double)g.nx * g.ny * g.nz));
        const double zbytes = nf * cb() * g.nkxc * g.nkyc * (double)(g.nkzc + g.nz);
        const bool zf = with_plan(g.nz, [&](auto Tc, auto Ec) {
            constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
            with_yz(true, [&](auto TXc, auto NTc) {
            constexpr int TX = decltype(TXc)::value;
            constexpr int G = yz_rows<T, TX, decltype(NTc)::value>();
            const size_t sm = yz_fast_smem<R>(T * E, T, TX, G);
            auto go = [&](auto k, auto pk, auto kt, auto pkt, auto kst, int nb) {
                set_smem(k, sm);
                const dim3 grid((g.nkxc + TX - 1) / TX, (g.nkyc + G * nb - 1) / (G * nb), nf);
                pk.g = g; pk.a = a; pk.tw = tpz; pk.norm = norm;
                const size_t tile = sizeof(cplx<R>) * (size_t)TX * G * nb * g.nz;
                if (use_tma && src == zi && tile + 8 <= sm - sizeof(cplx<R>) * 2 * T * E &&
                    make_field_tmap<R>(&pkt.tm, zi, g.pkx, g.nkyc, g.nz, nin_max, TX, G * nb, g.nz)) {
                    pkt.g = g; pkt.a = a; pkt.tw = tpz; pkt.norm = norm; pkt.tf = tma_fields(a.in, nf, zi, zsize);
                    // one row per thread: each output field's tile [nkzc][G][TX]
                    // by a tensor store (one map per compact output field)
                    bool stv = !rec && tma_zfst && nb == 1 && nf <= 16;
                    TmaMaps om;
                    for (int f = 0; stv && f < nf; ++f)
                        stv = make_field_tmap<R>(&om.m[f], a.out[f], g.pkx, g.nkyc, g.nkzc, 1, TX, G, g.nkzc);
                    if (stv) {
                        set_smem(kst, sm);
                        launch("zfwd", zbytes, [&] { kst<<<grid, TX * T * G, sm, st>>>(g, a, tpz, norm, pkt.tm, om, pkt.tf); });
                        return;
                    }
                    set_smem(kt, sm);
                    launch_p("zfwd", zbytes, grid, TX * T * G, sm, pkt,
                             [&] { kt<<<grid, TX * T * G, sm, st>>>(g, a, tpz, norm, pkt.tm, pkt.tf); });
                    return;
                }
                launch_p("zfwd", zbytes, grid, TX * T * G, sm, pk, [&] { k<<<grid, TX * T * G, sm, st>>>(g, a, tpz, norm); });
            };
            if (z_nbf == 2) {
                if (band_z) go(zfwd_fast<R, T, E, TX, G, true, 2>, ZfwdPack<R, T, E, TX, G, true, 2>{}, zfwd_tma<R, T, E, TX, G, true, 2>, ZfwdTmaPack<R, T, E, TX, G, true, 2>{}, zfwd_tma_st<R, T, E, TX, G, true>, 2);
                else go(zfwd_fast<R, T, E, TX, G, false, 2>, ZfwdPack<R, T, E, TX, G, false, 2>{}, zfwd_tma<R, T, E, TX, G, false, 2>, ZfwdTmaPack<R, T, E, TX, G, false, 2>{}, zfwd_tma_st<R, T, E, TX, G, false>, 2);
            } else {
                if (band_z) go(zfwd_fast<R, T, E, TX, G, true, 1>, ZfwdPack<R, T, E, TX, G, true, 1>{}, zfwd_tma<R, T, E, TX, G, true, 1>, ZfwdTmaPack<R, T, E, TX, G, true, 1>{}, zfwd_tma_st<R, T, E, TX, G, true>, 1);
                else go(zfwd_fast<R, T, E, TX, G, false, 1>, ZfwdPack<R, T, E, TX, G, false, 1>{}, zfwd_tma<R, T, E, TX, G, false, 1>, ZfwdTmaPack<R, T, E, TX, G, false, 1>{}, zfwd_tma_st<R, T, E, TX, G, false>, 1);
            }
            });
        });
        if (!zf) {
            const size_t smz = sizeof(cplx<R>) * (2 * (size_t)g.nz * TX + g.nz);
            launch("zfwd", zbytes, [&] { zfwd_kernel<R, TX><<<dim3(ntx, g.nkyc, nf), 256, smz, st>>>(g, a, twz, norm); });
        }
    }

    // threads of a fast x pass: the largest multiple of T up to 256 whose
    // shared memory stays within ~110 KB
    template <int T, int E>
    int x_threads(int np_slots, size_t &smem) const
    {
        int nt = x_ntmax;
        for (;;) {
            smem = sizeof(cplx<R>) * (2 * (size_t)T * E + (size_t)(nt / T) * xrow_stride<T, E>() + (size_t)np_slots * E * nt) +
                   (np_slots ? 2 * sizeof(R) * (size_t)E * nt : 0);
            if (smem <= 110 * 1024 || nt <= T) break;
            nt /= 2;
        }
        return nt;
    }

    XFastArgs<R> xargs(int nin, int nout) const
    {
        XFastArgs<R> a;
        a.nin = nin;
        a.nout = nout;
        a.dx_in_pass = 0;
        for (int f = 0; f < nin; ++f) a.in[f] = yi + (size_t)f * ysize;
        for (int f = 0; f < nout; ++f) a.out[f] = xo + (size_t)f * ysize;
        return a;
    }

    double xbytes(int nin, int nout, int nreal) const
    {
        return cb() * g.nkxc * (double)g.ny * g.nz * (nin + nout) + sizeof(R) * (double)ncell * nreal;
    }

    // fast phase-A x pass (3-D); uonly: u only (relaxation finish)
    void xa_launch(int nin, int nout, const PWA<R> &pw, bool grad, bool uonly, const char *name, int nreal)
    {
        const XFastArgs<R> a = xargs(nin, nout);
        const int nrows = g.ny * g.nz;
        with_plan(g.nx, [&](auto Tc, auto Ec) {
            constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
            auto go = [&](auto k, auto pk, int np) {
                size_t sm;
                const int nt = x_threads<T, E>(np, sm);
                set_smem(k, sm);
                const int rb = nt / T;
                const dim3 grid((nrows + rb - 1) / rb);
                pk.g = g; pk.a = a; pk.tw = tpx; pk.pw = pw;
                launch_p(name, xbytes(nin, nout, nreal), grid, nt, sm, pk, [&] { k<<<grid, nt, sm, st>>>(g, a, tpx, pw); });
            };
            auto go_regs = [&](auto k, auto pk) {
                int nt = std::min(256, x_ntmax) / T * T;
                size_t sm = xstaged_smem<R, T, E>(nt, g.pkx, 4, 0);
                // the blocks per SM the kernel is compiled for must fit: 228 KB
                // of shared memory per SM, 1 KB reserved per block
                const size_t cap = xstaged_minb<R, E>() == 2 ? 115712 : (size_t)smem_optin;
                while (sm > cap && nt > 32) {   // whole warps: each stages its own rows
                    nt /= 2;
                    sm = xstaged_smem<R, T, E>(nt, g.pkx, 4, 0);
                }
                set_smem(k, sm);
                const int rb = nt / T;
                const dim3 grid((nrows + rb - 1) / rb);
                pk.g = g; pk.a = a; pk.tw = tpx; pk.pw = pw;
                launch_p(name, xbytes(nin, nout, nreal), grid, nt, sm, pk, [&] { k<<<grid, nt, sm, st>>>(g, a, tpx, pw); });
            };
            const bool no_fd = !ph.has_tf && !ph.has_grad;
            if (staged_x && uonly) {
                if (band_x) go_regs(xa_regs<R, T, E, true, true>, XaRegsPack<R, T, E, true, true>{});
                else go_regs(xa_regs<R, T, E, true, false>, XaRegsPack<R, T, E, true, false>{});
            } else if (staged_x && !grad && no_fd) {
                if (band_x) go_regs(xa_regs<R, T, E, false, true>, XaRegsPack<R, T, E, false, true>{});
                else go_regs(xa_regs<R, T, E, false, false>, XaRegsPack<R, T, E, false, false>{});
            } else if (uonly) {
                go(xa_fast<R, T, E, 3, false, true>, XaFastPack<R, T, E, 3, false, true>{}, 2);
            } else if (grad) {
                go(xa_fast<R, T, E, 3, true, false>, XaFastPack<R, T, E, 3, true, false>{}, 4);
            } else {
                go(xa_fast<R, T, E, 3, false, false>, XaFastPack<R, T, E, 3, false, false>{}, 2);
            }
        });
    }

    void xb_launch(int nin, int nout, const PWB<R> &pw, int nreal, bool dx_in_pass)
    {
        XFastArgs<R> a = xargs(nin, nout);
        a.dx_in_pass = dx_in_pass ? 1 : 0;
        const int nrows = g.ny * g.nz;
        with_plan(g.nx, [&](auto Tc, auto Ec) {
            constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
            auto go = [&](auto k, auto pk) {
                size_t sm;
                const int nt = x_threads<T, E>(0, sm);
                set_smem(k, sm);
                const int rb = nt / T;
                const dim3 grid((nrows + rb - 1) / rb);
                pk.g = g; pk.a = a; pk.tw = tpx; pk.pw = pw;
                launch_p("xpass_b", xbytes(nin, nout, nreal), grid, nt, sm, pk, [&] { k<<<grid, nt, sm, st>>>(g, a, tpx, pw); });
            };
            auto go_rows = [&](auto k, auto pk, int nreal_rows) {
                int nt = std::min(256, x_ntmax) / T * T;
                size_t sm = xstaged_smem<R, T, E>(nt, g.pkx, 2, nreal_rows);
                // two blocks per SM: 228 KB of shared memory, 1 KB reserved per block
                while (sm > 115712 && nt > 32) {   // whole warps
                    nt /= 2;
                    sm = xstaged_smem<R, T, E>(nt, g.pkx, 2, nreal_rows);
                }
                set_smem(k, sm);
                const int rb = nt / T;
                const dim3 grid((nrows + rb - 1) / rb);
                pk.g = g; pk.a = a; pk.tw = tpx; pk.pw = pw;
                launch_p("xpass_b", xbytes(nin, nout, nreal), grid, nt, sm, pk, [&] { k<<<grid, nt, sm, st>>>(g, a, tpx, pw); });
            };
            const int extk = !ph.ext_active ? 0 : (ph.ext_kind == 3 ? 2 : 1);
            auto rows = [&](auto ev, auto ek) {
                constexpr bool EV = decltype(ev)::value;
                constexpr int EK = decltype(ek)::value;
                if (band_x) go_rows(xb_rows<R, T, E, EV, EK, true>, XbRowsPack<R, T, E, EV, EK, true>{}, EV ? 3 : 0);
                else go_rows(xb_rows<R, T, E, EV, EK, false>, XbRowsPack<R, T, E, EV, EK, false>{}, EV ? 3 : 0);
            };
            using std::integral_constant;
            using EvT = integral_constant<bool, true>;
            using EvF = integral_constant<bool, false>;
            if (staged_x && ph.evolve) {
                if (extk == 2) rows(EvT{}, integral_constant<int, 2>{});
                else if (extk == 1) rows(EvT{}, integral_constant<int, 1>{});
                else rows(EvT{}, integral_constant<int, 0>{});
            } else if (staged_x) {
                if (extk == 2) rows(EvF{}, integral_constant<int, 2>{});
                else if (extk == 1) rows(EvF{}, integral_constant<int, 1>{});
                else rows(EvF{}, integral_constant<int, 0>{});
            } else if (ph.evolve) {
                go(xb_fast<R, T, E, 3, true>, XbFastPack<R, T, E, 3, true>{});
            } else {
                go(xb_fast<R, T, E, 3, false>, XbFastPack<R, T, E, 3, false>{});
            }
        });
    }

    void xio_launch(int nin, int nout, const PWToReal<R> &dst, const PWFromReal<R> &src, const char *name)
    {
        const XFastArgs<R> a = xargs(nin, nout);
        const int nrows = g.ny * g.nz;
        with_plan(g.nx, [&](auto Tc, auto Ec) {
            constexpr int T = decltype(Tc)::value, E = decltype(Ec)::value;
            auto go = [&](auto k) {
                size_t sm;
                const int nt = x_threads<T, E>(0, sm);
                set_smem(k, sm);
                const int rb = nt / T;
                launch(name, xbytes(nin, nout, nin + nout), [&] { k<<<(nrows + rb - 1) / rb, nt, sm, st>>>(g, a, tpx, dst, src); });
            };
            if (nin > 0) go(xio_fast<R, T, E, true>);
            else go(xio_fast<R, T, E, false>);
        });
    }

    template <class PW>
    void xpass(int nin, int nout, const PW &pw, int rb, const char *name = "xpass", int nreal = 0)
    {
        XArgs<R> a;
        a.nin = nin;
        a.nout = nout;
        for (int f = 0; f < nin; ++f) a.in[f] = yi + (size_t)f * ysize;
        for (int f = 0; f < nout; ++f) a.out[f] = xo + (size_t)f * ysize;
        const int nrows = g.ny * g.nz;
        const size_t sm = xpass_smem<R>(g.nx, rb, nin, nout);
        const double bytes = cb() * g.nkxc * (double)nrows * (nin + nout) + sizeof(R) * (double)ncell * nreal;
        launch(name, bytes, [&] { xpass_kernel<R, PW><<<(nrows + rb - 1) / rb, 256, sm, st>>>(g, a, twx, pw, rb); });
    }

    // f(integral_constant<int, nm>): the momentum component count as a
    // compile-time constant
    template <class F>
    void with_nm(F &&f) const
    {
        if (nm == 3) f(std::integral_constant<int, 3>{});
        else if (nm == 2) f(std::integral_constant<int, 2>{});
        else f(std::integral_constant<int, 1>{});
    }

    int combine_grid() const
    {
        return (int)std::min<size_t>((csize + 255) / 256, 148 * 16);
    }

    // -------------------------------------------------------------- stage
    void phase_a(int stage, bool write_u)
    {
        const cplx<R> *src[MAXF];
        int ops[MAXF];
        int nf = 0;
        src[nf] = N; ops[nf++] = OP_ZK0;
        for (int d = 0; d < nm; ++d) { src[nf] = M[d]; ops[nf++] = OP_ID; }
        if (ph.has_grad) {
            for (int d = 0; d < nm; ++d) { src[nf] = N; ops[nf++] = OP_IKX + d; }
            src[nf] = N; ops[nf++] = OP_NK2;
        }
        inverse(nf, src, ops);
        PWA<R> pw;
        pw.ph = ph;
        pw.nm = nm;
        pw.nhat = N;
        pw.nmean = &ctrl->nmean;
        pw.fdtab = fdtab;
        pw.dn_real = dn_real;
        pw.u_real = write_u ? u_real : nullptr;
        pw.ncell = ncell;
        pw.status = &ctrl->status;
        const int nout = nm + nm * (nm + 1) / 2 + 1;
        if (fast_x) xa_launch(nf, nout, pw, ph.has_grad != 0, false, "xpass_a", write_u ? 1 + nm : 1);
        else xpass(nf, nout, pw, xrb_a, "xpass_a", write_u ? 1 + nm : 1);
        forward(nout, OA);
        CombineA<R> c;
        c.N = N;
        for (int d = 0; d < 3; ++d) c.M[d] = M[d];
        for (int q = 0; q < 6; ++q) { c.P[q] = P[q]; c.P0[q] = P0[q]; }
        for (int d = 0; d < 3; ++d) c.U[d] = OA[d];
        for (int q = 0; q < 6; ++q) c.F[q] = OA[nm + std::min(q, nm * (nm + 1) / 2 - 1)];
        c.G = OA[nout - 1];
        c.Klin = Klin;
        c.MU = MU;
        for (int d = 0; d < 3; ++d) c.Q[d] = Q[d];
        const double ncomp = (double)g.nkxc * g.nkyc * g.nkzc;
        const int nrw = 2 + nm + nm * (nm + 1) / 2 + 1 + nm + (ph.evolve ? 24 : 0);
        with_nm([&](auto n) {
            constexpr int NMc = decltype(n)::value;
            const dim3 grid(combine_grid());
            const CombineAPack<R, NMc> pk{g, ph, c, ctrl, stage};
            launch_p("combine_a", ncomp * (cb() * nrw + sizeof(R)), grid, 256, 0, pk,
                     [&] { combine_a_kernel<R, NMc><<<grid, 256, 0, st>>>(g, ph, c, ctrl, stage); });
        });
    }

    // phase B's inverse transforms into YI buffers 0..nf-1; returns nf.
    // dx_in_pass: the staged x pass takes d/dx itself, so the x and y
    // derivatives of mu and of each Pi component share one z transform (k_x
    // and k_y are constant along z) and each field is z-transformed twice,
    // not three times.
    int phase_b_inverse(bool &dx_in_pass)
    {
        const cplx<R> *src[MAXF];
        int ops[MAXF];
        int nf = 0;
        dx_in_pass = fast_x && staged_x && g.ny > 1 && has_plan(g.ny);
        if (dx_in_pass) {
            int nzf = 0, ysrc[MAXF], yops[MAXF];
            auto field = [&](const cplx<R> *f) {
                const int z0 = nzf;
                src[nzf] = f; ops[nzf++] = OP_ID;
                src[nzf] = f; ops[nzf++] = OP_IKZ;
                return z0;
            };
            const int zmu = field(MU);
            for (int d = 0; d < nm; ++d) {
                ysrc[nf] = d == 2 ? zmu + 1 : zmu;
                yops[nf++] = d == 1 ? OP_IKY : OP_ID;
            }
            if (ph.evolve) {
                int zq[6];
                for (int q = 0; q < 6; ++q) zq[q] = field(P[q]);
                for (int cp = 0; cp < 3; ++cp)
                    for (int d = 0; d < nm; ++d)
                        for (int h = 0; h < 2; ++h) {
                            const int z0 = zq[2 * cp + h];
                            ysrc[nf] = d == 2 ? z0 + 1 : z0;
                            yops[nf++] = d == 1 ? OP_IKY : OP_ID;
                        }
            }
            inverse_shared(nzf, src, ops, nf, ysrc, yops);
        } else {
            for (int d = 0; d < nm; ++d) { src[nf] = MU; ops[nf++] = OP_IKX + d; }
            if (ph.evolve)
                for (int cp = 0; cp < 3; ++cp)
                    for (int d = 0; d < nm; ++d)
                        for (int h = 0; h < 2; ++h) { src[nf] = P[2 * cp + h]; ops[nf++] = OP_IKX + d; }
            inverse(nf, src, ops);
        }
        return nf;
    }

    void phase_b(int stage, bool rhs_only)
    {
        bool dxp = false;
        const int nf = phase_b_inverse(dxp);
        PWB<R> pw;
        pw.ph = ph;
        pw.nm = nm;
        pw.nhat = N;
        pw.nmean = &ctrl->nmean;
        pw.dn_real = dn_real;
        pw.u_real = u_real;
        pw.ncell = ncell;
        pw.ex = ex; pw.ey = ey; pw.ez = ez;
        pw.gradv = gG;
        pw.ctrl = ctrl;
        pw.stage = stage;
        pw.status = &ctrl->status;
        const int nout = nm + (ph.evolve ? 6 : 0);
        if (ph.ext_active && ph.ext_kind == 3) {
            // mean of n F over the stage state (k = 0 of the momentum tendency)
            launch("force_mean", 0.0, [&] {
                gauss_force_mean_kernel<R><<<red_blocks, 256, 0, st>>>(g, N, Vg, spart);
            });
            launch("force_mean", 0.0, [&] { gauss_force_final_kernel<<<1, 32, 0, st>>>(spart, red_blocks, ctrl); });
        }
        if (fast_x) xb_launch(nf, nout, pw, ph.evolve ? 1 + nm : 1, dxp);
        else xpass(nf, nout, pw, xrb_b, "xpass_b", ph.evolve ? 1 + nm : 1);
        forward(nout, OB);
        CombineB<R> c;
        c.N = N; c.RN = RN; c.oN = HN;
        for (int d = 0; d < 3; ++d) {
            c.M[d] = M[d]; c.RM[d] = RM[d]; c.oM[d] = HM[d];
            c.Q[d] = Q[d];
            c.Gm[d] = OB[std::min(d, nm - 1)];
        }
        for (int q = 0; q < 6; ++q) {
            c.P[q] = P[q]; c.RP[q] = RP[q]; c.oP[q] = HP[q];
            c.V[q] = OB[ph.evolve ? nm + q : 0];
        }
        const double ncomp = (double)g.nkxc * g.nkyc * g.nkzc;
        const int nrw = 2 + 5 * nm + 2 + (ph.evolve ? 30 : 0);
        with_nm([&](auto n) {
            constexpr int NMc = decltype(n)::value;
            const dim3 grid(combine_grid());
            const int ro = rhs_only ? 1 : 0;
            const CombineBPack<R, NMc> pk{g, ph, c, ctrl, stage, ro};
            launch_p("combine_b", ncomp * cb() * nrw, grid, 256, 0, pk,
                     [&] { combine_b_kernel<R, NMc><<<grid, 256, 0, st>>>(g, ph, c, ctrl, stage, ro); });
        });
    }

    void begin_step()
    {
        const double omega = S.ext_kind == 2 ? S.ext_omega : 0.0;
        const BeginStepPack pk{ctrl, ph.evolve ? ph.tau : 0.0, S.ext_td, S.ext_amp, omega, S.ext_ramp};
        launch_p("step_ctrl", 0.0, dim3(1), 32, 0, pk, [&] {
            begin_step_kernel<<<1, 32, 0, st>>>(pk.ctrl, pk.tau, pk.ext_td, pk.amp0, pk.omega, pk.ramp);
        });
    }

    void one_step()
    {
        begin_step();
        for (int s = 0; s < 3; ++s) {
            phase_a(s, ph.evolve != 0);
            phase_b(s, false);
        }
        const EndStepPack pk{ctrl};
        launch_p("step_ctrl", 0.0, dim3(1), 32, 0, pk, [&] { end_step_kernel<<<1, 32, 0, st>>>(ctrl); });
    }

    // Maxwell: complete the last stage's relaxation from u of the new state
    void finish()
    {
        if (!ph.evolve) return;
        const cplx<R> *src[MAXF];
        int ops[MAXF];
        int nf = 0;
        src[nf] = N; ops[nf++] = OP_ZK0;
        for (int d = 0; d < nm; ++d) { src[nf] = M[d]; ops[nf++] = OP_ID; }
        inverse(nf, src, ops);
        if (fast_x) {
            PWA<R> pa;
            pa.ph = ph;
            pa.nm = nm;
            pa.nhat = N;
            pa.nmean = &ctrl->nmean;
            pa.fdtab = fdtab;
            pa.dn_real = nullptr;
            pa.u_real = nullptr;
            pa.ncell = ncell;
            pa.status = &ctrl->status;
            xa_launch(nf, nm, pa, false, true, "xpass_u", 0);
        } else {
            PWU<R> pw;
            pw.ph = ph;
            pw.nm = nm;
            pw.nhat = N;
        pw.nmean = &ctrl->nmean;
            pw.status = &ctrl->status;
            xpass(nf, nm, pw, xrb_io, "xpass_u");
        }
        forward(nm, OA);
        CombineU<R> c;
        for (int q = 0; q < 6; ++q) { c.P[q] = P[q]; c.P0[q] = P0[q]; }
        for (int d = 0; d < 3; ++d) c.U[d] = OA[std::min(d, nm - 1)];
        const double ncomp = (double)g.nkxc * g.nkyc * g.nkzc;
        launch("combine_u", ncomp * cb() * (nm + 18),
               [&] { with_nm([&](auto n) { combine_u_kernel<R, decltype(n)::value><<<combine_grid(), 256, 0, st>>>(g, ph, c, ctrl); }); });
        cudaMemsetAsync(&ctrl->pending, 0, sizeof(int), st);
    }

    void finish_if_pending()
    {
        if (host_pending) finish();
        host_pending = false;
    }

    int profile(int nsteps, std::vector<KernelStat> &out) override
    {
        std::vector<KStat> ks;
        int rc = profile_k(nsteps, ks);
        out.clear();
        for (auto &k : ks) {
            KernelStat o;
            o.name = k.name;
            o.ms = k.ms;
            o.bytes = k.bytes;
            o.n = k.n;
            out.push_back(o);
        }
        return rc;
    }

    // Runs nsteps uncaptured steps with an event pair around every launch.
    int profile_k(int nsteps, std::vector<KStat> &out)
    {
        CK(cudaStreamSynchronize(st));
        kstats.clear();
        evrecs.clear();
        profiling = true;
        for (int i = 0; i < nsteps; ++i) {
            std::vector<LaunchRec> recs;
            std::vector<size_t> off;
            int rc = 0;
            CK(cudaStreamSynchronize(st));
            const bool ens = upload_recorded(recs, off, rc);
            if (rc) { profiling = false; return rc; }
            if (ens) launch_recorded(recs, off);
            else one_step();
        }
        host_pending = ph.evolve != 0;
        profiling = false;
        CK(cudaStreamSynchronize(st));
        for (auto &e : evrecs) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e.a, e.b);
            kstats[e.k].ms += ms;
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        evrecs.clear();
        out = kstats;
        CK(cudaGetLastError());
        return check_status();
    }

    int check_status()
    {
        unsigned stv = 0;
        CK(cudaMemcpyAsync(&stv, &ctrl->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return take_status(stv);
    }

    int take_status(unsigned stv) override
    {
        if (stv) {
            CK(cudaMemsetAsync(&ctrl->status, 0, sizeof(unsigned), st));
            if (stv & ST_NONFINITE) { err = "state is not finite (NaN or Inf)"; return HYDFT_E_NONFINITE; }
            if (stv & ST_NONPOS) {
                err = "density became non-positive; reduce the amplitude or the time step";
                return HYDFT_E_NONPOS;
            }
        }
        return 0;
    }

    const unsigned *status_word() const override { return &ctrl->status; }

    int prepare() override { return tune(); }

    int radix_code(int axis) const override
    {
        const FFTPlan &p = axis == 0 ? g.px : (axis == 1 ? g.py : g.pz);
        int c = 0;
        for (int i = 0; i < p.nrad; ++i) c = 10 * c + p.rad[i];
        return radix_tuned ? c : -c;
    }
    void tiles(int *t) const override
    {
        t[0] = yz_tx;
        t[1] = yz_nt;
        t[2] = yz_txf;
        t[3] = yz_ntf;
        t[4] = x_ntmax;
    }

    int band_axes() const override { return (band_x ? 1 : 0) | (band_y ? 2 : 0) | (band_z ? 4 : 0); }

    // Grids of at least this many cells step with the plain kernels (their
    // arguments in the constant bank) alone and in ensembles: their launches
    // fill the GPU by themselves, and the ensemble form, which reads its
    // arguments from memory, holds them in registers (up to 25 % more per
    // thread in the transform passes).  Smaller grids step with the
    // ensemble form alone too, so that a model alone and the same model in
    // an ensemble group run the same kernels (bit-identical fields).
    // HYDFT_ENSEMBLE_MAX_CELLS overrides the 128^3 default.
    static size_t ensemble_max_cells()
    {
        const char *e = std::getenv("HYDFT_ENSEMBLE_MAX_CELLS");
        if (e && *e) return (size_t)std::strtoull(e, nullptr, 10);
        return (size_t)128 * 128 * 128;
    }

    int record_step(std::vector<LaunchRec> &out) override
    {
        if (int rc = tune()) return rc;
        out.clear();
        if (ncell >= ensemble_max_cells()) return HYDFT_E_UNSUPPORTED;
        rec = &out;
        rec_ok = true;
        one_step();
        rec = nullptr;
        if (!rec_ok) {
            out.clear();
            return HYDFT_E_UNSUPPORTED;
        }
        return 0;
    }

    void enqueue_steps(int k) override
    {
        for (int i = 0; i < k; ++i) one_step();
        if (k > 0) host_pending = ph.evolve != 0;
    }

    void mark_advanced() override { host_pending = ph.evolve != 0; }

    int64_t step_launches = 0;

    int advance(int nsteps) override
    {
        if (int rc = launch_steps(nsteps)) return rc;
        return check_status();
    }

    int poll_status() override { return check_status(); }

    void set_step(int64_t step) override
    {
        Ctrl c;
        cudaMemcpyAsync(&c, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        c.step = step;
        cudaMemcpyAsync(ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, st);
        cudaStreamSynchronize(st);
    }

    int probe_capacity() const override { return PROBE_CAP; }

    int probe_setup(int mx, int my, int mz) override
    {
        if (!pring) {
            if (int rc = alloc(pring, (size_t)5 * PROBE_CAP)) return rc;
            if (int rc = alloc(pcount, 1)) return rc;
        }
        CK(cudaMemsetAsync(pcount, 0, sizeof(int), st));
        // the compact index of the mode, as in mode()
        pconj = 0;
        if (mx < 0) { mx = -mx; my = -my; mz = -mz; pconj = 1; }
        auto wrapm = [](int m, int n) { m = ((m % n) + n) % n; return m <= n / 2 ? m : m - n; };
        my = g.ny > 1 ? wrapm(my, g.ny) : 0;
        mz = g.nz > 1 ? wrapm(mz, g.nz) : 0;
        if (mx > g.Mx || std::abs(my) > g.My || std::abs(mz) > g.Mz) {
            pidx = -1;
        } else {
            const int kyc = my >= 0 ? my : my + 2 * g.My + 1;
            const int kzc = mz >= 0 ? mz : mz + 2 * g.Mz + 1;
            pidx = ((long long)kzc * g.nkyc + kyc) * g.pkx + mx;
        }
        return 0;
    }

    int launch_steps_probed(int k, int every) override
    {
        if (!pring) { err = "probe_setup was not called"; return HYDFT_E_BAD; }
        Ctrl c;
        CK(cudaMemcpyAsync(&c, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        long long step = c.step;
        for (int i = 0; i < k; ++i) {
            if (int rc = launch_steps(1)) return rc;
            ++step;
            if (every > 0 && step % every == 0) {
                probe_kernel<R><<<1, 32, 0, st>>>(ctrl, N, M[0], pidx, pconj, pring, pcount, PROBE_CAP);
                launches++;
            }
        }
        CK(cudaGetLastError());
        return 0;
    }

    int read_probes(std::vector<double> &out) override
    {
        int cnt = 0;
        CK(cudaMemcpyAsync(&cnt, pcount, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        out.assign((size_t)5 * cnt, 0.0);
        if (cnt) CK(cudaMemcpyAsync(out.data(), pring, sizeof(double) * 5 * cnt, cudaMemcpyDeviceToHost, st));
        CK(cudaMemsetAsync(pcount, 0, sizeof(int), st));
        CK(cudaStreamSynchronize(st));
        return 0;
    }

    size_t device_bytes() const override { return alloc_bytes; }

    // Autotuner of the tile shapes and radix plans: times the phase-B
    // transform sequence (y/z inverse of its inputs, x pass B, y/z forward of
    // its outputs) with each candidate on the current data, writing only work
    // buffers.  Tile shapes (register-plan axes): it keeps for each of the
    // three groups the shape that ran it fastest; every shape gives the same
    // results to the bit (the same arithmetic per element, only the blocking
    // differs).  Radix plans (axes without a register plan, the generic
    // Stockham passes): it keeps the sequence whose whole phase-B time was
    // lowest; plans round differently, each within the oracle's tolerances.
    // The choice is shared by every model of the same grid, precision and
    // physics in the process.  HYDFT_TUNE=0 keeps the defaults, HYDFT_RADIX=0
    // the set-up radix plans.
    struct TuneKey {
        int nx, ny, nz, bytes, nm, evolve, ext;
        bool operator<(const TuneKey &o) const
        {
            return std::tie(nx, ny, nz, bytes, nm, evolve, ext) < std::tie(o.nx, o.ny, o.nz, o.bytes, o.nm, o.evolve, o.ext);
        }
    };
    // cached shape: kx columns and threads per y/z block of the inverse and
    // of the forward passes, threads per x block; and the radix plans of the
    // three axes
    struct TuneVal {
        std::array<int, 5> shape;
        FFTPlan px, py, pz;
    };
    static std::map<TuneKey, TuneVal> &tune_cache()
    {
        static std::map<TuneKey, TuneVal> m;
        return m;
    }

    // Radix plans the autotuner tries for an axis of length L = 2^a 3^b that
    // has no register plan (the generic Stockham passes): the 2^a part in
    // radix-8 steps or in radix-4 steps (a last 4 or 2 for the remainder),
    // the largest or the smallest radix first, the radix-3 steps after or
    // before them.  Every plan is the same transform; only the pass sequence
    // (and so the rounding) differs.
    static std::vector<FFTPlan> radix_candidates(int L)
    {
        std::vector<FFTPlan> out;
        int a = 0, b = 0, m = L;
        while (m % 2 == 0) { m /= 2; ++a; }
        while (m % 3 == 0) { m /= 3; ++b; }
        if (m != 1 || L < 2 || L > MAX_L) return out;
        for (int big : {8, 4}) {
            std::vector<int> twos;
            int r = a;
            const int lb = big == 8 ? 3 : 2;
            while (r >= lb) { twos.push_back(big); r -= lb; }
            if (r == 2) twos.push_back(4);
            else if (r == 1) twos.push_back(2);
            for (int asc = 0; asc < 2; ++asc)
                for (int threes_first = 0; threes_first < 2; ++threes_first) {
                    std::vector<int> t2 = twos, seq;
                    if (asc) std::sort(t2.begin(), t2.end());
                    else std::sort(t2.rbegin(), t2.rend());
                    const std::vector<int> t3(b, 3);
                    if (threes_first) { seq = t3; seq.insert(seq.end(), t2.begin(), t2.end()); }
                    else { seq = t2; seq.insert(seq.end(), t3.begin(), t3.end()); }
                    if (seq.empty() || (int)seq.size() > MAX_RAD) continue;
                    FFTPlan p{};
                    p.L = L;
                    p.nrad = (int)seq.size();
                    for (size_t i = 0; i < seq.size(); ++i) p.rad[i] = seq[i];
                    bool dup = false;
                    for (const FFTPlan &q : out) dup = dup || (q.nrad == p.nrad && std::equal(q.rad, q.rad + q.nrad, p.rad));
                    if (!dup) out.push_back(p);
                }
        }
        return out;
    }
    bool radix_tuned = false;
    static std::mutex &tune_mutex()
    {
        static std::mutex m;
        return m;
    }

    int tune()
    {
        if (tuned) return 0;
        tuned = true;
        const char *ev = std::getenv("HYDFT_TUNE");
        if (ev && std::string(ev) == "0") return 0;
        // fixed shapes on request (HYDFT_YZ_TILE = 8 | 16 | 32, HYDFT_YZ_THREADS =
        // YZ_NT | 2 YZ_NT, HYDFT_X_THREADS = 128 | 256)
        const char *fy = std::getenv("HYDFT_YZ_TILE"), *fx = std::getenv("HYDFT_X_THREADS");
        const char *fn = std::getenv("HYDFT_YZ_THREADS");
        // HYDFT_YZ_TILE_FWD / HYDFT_YZ_THREADS_FWD: the forward passes' shape alone
        const char *gy = std::getenv("HYDFT_YZ_TILE_FWD"), *gn = std::getenv("HYDFT_YZ_THREADS_FWD");
        auto set = [](const char *e) { return e && *e; };
        if (set(fy) || set(fx) || set(fn) || set(gy) || set(gn)) {
            auto tile = [](const char *e, int &a) {
                if (e && (std::atoi(e) == 8 || std::atoi(e) == 16 || std::atoi(e) == 32)) a = std::atoi(e);
            };
            auto nthr = [](const char *e, int &a) { if (e && (std::atoi(e) == YZ_NT || std::atoi(e) == 2 * YZ_NT)) a = std::atoi(e); };
            tile(fy, yz_tx);
            tile(fy, yz_txf);
            tile(gy, yz_txf);
            nthr(fn, yz_nt);
            nthr(fn, yz_ntf);
            nthr(gn, yz_ntf);
            if (fx && (std::string(fx) == "128" || std::string(fx) == "256")) x_ntmax = std::atoi(fx);
            return 0;
        }
        // the radix plans of axes without a register plan are tuned too
        // (HYDFT_RADIX=0 keeps the set-up plans)
        const char *er = std::getenv("HYDFT_RADIX");
        const bool radix_on = !(er && std::string(er) == "0");
        auto generic = [](int L) { return L > 1 && !has_plan(L); };
        const bool tile_tune = has_plan(g.ny) || has_plan(g.nz);
        const bool radix_tune = radix_on && (generic(g.nx) || generic(g.ny) || generic(g.nz));
        if (!tile_tune && !radix_tune) return 0;
        const TuneKey key{g.nx, g.ny, g.nz, (int)sizeof(R), nm, ph.evolve, ph.ext_active ? ph.ext_kind : 0};
        {
            std::lock_guard<std::mutex> lk(tune_mutex());
            auto it = tune_cache().find(key);
            if (it != tune_cache().end()) {
                yz_tx = it->second.shape[0];
                yz_nt = it->second.shape[1];
                yz_txf = it->second.shape[2];
                yz_ntf = it->second.shape[3];
                x_ntmax = it->second.shape[4];
                if (radix_tune) {
                    g.px = it->second.px;
                    g.py = it->second.py;
                    g.pz = it->second.pz;
                    radix_tuned = true;
                }
                return 0;
            }
        }
        // the phase-B pass sequence of stage 0
        const int nout = nm + (ph.evolve ? 6 : 0);
        PWB<R> pw;
        pw.ph = ph;
        pw.nm = nm;
        pw.nhat = N;
        pw.nmean = &ctrl->nmean;
        pw.dn_real = dn_real;
        pw.u_real = u_real;
        pw.ncell = ncell;
        pw.ex = ex; pw.ey = ey; pw.ez = ez;
        pw.gradv = gG;
        pw.ctrl = ctrl;
        pw.stage = 0;
        pw.status = &ctrl->status;
        const int64_t launches0 = launches;
        cudaEvent_t tev[4];
        for (auto &e : tev) CK(cudaEventCreate(&e));
        // one candidate: the inverse, x and forward groups timed apart (best
        // of two runs after a warm-up), so that each group's shape is chosen
        // by its own time
        auto time_it = [&](int tx, int ynt, int ntmax, float (&ms)[3]) {
            yz_tx = yz_txf = tx;
            yz_nt = yz_ntf = ynt;
            x_ntmax = ntmax;
            for (float &m : ms) m = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(tev[0], st);
                bool dxp = false;
                const int nf = phase_b_inverse(dxp);
                cudaEventRecord(tev[1], st);
                if (fast_x) xb_launch(nf, nout, pw, ph.evolve ? 1 + nm : 1, dxp);
                else xpass(nf, nout, pw, xrb_b, "xpass_b", ph.evolve ? 1 + nm : 1);
                cudaEventRecord(tev[2], st);
                forward(nout, OB);
                cudaEventRecord(tev[3], st);
                cudaEventSynchronize(tev[3]);
                for (int k = 0; k < 3; ++k) {
                    float t = 0.f;
                    cudaEventElapsedTime(&t, tev[k], tev[k + 1]);
                    if (rep > 0) ms[k] = std::min(ms[k], t);   // the first run warms up
                }
            }
        };
        const int txs[3] = {8, 16, 32};
        const int nts[2] = {128, 256};
        const int ynts[2] = {YZ_NT, 2 * YZ_NT};
        // the wide y/z blocks exist for the 256-point plan only
        const bool wide = g.ny == 256 || g.nz == 256;
        float bi = 1e30f, bx = 1e30f, bf = 1e30f;
        int btx = yz_tx, bynt = yz_nt, btxf = yz_txf, byntf = yz_ntf, bnt = x_ntmax;
        if (tile_tune)
            for (int tx : txs)
                for (int ynt : ynts)
                    for (int nt : nts) {
                        if (!fast_x && nt != 256) continue;
                        if (!wide && ynt != YZ_NT) continue;
                        float ms[3];
                        time_it(tx, ynt, nt, ms);
                        if (ms[0] < bi) { bi = ms[0]; btx = tx; bynt = ynt; }
                        if (ms[1] < bx) { bx = ms[1]; bnt = nt; }
                        if (ms[2] < bf) { bf = ms[2]; btxf = tx; byntf = ynt; }
                    }
        // radix plans: candidate i on every generic axis (an axis with fewer
        // candidates keeps its last), timed over the whole phase-B sequence
        // with the chosen tile shapes
        if (radix_tune) {
            const std::vector<FFTPlan> cx = generic(g.nx) ? radix_candidates(g.nx) : std::vector<FFTPlan>{g.px};
            const std::vector<FFTPlan> cy = generic(g.ny) ? radix_candidates(g.ny) : std::vector<FFTPlan>{g.py};
            const std::vector<FFTPlan> cz = generic(g.nz) ? radix_candidates(g.nz) : std::vector<FFTPlan>{g.pz};
            const size_t nc = std::max(cx.size(), std::max(cy.size(), cz.size()));
            FFTPlan best[3] = {g.px, g.py, g.pz};
            float bt = 1e30f;
            for (size_t i = 0; i < nc && !cx.empty() && !cy.empty() && !cz.empty(); ++i) {
                g.px = cx[std::min(i, cx.size() - 1)];
                g.py = cy[std::min(i, cy.size() - 1)];
                g.pz = cz[std::min(i, cz.size() - 1)];
                float ms[3];
                time_it(btx, bynt, bnt, ms);
                yz_txf = btxf;
                yz_ntf = byntf;
                const float tot = ms[0] + ms[1] + ms[2];
                if (tot < bt) { bt = tot; best[0] = g.px; best[1] = g.py; best[2] = g.pz; }
            }
            g.px = best[0];
            g.py = best[1];
            g.pz = best[2];
            radix_tuned = true;
        }
        for (auto &e : tev) cudaEventDestroy(e);
        launches = launches0;
        yz_tx = btx;
        yz_nt = bynt;
        yz_txf = btxf;
        yz_ntf = byntf;
        x_ntmax = bnt;
        CK(cudaGetLastError());
        std::lock_guard<std::mutex> lk(tune_mutex());
        tune_cache()[key] = TuneVal{{btx, bynt, btxf, byntf, bnt}, g.px, g.py, g.pz};
        return 0;
    }

    // The step's launches as an ensemble of one: each launch of one recorded
    // step is the ensemble form with n = 1 and the solver's own pack, so that
    // the model alone and the same model in an ensemble group run the same
    // compiled kernels (bit-identical fields).  upload_recorded records one
    // step and prepares the ensemble forms (outside any capture); it returns
    // false when a launch of the step has no ensemble form.
    bool upload_recorded(std::vector<LaunchRec> &recs, std::vector<size_t> &off, int &rc)
    {
        rc = 0;
        if (record_step(recs)) return false;
        off.assign(recs.size(), 0);
        cudaError_t e = cudaSuccess;
        for (size_t i = 0; e == cudaSuccess && i < recs.size(); ++i) e = recs[i].prepare(recs[i].smem);
        if (e != cudaSuccess) { err = std::string("ensemble form: ") + cudaGetErrorString(e); rc = HYDFT_E_CUDA; }
        return true;
    }

    void launch_recorded(const std::vector<LaunchRec> &recs, const std::vector<size_t> &off)
    {
        for (size_t i = 0; i < recs.size(); ++i) {
            const LaunchRec &r = recs[i];
            cudaEvent_t ea = nullptr, eb = nullptr;
            if (profiling) {
                cudaEventCreate(&ea);
                cudaEventCreate(&eb);
                cudaEventRecord(ea, st);
            }
            r.launch(r.pack.data(), 1, r.grid, r.block, r.smem, st);
            launches++;
            if (profiling) {
                cudaEventRecord(eb, st);
                int k = -1;
                for (size_t j = 0; j < kstats.size(); ++j)
                    if (kstats[j].name == r.name) k = (int)j;
                if (k < 0) {
                    kstats.push_back(KStat());
                    kstats.back().name = r.name;
                    k = (int)kstats.size() - 1;
                }
                kstats[k].bytes += r.bytes;
                kstats[k].n += 1;
                evrecs.push_back({k, ea, eb});
            }
        }
    }

    int launch_steps(int nsteps) override
    {
        if (int rc = tune()) return rc;
        if (nsteps <= 0) return 0;
        if (!gexec) {
            const int64_t before = launches;
            // the step is recorded and its ensemble forms prepared before the
            // capture begins
            std::vector<LaunchRec> recs;
            std::vector<size_t> off;
            int rc = 0;
            CK(cudaStreamSynchronize(st));
            const bool ens = upload_recorded(recs, off, rc);
            if (rc) return rc;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            if (ens) launch_recorded(recs, off);
            else one_step();
            cudaGraph_t gr = nullptr;
            CK(cudaStreamEndCapture(st, &gr));
            graph = gr;
            step_launches = launches - before;
            launches = before;
            CK(cudaGraphInstantiate(&gexec, graph, 0));
        }
        for (int i = 0; i < nsteps; ++i) {
            CK(cudaGraphLaunch(gexec, st));
            launches += step_launches;
        }
        host_pending = ph.evolve != 0;
        CK(cudaGetLastError());
        return 0;
    }

    int rhs(double t, double *dn, double *dmom, double *dpi) override
    {
        finish_if_pending();
        // t only enters through the external force: set the stage scalars of
        // stage 0 at time t
        double t0, dt0;
        int64_t s0;
        get_time(&t0, &dt0, &s0);
        set_time(t, dt0);
        begin_step();
        phase_a(0, ph.evolve != 0);
        phase_b(0, true);
        vlast_kernel<<<1, 32, 0, st>>>(ctrl, 0);
        launches++;
        set_time(t0, dt0);
        CK(cudaGetLastError());
        if (int rc = check_status()) return rc;
        // outputs to real space
        const cplx<R> *src[MAXF];
        R *dsts[MAXF];
        int nf = 0;
        src[nf] = HN; dsts[nf++] = io_real;
        for (int d = 0; d < 3; ++d) { src[nf] = HM[d]; dsts[nf++] = io_real + (1 + d) * ncell; }
        if (int rc = to_real(nf, src, dsts)) return rc;
        if (int rc = down(dn, io_real, 1, 0.0)) return rc;
        if (int rc = down(dmom, io_real + ncell, 3, 0.0)) return rc;
        if (ph.evolve && dpi) {
            nf = 0;
            for (int q = 0; q < 6; ++q) { src[nf] = HP[q]; dsts[nf++] = io_real + q * ncell; }
            if (int rc = to_real(nf, src, dsts)) return rc;
            if (int rc = down(dpi, io_real, 6, 0.0)) return rc;
        }
        return 0;
    }

    // compact fields -> real-space device arrays
    int to_real(int nf, const cplx<R> *const *src, R *const *dst)
    {
        int ops[MAXF];
        for (int f = 0; f < nf; ++f) ops[f] = OP_ID;
        inverse(nf, src, ops);
        PWToReal<R> pw;
        for (int f = 0; f < MAXF; ++f) pw.dst[f] = f < nf ? dst[f] : nullptr;
        pw.ncell = ncell;
        x_toreal(nf, pw);
        CK(cudaGetLastError());
        return 0;
    }

    void x_toreal(int nf, const PWToReal<R> &pw)
    {
        if (fast_x) {
            PWFromReal<R> none;
            for (int f = 0; f < MAXF; ++f) none.src[f] = nullptr;
            none.nf = 0;
            xio_launch(nf, 0, pw, none, "xpass_io");
        } else {
            xpass(nf, 0, pw, xrb_io, "xpass_io");
        }
    }

    // real-space device arrays -> compact fields (masked to the band)
    int from_real(int nf, const R *const *src, cplx<R> *const *dst)
    {
        PWFromReal<R> pw;
        for (int f = 0; f < MAXF; ++f) pw.src[f] = f < nf ? src[f] : nullptr;
        pw.nf = nf;
        if (fast_x) {
            PWToReal<R> none;
            for (int f = 0; f < MAXF; ++f) none.dst[f] = nullptr;
            none.ncell = ncell;
            xio_launch(0, nf, none, pw, "xpass_io");
        } else {
            xpass(0, nf, pw, xrb_io, "xpass_io");
        }
        forward(nf, const_cast<cplx<R> *const *>(dst));
        CK(cudaGetLastError());
        return 0;
    }

    // device real (R) -> host double, ncomp fields
    // device fields (R) -> host FP64 arrays, one component at a time through
    // the FP64 staging field
    int down(double *h, const R *d, int ncomp, double add)
    {
        for (int c = 0; c < ncomp; ++c) {
            real_to_double_kernel<R><<<592, 256, 0, st>>>(stage, d + (size_t)c * ncell, add, ncell);
            launches++;
            CK(cudaMemcpyAsync(h + (size_t)c * ncell, stage, ncell * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        CK(cudaStreamSynchronize(st));
        return 0;
    }

    // host FP64 arrays -> device fields (R) minus `sub`, through the staging field
    int up(R *d, const double *h, int ncomp, double sub)
    {
        for (int c = 0; c < ncomp; ++c) {
            CK(cudaMemcpyAsync(stage, h + (size_t)c * ncell, ncell * sizeof(double), cudaMemcpyHostToDevice, st));
            fill_real_kernel<R><<<592, 256, 0, st>>>(d + (size_t)c * ncell, stage, sub, ncell);
            launches++;
        }
        return 0;
    }

    int set_state(const double *n, const double *mom, const double *pi) override
    {
        if (!n || !mom) { err = "set_state: n and mom are required"; return HYDFT_E_BAD; }
        if (ph.evolve && !pi) { err = "set_state: pi is required for the Maxwell closure"; return HYDFT_E_BAD; }
        // the density in FP64 on the device: its mean (the k = 0 mode, kept
        // exactly; the deviations are transformed in R), minimum and
        // non-finite count
        CK(cudaMemcpyAsync(stage, n, ncell * sizeof(double), cudaMemcpyHostToDevice, st));
        density_stats_kernel<<<red_blocks, 256, 0, st>>>(stage, ncell, spart);
        launches++;
        std::vector<double> hp((size_t)red_blocks * NSUM);
        CK(cudaMemcpyAsync(hp.data(), spart, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double s = 0.0, c = 0.0, nmin = 1e300, bad = 0.0;
        for (int b = 0; b < red_blocks; ++b) {
            const double v = hp[(size_t)b * NSUM];
            const double t = s + v;
            if (std::fabs(s) >= std::fabs(v)) c += (s - t) + v; else c += (v - t) + s;
            s = t;
            nmin = std::min(nmin, hp[(size_t)b * NSUM + 1]);
            bad += hp[(size_t)b * NSUM + 2];
        }
        if (bad > 0.0 || !(nmin > 0.0)) {
            err = "initial density is not positive";
            return HYDFT_E_NONPOS;
        }
        const double nmean = (s + c) / (double)ncell;
        fill_real_kernel<R><<<592, 256, 0, st>>>(io_real, stage, nmean, ncell);
        launches++;
        if (int rc = up(io_real + ncell, mom, 3, 0.0)) return rc;
        const R *src[4] = {io_real, io_real + ncell, io_real + 2 * ncell, io_real + 3 * ncell};
        cplx<R> *dst[4] = {N, M[0], M[1], M[2]};
        if (int rc = from_real(4, src, dst)) return rc;
        set_k0_kernel<R><<<1, 32, 0, st>>>(N, nmean);
        launches++;
        CK(cudaMemcpyAsync(&ctrl->nmean, &nmean, sizeof(double), cudaMemcpyHostToDevice, st));
        if (ph.evolve) {
            if (int rc = up(io_real, pi, 6, 0.0)) return rc;
            const R *sp[6];
            cplx<R> *dp[6];
            for (int q = 0; q < 6; ++q) { sp[q] = io_real + q * ncell; dp[q] = P[q]; }
            if (int rc = from_real(6, sp, dp)) return rc;
        }
        CK(cudaMemsetAsync(&ctrl->pending, 0, sizeof(int), st));
        host_pending = false;
        CK(cudaStreamSynchronize(st));
        return 0;
    }

    int get_state(double *n, double *mom, double *pi) override
    {
        finish_if_pending();
        double nmean = 0.0;
        {
            CK(cudaMemcpyAsync(&nmean, &ctrl->nmean, sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        const cplx<R> *src[MAXF];
        R *dsts[MAXF];
        int nf = 0;
        src[nf] = N; dsts[nf++] = io_real;
        for (int d = 0; d < 3; ++d) { src[nf] = M[d]; dsts[nf++] = io_real + (1 + d) * ncell; }
        // n without its mean, added back in FP64
        {
            int ops[MAXF];
            ops[0] = OP_ZK0;
            for (int f = 1; f < nf; ++f) ops[f] = OP_ID;
            inverse(nf, src, ops);
            PWToReal<R> pw;
            for (int f = 0; f < MAXF; ++f) pw.dst[f] = f < nf ? dsts[f] : nullptr;
            pw.ncell = ncell;
            x_toreal(nf, pw);
        }
        if (n) if (int rc = down(n, io_real, 1, nmean)) return rc;
        if (mom) if (int rc = down(mom, io_real + ncell, 3, 0.0)) return rc;
        if (ph.evolve && pi) {
            nf = 0;
            for (int q = 0; q < 6; ++q) { src[nf] = P[q]; dsts[nf++] = io_real + q * ncell; }
            if (int rc = to_real(nf, src, dsts)) return rc;
            if (int rc = down(pi, io_real, 6, 0.0)) return rc;
        }
        return 0;
    }

    int reductions(double *sum_n, double sum_m[3], double *sum_m2n, double *nmin, double *nmax,
                   double *umax) override
    {
        const cplx<R> *src[4] = {N, M[0], M[1], M[2]};
        int ops[4] = {OP_ZK0, OP_ID, OP_ID, OP_ID};
        inverse(1 + nm, src, ops);
        PWToReal<R> pw;
        for (int f = 0; f < MAXF; ++f) pw.dst[f] = nullptr;
        pw.dst[0] = io_real;
        for (int d = 0; d < nm; ++d) pw.dst[1 + d] = io_real + (1 + d) * ncell;
        pw.ncell = ncell;
        x_toreal(1 + nm, pw);
        reduce_fields_kernel<R><<<red_blocks, 256, 0, st>>>(io_real, io_real + ncell, ncell, nm, &ctrl->nmean,
                                                            ph.inv_mass, rpart);
        reduce_final_kernel<R><<<1, 32, 0, st>>>(rpart, red_blocks, rout);
        launches += 2;
        RedPart h;
        CK(cudaMemcpyAsync(&h, rout, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        *sum_n = h.sn;
        for (int d = 0; d < 3; ++d) sum_m[d] = d < nm ? h.sm[d] : 0.0;
        *sum_m2n = h.sk;
        *nmin = h.nmin;
        *nmax = h.nmax;
        *umax = h.umax;
        return 0;
    }

    int energy(double *fe) override
    {
        const int ngr = ph.has_grad ? nm : 0;
        const cplx<R> *src[4] = {N, N, N, N};
        int ops[4] = {OP_ZK0, OP_IKX, OP_IKY, OP_IKZ};
        inverse(1 + ngr, src, ops);
        PWToReal<R> pw;
        for (int f = 0; f < MAXF; ++f) pw.dst[f] = nullptr;
        pw.dst[0] = io_real;
        for (int d = 0; d < ngr; ++d) pw.dst[1 + d] = io_real + (size_t)(1 + d) * ncell;
        pw.ncell = ncell;
        if (ph.has_grad && nm < 3)
            CK(cudaMemsetAsync(io_real + (size_t)(1 + nm) * ncell, 0, (3 - nm) * ncell * sizeof(R), st));
        x_toreal(1 + ngr, pw);
        double nmean = 0.0;
        CK(cudaMemcpyAsync(&nmean, &ctrl->nmean, sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double spec[NSUM], real[NSUM];
        energy_spec_kernel<R><<<red_blocks, 256, 0, st>>>(g, N, Kh, Kr, spart);
        sums_final_kernel<<<1, 32, 0, st>>>(spart, red_blocks, sout);
        CK(cudaMemcpyAsync(spec, sout, sizeof(spec), cudaMemcpyDeviceToHost, st));
        EnergyReal e;
        e.nref = nmean;
        e.fdtab = fdtab;
        e.cn = S.cn;
        e.ideal = ph.has_ideal;
        e.tf = ph.has_tf;
        e.grad = ph.has_grad;
        e.ext = !ph.ext_active ? 0 : (ph.ext_kind == 3 ? 2 : 1);
        e.ex = ex; e.ey = ey; e.ez = ez;
        e.ctrl = ctrl;
        energy_real_kernel<R><<<red_blocks, 256, 0, st>>>(g, io_real, io_real + ncell, gV, ncell, e, spart);
        sums_final_kernel<<<1, 32, 0, st>>>(spart, red_blocks, sout);
        CK(cudaMemcpyAsync(real, sout, sizeof(real), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        launches += 4;
        CK(cudaGetLastError());
        // terms in input order (functional.f90:80-90), each mean * volume
        const double nc = (double)ncell, vol = S.volume, beta = S.beta;
        double f = 0.0;
        for (int i = 0; i < S.neterms; ++i) {
            switch (S.eterm_order[i]) {
            case 1: f += real[2] / nc * vol / beta; break;
            case 2: f += real[3] / nc * vol / beta; break;
            case 3: f += S.cg * real[4] / nc * vol; break;
            case 4: f += 0.5 * (spec[0] + S.vk0 * nmean * nmean) * vol; break;
            case 5: {
                const double b0 = nmean - S.n0;
                f += -0.5 * (spec[1] + S.ck0 * b0 * b0) * vol / beta;
                break;
            }
            default: break;
            }
        }
        if (ph.ext_active) f += real[5] / nc * vol;
        *fe = f;
        return 0;
    }

    int mode(int field, int mx, int my, int mz, double *re, double *im) override
    {
        // the state is dealiased: coefficients outside the band are zero
        const cplx<R> *f = field == 0 ? N : M[field - 1];
        bool conjugate = false;
        if (mx < 0) { mx = -mx; my = -my; mz = -mz; conjugate = true; }
        // wrap to the signed range of each axis
        auto wrapm = [](int m, int n) { m = ((m % n) + n) % n; return m <= n / 2 ? m : m - n; };
        my = g.ny > 1 ? wrapm(my, g.ny) : 0;
        mz = g.nz > 1 ? wrapm(mz, g.nz) : 0;
        if (mx > g.Mx || std::abs(my) > g.My || std::abs(mz) > g.Mz) {
            *re = 0.0;
            *im = 0.0;
            return 0;
        }
        if (field == 0 && mx == 0 && my == 0 && mz == 0) {
            // the mean density, kept in FP64
            CK(cudaMemcpyAsync(re, &ctrl->nmean, sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            *im = 0.0;
            return 0;
        }
        const int kyc = my >= 0 ? my : my + 2 * g.My + 1;
        const int kzc = mz >= 0 ? mz : mz + 2 * g.Mz + 1;
        cplx<R> h;
        CK(cudaMemcpyAsync(&h, f + ((size_t)kzc * g.nkyc + kyc) * g.pkx + mx, sizeof(h), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        *re = (double)h.x;
        *im = conjugate ? -(double)h.y : (double)h.y;
        return 0;
    }

    void set_time(double t, double dt) override
    {
        Ctrl c;
        cudaMemcpyAsync(&c, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        c.t = t;
        c.dt = dt;
        cudaMemcpyAsync(ctrl, &c, sizeof(Ctrl), cudaMemcpyHostToDevice, st);
        cudaStreamSynchronize(st);
    }

    void get_time(double *t, double *dt, int64_t *step) override
    {
        Ctrl c;
        cudaMemcpyAsync(&c, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        if (t) *t = c.t;
        if (dt) *dt = c.dt;
        if (step) *step = c.step;
    }
};

// One precision per translation unit (solver_f32.cu / solver_f64.cu).
SolverBase *HYDFT_MAKE_FN(const SolverSetup &s, int device, std::string &err)
{
    auto *p = new Solver<HYDFT_REAL>();
    if (int rc = p->init(s, device)) {
        (void)rc;
        err = p->err;
        delete p;
        return nullptr;
    }
    return p;
}

}  // namespace hydft
