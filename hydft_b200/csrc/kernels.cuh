// Transform passes and fused pointwise/spectral kernels of the solver step.
//
// Data layouts (complex unless noted; kx runs padded to g.pkx):
//   compact  [kzc][kyc][kx]   the dealiased band: state, tendencies, mu
//   ZI       [z  ][kyc][kx]   after the z transform
//   YI / XF  [z  ][y  ][kx]   after the y transform (x still spectral)
//   real     [z  ][y  ][x ]   R, only for the few fields phase B re-reads
// A 3-D inverse transform is zinv -> yinv -> (x pass); a forward one is
// (x pass) -> yfwd -> zfwd.  The x pass does the c2r of its inputs, the
// pointwise physics and the r2c of its outputs for a block of rows without
// storing the real-space fields, so nonlinear products never touch HBM in
// real space.  Only modes inside the 2/3 band are read or written: every
// consumer of a forward transform multiplies by the dealiasing mask, so the
// pruned modes would be multiplied by zero.
#pragma once

#include "common.cuh"
#include "fermi_dirac.cuh"
#include "fft.cuh"

namespace hydft {

constexpr int MAXF = 24;

// spectral operators applied on load in zinv
enum : int { OP_ID = 0, OP_ZK0 = 1, OP_IKX = 2, OP_IKY = 3, OP_IKZ = 4, OP_NK2 = 5 };

template <typename R>
struct PassArgs {
    int nf;
    const cplx<R> *in[MAXF];
    cplx<R> *out[MAXF];
    int op[MAXF];
};

// twiddle tables exp(-2 pi i t/L), t < L, for the three axes
template <typename R>
struct Twiddles {
    const cplx<R> *x, *y, *z;
};

template <typename R>
__device__ __forceinline__ void load_tw(cplx<R> *dst, const cplx<R> *src, int L)
{
    for (int t = threadIdx.x; t < L; t += blockDim.x) dst[t] = src[t];
}

// ---------------------------------------------------------------- z inverse
// grid (ceil(nkxc/TX), nkyc, nf); smem 2*nz*TX + nz complex
template <typename R, int TX>
__global__ void __launch_bounds__(256) zinv_kernel(Grid g, PassArgs<R> a, const cplx<R> *twz)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *A = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *B = A + g.nz * TX;
    cplx<R> *tw = B + g.nz * TX;
    const int x0 = blockIdx.x * TX, kyc = blockIdx.y, f = blockIdx.z;
    const cplx<R> *__restrict__ in = a.in[f];
    cplx<R> *__restrict__ out = a.out[f];
    const int op = a.op[f];
    load_tw(tw, twz, g.nz);
    for (int i = threadIdx.x; i < g.nz * TX; i += blockDim.x) A[i] = cplx<R>{R(0), R(0)};
    __syncthreads();
    const int my = signed_idx(kyc, g.My);
    const R ky = R(my * g.ky0);
    for (int i = threadIdx.x; i < g.nkzc * TX; i += blockDim.x) {
        const int kzc = i / TX, c = i % TX, xx = x0 + c;
        if (xx >= g.nkxc) continue;
        cplx<R> v = in[((size_t)kzc * g.nkyc + kyc) * g.pkx + xx];
        const int mz = signed_idx(kzc, g.Mz);
        switch (op) {
        case OP_ZK0: if (xx == 0 && my == 0 && mz == 0) v = cplx<R>{R(0), R(0)}; break;
        case OP_IKX: v = ik_times(R(xx * g.kx0), v); break;
        case OP_IKY: v = ik_times(ky, v); break;
        case OP_IKZ: v = ik_times(R(mz * g.kz0), v); break;
        case OP_NK2: {
            const R kx = R(xx * g.kx0), kz = R(mz * g.kz0);
            v = R(-(kx * kx + ky * ky + kz * kz)) * v;
            break;
        }
        default: break;
        }
        A[fft_idx(mz, g.nz) * TX + c] = v;
    }
    __syncthreads();
    cplx<R> *res = fft_smem<+1>(A, B, g.pz, TX, TX, 1, true, tw);
    for (int i = threadIdx.x; i < g.nz * TX; i += blockDim.x) {
        const int z = i / TX, c = i % TX, xx = x0 + c;
        if (xx < g.nkxc) out[((size_t)z * g.nkyc + kyc) * g.pkx + xx] = res[i];
    }
}

// ---------------------------------------------------------------- y inverse
// grid (ceil(nkxc/TX), nz, nf)
template <typename R, int TX>
__global__ void __launch_bounds__(256) yinv_kernel(Grid g, PassArgs<R> a, const cplx<R> *twy)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *A = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *B = A + g.ny * TX;
    cplx<R> *tw = B + g.ny * TX;
    const int x0 = blockIdx.x * TX, z = blockIdx.y, f = blockIdx.z;
    const cplx<R> *__restrict__ in = a.in[f];
    cplx<R> *__restrict__ out = a.out[f];
    load_tw(tw, twy, g.ny);
    for (int i = threadIdx.x; i < g.ny * TX; i += blockDim.x) A[i] = cplx<R>{R(0), R(0)};
    __syncthreads();
    for (int i = threadIdx.x; i < g.nkyc * TX; i += blockDim.x) {
        const int kyc = i / TX, c = i % TX, xx = x0 + c;
        if (xx >= g.nkxc) continue;
        A[fft_idx(signed_idx(kyc, g.My), g.ny) * TX + c] = in[((size_t)z * g.nkyc + kyc) * g.pkx + xx];
    }
    __syncthreads();
    cplx<R> *res = fft_smem<+1>(A, B, g.py, TX, TX, 1, true, tw);
    for (int i = threadIdx.x; i < g.ny * TX; i += blockDim.x) {
        const int y = i / TX, c = i % TX, xx = x0 + c;
        if (xx < g.nkxc) out[((size_t)z * g.ny + y) * g.pkx + xx] = res[i];
    }
}

// ---------------------------------------------------------------- y forward
// grid (ceil(nkxc/TX), nz, nf)
template <typename R, int TX>
__global__ void __launch_bounds__(256) yfwd_kernel(Grid g, PassArgs<R> a, const cplx<R> *twy)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *A = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *B = A + g.ny * TX;
    cplx<R> *tw = B + g.ny * TX;
    const int x0 = blockIdx.x * TX, z = blockIdx.y, f = blockIdx.z;
    const cplx<R> *__restrict__ in = a.in[f];
    cplx<R> *__restrict__ out = a.out[f];
    load_tw(tw, twy, g.ny);
    for (int i = threadIdx.x; i < g.ny * TX; i += blockDim.x) {
        const int y = i / TX, c = i % TX, xx = x0 + c;
        A[i] = xx < g.nkxc ? in[((size_t)z * g.ny + y) * g.pkx + xx] : cplx<R>{R(0), R(0)};
    }
    __syncthreads();
    cplx<R> *res = fft_smem<-1>(A, B, g.py, TX, TX, 1, true, tw);
    for (int i = threadIdx.x; i < g.nkyc * TX; i += blockDim.x) {
        const int kyc = i / TX, c = i % TX, xx = x0 + c;
        if (xx < g.nkxc)
            out[((size_t)z * g.nkyc + kyc) * g.pkx + xx] = res[fft_idx(signed_idx(kyc, g.My), g.ny) * TX + c];
    }
}

// ---------------------------------------------------------------- z forward
// grid (ceil(nkxc/TX), nkyc, nf); applies the 1/(nx ny nz) normalisation
template <typename R, int TX>
__global__ void __launch_bounds__(256) zfwd_kernel(Grid g, PassArgs<R> a, const cplx<R> *twz, R norm)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *A = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *B = A + g.nz * TX;
    cplx<R> *tw = B + g.nz * TX;
    const int x0 = blockIdx.x * TX, kyc = blockIdx.y, f = blockIdx.z;
    const cplx<R> *__restrict__ in = a.in[f];
    cplx<R> *__restrict__ out = a.out[f];
    load_tw(tw, twz, g.nz);
    for (int i = threadIdx.x; i < g.nz * TX; i += blockDim.x) {
        const int z = i / TX, c = i % TX, xx = x0 + c;
        A[i] = xx < g.nkxc ? in[((size_t)z * g.nkyc + kyc) * g.pkx + xx] : cplx<R>{R(0), R(0)};
    }
    __syncthreads();
    cplx<R> *res = fft_smem<-1>(A, B, g.pz, TX, TX, 1, true, tw);
    for (int i = threadIdx.x; i < g.nkzc * TX; i += blockDim.x) {
        const int kzc = i / TX, c = i % TX, xx = x0 + c;
        if (xx < g.nkxc)
            out[((size_t)kzc * g.nkyc + kyc) * g.pkx + xx] = norm * res[fft_idx(signed_idx(kzc, g.Mz), g.nz) * TX + c];
    }
}

// ------------------------------------------------------------------ x pass
template <typename R>
struct XArgs {
    int nin, nout;
    const cplx<R> *in[MAXF];   // YI layout
    cplx<R> *out[MAXF];        // XF layout
};

// Shared-memory bytes of the x pass for RB rows.
template <typename R>
__host__ __device__ inline size_t xpass_smem(int nx, int RB, int nin, int nout)
{
    return sizeof(cplx<R>) * (size_t)(nx + 2 * RB * nx) + sizeof(R) * (size_t)RB * nx * (nin + nout);
}

// c2r of the inputs (two real fields per complex transform), pointwise
// functor, r2c of the outputs.  grid: ceil(ny*nz/RB) blocks.
template <typename R, class PW>
__global__ void __launch_bounds__(256) xpass_kernel(Grid g, XArgs<R> a, const cplx<R> *twx, PW pw, int RB)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    const int nx = g.nx;
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *A = tw + nx;
    cplx<R> *B = A + RB * nx;
    R *Fin = reinterpret_cast<R *>(B + RB * nx);
    R *Fout = Fin + (size_t)a.nin * RB * nx;
    const int stride = RB * nx;
    const int nrows = g.ny * g.nz;
    const int row0 = blockIdx.x * RB;
    const int Mx = g.Mx;
    load_tw(tw, twx, nx);
    // ---- c2r of the inputs, two at a time
    for (int p = 0; 2 * p < a.nin; ++p) {
        const int fa = 2 * p, fb = 2 * p + 1;
        const bool hasb = fb < a.nin;
        for (int i = threadIdx.x; i < stride; i += blockDim.x) {
            const int rr = i / nx, k = i % nx, row = row0 + rr;
            cplx<R> Z = {R(0), R(0)};
            if (row < nrows) {
                if (k <= Mx) {
                    cplx<R> va = a.in[fa][(size_t)row * g.pkx + k];
                    cplx<R> vb = hasb ? a.in[fb][(size_t)row * g.pkx + k] : cplx<R>{R(0), R(0)};
                    if (k == 0) { va.y = R(0); vb.y = R(0); }   // c2r keeps Re of the kx = 0 bin
                    Z = cplx<R>{va.x - vb.y, va.y + vb.x};       // A + iB
                } else if (k >= nx - Mx) {
                    const int kk = nx - k;
                    cplx<R> va = a.in[fa][(size_t)row * g.pkx + kk];
                    cplx<R> vb = hasb ? a.in[fb][(size_t)row * g.pkx + kk] : cplx<R>{R(0), R(0)};
                    Z = cplx<R>{va.x + vb.y, -va.y + vb.x};      // conj(A) + i conj(B)
                }
            }
            A[i] = Z;
        }
        __syncthreads();
        cplx<R> *res = fft_smem<+1>(A, B, g.px, RB, 1, nx, false, tw);
        for (int i = threadIdx.x; i < stride; i += blockDim.x) {
            Fin[(size_t)fa * stride + i] = res[i].x;
            if (hasb) Fin[(size_t)fb * stride + i] = res[i].y;
        }
        __syncthreads();
    }
    // ---- pointwise
    for (int i = threadIdx.x; i < stride; i += blockDim.x) {
        const int rr = i / nx, x = i % nx, row = row0 + rr;
        if (row < nrows) pw(g, row, x, Fin + i, Fout + i, stride);
    }
    __syncthreads();
    // ---- r2c of the outputs, two at a time
    for (int p = 0; 2 * p < a.nout; ++p) {
        const int fa = 2 * p, fb = 2 * p + 1;
        const bool hasb = fb < a.nout;
        for (int i = threadIdx.x; i < stride; i += blockDim.x)
            A[i] = cplx<R>{Fout[(size_t)fa * stride + i], hasb ? Fout[(size_t)fb * stride + i] : R(0)};
        __syncthreads();
        cplx<R> *res = fft_smem<-1>(A, B, g.px, RB, 1, nx, false, tw);
        const int nk = Mx + 1;
        for (int i = threadIdx.x; i < RB * nk; i += blockDim.x) {
            const int rr = i / nk, k = i % nk, row = row0 + rr;
            if (row >= nrows) continue;
            const cplx<R> zk = res[rr * nx + k];
            const cplx<R> zm = conj(res[rr * nx + (k == 0 ? 0 : nx - k)]);
            const cplx<R> s = R(0.5) * (zk + zm);
            const cplx<R> d = mul_i<-1>(R(0.5) * (zk - zm));
            a.out[fa][(size_t)row * g.pkx + k] = s;
            if (hasb) a.out[fb][(size_t)row * g.pkx + k] = d;
        }
        __syncthreads();
    }
}

// per-stage scalars in device memory (the step is graph-captured)
struct StageScal {
    double ts;        // stage time
    double amp;       // external amplitude A(ts)
    double ewr, ewi;  // exp(-i omega ts)
    double a, b;      // RK coefficients
    double phi, e;    // relaxation factors of this stage
};

struct Ctrl {
    double t, dt;
    long long step;
    StageScal st[3];
    double nkd_re, nkd_im;   // nhat at the drive mode, stage start
    double pend_phi, pend_e; // relaxation factors of the pending stage
    unsigned status;
    int pending;             // Maxwell relaxation pending
    // external potential as last evaluated (vext_t%v after the last rhs):
    // amplitude and exp(-i omega t) of that time
    double v_amp, v_ewr, v_ewi;
    double gf[3];            // mean of n F_ext for the gaussian potential, stage start
    double nmean;            // mean density in FP64 (conserved; the k = 0 mode of n)
};

// physics constants for the pointwise and spectral kernels
struct Phys {
    double beta, inv_beta, mass, inv_mass, n0;
    int has_ideal, has_tf, has_grad, term_order[8], nterms_local;
    double cn, cg, alpha_ref;
    int evolve, newtonian;   // Pi evolved / Newtonian stress from u
    double eta, xi, tau;
    int ext_active, ext_kind;     // 1 mode, 2 driven, 3 gaussian
    double ext_k[3], ext_amp, ext_omega, ext_ramp;
    int drive_in_band, drive_idx;  // compact index of the drive mode
    int drive_conj;                // drive mode stored as its conjugate
};

// --------------------------------------------------------- phase A functor
// inputs:  0 dn, 1..nm m_d, [grad: nm+1.. dn/dx_d (nm), lap n]
// outputs: 0..nm-1 u_d, fluxes m_i u_j (i<=j), mu_local
template <typename R>
struct PWA {
    Phys ph;
    int nm;
    const cplx<R> *nhat;       // compact n
    const double *nmean;       // the mean density in FP64
    const double *fdtab;
    R *dn_real;                // real-space dn for phase B
    R *u_real;                 // real-space u (3 fields) when Pi evolves
    size_t ncell;
    unsigned *status;

    __device__ void operator()(const Grid &g, int row, int x, const R *Fin, R *Fout, int stride) const
    {
        const double nref = *nmean;
        const R dn = Fin[0];
        const double n = nref + (double)dn;
        const size_t q = (size_t)row * g.nx + x;
        if (!(n > 0.0)) atomicOr(status, isfinite(n) ? ST_NONPOS : ST_NONFINITE);
        const R inv_mn = R(1.0 / (ph.mass * n));
        R m[3], u[3];
        for (int d = 0; d < nm; ++d) {
            m[d] = Fin[(1 + d) * stride];
            u[d] = m[d] * inv_mn;
            Fout[d * stride] = u[d];
        }
        int o = nm;
        for (int i = 0; i < nm; ++i)
            for (int j = i; j < nm; ++j) Fout[(o++) * stride] = m[i] * u[j];
        double mu = 0.0;
        bool have_alpha = false;
        double alpha = 0.0;
        for (int t = 0; t < ph.nterms_local; ++t) {
            const int id = ph.term_order[t];
            if (id == 1) {            // ideal: beta^-1 ln n, constant ln(nref) dropped
                mu += log1p((double)dn / nref) * ph.inv_beta;
            } else {                  // tf (2) / gradient (3): alpha(n) by FP64 Newton
                if (!have_alpha) {
                    bool ok = true;
                    alpha = fd::alpha_from_ip12(fdtab, n / ph.cn, &ok);
                    if (!ok) atomicOr(status, ST_NONPOS);
                    have_alpha = true;
                }
                if (id == 2) {
                    mu += (alpha - ph.alpha_ref) * ph.inv_beta;
                } else {
                    const int gi = 1 + nm;
                    const double xi = fd::xi(fdtab, alpha);
                    const double dxidn = fd::dxi(fdtab, alpha) / (0.5 * ph.cn * fd::im12(fdtab, alpha));
                    double g2 = 0.0;
                    for (int d = 0; d < nm; ++d) {
                        const double gd = (double)Fin[(gi + d) * stride];
                        g2 += gd * gd;
                    }
                    const double lapn = (double)Fin[(gi + nm) * stride];
                    mu -= ph.cg * (dxidn * g2 + 2.0 * xi * lapn);
                }
            }
        }
        Fout[o * stride] = R(mu);
        if (dn_real) dn_real[q] = dn;
        if (u_real)
            for (int d = 0; d < nm; ++d) u_real[d * ncell + q] = u[d];
    }
};

// --------------------------------------------------------- phase B functor
// inputs:  0..nm-1 d mu/dx_d, [Pi evolved: nm + 2((c/2) nm + d) + c%2  d Pi_c/dx_d]
// outputs: 0..nm-1 n (dmu/dx_i - F_ext,i), [6 x  -u.grad Pi_c]
template <typename R>
struct PWB {
    Phys ph;
    int nm;
    const cplx<R> *nhat;
    const double *nmean;       // the mean density in FP64
    const R *dn_real, *u_real;
    size_t ncell;
    const cplx<double> *ex, *ey, *ez;   // exp(i k_d x_d) per axis
    const R *gradv;                      // grad of the gaussian potential (3 fields)
    const Ctrl *ctrl;
    int stage;
    unsigned *status;

    __device__ void operator()(const Grid &g, int row, int x, const R *Fin, R *Fout, int stride) const
    {
        const size_t q = (size_t)row * g.nx + x;
        const double nref = *nmean;
        const R n = R(nref + (double)dn_real[q]);
        R f[3] = {R(0), R(0), R(0)};
        if (ph.ext_active && ph.ext_kind == 3) {
            for (int d = 0; d < nm; ++d) f[d] = -gradv[d * ncell + q];
        } else if (ph.ext_active) {
            const int y = row % g.ny, z = row / g.ny;
            const StageScal &s = ctrl->st[stage];
            cplx<double> e = ex[x] * ey[y];
            e = e * ez[z];
            e = e * cplx<double>{s.ewr, s.ewi};
            const double sf = s.amp * e.y;
            for (int d = 0; d < 3; ++d) f[d] = R(sf * ph.ext_k[d]);
        }
        for (int i = 0; i < nm; ++i) Fout[i * stride] = n * (Fin[i * stride] - f[i]);
        if (ph.evolve) {
            R u[3];
            for (int d = 0; d < nm; ++d) u[d] = u_real[d * ncell + q];
            // input order: for component pairs (c, c+1), c even, and d < nm,
            // the pair (d Pi_c/dx_d, d Pi_{c+1}/dx_d)
            for (int c = 0; c < 6; ++c) {
                R acc = R(0);
                for (int d = 0; d < nm; ++d) acc -= u[d] * Fin[(nm + 2 * ((c / 2) * nm + d) + (c % 2)) * stride];
                Fout[(nm + c) * stride] = acc;
            }
        }
    }
};

// ------------------------------------------------- u only (relaxation finish)
template <typename R>
struct PWU {
    Phys ph;
    int nm;
    const cplx<R> *nhat;
    const double *nmean;       // the mean density in FP64
    unsigned *status;
    __device__ void operator()(const Grid &g, int row, int x, const R *Fin, R *Fout, int stride) const
    {
        const double n = *nmean + (double)Fin[0];
        if (!(n > 0.0)) atomicOr(status, isfinite(n) ? ST_NONPOS : ST_NONFINITE);
        const R inv_mn = R(1.0 / (ph.mass * n));
        for (int d = 0; d < nm; ++d) Fout[d * stride] = Fin[(1 + d) * stride] * inv_mn;
    }
};

// ------------------------------------------- real-space read/write (I/O)
template <typename R>
struct PWToReal {
    R *dst[MAXF];
    size_t ncell;
    __device__ void operator()(const Grid &g, int row, int x, const R *Fin, R *, int stride) const
    {
        const size_t q = (size_t)row * g.nx + x;
        for (int f = 0; f < MAXF && dst[f]; ++f) dst[f][q] = Fin[f * stride];
    }
};

template <typename R>
struct PWFromReal {
    const R *src[MAXF];
    int nf;
    __device__ void operator()(const Grid &g, int row, int x, const R *, R *Fout, int stride) const
    {
        const size_t q = (size_t)row * g.nx + x;
        for (int f = 0; f < nf; ++f) Fout[f * stride] = src[f][q];
    }
};

// ---------------------------------------------------- spectral combines
// mode index -> (kx, ky, kz) compact indices.  The band holds fewer than
// 2^31 modes (the solver refuses larger grids), so the split uses 32-bit
// unsigned division: a 64-bit divide is a long software sequence per mode.
__host__ __device__ __forceinline__ void kvec(const Grid &g, size_t idx, int &kxc, int &kyc, int &kzc)
{
    const unsigned i = (unsigned)idx, px = (unsigned)g.pkx, ny = (unsigned)g.nkyc;
    const unsigned r = i / px;
    kxc = (int)(i - r * px);
    const unsigned z = r / ny;
    kyc = (int)(r - z * ny);
    kzc = (int)z;
}

template <typename R>
struct CombineA {
    const cplx<R> *N, *M[3];
    cplx<R> *P[6], *P0[6];          // Pi state and Pi0 of the stage start
    const cplx<R> *U[3], *F[6], *G;  // phase A outputs
    const R *Klin;                  // sum of the spectral (hartree, ry) mu kernels
    cplx<R> *MU, *Q[3];
};

// symmetric flux index of (i,j) in the packed i<=j order for nm components
__host__ __device__ __forceinline__ int sym_idx(int i, int j, int nm)
{
    if (i > j) { int t = i; i = j; j = t; }
    // rows: i=0 has nm entries, i=1 has nm-1, ...
    return i * nm - i * (i - 1) / 2 + (j - i);
}

// Pi component index of (i,j): xx,yy,zz,xy,xz,yz
__host__ __device__ __forceinline__ int pi_idx(int i, int j)
{
    if (i == j) return i;
    if (i > j) { int t = i; i = j; j = t; }
    return i == 0 ? (j == 1 ? 3 : 4) : 5;
}

// NM: the number of momentum components (1, 2, 3) as a compile-time
// constant, so that every small per-mode array below stays in registers
template <typename R, int NM>
__device__ __forceinline__ void combine_a_body(const BlockIx &bk, const Grid &g, const Phys &ph, const CombineA<R> &c,
                                               Ctrl *ctrl, int stage)
{
    constexpr int nm = NM;
    const size_t total = (size_t)g.nkzc * g.nkyc * g.pkx;
    const int pending = ctrl->pending;
    const double phi = ctrl->pend_phi;
    const double ee = ctrl->pend_e;
    const int nf = nm * (nm + 1) / 2;
    const bool need_u = ph.evolve || ph.newtonian;
    const cplx<R> zero = {R(0), R(0)};
    for (size_t idx = bk.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)bk.gx * blockDim.x) {
        int kxc, kyc, kzc;
        kvec(g, idx, kxc, kyc, kzc);
        if (kxc >= g.nkxc) continue;
        // every input of this element first (the stores below cannot move
        // ahead of loads the compiler does not know are unaliased)
        const cplx<R> nh = c.N[idx], gl = c.G[idx];
        const R kl = c.Klin[idx];
        cplx<R> F[6], U[3], Pv[6], P0v[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) F[f] = f < nf ? c.F[f][idx] : zero;
#pragma unroll
        for (int d = 0; d < 3; ++d) U[d] = (need_u && d < nm) ? c.U[d][idx] : zero;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            Pv[q] = ph.evolve ? c.P[q][idx] : zero;
            P0v[q] = (ph.evolve && pending) ? c.P0[q][idx] : zero;
        }
        const R k[3] = {R(kxc * g.kx0), R(signed_idx(kyc, g.My) * g.ky0), R(signed_idx(kzc, g.Mz) * g.kz0)};
        const bool k0 = kxc == 0 && kyc == 0 && kzc == 0;
        // chemical potential: local part + spectral kernels
        cplx<R> mu = gl + kl * nh;
        if (k0) mu = zero;
        // divergence of the momentum flux
        cplx<R> D[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            cplx<R> sm = zero;
            if (i < nm)
                for (int j = 0; j < nm; ++j) sm = sm + ik_times(k[j], F[sym_idx(i, j, nm)]);
            D[i] = sm;
        }
        cplx<R> fpi[3] = {zero, zero, zero};
        cplx<R> p0[6], pc[6];
        if (ph.evolve) {
            // Pi0 of the stage-start velocity, completes the previous stage's relaxation
            cplx<R> ku = zero;
            for (int d = 0; d < nm; ++d) ku = ku + ik_times(k[d], U[d]);   // i k.u
            const R eta = R(ph.eta), xi = R(ph.xi);
#pragma unroll
            for (int ii = 0; ii < 3; ++ii) {
                const cplx<R> du = ii < nm ? ik_times(k[ii], U[ii]) : zero;
                p0[ii] = eta * (R(2) * du - R(2.0 / 3.0) * ku) + xi * ku;
            }
            const int pi_i[3] = {0, 0, 1}, pi_j[3] = {1, 2, 2};
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int i = pi_i[q], j = pi_j[q];
                cplx<R> a1 = i < nm ? ik_times(k[j], U[i]) : zero;
                cplx<R> a2 = j < nm ? ik_times(k[i], U[j]) : zero;
                p0[3 + q] = eta * (a1 + a2);
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                cplx<R> pv = Pv[q];
                if (pending) {
                    const cplx<R> po = P0v[q];
                    pv = p0[q] - R(phi) * (p0[q] - po) + R(ee) * (pv - po);
                }
                pc[q] = pv;
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                cplx<R> sm = zero;
                if (i < nm)
                    for (int j = 0; j < nm; ++j) sm = sm + ik_times(k[j], pc[pi_idx(i, j)]);
                fpi[i] = sm;
            }
        } else if (ph.newtonian) {
            // div Pi0 = eta lap u + (eta/3 + xi) grad div u, spectrally
            cplx<R> kdu = zero;
            for (int d = 0; d < nm; ++d) kdu = kdu + k[d] * U[d];
            const R k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
            const R eta = R(ph.eta), b = R(ph.eta / 3.0 + ph.xi);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if (i < nm) fpi[i] = R(-1) * (eta * k2 * U[i] + (b * k[i]) * kdu);
        }
        // stores
        c.MU[idx] = mu;
        if (ph.evolve) {
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                if (pending) c.P[q][idx] = pc[q];
                c.P0[q][idx] = p0[q];
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < nm) c.Q[i][idx] = fpi[i] - D[i];
        if (k0 && ph.ext_active) {
            // n hat at the drive mode, read before this stage's update
            if (ph.drive_in_band) {
                cplx<R> v = c.N[ph.drive_idx];
                ctrl->nkd_re = (double)v.x;
                ctrl->nkd_im = ph.drive_conj ? -(double)v.y : (double)v.y;
            } else {
                ctrl->nkd_re = 0.0;
                ctrl->nkd_im = 0.0;
            }
        }
    }
}

template <typename R, int NM>
__global__ void combine_a_kernel(const __grid_constant__ Grid g, const __grid_constant__ Phys ph,
                                 const __grid_constant__ CombineA<R> c, Ctrl *ctrl, int stage)
{
    combine_a_body<R, NM>(hw_block(), g, ph, c, ctrl, stage);
}

template <typename R, int NM>
struct CombineAPack {
    static constexpr int MAXT = 256, MINB = 2;
    Grid g;
    Phys ph;
    CombineA<R> c;
    Ctrl *ctrl;
    int stage;
    __device__ __forceinline__ void run(const BlockIx &b) const { combine_a_body<R, NM>(b, g, ph, c, ctrl, stage); }
};

template <typename R>
struct CombineB {
    cplx<R> *N, *M[3], *P[6];        // state (updated in place)
    cplx<R> *RN, *RM[3], *RP[6];     // RK registers
    const cplx<R> *Q[3], *Gm[3], *V[6];
    cplx<R> *oN, *oM[3], *oP[6];     // rhs-only outputs (no update when set)
};

template <typename R, int NM>
__device__ __forceinline__ void combine_b_body(const BlockIx &bk, const Grid &g, const Phys &ph, const CombineB<R> &c,
                                               Ctrl *ctrl, int stage, int rhs_only)
{
    constexpr int nm = NM;
    const size_t total = (size_t)g.nkzc * g.nkyc * g.pkx;
    const StageScal s = ctrl->st[stage];
    const double dt = ctrl->dt;
    const R da = R(dt * s.a), db = R(dt * s.b);
    const cplx<R> zero = {R(0), R(0)};
    const bool regs = !rhs_only && stage != 0;   // the RK registers are read
    for (size_t idx = bk.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)bk.gx * blockDim.x) {
        int kxc, kyc, kzc;
        kvec(g, idx, kxc, kyc, kzc);
        if (kxc >= g.nkxc) continue;
        // every input of this element first
        cplx<R> M[3], Qv[3], Gv[3], RMv[3], Pv[6], Vv[6], RPv[6];
        cplx<R> Nv = zero, RNv = zero;
        if (!rhs_only) Nv = c.N[idx];
        if (regs) RNv = c.RN[idx];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const bool on = d < nm;
            M[d] = on ? c.M[d][idx] : zero;
            Qv[d] = on ? c.Q[d][idx] : zero;
            Gv[d] = on ? c.Gm[d][idx] : zero;
            RMv[d] = (on && regs) ? c.RM[d][idx] : zero;
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            Vv[q] = ph.evolve ? c.V[q][idx] : zero;
            Pv[q] = (ph.evolve && !rhs_only) ? c.P[q][idx] : zero;
            RPv[q] = (ph.evolve && regs) ? c.RP[q][idx] : zero;
        }
        const R k[3] = {R(kxc * g.kx0), R(signed_idx(kyc, g.My) * g.ky0), R(signed_idx(kzc, g.Mz) * g.kz0)};
        const bool k0 = kxc == 0 && kyc == 0 && kzc == 0;
        cplx<R> dn = zero;
        for (int d = 0; d < nm; ++d) dn = dn + ik_times(k[d], M[d]);
        dn = R(-ph.inv_mass) * dn;
        cplx<R> dm[3] = {zero, zero, zero};
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < nm) dm[i] = Qv[i] - Gv[i];
        if (k0) {
            // mean of the internal force removed; mean of n F_ext kept:
            // <n A sin(k.r - w t)> = A Im(exp(-i w t) conj(nhat(k)))
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (i >= nm) continue;
                double mf = 0.0;
                if (ph.ext_active && ph.ext_kind != 3) {
                    const double im = s.ewi * ctrl->nkd_re - s.ewr * ctrl->nkd_im;
                    mf = s.amp * ph.ext_k[i] * im;
                } else if (ph.ext_active) {
                    mf = ctrl->gf[i];
                }
                dm[i] = cplx<R>{R(mf), R(0)};
            }
        }
        if (rhs_only) {
            c.oN[idx] = dn;
#pragma unroll
            for (int i = 0; i < 3; ++i) c.oM[i][idx] = dm[i];
            if (ph.evolve)
#pragma unroll
                for (int q = 0; q < 6; ++q) c.oP[q][idx] = Vv[q];
            continue;
        }
        if (stage == 0) {
            c.N[idx] = Nv + da * dn;
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if (i < nm) c.M[i][idx] = M[i] + da * dm[i];
        } else {
            c.N[idx] = Nv + (da * dn + db * RNv);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if (i < nm) c.M[i][idx] = M[i] + (da * dm[i] + db * RMv[i]);
        }
        c.RN[idx] = dn;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < nm) c.RM[i][idx] = dm[i];
        if (ph.evolve) {
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const cplx<R> v = Vv[q];
                if (stage == 0) c.P[q][idx] = Pv[q] + da * v;
                else c.P[q][idx] = Pv[q] + (da * v + db * RPv[q]);
                c.RP[q][idx] = v;
            }
        }
    }
    if (!rhs_only && bk.x == 0 && threadIdx.x == 0 && ph.evolve) {
        ctrl->pending = 1;
        ctrl->pend_phi = s.phi;
        ctrl->pend_e = s.e;
    }
}

template <typename R, int NM>
__global__ void combine_b_kernel(const __grid_constant__ Grid g, const __grid_constant__ Phys ph,
                                 const __grid_constant__ CombineB<R> c, Ctrl *ctrl, int stage, int rhs_only)
{
    combine_b_body<R, NM>(hw_block(), g, ph, c, ctrl, stage, rhs_only);
}

template <typename R, int NM>
struct CombineBPack {
    static constexpr int MAXT = 256, MINB = 2;
    Grid g;
    Phys ph;
    CombineB<R> c;
    Ctrl *ctrl;
    int stage, rhs_only;
    __device__ __forceinline__ void run(const BlockIx &b) const
    {
        combine_b_body<R, NM>(b, g, ph, c, ctrl, stage, rhs_only);
    }
};

// Completes a pending relaxation from u of the current state (combine U).
template <typename R>
struct CombineU {
    cplx<R> *P[6];
    const cplx<R> *P0[6];
    const cplx<R> *U[3];
};

template <typename R, int NM>
__global__ void combine_u_kernel(Grid g, Phys ph, CombineU<R> c, Ctrl *ctrl)
{
    constexpr int nm = NM;
    const size_t total = (size_t)g.nkzc * g.nkyc * g.pkx;
    const double phi = ctrl->pend_phi, ee = ctrl->pend_e;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        int kxc, kyc, kzc;
        kvec(g, idx, kxc, kyc, kzc);
        if (kxc >= g.nkxc) continue;
        const R k[3] = {R(kxc * g.kx0), R(signed_idx(kyc, g.My) * g.ky0), R(signed_idx(kzc, g.Mz) * g.kz0)};
        cplx<R> ku = {R(0), R(0)};
        for (int d = 0; d < nm; ++d) ku = ku + ik_times(k[d], c.U[d][idx]);
        const R eta = R(ph.eta), xi = R(ph.xi);
        cplx<R> p0[6];
        for (int ii = 0; ii < 3; ++ii) {
            const cplx<R> du = ii < nm ? ik_times(k[ii], c.U[ii][idx]) : cplx<R>{R(0), R(0)};
            p0[ii] = eta * (R(2) * du - R(2.0 / 3.0) * ku) + xi * ku;
        }
        const int pi_i[3] = {0, 0, 1}, pi_j[3] = {1, 2, 2};
        for (int q = 0; q < 3; ++q) {
            const int i = pi_i[q], j = pi_j[q];
            cplx<R> a1 = i < nm ? ik_times(k[j], c.U[i][idx]) : cplx<R>{R(0), R(0)};
            cplx<R> a2 = j < nm ? ik_times(k[i], c.U[j][idx]) : cplx<R>{R(0), R(0)};
            p0[3 + q] = eta * (a1 + a2);
        }
        for (int q = 0; q < 6; ++q) {
            const cplx<R> po = c.P0[q][idx];
            c.P[q][idx] = p0[q] - R(phi) * (p0[q] - po) + R(ee) * (c.P[q][idx] - po);
        }
    }
}

// Per-step scalars: stage times, drive amplitude and phase, relaxation factors.
__device__ __forceinline__ void begin_step_body(const BlockIx &bk, Ctrl *ctrl, double tau, int ext_td, double amp0,
                                                double omega, double ramp)
{
    if (threadIdx.x != 0 || bk.x != 0) return;
    const double A[3] = {32.0 / 60.0, 25.0 / 60.0, 45.0 / 60.0};
    const double Bc[3] = {0.0, -17.0 / 60.0, -25.0 / 60.0};
    double ts = ctrl->t;
    const double dt = ctrl->dt;
    for (int s = 0; s < 3; ++s) {
        StageScal &st = ctrl->st[s];
        st.ts = ts;
        double a = amp0;
        if (ext_td && ramp > 0.0) a = a * fmin(1.0, ts / ramp);
        st.amp = a;
        double sn, cs;
        sincos(-omega * ts, &sn, &cs);
        st.ewr = cs;
        st.ewi = sn;
        st.a = A[s];
        st.b = Bc[s];
        const double dts = (A[s] + Bc[s]) * dt;
        if (tau > 0.0) {
            const double fac = exp(-dts / tau);
            st.e = fac;
            st.phi = (tau / dts) * (1.0 - fac);
        } else {
            st.e = 0.0;
            st.phi = 0.0;
        }
        ts = ts + dts;
    }
}

static __global__ void begin_step_kernel(Ctrl *ctrl, double tau, int ext_td, double amp0, double omega,
                                         double ramp)
{
    begin_step_body(hw_block(), ctrl, tau, ext_td, amp0, omega, ramp);
}

struct BeginStepPack {
    static constexpr int MAXT = 32, MINB = 1;
    Ctrl *ctrl;
    double tau;
    int ext_td;
    double amp0, omega, ramp;
    __device__ __forceinline__ void run(const BlockIx &b) const
    {
        begin_step_body(b, ctrl, tau, ext_td, amp0, omega, ramp);
    }
};

__device__ __forceinline__ void end_step_body(const BlockIx &bk, Ctrl *ctrl)
{
    if (threadIdx.x != 0 || bk.x != 0) return;
    ctrl->t = ctrl->t + ctrl->dt;
    ctrl->step = ctrl->step + 1;
    // the last right-hand side of the step was evaluated at stage 3's time
    ctrl->v_amp = ctrl->st[2].amp;
    ctrl->v_ewr = ctrl->st[2].ewr;
    ctrl->v_ewi = ctrl->st[2].ewi;
}

static __global__ void end_step_kernel(Ctrl *ctrl) { end_step_body(hw_block(), ctrl); }

struct EndStepPack {
    static constexpr int MAXT = 32, MINB = 1;
    Ctrl *ctrl;
    __device__ __forceinline__ void run(const BlockIx &b) const { end_step_body(b, ctrl); }
};

// one probe record: t, n and mom_x at compact index idx (conjugated when
// the mode is stored as its mirror), into ring slot *count
template <typename R>
__global__ void probe_kernel(const Ctrl *ctrl, const cplx<R> *N, const cplx<R> *M0, long long idx, int conj,
                             double *ring, int *count, int cap)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int slot = *count;
    if (slot >= cap) return;
    double nr = 0.0, ni = 0.0, mr = 0.0, mi = 0.0;
    if (idx >= 0) {
        nr = (double)N[idx].x;
        ni = (double)N[idx].y;
        mr = (double)M0[idx].x;
        mi = (double)M0[idx].y;
        if (conj) { ni = -ni; mi = -mi; }
    }
    double *r = ring + 5 * (size_t)slot;
    r[0] = ctrl->t;
    r[1] = nr; r[2] = ni; r[3] = mr; r[4] = mi;
    *count = slot + 1;
}

// the potential of a right-hand side evaluated at stage `stage`'s time
static __global__ void vlast_kernel(Ctrl *ctrl, int stage)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    ctrl->v_amp = ctrl->st[stage].amp;
    ctrl->v_ewr = ctrl->st[stage].ewr;
    ctrl->v_ewi = ctrl->st[stage].ewi;
}

}  // namespace hydft
