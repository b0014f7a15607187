// Persistent x passes fed by TMA bulk copies (cp.async.bulk, no multicast).
//
// Each block owns batches of RB rows of x; each row of an input field is a
// contiguous run of kx <= Mx complex values in the YI layout, copied into a
// ring of S shared-memory stages (one input pair of RB rows per stage) that
// complete on an mbarrier each.  Thread 0 keeps S-1 pairs in flight, across
// batch boundaries, so the loads of the next pairs overlap the transforms and
// physics of the current one.  The transforms and physics are the register
// FFT routines of regfft.cuh / passes_fast.cuh.  Every wait is bounded by
// %globaltimer (about 1 s); on expiry the block records ST_TIMEOUT, drains
// its own copies (again bounded) and returns.
#pragma once

#include "passes_fast.cuh"

namespace hydft {

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait for the phase with the given parity; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > 1000000000ull) return false;
    }
}

// global -> shared bulk copy completing on `bar` (sizes and both addresses
// multiples of 16 bytes)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Ring geometry shared by host and device.
struct RingGeom {
    int kp;          // complex slots per staged row (even; bank-shifted for T < 16)
    unsigned seg;    // bytes copied per row (even number of complex values)
    int stages;
};

__host__ __device__ inline int ring_kp(int nkxc, int T)
{
    const int even = (nkxc + 1) / 2 * 2;
    if (T >= 16) return even;
    return (nkxc + 15) / 16 * 16 + T;   // row r starts at bank group r*T
}

// The pair schedule of one batch: input field indices (fa, fb), fb < 0 if
// single.
struct PairList {
    int n;
    signed char fa[24], fb[24];
};

// Producer: issue the copies of global sequence index q (batch iteration
// q / np, pair q % np) into stage q % S.
template <typename R>
__device__ __forceinline__ void ring_issue(long q, int np, const PairList &pl, int rb, int nrows, int nbatch,
                                           long nmy, const XFastArgs<R> &a, const Grid &g, const RingGeom &rg,
                                           cplx<R> *ring, uint64_t *bars)
{
    const long it = q / np;
    if (it >= nmy) return;
    const int p = (int)(q % np);
    const int s = (int)(q % rg.stages);
    const int b = blockIdx.x + (int)(it * gridDim.x);
    (void)nbatch;
    cplx<R> *st = ring + (size_t)s * 2 * rb * rg.kp;
    const int rows = min(rb, nrows - b * rb);
    const int nf = pl.fb[p] >= 0 ? 2 : 1;
    fence_proxy_async();
    mbar_arrive_expect_tx(&bars[s], (unsigned)(rows * nf) * rg.seg);
    for (int h = 0; h < nf; ++h) {
        const cplx<R> *src = a.in[h == 0 ? pl.fa[p] : pl.fb[p]];
        for (int rr = 0; rr < rows; ++rr) {
            const size_t row = (size_t)b * rb + rr;
            bulk_load(st + ((size_t)h * rb + rr) * rg.kp, src + row * g.pkx, rg.seg, &bars[s]);
        }
    }
}

// c2r input of a staged pair (rows of kx <= Mx) -> block layout
template <typename R, int T, int E>
__device__ __forceinline__ void staged_c2r(cplx<R> (&v)[E], const cplx<R> *sa, const cplx<R> *sb, bool rowok,
                                           int t, int Mx, cplx<R> *xrow, const cplx<R> *tw)
{
    constexpr int L = T * E;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int k = t + T * e;
        cplx<R> Z = {R(0), R(0)};
        if (rowok) {
            if (k <= Mx) {
                cplx<R> va = sa[k];
                cplx<R> vb = sb ? sb[k] : cplx<R>{R(0), R(0)};
                if (k == 0) { va.y = R(0); vb.y = R(0); }
                Z = cplx<R>{va.x - vb.y, va.y + vb.x};
            } else if (k >= L - Mx) {
                const int kk = L - k;
                const cplx<R> va = sa[kk];
                const cplx<R> vb = sb ? sb[kk] : cplx<R>{R(0), R(0)};
                Z = cplx<R>{va.x + vb.y, -va.y + vb.x};
            }
        }
        v[e] = Z;
    }
    stride_to_block<T, E, +1, R, BarWarp, 1>(v, t, xrow, tw);
}

// smem layout of the persistent x passes
template <typename R, int T, int E>
__host__ __device__ inline size_t tma_smem(int rb, const RingGeom &rg, int nslots, bool scal)
{
    const size_t nt = (size_t)rb * T;
    size_t b = 0;
    b += sizeof(uint64_t) * 8;                                      // mbarriers (up to 8 stages)
    b += sizeof(cplx<R>) * (T * E);                                 // twiddles
    b += sizeof(cplx<R>) * (size_t)rb * xrow_stride<T, E>();       // exchange rows
    b += sizeof(cplx<R>) * (size_t)rg.stages * 2 * rb * rg.kp;     // ring
    b += sizeof(cplx<R>) * (size_t)nslots * E * nt;                // input slots
    if (scal) b += 2 * sizeof(R) * (size_t)E * nt;                 // mu and 1/(mn)
    return b;
}

// ------------------------------------------------------------- phase A
template <typename R, int T, int E, bool GRAD, bool UONLY>
__global__ void __launch_bounds__(128) xa_tma(Grid g, XFastArgs<R> a, const cplx<R> *twx, PWA<R> pw, int rb,
                                              RingGeom rg, PairList pl)
{
    constexpr int NM = 3;
    constexpr int NIN = 1 + NM + (GRAD ? NM + 1 : 0);
    constexpr int NP = (NIN + 1) / 2;
    constexpr int NF = NM * (NM + 1) / 2;
    constexpr int NOUT = UONLY ? NM : NM + NF + 1;
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw);
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw + sizeof(uint64_t) * 8);
    cplx<R> *xbuf = tw + L;
    cplx<R> *ring = xbuf + (size_t)rb * xrow_stride<T, E>();
    const int nt = blockDim.x;
    cplx<R> *slots = ring + (size_t)rg.stages * 2 * rb * rg.kp;
    R *muslot = reinterpret_cast<R *>(slots + (size_t)NP * E * nt);
    R *invslot = muslot + (size_t)E * nt;
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int nrows = g.ny * g.nz;
    const int nbatch = (nrows + rb - 1) / rb;
    const long nmy = blockIdx.x < nbatch ? (nbatch - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    for (int i = tid; i < L; i += nt) tw[i] = twx[i];
    if (tid == 0) {
        for (int s = 0; s < rg.stages; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    const long nq = nmy * NP;
    if (tid == 0)
        for (long q = 0; q < rg.stages - 1 && q < nq; ++q)
            ring_issue<R>(q, NP, pl, rb, nrows, nbatch, nmy, a, g, rg, ring, bars);
    const R nref = pw.nhat[0].x;
    const R inv_nref = R(1) / nref, inv_beta = R(pw.ph.inv_beta), mass = R(pw.ph.mass);
    long qfail = -1, qissued = nq < rg.stages - 1 ? nq : rg.stages - 1;
    for (long q = 0; q < nq; ++q) {
        const int s = (int)(q % rg.stages);
        const bool ok = mbar_wait(&bars[s], (unsigned)((q / rg.stages) & 1));
        // uniform over the block; also every thread has finished pair q-1,
        // so its stage can be refilled
        if (__syncthreads_or(!ok)) { qfail = q; break; }
        if (q + rg.stages - 1 < nq) {
            if (tid == 0) ring_issue<R>(q + rg.stages - 1, NP, pl, rb, nrows, nbatch, nmy, a, g, rg, ring, bars);
            qissued = q + rg.stages;
        }
        const int p = (int)(q % NP);
        const int b = blockIdx.x + (int)((q / NP) * gridDim.x);
        const int row = b * rb + rr;
        const bool rowok = row < nrows;
        const cplx<R> *st = ring + (size_t)s * 2 * rb * rg.kp;
        cplx<R> v[E];
        staged_c2r<R, T, E>(v, st + (size_t)rr * rg.kp, pl.fb[p] >= 0 ? st + ((size_t)rb + rr) * rg.kp : nullptr,
                            rowok, t, g.Mx, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) slots[(p * E + r) * nt + tid] = v[r];
        if (p != NP - 1) continue;
        // -------- all inputs of this batch are in the slots
        auto input = [&](int f, int r) -> R {
            const cplx<R> sv = slots[((f / 2) * E + r) * nt + tid];
            return (f & 1) ? sv.y : sv.x;
        };
        const size_t rowbase = (size_t)row * g.nx;
#pragma unroll 1
        for (int r = 0; r < E; ++r) {
            const int xx = block_pos<T, E>(t, r);
            const R dn = input(0, r);
            const R n = nref + dn;
            const R inv_mn = R(1) / (mass * n);
            invslot[r * nt + tid] = inv_mn;
            if (rowok) {
                if (!(n > R(0))) atomicOr(pw.status, isfinite(n) ? ST_NONPOS : ST_NONFINITE);
                if (pw.dn_real) pw.dn_real[rowbase + xx] = dn;
                if (pw.u_real)
                    for (int d = 0; d < NM; ++d) pw.u_real[d * pw.ncell + rowbase + xx] = input(1 + d, r) * inv_mn;
            }
            if (!UONLY) {
                R mu = R(0);
                double mu64 = 0.0, alpha = 0.0;
                bool have_alpha = false, any64 = false;
                for (int tt = 0; tt < pw.ph.nterms_local; ++tt) {
                    const int id = pw.ph.term_order[tt];
                    if (id == 1) {
                        mu += log1p(dn * inv_nref) * inv_beta;
                    } else {
                        const double n64 = (double)nref + (double)dn;
                        any64 = true;
                        if (!have_alpha) {
                            bool ok = true;
                            alpha = fd::alpha_from_ip12(pw.fdtab, n64 / pw.ph.cn, &ok);
                            if (!ok && rowok) atomicOr(pw.status, ST_NONPOS);
                            have_alpha = true;
                        }
                        if (id == 2) {
                            mu64 += (alpha - pw.ph.alpha_ref) * pw.ph.inv_beta;
                        } else if (GRAD) {
                            const double xi = fd::xi(pw.fdtab, alpha);
                            const double dxidn = fd::dxi(pw.fdtab, alpha) / (0.5 * pw.ph.cn * fd::im12(pw.fdtab, alpha));
                            double g2 = 0.0;
                            for (int d = 0; d < NM; ++d) {
                                const double gd = (double)input(1 + NM + d, r);
                                g2 += gd * gd;
                            }
                            const double lapn = (double)input(1 + 2 * NM, r);
                            mu64 -= pw.ph.cg * (dxidn * g2 + 2.0 * xi * lapn);
                        }
                    }
                }
                muslot[r * nt + tid] = any64 ? R((double)mu + mu64) : mu;
            }
        }
#pragma unroll
        for (int qo = 0; 2 * qo < NOUT; ++qo) {
            cplx<R> w[E];
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const R inv_mn = invslot[r * nt + tid];
                R val[2] = {R(0), R(0)};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int o = 2 * qo + h;
                    if (o < NM) val[h] = input(1 + o, r) * inv_mn;
                    else if (o < NM + NF) val[h] = input(1 + flux_i3(o - NM), r) * (input(1 + flux_j3(o - NM), r) * inv_mn);
                    else if (o < NOUT) val[h] = muslot[r * nt + tid];
                }
                w[r] = cplx<R>{val[0], val[1]};
            }
            x_r2c_pair<R, T, E>(w, a.out[2 * qo], 2 * qo + 1 < NOUT ? a.out[2 * qo + 1] : nullptr, row, rowok, t, g,
                                xrow, tw);
        }
    }
    if (qfail >= 0 && tid == 0) {
        atomicOr(pw.status, ST_TIMEOUT);
        // copies issued but not consumed must land before the block exits
        for (long q = qfail; q < qissued; ++q) mbar_wait(&bars[q % rg.stages], (unsigned)((q / rg.stages) & 1));
    }
}

// ------------------------------------------------------------- phase B
template <typename R, int T, int E, bool EVOLVE>
__global__ void __launch_bounds__(128) xb_tma(Grid g, XFastArgs<R> a, const cplx<R> *twx, PWB<R> pw, int rb,
                                              RingGeom rg, PairList pl)
{
    constexpr int NM = 3;
    constexpr int L = T * E;
    constexpr int NGP = (NM + 1) / 2;                  // pairs of n(dmu - F)
    constexpr int NP = NGP + (EVOLVE ? 3 * NM : 0);    // input pairs per batch
    extern __shared__ __align__(16) unsigned char smraw[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smraw);
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw + sizeof(uint64_t) * 8);
    cplx<R> *xbuf = tw + L;
    cplx<R> *ring = xbuf + (size_t)rb * xrow_stride<T, E>();
    const int nt = blockDim.x;
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int nrows = g.ny * g.nz;
    const int nbatch = (nrows + rb - 1) / rb;
    const long nmy = blockIdx.x < nbatch ? (nbatch - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    for (int i = tid; i < L; i += nt) tw[i] = twx[i];
    if (tid == 0) {
        for (int s = 0; s < rg.stages; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();
    const long nq = nmy * NP;
    if (tid == 0)
        for (long q = 0; q < rg.stages - 1 && q < nq; ++q)
            ring_issue<R>(q, NP, pl, rb, nrows, nbatch, nmy, a, g, rg, ring, bars);
    const R nref = pw.nhat[0].x;
    long qfail = -1, qissued = nq < rg.stages - 1 ? nq : rg.stages - 1;
    cplx<R> acc[E];
    for (long q = 0; q < nq; ++q) {
        const int s = (int)(q % rg.stages);
        const bool ok = mbar_wait(&bars[s], (unsigned)((q / rg.stages) & 1));
        if (__syncthreads_or(!ok)) { qfail = q; break; }
        if (q + rg.stages - 1 < nq) {
            if (tid == 0) ring_issue<R>(q + rg.stages - 1, NP, pl, rb, nrows, nbatch, nmy, a, g, rg, ring, bars);
            qissued = q + rg.stages;
        }
        const int p = (int)(q % NP);
        const int b = blockIdx.x + (int)((q / NP) * gridDim.x);
        const int row = b * rb + rr;
        const bool rowok = row < nrows;
        const size_t rowbase = (size_t)row * g.nx;
        const cplx<R> *st = ring + (size_t)s * 2 * rb * rg.kp;
        cplx<R> v[E];
        staged_c2r<R, T, E>(v, st + (size_t)rr * rg.kp, pl.fb[p] >= 0 ? st + ((size_t)rb + rr) * rg.kp : nullptr,
                            rowok, t, g.Mx, xrow, tw);
        if (p < NGP) {
            // n (dmu/dx_i - F_i) for the component pair (2p, 2p+1)
            const int i0 = 2 * p, i1 = 2 * p + 1;
            const int y = rowok ? row % g.ny : 0, z = rowok ? row / g.ny : 0;
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int xx = block_pos<T, E>(t, r);
                const R n = rowok ? nref + pw.dn_real[rowbase + xx] : R(0);
                R f0 = R(0), f1 = R(0);
                if (pw.ph.ext_active) {
                    const StageScal &ss = pw.ctrl->st[pw.stage];
                    cplx<double> e = pw.ex[xx] * pw.ey[y];
                    e = e * pw.ez[z];
                    e = e * cplx<double>{ss.ewr, ss.ewi};
                    const double sf = ss.amp * e.y;
                    f0 = R(sf * pw.ph.ext_k[i0]);
                    if (i1 < NM) f1 = R(sf * pw.ph.ext_k[i1]);
                }
                v[r] = cplx<R>{n * (v[r].x - f0), n * (v[r].y - f1)};
            }
            x_r2c_pair<R, T, E>(v, a.out[i0], i1 < NM ? a.out[i1] : nullptr, row, rowok, t, g, xrow, tw);
        } else {
            // -u.grad Pi for the component pair (2cp, 2cp+1), derivative d
            const int k = p - NGP, cp = k / NM, d = k % NM;
            if (d == 0) {
#pragma unroll
                for (int r = 0; r < E; ++r) acc[r] = cplx<R>{R(0), R(0)};
            }
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int xx = block_pos<T, E>(t, r);
                const R u = rowok ? pw.u_real[d * pw.ncell + rowbase + xx] : R(0);
                acc[r] = acc[r] - u * v[r];
            }
            if (d == NM - 1)
                x_r2c_pair<R, T, E>(acc, a.out[NM + 2 * cp], a.out[NM + 2 * cp + 1], row, rowok, t, g, xrow, tw);
        }
    }
    if (qfail >= 0 && tid == 0) {
        atomicOr(pw.status, ST_TIMEOUT);
        for (long q = qfail; q < qissued; ++q) mbar_wait(&bars[q % rg.stages], (unsigned)((q / rg.stages) & 1));
    }
}

}  // namespace hydft
