// Batched 1-D complex FFTs in shared memory (Stockham autosort, radices
// 2, 3, 4, 8), used by every transform pass of the solver.
//
// A CTA transforms `ncols` independent columns of length L held in shared
// memory at addr(e, c) = e*es + c*cs.  Each radix-R pass reads R elements
// j + r*L/R of a column, applies the twiddles exp(-+2 pi i k r / (Ns R)),
// does an R-point DFT and writes the results at (j/Ns)*Ns*R + k + q*Ns
// (k = j mod Ns, Ns = product of the radices already applied); passes
// ping-pong between two buffers, so the output is in natural order with no
// digit-reversal step.  `colfast` chooses which index consecutive threads
// walk: columns (the Y/Z passes, whose columns are contiguous kx runs) or
// butterflies (the X pass, whose columns are rows of x).
#pragma once

#include "common.cuh"

namespace hydft {

template <int DIR, typename R>
__device__ __forceinline__ void dft2(cplx<R> *v)
{
    cplx<R> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
}

template <int DIR, typename R>
__device__ __forceinline__ void dft3(cplx<R> *v)
{
    const R s = R(0.86602540378443864676372317075293618);   // sqrt(3)/2
    cplx<R> t1 = v[1] + v[2];
    cplx<R> m = v[0] - R(0.5) * t1;
    cplx<R> d = s * (v[1] - v[2]);
    cplx<R> jd = mul_i<DIR>(d);
    v[0] = v[0] + t1;
    v[1] = m + jd;
    v[2] = m - jd;
}

template <int DIR, typename R>
__device__ __forceinline__ void dft4v(cplx<R> &x0, cplx<R> &x1, cplx<R> &x2, cplx<R> &x3)
{
    cplx<R> a0 = x0 + x2, a1 = x0 - x2, b0 = x1 + x3, b1 = mul_i<DIR>(x1 - x3);
    x0 = a0 + b0;
    x2 = a0 - b0;
    x1 = a1 + b1;
    x3 = a1 - b1;
}

template <int DIR, typename R>
__device__ __forceinline__ void dft4(cplx<R> *v) { dft4v<DIR>(v[0], v[1], v[2], v[3]); }

template <int DIR, typename R>
__device__ __forceinline__ void dft8(cplx<R> *v)
{
    const R h = R(0.70710678118654752440084436210484904);   // sqrt(1/2)
    cplx<R> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cplx<R> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4v<DIR>(e0, e1, e2, e3);
    dft4v<DIR>(o0, o1, o2, o3);
    // o_q *= W8^q, W8 = exp(DIR * 2 pi i / 8)
    cplx<R> w1 = {h, R(DIR) * h};
    cplx<R> w3 = {-h, R(DIR) * h};
    o1 = o1 * w1;
    o2 = mul_i<DIR>(o2);
    o3 = o3 * w3;
    v[0] = e0 + o0; v[4] = e0 - o0;
    v[1] = e1 + o1; v[5] = e1 - o1;
    v[2] = e2 + o2; v[6] = e2 - o2;
    v[3] = e3 + o3; v[7] = e3 - o3;
}

// One Stockham pass.
template <int DIR, typename R, int RAD>
__device__ __forceinline__ void stockham_pass(const cplx<R> *__restrict__ in, cplx<R> *__restrict__ out,
                                              int L, int Ns, int ncols, int es, int cs, bool colfast,
                                              const cplx<R> *__restrict__ tw)
{
    const int m = L / RAD;
    const int tw_step = L / (Ns * RAD);
    const int items = m * ncols;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        int c, j;
        if (colfast) { c = it % ncols; j = it / ncols; }
        else { j = it % m; c = it / m; }
        const int k = j % Ns;
        cplx<R> v[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r) {
            cplx<R> x = in[(j + r * m) * es + c * cs];
            if (r > 0) {
                cplx<R> w = tw[k * r * tw_step];
                if (DIR > 0) w.y = -w.y;
                x = x * w;
            }
            v[r] = x;
        }
        if (RAD == 2) dft2<DIR>(v);
        else if (RAD == 3) dft3<DIR>(v);
        else if (RAD == 4) dft4<DIR>(v);
        else dft8<DIR>(v);
        const int base = (j / Ns) * Ns * RAD + k;
#pragma unroll
        for (int q = 0; q < RAD; ++q) out[(base + q * Ns) * es + c * cs] = v[q];
    }
}

// Runs all passes of plan p.  Data starts in `a`; the result pointer (a or b)
// is returned.  Ends with a __syncthreads().
template <int DIR, typename R>
__device__ cplx<R> *fft_smem(cplx<R> *a, cplx<R> *b, const FFTPlan &p, int ncols, int es, int cs,
                             bool colfast, const cplx<R> *tw)
{
    int Ns = 1;
    for (int s = 0; s < p.nrad; ++s) {
        const int rad = p.rad[s];
        switch (rad) {
        case 2: stockham_pass<DIR, R, 2>(a, b, p.L, Ns, ncols, es, cs, colfast, tw); break;
        case 3: stockham_pass<DIR, R, 3>(a, b, p.L, Ns, ncols, es, cs, colfast, tw); break;
        case 4: stockham_pass<DIR, R, 4>(a, b, p.L, Ns, ncols, es, cs, colfast, tw); break;
        default: stockham_pass<DIR, R, 8>(a, b, p.L, Ns, ncols, es, cs, colfast, tw); break;
        }
        __syncthreads();
        cplx<R> *t = a; a = b; b = t;
        Ns *= rad;
    }
    return a;
}

}  // namespace hydft
