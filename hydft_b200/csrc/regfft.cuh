// Register-resident FFTs: a column of length L = T*E is transformed by T
// cooperating threads holding E values each, with one shared-memory
// exchange (the four-step algorithm):
//
//   x[n], n = t + T e              (thread t holds e = 0..E-1, "stride" layout)
//   X[k], k = k2 + E k1            (thread t holds k2 = t + T j, j < E/T, and
//                                   k1 = 0..T-1, "block" layout)
//   X[k2 + E k1] = sum_t W_T^{t k1} W_L^{t k2} sum_e x[t + T e] W_E^{e k2}
//
// stride_to_block: E-point DFT in registers, twiddle W_L^{t k2}, exchange,
// T-point DFTs.  block_to_stride is its transpose (T-point DFTs, twiddle,
// exchange, E-point DFT) and takes input in block layout and returns
// X[t + T m] in stride layout.  The small DFTs are unrolled at compile
// time: radices 2, 3, 4, 8 and products of them (6, 12, 16, 24, 32) by the
// same four-step rule inside the registers.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace hydft {

// W_N^j = exp(-2 pi i j/N) for the composite register DFTs, in constant
// memory (indices are compile-time constants after unrolling).
struct RegTw {
    double w6[6][2], w12[12][2], w16[16][2], w24[24][2], w32[32][2];
};
static __constant__ RegTw c_regtw;

template <int N>
__device__ __forceinline__ const double *regtw_table()
{
    if (N == 6) return &c_regtw.w6[0][0];
    if (N == 12) return &c_regtw.w12[0][0];
    if (N == 16) return &c_regtw.w16[0][0];
    if (N == 24) return &c_regtw.w24[0][0];
    return &c_regtw.w32[0][0];
}

template <int N, int DIR, typename R>
struct RegDFT;

template <int DIR, typename R>
struct RegDFT<1, DIR, R> {
    static __device__ __forceinline__ void run(cplx<R> *) {}
};
template <int DIR, typename R>
struct RegDFT<2, DIR, R> {
    static __device__ __forceinline__ void run(cplx<R> *v) { dft2<DIR>(v); }
};
template <int DIR, typename R>
struct RegDFT<3, DIR, R> {
    static __device__ __forceinline__ void run(cplx<R> *v) { dft3<DIR>(v); }
};
template <int DIR, typename R>
struct RegDFT<4, DIR, R> {
    static __device__ __forceinline__ void run(cplx<R> *v) { dft4<DIR>(v); }
};
template <int DIR, typename R>
struct RegDFT<8, DIR, R> {
    static __device__ __forceinline__ void run(cplx<R> *v) { dft8<DIR>(v); }
};

// N = A*B in registers: n = a + A b, k = kb + B ka
template <int A, int B, int DIR, typename R>
struct RegDFTComp {
    static __device__ __forceinline__ void run(cplx<R> *v)
    {
        constexpr int N = A * B;
        const double *w = regtw_table<N>();
        cplx<R> u[A][B];
#pragma unroll
        for (int a = 0; a < A; ++a) {
#pragma unroll
            for (int b = 0; b < B; ++b) u[a][b] = v[a + A * b];
            RegDFT<B, DIR, R>::run(u[a]);
#pragma unroll
            for (int kb = 1; kb < B; ++kb) {
                if (a == 0) continue;
                const int j = (a * kb) % N;
                const cplx<R> tw = {R(w[2 * j]), R(-DIR) * R(w[2 * j + 1])};
                u[a][kb] = u[a][kb] * tw;
            }
        }
#pragma unroll
        for (int kb = 0; kb < B; ++kb) {
            cplx<R> c[A];
#pragma unroll
            for (int a = 0; a < A; ++a) c[a] = u[a][kb];
            RegDFT<A, DIR, R>::run(c);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) v[kb + B * ka] = c[ka];
        }
    }
};

template <int DIR, typename R>
struct RegDFT<6, DIR, R> : RegDFTComp<2, 3, DIR, R> {};
template <int DIR, typename R>
struct RegDFT<12, DIR, R> : RegDFTComp<4, 3, DIR, R> {};
template <int DIR, typename R>
struct RegDFT<16, DIR, R> : RegDFTComp<4, 4, DIR, R> {};
template <int DIR, typename R>
struct RegDFT<24, DIR, R> : RegDFTComp<8, 3, DIR, R> {};
template <int DIR, typename R>
struct RegDFT<32, DIR, R> : RegDFTComp<4, 8, DIR, R> {};

// Shared-memory exchange buffer of one column: element e at
// sm[(e + e/T) * ES] (one pad slot every T elements, so that the strided
// reads of the exchange hit distinct banks).  The index expressions below
// are that formula with t < T and E % T == 0 folded in, so every access is
// a per-thread base plus a compile-time offset.
template <int T>
__device__ __forceinline__ int xidx(int e) { return e + e / T; }

// Barrier policies of the exchange: the whole block (a column's threads
// span warps) or one warp (a column's threads are lanes of one warp).
struct BarBlock {
    static __device__ __forceinline__ void sync() { __syncthreads(); }
};
struct BarWarp {
    static __device__ __forceinline__ void sync() { __syncwarp(); }
};

// x in stride layout (v[e] = x[t + T e]) -> X in block layout
// (v[j*T + k1] = X[(t + T j) + E k1]).  `sm` is this column's exchange
// buffer (element stride ES).  `tw` is the planned twiddle table of 2L
// entries: W_L^{t k2} at [k2 T + t] (k2 < E, t < T) for this routine, then
// W_L^{k2 m1} at [L + m1 E + k2] (m1 < T, k2 < E) for block_to_stride, laid
// out so that the T threads of a column read consecutive entries.
template <int T, int E, int DIR, typename R, class BAR = BarBlock, int ES = 1>
__device__ __forceinline__ void stride_to_block(cplx<R> (&v)[E], int t, cplx<R> *sm,
                                                const cplx<R> *__restrict__ tw)
{
    RegDFT<E, DIR, R>::run(v);
#pragma unroll
    for (int k2 = 1; k2 < E; ++k2) {
        cplx<R> w = tw[k2 * T + t];   // W_L^{t k2}
        if (DIR > 0) w.y = -w.y;
        v[k2] = v[k2] * w;
    }
    cplx<R> *wp = sm + t * ES;
#pragma unroll
    for (int k2 = 0; k2 < E; ++k2) wp[k2 * (T + 1) * ES] = v[k2];   // element k2*T + t
    BAR::sync();
#pragma unroll
    for (int j = 0; j < E / T; ++j) {
        const cplx<R> *rp = sm + (t + T * j) * (T + 1) * ES;         // element (t + T j)*T + n1
        cplx<R> u[T];
#pragma unroll
        for (int n1 = 0; n1 < T; ++n1) u[n1] = rp[n1 * ES];
        RegDFT<T, DIR, R>::run(u);
#pragma unroll
        for (int k1 = 0; k1 < T; ++k1) v[j * T + k1] = u[k1];
    }
    BAR::sync();
}

// z in block layout (v[j*T + k1] = z[(t + T j) + E k1]) -> X in stride
// layout (v[m] = X[t + T m]).
template <int T, int E, int DIR, typename R, class BAR = BarBlock, int ES = 1>
__device__ __forceinline__ void block_to_stride(cplx<R> (&v)[E], int t, cplx<R> *sm,
                                                const cplx<R> *__restrict__ tw)
{
    constexpr int EP = E + E / T;   // padded length of E elements
#pragma unroll
    for (int j = 0; j < E / T; ++j) {
        const int k2 = t + T * j;
        cplx<R> u[T];
#pragma unroll
        for (int k1 = 0; k1 < T; ++k1) u[k1] = v[j * T + k1];
        RegDFT<T, DIR, R>::run(u);
        cplx<R> *wp = sm + (t + j * (T + 1)) * ES;                   // element m1*E + k2
#pragma unroll
        for (int m1 = 0; m1 < T; ++m1) {
            cplx<R> w = tw[T * E + m1 * E + k2];   // W_L^{k2 m1}
            if (DIR > 0) w.y = -w.y;
            wp[m1 * EP * ES] = m1 == 0 ? u[0] : u[m1] * w;
        }
    }
    BAR::sync();
    const cplx<R> *rp = sm + t * EP * ES;                             // element t*E + k2
#pragma unroll
    for (int k2 = 0; k2 < E; ++k2) v[k2] = rp[(k2 + k2 / T) * ES];
    RegDFT<E, DIR, R>::run(v);
    BAR::sync();
}

// position (index along the axis) of register r in block layout
template <int T, int E>
__device__ __forceinline__ int block_pos(int t, int r)
{
    return (t + T * (r / T)) + E * (r % T);
}

// the register plan of an axis length (T threads x E values); 0 if none
__host__ __device__ inline int reg_plan_T(int L)
{
    switch (L) {
    case 32: return 4;
    case 48: return 4;
    case 64: return 8;
    case 96: return 4;
    case 128: return 8;
    case 192: return 8;
    case 256: return 16;
    default: return 0;
    }
}

}  // namespace hydft
