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

#include <type_traits>

#include "common.cuh"
#include "fft.cuh"

namespace hydft {

// W_N^j = exp(-2 pi i j/N) = {cos, -sin}(2 pi j/N) for the composite
// register DFTs, as compile-time constants: after unrolling every factor is
// an immediate operand, and the quarter turns become sign changes and swaps.
// f(integral_constant<int, i>) for i = 0 .. N-1, unrolled at compile time
template <int I, int N, class F>
__device__ __forceinline__ void unroll_for_impl(F &&f)
{
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        unroll_for_impl<I + 1, N>(f);
    }
}
template <int N, class F>
__device__ __forceinline__ void unroll_for(F &&f) { unroll_for_impl<0, N>(f); }

template <int N>
struct RegTwC;
template <>
struct RegTwC<6> {
    static constexpr double w[6][2] = {{1.0, -0.0},
                                      {0.5000000000000001, -0.8660254037844386},
                                      {-0.4999999999999998, -0.8660254037844387},
                                      {-1.0, -1.2246467991473532e-16},
                                      {-0.5000000000000004, 0.8660254037844384},
                                      {0.5000000000000001, 0.8660254037844386}};
};
template <>
struct RegTwC<12> {
    static constexpr double w[12][2] = {{1.0, -0.0},
                                      {0.8660254037844387, -0.49999999999999994},
                                      {0.5000000000000001, -0.8660254037844386},
                                      {6.123233995736766e-17, -1.0},
                                      {-0.4999999999999998, -0.8660254037844387},
                                      {-0.8660254037844387, -0.49999999999999994},
                                      {-1.0, -1.2246467991473532e-16},
                                      {-0.8660254037844388, 0.4999999999999997},
                                      {-0.5000000000000004, 0.8660254037844384},
                                      {-1.8369701987210297e-16, 1.0},
                                      {0.5000000000000001, 0.8660254037844386},
                                      {0.8660254037844384, 0.5000000000000004}};
};
template <>
struct RegTwC<16> {
    static constexpr double w[16][2] = {{1.0, -0.0},
                                      {0.9238795325112867, -0.3826834323650898},
                                      {0.7071067811865476, -0.7071067811865475},
                                      {0.38268343236508984, -0.9238795325112867},
                                      {6.123233995736766e-17, -1.0},
                                      {-0.3826834323650897, -0.9238795325112867},
                                      {-0.7071067811865475, -0.7071067811865476},
                                      {-0.9238795325112867, -0.3826834323650899},
                                      {-1.0, -1.2246467991473532e-16},
                                      {-0.9238795325112868, 0.38268343236508967},
                                      {-0.7071067811865477, 0.7071067811865475},
                                      {-0.38268343236509034, 0.9238795325112865},
                                      {-1.8369701987210297e-16, 1.0},
                                      {0.38268343236509, 0.9238795325112866},
                                      {0.7071067811865474, 0.7071067811865477},
                                      {0.9238795325112865, 0.3826834323650904}};
};
template <>
struct RegTwC<24> {
    static constexpr double w[24][2] = {{1.0, -0.0},
                                      {0.9659258262890683, -0.25881904510252074},
                                      {0.8660254037844387, -0.49999999999999994},
                                      {0.7071067811865476, -0.7071067811865475},
                                      {0.5000000000000001, -0.8660254037844386},
                                      {0.25881904510252074, -0.9659258262890683},
                                      {6.123233995736766e-17, -1.0},
                                      {-0.25881904510252063, -0.9659258262890683},
                                      {-0.4999999999999998, -0.8660254037844387},
                                      {-0.7071067811865475, -0.7071067811865476},
                                      {-0.8660254037844387, -0.49999999999999994},
                                      {-0.9659258262890682, -0.258819045102521},
                                      {-1.0, -1.2246467991473532e-16},
                                      {-0.9659258262890683, 0.2588190451025208},
                                      {-0.8660254037844388, 0.4999999999999997},
                                      {-0.7071067811865479, 0.7071067811865471},
                                      {-0.5000000000000004, 0.8660254037844384},
                                      {-0.25881904510252063, 0.9659258262890683},
                                      {-1.8369701987210297e-16, 1.0},
                                      {0.2588190451025203, 0.9659258262890684},
                                      {0.5000000000000001, 0.8660254037844386},
                                      {0.7071067811865474, 0.7071067811865477},
                                      {0.8660254037844384, 0.5000000000000004},
                                      {0.9659258262890681, 0.25881904510252157}};
};
template <>
struct RegTwC<32> {
    static constexpr double w[32][2] = {{1.0, -0.0},
                                      {0.9807852804032304, -0.19509032201612825},
                                      {0.9238795325112867, -0.3826834323650898},
                                      {0.8314696123025452, -0.5555702330196022},
                                      {0.7071067811865476, -0.7071067811865475},
                                      {0.5555702330196023, -0.8314696123025452},
                                      {0.38268343236508984, -0.9238795325112867},
                                      {0.19509032201612833, -0.9807852804032304},
                                      {6.123233995736766e-17, -1.0},
                                      {-0.1950903220161282, -0.9807852804032304},
                                      {-0.3826834323650897, -0.9238795325112867},
                                      {-0.555570233019602, -0.8314696123025455},
                                      {-0.7071067811865475, -0.7071067811865476},
                                      {-0.8314696123025453, -0.5555702330196022},
                                      {-0.9238795325112867, -0.3826834323650899},
                                      {-0.9807852804032304, -0.1950903220161286},
                                      {-1.0, -1.2246467991473532e-16},
                                      {-0.9807852804032304, 0.19509032201612836},
                                      {-0.9238795325112868, 0.38268343236508967},
                                      {-0.8314696123025455, 0.555570233019602},
                                      {-0.7071067811865477, 0.7071067811865475},
                                      {-0.5555702330196022, 0.8314696123025452},
                                      {-0.38268343236509034, 0.9238795325112865},
                                      {-0.19509032201612866, 0.9807852804032303},
                                      {-1.8369701987210297e-16, 1.0},
                                      {0.1950903220161283, 0.9807852804032304},
                                      {0.38268343236509, 0.9238795325112866},
                                      {0.5555702330196018, 0.8314696123025455},
                                      {0.7071067811865474, 0.7071067811865477},
                                      {0.8314696123025452, 0.5555702330196022},
                                      {0.9238795325112865, 0.3826834323650904},
                                      {0.9807852804032303, 0.19509032201612872}};
};

// x * exp(DIR i 2 pi j / N), j a compile-time constant
template <int N, int J, int DIR, typename R>
__device__ __forceinline__ cplx<R> twiddle_mul(cplx<R> x)
{
    constexpr int j = J % N;
    if constexpr (j == 0) {
        return x;
    } else if constexpr (4 * j == N) {
        return mul_i<DIR>(x);
    } else if constexpr (2 * j == N) {
        return cplx<R>{-x.x, -x.y};
    } else if constexpr (4 * j == 3 * N) {
        return mul_i<-DIR>(x);
    } else {
        constexpr double c = RegTwC<N>::w[j][0], sn = -RegTwC<N>::w[j][1];   // cos, sin
        const R cr = R(c), si = R(DIR * sn);
        return cplx<R>{x.x * cr - x.y * si, x.x * si + x.y * cr};
    }
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
        cplx<R> u[A][B];
        unroll_for<A>([&](auto ac) {
            constexpr int a = decltype(ac)::value;
#pragma unroll
            for (int b = 0; b < B; ++b) u[a][b] = v[a + A * b];
            RegDFT<B, DIR, R>::run(u[a]);
            unroll_for<B>([&](auto kc) {
                constexpr int kb = decltype(kc)::value;
                u[a][kb] = twiddle_mul<N, a * kb, DIR>(u[a][kb]);
            });
        });
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
