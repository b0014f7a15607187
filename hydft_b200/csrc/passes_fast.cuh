// Transform passes built on the register FFT (regfft.cuh) for axis lengths
// with a register plan (32, 48, 64, 96, 128, 192, 256).  Same data layouts
// and semantics as the generic passes in kernels.cuh; these move each value
// through shared memory once per transform instead of once per radix pass.
//
// y/z passes: TX consecutive kx columns on the fastest thread index (coalesced
// 128-byte rows), T threads per column, G rows of the other axis per block.
// x passes: T threads per row of x, blockDim/T rows per block; the phase A
// and B physics runs in registers in block layout between the c2r and the
// r2c, streamed over pairs of output fields.
#pragma once

#include "kernels.cuh"
#include "regfft.cuh"
#include "tma.cuh"

namespace hydft {

__device__ __forceinline__ int fft_signed(int n, int L) { return n <= L / 2 ? n : n - L; }

// a b + c with one rounding, and a b rounded on its own (never contracted)
__device__ __forceinline__ float fma_r(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// ------------------------------------------------------------ y/z passes
// Column element addressing with 32-bit offsets from a per-thread base: a
// column of length L has its elements `rs` array elements apart.
//
// Band layout (the compact axis of the spectral arrays): signed index m
// with |m| <= M stored at c = m (m >= 0) or m + nc (m < 0); the thread's
// stride-layout elements are n = t + T e, so the offset of element e is
// (t or t - L + nc) * rs + e * T * rs and lies in the band when n <= M or
// n >= L - M.
// With BAND the band limit is the two-thirds rule's M = (L - 1) / 3, a
// compile-time constant: the elements e whose n = t + T e is in the low
// half (n <= M), in the high half (n >= L - M) or outside the band for every
// thread t < T are classified at compile time, so they need no per-element
// test, and the ones outside the band are neither loaded nor stored.  Only
// the (at most two) elements that straddle an edge keep a runtime test.
template <int T, int E>
__host__ __device__ constexpr int band_m() { return (T * E - 1) / 3; }
template <int T, int E>
__host__ __device__ constexpr bool band_all_lo(int e) { return T * e + T - 1 <= band_m<T, E>(); }
template <int T, int E>
__host__ __device__ constexpr bool band_all_hi(int e) { return T * e >= T * E - band_m<T, E>(); }
template <int T, int E>
__host__ __device__ constexpr bool band_none(int e)
{
    return T * e > band_m<T, E>() && T * e + T - 1 < T * E - band_m<T, E>();
}

// k0 times the signed index of stride-layout element e (n = t + T e) of an
// axis of length L, as kt + (T e or T e - L) k0 with kt = t k0: one fused
// multiply-add, whose half BAND fixes at compile time (the same expression
// either way, so both paths round alike)
template <typename R, int T, int E, bool BAND>
__device__ __forceinline__ R band_k(int e, int t, R k0, R kt)
{
    constexpr int L = T * E;
    if (BAND && band_all_lo<T, E>(e)) return kt + R(T * e) * k0;
    if (BAND && band_all_hi<T, E>(e)) return kt + R(T * e - L) * k0;
    return kt + R(t + T * e <= L / 2 ? T * e : T * e - L) * k0;
}

template <typename R, int T, int E, bool BAND>
__device__ __forceinline__ void load_band(cplx<R> (&v)[E], const cplx<R> *__restrict__ col, int rs, int t, int Mrt,
                                          int nc, bool valid)
{
    constexpr int L = T * E;
    const int M = BAND ? band_m<T, E>() : Mrt;
    const int lo_off = t * rs, hi_off = (t - L + nc) * rs, step = T * rs;
    const cplx<R> zero = {R(0), R(0)};
#pragma unroll
    for (int e = 0; e < E; ++e) {
        if (BAND && band_none<T, E>(e)) {
            v[e] = cplx<R>{R(-0.0), R(-0.0)};
        } else if (BAND && band_all_lo<T, E>(e)) {
            v[e] = valid ? col[lo_off + e * step] : zero;
        } else if (BAND && band_all_hi<T, E>(e)) {
            v[e] = valid ? col[hi_off + e * step] : zero;
        } else {
            const int n = t + T * e;
            const bool lo = n <= M, hi = n >= L - M;
            const int off = (lo ? lo_off : hi_off) + e * step;
            v[e] = (valid && (lo || hi)) ? col[off] : zero;
        }
    }
}

template <typename R, int T, int E, bool BAND>
__device__ __forceinline__ void store_band(cplx<R> *__restrict__ col, const cplx<R> (&v)[E], int rs, int t, int Mrt,
                                           int nc, R scale)
{
    constexpr int L = T * E;
    const int M = BAND ? band_m<T, E>() : Mrt;
    const int lo_off = t * rs, hi_off = (t - L + nc) * rs, step = T * rs;
#pragma unroll
    for (int e = 0; e < E; ++e) {
        if (BAND && band_none<T, E>(e)) continue;
        if (BAND && band_all_lo<T, E>(e)) {
            col[lo_off + e * step] = scale * v[e];
        } else if (BAND && band_all_hi<T, E>(e)) {
            col[hi_off + e * step] = scale * v[e];
        } else {
            const int n = t + T * e;
            const bool lo = n <= M, hi = n >= L - M;
            if (lo || hi) col[(lo ? lo_off : hi_off) + e * step] = scale * v[e];
        }
    }
}

// Full layout, block order: register r holds position block_pos(t, r)
template <typename R, int T, int E>
__device__ __forceinline__ void load_block(cplx<R> (&v)[E], const cplx<R> *__restrict__ col, int rs, int t, bool valid)
{
    const int base = t * rs;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int off = base + (T * (r / T) + E * (r % T)) * rs;
        v[r] = valid ? col[off] : cplx<R>{R(0), R(0)};
    }
}

template <typename R, int T, int E>
__device__ __forceinline__ void store_block(cplx<R> *__restrict__ col, const cplx<R> (&v)[E], int rs, int t)
{
    const int base = t * rs;
#pragma unroll
    for (int r = 0; r < E; ++r) col[base + (T * (r / T) + E * (r % T)) * rs] = v[r];
}

// z passes: NB ky rows (G apart) per thread, all NB columns loaded before the
// first is transformed, so that a thread keeps NB x E loads in flight
template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
__device__ __forceinline__ void zinv_body(const BlockIx &bk, const Grid &g, const PassArgs<R> &a, const cplx<R> *twz,
                                          const cplx<R> *tile = nullptr, const CUtensorMap *otm = nullptr,
                                          int odst = 0)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xb = tw + 2 * L;
    const int tid = threadIdx.x, c = tid % TX, t = (tid / TX) % T, gi = tid / (TX * T);
    const int x = bk.x * TX + c, f = bk.z;
    const int op = a.op[f];
    for (int i = tid; i < 2 * L; i += blockDim.x) tw[i] = twz[i];
    const R kx = R(x * g.kx0);
    const R kz0 = R(g.kz0), kzt = R(t) * kz0;
    // kz runs over the compact band: element stride nkyc * pkx
    const int rs = g.nkyc * g.pkx;
    cplx<R> v[NB][E];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int kyc = (bk.y * NB + b) * G + gi;
        const bool valid = x < g.nkxc && kyc < g.nkyc;
        if (tile)   // the block's input tile, [nkzc][G NB][TX], loaded by TMA
            load_band<R, T, E, BAND>(v[b], tile + (size_t)(b * G + gi) * TX + c, G * NB * TX, t, g.Mz, g.nkzc, valid);
        else
            load_band<R, T, E, BAND>(v[b], a.in[f] + (size_t)kyc * g.pkx + x, rs, t, g.Mz, g.nkzc, valid);
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int kyc = (bk.y * NB + b) * G + gi;
        const bool valid = x < g.nkxc && kyc < g.nkyc;
        const int my = valid ? signed_idx(kyc, g.My) : 0;
        const R ky = R(my * g.ky0);
        // the operator is uniform over the block
        switch (op) {
        case OP_ZK0:
            if (x == 0 && my == 0 && t == 0) v[b][0] = cplx<R>{R(0), R(0)};
            break;
        case OP_IKX:
#pragma unroll
            for (int e = 0; e < E; ++e)
                if (!(BAND && band_none<T, E>(e))) v[b][e] = ik_times(kx, v[b][e]);
            break;
        case OP_IKY:
#pragma unroll
            for (int e = 0; e < E; ++e)
                if (!(BAND && band_none<T, E>(e))) v[b][e] = ik_times(ky, v[b][e]);
            break;
        case OP_IKZ:
#pragma unroll
            for (int e = 0; e < E; ++e)
                if (!(BAND && band_none<T, E>(e))) v[b][e] = ik_times(band_k<R, T, E, BAND>(e, t, kz0, kzt), v[b][e]);
            break;
        case OP_NK2:
#pragma unroll
            for (int e = 0; e < E; ++e) {
                if (BAND && band_none<T, E>(e)) continue;
                const R kz = band_k<R, T, E, BAND>(e, t, kz0, kzt);
                v[b][e] = R(-(kx * kx + ky * ky + kz * kz)) * v[b][e];
            }
            break;
        default: break;
        }
        if (b == 0) __syncthreads();   // the twiddles (later rows: the exchange's own barriers)
        stride_to_block<T, E, +1, R, BarBlock, TX>(v[b], t, xb + gi * (L + L / T) * TX + c, tw);
        if (NB == 1 && otm) {
            // output tile [nz][G][TX] in the exchange space (nz = L <= the
            // space's L + L/T rows per G row), one tensor store
            store_block<R, T, E>(xb + (size_t)gi * TX + c, v[b], G * TX, t);
            tma_store_tile_4d(otm, xb, 2 * TX * (int)bk.x, G * (int)bk.y, 0, odst);
            return;
        }
        // z runs over the full axis: element stride nkyc * pkx in the ZI layout
        if (valid) store_block<R, T, E>(a.out[f] + (size_t)kyc * g.pkx + x, v[b], rs, t);
    }
}

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
__global__ void __launch_bounds__(TX * T * G) zinv_fast(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a, const cplx<R> *twz)
{
    zinv_body<R, T, E, TX, G, BAND, NB>(hw_block(), g, a, twz);
}

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
struct ZinvPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    __device__ __forceinline__ void run(const BlockIx &b) const { zinv_body<R, T, E, TX, G, BAND, NB>(b, g, a, tw); }
};

template <typename R, int T, int E, int TX, int G, bool BAND>
__device__ __forceinline__ void yinv_body(const BlockIx &bk, const Grid &g, const PassArgs<R> &a, const cplx<R> *twy,
                                          const cplx<R> *tile = nullptr, const CUtensorMap *otm = nullptr,
                                          int odst = 0)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xb = tw + 2 * L;
    const int tid = threadIdx.x, c = tid % TX, t = (tid / TX) % T, gi = tid / (TX * T);
    const int x = bk.x * TX + c, z = bk.y * G + gi, f = bk.z;
    const bool valid = x < g.nkxc && z < g.nz;
    for (int i = tid; i < 2 * L; i += blockDim.x) tw[i] = twy[i];
    cplx<R> v[E];
    if (tile)   // the block's input tile, [G][nkyc][TX], loaded by TMA
        load_band<R, T, E, BAND>(v, tile + (size_t)gi * g.nkyc * TX + c, TX, t, g.My, g.nkyc, valid);
    else
        load_band<R, T, E, BAND>(v, a.in[f] + (size_t)z * g.nkyc * g.pkx + x, g.pkx, t, g.My, g.nkyc, valid);
    // OP_IKY: the y derivative of a field whose z transform is shared with
    // other derivatives (k_y is constant along z); uniform over the block
    if (a.op[f] == OP_IKY) {
        const R ky0 = R(g.ky0), kyt = R(t) * ky0;
#pragma unroll
        for (int e = 0; e < E; ++e)
            if (!(BAND && band_none<T, E>(e))) v[e] = ik_times(band_k<R, T, E, BAND>(e, t, ky0, kyt), v[e]);
    }
    __syncthreads();
    stride_to_block<T, E, +1, R, BarBlock, TX>(v, t, xb + gi * (L + L / T) * TX + c, tw);
    if (otm) {
        // the exchange ended with a block barrier, so its space holds the
        // output tile [G][ny][TX] (ny <= L + L/T); columns past the band
        // hold zeros and land in the row padding, z planes past the grid
        // are clipped by the tensor store
        cplx<R> *ot = xb + (size_t)gi * g.ny * TX + c;
#pragma unroll
        for (int r = 0; r < E; ++r) ot[(size_t)block_pos<T, E>(t, r) * TX] = v[r];
        tma_store_tile_4d(otm, xb, 2 * TX * (int)bk.x, 0, G * (int)bk.y, odst);
        return;
    }
    if (valid) store_block<R, T, E>(a.out[f] + (size_t)z * g.ny * g.pkx + x, v, g.pkx, t);
}

template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) yinv_fast(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a, const cplx<R> *twy)
{
    yinv_body<R, T, E, TX, G, BAND>(hw_block(), g, a, twy);
}

template <typename R, int T, int E, int TX, int G, bool BAND>
struct YinvPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    __device__ __forceinline__ void run(const BlockIx &b) const { yinv_body<R, T, E, TX, G, BAND>(b, g, a, tw); }
};

template <typename R, int T, int E, int TX, int G, bool BAND>
__device__ __forceinline__ void yfwd_body(const BlockIx &bk, const Grid &g, const PassArgs<R> &a, const cplx<R> *twy,
                                          const cplx<R> *tile = nullptr, const CUtensorMap *otm = nullptr,
                                          int odst = 0)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xb = tw + 2 * L;
    const int tid = threadIdx.x, c = tid % TX, t = (tid / TX) % T, gi = tid / (TX * T);
    const int x = bk.x * TX + c, z = bk.y * G + gi, f = bk.z;
    const bool valid = x < g.nkxc && z < g.nz;
    for (int i = tid; i < 2 * L; i += blockDim.x) tw[i] = twy[i];
    cplx<R> v[E];
    if (tile)   // the block's input tile, [G][ny][TX], loaded by TMA
        load_block<R, T, E>(v, tile + (size_t)gi * g.ny * TX + c, TX, t, valid);
    else
        load_block<R, T, E>(v, a.in[f] + (size_t)z * g.ny * g.pkx + x, g.pkx, t, valid);
    __syncthreads();
    block_to_stride<T, E, -1, R, BarBlock, TX>(v, t, xb + gi * (L + L / T) * TX + c, tw);
    if (otm) {
        // output tile [G][nkyc][TX] in the exchange space (free after the
        // exchange's closing barrier); see yinv_body
        store_band<R, T, E, BAND>(xb + (size_t)gi * g.nkyc * TX + c, v, TX, t, g.My, g.nkyc, R(1));
        tma_store_tile_4d(otm, xb, 2 * TX * (int)bk.x, 0, G * (int)bk.y, odst);
        return;
    }
    if (valid) store_band<R, T, E, BAND>(a.out[f] + (size_t)z * g.nkyc * g.pkx + x, v, g.pkx, t, g.My, g.nkyc, R(1));
}

template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) yfwd_fast(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a, const cplx<R> *twy)
{
    yfwd_body<R, T, E, TX, G, BAND>(hw_block(), g, a, twy);
}

template <typename R, int T, int E, int TX, int G, bool BAND>
struct YfwdPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    __device__ __forceinline__ void run(const BlockIx &b) const { yfwd_body<R, T, E, TX, G, BAND>(b, g, a, tw); }
};

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
__device__ __forceinline__ void zfwd_body(const BlockIx &bk, const Grid &g, const PassArgs<R> &a, const cplx<R> *twz, R norm,
                                          const cplx<R> *tile = nullptr, const CUtensorMap *otm = nullptr)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xb = tw + 2 * L;
    const int tid = threadIdx.x, c = tid % TX, t = (tid / TX) % T, gi = tid / (TX * T);
    const int x = bk.x * TX + c, f = bk.z;
    for (int i = tid; i < 2 * L; i += blockDim.x) tw[i] = twz[i];
    const int rs = g.nkyc * g.pkx;
    cplx<R> v[NB][E];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int kyc = (bk.y * NB + b) * G + gi;
        const bool valid = x < g.nkxc && kyc < g.nkyc;
        if (tile)   // the block's input tile, [nz][G NB][TX], loaded by TMA
            load_block<R, T, E>(v[b], tile + (size_t)(b * G + gi) * TX + c, G * NB * TX, t, valid);
        else
            load_block<R, T, E>(v[b], a.in[f] + (size_t)kyc * g.pkx + x, rs, t, valid);
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int kyc = (bk.y * NB + b) * G + gi;
        const bool valid = x < g.nkxc && kyc < g.nkyc;
        if (b == 0) __syncthreads();   // the twiddles (later rows: the exchange's own barriers)
        block_to_stride<T, E, -1, R, BarBlock, TX>(v[b], t, xb + gi * (L + L / T) * TX + c, tw);
        if (NB == 1 && otm) {
            // output tile [nkzc][G][TX] of field f's compact array (map otm
            // covers that field alone), in the exchange space
            store_band<R, T, E, BAND>(xb + (size_t)gi * TX + c, v[b], G * TX, t, g.Mz, g.nkzc, norm);
            tma_store_tile_4d(otm, xb, 2 * TX * (int)bk.x, G * (int)bk.y, 0, 0);
            return;
        }
        if (valid) store_band<R, T, E, BAND>(a.out[f] + (size_t)kyc * g.pkx + x, v[b], rs, t, g.Mz, g.nkzc, norm);
    }
}

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
__global__ void __launch_bounds__(TX * T * G) zfwd_fast(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a, const cplx<R> *twz, R norm)
{
    zfwd_body<R, T, E, TX, G, BAND, NB>(hw_block(), g, a, twz, norm);
}

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
struct ZfwdPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    R norm;
    __device__ __forceinline__ void run(const BlockIx &b) const { zfwd_body<R, T, E, TX, G, BAND, NB>(b, g, a, tw, norm); }
};

// The TMA forms of the y inverse, y forward and z forward passes: thread 0
// loads the block's whole input tile into the exchange buffer's space with
// one tensor load (the tile is read into registers before the exchange
// reuses that space), then the block runs the same body on the tile.  The
// field coordinate of output f is src[f]; a wait that runs out sets
// ST_TIMEOUT in *status and the block returns without storing.
struct TmaFields {
    int src[MAXF];
    int dst[MAXF];     // output field coordinate (passes with a tensor store)
    unsigned *status;
};

// The tile goes at complex offset `off`: where the exchange buffer will be
// (after the 2L twiddles), or past the pass's own shared memory when it
// does not fit there (z inverse); its mbarrier goes right after the tile
// (the host sizes the space for tile + 8 bytes); the barrier is
// invalidated before the body reuses that space.  Returns the tile, or
// null when the destination is not 128-byte aligned (the block then reads
// global memory as the plain pass does); ok is false when the wait ran out.
template <typename R, int L>
__device__ __forceinline__ cplx<R> *tma_tile_begin(const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                                   unsigned bytes, bool &ok, size_t off = 2 * L)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tile = reinterpret_cast<cplx<R> *>(smraw) + off;
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(reinterpret_cast<unsigned char *>(tile) + bytes);
    ok = true;
    if ((smem_u32(tile) & 127u) != 0) return nullptr;   // uniform over the block
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, bytes);
        tma_load_4d(tile, tm, c0, c1, c2, c3, bar);
    }
    __syncthreads();
    // the block decides together, so that no thread leaves while others
    // wait at a later barrier
    ok = __syncthreads_and(mbar_wait_bounded(bar, 0)) != 0;
    if (ok && threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
    return tile;
}

// per-field tensor maps of the z inverse pass, whose inputs are separate
// compact fields (map f covers in[f] alone)
struct TmaMaps {
    CUtensorMap m[16];
};

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
__global__ void __launch_bounds__(TX * T * G) zinv_tma(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a,
                                                      const cplx<R> *twz, const __grid_constant__ TmaMaps tm,
                                                      unsigned tile_off, unsigned *status)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm.m[bk.z], 2 * TX * (int)bk.x, G * NB * (int)bk.y, 0, 0,
                                                   (unsigned)(2 * TX * G * NB * g.nkzc * sizeof(R)), ok, tile_off);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(status, ST_TIMEOUT);
        return;
    }
    zinv_body<R, T, E, TX, G, BAND, NB>(bk, g, a, twz, tile);
}

template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) yinv_tma(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a,
                                                      const cplx<R> *twy, const __grid_constant__ CUtensorMap tm,
                                                      const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, 0, G * (int)bk.y, tf.src[bk.z],
                                                   (unsigned)(2 * TX * g.nkyc * G * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    yinv_body<R, T, E, TX, G, BAND>(bk, g, a, twy, tile);
}

// The y inverse pass with a tensor load of its input tile and a tensor
// store of its output tile (map otm over the YI buffer)
template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) yinv_tma_st(const __grid_constant__ Grid g,
    const __grid_constant__ PassArgs<R> a, const cplx<R> *twy, const __grid_constant__ CUtensorMap tm,
    const __grid_constant__ CUtensorMap otm, const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, 0, G * (int)bk.y, tf.src[bk.z],
                                                   (unsigned)(2 * TX * g.nkyc * G * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    yinv_body<R, T, E, TX, G, BAND>(bk, g, a, twy, tile, &otm, tf.dst[bk.z]);
}

template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) yfwd_tma(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a,
                                                      const cplx<R> *twy, const __grid_constant__ CUtensorMap tm,
                                                      const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, 0, G * (int)bk.y, tf.src[bk.z],
                                                   (unsigned)(2 * TX * g.ny * G * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    yfwd_body<R, T, E, TX, G, BAND>(bk, g, a, twy, tile);
}

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
__global__ void __launch_bounds__(TX * T * G) zfwd_tma(const __grid_constant__ Grid g, const __grid_constant__ PassArgs<R> a,
                                                      const cplx<R> *twz, R norm, const __grid_constant__ CUtensorMap tm,
                                                      const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, G * NB * (int)bk.y, 0, tf.src[bk.z],
                                                   (unsigned)(2 * TX * G * NB * g.nz * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    zfwd_body<R, T, E, TX, G, BAND, NB>(bk, g, a, twz, norm, tile);
}

// The forward y pass with tensor load and tensor store (map otm over the
// ZI buffer)
template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) yfwd_tma_st(const __grid_constant__ Grid g,
    const __grid_constant__ PassArgs<R> a, const cplx<R> *twy, const __grid_constant__ CUtensorMap tm,
    const __grid_constant__ CUtensorMap otm, const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, 0, G * (int)bk.y, tf.src[bk.z],
                                                   (unsigned)(2 * TX * g.ny * G * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    yfwd_body<R, T, E, TX, G, BAND>(bk, g, a, twy, tile, &otm, tf.dst[bk.z]);
}

// The forward z pass (one row per thread) with tensor load and a tensor
// store into each output field's compact array (om.m[f] covers field f)
template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) zfwd_tma_st(const __grid_constant__ Grid g,
    const __grid_constant__ PassArgs<R> a, const cplx<R> *twz, R norm, const __grid_constant__ CUtensorMap tm,
    const __grid_constant__ TmaMaps om, const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, G * (int)bk.y, 0, tf.src[bk.z],
                                                   (unsigned)(2 * TX * G * g.nz * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    zfwd_body<R, T, E, TX, G, BAND, 1>(bk, g, a, twz, norm, tile, &om.m[bk.z]);
}

// The inverse z pass (one row per thread) with a tensor load of its input
// tile into the exchange space (every column is read into registers before
// the first exchange) and a tensor store of its output tile
template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) zinv_tma_st(const __grid_constant__ Grid g,
    const __grid_constant__ PassArgs<R> a, const cplx<R> *twz, const __grid_constant__ TmaMaps tm,
    const __grid_constant__ CUtensorMap otm, const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    bool ok;
    const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm.m[bk.z], 2 * TX * (int)bk.x, G * (int)bk.y, 0, 0,
                                                   (unsigned)(2 * TX * G * g.nkzc * sizeof(R)), ok);
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
        return;
    }
    zinv_body<R, T, E, TX, G, BAND, 1>(bk, g, a, twz, tile, &otm, tf.dst[bk.z]);
}

// The inverse z pass (one row per thread) with a tensor store of its output
// tile (map otm over the ZI buffer, field coordinate dst[f])
template <typename R, int T, int E, int TX, int G, bool BAND>
__global__ void __launch_bounds__(TX * T * G) zinv_st(const __grid_constant__ Grid g,
    const __grid_constant__ PassArgs<R> a, const cplx<R> *twz, const __grid_constant__ CUtensorMap otm,
    const __grid_constant__ TmaFields tf)
{
    const BlockIx bk = hw_block();
    zinv_body<R, T, E, TX, G, BAND, 1>(bk, g, a, twz, nullptr, &otm, tf.dst[bk.z]);
}

// The ensemble forms of the TMA passes: each pack carries its simulation's
// tensor map (kernel parameter space, from which a tensor load may read its
// map) and field coordinates, and runs the TMA kernel's body.
template <typename R, int T, int E, int TX, int G, bool BAND>
struct YinvTmaPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    CUtensorMap tm;
    CUtensorMap otm;   // the output tile's tensor store when store != 0
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    TmaFields tf;
    int store;
    __device__ __forceinline__ void run(const BlockIx &bk) const
    {
        bool ok;
        const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, 0, G * (int)bk.y, tf.src[bk.z],
                                                       (unsigned)(2 * TX * g.nkyc * G * sizeof(R)), ok);
        if (!ok) {
            if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
            return;
        }
        yinv_body<R, T, E, TX, G, BAND>(bk, g, a, tw, tile, store ? &otm : nullptr, tf.dst[bk.z]);
    }
};

template <typename R, int T, int E, int TX, int G, bool BAND>
struct YfwdTmaPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    CUtensorMap tm;
    CUtensorMap otm;   // the output tile's tensor store when store != 0
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    TmaFields tf;
    int store;
    __device__ __forceinline__ void run(const BlockIx &bk) const
    {
        bool ok;
        const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, 0, G * (int)bk.y, tf.src[bk.z],
                                                       (unsigned)(2 * TX * g.ny * G * sizeof(R)), ok);
        if (!ok) {
            if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
            return;
        }
        yfwd_body<R, T, E, TX, G, BAND>(bk, g, a, tw, tile, store ? &otm : nullptr, tf.dst[bk.z]);
    }
};

template <typename R, int T, int E, int TX, int G, bool BAND, int NB>
struct ZfwdTmaPack {
    static constexpr int MAXT = TX * T * G, MINB = 1;
    CUtensorMap tm;
    Grid g;
    PassArgs<R> a;
    const cplx<R> *tw;
    R norm;
    TmaFields tf;
    __device__ __forceinline__ void run(const BlockIx &bk) const
    {
        bool ok;
        const cplx<R> *tile = tma_tile_begin<R, T * E>(&tm, 2 * TX * (int)bk.x, G * NB * (int)bk.y, 0, tf.src[bk.z],
                                                       (unsigned)(2 * TX * G * NB * g.nz * sizeof(R)), ok);
        if (!ok) {
            if (threadIdx.x == 0) atomicOr(tf.status, ST_TIMEOUT);
            return;
        }
        zfwd_body<R, T, E, TX, G, BAND, NB>(bk, g, a, tw, norm, tile);
    }
};

// smem bytes of a y/z fast pass
template <typename R>
inline size_t yz_fast_smem(int L, int T, int TX, int G)
{
    return sizeof(cplx<R>) * (2 * (size_t)L + (size_t)G * (L + L / T) * TX);
}

// --------------------------------------------------------------- x passes
// row exchange buffer stride: the padded row (L + L/T elements) rounded up
// to 16 elements, plus T when several rows share a half-warp, so that row r
// starts at bank group r*T and the rows of a half-warp never collide
template <int T, int E>
__host__ __device__ constexpr int xrow_stride() { return (T * E + E + 15) / 16 * 16 + (T < 16 ? T : 0); }

// c2r input of a pair of half spectra (kx <= Mx, XF/YI layout) in stride
// layout, then inverse FFT to block layout: v[r] = a(x) + i b(x) at
// x = block_pos(t, r).  inb may be null (b = 0).  BAND: Mx is the
// two-thirds rule's band_m (see load_band).
//
// dxa / dxb: the input is differentiated along x on the way in (a_k becomes
// i k kx0 a_k), for fields whose z and y transforms are shared with their
// other derivatives.  BM: inb is null (0), not null (1) or tested (2).
// Loads from rows staged in shared memory pass rowok = true: every staged
// row slot exists (unused ones hold stale data whose results are not
// stored).
template <typename R, int T, int E, bool BAND = false, int BM = 2>
__device__ __forceinline__ void x_c2r_load(cplx<R> (&v)[E], const cplx<R> *__restrict__ ina,
                                           const cplx<R> *__restrict__ inb, size_t base, bool rowok, int t, int Mrt,
                                           bool dxa = false, bool dxb = false, R kx0 = R(0))
{
    constexpr int L = T * E;
    const int Mx = BAND ? band_m<T, E>() : Mrt;
    const cplx<R> zero = {R(0), R(0)};
    const R kxt = R(t) * kx0;
    // half-spectrum entries kk of a and b; kxk = kk kx0 for the derivative
    // the derivative's products are rounded on their own (not contracted
    // into the sums below), the same in every instantiation
    auto ikx = [](R k, cplx<R> v) { return cplx<R>{mul_rn(-k, v.y), mul_rn(k, v.x)}; };
    auto get = [&](int kk, R kxk, cplx<R> &va, cplx<R> &vb) {
        va = ina[base + kk];
        vb = (BM == 1 || (BM == 2 && inb)) ? inb[base + kk] : zero;
        if (dxa) va = ikx(kxk, va);
        if (dxb) vb = ikx(kxk, vb);
    };
    // k = t + T e <= Mx: a_k + i b_k; k >= L - Mx: conj(a_{L-k}) + i conj(b_{L-k})
    auto lo = [&](int k, int e) {
        cplx<R> va, vb;
        get(k, kxt + R(T * e) * kx0, va, vb);
        if (k == 0) { va.y = R(0); vb.y = R(0); }
        return cplx<R>{va.x - vb.y, va.y + vb.x};
    };
    auto hi = [&](int k, int e) {
        cplx<R> va, vb;
        get(L - k, R(L - T * e) * kx0 - kxt, va, vb);
        return cplx<R>{va.x + vb.y, -va.y + vb.x};
    };
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const int k = t + T * e;
        if (BAND && band_none<T, E>(e)) {
            v[e] = cplx<R>{R(-0.0), R(-0.0)};
        } else if (BAND && band_all_lo<T, E>(e)) {
            v[e] = rowok ? lo(k, e) : zero;
        } else if (BAND && band_all_hi<T, E>(e)) {
            v[e] = rowok ? hi(k, e) : zero;
        } else {
            cplx<R> Z = zero;
            if (rowok) {
                if (k <= Mx) Z = lo(k, e);
                else if (k >= L - Mx) Z = hi(k, e);
            }
            v[e] = Z;
        }
    }
}

template <typename R, int T, int E, bool BAND = false>
__device__ __forceinline__ void x_c2r_pair(cplx<R> (&v)[E], const cplx<R> *__restrict__ ina,
                                           const cplx<R> *__restrict__ inb, int row, bool rowok, int t,
                                           const Grid &g, cplx<R> *xrow, const cplx<R> *tw)
{
    x_c2r_load<R, T, E, BAND>(v, ina, inb, (size_t)row * g.pkx, rowok, t, g.Mx);
    stride_to_block<T, E, +1, R, BarWarp, 1>(v, t, xrow, tw);
}

// r2c of z = a + i b given in block layout; writes the half spectra of a
// and b for kx <= Mx (outb null (BM 0), not null (1) or tested (2)).  UNR
// with BAND: the output loop is unrolled over the compile-time band
// classification (no divergent trip count; more registers live)
template <typename R, int T, int E, bool BAND = false, int BM = 2, bool UNR = false>
__device__ __forceinline__ void x_r2c_pair(cplx<R> (&v)[E], cplx<R> *__restrict__ outa, cplx<R> *__restrict__ outb,
                                           int row, bool rowok, int t, const Grid &g, cplx<R> *xrow,
                                           const cplx<R> *tw)
{
    constexpr int L = T * E;
    block_to_stride<T, E, -1, R, BarWarp, 1>(v, t, xrow, tw);
    // element t + T m; with BAND the ones outside the band for every t are
    // never read below, so neither they nor their last butterflies are made
#pragma unroll
    for (int m = 0; m < E; ++m)
        if (!(BAND && band_none<T, E>(m))) xrow[t + m * (T + 1)] = v[m];
    __syncwarp();
    const size_t base = (size_t)row * g.pkx;
    auto put = [&](int k) {
        const cplx<R> zk = xrow[xidx<T>(k)];
        const cplx<R> zm = conj(xrow[xidx<T>(k == 0 ? 0 : L - k)]);
        outa[base + k] = R(0.5) * (zk + zm);
        if (BM == 1 || (BM == 2 && outb)) outb[base + k] = mul_i<-1>(R(0.5) * (zk - zm));
    };
    if (rowok) {
        if (BAND && UNR) {
#pragma unroll
            for (int e = 0; e < E; ++e) {
                if (band_all_lo<T, E>(e)) put(t + T * e);
                else if (T * e <= band_m<T, E>() && t + T * e <= band_m<T, E>()) put(t + T * e);
            }
        } else {
            const int Mx = BAND ? band_m<T, E>() : g.Mx;
            for (int k = t; k <= Mx; k += T) put(k);
        }
    }
    __syncwarp();
}

template <typename R>
struct XFastArgs {
    const cplx<R> *in[MAXF];
    cplx<R> *out[MAXF];
    int nin, nout;
    int dx_in_pass;   // phase B (xb_rows): the x derivatives arrive underived
};

// packed (i <= j) flux index -> (i, j) for three components
__host__ __device__ constexpr int flux_i3(int f) { return f < 3 ? 0 : (f < 5 ? 1 : 2); }
__host__ __device__ constexpr int flux_j3(int f) { return f < 3 ? f : (f < 5 ? f - 2 : 2); }

// Phase A (3-D): inputs dn, m_0..m_2 [, dn/dx_0..2, lap n]; outputs u_d,
// the fluxes m_i u_j (i <= j) and mu_local (UONLY: u_d only).  Input pairs
// and mu_local are kept in per-thread shared-memory slots (block layout);
// each output pair is then computed, transformed and written in turn.
#ifndef HYDFT_XMINB
#define HYDFT_XMINB 1
#endif

template <typename R, int T, int E, int NM, bool GRAD, bool UONLY>
__device__ __forceinline__ void xa_fast_body(const BlockIx &bk, const Grid &g, const XFastArgs<R> &a,
    const cplx<R> *twx, const PWA<R> &pw)
{
    static_assert(NM == 3, "fast x pass is for 3-D grids");
    constexpr int L = T * E;
    constexpr int NIN = 1 + NM + (GRAD ? NM + 1 : 0);
    constexpr int NP = (NIN + 1) / 2;
    constexpr int NF = NM * (NM + 1) / 2;
    constexpr int NOUT = UONLY ? NM : NM + NF + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xbuf = tw + 2 * L;
    const int nt = blockDim.x, rb = nt / T;
    cplx<R> *slots = xbuf + rb * xrow_stride<T, E>();
    R *muslot = reinterpret_cast<R *>(slots + NP * E * nt);
    R *invslot = muslot + E * nt;
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int row = bk.x * rb + rr;
    const bool rowok = row < g.ny * g.nz;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    for (int i = tid; i < 2 * L; i += nt) tw[i] = twx[i];
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < NP; ++p) {
        cplx<R> v[E];
        x_c2r_pair<R, T, E>(v, a.in[2 * p], 2 * p + 1 < NIN ? a.in[2 * p + 1] : nullptr, row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) slots[(p * E + r) * nt + tid] = v[r];
    }
    auto input = [&](int f, int r) -> R {
        const cplx<R> s = slots[((f / 2) * E + r) * nt + tid];
        return (f & 1) ? s.y : s.x;
    };
    // the mean density is exact in the k = 0 mode; deviations carry the
    // signal, so n, 1/(m n) and ln(n/nref) are formed in the field precision
    const double nref64 = *pw.nmean;
    const R nref = R(nref64);
    const R inv_nref = R(1) / nref, inv_beta = R(pw.ph.inv_beta), mass = R(pw.ph.mass);
    const size_t rowbase = (size_t)row * g.nx;
    // density check, real-space dn and u for phase B, 1/(m n) and the local
    // chemical potential into per-thread slots
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
            if (pw.u_real) {
                for (int d = 0; d < NM; ++d) pw.u_real[d * pw.ncell + rowbase + xx] = input(1 + d, r) * inv_mn;
            }
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
                    // alpha(n) by FP64 Newton on the Fermi-Dirac table
                    const double n64 = nref64 + (double)dn;
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
    // output pairs
#pragma unroll
    for (int q = 0; 2 * q < NOUT; ++q) {
        cplx<R> v[E];
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const R inv_mn = invslot[r * nt + tid];
            R val[2] = {R(0), R(0)};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = 2 * q + h;
                if (o < NM) val[h] = input(1 + o, r) * inv_mn;
                else if (o < NM + NF) val[h] = input(1 + flux_i3(o - NM), r) * (input(1 + flux_j3(o - NM), r) * inv_mn);
                else if (o < NOUT) val[h] = muslot[r * nt + tid];
            }
            v[r] = cplx<R>{val[0], val[1]};
        }
        x_r2c_pair<R, T, E>(v, a.out[2 * q], 2 * q + 1 < NOUT ? a.out[2 * q + 1] : nullptr, row, rowok, t, g, xrow, tw);
    }
}

template <typename R, int T, int E, int NM, bool GRAD, bool UONLY>
__global__ void __launch_bounds__(256, HYDFT_XMINB) xa_fast(const __grid_constant__ Grid g, const __grid_constant__ XFastArgs<R> a,
    const cplx<R> *twx, const __grid_constant__ PWA<R> pw)
{
    xa_fast_body<R, T, E, NM, GRAD, UONLY>(hw_block(), g, a, twx, pw);
}

template <typename R, int T, int E, int NM, bool GRAD, bool UONLY>
struct XaFastPack {
    static constexpr int MAXT = 256, MINB = HYDFT_XMINB;
    Grid g;
    XFastArgs<R> a;
    const cplx<R> *tw;
    PWA<R> pw;
    __device__ __forceinline__ void run(const BlockIx &b) const { xa_fast_body<R, T, E, NM, GRAD, UONLY>(b, g, a, tw, pw); }
};

// Phase B: inputs [d mu/dx_0 ..], then for each Pi component pair (c, c+1)
// and d < NM the pair (d Pi_c/dx_d, d Pi_{c+1}/dx_d); outputs
// n (d mu/dx_i - F_i) and, when Pi evolves, -u.grad Pi_c.
template <typename R, int T, int E, int NM, bool EVOLVE>
__device__ __forceinline__ void xb_fast_body(const BlockIx &bk, const Grid &g, const XFastArgs<R> &a,
    const cplx<R> *twx, const PWB<R> &pw)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xbuf = tw + 2 * L;
    const int nt = blockDim.x, rb = nt / T;
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int row = bk.x * rb + rr;
    const bool rowok = row < g.ny * g.nz;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    for (int i = tid; i < 2 * L; i += nt) tw[i] = twx[i];
    __syncthreads();
    const double nref64 = *pw.nmean;
    const R nref = R(nref64);
    const size_t rowbase = (size_t)row * g.nx;
    const int y = rowok ? row % g.ny : 0, z = rowok ? row / g.ny : 0;
    // n (dmu - F): pairs of components
#pragma unroll
    for (int q = 0; 2 * q < NM; ++q) {
        const int i0 = 2 * q, i1 = 2 * q + 1;
        cplx<R> v[E];
        x_c2r_pair<R, T, E>(v, a.in[i0], i1 < NM ? a.in[i1] : nullptr, row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int xx = block_pos<T, E>(t, r);
            const R n = rowok ? nref + pw.dn_real[rowbase + xx] : R(0);
            R f0 = R(0), f1 = R(0);
            if (pw.ph.ext_active && pw.ph.ext_kind == 3) {
                f0 = rowok ? -pw.gradv[(size_t)i0 * pw.ncell + rowbase + xx] : R(0);
                if (i1 < NM) f1 = rowok ? -pw.gradv[(size_t)i1 * pw.ncell + rowbase + xx] : R(0);
            } else if (pw.ph.ext_active) {
                const StageScal &s = pw.ctrl->st[pw.stage];
                cplx<double> e = pw.ex[xx] * pw.ey[y];
                e = e * pw.ez[z];
                e = e * cplx<double>{s.ewr, s.ewi};
                const double sf = s.amp * e.y;
                f0 = R(sf * pw.ph.ext_k[i0]);
                if (i1 < NM) f1 = R(sf * pw.ph.ext_k[i1]);
            }
            v[r] = cplx<R>{n * (v[r].x - f0), n * (v[r].y - f1)};
        }
        x_r2c_pair<R, T, E>(v, a.out[i0], i1 < NM ? a.out[i1] : nullptr, row, rowok, t, g, xrow, tw);
    }
    if (EVOLVE) {
        // -u.grad Pi for component pairs (0,1), (2,3), (4,5)
#pragma unroll 1
        for (int cp = 0; cp < 3; ++cp) {
            cplx<R> acc[E];
#pragma unroll
            for (int r = 0; r < E; ++r) acc[r] = cplx<R>{R(0), R(0)};
#pragma unroll
            for (int d = 0; d < NM; ++d) {
                const int f = NM + 2 * (cp * NM + d);
                cplx<R> v[E];
                x_c2r_pair<R, T, E>(v, a.in[f], a.in[f + 1], row, rowok, t, g, xrow, tw);
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int xx = block_pos<T, E>(t, r);
                    const R u = rowok ? pw.u_real[d * pw.ncell + rowbase + xx] : R(0);
                    acc[r] = acc[r] - u * v[r];
                }
            }
            x_r2c_pair<R, T, E>(acc, a.out[NM + 2 * cp], a.out[NM + 2 * cp + 1], row, rowok, t, g, xrow, tw);
        }
    }
}

template <typename R, int T, int E, int NM, bool EVOLVE>
__global__ void __launch_bounds__(256, HYDFT_XMINB) xb_fast(const __grid_constant__ Grid g, const __grid_constant__ XFastArgs<R> a,
    const cplx<R> *twx, const __grid_constant__ PWB<R> pw)
{
    xb_fast_body<R, T, E, NM, EVOLVE>(hw_block(), g, a, twx, pw);
}

template <typename R, int T, int E, int NM, bool EVOLVE>
struct XbFastPack {
    static constexpr int MAXT = 256, MINB = HYDFT_XMINB;
    Grid g;
    XFastArgs<R> a;
    const cplx<R> *tw;
    PWB<R> pw;
    __device__ __forceinline__ void run(const BlockIx &b) const { xb_fast_body<R, T, E, NM, EVOLVE>(b, g, a, tw, pw); }
};

// Staging of the x passes' input rows.  The rows of x a warp transforms
// (32/T of them) are its own: lane 0 copies the warp's rows of each staged
// field into shared memory with one bulk copy per field (the rows of a
// block are contiguous in every field), completing on the warp's own
// mbarrier, so no block-wide barrier follows the start of the pass.  The
// barriers sit past the pass's other shared memory, 16 bytes per warp.
template <int T>
__host__ __device__ constexpr int x_rows_per_warp() { return 32 / T; }

// the warp's rows that exist: inside its block (rb rows) and the grid
template <int T>
__device__ __forceinline__ int warp_rows(int w, int rb, int row0, int nrows)
{
    constexpr int RPW = x_rows_per_warp<T>();
    return max(0, min(min(RPW, rb - w * RPW), nrows - row0 - w * RPW));
}

// Waits for phase `parity` of a warp's staging barrier.  A wait that runs
// out (it is bounded) sets ST_TIMEOUT, which fails the step, and returns.
__device__ __forceinline__ void warp_stage_wait(unsigned long long *bar, unsigned parity, unsigned *status)
{
    if (!mbar_wait_bounded(bar, parity) && (threadIdx.x & 31) == 0) atomicOr(status, ST_TIMEOUT);
    __syncwarp();
}

// bulk prefetch of a 16-byte aligned global range (a multiple of 16 bytes)
// into L2; no completion to wait for
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// The spectral input rows of one block of x rows are contiguous in every
// field (row stride pkx).  XPrefetch keeps the rows of the next fields in
// flight to L2 (thread 0 of the block issues one bulk prefetch per field)
// while the current field pair is transformed.
template <typename R>
struct XPrefetch {
    const XFastArgs<R> &a;
    size_t off;
    unsigned bytes;
    int next = 0;
    bool issuer;
    __device__ XPrefetch(const XFastArgs<R> &a_, const Grid &g, int row0, int rows, bool is0)
        : a(a_), off((size_t)row0 * g.pkx), bytes((unsigned)((size_t)rows * g.pkx * sizeof(cplx<R>))), issuer(is0) {}
    // prefetch every field up to index f (inclusive)
    __device__ __forceinline__ void upto(int f)
    {
        for (; next <= f && next < a.nin; ++next)
            if (issuer && bytes) prefetch_l2(a.in[next] + off, bytes);
    }
};

// Staged real rows: each row of x holds its nreal fields back to back (one
// row of x each), and rows are nreal L + T elements apart, so that the rows
// read by one warp start T banks apart (L is a multiple of 16, and of 32
// where T > 4) and never collide
template <int T, int E>
__host__ __device__ constexpr int xreal_stride(int nreal) { return nreal * T * E + T; }

// shared-memory bytes of the staged x passes before the warps' staging
// barriers: twiddles, staged spectral rows (nstage fields), exchange rows,
// staged real rows (nreal fields), rounded up to 16
template <typename R, int T, int E>
__host__ __device__ inline size_t xstaged_body_bytes(int nt, int pkx, int nstage, int nreal)
{
    const int rb = nt / T;
    const size_t b = sizeof(cplx<R>) * (2 * (size_t)T * E + (size_t)nstage * rb * pkx + (size_t)rb * xrow_stride<T, E>()) +
                     (nreal ? sizeof(R) * (size_t)rb * xreal_stride<T, E>(nreal) : 0);
    return (b + 15) / 16 * 16;
}
// all of it: two 8-byte barriers per warp after the body
template <typename R, int T, int E>
inline size_t xstaged_smem(int nt, int pkx, int nstage, int nreal)
{
    return xstaged_body_bytes<R, T, E>(nt, pkx, nstage, nreal) + 16 * (size_t)((nt + 31) / 32);
}

// blocks per SM the staged x passes are compiled for: two 256-thread blocks
// in single precision with up to 16 values per thread, else one
template <typename R, int E>
__host__ __device__ constexpr int xstaged_minb() { return sizeof(R) == 4 && E <= 16 ? 2 : 1; }

// Phase A without Fermi-Dirac terms (ideal / Hartree / RY ions and the u-only
// relaxation finish): the four inputs dn, m_0..m_2 stay in registers as two
// pairs, so no per-thread shared-memory slots are needed and two 256-thread
// blocks fit on an SM.  The block's spectral input rows are copied into
// shared memory first (each warp its own rows, by bulk copies: pair 1
// lands while pair 0 is transformed).  The output pairs are ordered so that dn is consumed
// first: (mu_local, u_0), (u_1, u_2), (m0u0, m0u1), (m0u2, m1u1), (m1u2, m2u2);
// UONLY: (u_0, u_1), (u_2, -).  Outputs go to the same fields as xa_fast's.
template <typename R, int T, int E, bool UONLY, bool BAND>
__device__ __forceinline__ void xa_regs_body(const BlockIx &bk, const Grid &g, const XFastArgs<R> &a,
    const cplx<R> *twx, const PWA<R> &pw)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    const int nt = blockDim.x, rb = nt / T, pk = g.pkx;
    cplx<R> *sb = tw + 2 * L;                      // [4][rb][pkx] the staged inputs
    cplx<R> *xbuf = sb + 4 * (size_t)rb * pk;
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int row0 = bk.x * rb, row = row0 + rr;
    const bool rowok = row < g.ny * g.nz;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    // the warp's rows of all four inputs on their way at once, one barrier
    // per pair: pair 1 lands while pair 0 is transformed
    constexpr int RPW = x_rows_per_warp<T>();
    const int lane = tid & 31, w = tid >> 5;
    const int wrows = warp_rows<T>(w, rb, row0, g.ny * g.nz);
    unsigned long long *bars =
        reinterpret_cast<unsigned long long *>(smraw + xstaged_body_bytes<R, T, E>(nt, pk, 4, 0)) + 2 * w;
    if (lane == 0) {
        mbar_init(bars, 1);
        mbar_init(bars + 1, 1);
        if (wrows > 0) {
            const unsigned bytes = (unsigned)(wrows * pk * sizeof(cplx<R>));
            const size_t src = (size_t)(row0 + w * RPW) * pk;
            for (int q = 0; q < 2; ++q) {
                mbar_expect_tx(bars + q, 2 * bytes);
                for (int f = 2 * q; f < 2 * q + 2; ++f)
                    bulk_load(sb + ((size_t)f * rb + w * RPW) * pk, a.in[f] + src, bytes, bars + q);
            }
        }
    }
    for (int i = tid; i < 2 * L; i += nt) tw[i] = twx[i];
    __syncthreads();
    cplx<R> p0[E], p1[E];   // (dn, m_0), (m_1, m_2)
    const size_t sbase = (size_t)rr * pk;
    if (wrows > 0) warp_stage_wait(bars, 0, pw.status);
    x_c2r_load<R, T, E, BAND, 1>(p0, sb, sb + (size_t)rb * pk, sbase, true, t, g.Mx);
    stride_to_block<T, E, +1, R, BarWarp, 1>(p0, t, xrow, tw);
    if (wrows > 0) warp_stage_wait(bars + 1, 0, pw.status);
    x_c2r_load<R, T, E, BAND, 1>(p1, sb + 2 * (size_t)rb * pk, sb + 3 * (size_t)rb * pk, sbase, true, t, g.Mx);
    stride_to_block<T, E, +1, R, BarWarp, 1>(p1, t, xrow, tw);
    const double nref64 = *pw.nmean;
    const R nref = R(nref64);
    const R inv_nref = R(1) / nref, inv_beta = R(pw.ph.inv_beta), mass = R(pw.ph.mass);
    const size_t rowbase = (size_t)row * g.nx;
    // occurrences of the ideal term (the only local term this kernel has) in
    // the term list, counted once rather than per element
    int nid = 0;
    for (int tt = 0; tt < pw.ph.nterms_local; ++tt) nid += pw.ph.term_order[tt] == 1;
    // mu_local (ideal terms in the given order) and 1/(m n); p0[r].x becomes 1/(m n)
    cplx<R> v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int xx = block_pos<T, E>(t, r);
        const R dn = p0[r].x;
        const R n = nref + dn;
        const R inv_mn = R(1) / (mass * n);
        if (rowok) {
            if (!(n > R(0))) atomicOr(pw.status, isfinite(n) ? ST_NONPOS : ST_NONFINITE);
            if (pw.dn_real) pw.dn_real[rowbase + xx] = dn;
            if (pw.u_real) {
                pw.u_real[rowbase + xx] = p0[r].y * inv_mn;
                pw.u_real[pw.ncell + rowbase + xx] = p1[r].x * inv_mn;
                pw.u_real[2 * pw.ncell + rowbase + xx] = p1[r].y * inv_mn;
            }
        }
        if (!UONLY) {
            R mu = R(0);
            if (nid > 0) {
                const R l = log1p(dn * inv_nref) * inv_beta;
                mu += l;
                for (int c = 1; c < nid; ++c) mu += l;
            }
            v[r] = cplx<R>{mu, p0[r].y * inv_mn};
        } else {
            v[r] = cplx<R>{p0[r].y * inv_mn, p1[r].x * inv_mn};
        }
        p0[r].x = inv_mn;
    }
    if (!UONLY) {
        // (m_1, m_2) wait in the warp's own staging space, whose inputs are
        // consumed, while the output pairs are transformed: 2E fewer live
        // registers per thread (the kernel spilled with them all in
        // registers).  Lane l keeps element r at entry r 32 + l of the warp's
        // four field slices (4 x 32/T rows x pkx entries >= 32 E, as
        // pkx > L/3); the warp reads the same entries it wrote.
        const int slice = RPW * pk;
        auto stash = [&](int r) -> cplx<R> & {
            const int e = r * 32 + lane;
            return sb[((size_t)(e / slice) * rb + w * RPW) * pk + e % slice];
        };
        __syncwarp();
#pragma unroll
        for (int r = 0; r < E; ++r) stash(r) = p1[r];
        // outputs: 0..2 u_d, 3..8 fluxes (00, 01, 02, 11, 12, 22), 9 mu
        x_r2c_pair<R, T, E, BAND, 1>(v, a.out[9], a.out[0], row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const cplx<R> q = stash(r);
            v[r] = cplx<R>{q.x * p0[r].x, q.y * p0[r].x};
        }
        x_r2c_pair<R, T, E, BAND, 1>(v, a.out[1], a.out[2], row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const cplx<R> q = stash(r);
            const R u0 = p0[r].y * p0[r].x;
            v[r] = cplx<R>{p0[r].y * u0, p0[r].y * (q.x * p0[r].x)};
        }
        x_r2c_pair<R, T, E, BAND, 1>(v, a.out[3], a.out[4], row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const cplx<R> q = stash(r);
            const R u1 = q.x * p0[r].x, u2 = q.y * p0[r].x;
            v[r] = cplx<R>{p0[r].y * u2, q.x * u1};
        }
        x_r2c_pair<R, T, E, BAND, 1>(v, a.out[5], a.out[6], row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const cplx<R> q = stash(r);
            const R u2 = q.y * p0[r].x;
            v[r] = cplx<R>{q.x * u2, q.y * u2};
        }
        x_r2c_pair<R, T, E, BAND, 1>(v, a.out[7], a.out[8], row, rowok, t, g, xrow, tw);
    } else {
        x_r2c_pair<R, T, E, BAND, 1>(v, a.out[0], a.out[1], row, rowok, t, g, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = cplx<R>{p1[r].y * p0[r].x, R(0)};
        x_r2c_pair<R, T, E, BAND, 0>(v, a.out[2], nullptr, row, rowok, t, g, xrow, tw);
    }
}

template <typename R, int T, int E, bool UONLY, bool BAND>
__global__ void __launch_bounds__(256, xstaged_minb<R, E>()) xa_regs(const __grid_constant__ Grid g, const __grid_constant__ XFastArgs<R> a,
    const cplx<R> *twx, const __grid_constant__ PWA<R> pw)
{
    xa_regs_body<R, T, E, UONLY, BAND>(hw_block(), g, a, twx, pw);
}

template <typename R, int T, int E, bool UONLY, bool BAND>
struct XaRegsPack {
    static constexpr int MAXT = 256, MINB = xstaged_minb<R, E>();
    Grid g;
    XFastArgs<R> a;
    const cplx<R> *tw;
    PWA<R> pw;
    __device__ __forceinline__ void run(const BlockIx &b) const { xa_regs_body<R, T, E, UONLY, BAND>(b, g, a, tw, pw); }
};

// Phase B with each warp's real-space u_d rows (when Pi evolves) copied into
// shared memory at the start with the first input pair, and each input pair
// staged one pair ahead of the transform that reads it (bulk copies on the
// warp's own barrier, whose phases follow the pairs); the spectral inputs
// are prefetched to L2 a few fields ahead and dn comes straight into
// registers.  Same inputs, outputs and arithmetic as xb_fast, except that
// with a.dx_in_pass the x derivatives (of mu and of each Pi component)
// arrive underived, sharing their z and y transforms with the y derivative,
// and are differentiated here on the way in.  EXTK: no external force (0), a
// plane-wave potential (1), the gaussian potential's static force field (2).
template <typename R, int T, int E, bool EVOLVE, int EXTK, bool BAND>
__device__ __forceinline__ void xb_rows_body(const BlockIx &bk, const Grid &g, const XFastArgs<R> &a,
    const cplx<R> *twx, const PWB<R> &pw)
{
    constexpr int L = T * E, NM = 3;
    constexpr int RS = xreal_stride<T, E>(NM);
    constexpr int RPW = x_rows_per_warp<T>();
    constexpr int AHEAD = 6;                        // fields prefetched to L2 ahead
    constexpr int NPAIR = EVOLVE ? 2 + 3 * NM : 2;  // (dmu_0, dmu_1), (dmu_2), (dPi pairs)
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    const int nt = blockDim.x, rb = nt / T, pk = g.pkx;
    cplx<R> *sb = tw + 2 * L;                       // [2][rb][pkx] the staged input pair
    cplx<R> *xbuf = sb + 2 * (size_t)rb * pk;
    R *rs = reinterpret_cast<R *>(xbuf + rb * xrow_stride<T, E>());   // [rb][RS]: u rows, 3 per row of x
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int nrows = g.ny * g.nz;
    const int row0 = bk.x * rb;
    const int row = row0 + rr;
    const bool rowok = row < nrows;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    const int vrows = max(0, min(rb, nrows - row0));
    const size_t rowbase = (size_t)row * L;
    const int lane = tid & 31, w = tid >> 5, wr0 = w * RPW;
    const int wrows = warp_rows<T>(w, rb, row0, nrows);
    unsigned long long *bar = reinterpret_cast<unsigned long long *>(
                                  smraw + xstaged_body_bytes<R, T, E>(nt, pk, 2, EVOLVE ? NM : 0)) + 2 * w;
    unsigned phase = 0;
    // fields of pair p: (0, 1), (2, -), then (3 + 2q, 4 + 2q)
    auto fields = [&](int p, int &fa, int &fb) {
        if (p == 0) { fa = 0; fb = 1; }
        else if (p == 1) { fa = 2; fb = -1; }
        else { fa = NM + 2 * (p - 2); fb = fa + 1; }
    };
    // the warp's rows of pair p (and with pair 0 its u rows) on their way;
    // the lanes have read the previous pair from the same space (the caller
    // synchronises the warp), hence the proxy fence
    auto stage = [&](int p) {
        if (p >= NPAIR || lane != 0 || wrows == 0) return;
        int fa, fb;
        fields(p, fa, fb);
        const unsigned bytes = (unsigned)(wrows * pk * sizeof(cplx<R>));
        const unsigned ubytes = (unsigned)(L * sizeof(R));
        unsigned total = bytes * (fb >= 0 ? 2u : 1u);
        if (EVOLVE && p == 0) total += NM * wrows * ubytes;
        fence_proxy_async_shared();
        mbar_expect_tx(bar, total);
        const size_t src = (size_t)(row0 + wr0) * pk;
        bulk_load(sb + (size_t)wr0 * pk, a.in[fa] + src, bytes, bar);
        if (fb >= 0) bulk_load(sb + (size_t)(rb + wr0) * pk, a.in[fb] + src, bytes, bar);
        if (EVOLVE && p == 0)
            for (int f = 0; f < NM; ++f)
                for (int j = 0; j < wrows; ++j)
                    bulk_load(rs + (size_t)(wr0 + j) * RS + f * L,
                              pw.u_real + (size_t)f * pw.ncell + (size_t)(row0 + wr0 + j) * L, ubytes, bar);
    };
    if (lane == 0) mbar_init(bar, 1);
    __syncwarp();
    stage(0);
    XPrefetch<R> pf(a, g, row0, vrows, tid == 0);
    pf.upto(AHEAD);
    R dnv[E];
#pragma unroll
    for (int r = 0; r < E; ++r) dnv[r] = rowok ? pw.dn_real[rowbase + block_pos<T, E>(t, r)] : R(0);
    for (int i = tid; i < 2 * L; i += nt) tw[i] = twx[i];
    __syncthreads();
    // the staged pair p into registers, then pair p + 1 on its way
    const R kx0 = R(g.kx0);
    const bool dxs = a.dx_in_pass != 0;
    using B0 = std::integral_constant<int, 0>;   // a pair without its second field
    using B1 = std::integral_constant<int, 1>;
    auto load = [&](int p, cplx<R> (&v)[E], bool dxa, bool dxb, auto bm) {
        constexpr int BM = decltype(bm)::value;
        int fa, fb;
        fields(p, fa, fb);
        if (wrows > 0) {
            warp_stage_wait(bar, phase, pw.status);
            phase ^= 1u;
        }
        x_c2r_load<R, T, E, BAND, BM>(v, sb, BM ? sb + (size_t)rb * pk : nullptr, (size_t)rr * pk, true, t, g.Mx,
                                      dxa, dxb, kx0);
        __syncwarp();
        stage(p + 1);
        pf.upto((fb >= 0 ? fb : fa) + 2 + AHEAD);
    };
    const double nref64 = *pw.nmean;
    const R nref = R(nref64);
    const int y = rowok ? row % g.ny : 0, z = rowok ? row / g.ny : 0;
    // n (dmu - F): pairs of components
#pragma unroll
    for (int q = 0; 2 * q < NM; ++q) {
        const int i0 = 2 * q, i1 = 2 * q + 1;
        cplx<R> v[E];
        if (i1 < NM) load(q, v, dxs && q == 0, false, B1{});   // d/dx of mu
        else load(q, v, false, false, B0{});
        stride_to_block<T, E, +1, R, BarWarp, 1>(v, t, xrow, tw);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int xx = block_pos<T, E>(t, r);
            const R n = nref + dnv[r];
            R f0 = R(0), f1 = R(0);
            if (EXTK == 2) {
                f0 = rowok ? -pw.gradv[(size_t)i0 * pw.ncell + rowbase + xx] : R(0);
                if (i1 < NM) f1 = rowok ? -pw.gradv[(size_t)i1 * pw.ncell + rowbase + xx] : R(0);
            } else if (EXTK == 1) {
                const StageScal &s = pw.ctrl->st[pw.stage];
                cplx<double> e = pw.ex[xx] * pw.ey[y];
                e = e * pw.ez[z];
                e = e * cplx<double>{s.ewr, s.ewi};
                const double sf = s.amp * e.y;
                f0 = R(sf * pw.ph.ext_k[i0]);
                if (i1 < NM) f1 = R(sf * pw.ph.ext_k[i1]);
            }
            v[r] = cplx<R>{n * (v[r].x - f0), n * (v[r].y - f1)};
        }
        if (i1 < NM) x_r2c_pair<R, T, E, BAND, 1, true>(v, a.out[i0], a.out[i1], row, rowok, t, g, xrow, tw);
        else x_r2c_pair<R, T, E, BAND, 0, true>(v, a.out[i0], nullptr, row, rowok, t, g, xrow, tw);
    }
    if (EVOLVE) {
        // -u.grad Pi for component pairs (0,1), (2,3), (4,5)
#pragma unroll 1
        for (int cp = 0; cp < 3; ++cp) {
            cplx<R> acc[E];
#pragma unroll
            for (int r = 0; r < E; ++r) acc[r] = cplx<R>{R(0), R(0)};
#pragma unroll
            for (int d = 0; d < NM; ++d) {
                cplx<R> v[E];
                load(2 + cp * NM + d, v, dxs && d == 0, dxs && d == 0, B1{});   // d/dx of Pi
                stride_to_block<T, E, +1, R, BarWarp, 1>(v, t, xrow, tw);
                const R *urow = rs + (size_t)rr * RS + d * L;
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    // explicit fused multiply-adds: the rounding does not depend
                    // on how the compiler contracts this instantiation
                    const R u = urow[block_pos<T, E>(t, r)];
                    acc[r] = cplx<R>{fma_r(-u, v[r].x, acc[r].x), fma_r(-u, v[r].y, acc[r].y)};
                }
            }
            x_r2c_pair<R, T, E, BAND, 1, true>(acc, a.out[NM + 2 * cp], a.out[NM + 2 * cp + 1], row, rowok, t, g,
                                               xrow, tw);
        }
    }
}

template <typename R, int T, int E, bool EVOLVE, int EXTK, bool BAND>
__global__ void __launch_bounds__(256, xstaged_minb<R, E>()) xb_rows(const __grid_constant__ Grid g, const __grid_constant__ XFastArgs<R> a,
    const cplx<R> *twx, const __grid_constant__ PWB<R> pw)
{
    xb_rows_body<R, T, E, EVOLVE, EXTK, BAND>(hw_block(), g, a, twx, pw);
}

template <typename R, int T, int E, bool EVOLVE, int EXTK, bool BAND>
struct XbRowsPack {
    static constexpr int MAXT = 256, MINB = xstaged_minb<R, E>();
    Grid g;
    XFastArgs<R> a;
    const cplx<R> *tw;
    PWB<R> pw;
    __device__ __forceinline__ void run(const BlockIx &b) const { xb_rows_body<R, T, E, EVOLVE, EXTK, BAND>(b, g, a, tw, pw); }
};



// Real-space I/O: half spectra -> real fields (TOREAL) or back.
template <typename R, int T, int E, bool TOREAL>
__global__ void __launch_bounds__(256) xio_fast(Grid g, XFastArgs<R> a, const cplx<R> *twx, PWToReal<R> dst,
                                                PWFromReal<R> src)
{
    constexpr int L = T * E;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tw = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *xbuf = tw + 2 * L;
    const int nt = blockDim.x, rb = nt / T;
    const int tid = threadIdx.x, t = tid % T, rr = tid / T;
    const int row = blockIdx.x * rb + rr;
    const bool rowok = row < g.ny * g.nz;
    cplx<R> *xrow = xbuf + rr * xrow_stride<T, E>();
    for (int i = tid; i < 2 * L; i += nt) tw[i] = twx[i];
    __syncthreads();
    const size_t rowbase = (size_t)row * g.nx;
    const int nf = TOREAL ? a.nin : a.nout;
    for (int p = 0; 2 * p < nf; ++p) {
        const int fa = 2 * p, fb = 2 * p + 1;
        cplx<R> v[E];
        if (TOREAL) {
            x_c2r_pair<R, T, E>(v, a.in[fa], fb < nf ? a.in[fb] : nullptr, row, rowok, t, g, xrow, tw);
            if (rowok) {
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int xx = block_pos<T, E>(t, r);
                    dst.dst[fa][rowbase + xx] = v[r].x;
                    if (fb < nf) dst.dst[fb][rowbase + xx] = v[r].y;
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int xx = block_pos<T, E>(t, r);
                v[r] = rowok ? cplx<R>{src.src[fa][rowbase + xx], fb < nf ? src.src[fb][rowbase + xx] : R(0)}
                             : cplx<R>{R(0), R(0)};
            }
            x_r2c_pair<R, T, E>(v, a.out[fa], fb < nf ? a.out[fb] : nullptr, row, rowok, t, g, xrow, tw);
        }
    }
}

}  // namespace hydft
