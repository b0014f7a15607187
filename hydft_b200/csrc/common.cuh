// Common device types and helpers for the HyDFT B200 solver.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace hydft {

template <typename R>
struct alignas(2 * sizeof(R)) cplx {
    R x, y;
};

template <typename R>
__host__ __device__ __forceinline__ cplx<R> mk(R a, R b) { return cplx<R>{a, b}; }
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator+(cplx<R> a, cplx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator-(cplx<R> a, cplx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator*(cplx<R> a, cplx<R> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R>
__host__ __device__ __forceinline__ cplx<R> operator*(R s, cplx<R> a) { return {s * a.x, s * a.y}; }
template <typename R>
__host__ __device__ __forceinline__ cplx<R> conj(cplx<R> a) { return {a.x, -a.y}; }
// multiply by +i (DIR=+1) or -i (DIR=-1)
template <int DIR, typename R>
__host__ __device__ __forceinline__ cplx<R> mul_i(cplx<R> a)
{
    return DIR > 0 ? cplx<R>{-a.y, a.x} : cplx<R>{a.y, -a.x};
}
// i*k*a with real k: (0 + i k)(a.x + i a.y) = (-k a.y, k a.x)
template <typename R>
__host__ __device__ __forceinline__ cplx<R> ik_times(R k, cplx<R> a) { return {-k * a.y, k * a.x}; }

// status bits written by kernels (plain stores of OR-ed flags)
enum : unsigned {
    ST_NONPOS = 1u,       // density <= 0 (model.f90:91)
    ST_NONFINITE = 2u,    // NaN / Inf in the state
    ST_NEWTON = 4u,       // Fermi-Dirac inverse did not converge
    ST_TIMEOUT = 8u,
};

// Largest FFT length along one axis and the radix plan.
constexpr int MAX_L = 512;
constexpr int MAX_RAD = 12;

struct FFTPlan {
    int L;
    int nrad;
    int rad[MAX_RAD];
};

// Grid description shared by all kernels of one simulation.
// Compact spectral arrays hold the dealiased band only:
//   kx index c in [0, Mx]                (signed m = c)
//   ky index c in [0, 2My]  (c <= My: m = c, else m = c - (2My+1))
//   kz index c in [0, 2Mz]
// stored [kzc][kyc][kxc] with the kx run padded to pkx elements.
struct Grid {
    int nx, ny, nz, ndim;
    int Mx, My, Mz;
    int nkxc, nkyc, nkzc, pkx;
    double kx0, ky0, kz0;   // 2 pi / L per axis (0 on a collapsed axis)
    double dx, dy, dz;
    FFTPlan px, py, pz;
};

__host__ __device__ __forceinline__ int signed_idx(int c, int M) { return c <= M ? c : c - (2 * M + 1); }
__host__ __device__ __forceinline__ int fft_idx(int m, int n) { return m >= 0 ? m : m + n; }

// Block coordinates and grid extent of one simulation's share of a launch.
// A plain launch uses the hardware's.  An ensemble launch runs one kernel
// for many simulations of the same shape: their grids are stacked along z,
// and each block finds its simulation and its coordinates in that
// simulation's grid (ensemble_kernel below).
struct BlockIx {
    unsigned x, y, z;
    unsigned gx, gy, gz;
};

__device__ __forceinline__ BlockIx hw_block()
{
    return BlockIx{blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y, gridDim.z};
}

// The ensemble form of a kernel.  P (a "pack") holds one simulation's
// launch arguments and runs the kernel body for one block of that
// simulation's grid.  The packs of up to PackSet<P>::N simulations travel as
// one kernel parameter (__grid_constant__, under the 32 KB parameter limit),
// set.p[m] being simulation m's, and zper is the z extent of one
// simulation's grid, so block z = m zper + z'.  The body then reads its
// arguments from the parameter space, which is read-only and which no
// global store can alias, with a block-uniform index (no per-block copy, no
// table in device memory).  A model on its own runs the same kernel with one
// pack.
template <class P>
struct PackSet {
    static constexpr int FIT = (int)(30720 / sizeof(P));
    static constexpr int N = FIT < 1 ? 1 : (FIT > 64 ? 64 : FIT);
    P p[N];
};

template <class P>
__global__ void __launch_bounds__(P::MAXT, P::MINB) ensemble_kernel(const __grid_constant__ PackSet<P> set, unsigned zper)
{
    static_assert(sizeof(PackSet<P>) <= 32000, "kernel parameters are limited to 32 KB");
    const unsigned m = blockIdx.z / zper;
    const BlockIx b{blockIdx.x, blockIdx.y, blockIdx.z - m * zper, gridDim.x, gridDim.y, zper};
    set.p[m].run(b);
}

}  // namespace hydft
