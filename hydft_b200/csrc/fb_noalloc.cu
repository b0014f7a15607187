// Allocation-free Fourier-Bessel transform.
//
// hydft_gpu_fourier_bessel allocates device buffers for its input, output
// and tables on every call.  Some callers cannot allocate device memory at
// the point where they need the transform: code running inside a region
// where device allocation is not allowed or would be too slow (a solver
// loop that must not synchronise the device, a host that reserved all
// device memory up front for its own pool, a plugin whose host framework
// owns every allocation).  hydft_gpu_fourier_bessel_noalloc serves them: the
// caller passes device input and output arrays, and the tables the
// transform needs (the sine table and the radial weights) live in a fixed
// scratch array compiled into the library.
//
// The scratch array holds 2(n+1) + 2n doubles for n up to
// HYDFT_FB_NOALLOC_MAX_N = 8192, 262 160 bytes, and every GPU that loads
// the library keeps it until the process exits.  Each call rebuilds the
// tables for its own n and rmax before transforming, so calls do not depend
// on one another's contents; two calls whose work overlaps on the GPU (on
// different streams, or from different host threads) share the array and
// race.  The input and output arrays must not overlap: every block reads
// the whole input while other blocks write their outputs.
//
// Every call looks up the array's device address in the current context
// (cudaGetSymbolAddress, which allocates nothing) and sets the transform
// kernel's shared-memory limit, so a reset device or a new context never
// sees a stale address.  The first call on a device also loads the
// library's kernels into that context; make that first call before any
// stream capture.  A NULL stream is the calling thread's per-thread default
// stream (the library is compiled with --default-stream per-thread).
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/hydft_gpu.h"

namespace hydft {
void set_thread_error(const std::string &msg);
}

namespace {

constexpr int FB_MAX_N = HYDFT_FB_NOALLOC_MAX_N;
constexpr size_t FB_SCRATCH = 2 * ((size_t)FB_MAX_N + 1) + 2 * (size_t)FB_MAX_N;

// the transform's scratch: sine table, then the input weights, then the
// output weights
static __device__ __align__(256) double fb_scratch[FB_SCRATCH];

// sin(pi m/(n+1)) for m < 2(n+1); the weights of direction 0 (r2k: r_j in,
// 2 pi dr/k_j out) or 1 (k2r: k_j in, dk/(4 pi^2 r_j) out)
__global__ void fb_tables_kernel(double *scr, int n, double rmax, int direction)
{
    const double pi = 3.14159265358979323846264338327950288;
    const int M = 2 * (n + 1);
    double *pre = scr + M, *post = pre + n;
    const double dr = rmax / (n + 1), dk = pi / ((n + 1) * dr);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        scr[m] = sinpi((double)m / (double)(n + 1));
        if (m < n) {
            const double r = (m + 1) * dr, k = (m + 1) * dk;
            pre[m] = direction == 0 ? r : k;
            post[m] = direction == 0 ? 2.0 * pi * dr / k : dk / (4.0 * pi * pi * r);
        }
    }
}

// out_k = post_k 2 sum_j pre_j x_j sin(pi (j+1)(k+1)/(n+1)), the integer
// phase (j+1)(k+1) mod 2(n+1) advancing by k+1 per term
__global__ void fb_dst_kernel(const double *__restrict__ x, double *__restrict__ out, int n, const double *scr)
{
    extern __shared__ double sm[];
    const int M = 2 * (n + 1);
    const double *pre = scr + M, *post = pre + n;
    double *st = sm, *xs = sm + M;
    for (int m = threadIdx.x; m < M; m += blockDim.x) st[m] = scr[m];
    for (int j = threadIdx.x; j < n; j += blockDim.x) xs[j] = pre[j] * x[j];
    __syncthreads();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int step = k + 1;
    int ph = step;
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

// with the device current: the scratch array's device address in the
// current context and the shared-memory limit of the transform kernel
int setup_context(double **ptr)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, fb_scratch);
    if (e != cudaSuccess || !p) {
        hydft::set_thread_error(std::string("fourier_bessel_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return HYDFT_ERR_CUDA;
    }
    const int smax = (int)(sizeof(double) * (2 * ((size_t)FB_MAX_N + 1) + FB_MAX_N));
    e = cudaFuncSetAttribute(fb_dst_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
    if (e != cudaSuccess) {
        hydft::set_thread_error(std::string("fourier_bessel_noalloc: cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        return HYDFT_ERR_CUDA;
    }
    *ptr = static_cast<double *>(p);
    return HYDFT_OK;
}

}  // namespace

extern "C" int hydft_gpu_fourier_bessel_noalloc(const double *d_in, double *d_out, int n, double rmax,
                                                int direction, void *stream)
{
    if (!d_in || !d_out || !(rmax > 0.0) || (direction != 0 && direction != 1)) {
        hydft::set_thread_error("fourier_bessel_noalloc: bad arguments");
        return HYDFT_ERR_BAD_ARG;
    }
    if (n < 1 || n > FB_MAX_N) {
        hydft::set_thread_error("fourier_bessel_noalloc: n = " + std::to_string(n) + " is outside 1.." +
                                std::to_string(FB_MAX_N) + ", the size of the fixed scratch array");
        return HYDFT_ERR_BAD_ARG;
    }
    const uintptr_t a0 = reinterpret_cast<uintptr_t>(d_in), b0 = reinterpret_cast<uintptr_t>(d_out);
    const uintptr_t bytes = sizeof(double) * (uintptr_t)n;
    if (a0 < b0 + bytes && b0 < a0 + bytes) {
        hydft::set_thread_error("fourier_bessel_noalloc: the input and output arrays overlap");
        return HYDFT_ERR_BAD_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        hydft::set_thread_error("fourier_bessel_noalloc: no usable current CUDA device");
        return HYDFT_ERR_CUDA;
    }
    double *scr = nullptr;
    if (int rc = setup_context(&scr)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int M = 2 * (n + 1);
    fb_tables_kernel<<<(M + 255) / 256, 256, 0, st>>>(scr, n, rmax, direction);
    const size_t smem = sizeof(double) * ((size_t)M + n);
    fb_dst_kernel<<<(n + 127) / 128, 128, smem, st>>>(d_in, d_out, n, scr);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        hydft::set_thread_error(std::string("fourier_bessel_noalloc: launch: ") + cudaGetErrorString(e));
        return HYDFT_ERR_CUDA;
    }
    return HYDFT_OK;
}
