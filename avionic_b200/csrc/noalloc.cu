// TV norm without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// result: code running inside a pre-sized memory budget of a scanner
// pipeline, a host-language binding with no CUDA allocator of its own, or a
// process that must not grow its footprint after start-up.  For them,
// avx_tv_norm_noalloc computes utils::TVNorm like avx_tv_norm, but its
// per-block partial sums live in a fixed file-scope __device__ array instead
// of memory obtained from cudaMalloc.
//
// Limits and behaviour:
//  * the array holds AVX_NOALLOC_MAX_BLOCKS partial sums (64 KiB of FP64), one
//    per 256-pixel block, so W*H*T may be at most AVX_NOALLOC_MAX_PIXELS;
//    larger images are rejected with AVX_E_ARG before any launch;
//  * every GPU that loads the library holds the array until process exit;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (the host-side name of a __device__ variable is
//    only a stand-in and must not be passed to a kernel); make that first
//    call before any stream capture.  The address is kept for the life of
//    the process: do not call this entry point after cudaDeviceReset on that
//    device (the reset unloads the module that holds the array);
//  * all calls share the array and it keeps the last call's contents; each
//    call overwrites every slot it later reads, so nothing needs clearing,
//    but calls that overlap on the GPU (different streams or threads) race.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/avionic.h"
#include "stencil.cuh"

#define AVX_NOALLOC_THREADS 256
#define AVX_NOALLOC_MAX_BLOCKS 8192
#define AVX_NOALLOC_MAX_PIXELS (AVX_NOALLOC_THREADS * AVX_NOALLOC_MAX_BLOCKS)

// slots [0, MAX_BLOCKS): block partials; slot MAX_BLOCKS: the final sum
static __device__ __align__(256) double g_noalloc_scratch[AVX_NOALLOC_MAX_BLOCKS + 1];

namespace {

__global__ void __launch_bounds__(AVX_NOALLOC_THREADS)
    tv_norm_partial_kernel(const float2* __restrict__ u, int W, int H, int T, Wts w, double* scratch) {
  __shared__ double red[32];
  const long long HW = (long long)W * H;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  if (i < HW * T) {
    const int t = (int)(i / HW);
    const int r = (int)(i - t * HW);
    const PixCoord p = make_pix(r % W, r / W, t, W, H, T);
    float2 g[3];
    grad3(u, p, w, g);
    acc[0] = (double)nrm3(g);
  }
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) scratch[blockIdx.x] = acc[0];
}

__global__ void __launch_bounds__(AVX_NOALLOC_THREADS) tv_norm_final_kernel(double* scratch, int nblocks) {
  __shared__ double red[32];
  double acc[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc[0] += scratch[b];
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) scratch[AVX_NOALLOC_MAX_BLOCKS] = acc[0];
}

std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {nullptr};  // per device

}  // namespace

// sets the message avx_last_error() returns (core.cu)
void avx_internal_set_error(const char* msg);

static avx_status cuda_fail(const char* what, cudaError_t e) {
  char msg[200];
  std::snprintf(msg, sizeof(msg), "avx_tv_norm_noalloc: %s failed: %s", what, cudaGetErrorString(e));
  avx_internal_set_error(msg);
  return AVX_E_CUDA;
}

extern "C" avx_status avx_tv_norm_noalloc(const avx_cf32* d_u, unsigned W, unsigned H, unsigned T, float dx,
                                          float dy, float dt, double* out) {
  if (!d_u || !out || !W || !H || !T) {
    avx_internal_set_error("avx_tv_norm_noalloc: null pointer or zero dimension");
    return AVX_E_ARG;
  }
  const unsigned long long n = (unsigned long long)W * H * T;
  if (n > (unsigned long long)AVX_NOALLOC_MAX_PIXELS) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "avx_tv_norm_noalloc: %llu pixels exceed the fixed scratch limit of %d pixels", n,
                  AVX_NOALLOC_MAX_PIXELS);
    avx_internal_set_error(msg);
    return AVX_E_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  if (dev < 0 || dev >= 64) {
    avx_internal_set_error("avx_tv_norm_noalloc: device ordinal beyond 63");
    return AVX_E_ARG;
  }
  double* scratch;
  {
    // set-up once per device, with that device current
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress", e);
      if (!p) return cuda_fail("cudaGetSymbolAddress", cudaErrorInvalidSymbol);
      g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_noalloc_addr[dev];
  }
  Wts w;
  w.ix = (float)(1.0 / (double)dx);
  w.iy = (float)(1.0 / (double)dy);
  w.it = (float)(1.0 / (double)dt);
  w.hx = (float)(1.0 / (2.0 * (double)dx));
  w.hy = (float)(1.0 / (2.0 * (double)dy));
  w.ht = (float)(1.0 / (2.0 * (double)dt));
  const int nblocks = (int)((n + AVX_NOALLOC_THREADS - 1) / AVX_NOALLOC_THREADS);
  // an error left pending by an earlier, unrelated call is not this call's failure
  (void)cudaGetLastError();
  tv_norm_partial_kernel<<<nblocks, AVX_NOALLOC_THREADS>>>(reinterpret_cast<const float2*>(d_u), (int)W, (int)H,
                                                          (int)T, w, scratch);
  tv_norm_final_kernel<<<1, AVX_NOALLOC_THREADS>>>(scratch, nblocks);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("kernel launch", e);
  e = cudaMemcpy(out, scratch + AVX_NOALLOC_MAX_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail("cudaMemcpy of the result", e);
  return AVX_OK;
}
