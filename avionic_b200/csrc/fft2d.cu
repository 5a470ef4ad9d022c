#include "fft.cuh"
#include "fft2d.cuh"

namespace avx {

#define FFT2D_KC 16

__global__ void __launch_bounds__(256) fft2d_rows_kernel(Fft2dPlan p, float2* data, int sign) {
  constexpr int KC = FFT2D_KC, KCP = AVX_FFT_PITCH(KC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int G = p.W;
  float2* A = reinterpret_cast<float2*>(smem_raw);
  float2* B = A + (size_t)G * KCP;
  float2* tw = B + (size_t)G * KCP;
  const int r0 = blockIdx.x * KC;
  const int rows = min(KC, p.H - r0);
  float2* base = data + (long long)blockIdx.y * p.W * p.H;
  __shared__ int splan[12];
  stage_plan(p.radx, splan);
  for (int j = threadIdx.x; j < G; j += blockDim.x) tw[j] = p.twx[j];
  for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
    const int kk = e / G, x = e % G;
    A[x * KCP + kk] = kk < rows ? base[(long long)(r0 + kk) * G + x] : czero();
  }
  __syncthreads();
  const float2* R = row_fft<KC>(A, B, tw, G, p.nradx, splan, sign);
  for (int e = threadIdx.x; e < rows * G; e += blockDim.x) {
    const int kk = e / G, x = e % G;
    base[(long long)(r0 + kk) * G + x] = R[x * KCP + kk];
  }
}

__global__ void __launch_bounds__(256) fft2d_cols_kernel(Fft2dPlan p, float2* data, int sign) {
  constexpr int KC = FFT2D_KC, KCP = AVX_FFT_PITCH(KC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int G = p.H;
  float2* A = reinterpret_cast<float2*>(smem_raw);
  float2* B = A + (size_t)G * KCP;
  float2* tw = B + (size_t)G * KCP;
  const int c0 = blockIdx.x * KC;
  const int cols = min(KC, p.W - c0);
  float2* base = data + (long long)blockIdx.y * p.W * p.H;
  __shared__ int splan[12];
  stage_plan(p.rady, splan);
  for (int j = threadIdx.x; j < G; j += blockDim.x) tw[j] = p.twy[j];
  for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
    const int kk = e % KC, y = e / KC;
    A[y * KCP + kk] = kk < cols ? base[(long long)y * p.W + c0 + kk] : czero();
  }
  __syncthreads();
  const float2* R = row_fft<KC>(A, B, tw, G, p.nrady, splan, sign);
  for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
    const int kk = e % KC, y = e / KC;
    if (kk < cols) base[(long long)y * p.W + c0 + kk] = R[y * KCP + kk];
  }
}

size_t fft2d_smem_bytes(int n) { return sizeof(float2) * (2 * (size_t)n * AVX_FFT_PITCH(FFT2D_KC) + n); }

cudaError_t configure_fft2d_kernels() {
  cudaError_t e = cudaFuncSetAttribute(fft2d_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fft2d_cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);
}

void launch_fft2d(const Fft2dPlan& p, float2* data, int nslices, int sign, cudaStream_t s) {
  dim3 gr((p.H + FFT2D_KC - 1) / FFT2D_KC, nslices);
  fft2d_rows_kernel<<<gr, 256, fft2d_smem_bytes(p.W), s>>>(p, data, sign);
  dim3 gc((p.W + FFT2D_KC - 1) / FFT2D_KC, nslices);
  fft2d_cols_kernel<<<gc, 256, fft2d_smem_bytes(p.H), s>>>(p, data, sign);
}

}  // namespace avx
