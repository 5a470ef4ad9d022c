// Shared device types and helpers for the AVIONIC B200 reconstruction core.
//
// complex64 is carried as float2 (re, im), the memory layout of
// std::complex<float> that the reference's CVector uses (CUDA/include/types.h:16-19).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define AVX_HD __host__ __device__ __forceinline__
#define AVX_D __device__ __forceinline__

// Dynamic shared memory a kernel may request: the 227 KB a CTA can hold on
// sm_100, less 1 KB for the small static __shared__ arrays some kernels add.
#define AVX_DYN_SMEM_MAX (227 * 1024 - 1024)

AVX_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
AVX_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
AVX_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
AVX_HD float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
AVX_HD float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// acc += a * b
AVX_HD void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
  acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
}
AVX_HD float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
AVX_HD float2 czero() { return make_float2(0.f, 0.f); }

// Reconstruction methods, numbered as the reference's Method enum
// (CUDA/include/options_parser.h: TV, TVtemp, TGV2, TGV2_3D, ICTV, ICTGV2, ...).
enum : int { AVX_M_TV = 0, AVX_M_TVTEMP = 1, AVX_M_TGV2 = 2, AVX_M_ICTV = 4, AVX_M_ICTGV2 = 5 };

template <int M>
struct MethodDims;
template <>
struct MethodDims<AVX_M_TV> {
  static constexpr int P = 1, D = 3;
};
template <>
struct MethodDims<AVX_M_TVTEMP> {
  static constexpr int P = 1, D = 1;
};
template <>
struct MethodDims<AVX_M_ICTV> {
  static constexpr int P = 2, D = 6;
};
template <>
struct MethodDims<AVX_M_TGV2> {
  static constexpr int P = 4, D = 9;
};
template <>
struct MethodDims<AVX_M_ICTGV2> {
  static constexpr int P = 8, D = 18;
};

// Device-resident solver scalars.  The step rule and the gap test run on the
// device so that an iteration never waits on the host.
struct DevState {
  double sigma, tau;      // current primal/dual step sizes
  double nKx2, nx2;       // last step-rule norms (squared)
  double gap;             // last normalised gap
  int stop;               // 1 once gap/N < stopPDGap
  int ngap;               // records written to the gap history
  int iters;              // iterations started (dual_kernel increments it)
  int err;                // non-zero when a device-side check failed
  double d_off;           // energy of the data outside the sampled rows (gap constant)
  double gap0;            // first normalised gap of the run (relative stop criterion)
};

// Number of FP64 partial-sum slots a reduction writes per block.
#define AVX_RED_SLOTS 12
#define AVX_RED_BLOCKS 592  // 4 x 148 SMs

// Block-wide sum of NS doubles; results valid in thread 0.
template <int NS>
AVX_D void block_sum(double (&v)[NS], double* smem /* >= 32*NS */) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31;
  const int wid = tid >> 5;
  const int nw = (nthr + 31) >> 5;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double a = v[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) smem[s * 32 + wid] = a;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      double a = lane < nw ? smem[s * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      v[s] = a;
    }
  }
  __syncthreads();
}
