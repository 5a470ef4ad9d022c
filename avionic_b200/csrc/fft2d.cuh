// Batched in-place 2D DFT of complex slices [slice][H][W] (fft2d.cu): one
// pass of row FFTs and one of column FFTs through global memory, each CTA
// transforming 16 lines in shared memory (fft.cuh).  Unnormalised;
// sign -1 is the e^{-2 pi i} kernel, +1 the e^{+2 pi i} kernel.
#pragma once

#include "common.cuh"

struct Fft2dPlan {
  int W, H;
  const float2* twx;  // [W] exp(+2 pi i j / W)
  const float2* twy;  // [H]
  int nradx, radx[12];
  int nrady, rady[12];
};

namespace avx {

size_t fft2d_smem_bytes(int n);
cudaError_t configure_fft2d_kernels();
void launch_fft2d(const Fft2dPlan& p, float2* data, int nslices, int sign, cudaStream_t s);

}  // namespace avx
