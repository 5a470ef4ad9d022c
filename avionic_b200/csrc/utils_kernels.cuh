// Launchers of the stand-alone utils kernels (utils_kernels.cu).
#pragma once

#include "pd_args.cuh"

namespace avx {

struct Ptr18 {
  float2* p[18];
};

void launch_gradient(const float2* u, const Ptr18& g, int W, int H, int T, Wts w, cudaStream_t s);
void launch_divergence(const Ptr18& y, float2* out, int W, int H, int T, Wts w, cudaStream_t s);
void launch_symgrad(const Ptr18& v, const Ptr18& e, int W, int H, int T, Wts w, cudaStream_t s);
void launch_symdiv(const Ptr18& wv, const Ptr18& d, int W, int H, int T, Wts w, cudaStream_t s);
void launch_prox(const Ptr18& y, int K, long long N, float scale, cudaStream_t s);
void launch_norm(const Ptr18& g, int K, float* out, long long N, cudaStream_t s);
void launch_regnorm(const float2* u, const float2* u2, const Ptr18& v, int has_v, int W, int H, int T, Wts w,
                    double* partial, int nblocks, cudaStream_t s);

}  // namespace avx
