// Coil-sensitivity estimation kernels (coils.cu).
#pragma once

#include "common.cuh"

// State of one 2D primal-dual loop (UTGV2Recon or B1Recon); updates are in place.
struct CoilPD {
  int W, H;
  float sigma, tau;
  float s1, s2;           // prox scales 1/(alpha1 nu), 1/(alpha0 nu) (UTGV2)
  float mu;               // H1 weight (B1Recon)
  float2* x1;
  float2* ext1;
  float2* x1n;            // where the new x1 goes (may equal x1)
  float2* ext1n;          // where the new extragradient goes (may equal ext1)
  float2* x2[2];
  float2* ext2[2];
  float2* ext2n[2];
  float2* y1[2];
  float2* y2[3];
  const float2* Lw;
  const float2* Ib;
};

// double-buffered extragradient and duals of one fused B1Recon iteration
struct B1Buffers {
  const float2* ext_in;
  float2* ext_out;
  const float2* y0_in;
  const float2* y1_in;
  float2* y0_out;
  float2* y1_out;
};

// double-buffered extragradients and duals of one fused UTGV2Recon iteration
struct UtgvBuffers {
  const float2* ext1_in;
  float2* ext1_out;
  const float2* ext2_in[2];
  float2* ext2_out[2];
  const float2* y1_in[2];
  float2* y1_out[2];
  const float2* y2_in[3];
  float2* y2_out[3];
};

namespace avx {

void launch_ta_sum(const float2* kdata, const float* mask, float2* out, int HW, int C, int T, cudaStream_t s);
void launch_ta_combine(float2* crec, float2* u, int HW, int C, float scale, int apply_phase, cudaStream_t s);
void launch_h1_cg(const float2* u, const float2* crec, double mu, int W, int H, int C, int max_it, double rel_tol,
                  double2* work, double* muu, float2* out, int* iters, cudaStream_t s);
void launch_h1_normalize(float2* b1, int HW, int C, cudaStream_t s);
void launch_utgv_prep(const float2* b10, const float2* crec0, const int* inds, int ninds, float tau, int HW,
                      float2* Lw, float2* Ib, cudaStream_t s);
void launch_utgv_fused(const CoilPD& a, const UtgvBuffers& b, cudaStream_t s);
void launch_absmax(const float2* v, int n, unsigned* out, cudaStream_t s);
void launch_b1r_prep(const float2* u0, const unsigned* umax, const float2* crec, int coils, int HW, float tau,
                     float2* Lw, float2* Iu, cudaStream_t s);
void launch_b1r_fused(const CoilPD& a, int coils, const B1Buffers& b, cudaStream_t s);
void launch_b1r_normalize(const float2* x, float2* out, int HW, int coils, cudaStream_t s);
void launch_phase_apply(const float2* absb1, const float2* x1, float2* out, int HW, cudaStream_t s);
void launch_weight_update(float2* w, const float2* b, int HW, cudaStream_t s);
void launch_greedy_inputs(const float2* absb1, const float2* u, const float2* w, const float2* crec, float2* u_in,
                          float2* crec_in, int HW, cudaStream_t s);
void launch_cscale(float2* v, long long n, float f, cudaStream_t s);
void launch_abs_sum(const float2* a, const float2* b, int HW, double* partial, int nblocks, cudaStream_t s);

}  // namespace avx
