// Power-iteration estimate of a primal-dual operator's norm (getopnorm,
// matlab/getopnorm.m:1-17): the kernels that apply K^H K with FP64
// reductions of the iterate.
#pragma once

#include "pd_args.cuh"

// Method id of the encoding operator alone (no regularisation part).
#define AVX_M_ENCODING (-1)

namespace avx {

struct OpnArgs {
  int W, H, T;
  long long N;
  const float2* x[8];  // primal components of the iterate
  float2* y[8];        // K^H K x, primal components
  float2* d[18];       // K_reg x, dual components (layout of the solver's dual fields)
  const float2* khk;   // A^H A x[0] (encoding operator)
  Wts w1, w2;          // branch weights, as the solver's
  double* partial;     // [3][AVX_RED_BLOCKS]: |y|^2, Re y^H x, Im y^H x
};

// d = K_reg x (the linear part of the method's dual update)
void launch_opn_dual(int method, const OpnArgs& a, cudaStream_t s);
// y = K_reg^H d + (A^H A x[0] on component 0), with the block partial sums
void launch_opn_primal(int method, const OpnArgs& a, cudaStream_t s);
// out[0..2] = the sums of the partials
void launch_opn_finalize(const double* partial, double* out, cudaStream_t s);
// x_c = y_c / sqrt(ss[0]) for every component (x = y when ss[0] == 0)
void launch_opn_normalise(const OpnArgs& a, int P, float2* const* x, const double* ss, cudaStream_t s);

}  // namespace avx
