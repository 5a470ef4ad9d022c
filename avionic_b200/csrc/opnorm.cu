// K^H K of the primal-dual operators, for the power-iteration estimate of
// their norm (getopnorm, matlab/getopnorm.m:1-17).
//
// K is the linear map of a method's dual update, K x = (K_reg x, A x), and
// K^H is the map of its primal update, x <- x - tau K^H (y, z) (tv.cpp:137-198,
// tgv2.cpp:234-335, ictgv2.cpp:334-490, tv_temp.cpp:94-182, ictv.cpp:227-370):
//   TV      K_reg u = grad_w u                              K_reg^H y = -div_w y
//   TVtemp  K_reg u = D+_t u / dt                           K_reg^H y = -div_t y
//   TGV2    K_reg (u, v) = (grad u - v, E v)                K_reg^H (p, q) = (-div p, -(p + div_sym q))
//   ICTV    K_reg (u, w) = (grad_1 (u - w), grad_2 w)       K_reg^H (p, r) = (-div_1 p, div_1 p - div_2 r)
//   ICTGV2  K_reg (u, v, w, s) = (grad_1 (u - w) - v, E_1 v, grad_2 w - s, E_2 s)
//           K_reg^H (p, q, r, o) = (-div_1 p, -(p + div_sym1 q), div_1 p - div_2 r, -(r + div_sym2 o))
// with the off-diagonal entries of the symmetrised gradient counted twice in
// the dual inner product, as the step rule counts them (utils.cpp SumOfSquares6).
// The encoding part A^H A x[0] is applied by the operator's own kernels and
// arrives as an image.  One kernel forms K_reg x, a second forms K^H K x and
// its FP64 block sums of |y|^2 and y^H x; a one-block kernel adds the sums.
#include "opnorm.cuh"
#include "stencil.cuh"

namespace avx {

template <int M>
__global__ void __launch_bounds__(256) opn_dual_kernel(OpnArgs a) {
  const long long HW = (long long)a.W * a.H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / HW);
    const int r = (int)(i - t * HW);
    const PixCoord p = make_pix(r % a.W, r / a.W, t, a.W, a.H, a.T);
    if (M == AVX_M_TV) {
      float2 g[3];
      grad3(a.x[0], p, a.w1, g);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.d[k][i] = g[k];
    } else if (M == AVX_M_TVTEMP) {
      a.d[0][i] = tgrad(a.x[0], p, a.w1);
    } else if (M == AVX_M_ICTV) {
      float2 g[3];
      grad3_diff(a.x[0], a.x[1], p, a.w1, g);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.d[k][i] = g[k];
      grad3(a.x[1], p, a.w2, g);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.d[3 + k][i] = g[k];
    } else if (M == AVX_M_TGV2 || M == AVX_M_ICTGV2) {
      float2 g[3], e[6];
      if (M == AVX_M_TGV2)
        grad3(a.x[0], p, a.w1, g);
      else
        grad3_diff(a.x[0], a.x[4], p, a.w1, g);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.d[k][i] = csub(g[k], ldc(a.x[1 + k], i));
      symgrad(a.x[1], a.x[2], a.x[3], p, a.w1, e);
#pragma unroll
      for (int k = 0; k < 6; ++k) a.d[3 + k][i] = e[k];
      if (M == AVX_M_ICTGV2) {
        grad3(a.x[4], p, a.w2, g);
#pragma unroll
        for (int k = 0; k < 3; ++k) a.d[9 + k][i] = csub(g[k], ldc(a.x[5 + k], i));
        symgrad(a.x[5], a.x[6], a.x[7], p, a.w2, e);
#pragma unroll
        for (int k = 0; k < 6; ++k) a.d[12 + k][i] = e[k];
      }
    }
  }
}

AVX_D void opn_acc(double (&acc)[3], float2 y, float2 x) {
  acc[0] += (double)y.x * y.x + (double)y.y * y.y;
  // y^H x = sum conj(y) x
  acc[1] += (double)y.x * x.x + (double)y.y * x.y;
  acc[2] += (double)y.x * x.y - (double)y.y * x.x;
}

template <int M>
__global__ void __launch_bounds__(256) opn_primal_kernel(OpnArgs a) {
  __shared__ double red[32 * 3];
  double acc[3] = {0.0, 0.0, 0.0};
  const long long HW = (long long)a.W * a.H;
  float2* const* d = a.d;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / HW);
    const int r = (int)(i - t * HW);
    const PixCoord p = make_pix(r % a.W, r / a.W, t, a.W, a.H, a.T);
    float2 y0 = a.khk[i];
    if (M == AVX_M_TV) {
      y0 = csub(y0, div3(d[0], d[1], d[2], p, a.w1));
    } else if (M == AVX_M_TVTEMP) {
      y0 = csub(y0, tdiv(d[0], p, a.w1));
    } else if (M == AVX_M_ICTV) {
      const float2 div1 = div3(d[0], d[1], d[2], p, a.w1);
      y0 = csub(y0, div1);
      const float2 y1 = csub(div1, div3(d[3], d[4], d[5], p, a.w2));
      a.y[1][i] = y1;
      opn_acc(acc, y1, a.x[1][i]);
    } else if (M == AVX_M_TGV2 || M == AVX_M_ICTGV2) {
      const float2 div1 = div3(d[0], d[1], d[2], p, a.w1);
      y0 = csub(y0, div1);
      float2 sd[3];
      symdiv(d + 3, p, a.w1, sd);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float2 v = ldc(d[k], i);
        const float2 yk = make_float2(-(v.x + sd[k].x), -(v.y + sd[k].y));
        a.y[1 + k][i] = yk;
        opn_acc(acc, yk, a.x[1 + k][i]);
      }
      if (M == AVX_M_ICTGV2) {
        const float2 y4 = csub(div1, div3(d[9], d[10], d[11], p, a.w2));
        a.y[4][i] = y4;
        opn_acc(acc, y4, a.x[4][i]);
        symdiv(d + 12, p, a.w2, sd);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float2 v = ldc(d[9 + k], i);
          const float2 yk = make_float2(-(v.x + sd[k].x), -(v.y + sd[k].y));
          a.y[5 + k][i] = yk;
          opn_acc(acc, yk, a.x[5 + k][i]);
        }
      }
    }
    a.y[0][i] = y0;
    opn_acc(acc, y0, a.x[0][i]);
  }
  block_sum<3>(acc, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < 3; ++s) a.partial[s * gridDim.x + blockIdx.x] = acc[s];
  }
}

__global__ void opn_finalize_kernel(const double* partial, int nb, double* out) {
  __shared__ double red[32 * 3];
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
#pragma unroll
    for (int s = 0; s < 3; ++s) v[s] += partial[s * nb + i];
  }
  block_sum<3>(v, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < 3; ++s) out[s] = v[s];
  }
}

struct OpnPtrs {
  float2* x[8];
  const float2* y[8];
};

// x = y / ||y|| in FP64, rounded once to fp32 (getopnorm.m:7-11)
__global__ void __launch_bounds__(256) opn_normalise_kernel(OpnPtrs q, int P, long long N, const double* ss) {
  const double s = ss[0];
  const double inv = s != 0.0 ? 1.0 / sqrt(s) : 1.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < P; ++c) {
      const float2 v = q.y[c][i];
      q.x[c][i] = make_float2((float)((double)v.x * inv), (float)((double)v.y * inv));
    }
  }
}

void launch_opn_dual(int method, const OpnArgs& a, cudaStream_t s) {
  if (method == AVX_M_TV) opn_dual_kernel<AVX_M_TV><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_TVTEMP) opn_dual_kernel<AVX_M_TVTEMP><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_TGV2) opn_dual_kernel<AVX_M_TGV2><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_ICTV) opn_dual_kernel<AVX_M_ICTV><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_ICTGV2) opn_dual_kernel<AVX_M_ICTGV2><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
}

void launch_opn_primal(int method, const OpnArgs& a, cudaStream_t s) {
  if (method == AVX_M_TV) opn_primal_kernel<AVX_M_TV><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_TVTEMP) opn_primal_kernel<AVX_M_TVTEMP><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_TGV2) opn_primal_kernel<AVX_M_TGV2><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_ICTV) opn_primal_kernel<AVX_M_ICTV><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else if (method == AVX_M_ICTGV2) opn_primal_kernel<AVX_M_ICTGV2><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
  else opn_primal_kernel<AVX_M_ENCODING><<<AVX_RED_BLOCKS, 256, 0, s>>>(a);
}

void launch_opn_finalize(const double* partial, double* out, cudaStream_t s) {
  opn_finalize_kernel<<<1, 256, 0, s>>>(partial, AVX_RED_BLOCKS, out);
}

void launch_opn_normalise(const OpnArgs& a, int P, float2* const* x, const double* ss, cudaStream_t s) {
  OpnPtrs q;
  for (int c = 0; c < 8; ++c) {
    q.x[c] = c < P ? x[c] : nullptr;
    q.y[c] = c < P ? a.y[c] : nullptr;
  }
  opn_normalise_kernel<<<AVX_RED_BLOCKS, 256, 0, s>>>(q, P, a.N, ss);
}

}  // namespace avx
