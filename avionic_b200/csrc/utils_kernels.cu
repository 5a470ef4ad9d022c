// Stand-alone stencil, norm and proximal-map kernels behind the utils part of
// the C ABI (reference namespace utils, CUDA/src/utils.cpp).  They share the
// per-pixel stencil code (stencil.cuh) with the fused solver kernels, so the
// reference's derivative and norm known-answer tests exercise the same
// arithmetic the solver runs.
#include "utils_kernels.cuh"
#include "stencil.cuh"

namespace avx {

static __device__ __forceinline__ bool pix_of(long long i, int W, int H, int T, PixCoord& p) {
  const long long HW = (long long)W * H;
  if (i >= HW * T) return false;
  const int t = (int)(i / HW);
  const int r = (int)(i - t * HW);
  p = make_pix(r % W, r / W, t, W, H, T);
  return true;
}

__global__ void gradient_kernel(const float2* u, Ptr18 g, int W, int H, int T, Wts w) {
  PixCoord p;
  if (!pix_of(blockIdx.x * (long long)blockDim.x + threadIdx.x, W, H, T, p)) return;
  float2 r[3];
  grad3(u, p, w, r);
  for (int k = 0; k < 3; ++k) g.p[k][p.i] = r[k];
}

__global__ void divergence_kernel(Ptr18 y, float2* out, int W, int H, int T, Wts w) {
  PixCoord p;
  if (!pix_of(blockIdx.x * (long long)blockDim.x + threadIdx.x, W, H, T, p)) return;
  out[p.i] = div3(y.p[0], y.p[1], y.p[2], p, w);
}

__global__ void symgrad_kernel(Ptr18 v, Ptr18 e, int W, int H, int T, Wts w) {
  PixCoord p;
  if (!pix_of(blockIdx.x * (long long)blockDim.x + threadIdx.x, W, H, T, p)) return;
  float2 r[6];
  symgrad(v.p[0], v.p[1], v.p[2], p, w, r);
  for (int k = 0; k < 6; ++k) e.p[k][p.i] = r[k];
}

__global__ void symdiv_kernel(Ptr18 wv, Ptr18 d, int W, int H, int T, Wts w) {
  PixCoord p;
  if (!pix_of(blockIdx.x * (long long)blockDim.x + threadIdx.x, W, H, T, p)) return;
  float2 r[3];
  symdiv(wv.p, p, w, r);
  for (int k = 0; k < 3; ++k) d.p[k][p.i] = r[k];
}

template <int K>
__global__ void prox_kernel(Ptr18 y, long long N, float scale) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  float2 v[K];
  for (int k = 0; k < K; ++k) v[k] = y.p[k][i];
  float n;
  if (K == 3) {
    n = sqrtf(cabs2(v[0]) + cabs2(v[1]) + cabs2(v[2]));
  } else {
    float s = cabs2(v[0]) + cabs2(v[1]) + cabs2(v[2]);
    for (int k = 3; k < K; ++k) s += 2.f * cabs2(v[k]);
    n = sqrtf(s);
  }
  prox_div<K>(v, n, scale);
  for (int k = 0; k < K; ++k) y.p[k][i] = v[k];
}

template <int K>
__global__ void norm_kernel(Ptr18 g, float* out, long long N) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  float s = 0.f;
  for (int k = 0; k < 3; ++k) s += cabs2(g.p[k][i]);
  for (int k = 3; k < K; ++k) s += 2.f * cabs2(g.p[k][i]);
  out[i] = sqrtf(s);
}

// L1 sums for the regulariser norms: slot 0 = sum |grad u - v|_3,
// slot 1 = sum |E v|_6 (v may be absent: TV norm)
__global__ void regnorm_kernel(const float2* u, const float2* u2, Ptr18 v, int has_v, int W, int H, int T, Wts w,
                               double* partial) {
  __shared__ double red[64];
  double acc[2] = {0.0, 0.0};
  const long long N = (long long)W * H * T;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    PixCoord p;
    pix_of(i, W, H, T, p);
    float2 g[3];
    if (u2)
      grad3_diff(u, u2, p, w, g);
    else
      grad3(u, p, w, g);
    if (has_v) {
      for (int k = 0; k < 3; ++k) g[k] = csub(g[k], ldc(v.p[k], p.i));
      float2 e[6];
      symgrad(v.p[0], v.p[1], v.p[2], p, w, e);
      acc[1] += (double)nrm6(e);
    }
    acc[0] += (double)nrm3(g);
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = acc[0];
    partial[gridDim.x + blockIdx.x] = acc[1];
  }
}

static inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }

void launch_gradient(const float2* u, const Ptr18& g, int W, int H, int T, Wts w, cudaStream_t s) {
  gradient_kernel<<<nblk((long long)W * H * T), 256, 0, s>>>(u, g, W, H, T, w);
}
void launch_divergence(const Ptr18& y, float2* out, int W, int H, int T, Wts w, cudaStream_t s) {
  divergence_kernel<<<nblk((long long)W * H * T), 256, 0, s>>>(y, out, W, H, T, w);
}
void launch_symgrad(const Ptr18& v, const Ptr18& e, int W, int H, int T, Wts w, cudaStream_t s) {
  symgrad_kernel<<<nblk((long long)W * H * T), 256, 0, s>>>(v, e, W, H, T, w);
}
void launch_symdiv(const Ptr18& wv, const Ptr18& d, int W, int H, int T, Wts w, cudaStream_t s) {
  symdiv_kernel<<<nblk((long long)W * H * T), 256, 0, s>>>(wv, d, W, H, T, w);
}
void launch_prox(const Ptr18& y, int K, long long N, float scale, cudaStream_t s) {
  if (K == 3) prox_kernel<3><<<nblk(N), 256, 0, s>>>(y, N, scale);
  else prox_kernel<6><<<nblk(N), 256, 0, s>>>(y, N, scale);
}
void launch_norm(const Ptr18& g, int K, float* out, long long N, cudaStream_t s) {
  if (K == 3) norm_kernel<3><<<nblk(N), 256, 0, s>>>(g, out, N);
  else norm_kernel<6><<<nblk(N), 256, 0, s>>>(g, out, N);
}
void launch_regnorm(const float2* u, const float2* u2, const Ptr18& v, int has_v, int W, int H, int T, Wts w,
                    double* partial, int nblocks, cudaStream_t s) {
  regnorm_kernel<<<nblocks, 256, 0, s>>>(u, u2, v, has_v, W, H, T, w, partial);
}

}  // namespace avx
