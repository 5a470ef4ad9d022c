// Finite-difference stencils of the reference's AGILE kernels, per pixel.
//
// Boundary semantics (pinned by CUDA/test/derivatives.cc:169-650):
//   D+  (diff3, no wrap):   (D+u)_i = u_{i+1} - u_i, 0 at the last index
//   D-  (bdiff3, no wrap):  -(D+)^T: u_0 at 0, u_i - u_{i-1} inside, -u_{n-2} last
//   (D+)^T (diff3trans):    u_{i-1} [i>0] - u_i [i<n-1]
//   (D-)^T (bdiff3trans):   -D+
// Each helper takes the pixel's linear index i, its coordinate c along the
// difference direction, the extent n and the stride s of that direction.
#pragma once

#include "pd_args.cuh"

AVX_D float2 ldc(const float2* __restrict__ u, long long i) { return __ldg(u + i); }

AVX_D float2 d_fwd(const float2* __restrict__ u, long long i, int c, int n, long long s) {
  return (c < n - 1) ? csub(ldc(u, i + s), ldc(u, i)) : czero();
}
// D+ of (u - v), formed as the reference forms it (difference first).
AVX_D float2 d_fwd2(const float2* __restrict__ u, const float2* __restrict__ v, long long i,
                    int c, int n, long long s) {
  if (c >= n - 1) return czero();
  float2 a = csub(ldc(u, i + s), ldc(v, i + s));
  float2 b = csub(ldc(u, i), ldc(v, i));
  return csub(a, b);
}
AVX_D float2 d_bwd(const float2* __restrict__ u, long long i, int c, int n, long long s) {
  float2 a = (c < n - 1) ? ldc(u, i) : czero();
  float2 b = (c > 0) ? ldc(u, i - s) : czero();
  return csub(a, b);
}
AVX_D float2 d_fwd_t(const float2* __restrict__ u, long long i, int c, int n, long long s) {
  float2 a = (c > 0) ? ldc(u, i - s) : czero();
  float2 b = (c < n - 1) ? ldc(u, i) : czero();
  return csub(a, b);
}
AVX_D float2 d_bwd_t(const float2* __restrict__ u, long long i, int c, int n, long long s) {
  return (c < n - 1) ? csub(ldc(u, i), ldc(u, i + s)) : czero();
}

struct PixCoord {
  int x, y, t, W, H, T;
  long long i, sW, sWH;
};

AVX_D PixCoord make_pix(int x, int y, int t, int W, int H, int T) {
  PixCoord p;
  p.x = x; p.y = y; p.t = t; p.W = W; p.H = H; p.T = T;
  p.sW = W;
  p.sWH = (long long)W * H;
  p.i = x + p.sW * y + p.sWH * t;
  return p;
}

// utils::Gradient (utils.cpp:99-118)
AVX_D void grad3(const float2* u, const PixCoord& p, const Wts& w, float2 (&g)[3]) {
  g[0] = cscale(d_fwd(u, p.i, p.x, p.W, 1), w.ix);
  g[1] = cscale(d_fwd(u, p.i, p.y, p.H, p.sW), w.iy);
  g[2] = cscale(d_fwd(u, p.i, p.t, p.T, p.sWH), w.it);
}
AVX_D void grad3_diff(const float2* u, const float2* v, const PixCoord& p, const Wts& w,
                      float2 (&g)[3]) {
  g[0] = cscale(d_fwd2(u, v, p.i, p.x, p.W, 1), w.ix);
  g[1] = cscale(d_fwd2(u, v, p.i, p.y, p.H, p.sW), w.iy);
  g[2] = cscale(d_fwd2(u, v, p.i, p.t, p.T, p.sWH), w.it);
}

// utils::SymmetricGradient, 7-argument form (utils.cpp:397-456).  The yt
// entry scales its y-difference by 1/(2 dx), as the reference does (:453).
AVX_D void symgrad(const float2* v0, const float2* v1, const float2* v2, const PixCoord& p,
                   const Wts& w, float2 (&e)[6]) {
  e[0] = cscale(d_bwd(v0, p.i, p.x, p.W, 1), w.ix);
  e[1] = cscale(d_bwd(v1, p.i, p.y, p.H, p.sW), w.iy);
  e[2] = cscale(d_bwd(v2, p.i, p.t, p.T, p.sWH), w.it);
  e[3] = cadd(cscale(d_bwd(v0, p.i, p.y, p.H, p.sW), w.hy), cscale(d_bwd(v1, p.i, p.x, p.W, 1), w.hx));
  e[4] = cadd(cscale(d_bwd(v0, p.i, p.t, p.T, p.sWH), w.ht), cscale(d_bwd(v2, p.i, p.x, p.W, 1), w.hx));
  e[5] = cadd(cscale(d_bwd(v1, p.i, p.t, p.T, p.sWH), w.ht), cscale(d_bwd(v2, p.i, p.y, p.H, p.sW), w.hx));
}

// utils::Divergence (utils.cpp:733-757) = -grad^T y
AVX_D float2 div3(const float2* y0, const float2* y1, const float2* y2, const PixCoord& p,
                  const Wts& w) {
  float2 a = cscale(d_fwd_t(y0, p.i, p.x, p.W, 1), w.ix);
  a = cadd(a, cscale(d_fwd_t(y1, p.i, p.y, p.H, p.sW), w.iy));
  a = cadd(a, cscale(d_fwd_t(y2, p.i, p.t, p.T, p.sWH), w.it));
  return make_float2(-a.x, -a.y);
}

// utils::Gradient_temp (utils.cpp:134-143): the temporal component alone
AVX_D float2 tgrad(const float2* u, const PixCoord& p, const Wts& w) {
  return cscale(d_fwd(u, p.i, p.t, p.T, p.sWH), w.it);
}

// utils::Divergence_temp (utils.cpp:795-805) = -(D+_t)^T y / dt
AVX_D float2 tdiv(const float2* y, const PixCoord& p, const Wts& w) {
  const float2 a = cscale(d_fwd_t(y, p.i, p.t, p.T, p.sWH), w.it);
  return make_float2(-a.x, -a.y);
}

// utils::SymmetricDivergence, 8-argument form (utils.cpp:961-1012)
AVX_D void symdiv(float2* const* wv, const PixCoord& p, const Wts& w, float2 (&d)[3]) {
  const float2 *w0 = wv[0], *w1 = wv[1], *w2 = wv[2], *w3 = wv[3], *w4 = wv[4], *w5 = wv[5];
  float2 a = cscale(d_bwd_t(w0, p.i, p.x, p.W, 1), w.ix);
  a = cadd(a, cscale(d_bwd_t(w3, p.i, p.y, p.H, p.sW), w.iy));
  a = cadd(a, cscale(d_bwd_t(w4, p.i, p.t, p.T, p.sWH), w.it));
  d[0] = make_float2(-a.x, -a.y);
  a = cscale(d_bwd_t(w3, p.i, p.x, p.W, 1), w.ix);
  a = cadd(a, cscale(d_bwd_t(w1, p.i, p.y, p.H, p.sW), w.iy));
  a = cadd(a, cscale(d_bwd_t(w5, p.i, p.t, p.T, p.sWH), w.it));
  d[1] = make_float2(-a.x, -a.y);
  a = cscale(d_bwd_t(w4, p.i, p.x, p.W, 1), w.ix);
  a = cadd(a, cscale(d_bwd_t(w5, p.i, p.y, p.H, p.sW), w.iy));
  a = cadd(a, cscale(d_bwd_t(w2, p.i, p.t, p.T, p.sWH), w.it));
  d[2] = make_float2(-a.x, -a.y);
}

AVX_D float nrm3(const float2 (&g)[3]) { return sqrtf(cabs2(g[0]) + cabs2(g[1]) + cabs2(g[2])); }
AVX_D float nrm6(const float2 (&g)[6]) {
  float s = cabs2(g[0]) + cabs2(g[1]) + cabs2(g[2]);
  s += 2.f * cabs2(g[3]);
  s += 2.f * cabs2(g[4]);
  s += 2.f * cabs2(g[5]);
  return sqrtf(s);
}
AVX_D float ss3(const float2 (&g)[3]) { return cabs2(g[0]) + cabs2(g[1]) + cabs2(g[2]); }
AVX_D float ss6(const float2 (&g)[6]) {
  return cabs2(g[0]) + cabs2(g[1]) + cabs2(g[2]) + 2.f * (cabs2(g[3]) + cabs2(g[4]) + cabs2(g[5]));
}

// y / max(1, scale * |y|): utils::ProximalMap3/6 (utils.cpp:1297-1351).
// Inside the ball y is left as it is; outside it is multiplied by one
// reciprocal (one division per pixel instead of one per component).
template <int K>
AVX_D void prox_div(float2 (&y)[K], float n, float scale) {
  const float den = scale * n;
  if (den > 1.f) {
    const float inv = 1.f / den;
#pragma unroll
    for (int k = 0; k < K; ++k) y[k] = make_float2(y[k].x * inv, y[k].y * inv);
  }
}
