// Primal-dual kernels of the AVIONIC B200 reconstruction core.
//
// One PD iteration of TV / TGV2 / ICTGV2 (reference loops: CUDA/src/tv.cpp:137-198,
// tgv2.cpp:234-335, ictgv2.cpp:334-490) with the Cartesian operator runs as
// five kernels:
//   dual_kernel    y <- prox(y + sigma * K_reg xbar)        (pointwise + stencils)
//   ydft_kernel    y-transform of b1 xbar onto the sampled rows (all coils)
//   rows_kernel    x-FFT of those rows, z <- prox(z + sigma (K xbar - d)),
//                  Q' = row-IFFT(mask z); one CTA per (coil, frame)
//   coladj_kernel  K^H z = sum_c conj(b1_c) column-IDFT(Q'_c)
//   primal_kernel  divergence stencils, primal update and extragradient
// The step-size rule (pd_recon.cpp:40-61) and the primal-dual gap
// (tv.cpp:202-235, tgv2.cpp:130-176, ictgv2.cpp:163-249) are FP64 block
// reductions plus a one-block finaliser that updates device-resident scalars.
#include <algorithm>

#include "pd_kernels.cuh"
#include "stencil.cuh"
#include "fft.cuh"
#include "tc_dft.cuh"

namespace avx {

// ---------------------------------------------------------------------------
// dual update
// ---------------------------------------------------------------------------

template <int M, int NT>
__global__ void __launch_bounds__(NT) dual_kernel(PDArgs a) {
  if (a.st->stop) return;
  // iteration counter (loopCnt of the reference) kept on the device so that
  // every iteration launches identical work and can be replayed from a graph
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) a.st->iters += 1;
  const int HW = a.W * a.H;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= HW) return;
  const int t = blockIdx.y;
  const PixCoord p = make_pix(j % a.W, j / a.W, t, a.W, a.H, a.T);
  const float sig = (float)a.st->sigma;

  if (M == AVX_M_TV) {
    float2 g[3], y[3];
    grad3(a.xb[0], p, a.w1, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float2 v = a.y[k][p.i];
      y[k] = make_float2(v.x + sig * g[k].x, v.y + sig * g[k].y);
    }
    prox_div<3>(y, nrm3(y), a.r1);
#pragma unroll
    for (int k = 0; k < 3; ++k) a.y[k][p.i] = y[k];
  } else if (M == AVX_M_TVTEMP) {
    // y += sigma D_t xbar / dt, y /= max(1, |y|) (tv_temp.cpp:129-136, ProximalMap1D utils.cpp:1307-1311)
    const float2 g = tgrad(a.xb[0], p, a.w1);
    const float2 v = a.y[0][p.i];
    float2 y[1] = {make_float2(v.x + sig * g.x, v.y + sig * g.y)};
    prox_div<1>(y, sqrtf(cabs2(y[0])), a.r1);
    a.y[0][p.i] = y[0];
  } else if (M == AVX_M_ICTV) {
    // y1 += sigma grad_w1 (xbar1 - xbar3), y3 += sigma grad_w2 xbar3, each
    // projected onto its ball (ictv.cpp:255-285)
    float2 g[3], y1[3];
    grad3_diff(a.xb[0], a.xb[1], p, a.w1, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 v = a.y[k][p.i];
      y1[k] = make_float2(v.x + sig * g[k].x, v.y + sig * g[k].y);
    }
    prox_div<3>(y1, nrm3(y1), a.r1);
#pragma unroll
    for (int k = 0; k < 3; ++k) a.y[k][p.i] = y1[k];
    grad3(a.xb[1], p, a.w2, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 v = a.y[3 + k][p.i];
      y1[k] = make_float2(v.x + sig * g[k].x, v.y + sig * g[k].y);
    }
    prox_div<3>(y1, nrm3(y1), a.r3);
#pragma unroll
    for (int k = 0; k < 3; ++k) a.y[3 + k][p.i] = y1[k];
  } else {
    // branch 1: y1 += sigma (grad u - v), y2 += sigma E v
    // TGV2: u = xbar1, v = xbar2.  ICTGV2: u = xbar1 - xbar3, v = xbar2.
    // Every load of a branch is issued before its first store: the dual
    // pointers may alias as far as the compiler knows, so a store would keep
    // the loads after it from being moved up.
    {
      float2 g[3], y1[3], e[6], y2[6];
#pragma unroll
      for (int k = 0; k < 3; ++k) y1[k] = a.y[k][p.i];
#pragma unroll
      for (int k = 0; k < 6; ++k) y2[k] = a.y[3 + k][p.i];
      if (M == AVX_M_TGV2)
        grad3(a.xb[0], p, a.w1, g);
      else
        grad3_diff(a.xb[0], a.xb[4], p, a.w1, g);
      symgrad(a.xb[1], a.xb[2], a.xb[3], p, a.w1, e);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float2 d = csub(g[k], ldc(a.xb[1 + k], p.i));
        y1[k] = make_float2(y1[k].x + sig * d.x, y1[k].y + sig * d.y);
      }
      prox_div<3>(y1, nrm3(y1), a.r1);
#pragma unroll
      for (int k = 0; k < 6; ++k) y2[k] = make_float2(y2[k].x + sig * e[k].x, y2[k].y + sig * e[k].y);
      prox_div<6>(y2, nrm6(y2), a.r2);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.y[k][p.i] = y1[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) a.y[3 + k][p.i] = y2[k];
    }
    if (M == AVX_M_ICTGV2) {
      // branch 2: y3 += sigma (grad2 xbar3 - xbar4), y4 += sigma E2 xbar4
      float2 g[3], y3[3], e[6], y4[6];
#pragma unroll
      for (int k = 0; k < 3; ++k) y3[k] = a.y[9 + k][p.i];
#pragma unroll
      for (int k = 0; k < 6; ++k) y4[k] = a.y[12 + k][p.i];
      grad3(a.xb[4], p, a.w2, g);
      symgrad(a.xb[5], a.xb[6], a.xb[7], p, a.w2, e);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float2 d = csub(g[k], ldc(a.xb[5 + k], p.i));
        y3[k] = make_float2(y3[k].x + sig * d.x, y3[k].y + sig * d.y);
      }
      prox_div<3>(y3, nrm3(y3), a.r3);
#pragma unroll
      for (int k = 0; k < 6; ++k) y4[k] = make_float2(y4[k].x + sig * e[k].x, y4[k].y + sig * e[k].y);
      prox_div<6>(y4, nrm6(y4), a.r4);
#pragma unroll
      for (int k = 0; k < 3; ++k) a.y[9 + k][p.i] = y3[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) a.y[12 + k][p.i] = y4[k];
    }
  }
}

// ---------------------------------------------------------------------------
// dual update, two pixels per thread (x0, x0 + 1 with x0 even; W even) for
// TGV2 / ICTGV2: every field is read and written as 128-bit pairs, the
// stencil neighbours along y and t as pairs too, along x the one value past
// each end.  Per pixel the arithmetic of dual_kernel (results agree to
// rounding: the compiler may fuse multiply-adds differently).
// ---------------------------------------------------------------------------

struct V2 {
  float2 a, b;  // pixel x0, x0 + 1
};
AVX_D V2 ld4(const float2* p, long long i) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p + i));
  return V2{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
AVX_D void st4(float2* p, long long i, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p + i) = make_float4(a.x, a.y, b.x, b.y);
}

// neighbourhood of one field at a pixel pair
struct Nb {
  V2 c, yp, ym, tp, tm;
  float2 xp, xm;  // x0 + 2, x0 - 1
};

template <bool FWD, bool BWD>
AVX_D Nb load_nb(const float2* u, long long i, int x0, int y, int t, int W, int H, int T, long long sW, long long sWH) {
  Nb n;
  n.c = ld4(u, i);
  if (FWD) {
    n.xp = (x0 + 2 < W) ? __ldg(u + i + 2) : czero();
    n.yp = (y < H - 1) ? ld4(u, i + sW) : V2{czero(), czero()};
    n.tp = (t < T - 1) ? ld4(u, i + sWH) : V2{czero(), czero()};
  }
  if (BWD) {
    n.xm = (x0 > 0) ? __ldg(u + i - 1) : czero();
    n.ym = (y > 0) ? ld4(u, i - sW) : V2{czero(), czero()};
    n.tm = (t > 0) ? ld4(u, i - sWH) : V2{czero(), czero()};
  }
  return n;
}

// per pixel k (0, 1) of the pair: the values stencil.cuh reads
AVX_D float2 pick(const V2& v, int k) { return k ? v.b : v.a; }
AVX_D float2 nb_xp(const Nb& n, int k) { return k ? n.xp : n.c.b; }  // u(i + 1)
AVX_D float2 nb_xm(const Nb& n, int k) { return k ? n.c.a : n.xm; }  // u(i - 1)

// d_fwd of stencil.cuh along x / y / t for pixel k
AVX_D float2 fx(const Nb& n, int k, int x, int W) { return (x < W - 1) ? csub(nb_xp(n, k), pick(n.c, k)) : czero(); }
AVX_D float2 fy(const Nb& n, int k, int y, int H) { return (y < H - 1) ? csub(pick(n.yp, k), pick(n.c, k)) : czero(); }
AVX_D float2 ft(const Nb& n, int k, int t, int T) { return (t < T - 1) ? csub(pick(n.tp, k), pick(n.c, k)) : czero(); }
// d_fwd2: D+ of (u - v), the difference formed first
AVX_D float2 fx2(const Nb& u, const Nb& v, int k, int x, int W) {
  if (x >= W - 1) return czero();
  return csub(csub(nb_xp(u, k), nb_xp(v, k)), csub(pick(u.c, k), pick(v.c, k)));
}
AVX_D float2 fy2(const Nb& u, const Nb& v, int k, int y, int H) {
  if (y >= H - 1) return czero();
  return csub(csub(pick(u.yp, k), pick(v.yp, k)), csub(pick(u.c, k), pick(v.c, k)));
}
AVX_D float2 ft2(const Nb& u, const Nb& v, int k, int t, int T) {
  if (t >= T - 1) return czero();
  return csub(csub(pick(u.tp, k), pick(v.tp, k)), csub(pick(u.c, k), pick(v.c, k)));
}
// d_bwd
AVX_D float2 bx(const Nb& n, int k, int x, int W) {
  const float2 a = (x < W - 1) ? pick(n.c, k) : czero();
  const float2 b = (x > 0) ? nb_xm(n, k) : czero();
  return csub(a, b);
}
AVX_D float2 by(const Nb& n, int k, int y, int H) {
  const float2 a = (y < H - 1) ? pick(n.c, k) : czero();
  const float2 b = (y > 0) ? pick(n.ym, k) : czero();
  return csub(a, b);
}
AVX_D float2 bt(const Nb& n, int k, int t, int T) {
  const float2 a = (t < T - 1) ? pick(n.c, k) : czero();
  const float2 b = (t > 0) ? pick(n.tm, k) : czero();
  return csub(a, b);
}

template <int M, int NT>
__global__ void __launch_bounds__(NT) dual_vec_kernel(PDArgs a) {
  if (a.st->stop) return;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) a.st->iters += 1;
  const int HW2 = (a.W >> 1) * a.H;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= HW2) return;
  const int t = blockIdx.y;
  const int y = j / (a.W >> 1);
  const int x0 = 2 * (j - y * (a.W >> 1));
  const long long sW = a.W, sWH = (long long)a.W * a.H;
  const long long i = x0 + sW * y + sWH * t;
  const float sig = (float)a.st->sigma;
  // branch 1
  {
    V2 y1v[3], y2v[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) y1v[k] = ld4(a.y[k], i);
#pragma unroll
    for (int k = 0; k < 6; ++k) y2v[k] = ld4(a.y[3 + k], i);
    const Nb u = load_nb<true, false>(a.xb[0], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    Nb w;
    if (M == AVX_M_ICTGV2) w = load_nb<true, false>(a.xb[4], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    const Nb v0 = load_nb<false, true>(a.xb[1], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    const Nb v1 = load_nb<false, true>(a.xb[2], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    const Nb v2 = load_nb<false, true>(a.xb[3], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    float2 o1[2][3], o2[2][6];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int x = x0 + k;
      float2 g[3], e[6], y1[3], y2[6];
#pragma unroll
      for (int c = 0; c < 3; ++c) y1[c] = pick(y1v[c], k);
#pragma unroll
      for (int c = 0; c < 6; ++c) y2[c] = pick(y2v[c], k);
      if (M == AVX_M_TGV2) {
        g[0] = cscale(fx(u, k, x, a.W), a.w1.ix);
        g[1] = cscale(fy(u, k, y, a.H), a.w1.iy);
        g[2] = cscale(ft(u, k, t, a.T), a.w1.it);
      } else {
        g[0] = cscale(fx2(u, w, k, x, a.W), a.w1.ix);
        g[1] = cscale(fy2(u, w, k, y, a.H), a.w1.iy);
        g[2] = cscale(ft2(u, w, k, t, a.T), a.w1.it);
      }
      e[0] = cscale(bx(v0, k, x, a.W), a.w1.ix);
      e[1] = cscale(by(v1, k, y, a.H), a.w1.iy);
      e[2] = cscale(bt(v2, k, t, a.T), a.w1.it);
      e[3] = cadd(cscale(by(v0, k, y, a.H), a.w1.hy), cscale(bx(v1, k, x, a.W), a.w1.hx));
      e[4] = cadd(cscale(bt(v0, k, t, a.T), a.w1.ht), cscale(bx(v2, k, x, a.W), a.w1.hx));
      e[5] = cadd(cscale(bt(v1, k, t, a.T), a.w1.ht), cscale(by(v2, k, y, a.H), a.w1.hx));
      const Nb* vv[3] = {&v0, &v1, &v2};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 d = csub(g[c], pick(vv[c]->c, k));
        y1[c] = make_float2(y1[c].x + sig * d.x, y1[c].y + sig * d.y);
      }
      prox_div<3>(y1, nrm3(y1), a.r1);
#pragma unroll
      for (int c = 0; c < 6; ++c) y2[c] = make_float2(y2[c].x + sig * e[c].x, y2[c].y + sig * e[c].y);
      prox_div<6>(y2, nrm6(y2), a.r2);
#pragma unroll
      for (int c = 0; c < 3; ++c) o1[k][c] = y1[c];
#pragma unroll
      for (int c = 0; c < 6; ++c) o2[k][c] = y2[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) st4(a.y[c], i, o1[0][c], o1[1][c]);
#pragma unroll
    for (int c = 0; c < 6; ++c) st4(a.y[3 + c], i, o2[0][c], o2[1][c]);
  }
  if (M == AVX_M_ICTGV2) {
    V2 y3v[3], y4v[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) y3v[k] = ld4(a.y[9 + k], i);
#pragma unroll
    for (int k = 0; k < 6; ++k) y4v[k] = ld4(a.y[12 + k], i);
    const Nb w = load_nb<true, false>(a.xb[4], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    const Nb v0 = load_nb<false, true>(a.xb[5], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    const Nb v1 = load_nb<false, true>(a.xb[6], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    const Nb v2 = load_nb<false, true>(a.xb[7], i, x0, y, t, a.W, a.H, a.T, sW, sWH);
    float2 o1[2][3], o2[2][6];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int x = x0 + k;
      float2 g[3], e[6], y3[3], y4[6];
#pragma unroll
      for (int c = 0; c < 3; ++c) y3[c] = pick(y3v[c], k);
#pragma unroll
      for (int c = 0; c < 6; ++c) y4[c] = pick(y4v[c], k);
      g[0] = cscale(fx(w, k, x, a.W), a.w2.ix);
      g[1] = cscale(fy(w, k, y, a.H), a.w2.iy);
      g[2] = cscale(ft(w, k, t, a.T), a.w2.it);
      e[0] = cscale(bx(v0, k, x, a.W), a.w2.ix);
      e[1] = cscale(by(v1, k, y, a.H), a.w2.iy);
      e[2] = cscale(bt(v2, k, t, a.T), a.w2.it);
      e[3] = cadd(cscale(by(v0, k, y, a.H), a.w2.hy), cscale(bx(v1, k, x, a.W), a.w2.hx));
      e[4] = cadd(cscale(bt(v0, k, t, a.T), a.w2.ht), cscale(bx(v2, k, x, a.W), a.w2.hx));
      e[5] = cadd(cscale(bt(v1, k, t, a.T), a.w2.ht), cscale(by(v2, k, y, a.H), a.w2.hx));
      const Nb* vv[3] = {&v0, &v1, &v2};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float2 d = csub(g[c], pick(vv[c]->c, k));
        y3[c] = make_float2(y3[c].x + sig * d.x, y3[c].y + sig * d.y);
      }
      prox_div<3>(y3, nrm3(y3), a.r3);
#pragma unroll
      for (int c = 0; c < 6; ++c) y4[c] = make_float2(y4[c].x + sig * e[c].x, y4[c].y + sig * e[c].y);
      prox_div<6>(y4, nrm6(y4), a.r4);
#pragma unroll
      for (int c = 0; c < 3; ++c) o1[k][c] = y3[c];
#pragma unroll
      for (int c = 0; c < 6; ++c) o2[k][c] = y4[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) st4(a.y[9 + c], i, o1[0][c], o1[1][c]);
#pragma unroll
    for (int c = 0; c < 6; ++c) st4(a.y[12 + c], i, o2[0][c], o2[1][c]);
  }
}

// ---------------------------------------------------------------------------
// primal update, two pixels per thread (W even) for TGV2 / ICTGV2, with
// 128-bit accesses as in dual_vec_kernel; per pixel the arithmetic of
// primal_kernel
// ---------------------------------------------------------------------------

// d_fwd_t / d_bwd_t of stencil.cuh for pixel k of a pair
AVX_D float2 tfx(const Nb& n, int k, int x, int W) {
  const float2 a = (x > 0) ? nb_xm(n, k) : czero();
  const float2 b = (x < W - 1) ? pick(n.c, k) : czero();
  return csub(a, b);
}
AVX_D float2 tfy(const Nb& n, int k, int y, int H) {
  const float2 a = (y > 0) ? pick(n.ym, k) : czero();
  const float2 b = (y < H - 1) ? pick(n.c, k) : czero();
  return csub(a, b);
}
AVX_D float2 tft(const Nb& n, int k, int t, int T) {
  const float2 a = (t > 0) ? pick(n.tm, k) : czero();
  const float2 b = (t < T - 1) ? pick(n.c, k) : czero();
  return csub(a, b);
}
AVX_D float2 tbx(const Nb& n, int k, int x, int W) { return (x < W - 1) ? csub(pick(n.c, k), nb_xp(n, k)) : czero(); }
AVX_D float2 tby(const Nb& n, int k, int y, int H) { return (y < H - 1) ? csub(pick(n.c, k), pick(n.yp, k)) : czero(); }
AVX_D float2 tbt(const Nb& n, int k, int t, int T) { return (t < T - 1) ? csub(pick(n.c, k), pick(n.tp, k)) : czero(); }

// the pair's neighbours that one field needs: bit 0 x+1, 1 y+1, 2 t+1, 3 x-1, 4 y-1, 5 t-1
template <int F>
AVX_D Nb load_sel(const float2* u, long long i, int x0, int y, int t, int W, int H, int T, long long sW,
                  long long sWH) {
  Nb n;
  const V2 z{czero(), czero()};
  n.c = ld4(u, i);
  n.xp = (F & 1) && x0 + 2 < W ? __ldg(u + i + 2) : czero();
  n.yp = (F & 2) && y < H - 1 ? ld4(u, i + sW) : z;
  n.tp = (F & 4) && t < T - 1 ? ld4(u, i + sWH) : z;
  n.xm = (F & 8) && x0 > 0 ? __ldg(u + i - 1) : czero();
  n.ym = (F & 16) && y > 0 ? ld4(u, i - sW) : z;
  n.tm = (F & 32) && t > 0 ? ld4(u, i - sWH) : z;
  return n;
}

// div3 (D- transposed of the gradient, negated) and symdiv of one branch for pixel k
struct DivBranch {
  Nb y0, y1, y2, w0, w1, w2, w3, w4, w5;
};
AVX_D DivBranch load_branch(float2* const* yv, long long i, int x0, int y, int t, int W, int H, int T, long long sW,
                            long long sWH, bool sym) {
  DivBranch b;
  b.y0 = load_sel<8>(yv[0], i, x0, y, t, W, H, T, sW, sWH);
  b.y1 = load_sel<16>(yv[1], i, x0, y, t, W, H, T, sW, sWH);
  b.y2 = load_sel<32>(yv[2], i, x0, y, t, W, H, T, sW, sWH);
  if (sym) {
    b.w0 = load_sel<1>(yv[3], i, x0, y, t, W, H, T, sW, sWH);
    b.w1 = load_sel<2>(yv[4], i, x0, y, t, W, H, T, sW, sWH);
    b.w2 = load_sel<4>(yv[5], i, x0, y, t, W, H, T, sW, sWH);
    b.w3 = load_sel<3>(yv[6], i, x0, y, t, W, H, T, sW, sWH);
    b.w4 = load_sel<5>(yv[7], i, x0, y, t, W, H, T, sW, sWH);
    b.w5 = load_sel<6>(yv[8], i, x0, y, t, W, H, T, sW, sWH);
  }
  return b;
}
AVX_D float2 pair_div3(const DivBranch& b, int k, int x, int y, int t, int W, int H, int T, const Wts& w) {
  float2 a = cscale(tfx(b.y0, k, x, W), w.ix);
  a = cadd(a, cscale(tfy(b.y1, k, y, H), w.iy));
  a = cadd(a, cscale(tft(b.y2, k, t, T), w.it));
  return make_float2(-a.x, -a.y);
}
AVX_D void pair_symdiv(const DivBranch& b, int k, int x, int y, int t, int W, int H, int T, const Wts& w,
                       float2 (&d)[3]) {
  float2 a = cscale(tbx(b.w0, k, x, W), w.ix);
  a = cadd(a, cscale(tby(b.w3, k, y, H), w.iy));
  a = cadd(a, cscale(tbt(b.w4, k, t, T), w.it));
  d[0] = make_float2(-a.x, -a.y);
  a = cscale(tbx(b.w3, k, x, W), w.ix);
  a = cadd(a, cscale(tby(b.w1, k, y, H), w.iy));
  a = cadd(a, cscale(tbt(b.w5, k, t, T), w.it));
  d[1] = make_float2(-a.x, -a.y);
  a = cscale(tbx(b.w4, k, x, W), w.ix);
  a = cadd(a, cscale(tby(b.w5, k, y, H), w.iy));
  a = cadd(a, cscale(tbt(b.w2, k, t, T), w.it));
  d[2] = make_float2(-a.x, -a.y);
}

// Two phases per pair, to keep fewer values live: branch 1 (div and symdiv
// of y1, y2: components 0-3) is loaded, updated and stored before branch 2
// (ICTGV2: y3, y4, components 4-7) is loaded; component 4 needs branch 1's
// divergence, which is all that crosses the phases.
template <int M, int NT>
__global__ void __launch_bounds__(NT) primal_vec_kernel(PDArgs a) {
  if (a.st->stop) return;
  const int HW2 = (a.W >> 1) * a.H;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= HW2) return;
  const int t = blockIdx.y;
  const int y = j / (a.W >> 1);
  const int x0 = 2 * (j - y * (a.W >> 1));
  const long long sW = a.W, sWH = (long long)a.W * a.H;
  const long long i = x0 + sW * y + sWH * t;
  const float tau = (float)a.st->tau;
  float2 dv1[2];
  {
    const V2 kh = ld4(a.khz, i);
    const DivBranch b1 = load_branch(a.y, i, x0, y, t, a.W, a.H, a.T, sW, sWH, true);
    V2 xo[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) xo[c] = ld4(a.x[c], i);
    float2 xn[2][4], xbv[2][4];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int x = x0 + k;
      dv1[k] = pair_div3(b1, k, x, y, t, a.W, a.H, a.T, a.w1);
      float2 sd1[3];
      pair_symdiv(b1, k, x, y, t, a.W, a.H, a.T, a.w1, sd1);
      const float2 y1[3] = {pick(b1.y0.c, k), pick(b1.y1.c, k), pick(b1.y2.c, k)};
      float2 r[4];
      r[0] = csub(dv1[k], pick(kh, k));
#pragma unroll
      for (int c = 0; c < 3; ++c) r[1 + c] = cadd(y1[c], sd1[c]);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float2 o = pick(xo[c], k);
        const float2 n = make_float2(o.x + tau * r[c].x, o.y + tau * r[c].y);
        xn[k][c] = n;
        xbv[k][c] = make_float2(2.f * n.x - o.x, 2.f * n.y - o.y);
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      st4(a.x[c], i, xn[0][c], xn[1][c]);
      st4(a.xb[c], i, xbv[0][c], xbv[1][c]);
    }
  }
  if (M == AVX_M_ICTGV2) {
    const DivBranch b2 = load_branch(a.y + 9, i, x0, y, t, a.W, a.H, a.T, sW, sWH, true);
    V2 xo[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) xo[c] = ld4(a.x[4 + c], i);
    float2 xn[2][4], xbv[2][4];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int x = x0 + k;
      const float2 dv3 = pair_div3(b2, k, x, y, t, a.W, a.H, a.T, a.w2);
      float2 sd2[3];
      pair_symdiv(b2, k, x, y, t, a.W, a.H, a.T, a.w2, sd2);
      const float2 y3[3] = {pick(b2.y0.c, k), pick(b2.y1.c, k), pick(b2.y2.c, k)};
      float2 r[4];
      r[0] = csub(dv3, dv1[k]);
#pragma unroll
      for (int c = 0; c < 3; ++c) r[1 + c] = cadd(y3[c], sd2[c]);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float2 o = pick(xo[c], k);
        const float2 n = make_float2(o.x + tau * r[c].x, o.y + tau * r[c].y);
        xn[k][c] = n;
        xbv[k][c] = make_float2(2.f * n.x - o.x, 2.f * n.y - o.y);
      }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      st4(a.x[4 + c], i, xn[0][c], xn[1][c]);
      st4(a.xb[4 + c], i, xbv[0][c], xbv[1][c]);
    }
  }
}

// ---------------------------------------------------------------------------
// y-transform: frame t, a strip of YD_XS image columns, every coil.
//   P[t,c,k,x] = 1/sqrt(H) sum_y e^{+2 pi i (ky_k-sy)(y-sy)/H} b1[c,y,x] u[t,y,x]
// (u = in - in2 when in2 is given), written into k.qp in the compact layout
// of z.  The strip of u is staged in shared memory once; coefficient rows
// are staged in chunks of KC compact rows.  Thread (x, cs) handles the
// coils cs, cs + YD_CG, ...
// ---------------------------------------------------------------------------

template <int KC>
__global__ void __launch_bounds__(YD_XS* YD_CG) ydft_kernel(KArgs a) {
  if (a.st && a.st->stop) return;
  constexpr int KCP = KC + 2;  // padded row stride (keeps 16-byte alignment)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const CartGeomDev& g = a.g;
  const int W = g.W, H = g.H, C = g.C;
  const int t = blockIdx.y;
  const int x0 = blockIdx.x * YD_XS;
  const int tx = threadIdx.x, cs = threadIdx.y;
  const int tid = tx + YD_XS * cs, nt = YD_XS * YD_CG;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const int S = r1 - r0;
  if (S == 0) return;
  const long long HW = (long long)W * H;
  float2* su = reinterpret_cast<float2*>(smem_raw);  // [H][YD_XS]
  float2* coef = su + (size_t)H * YD_XS;            // [H][KCP]
  const float2* __restrict__ u = a.in + (long long)t * HW;
  const float2* __restrict__ u2 = a.in2 ? a.in2 + (long long)t * HW : nullptr;
  for (int e = tid; e < H * YD_XS; e += nt) {
    const int y = e / YD_XS, x = x0 + e % YD_XS;
    float2 v = czero();
    if (x < W) {
      v = u[(long long)y * W + x];
      if (u2) v = csub(v, u2[(long long)y * W + x]);
    }
    su[e] = v;
  }
  const int x = x0 + tx;
  for (int k0 = 0; k0 < S; k0 += KC) {
    const int kc = min(KC, S - k0);
    __syncthreads();
    for (int e = tid; e < H * KC; e += nt) {
      const int y = e / KC, kk = e % KC;
      float2 v = czero();
      if (kk < kc) {
        const int ky = g.rows[r0 + k0 + kk];
        const int a1 = (ky - g.sy + H) % H, a2 = (y - g.sy + H) % H;
        v = cscale(g.twy[(a1 * a2) % H], g.inv_sqrt_h);
      }
      coef[y * KCP + kk] = v;
    }
    __syncthreads();
    if (x >= W) continue;
    for (int c = cs; c < C; c += YD_CG) {
      const float2* __restrict__ bc = a.b1 + (long long)c * HW + x;
      float2 acc[KC];
#pragma unroll
      for (int kk = 0; kk < KC; ++kk) acc[kk] = czero();
#pragma unroll 4
      for (int y = 0; y < H; ++y) {
        const float2 v = cmul(__ldg(bc + (long long)y * W), su[y * YD_XS + tx]);
        const float4* cy = reinterpret_cast<const float4*>(coef + y * KCP);
#pragma unroll
        for (int kk = 0; kk < KC; kk += 2) {
          const float4 q = cy[kk >> 1];
          cfma(acc[kk], make_float2(q.x, q.y), v);
          cfma(acc[kk + 1], make_float2(q.z, q.w), v);
        }
      }
      float2* out = a.qp + kbase(g, t, c, r0, r1) + (long long)k0 * W + x;
#pragma unroll
      for (int kk = 0; kk < KC; ++kk)
        if (kk < kc) out[(long long)kk * W] = acc[kk];
    }
  }
}

size_t ydft_smem_bytes(int H) { return sizeof(float2) * (size_t)H * (YD_XS + KSPACE_KC + 2); }

// ---------------------------------------------------------------------------
// Row kernel: one CTA per (coil, frame), compact rows in chunks of KC.  For
// the chunk's y-transformed rows P (from ydft_kernel, in k.qp):
//   X[k][kx] = 1/sqrt(W) sum_x e^{+2 pi i (kx-sx)(x-sx)/W} P[k][x]
// which completes the unitary image -> k-space transform of the reference
// restricted to the kept rows (see oracle/cartesian.py for the sign).  Then,
// by mode:
//   0  PD step:   z <- mask * (z + sigma mask X - sigma d) / (1 + sigma/lambda)
//                 (tgv2.cpp:254-264 followed by the in-place masking of
//                 ForwardOperation, cartesian_operator.cpp:83-88), and
//                 Q'[k][x] = 1/sqrt(W) sum_kx e^{-2 pi i ..} z[k][kx] into k.qp
//   1  step rule: sum |mask X|^2
//   2  gap:       sum |mask X - d|^2, Re<d,z>, |z|^2, then z <- mask z and Q'
//   3  apply:     dense_out[t,c,ky,kx] = mask X
// Each CTA reads and rewrites only its own block of k.qp.
// ---------------------------------------------------------------------------

template <int KC, int PLAN>
__global__ void __launch_bounds__(256, 4) rows_kernel(KArgs a, int mode) {
  if (a.st && a.st->stop && mode != 3) return;
  constexpr int KCP = AVX_FFT_PITCH(KC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const CartGeomDev& g = a.g;
  const int W = PLAN > 1 ? PLAN : g.W, C = g.C;  // W compile-time with a fixed plan
  const int c = blockIdx.x % C;
  const int t = blockIdx.x / C;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const int S = r1 - r0;
  const long long zb = kbase(g, t, c, r0, r1);

  float2* P = reinterpret_cast<float2*>(smem_raw);  // [W][KCP]
  float2* X = P + (size_t)W * KCP;                   // [W][KCP]
  float2* twx = X + (size_t)W * KCP;                 // [W]
  double* red = reinterpret_cast<double*>(twx + W);  // [32*3]

  const int tid = threadIdx.x, nt = blockDim.x;
  __shared__ int splan[12];
  stage_plan(g.rad, splan);
  for (int j = tid; j < W; j += nt) twx[j] = g.twx[j];
  const unsigned mW = div_magic((unsigned)W);  // e < KC W < 2^16

  const float sig = a.st ? (float)a.st->sigma : 0.f;
  const float zscale = (mode == 0) ? (float)(1.0 / (1.0 + a.st->sigma / (double)a.lam)) : 1.f;
  double acc_r[3] = {0.0, 0.0, 0.0};

  for (int k0 = 0; k0 < S; k0 += KC) {
    const int kc = min(KC, S - k0);
    __syncthreads();
    // with the FFT, sequence position n holds x = n + sx (the ifftshift of the
    // centred transform); the dense DFT indexes x directly
    // ROWS_RB loads per thread are issued before any is stored, so that their
    // latencies overlap
    for (int e0 = tid; e0 < KC * W; e0 += ROWS_RB * nt) {
      float2 v[ROWS_RB];
#pragma unroll
      for (int b = 0; b < ROWS_RB; ++b) {
        const int e = e0 + b * nt;
        const int kk = fast_div(e, (unsigned)W, mW), x = e - kk * W;
        v[b] = (e < KC * W && kk < kc) ? a.qp[zb + (long long)(k0 + kk) * W + x] : czero();
      }
#pragma unroll
      for (int b = 0; b < ROWS_RB; ++b) {
        const int e = e0 + b * nt;
        if (e >= KC * W) break;
        const int kk = fast_div(e, (unsigned)W, mW), x = e - kk * W;
        int xs = x;
        if (g.nrad) {
          xs = x - g.sx;
          if (xs < 0) xs += W;
        }
        P[xs * KCP + kk] = v[b];
      }
    }
    __syncthreads();
    float2* Xb = X;  // buffer holding the row transform, index (kx - sx) mod W with the FFT
    if (g.nrad) {
      Xb = row_fft_planned<KC, PLAN, +1>(P, X, twx, W, g.nrad, splan);
    } else {
      // dense DFT along x: thread per kx
      for (int kx = tid; kx < W; kx += nt) {
        float2 acc[KC];
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) acc[kk] = czero();
        const int step = (kx - g.sx + W) % W;
        int jj = (step * ((W - g.sx) % W)) % W;  // index for x = 0
        for (int x = 0; x < W; ++x) {
          const float2 tw = twx[jj];
          const float2* pr = P + x * KCP;
#pragma unroll
          for (int kk = 0; kk < KC; ++kk) cfma(acc[kk], tw, pr[kk]);
          jj += step;
          if (jj >= W) jj -= W;
        }
        float2* xr = X + kx * KCP;
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) xr[kk] = acc[kk];
      }
      __syncthreads();
    }
    // pointwise stage on the kept samples; Xb[n] holds kx = n + sx (FFT) or kx.
    // The mask, z and d values of ROWS_RB samples are loaded first.
    const bool need_zd = mode == 0 || mode == 2;
    for (int e0 = tid; e0 < kc * W; e0 += ROWS_RB * nt) {
      float mb[ROWS_RB];
      float2 zpre[ROWS_RB], dpre[ROWS_RB];
#pragma unroll
      for (int b = 0; b < ROWS_RB; ++b) {
        const int e = e0 + b * nt;
        mb[b] = 0.f;
        zpre[b] = dpre[b] = czero();
        if (e < kc * W) {
          const int kk = fast_div(e, (unsigned)W, mW), kx = e - kk * W;
          const long long gi = zb + (long long)(k0 + kk) * W + kx;
          mb[b] = g.mrow[(long long)(r0 + k0 + kk) * W + kx];
          if (need_zd) {
            zpre[b] = a.z[gi];
            dpre[b] = a.d[gi];
          }
        }
      }
#pragma unroll
      for (int b = 0; b < ROWS_RB; ++b) {
        const int e = e0 + b * nt;
        if (e >= kc * W) break;
        const int kk = fast_div(e, (unsigned)W, mW), kx = e - kk * W;
        int n = kx;
        if (g.nrad) {
          n = kx - g.sx;
          if (n < 0) n += W;
        }
        const long long gi = zb + (long long)(k0 + kk) * W + kx;
        const float m = mb[b];
        const float2 Xv = cscale(Xb[n * KCP + kk], g.inv_sqrt_w);
        const float2 mX = cscale(Xv, m);
        if (mode == 0) {
          const float2 zo = zpre[b], dv = dpre[b];
          // z += sigma * (mask X); z = (z - sigma d) * 1/(1 + sigma/lambda); z *= mask
          float2 zn = make_float2(zo.x + sig * mX.x, zo.y + sig * mX.y);
          zn = make_float2(zn.x - sig * dv.x, zn.y - sig * dv.y);
          zn = cscale(zn, zscale);
          zn = cscale(zn, m);
          a.z[gi] = zn;
          Xb[n * KCP + kk] = zn;
        } else if (mode == 1) {
          acc_r[0] += (double)cabs2(mX);
        } else if (mode == 2) {
          const float2 zo = zpre[b], dv = dpre[b];
          const float2 r = csub(mX, dv);
          acc_r[0] += (double)cabs2(r);
          acc_r[1] += (double)dv.x * zo.x + (double)dv.y * zo.y;
          acc_r[2] += (double)cabs2(zo);
          const float2 zm = cscale(zo, m);
          if (!a.binary_mask) a.z[gi] = zm;
          Xb[n * KCP + kk] = zm;
        } else if (mode == 4) {
          Xb[n * KCP + kk] = cscale(mX, m);
        } else {
          const int ky = g.rows[r0 + k0 + kk];
          a.dense_out[(((long long)t * C + c) * g.H + ky) * W + kx] = mX;
        }
      }
    }
    if (mode == 1 || mode == 3) continue;
    __syncthreads();
    if (g.nrad) {
      // inverse row FFT; Xb position n holds kx = n + sx, the result position n holds x = n + sx
      float2* Qb = row_fft_planned<KC, PLAN, -1>(Xb, Xb == X ? P : X, twx, W, g.nrad, splan);
      for (int e = tid; e < kc * W; e += nt) {
        const int kk = fast_div(e, (unsigned)W, mW), x = e - kk * W;
        int n = x - g.sx;
        if (n < 0) n += W;
        a.qp[zb + (long long)(k0 + kk) * W + x] = cscale(Qb[n * KCP + kk], g.inv_sqrt_w);
      }
      continue;
    }
    // dense inverse DFT along x: thread per x
    for (int x = tid; x < W; x += nt) {
      float2 acc[KC];
#pragma unroll
      for (int kk = 0; kk < KC; ++kk) acc[kk] = czero();
      const int step = (x - g.sx + W) % W;
      int jj = (step * ((W - g.sx) % W)) % W;  // index for kx = 0
      for (int kx = 0; kx < W; ++kx) {
        const float2 tw = twx[jj];
        const float2 twc = make_float2(tw.x, -tw.y);
        const float2* xr = X + kx * KCP;
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) cfma(acc[kk], twc, xr[kk]);
        jj += step;
        if (jj >= W) jj -= W;
      }
#pragma unroll
      for (int kk = 0; kk < KC; ++kk)
        if (kk < kc) a.qp[zb + (long long)(k0 + kk) * W + x] = cscale(acc[kk], g.inv_sqrt_w);
    }
  }
  if (mode == 1 || mode == 2) {
    block_sum<3>(acc_r, red);
    if (tid == 0) {
      const int nb = gridDim.x;
      a.partial[0 * nb + blockIdx.x] = acc_r[0];
      a.partial[1 * nb + blockIdx.x] = acc_r[1];
      a.partial[2 * nb + blockIdx.x] = acc_r[2];
    }
  }
}

size_t rows_smem_bytes(int W, int KC) {
  const int KCP = AVX_FFT_PITCH(KC);
  return sizeof(float2) * (2 * (size_t)W * KCP + W) + sizeof(double) * 32 * 3;
}

size_t kspace_smem_bytes(int W, int H) { return std::max(ydft_smem_bytes(H), rows_smem_bytes(W, KSPACE_KC)); }

// ---------------------------------------------------------------------------
// Column adjoint of the compact rows (completes K^H, cartesian_operator.cpp:65-111):
//   img[t,y,x] = sum_c conj(b1[c,y,x]) 1/sqrt(H) sum_k e^{-2 pi i (ky_k-sy)(y-sy)/H} Q'[t,c,k,x]
// CTA tile 2 CA_TX columns x CA_TY CA_YP rows of frame t; thread (tx, ty)
// owns columns x0+tx, x0+tx+CA_TX and rows y0+ty*CA_YP .. +CA_YP-1, a 2 x
// CA_YP register tile.  Coefficients are staged per chunk of CA_KQ rows;
// Q' is read from global memory (L2 resident), one value per column and row.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(CA_TX* CA_TY) coladj_kernel(KArgs k, float2* img) {
  if (k.st && k.st->stop) return;
  constexpr int TH = CA_TY * CA_YP;
  __shared__ __align__(16) float2 sg[CA_KQ * TH];  // [kk][y] conjugated coefficients
  const CartGeomDev& g = k.g;
  const int W = g.W, H = g.H, C = g.C;
  const int t = blockIdx.z;
  const int x0 = blockIdx.x * 2 * CA_TX, y0 = blockIdx.y * TH;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + CA_TX * ty, nt = CA_TX * CA_TY;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const int S = r1 - r0;
  const long long HW = (long long)W * H;
  const int xa = x0 + tx, xb = x0 + tx + CA_TX;
  const bool va = xa < W, vb = xb < W;
  float2 acc[2][CA_YP];
#pragma unroll
  for (int j = 0; j < CA_YP; ++j) acc[0][j] = acc[1][j] = czero();
  for (int k0 = 0; k0 < S; k0 += CA_KQ) {
    const int kc = min(CA_KQ, S - k0);
    __syncthreads();
    for (int e = tid; e < CA_KQ * TH; e += nt) {
      const int kk = e / TH, yy = e % TH;
      float2 v = czero();
      if (kk < kc && y0 + yy < H) {
        const int ky = g.rows[r0 + k0 + kk];
        const int a1 = (ky - g.sy + H) % H, a2 = (y0 + yy - g.sy + H) % H;
        const float2 w = g.twy[(a1 * a2) % H];
        v = make_float2(w.x * g.inv_sqrt_h, -w.y * g.inv_sqrt_h);
      }
      sg[e] = v;
    }
    __syncthreads();
    for (int c = 0; c < C; ++c) {
      const float2* __restrict__ q = k.qp + kbase(g, t, c, r0, r1) + (long long)k0 * W;
      float2 racc[2][CA_YP];
#pragma unroll
      for (int j = 0; j < CA_YP; ++j) racc[0][j] = racc[1][j] = czero();
#pragma unroll 4
      for (int kk = 0; kk < kc; ++kk) {
        const float2 qa = va ? __ldg(q + (long long)kk * W + xa) : czero();
        const float2 qb = vb ? __ldg(q + (long long)kk * W + xb) : czero();
        const float4* gy = reinterpret_cast<const float4*>(sg + kk * TH + ty * CA_YP);
#pragma unroll
        for (int j = 0; j < CA_YP; j += 2) {
          const float4 c2 = gy[j >> 1];
          const float2 g0 = make_float2(c2.x, c2.y), g1 = make_float2(c2.z, c2.w);
          cfma(racc[0][j], g0, qa);
          cfma(racc[0][j + 1], g1, qa);
          cfma(racc[1][j], g0, qb);
          cfma(racc[1][j + 1], g1, qb);
        }
      }
      const float2* __restrict__ bc = k.b1 + (long long)c * HW;
#pragma unroll
      for (int j = 0; j < CA_YP; ++j) {
        const int y = y0 + ty * CA_YP + j;
        if (y >= H) break;
        if (va) acc[0][j] = cadd(acc[0][j], cmulc(__ldg(bc + (long long)y * W + xa), racc[0][j]));
        if (vb) acc[1][j] = cadd(acc[1][j], cmulc(__ldg(bc + (long long)y * W + xb), racc[1][j]));
      }
    }
  }
  float2* out = img + (long long)t * HW;
#pragma unroll
  for (int j = 0; j < CA_YP; ++j) {
    const int y = y0 + ty * CA_YP + j;
    if (y >= H) break;
    if (va) out[(long long)y * W + xa] = acc[0][j];
    if (vb) out[(long long)y * W + xb] = acc[1][j];
  }
}

// ---------------------------------------------------------------------------
// primal update; K^H z is read from the image a.khz (column adjoint or
// gridding adjoint)
// ---------------------------------------------------------------------------

template <int M, int PR_TX, int PR_TY, int PR_YP>
__global__ void __launch_bounds__(PR_TX* PR_TY) primal_kernel(PDArgs a) {
  if (a.st->stop) return;
  constexpr int PR_TH = PR_TY * PR_YP;
  const int t = blockIdx.z;
  const int x0 = blockIdx.x * PR_TX, y0 = blockIdx.y * PR_TH;
  float2 kh[PR_YP];
#pragma unroll
  for (int j = 0; j < PR_YP; ++j) {
    const int y = y0 + threadIdx.y * PR_YP + j;
    const int x = x0 + threadIdx.x;
    kh[j] = (x < a.W && y < a.H) ? a.khz[((long long)t * a.H + y) * a.W + x] : czero();
  }
  const int x = x0 + threadIdx.x;
  if (x >= a.W) return;
  const float tau = (float)a.st->tau;
#pragma unroll
  for (int j = 0; j < PR_YP; ++j) {
    const int y = y0 + threadIdx.y * PR_YP + j;
    if (y >= a.H) continue;
    const PixCoord p = make_pix(x, y, t, a.W, a.H, a.T);
    // every load of the pixel first (the stores below would otherwise order them)
    const float2 dv1 = M == AVX_M_TVTEMP ? tdiv(a.y[0], p, a.w1) : div3(a.y[0], a.y[1], a.y[2], p, a.w1);
    float2 sd1[3], y1[3], sd2[3], y3[3], xo[8];
    float2 dv3 = czero();
    if (M == AVX_M_ICTV) dv3 = div3(a.y[3], a.y[4], a.y[5], p, a.w2);
    if (M == AVX_M_TGV2 || M == AVX_M_ICTGV2) {
      symdiv(a.y + 3, p, a.w1, sd1);
#pragma unroll
      for (int c = 0; c < 3; ++c) y1[c] = ldc(a.y[c], p.i);
    }
    if (M == AVX_M_ICTGV2) {
      dv3 = div3(a.y[9], a.y[10], a.y[11], p, a.w2);
      symdiv(a.y + 12, p, a.w2, sd2);
#pragma unroll
      for (int c = 0; c < 3; ++c) y3[c] = ldc(a.y[9 + c], p.i);
    }
    constexpr int P = MethodDims<M>::P;
#pragma unroll
    for (int c = 0; c < P; ++c) xo[c] = a.x[c][p.i];
    // updates: x' = x + tau r, xbar = 2 x' - x
    float2 r[8];
    r[0] = csub(dv1, kh[j]);                       // x1 <- x1 - tau (K^H z - div y1)
    if (M == AVX_M_ICTV) r[1] = csub(dv3, dv1);    // x3 <- x3 - tau (div1 y1 - div2 y3) (ictv.cpp:300-318)
    if (M == AVX_M_TGV2 || M == AVX_M_ICTGV2)
#pragma unroll
      for (int c = 0; c < 3; ++c) r[1 + c] = cadd(y1[c], sd1[c]);  // x2 <- x2 + tau (y1 + symdiv y2)
    if (M == AVX_M_ICTGV2) {
      r[4] = csub(dv3, dv1);                       // x3 <- x3 - tau (div1 y1 - div2 y3)
#pragma unroll
      for (int c = 0; c < 3; ++c) r[5 + c] = cadd(y3[c], sd2[c]);  // x4 <- x4 + tau (y3 + symdiv2 y4)
    }
#pragma unroll
    for (int c = 0; c < P; ++c) {
      const float2 xn = make_float2(xo[c].x + tau * r[c].x, xo[c].y + tau * r[c].y);
      a.x[c][p.i] = xn;
      a.xb[c][p.i] = make_float2(2.f * xn.x - xo[c].x, 2.f * xn.y - xo[c].y);
    }
  }
}

// ---------------------------------------------------------------------------
// step rule: image-side norms of e = xbar - x
// (TV::AdaptStepSize tv.cpp:79-97, TGV2 tgv2.cpp:89-128, ICTGV2 ictgv2.cpp:97-161)
// slot 0: sum of squared regulariser-operator norms; slot 1: sum |e|^2
// ---------------------------------------------------------------------------

template <int M>
__global__ void __launch_bounds__(256) step_img_kernel(PDArgs a, Ptr8 e, double* partial) {
  if (a.st->stop) return;
  __shared__ double red[32 * 2];
  double acc[2] = {0.0, 0.0};
  const long long HW = (long long)a.W * a.H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / HW);
    const int r = (int)(i - t * HW);
    const PixCoord p = make_pix(r % a.W, r / a.W, t, a.W, a.H, a.T);
    if (M == AVX_M_TV) {
      float2 g[3];
      grad3(e.p[0], p, a.w1, g);
      acc[0] += (double)ss3(g);
      acc[1] += (double)cabs2(ldc(e.p[0], p.i));
    } else if (M == AVX_M_TVTEMP) {
      // TVTEMP::AdaptStepSize (tv_temp.cpp:80-95): temporal gradient only
      acc[0] += (double)cabs2(tgrad(e.p[0], p, a.w1));
      acc[1] += (double)cabs2(ldc(e.p[0], p.i));
    } else if (M == AVX_M_ICTV) {
      // ICTV::AdaptStepSize (ictv.cpp:97-128) forms the gradient sums in a
      // buffer that the next statement overwrites: |K e1| and |e1|, |e3| remain
      acc[1] += (double)(cabs2(ldc(e.p[0], p.i)) + cabs2(ldc(e.p[1], p.i)));
    } else {
      float2 g[3], s[6];
      if (M == AVX_M_TGV2)
        grad3(e.p[0], p, a.w1, g);
      else
        grad3_diff(e.p[0], e.p[4], p, a.w1, g);
#pragma unroll
      for (int c = 0; c < 3; ++c) g[c] = csub(g[c], ldc(e.p[1 + c], p.i));
      acc[0] += (double)ss3(g);
      symgrad(e.p[1], e.p[2], e.p[3], p, a.w1, s);
      acc[0] += (double)ss6(s);
      float nx = cabs2(ldc(e.p[0], p.i));
#pragma unroll
      for (int c = 0; c < 3; ++c) nx += cabs2(ldc(e.p[1 + c], p.i));
      if (M == AVX_M_ICTGV2) {
        grad3(e.p[4], p, a.w2, g);
#pragma unroll
        for (int c = 0; c < 3; ++c) g[c] = csub(g[c], ldc(e.p[5 + c], p.i));
        acc[0] += (double)ss3(g);
        symgrad(e.p[5], e.p[6], e.p[7], p, a.w2, s);
        acc[0] += (double)ss6(s);
        nx += cabs2(ldc(e.p[4], p.i));
#pragma unroll
        for (int c = 0; c < 3; ++c) nx += cabs2(ldc(e.p[5 + c], p.i));
      }
      acc[1] += (double)nx;
    }
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) {
    partial[0 * gridDim.x + blockIdx.x] = acc[0];
    partial[1 * gridDim.x + blockIdx.x] = acc[1];
  }
}

// e = xbar - x for every primal component (the reference's subVector before
// AdaptStepSize, tgv2.cpp:306-314)
__global__ void diff_kernel(PDArgs a, Ptr8 e, int P) {
  if (a.st->stop) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.N;
       i += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < P; ++c) e.p[c][i] = csub(a.xb[c][i], a.x[c][i]);
  }
}

__global__ void step_finalize_kernel(DevState* st, const double* pimg, int nimg, const double* pk,
                                     int nk, double ratio) {
  if (st->stop) return;
  __shared__ double red[32 * 3];
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < nimg; i += blockDim.x) {
    v[0] += pimg[i];
    v[1] += pimg[nimg + i];
  }
  for (int i = threadIdx.x; i < nk; i += blockDim.x) v[2] += pk[i];
  block_sum<3>(v, red);
  if (threadIdx.x == 0) {
    const double nKx = sqrt(fabs(v[0] + v[2]));
    const double nx = sqrt(fabs(v[1]));
    st->nKx2 = v[0] + v[2];
    st->nx2 = v[1];
    // PDRecon::AdaptStepSize (pd_recon.cpp:40-61)
    const double tmp = nx / nKx;
    const double theta = 0.95;
    double s = st->sigma, tt = st->tau;
    if (s * tt > tmp * tmp) {
      if (theta * theta * s * tt < tmp * tmp) {
        s *= theta;
        tt *= theta;
      } else {
        s = tmp * ratio;
        tt = tmp / ratio;
      }
    }
    st->sigma = (double)(float)s;
    st->tau = (double)(float)tt;
  }
}

// ---------------------------------------------------------------------------
// primal-dual gap, image side (needs a fresh K^H z image in a.khz).
// slots: 0 g3 = |K^H z - div y1|_1, 1 g4, 2 g5, 3 g6,
//        4..7 regulariser L1 sums n1..n4 (see gap_finalize_kernel)
// ---------------------------------------------------------------------------

template <int M>
__global__ void __launch_bounds__(ADJ_TX* ADJ_TY) gap_img_kernel(PDArgs a, double* partial) {
  if (a.st->stop) return;
  __shared__ double red[32 * 8];
  const int t = blockIdx.z;
  const int x0 = blockIdx.x * ADJ_TX, y0 = blockIdx.y * ADJ_TH;
  float2 kh[ADJ_YP];
#pragma unroll
  for (int j = 0; j < ADJ_YP; ++j) {
    const int y = y0 + threadIdx.y * ADJ_YP + j;
    const int x = x0 + threadIdx.x;
    kh[j] = (x < a.W && y < a.H) ? a.khz[((long long)t * a.H + y) * a.W + x] : czero();
  }
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int x = x0 + threadIdx.x;
  if (x < a.W) {
#pragma unroll
    for (int j = 0; j < ADJ_YP; ++j) {
      const int y = y0 + threadIdx.y * ADJ_YP + j;
      if (y >= a.H) continue;
      const PixCoord p = make_pix(x, y, t, a.W, a.H, a.T);
      const float2 dv1 = M == AVX_M_TVTEMP ? tdiv(a.y[0], p, a.w1) : div3(a.y[0], a.y[1], a.y[2], p, a.w1);
      acc[0] += (double)sqrtf(cabs2(csub(kh[j], dv1)));
      float2 g[3];
      if (M == AVX_M_TV || M == AVX_M_TVTEMP) {
        // TVTEMP::ComputePDGap adds the full TVNorm (tv_temp.cpp:214-222)
        grad3(a.x[0], p, a.w1, g);
        acc[4] += (double)nrm3(g);
        continue;
      }
      if (M == AVX_M_ICTV) {
        // ICTV::ComputeGStar g5 and ICTVNorm's two TV norms (ictv.cpp:148-190, utils.cpp:1221-1242)
        const float2 dv3 = div3(a.y[3], a.y[4], a.y[5], p, a.w2);
        acc[2] += (double)sqrtf(cabs2(csub(dv1, dv3)));
        grad3_diff(a.x[0], a.x[1], p, a.w1, g);
        acc[4] += (double)nrm3(g);
        grad3(a.x[1], p, a.w2, g);
        acc[6] += (double)nrm3(g);
        continue;
      }
      float2 sd[3], e[6];
      symdiv(a.y + 3, p, a.w1, sd);
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[1] += (double)sqrtf(cabs2(cadd(sd[c], ldc(a.y[c], p.i))));
      if (M == AVX_M_TGV2)
        grad3(a.x[0], p, a.w1, g);
      else
        grad3_diff(a.x[0], a.x[4], p, a.w1, g);
#pragma unroll
      for (int c = 0; c < 3; ++c) g[c] = csub(g[c], ldc(a.x[1 + c], p.i));
      acc[4] += (double)nrm3(g);
      symgrad(a.x[1], a.x[2], a.x[3], p, a.w1, e);
      acc[5] += (double)nrm6(e);
      if (M == AVX_M_ICTGV2) {
        const float2 dv3 = div3(a.y[9], a.y[10], a.y[11], p, a.w2);
        acc[2] += (double)sqrtf(cabs2(csub(dv1, dv3)));
        symdiv(a.y + 12, p, a.w2, sd);
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[3] += (double)sqrtf(cabs2(cadd(sd[c], ldc(a.y[9 + c], p.i))));
        grad3(a.x[4], p, a.w2, g);
#pragma unroll
        for (int c = 0; c < 3; ++c) g[c] = csub(g[c], ldc(a.x[5 + c], p.i));
        acc[6] += (double)nrm3(g);
        symgrad(a.x[5], a.x[6], a.x[7], p, a.w2, e);
        acc[7] += (double)nrm6(e);
      }
    }
  }
  block_sum<8>(acc, red);
  const int nb = gridDim.x * gridDim.y * gridDim.z;
  const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
#pragma unroll
    for (int s = 0; s < 8; ++s) partial[s * nb + b] = acc[s];
  }
}

// Assembles G* + R (tv.cpp:202-235, tgv2.cpp:130-176, ictgv2.cpp:163-249),
// records the history and raises the stop flag.
template <int M>
__global__ void gap_finalize_kernel(DevState* st, const double* pk, int nk, const double* pimg, int nimg,
                                    GapConst gc, double* hist_gap, double* hist_norm, double* hist_fid,
                                    int cap, int init_only) {
  if (st->stop) return;
  __shared__ double red[32 * 11];
  double v[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < nk; i += blockDim.x) {
    v[0] += pk[i];
    v[1] += pk[nk + i];
    v[2] += pk[2 * nk + i];
  }
  for (int i = threadIdx.x; i < nimg; i += blockDim.x) {
#pragma unroll
    for (int s = 0; s < 8; ++s) v[3 + s] += pimg[s * nimg + i];
  }
  block_sum<11>(v, red);
  if (threadIdx.x != 0) return;
  const double lam = gc.lam;
  const double res2 = v[0] + st->d_off;
  const double g1 = 0.5 * lam * res2;
  const double g2 = v[1] + v[2] / (2.0 * lam);
  const double g36 = v[3] + v[4] + v[5] + v[6];
  double reg;
  if (M == AVX_M_TV || M == AVX_M_TVTEMP)
    reg = v[7];
  else if (M == AVX_M_ICTV)
    reg = gc.alpha1 * gc.ic_a * v[7] + gc.alpha1 * gc.ic_b * v[9];
  else if (M == AVX_M_TGV2)
    reg = gc.alpha1 * v[7] + gc.alpha0 * v[8];
  else
    reg = gc.ic_a * (gc.alpha1 * v[7] + gc.alpha0 * v[8]) + gc.ic_b * (gc.alpha1 * v[9] + gc.alpha0 * v[10]);
  const double gap = fabs(g1 + g2 + g36 + reg) / gc.N;
  const double fid = sqrt(fabs(res2)) * lam / 2.0;
  if (init_only) {
    // ICTGV2 records norm and data fidelity once before its loop (ictgv2.cpp:318-328)
    if (hist_norm) hist_norm[0] = reg;
    if (hist_fid) hist_fid[0] = fid;
    return;
  }
  st->gap = gap;
  if (st->gap0 == 0.0) st->gap0 = gap;
  const bool stop = gap < gc.stop_gap || (gc.stop_rel > 0.0 && gap <= gc.stop_rel * st->gap0);
  // TGV2 returns before recording the gap that stops it (tgv2.cpp:325-328)
  const bool record = !(M == AVX_M_TGV2 && stop);
  // ICTGV2's norm and fidelity histories start with the pre-loop record
  const int off = M == AVX_M_ICTGV2 ? 1 : 0;
  if (record && st->ngap < cap) {
    hist_gap[st->ngap] = gap;
    if (hist_norm) hist_norm[st->ngap + off] = reg;
    if (hist_fid) hist_fid[st->ngap + off] = fid;
    st->ngap += 1;
  }
  if (stop) st->stop = 1;
}

// ---------------------------------------------------------------------------
// data movement helpers
// ---------------------------------------------------------------------------

// dense (T,C,H,W) -> compact rows, optionally multiplied by the mask
__global__ void gather_rows_kernel(CartGeomDev g, const float2* dense, float2* compact, int apply_mask) {
  const int c = blockIdx.x % g.C, t = blockIdx.x / g.C;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const long long zb = kbase(g, t, c, r0, r1);
  for (int e = threadIdx.x; e < (r1 - r0) * g.W; e += blockDim.x) {
    const int kk = e / g.W, kx = e % g.W;
    const int ky = g.rows[r0 + kk];
    float2 v = dense[(((long long)t * g.C + c) * g.H + ky) * g.W + kx];
    if (apply_mask) v = cscale(v, g.mrow[(long long)(r0 + kk) * g.W + kx]);
    compact[zb + (long long)kk * g.W + kx] = v;
  }
}

// k-space -> image transform of a dense k-space vector, first stage: mask the
// input in place (cartesian_operator.cpp:83-88; rows outside the kept set
// carry mask 0 and are cleared) and row-IDFT the kept rows into Q'.
__global__ void dense_rowidft_kernel(CartGeomDev g, float2* dense, float2* qp, const float* mask_dense) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* row = reinterpret_cast<float2*>(smem_raw);  // [W]
  const int c = blockIdx.x % g.C, t = blockIdx.x / g.C;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const long long zb = kbase(g, t, c, r0, r1);
  float2* slice = dense + ((long long)t * g.C + c) * g.H * g.W;
  if (mask_dense) {
    const float* ms = mask_dense + (long long)t * g.H * g.W;
    for (long long e = threadIdx.x; e < (long long)g.H * g.W; e += blockDim.x) slice[e] = cscale(slice[e], ms[e]);
  }
  __syncthreads();
  for (int kk = 0; kk < r1 - r0; ++kk) {
    const int ky = g.rows[r0 + kk];
    for (int kx = threadIdx.x; kx < g.W; kx += blockDim.x) row[kx] = slice[(long long)ky * g.W + kx];
    __syncthreads();
    for (int x = threadIdx.x; x < g.W; x += blockDim.x) {
      float2 acc = czero();
      const int step = (x - g.sx + g.W) % g.W;
      int jj = (step * ((g.W - g.sx) % g.W)) % g.W;
      for (int kx = 0; kx < g.W; ++kx) {
        const float2 tw = g.twx[jj];
        cfma(acc, make_float2(tw.x, -tw.y), row[kx]);
        jj += step;
        if (jj >= g.W) jj -= g.W;
      }
      qp[zb + (long long)kk * g.W + x] = cscale(acc, g.inv_sqrt_w);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// explicit template instantiations and launch helpers
// ---------------------------------------------------------------------------

static void rec(cudaEvent_t* ev, int i, cudaStream_t s) {
  if (ev) cudaEventRecord(ev[i], s);
}

// tuning tables (AVX_PRIMAL_TILES, AVX_DUAL_BLOCKS entries, in the order of
// the switches below); 32 x 8 x 1 and 256 threads measured fastest at
// 192 x 192 x 30 ICTGV2 (primal 68 us against 90 us for 32 x 4 x 4)
static const char* kPrimalTileNames[AVX_PRIMAL_TILES] = {"32x8x1", "32x4x2", "64x4x1", "32x4x4", "32x16x1",
                                                          "128x1 pairs", "256x1 pairs"};
static const int kDualBlocks[AVX_DUAL_BLOCKS] = {256, 128, 512, 256, 128, 512};

const char* primal_tile_name(int i) { return kPrimalTileNames[(i >= 0 && i < AVX_PRIMAL_TILES) ? i : 0]; }
int dual_block_threads(int i) { return kDualBlocks[(i >= 0 && i < AVX_DUAL_BLOCKS) ? i : 0]; }

template <int NT>
static void launch_dual_nt(int method, const PDArgs& a, cudaStream_t s) {
  dim3 gd((a.W * a.H + NT - 1) / NT, a.T);
  if (method == AVX_M_TV) dual_kernel<AVX_M_TV, NT><<<gd, NT, 0, s>>>(a);
  else if (method == AVX_M_TVTEMP) dual_kernel<AVX_M_TVTEMP, NT><<<gd, NT, 0, s>>>(a);
  else if (method == AVX_M_TGV2) dual_kernel<AVX_M_TGV2, NT><<<gd, NT, 0, s>>>(a);
  else if (method == AVX_M_ICTV) dual_kernel<AVX_M_ICTV, NT><<<gd, NT, 0, s>>>(a);
  else dual_kernel<AVX_M_ICTGV2, NT><<<gd, NT, 0, s>>>(a);
}

bool dual_pairs(int method, int W) { return (method == AVX_M_TGV2 || method == AVX_M_ICTGV2) && W % 2 == 0; }

template <int NT>
static void launch_dual_vec(int method, const PDArgs& a, cudaStream_t s) {
  dim3 gd(((a.W / 2) * a.H + NT - 1) / NT, a.T);
  if (method == AVX_M_TGV2) dual_vec_kernel<AVX_M_TGV2, NT><<<gd, NT, 0, s>>>(a);
  else dual_vec_kernel<AVX_M_ICTGV2, NT><<<gd, NT, 0, s>>>(a);
}

void launch_dual(int method, const PDArgs& a, cudaStream_t s) {
  if (a.dual_block >= 3 && dual_pairs(method, a.W)) {
    switch (dual_block_threads(a.dual_block)) {
      case 128: launch_dual_vec<128>(method, a, s); break;
      case 512: launch_dual_vec<512>(method, a, s); break;
      default: launch_dual_vec<256>(method, a, s); break;
    }
    return;
  }
  switch (dual_block_threads(a.dual_block)) {
    case 128: launch_dual_nt<128>(method, a, s); break;
    case 512: launch_dual_nt<512>(method, a, s); break;
    default: launch_dual_nt<256>(method, a, s); break;
  }
}

template <int TX, int TY, int YP>
static void launch_primal_tile(int method, const PDArgs& a, cudaStream_t s) {
  dim3 gp((a.W + TX - 1) / TX, (a.H + TY * YP - 1) / (TY * YP), a.T);
  dim3 bl(TX, TY);
  if (method == AVX_M_TV) primal_kernel<AVX_M_TV, TX, TY, YP><<<gp, bl, 0, s>>>(a);
  else if (method == AVX_M_TVTEMP) primal_kernel<AVX_M_TVTEMP, TX, TY, YP><<<gp, bl, 0, s>>>(a);
  else if (method == AVX_M_TGV2) primal_kernel<AVX_M_TGV2, TX, TY, YP><<<gp, bl, 0, s>>>(a);
  else if (method == AVX_M_ICTV) primal_kernel<AVX_M_ICTV, TX, TY, YP><<<gp, bl, 0, s>>>(a);
  else primal_kernel<AVX_M_ICTGV2, TX, TY, YP><<<gp, bl, 0, s>>>(a);
}

template <int NT>
static void launch_primal_vec(int method, const PDArgs& a, cudaStream_t s) {
  dim3 gd(((a.W / 2) * a.H + NT - 1) / NT, a.T);
  if (method == AVX_M_TGV2) primal_vec_kernel<AVX_M_TGV2, NT><<<gd, NT, 0, s>>>(a);
  else primal_vec_kernel<AVX_M_ICTGV2, NT><<<gd, NT, 0, s>>>(a);
}

void launch_primal(int method, const PDArgs& a, cudaStream_t s) {
  if (a.primal_tile >= 5 && dual_pairs(method, a.W)) {
    if (a.primal_tile == 5)
      launch_primal_vec<128>(method, a, s);
    else
      launch_primal_vec<256>(method, a, s);
    return;
  }
  switch (a.primal_tile) {
    case 1: launch_primal_tile<32, 4, 2>(method, a, s); break;
    case 2: launch_primal_tile<64, 4, 1>(method, a, s); break;
    case 3: launch_primal_tile<32, 4, 4>(method, a, s); break;
    case 4: launch_primal_tile<32, 16, 1>(method, a, s); break;
    default: launch_primal_tile<32, 8, 1>(method, a, s); break;
  }
}

void launch_ydft(const KArgs& k, cudaStream_t s) {
  if (k.tc_ytab) {
    launch_ydft_tc(k, s);
    return;
  }
  dim3 gr((k.g.W + YD_XS - 1) / YD_XS, k.g.T);
  ydft_kernel<KSPACE_KC><<<gr, dim3(YD_XS, YD_CG), ydft_smem_bytes(k.g.H), s>>>(k);
}

template <int KC>
static void launch_rows_kc(const KArgs& k, int mode, cudaStream_t s) {
  // 256 threads, as the compile-time FFT plans assume
  const int id = k.rows_rt ? fft_plan_id_runtime(k.g.nrad, k.g.rad) : fft_plan_id(k.g.W, k.g.nrad, k.g.rad);
#define CALL_R(ID) rows_kernel<KC, ID><<<k.g.C * k.g.T, 256, rows_smem_bytes(k.g.W, KC), s>>>(k, mode)
  AVX_FFT_PLAN_DISPATCH(id, CALL_R)
#undef CALL_R
}

void launch_rows(const KArgs& k, int mode, cudaStream_t s) {
  switch (k.rows_kc) {
    case 8: launch_rows_kc<8>(k, mode, s); break;
    case 12: launch_rows_kc<12>(k, mode, s); break;
    default: launch_rows_kc<KSPACE_KC>(k, mode, s); break;
  }
}

void launch_kspace(const KArgs& k, int mode, cudaStream_t s) {
  launch_ydft(k, s);
  launch_rows(k, mode, s);
}

void launch_adjoint(const KArgs& k, float2* img, cudaStream_t s) {
  if (k.tc_ctab) {
    launch_coladj_tc(k, img, s);
    return;
  }
  dim3 gr((k.g.W + 2 * CA_TX - 1) / (2 * CA_TX), (k.g.H + CA_TY * CA_YP - 1) / (CA_TY * CA_YP), k.g.T);
  coladj_kernel<<<gr, dim3(CA_TX, CA_TY), 0, s>>>(k, img);
}

void launch_iteration(int method, const PDArgs& a, const KArgs& k, float2* khz, cudaStream_t s, cudaEvent_t* ev) {
  rec(ev, 0, s);
  launch_dual(method, a, s);
  rec(ev, 1, s);
  launch_ydft(k, s);
  rec(ev, 2, s);
  launch_rows(k, 0, s);
  rec(ev, 3, s);
  launch_adjoint(k, khz, s);
  rec(ev, 4, s);
  launch_primal(method, a, s);
  rec(ev, 5, s);
}

int gap_img_blocks(int W, int H, int T) {
  return ((W + ADJ_TX - 1) / ADJ_TX) * ((H + ADJ_TH - 1) / ADJ_TH) * T;
}

void launch_step_img(int method, const PDArgs& a, const Ptr8& e_dev, int P, double* pimg, cudaStream_t s) {
  diff_kernel<<<AVX_RED_BLOCKS, 256, 0, s>>>(a, e_dev, P);
  if (method == AVX_M_TV) step_img_kernel<AVX_M_TV><<<AVX_RED_BLOCKS, 256, 0, s>>>(a, e_dev, pimg);
  else if (method == AVX_M_TVTEMP) step_img_kernel<AVX_M_TVTEMP><<<AVX_RED_BLOCKS, 256, 0, s>>>(a, e_dev, pimg);
  else if (method == AVX_M_TGV2) step_img_kernel<AVX_M_TGV2><<<AVX_RED_BLOCKS, 256, 0, s>>>(a, e_dev, pimg);
  else if (method == AVX_M_ICTV) step_img_kernel<AVX_M_ICTV><<<AVX_RED_BLOCKS, 256, 0, s>>>(a, e_dev, pimg);
  else step_img_kernel<AVX_M_ICTGV2><<<AVX_RED_BLOCKS, 256, 0, s>>>(a, e_dev, pimg);
}

void launch_step_finalize(const PDArgs& a, double* pimg, double* pk, int nk, double ratio, cudaStream_t s) {
  step_finalize_kernel<<<1, 256, 0, s>>>(a.st, pimg, AVX_RED_BLOCKS, pk, nk, ratio);
}

void launch_step(int method, const PDArgs& a, const KArgs& k_e, const Ptr8& e_dev, int P,
                 double* pimg, double* pk, double ratio, cudaStream_t s) {
  launch_step_img(method, a, e_dev, P, pimg, s);
  launch_kspace(k_e, 1, s);
  launch_step_finalize(a, pimg, pk, k_e.g.C * k_e.g.T, ratio, s);
}

void launch_gap_tail(int method, const PDArgs& a, const KArgs& k_x, double* pimg, double* pk, int nk,
                     const GapConst& gc, double* hg, double* hn, double* hf, int cap, int init_only,
                     cudaStream_t s) {
  (void)k_x;
  dim3 gp((a.W + ADJ_TX - 1) / ADJ_TX, (a.H + ADJ_TH - 1) / ADJ_TH, a.T);
  dim3 bl(ADJ_TX, ADJ_TY);
  const int nimg = gap_img_blocks(a.W, a.H, a.T);
#define GAP_IMG(MM)                                              \
  gap_img_kernel<MM><<<gp, bl, 0, s>>>(a, pimg);                \
  gap_finalize_kernel<MM><<<1, 256, 0, s>>>(a.st, pk, nk, pimg, nimg, gc, hg, hn, hf, cap, init_only);
  if (method == AVX_M_TV) {
    GAP_IMG(AVX_M_TV)
  } else if (method == AVX_M_TVTEMP) {
    GAP_IMG(AVX_M_TVTEMP)
  } else if (method == AVX_M_TGV2) {
    GAP_IMG(AVX_M_TGV2)
  } else if (method == AVX_M_ICTV) {
    GAP_IMG(AVX_M_ICTV)
  } else {
    GAP_IMG(AVX_M_ICTGV2)
  }
#undef GAP_IMG
}

void launch_gap(int method, const PDArgs& a, const KArgs& k_x, float2* khz, double* pimg, double* pk,
                const GapConst& gc, double* hg, double* hn, double* hf, int cap, int init_only, cudaStream_t s) {
  launch_kspace(k_x, 2, s);
  launch_adjoint(k_x, khz, s);
  PDArgs ag = a;
  ag.khz = khz;
  launch_gap_tail(method, ag, k_x, pimg, pk, k_x.g.C * k_x.g.T, gc, hg, hn, hf, cap, init_only, s);
}

void launch_gather_rows(const CartGeomDev& g, const float2* dense, float2* compact, int apply_mask, cudaStream_t s) {
  gather_rows_kernel<<<g.C * g.T, 256, 0, s>>>(g, dense, compact, apply_mask);
}

void launch_dense_rowidft(const CartGeomDev& g, float2* dense, float2* qp, const float* mask_dense, cudaStream_t s) {
  dense_rowidft_kernel<<<g.C * g.T, 256, sizeof(float2) * g.W, s>>>(g, dense, qp, mask_dense);
}

cudaError_t configure_kernels() {
  // opt in to the full 227 KB of dynamic shared memory per CTA (sm_100)
  cudaError_t e = cudaFuncSetAttribute(ydft_kernel<KSPACE_KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);
  if (e != cudaSuccess) return e;
  for (int id : {96, 128, 160, 192, 256, 320, 1, 0}) {
#define SET_R(ID)                                                                                                  \
  e = cudaFuncSetAttribute(rows_kernel<8, ID>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);       \
  if (e == cudaSuccess)                                                                                            \
    e = cudaFuncSetAttribute(rows_kernel<12, ID>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);    \
  if (e == cudaSuccess)                                                                                            \
    e = cudaFuncSetAttribute(rows_kernel<KSPACE_KC, ID>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX)
    AVX_FFT_PLAN_DISPATCH(id, SET_R)
#undef SET_R
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace avx
