// Variational H1 coil-sensitivity estimation kernels (reference:
// CUDA/src/coil_construction.cpp:55-556, cartesian_coil_construction.cpp:23-86).
//
// Images are single W x H slices (coil images stacked [coil][H][W]); the 2D
// stencils are the (x, y) restriction of the 3D ones: gradient (D+x, D+y),
// symmetrised gradient (xx, yy, xy with 1/2 on the off-diagonal),
// divergences as their negative adjoints (utils.cpp:156-181, 525-568,
// 664-684, 817-844, 1078-1117).
#include <algorithm>

#include <cooperative_groups.h>

#include "coils.cuh"
#include "stencil.cuh"

namespace avx {

struct P2 {
  int x, y, W, H;
  long long i;
};

AVX_D P2 p2_of(int idx, int W, int H) {
  P2 p;
  p.x = idx % W;
  p.y = idx / W;
  p.W = W;
  p.H = H;
  p.i = idx;
  return p;
}

AVX_D void grad2(const float2* u, const P2& p, float2 (&g)[2]) {
  g[0] = d_fwd(u, p.i, p.x, p.W, 1);
  g[1] = d_fwd(u, p.i, p.y, p.H, p.W);
}
AVX_D float2 div2(const float2* y0, const float2* y1, const P2& p) {
  const float2 a = cadd(d_fwd_t(y0, p.i, p.x, p.W, 1), d_fwd_t(y1, p.i, p.y, p.H, p.W));
  return make_float2(-a.x, -a.y);
}
// SymmetricGradient2D (utils.cpp:525-556): (D-x v0, D-y v1, (D-y v0 + D-x v1) / 2)
AVX_D void symgrad2(const float2* v0, const float2* v1, const P2& p, float2 (&e)[3]) {
  e[0] = d_bwd(v0, p.i, p.x, p.W, 1);
  e[1] = d_bwd(v1, p.i, p.y, p.H, p.W);
  e[2] = cadd(cscale(d_bwd(v0, p.i, p.y, p.H, p.W), 0.5f), cscale(d_bwd(v1, p.i, p.x, p.W, 1), 0.5f));
}
// SymmetricDivergence2D (utils.cpp:1078-1117)
AVX_D void symdiv2(const float2* w0, const float2* w1, const float2* w2, const P2& p, float2 (&d)[2]) {
  float2 a = cadd(d_bwd_t(w0, p.i, p.x, p.W, 1), d_bwd_t(w2, p.i, p.y, p.H, p.W));
  d[0] = make_float2(-a.x, -a.y);
  a = cadd(d_bwd_t(w2, p.i, p.x, p.W, 1), d_bwd_t(w1, p.i, p.y, p.H, p.W));
  d[1] = make_float2(-a.x, -a.y);
}

// ---------------------------------------------------------------------------
// time-averaged reconstruction
// ---------------------------------------------------------------------------

__global__ void ta_sum_kernel(const float2* kdata, const float* mask, float2* out, int HW, int C, int T) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)C * HW) return;
  const int c = (int)(i / HW), p = (int)(i % HW);
  float2 s = czero();
  float m = 0.f;
  for (int t = 0; t < T; ++t) {
    s = cadd(s, kdata[((long long)t * C + c) * HW + p]);
    m += mask ? mask[(long long)t * HW + p] : 1.f;
  }
  m = fmaxf(m, 1.f);
  out[i] = make_float2(s.x / m, s.y / m);
}

__global__ void ta_combine_kernel(float2* crec, float2* u, int HW, int C, float scale, int apply_phase) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  float s = 0.f;
  float2 sum = czero();
  for (int c = 0; c < C; ++c) {
    const float2 v = cscale(crec[(long long)c * HW + p], scale);
    crec[(long long)c * HW + p] = v;
    s += cabs2(v);
    sum = cadd(sum, v);
  }
  float2 r = make_float2(sqrtf(s), 0.f);
  if (apply_phase) {
    const float ang = atan2f(sum.y, sum.x);
    r = cmul(r, make_float2(cosf(ang), sinf(ang)));
  }
  u[p] = r;
}

// ---------------------------------------------------------------------------
// H1 solve: (mu |u|^2 - Laplace_periodic) x = conj(u) mu |crec_c|, complex CG
// in FP64 (cg_forward_operation.h:47-70)
// ---------------------------------------------------------------------------

AVX_D double2 h1_apply(const double2* v, const double* muu, int x, int y, int W, int H) {
  const int i = y * W + x;
  const int xp = x + 1 == W ? 0 : x + 1, xm = x == 0 ? W - 1 : x - 1;
  const int yp = y + 1 == H ? 0 : y + 1, ym = y == 0 ? H - 1 : y - 1;
  const double2 c = v[i];
  const double2 a = v[y * W + xp], b = v[y * W + xm], d = v[yp * W + x], e = v[ym * W + x];
  const double m = muu[i] + 4.0;
  return make_double2(m * c.x - a.x - b.x - d.x - e.x, m * c.y - a.y - b.y - d.y - e.y);
}

template <int NT>
AVX_D double block_dsum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double r = 0.0;
  for (int k = 0; k < NT / 32; ++k) r += red[k];
  return r;
}

// Each coil's system is solved by a cluster of H1_CLUSTER CTAs (contiguous
// blocks of pixels per CTA).  The vectors stay in global
// memory; the stencil reads its neighbours there after a cluster barrier
// (release/acquire at cluster scope).  Every inner product is a block sum per
// CTA, the CTA sums written into a slot of every CTA's shared memory, and one
// cluster barrier, after which each CTA adds the slots in rank order: every
// CTA holds the same value, so all take the same branch of the stopping test.
#define H1_CLUSTER 8

__global__ void __cluster_dims__(H1_CLUSTER, 1, 1) __launch_bounds__(1024)
    h1_cg_cluster_kernel(const float2* u, const float2* crec, double mu, int W, int H, int max_it, double rel_tol,
                         double2* work, double* muu_buf, float2* out, int* iters) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double red[32];
  __shared__ double slots[2][H1_CLUSTER];  // the CTA sums of the two most recent reductions
  const int rank = (int)cl.block_rank();
  const int c = blockIdx.x / H1_CLUSTER;
  const int N = W * H;
  const int i0 = (int)((long long)N * rank / H1_CLUSTER), i1 = (int)((long long)N * (rank + 1) / H1_CLUSTER);
  double2* x = work + (size_t)c * 4 * N;
  double2* r = x + N;
  double2* p = r + N;
  double2* q = p + N;
  double* muu = muu_buf + (size_t)c * N;
  int nred = 0;
  auto csum = [&](double v) {
    v = block_dsum<1024>(v, red);
    double* buf = slots[nred & 1];
    if (threadIdx.x == 0)
      for (int k = 0; k < H1_CLUSTER; ++k) cl.map_shared_rank(buf, k)[rank] = v;
    cl.sync();
    double t = 0.0;
    for (int k = 0; k < H1_CLUSTER; ++k) t += buf[k];
    ++nred;
    return t;
  };
  double rr = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    const float2 uu = u[i];
    const double au2 = (double)uu.x * uu.x + (double)uu.y * uu.y;
    muu[i] = mu * au2;
    const float2 cr = crec[(size_t)c * N + i];
    const double ac = mu * sqrt((double)cr.x * cr.x + (double)cr.y * cr.y);
    const double2 y = make_double2((double)uu.x * ac, -(double)uu.y * ac);
    x[i] = make_double2(0.0, 0.0);
    r[i] = y;
    p[i] = y;
    rr += y.x * y.x + y.y * y.y;
  }
  rr = csum(rr);  // the barrier also publishes p and muu to the cluster
  const double rr0 = rr;
  int it = 0;
  for (; it < max_it && rr > rel_tol * rel_tol * rr0 && rr > 0.0; ++it) {
    double pq = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const double2 a = h1_apply(p, muu, i % W, i / W, W, H);
      q[i] = a;
      const double2 pv = p[i];
      pq += pv.x * a.x + pv.y * a.y;
    }
    pq = csum(pq);
    const double alpha = rr / pq;
    double rn = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const double2 pv = p[i], qv = q[i];
      double2 xv = x[i], rv = r[i];
      xv.x += alpha * pv.x;
      xv.y += alpha * pv.y;
      rv.x -= alpha * qv.x;
      rv.y -= alpha * qv.y;
      x[i] = xv;
      r[i] = rv;
      rn += rv.x * rv.x + rv.y * rv.y;
    }
    rn = csum(rn);
    const double beta = rn / rr;
    rr = rn;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      const double2 rv = r[i], pv = p[i];
      p[i] = make_double2(rv.x + beta * pv.x, rv.y + beta * pv.y);
    }
    cl.sync();  // the new p before any CTA applies the stencil to it
  }
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) out[(size_t)c * N + i] = make_float2((float)x[i].x, (float)x[i].y);
  if (rank == 0 && threadIdx.x == 0 && iters) iters[c] = it;
}

// b1 <- |b1_c / sqrt(sum_c |b1_c|^2)| (coil_construction.cpp:428-444)
__global__ void h1_normalize_kernel(float2* b1, int HW, int C) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  float s = 0.f;
  for (int c = 0; c < C; ++c) s += cabs2(b1[(long long)c * HW + p]);
  const float n = sqrtf(s);
  for (int c = 0; c < C; ++c) {
    const float2 v = b1[(long long)c * HW + p];
    const float2 w = make_float2(v.x / n, v.y / n);
    b1[(long long)c * HW + p] = make_float2(sqrtf(cabs2(w)), 0.f);
  }
}

// ---------------------------------------------------------------------------
// UTGV2Recon (coil_construction.cpp:75-215)
// ---------------------------------------------------------------------------

__global__ void utgv_prep_kernel(const float2* b10, const float2* crec0, const int* inds, int ninds, float tau, int HW,
                                 float2* Lw, float2* Ib) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  float2 lw = czero(), sb = czero();
  for (int k = 0; k < ninds; ++k) {
    const float2 b = b10[(long long)inds[k] * HW + p];
    const float2 cr = crec0[(long long)inds[k] * HW + p];
    lw = cadd(lw, cmulc(b, cr));
    sb = cadd(sb, cmulc(b, b));
  }
  Lw[p] = lw;
  // Ib = 1 / (1 + tau sumB1) (complex division of 1 by a real-valued complex)
  const float2 den = make_float2(1.f + tau * sb.x, tau * sb.y);
  const float dd = cabs2(den);
  Ib[p] = make_float2(den.x / dd, -den.y / dd);
}

// One UTGV2Recon iteration (coil_construction.cpp:75-215) in one kernel: the
// dual update (y1 += sigma (grad x1bar - x2bar), y2 += sigma E x2bar, each
// projected onto its ball) at this pixel and at the neighbours the primal
// update reads (the divergence: x - 1, y - W; the symmetrised divergence:
// x + 1, y + W), recomputed from the old extragradients and duals, then the
// primal update (x1 <- (x1 + tau (div y1 + Lw)) Ib, x2 += tau (y1 + div_sym
// y2), extragradients 2 new - old).  The extragradients and the duals are
// double-buffered; x1 and x2 are updated in place by their own thread.
__global__ void utgv_fused_kernel(CoilPD a, UtgvBuffers b) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.W * a.H) return;
  const P2 p = p2_of(idx, a.W, a.H);
  // the dual update at pixel (qx, qy)
  auto dual = [&](int qx, int qy, float2 (&y1)[2], float2 (&y2)[3]) {
    P2 q;
    q.x = qx;
    q.y = qy;
    q.W = a.W;
    q.H = a.H;
    q.i = (long long)qy * a.W + qx;
    float2 g[2], e[3];
    grad2(b.ext1_in, q, g);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const float2 d = csub(g[k], ldc(b.ext2_in[k], q.i));
      const float2 v = ldc(b.y1_in[k], q.i);
      y1[k] = make_float2(v.x + a.sigma * d.x, v.y + a.sigma * d.y);
    }
    symgrad2(b.ext2_in[0], b.ext2_in[1], q, e);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float2 v = ldc(b.y2_in[k], q.i);
      y2[k] = make_float2(v.x + a.sigma * e[k].x, v.y + a.sigma * e[k].y);
    }
    const float n1 = sqrtf(cabs2(y1[0]) + cabs2(y1[1]));
    const float n2 = sqrtf(cabs2(y2[0]) + cabs2(y2[1]) + 2.f * cabs2(y2[2]));
    const float d1 = fmaxf(1.f, a.s1 * n1), d2 = fmaxf(1.f, a.s2 * n2);
#pragma unroll
    for (int k = 0; k < 2; ++k) y1[k] = make_float2(y1[k].x / d1, y1[k].y / d1);
#pragma unroll
    for (int k = 0; k < 3; ++k) y2[k] = make_float2(y2[k].x / d2, y2[k].y / d2);
  };
  float2 y1[2], y2[3];
  dual(p.x, p.y, y1, y2);
#pragma unroll
  for (int k = 0; k < 2; ++k) b.y1_out[k][idx] = y1[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) b.y2_out[k][idx] = y2[k];
  float2 n1[2], n2[3];
  // div2 (d_fwd_t along x of y1_0, along y of y1_1), negated
  float2 xm = czero(), ym = czero();
  if (p.x > 0) {
    dual(p.x - 1, p.y, n1, n2);
    xm = n1[0];
  }
  if (p.y > 0) {
    dual(p.x, p.y - 1, n1, n2);
    ym = n1[1];
  }
  const float2 ax = csub(xm, p.x < a.W - 1 ? y1[0] : czero());
  const float2 ay = csub(ym, p.y < a.H - 1 ? y1[1] : czero());
  const float2 s2 = cadd(ax, ay);
  const float2 dv = make_float2(-s2.x, -s2.y);
  const float2 xo = a.x1[idx];
  float2 x1n = make_float2(xo.x + a.tau * dv.x, xo.y + a.tau * dv.y);
  const float2 lw = a.Lw[idx];
  x1n = make_float2(x1n.x + a.tau * lw.x, x1n.y + a.tau * lw.y);
  x1n = cmul(x1n, a.Ib[idx]);
  a.x1[idx] = x1n;
  b.ext1_out[idx] = make_float2(2.f * x1n.x - xo.x, 2.f * x1n.y - xo.y);
  // symdiv2 (d_bwd_t: w0 and w2 along x, w2 and w1 along y), negated
  float2 w0p = czero(), w2x = czero(), w2y = czero(), w1p = czero();
  if (p.x < a.W - 1) {
    dual(p.x + 1, p.y, n1, n2);
    w0p = n2[0];
    w2x = n2[2];
  }
  if (p.y < a.H - 1) {
    dual(p.x, p.y + 1, n1, n2);
    w1p = n2[1];
    w2y = n2[2];
  }
  const float2 z = czero();
  float2 sd[2];
  float2 t0 = cadd(p.x < a.W - 1 ? csub(y2[0], w0p) : z, p.y < a.H - 1 ? csub(y2[2], w2y) : z);
  sd[0] = make_float2(-t0.x, -t0.y);
  t0 = cadd(p.x < a.W - 1 ? csub(y2[2], w2x) : z, p.y < a.H - 1 ? csub(y2[1], w1p) : z);
  sd[1] = make_float2(-t0.x, -t0.y);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const float2 r = cadd(y1[k], sd[k]);
    const float2 x2 = a.x2[k][idx];
    const float2 m = make_float2(x2.x + a.tau * r.x, x2.y + a.tau * r.y);
    a.x2[k][idx] = m;
    b.ext2_out[k][idx] = make_float2(2.f * m.x - x2.x, 2.f * m.y - x2.y);
  }
}

// ---------------------------------------------------------------------------
// B1Recon (coil_construction.cpp:217-361)
// ---------------------------------------------------------------------------

__global__ void absmax_kernel(const float2* v, int n, unsigned* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float m = 0.f;
  if (i < n) m = sqrtf(cabs2(v[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  // non-negative floats order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void b1r_prep_kernel(const float2* u0, const unsigned* umax, const float2* crec, int coils, int HW,
                                float tau, float2* Lw, float2* Iu) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  const float mx = __uint_as_float(*umax);
  const float2 un = make_float2(u0[p].x / mx, u0[p].y / mx);
  const float2 sumU = make_float2(1.f + tau * cabs2(un), 0.f);
  const float2 iu = make_float2(1.f / sumU.x, 0.f);
  for (int c = 0; c < coils; ++c) {
    Lw[(long long)c * HW + p] = cmulc(un, crec[(long long)c * HW + p]);
    Iu[(long long)c * HW + p] = iu;
  }
}

// One B1Recon iteration (coil_construction.cpp:217-361) in one kernel: the
// dual update (y = (y + sigma grad xbar) / (1 + sigma / mu)) at this pixel and
// at the neighbours the divergence reads (x - 1 for the x component, x - W for
// the y component), recomputed from the old extragradient and duals, then the
// primal update (x <- (x + tau (div y + Lw)) Iu, extragradient 2 new - old).
// The extragradient and the duals are double-buffered (neighbouring threads
// read the old values while the owner writes the new ones); x is updated in
// place (read and written by its own thread only).
__global__ void b1r_fused_kernel(CoilPD a, int coils, B1Buffers b) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int HW = a.W * a.H;
  if (idx >= (long long)coils * HW) return;
  const int c = (int)(idx / HW);
  const int pix = (int)(idx % HW);
  const P2 p = p2_of(pix, a.W, a.H);
  const long long cb = (long long)c * HW;
  const float2* e = b.ext_in + cb;
  const float sc = 1.f / (1.f + a.sigma / a.mu);
  // dual component k at coil pixel q
  auto dual = [&](int k, int qx, int qy) {
    const long long q = (long long)qy * a.W + qx;
    const float2 g = k == 0 ? d_fwd(e, q, qx, a.W, 1) : d_fwd(e, q, qy, a.H, a.W);
    const float2 v = (k == 0 ? b.y0_in : b.y1_in)[cb + q];
    return cscale(make_float2(v.x + a.sigma * g.x, v.y + a.sigma * g.y), sc);
  };
  const float2 y0 = dual(0, p.x, p.y), y1 = dual(1, p.x, p.y);
  b.y0_out[idx] = y0;
  b.y1_out[idx] = y1;
  // divergence (div2 of coils.cu) from the new duals
  const float2 y0m = p.x > 0 ? dual(0, p.x - 1, p.y) : czero();
  const float2 y1m = p.y > 0 ? dual(1, p.x, p.y - 1) : czero();
  const float2 ax = csub(y0m, p.x < a.W - 1 ? y0 : czero());
  const float2 ay = csub(y1m, p.y < a.H - 1 ? y1 : czero());
  const float2 s2 = cadd(ax, ay);
  const float2 dv = make_float2(-s2.x, -s2.y);
  const float2 xo = a.x1[idx];
  float2 n1 = make_float2(xo.x + a.tau * dv.x, xo.y + a.tau * dv.y);
  const float2 lw = a.Lw[idx];
  n1 = cmul(make_float2(n1.x + a.tau * lw.x, n1.y + a.tau * lw.y), a.Ib[idx]);
  a.x1n[idx] = n1;
  b.ext_out[idx] = make_float2(2.f * n1.x - xo.x, 2.f * n1.y - xo.y);
}

__global__ void b1r_normalize_kernel(const float2* x, float2* out, int HW, int coils) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  float s = 0.f;
  for (int c = 0; c < coils; ++c) s += cabs2(x[(long long)c * HW + p]);
  const float n = sqrtf(s);
  for (int c = 0; c < coils; ++c) {
    const float2 v = x[(long long)c * HW + p];
    out[(long long)c * HW + p] = make_float2(v.x / n, v.y / n);
  }
}

// b1 = |absb1| * exp(i angle(x1))
__global__ void phase_apply_kernel(const float2* absb1, const float2* x1, float2* out, int HW) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  const float ang = atan2f(x1[p].y, x1[p].x);
  out[p] = cmul(absb1[p], make_float2(cosf(ang), sinf(ang)));
}

// w = sqrt(w*w + conj(b) b); crec_abs products and sums for the greedy order
__global__ void weight_update_kernel(float2* w, const float2* b, int HW) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  const float2 ww = cmul(w[p], w[p]);
  const float2 s = cadd(ww, cmulc(b[p], b[p]));
  // complex square root of a value with zero imaginary part here
  const float r = sqrtf(sqrtf(cabs2(s)));
  const float th = 0.5f * atan2f(s.y, s.x);
  w[p] = make_float2(r * cosf(th), r * sinf(th));
}

// u_in = absb1 * u * w; crec_in = crec * w
__global__ void greedy_inputs_kernel(const float2* absb1, const float2* u, const float2* w, const float2* crec,
                                     float2* u_in, float2* crec_in, int HW) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  u_in[p] = cmul(cmul(absb1[p], u[p]), w[p]);
  crec_in[p] = cmul(crec[p], w[p]);
}

// FP64 sums over a coil image of |a| (b == null) or |a| |b|
__global__ void abs_sum_kernel(const float2* a, const float2* b, int HW, double* partial) {
  __shared__ double red[32];
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < HW; i += gridDim.x * blockDim.x) {
    float v = sqrtf(cabs2(a[i]));
    if (b) v *= sqrtf(cabs2(b[i]));
    acc[0] += (double)v;
  }
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

static inline unsigned nb256(long long n) { return (unsigned)((n + 255) / 256); }

void launch_ta_sum(const float2* kdata, const float* mask, float2* out, int HW, int C, int T, cudaStream_t s) {
  ta_sum_kernel<<<nb256((long long)C * HW), 256, 0, s>>>(kdata, mask, out, HW, C, T);
}
void launch_ta_combine(float2* crec, float2* u, int HW, int C, float scale, int apply_phase, cudaStream_t s) {
  ta_combine_kernel<<<nb256(HW), 256, 0, s>>>(crec, u, HW, C, scale, apply_phase);
}
void launch_h1_cg(const float2* u, const float2* crec, double mu, int W, int H, int C, int max_it, double rel_tol,
                  double2* work, double* muu, float2* out, int* iters, cudaStream_t s) {
  h1_cg_cluster_kernel<<<C * H1_CLUSTER, 1024, 0, s>>>(u, crec, mu, W, H, max_it, rel_tol, work, muu, out, iters);
}
void launch_h1_normalize(float2* b1, int HW, int C, cudaStream_t s) {
  h1_normalize_kernel<<<nb256(HW), 256, 0, s>>>(b1, HW, C);
}
void launch_utgv_prep(const float2* b10, const float2* crec0, const int* inds, int ninds, float tau, int HW,
                      float2* Lw, float2* Ib, cudaStream_t s) {
  utgv_prep_kernel<<<nb256(HW), 256, 0, s>>>(b10, crec0, inds, ninds, tau, HW, Lw, Ib);
}
void launch_utgv_fused(const CoilPD& a, const UtgvBuffers& b, cudaStream_t s) {
  utgv_fused_kernel<<<nb256((long long)a.W * a.H), 256, 0, s>>>(a, b);
}
void launch_absmax(const float2* v, int n, unsigned* out, cudaStream_t s) {
  absmax_kernel<<<nb256(n), 256, 0, s>>>(v, n, out);
}
void launch_b1r_prep(const float2* u0, const unsigned* umax, const float2* crec, int coils, int HW, float tau,
                     float2* Lw, float2* Iu, cudaStream_t s) {
  b1r_prep_kernel<<<nb256(HW), 256, 0, s>>>(u0, umax, crec, coils, HW, tau, Lw, Iu);
}
void launch_b1r_fused(const CoilPD& a, int coils, const B1Buffers& b, cudaStream_t s) {
  const long long n = (long long)coils * a.W * a.H;
  b1r_fused_kernel<<<nb256(n), 256, 0, s>>>(a, coils, b);
}
void launch_b1r_normalize(const float2* x, float2* out, int HW, int coils, cudaStream_t s) {
  b1r_normalize_kernel<<<nb256(HW), 256, 0, s>>>(x, out, HW, coils);
}
void launch_phase_apply(const float2* absb1, const float2* x1, float2* out, int HW, cudaStream_t s) {
  phase_apply_kernel<<<nb256(HW), 256, 0, s>>>(absb1, x1, out, HW);
}
void launch_weight_update(float2* w, const float2* b, int HW, cudaStream_t s) {
  weight_update_kernel<<<nb256(HW), 256, 0, s>>>(w, b, HW);
}
void launch_greedy_inputs(const float2* absb1, const float2* u, const float2* w, const float2* crec, float2* u_in,
                          float2* crec_in, int HW, cudaStream_t s) {
  greedy_inputs_kernel<<<nb256(HW), 256, 0, s>>>(absb1, u, w, crec, u_in, crec_in, HW);
}
void launch_abs_sum(const float2* a, const float2* b, int HW, double* partial, int nblocks, cudaStream_t s) {
  abs_sum_kernel<<<nblocks, 256, 0, s>>>(a, b, HW, partial);
}

// v *= f (agile::scale of the data normalisation, raw_data_preparation.cpp:792, 842)
__global__ void cscale_kernel(float2* v, long long n, float f) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = v[i];
    v[i] = make_float2(a.x * f, a.y * f);
  }
}

void launch_cscale(float2* v, long long n, float f, cudaStream_t s) {
  const long long nb = std::min<long long>((n + 255) / 256, 148 * 16);
  if (nb > 0) cscale_kernel<<<(int)nb, 256, 0, s>>>(v, n, f);
}

}  // namespace avx
