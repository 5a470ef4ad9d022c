// Radial gridding operator kernels (see radial.cuh and oracle/radial.py).
//
// Forward  (image -> samples): row DFT fused with pad+deapodise (sign -1) ->
//                              column DFT -> interpolate
// Adjoint  (samples -> image): spread (sector gather) -> column DFT (sign +1) ->
//                              row DFT fused with crop+deapodise+coil-combine
// The spreading step gathers: one CTA per (frame, sector) owns the sector's
// grid cells and reads every sample of the 3x3 neighbouring sectors, so each
// grid value is a fixed-order sum (no floating-point atomics, deterministic).
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "fft.cuh"
#include "radial.cuh"

namespace avx {

#define RAD_FFT_KC 16
#define RAD_ADJ_KC 8  // image rows per CTA of the adjoint's fused row pass
#define RAD_SPREAD_BATCH 64
#define RAD_MAX_SW 32  // largest sector width (the operator accepts 2..32; one thread per cell)

// tapered Kaiser-Bessel weight at offset u (grid units); zero for |u| >= J/2
AVX_D float kbw(float u, const RadialGeomDev& g) {
  if (!(fabsf(u) < 0.5f * g.J)) return 0.f;
  const float r = 2.f * u / g.J;
  return (cyl_bessel_i0f(g.beta * sqrtf(fmaxf(1.f - r * r, 0.f))) - 1.f) * g.kb_norm;
}

AVX_D int imod(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}

// a mod n for -n <= a < 2n.  Window offsets on the grid lie in that range:
// window starts g0 = floor(k G - J/2) with k in [-1/2, 1/2) lie in
// [-G/2 - J/2 - 1, G/2), and the operator requires G > J + 2.
AVX_D int wrap1(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

// grid index -> image index along one axis, or -1 outside the image
AVX_D int grid_to_img(int m, int d, int G) {
  const int h = d / 2;
  if (m < d - h) return m + h;
  if (m >= G - h) return m - G + h;
  return -1;
}

// Forward, first pass: 16 grid rows of slice (f, c) per CTA, each formed from
// the zero-padded, deapodised b1 (in - in2) and transformed along x with
// sign -1.  Chunks without image rows store zeros.
template <int PLAN>
__global__ void __launch_bounds__(256) rad_rows_fwd_kernel(RArgs a) {
  constexpr int KC = RAD_FFT_KC, KCP = AVX_FFT_PITCH(KC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RadialGeomDev& g = a.g;
  const int G = PLAN > 1 ? PLAN : g.Gx;  // compile-time with a fixed plan
  const int slice = blockIdx.y;
  const int c = slice % g.C, f = slice / g.C;
  const int r0 = blockIdx.x * KC;
  const int rows = min(KC, g.Gy - r0);
  float2* base = a.grid + (long long)slice * g.Gx * g.Gy;
  bool any = false;  // the same for every thread of the CTA
  for (int kk = 0; kk < rows; ++kk) any = any || grid_to_img(r0 + kk, g.H, g.Gy) >= 0;
  if (!any) {
    for (int e = threadIdx.x; e < rows * G; e += blockDim.x) base[(long long)r0 * G + e] = czero();
    return;
  }
  float2* A = reinterpret_cast<float2*>(smem_raw);
  float2* B = A + (size_t)G * KCP;
  float2* tw = B + (size_t)G * KCP;
  __shared__ int splan[12];
  stage_plan(g.radx, splan);
  for (int j = threadIdx.x; j < G; j += blockDim.x) tw[j] = g.twgx[j];
  for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
    const int kk = e / G, mx = e % G;
    const int ny = kk < rows ? grid_to_img(r0 + kk, g.H, g.Gy) : -1, nx = grid_to_img(mx, g.W, g.Gx);
    float2 v = czero();
    if (ny >= 0 && nx >= 0) {
      const long long pi = ((long long)f * g.H + ny) * g.W + nx;
      float2 u = a.in[pi];
      if (a.in2) u = csub(u, a.in2[pi]);
      v = cscale(cmul(a.b1[((long long)c * g.H + ny) * g.W + nx], u), g.inv_psi_y[ny] * g.inv_psi_x[nx]);
    }
    A[mx * KCP + kk] = v;
  }
  __syncthreads();
  const float2* R = row_fft_planned<KC, PLAN, -1>(A, B, tw, G, g.nradx, splan);
  for (int e = threadIdx.x; e < rows * G; e += blockDim.x) {
    const int kk = e / G, x = e % G;
    base[(long long)(r0 + kk) * G + x] = R[x * KCP + kk];
  }
}

// Adjoint, last pass: RAD_ADJ_KC image rows of frame f per CTA.  For every
// coil the matching grid rows are transformed along x with sign +1, cropped,
// multiplied by conj(b1) and summed; the sum is deapodised into img.
template <int PLAN>
__global__ void __launch_bounds__(256) rad_rows_adj_kernel(RArgs a, float2* img) {
  if (a.st && a.st->stop) return;
  constexpr int KC = RAD_ADJ_KC, KCP = AVX_FFT_PITCH(KC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RadialGeomDev& g = a.g;
  const int G = PLAN > 1 ? PLAN : g.Gx, W = g.W;  // G compile-time with a fixed plan
  const int f = blockIdx.y;
  const int y0 = blockIdx.x * KC;
  const int rows = min(KC, g.H - y0);
  float2* A = reinterpret_cast<float2*>(smem_raw);
  float2* B = A + (size_t)G * KCP;
  float2* tw = B + (size_t)G * KCP;
  float2* acc = tw + G;  // [KC][W]
  __shared__ int splan[12];
  stage_plan(g.radx, splan);
  for (int j = threadIdx.x; j < G; j += blockDim.x) tw[j] = g.twgx[j];
  for (int e = threadIdx.x; e < KC * W; e += blockDim.x) acc[e] = czero();
  for (int c = 0; c < g.C; ++c) {
    const float2* base = a.grid + ((long long)f * g.C + c) * g.Gx * g.Gy;
    __syncthreads();
    for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
      const int kk = e / G, mx = e % G;
      const int my = imod(y0 + kk - g.H / 2, g.Gy);
      A[mx * KCP + kk] = kk < rows ? base[(long long)my * G + mx] : czero();
    }
    __syncthreads();
    const float2* R = row_fft_planned<KC, PLAN, +1>(A, B, tw, G, g.nradx, splan);
    // each thread owns the same entries of acc in every coil pass
    for (int e = threadIdx.x; e < rows * W; e += blockDim.x) {
      const int kk = e / W, x = e % W;
      const int mx = imod(x - W / 2, G);
      const float2 bv = a.b1[((long long)c * g.H + y0 + kk) * W + x];
      acc[e] = cadd(acc[e], cmulc(bv, R[mx * KCP + kk]));
    }
  }
  for (int e = threadIdx.x; e < rows * W; e += blockDim.x) {
    const int kk = e / W, x = e % W, y = y0 + kk;
    img[((long long)f * g.H + y) * W + x] = cscale(acc[e], g.inv_psi_y[y] * g.inv_psi_x[x]);
  }
}

// columns (along y) of 16 grid columns per CTA, in place
template <int PLAN, int SIGN>
__global__ void __launch_bounds__(256) rad_fft_cols_kernel(RArgs a) {
  constexpr int KC = RAD_FFT_KC, KCP = AVX_FFT_PITCH(KC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const RadialGeomDev& g = a.g;
  const int G = PLAN > 1 ? PLAN : g.Gy;  // compile-time with a fixed plan
  float2* A = reinterpret_cast<float2*>(smem_raw);
  float2* B = A + (size_t)G * KCP;
  float2* tw = B + (size_t)G * KCP;
  const int slice = blockIdx.y;
  const int c0 = blockIdx.x * KC;
  const int cols = min(KC, g.Gx - c0);
  float2* base = a.grid + (long long)slice * g.Gx * g.Gy;
  __shared__ int splan[12];
  stage_plan(g.rady, splan);
  for (int j = threadIdx.x; j < G; j += blockDim.x) tw[j] = g.twgy[j];
  for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
    const int kk = e % KC, y = e / KC;
    A[y * KCP + kk] = kk < cols ? base[(long long)y * g.Gx + c0 + kk] : czero();
  }
  __syncthreads();
  const float2* R = row_fft_planned<KC, PLAN, SIGN>(A, B, tw, G, g.nrady, splan);
  for (int e = threadIdx.x; e < KC * G; e += blockDim.x) {
    const int kk = e % KC, y = e / KC;
    if (kk < cols) base[(long long)y * g.Gx + c0 + kk] = R[y * KCP + kk];
  }
}

// window of one sample along one axis: start index (unwrapped) and weights
template <int NW>
AVX_D int sample_window(float kappa, const RadialGeomDev& g, float (&w)[NW]) {
  const int g0 = (int)floorf(kappa - 0.5f * g.J);
#pragma unroll
  for (int o = 0; o < NW; ++o) w[o] = kbw(kappa - (float)(g0 + o), g);
  return g0;
}

template <int NW>
__global__ void rad_window_kernel(RadialGeomDev g, int2* win0, float* winw) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)g.T * g.S;
       i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i / g.S), s = (int)(i % g.S);
    float wx[NW], wy[NW];
    const int g0x = sample_window<NW>(g.traj[((long long)f * 2 + 0) * g.S + s] * (float)g.Gx, g, wx);
    const int g0y = sample_window<NW>(g.traj[((long long)f * 2 + 1) * g.S + s] * (float)g.Gy, g, wy);
    win0[i] = make_int2(g0x, g0y);
#pragma unroll
    for (int o = 0; o < NW; ++o) {
      winw[i * 2 * NW + o] = wx[o];
      winw[i * 2 * NW + NW + o] = wy[o];
    }
  }
}

template <int NW>
__global__ void __launch_bounds__(256) rad_interp_kernel(RArgs a, int mode) {
  if (a.st && a.st->stop && mode != 3) return;
  __shared__ double red[32 * 3];
  const RadialGeomDev& g = a.g;
  // one thread per (frame, coil, sample), in the layout of z and d
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double acc_r[3] = {0.0, 0.0, 0.0};
  if (i < (long long)g.T * g.C * g.S) {
    const int s = (int)(i % g.S);
    const long long fc = i / g.S;  // f * C + c
    const int f = (int)(fc / g.C);
    const long long fs = (long long)f * g.S + s;
    const int2 g0 = g.win0[fs];
    const int g0x = g0.x, g0y = g0.y;
    float wx[NW], wy[NW];
#pragma unroll
    for (int o = 0; o < NW; ++o) {
      wx[o] = g.winw[fs * 2 * NW + o];
      wy[o] = g.winw[fs * 2 * NW + NW + o];
    }
    int ix[NW], iy[NW];
#pragma unroll
    for (int o = 0; o < NW; ++o) {
      ix[o] = wrap1(g0x + o, g.Gx);
      iy[o] = wrap1(g0y + o, g.Gy);
    }
    const float sc = g.sqrt_w[fs] * g.norm;
    const float sig = a.st ? (float)a.st->sigma : 0.f;
    const float zscale = (mode == 0) ? (float)(1.0 / (1.0 + a.st->sigma / (double)a.lam)) : 1.f;
    {
      const float2* gr = a.grid + fc * g.Gx * g.Gy;
      float2 v = czero();
#pragma unroll
      for (int oy = 0; oy < NW; ++oy) {
        float2 row = czero();
#pragma unroll
        for (int ox = 0; ox < NW; ++ox) {
          const float2 q = gr[(long long)iy[oy] * g.Gx + ix[ox]];
          row.x = fmaf(wx[ox], q.x, row.x);
          row.y = fmaf(wx[ox], q.y, row.y);
        }
        v.x = fmaf(wy[oy], row.x, v.x);
        v.y = fmaf(wy[oy], row.y, v.y);
      }
      const float2 k = cscale(v, sc);
      const long long zi = i;
      if (mode == 0) {
        // z += sigma K x; z = (z - sigma d) / (1 + sigma / lambda)   (tgv2.cpp:254-264)
        const float2 zo = a.z[zi], dv = a.d[zi];
        float2 zn = make_float2(zo.x + sig * k.x, zo.y + sig * k.y);
        zn = make_float2(zn.x - sig * dv.x, zn.y - sig * dv.y);
        a.z[zi] = cscale(zn, zscale);
      } else if (mode == 1) {
        acc_r[0] += (double)cabs2(k);
      } else if (mode == 2) {
        const float2 zo = a.z[zi], dv = a.d[zi];
        acc_r[0] += (double)cabs2(csub(k, dv));
        acc_r[1] += (double)dv.x * zo.x + (double)dv.y * zo.y;
        acc_r[2] += (double)cabs2(zo);
      } else {
        a.out[zi] = k;
      }
    }
  }
  if (mode == 1 || mode == 2) {
    block_sum<3>(acc_r, red);
    if (threadIdx.x == 0) {
      const int nb = gridDim.x;
      a.partial[blockIdx.x] = acc_r[0];
      a.partial[nb + blockIdx.x] = acc_r[1];
      a.partial[2 * nb + blockIdx.x] = acc_r[2];
    }
  }
}

// one CTA per (sector, frame); thread = grid cell of the sector; CC coils
// accumulated per pass over the sector's work list: the samples whose window
// reaches the sector, in the order of the 3x3 neighbouring sectors and of the
// sorted order within each (built with the operator).  The CTAs are numbered
// through g.spread_blocks, longest list first, so that the central sectors
// (which every spoke crosses) start in the first wave.
template <int NW, int CC>
__global__ void rad_spread_kernel(RArgs a, const float2* __restrict__ samples) {
  if (a.st && a.st->stop) return;
  constexpr int NB = RAD_SPREAD_BATCH, NBP = NB + 1;  // NBP: padded rows, conflict-free column reads
  const RadialGeomDev& g = a.g;
  __shared__ int s_g0x[NB], s_g0y[NB];
  __shared__ float s_wx[NW][NBP], s_wy[NW][NBP];
  __shared__ float2 s_v[CC][NB];
  // per sector row: the staged samples whose window covers that row (two
  // batches' worth, alternating), so that a cell visits only those
  __shared__ unsigned long long s_rowm[2][RAD_MAX_SW];
  const int nsec = g.nsx * g.nsy;
  const int blk = g.spread_blocks[blockIdx.x];
  const int f = blk / nsec;
  const int sec = blk - f * nsec;
  const int sxi = sec % g.nsx, syi = sec / g.nsx;
  const int X0 = sxi * g.sw, Y0 = syi * g.sw;
  const int lx = threadIdx.x % g.sw, ly = threadIdx.x / g.sw;
  const int gx = X0 + lx, gy = Y0 + ly;
  const bool active = gx < g.Gx && gy < g.Gy;
  const int* list = g.spread_list + g.spread_off[blk];
  const int tot = g.spread_off[blk + 1] - g.spread_off[blk];
  for (int i = threadIdx.x; i < RAD_MAX_SW; i += blockDim.x) s_rowm[0][i] = s_rowm[1][i] = 0ull;
  __syncthreads();
  const int swy = min(g.sw, g.Gy - Y0);
  int bi = 0;  // batch counter over all coil passes (selects s_rowm)
  for (int c0 = 0; c0 < g.C; c0 += CC) {
    const int cc = min(CC, g.C - c0);
    float2 acc[CC];
#pragma unroll
    for (int k = 0; k < CC; ++k) acc[k] = czero();
    for (int b0 = 0; b0 < tot; b0 += NB, ++bi) {
      const int nb = min(NB, tot - b0);
      unsigned long long* rowm = s_rowm[bi & 1];
      __syncthreads();
      for (int e = threadIdx.x; e < nb; e += blockDim.x) {
        const int j = list[b0 + e];
        const long long fj = (long long)f * g.S + j;
        const int2 g0 = g.win0[fj];
        // the sector rows the window covers (bitwise OR: the result does not depend on the order)
#pragma unroll
        for (int o = 0; o < NW; ++o) {
          const int ly = wrap1(g0.y + o, g.Gy) - Y0;
          if (ly >= 0 && ly < swy) atomicOr(&rowm[ly], 1ull << e);
        }
        s_g0x[e] = g0.x;
        s_g0y[e] = g0.y;
#pragma unroll
        for (int o = 0; o < NW; ++o) {
          s_wx[o][e] = g.winw[fj * 2 * NW + o];
          s_wy[o][e] = g.winw[fj * 2 * NW + NW + o];
        }
        const float sc = g.sqrt_w[fj] * g.norm;
#pragma unroll
        for (int kc = 0; kc < CC; ++kc)
          s_v[kc][e] = kc < cc ? cscale(samples[((long long)f * g.C + c0 + kc) * g.S + j], sc) : czero();
      }
      __syncthreads();
      unsigned long long m = active ? rowm[ly] : 0ull;
      // the other batch's row masks are free again (every thread read them
      // before this batch's first barrier)
      for (int i = threadIdx.x; i < RAD_MAX_SW; i += blockDim.x) s_rowm[(bi + 1) & 1][i] = 0ull;
      if (!active) continue;
      while (m) {  // the staged samples covering this row, in staging order
        const int e = __ffsll((long long)m) - 1;
        m &= m - 1;
        // window starts lie within J of the grid, so one wrap suffices
        const int ox = wrap1(gx - s_g0x[e], g.Gx), oy = wrap1(gy - s_g0y[e], g.Gy);
        if (ox < NW && oy < NW) {
          const float w = s_wx[ox][e] * s_wy[oy][e];
#pragma unroll
          for (int k = 0; k < CC; ++k) {
            acc[k].x = fmaf(w, s_v[k][e].x, acc[k].x);
            acc[k].y = fmaf(w, s_v[k][e].y, acc[k].y);
          }
        }
      }
    }
    if (active) {
#pragma unroll
      for (int k = 0; k < CC; ++k)
        if (k < cc) a.grid[(((long long)f * g.C + c0 + k) * g.Gy + gy) * g.Gx + gx] = acc[k];
    }
  }
}

// ---------------------------------------------------------------------------

size_t radial_fft_smem_bytes(int G) { return sizeof(float2) * (2 * (size_t)G * AVX_FFT_PITCH(RAD_FFT_KC) + G); }
size_t radial_adj_smem_bytes(int G, int W) {
  return sizeof(float2) * (2 * (size_t)G * AVX_FFT_PITCH(RAD_ADJ_KC) + G + (size_t)RAD_ADJ_KC * W);
}

int radial_interp_blocks(const RadialGeomDev& g) { return (int)(((long long)g.T * g.C * g.S + 255) / 256); }

cudaError_t configure_radial_kernels() {
  cudaError_t e = cudaSuccess;
  for (int id : {96, 128, 160, 192, 256, 320, 1, 0}) {
#define SET_K(ID)                                                                                                   \
  e = cudaFuncSetAttribute(rad_fft_cols_kernel<ID, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX); \
  if (e == cudaSuccess)                                                                                             \
    e = cudaFuncSetAttribute(rad_fft_cols_kernel<ID, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);  \
  if (e == cudaSuccess)                                                                                             \
    e = cudaFuncSetAttribute(rad_rows_fwd_kernel<ID>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);     \
  if (e == cudaSuccess)                                                                                             \
    e = cudaFuncSetAttribute(rad_rows_adj_kernel<ID>, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX)
    AVX_FFT_PLAN_DISPATCH(id, SET_K)
#undef SET_K
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// every FFT kernel runs 256 threads, as the compile-time plans assume
void launch_rad_forward_grid(const RArgs& a, cudaStream_t s) {
  dim3 gr((a.g.Gy + RAD_FFT_KC - 1) / RAD_FFT_KC, a.g.C * a.g.T);
#define CALL_F(ID) rad_rows_fwd_kernel<ID><<<gr, 256, radial_fft_smem_bytes(a.g.Gx), s>>>(a)
  AVX_FFT_PLAN_DISPATCH(fft_plan_id(a.g.Gx, a.g.nradx, a.g.radx), CALL_F)
#undef CALL_F
  dim3 gc((a.g.Gx + RAD_FFT_KC - 1) / RAD_FFT_KC, a.g.C * a.g.T);
#define CALL_C(ID) rad_fft_cols_kernel<ID, -1><<<gc, 256, radial_fft_smem_bytes(a.g.Gy), s>>>(a)
  AVX_FFT_PLAN_DISPATCH(fft_plan_id(a.g.Gy, a.g.nrady, a.g.rady), CALL_C)
#undef CALL_C
}

void launch_rad_adjoint_image(const RArgs& a, float2* img, cudaStream_t s) {
  dim3 gc((a.g.Gx + RAD_FFT_KC - 1) / RAD_FFT_KC, a.g.C * a.g.T);
#define CALL_C(ID) rad_fft_cols_kernel<ID, 1><<<gc, 256, radial_fft_smem_bytes(a.g.Gy), s>>>(a)
  AVX_FFT_PLAN_DISPATCH(fft_plan_id(a.g.Gy, a.g.nrady, a.g.rady), CALL_C)
#undef CALL_C
  dim3 gr((a.g.H + RAD_ADJ_KC - 1) / RAD_ADJ_KC, a.g.T);
#define CALL_A(ID) rad_rows_adj_kernel<ID><<<gr, 256, radial_adj_smem_bytes(a.g.Gx, a.g.W), s>>>(a, img)
  AVX_FFT_PLAN_DISPATCH(fft_plan_id(a.g.Gx, a.g.nradx, a.g.radx), CALL_A)
#undef CALL_A
}

#define RAD_NW_DISPATCH(NWV, CALL) \
  switch (NWV) {                   \
    case 2: CALL(2); break;        \
    case 3: CALL(3); break;        \
    case 4: CALL(4); break;        \
    case 5: CALL(5); break;        \
    case 6: CALL(6); break;        \
    case 7: CALL(7); break;        \
    default: CALL(8); break;       \
  }

void launch_rad_interp(const RArgs& a, int mode, cudaStream_t s) {
  const int nb = radial_interp_blocks(a.g);
#define CALL_I(N) rad_interp_kernel<N><<<nb, 256, 0, s>>>(a, mode)
  RAD_NW_DISPATCH(a.g.nw, CALL_I)
#undef CALL_I
}

// ---------------------------------------------------------------------------
// Per-sample tables of an operator, built on the device.
// ---------------------------------------------------------------------------

__global__ void rad_validate_kernel(const float* traj, long long nt, const float* dens, long long nd, int* flags) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nt; i += (long long)gridDim.x * blockDim.x)
    if (!(fabsf(traj[i]) <= 0.5f)) atomicOr(flags, 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nd; i += (long long)gridDim.x * blockDim.x)
    if (!(dens[i] >= 0.f)) atomicOr(flags, 2);
}

// sector of every sample in float32 arithmetic (multiply, wrap, divide:
// each rounded once), key f nsec + sector, value the sample index, the
// per-key counts, and sqrt(w) per sample
__global__ void rad_keys_kernel(RadialGeomDev g, const float* dens, float* sqrt_w, int* key, int* val, int* cnt) {
  const int nsec = g.nsx * g.nsy;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)g.T * g.S;
       i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i / g.S), s = (int)(i % g.S);
    float px = __fmul_rn(g.traj[((long long)f * 2 + 0) * g.S + s], (float)g.Gx);
    float py = __fmul_rn(g.traj[((long long)f * 2 + 1) * g.S + s], (float)g.Gy);
    if (px < 0.f) px = __fadd_rn(px, (float)g.Gx);
    if (py < 0.f) py = __fadd_rn(py, (float)g.Gy);
    int sx = (int)floorf(__fdiv_rn(px, (float)g.sw)), sy = (int)floorf(__fdiv_rn(py, (float)g.sw));
    sx = min(max(sx, 0), g.nsx - 1);
    sy = min(max(sy, 0), g.nsy - 1);
    const int k = f * nsec + sy * g.nsx + sx;
    key[i] = k;
    val[i] = s;
    atomicAdd(cnt + k, 1);
    sqrt_w[i] = (float)sqrt((double)dens[i]);
  }
}

// sec_start[f][k] = offset of frame f's sector k within the frame's sorted order
__global__ void rad_sec_start_kernel(RadialGeomDev g, const int* off, int* sec_start) {
  const int nsec = g.nsx * g.nsy;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)g.T * (nsec + 1);
       i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i / (nsec + 1)), k = (int)(i % (nsec + 1));
    sec_start[i] = k < nsec ? off[(long long)f * nsec + k] - f * g.S : g.S;
  }
}

// The spreading work list of (frame, sector) item `it`, one warp per item:
// the samples of the distinct 3x3 neighbouring sectors in (dy, dx) order,
// each sector's in sorted order, that pass the window test of
// rad_spread_kernel.  Counts (list == nullptr) or writes them from off[it].
__global__ void rad_lists_kernel(RadialGeomDev g, const int* order, const int* sec_start, const int2* win0,
                                 int* count, const int* off, int* list) {
  const int nsec = g.nsx * g.nsy;
  const int lane = threadIdx.x & 31;
  const long long it = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (it >= (long long)g.T * nsec) return;
  const int f = (int)(it / nsec), sec = (int)(it % nsec);
  const int sxi = sec % g.nsx, syi = sec / g.nsx;
  const int X0 = sxi * g.sw, Y0 = syi * g.sw;
  const int swx = min(g.sw, g.Gx - X0), swy = min(g.sw, g.Gy - Y0);
  const int dxn = g.nsx >= 3 ? 3 : g.nsx, dyn = g.nsy >= 3 ? 3 : g.nsy;
  const int* ord = order + (long long)f * g.S;
  const int* st = sec_start + (long long)f * (nsec + 1);
  int n = 0;
  int* out = list ? list + off[it] : nullptr;
  for (int dy = 0; dy < dyn; ++dy)
    for (int dx = 0; dx < dxn; ++dx) {
      const int nx = imod(sxi + (dxn == 3 ? dx - 1 : dx), g.nsx);
      const int ny = imod(syi + (dyn == 3 ? dy - 1 : dy), g.nsy);
      const int ns = ny * g.nsx + nx;
      for (int q0 = st[ns]; q0 < st[ns + 1]; q0 += 32) {
        const int q = q0 + lane;
        bool hit = false;
        int j = 0;
        if (q < st[ns + 1]) {
          j = ord[q];
          const int2 a0 = win0[(long long)f * g.S + j];
          const int dx0 = wrap1(X0 - a0.x, g.Gx), dy0 = wrap1(Y0 - a0.y, g.Gy);
          hit = (dx0 < g.nw || dx0 + swx > g.Gx) && (dy0 < g.nw || dy0 + swy > g.Gy);
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (out && hit) out[n + __popc(m & ((1u << lane) - 1u))] = j;
        n += __popc(m);
      }
    }
  if (!list && lane == 0) count[it] = n;
}

__global__ void rad_list_len_kernel(const int* off, int n, int* len) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) len[i] = off[i + 1] - off[i];
}

__global__ void rad_iota_kernel(int* v, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// stream-ordered scratch memory, returned on its stream when it goes out of scope
struct AsyncScratch {
  void* p = nullptr;
  cudaStream_t s;
  explicit AsyncScratch(cudaStream_t st) : s(st) {}
  ~AsyncScratch() {
    if (p) cudaFreeAsync(p, s);
  }
  cudaError_t alloc(size_t bytes) { return cudaMallocAsync(&p, bytes, s); }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

static int key_bits(long long n) {
  int b = 1;
  while ((1ll << b) < n) ++b;
  return b;
}

cudaError_t rad_validate(const float* traj, long long nt, const float* dens, long long nd, int* flags_host,
                         cudaStream_t s) {
  AsyncScratch d(s);
  cudaError_t e = d.alloc(sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(d.p, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  rad_validate_kernel<<<148 * 8, 256, 0, s>>>(traj, nt, dens, nd, d.as<int>());
  e = cudaMemcpyAsync(flags_host, d.p, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

cudaError_t rad_build_order(const RadialGeomDev& g, const float* dens, float* sqrt_w, int* order, int* sec_start,
                            cudaStream_t s) {
  const long long n = (long long)g.T * g.S;
  const long long nk = (long long)g.T * g.nsx * g.nsy;
  size_t tb_sort = 0, tb_scan = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, tb_sort, (int*)nullptr, (int*)nullptr, (int*)nullptr,
                                                  order, (int)n, 0, key_bits(nk), s);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, (int*)nullptr, (int*)nullptr, (int)nk, s);
  AsyncScratch keys(s), counts(s), tmp(s);
  if (e == cudaSuccess) e = keys.alloc(3 * n * sizeof(int));
  if (e == cudaSuccess) e = counts.alloc(2 * (nk + 1) * sizeof(int));
  if (e == cudaSuccess) e = tmp.alloc(std::max(tb_sort, tb_scan) + 16);
  if (e == cudaSuccess) e = cudaMemsetAsync(counts.p, 0, (nk + 1) * sizeof(int), s);
  if (e != cudaSuccess) return e;
  int *key = keys.as<int>(), *key2 = key + n, *val = key + 2 * n;
  int *cnt = counts.as<int>(), *off = cnt + nk + 1;
  const int nb = (int)std::min<long long>((n + 255) / 256, 148 * 16);
  rad_keys_kernel<<<nb, 256, 0, s>>>(g, dens, sqrt_w, key, val, cnt);
  // a stable sort: within a key, samples stay in index order
  e = cub::DeviceRadixSort::SortPairs(tmp.p, tb_sort, key, key2, val, order, (int)n, 0, key_bits(nk), s);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp.p, tb_scan, cnt, off, (int)nk, s);
  if (e == cudaSuccess) {
    const long long ns = (long long)g.T * (g.nsx * g.nsy + 1);
    rad_sec_start_kernel<<<(int)std::min<long long>((ns + 255) / 256, 148 * 16), 256, 0, s>>>(g, off, sec_start);
    e = cudaGetLastError();
  }
  return e;
}

cudaError_t rad_count_lists(const RadialGeomDev& g, const int* order, const int* sec_start, const int2* win0,
                            int* off, long long* total, cudaStream_t s) {
  const long long nk = (long long)g.T * g.nsx * g.nsy;
  size_t tb = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tb, (int*)nullptr, off, (int)(nk + 1), s);
  AsyncScratch counts(s), tmp(s);
  if (e == cudaSuccess) e = counts.alloc((nk + 1) * sizeof(int));
  if (e == cudaSuccess) e = tmp.alloc(tb + 16);
  if (e == cudaSuccess) e = cudaMemsetAsync(counts.p, 0, (nk + 1) * sizeof(int), s);
  if (e != cudaSuccess) return e;
  rad_lists_kernel<<<(int)((nk * 32 + 255) / 256), 256, 0, s>>>(g, order, sec_start, win0, counts.as<int>(), nullptr,
                                                                   nullptr);
  e = cub::DeviceScan::ExclusiveSum(tmp.p, tb, counts.as<int>(), off, (int)(nk + 1), s);
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, off + nk, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  *total = h;
  return e;
}

cudaError_t rad_fill_lists(const RadialGeomDev& g, const int* order, const int* sec_start, const int2* win0,
                           const int* off, int* list, int* blocks, cudaStream_t s) {
  const long long nk = (long long)g.T * g.nsx * g.nsy;
  rad_lists_kernel<<<(int)((nk * 32 + 255) / 256), 256, 0, s>>>(g, order, sec_start, win0, nullptr, off, list);
  // CTAs longest list first (a stable sort: equal lengths keep item order)
  size_t tb = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, (int*)nullptr, (int*)nullptr, (int*)nullptr,
                                                            blocks, (int)nk, 0, 32, s);
  AsyncScratch lens(s), tmp(s);
  if (e == cudaSuccess) e = lens.alloc(3 * nk * sizeof(int));
  if (e == cudaSuccess) e = tmp.alloc(tb + 16);
  if (e != cudaSuccess) return e;
  int *len = lens.as<int>(), *len2 = len + nk, *ids = len + 2 * nk;
  rad_list_len_kernel<<<(int)((nk + 255) / 256), 256, 0, s>>>(off, (int)nk, len);
  rad_iota_kernel<<<(int)((nk + 255) / 256), 256, 0, s>>>(ids, (int)nk);
  e = cub::DeviceRadixSort::SortPairsDescending(tmp.p, tb, len, len2, ids, blocks, (int)nk, 0, 32, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

void launch_rad_windows(const RadialGeomDev& g, int2* win0, float* winw, cudaStream_t s) {
  const int nb = (int)std::min<long long>(((long long)g.T * g.S + 255) / 256, 148 * 16);
#define CALL_W(N) rad_window_kernel<N><<<nb, 256, 0, s>>>(g, win0, winw)
  RAD_NW_DISPATCH(g.nw, CALL_W)
#undef CALL_W
}

void launch_rad_spread(const RArgs& a, const float2* samples, cudaStream_t s) {
  const int grid = a.g.nsx * a.g.nsy * a.g.T;
  const int threads = a.g.sw * a.g.sw;
  // coils per pass: every pass re-reads the neighbouring sectors' samples
  if (a.g.C <= 4) {
#define CALL_S(N) rad_spread_kernel<N, 4><<<grid, threads, 0, s>>>(a, samples)
    RAD_NW_DISPATCH(a.g.nw, CALL_S)
#undef CALL_S
  } else if (a.g.C <= 8) {
#define CALL_S(N) rad_spread_kernel<N, 8><<<grid, threads, 0, s>>>(a, samples)
    RAD_NW_DISPATCH(a.g.nw, CALL_S)
#undef CALL_S
  } else if (a.g.C == 12) {
#define CALL_S(N) rad_spread_kernel<N, 12><<<grid, threads, 0, s>>>(a, samples)
    RAD_NW_DISPATCH(a.g.nw, CALL_S)
#undef CALL_S
  } else {
#define CALL_S(N) rad_spread_kernel<N, 16><<<grid, threads, 0, s>>>(a, samples)
    RAD_NW_DISPATCH(a.g.nw, CALL_S)
#undef CALL_S
  }
}


}  // namespace avx
