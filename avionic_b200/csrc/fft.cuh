// Shared-memory mixed-radix FFT of many short sequences (device code).
#pragma once

#include "common.cuh"

// ---------------------------------------------------------------------------
// KC independent length-W sequences stored [x][KCP] (row index kk
// fastest), mixed-radix Stockham autosort passes ping-ponging between two
// shared-memory buffers.  Pass with radix R over sub-transforms of size Ns:
//   v_r = src[j + r W/R] * w^(r (j mod Ns) W/(Ns R)),  V = DFT_R(v),
//   dst[(j / Ns) Ns R + (j mod Ns) + r Ns] = V_r
// with w = exp(sign 2 pi i / W) from the twiddle table.  Returns the buffer
// holding the natural-order result.
// ---------------------------------------------------------------------------

AVX_D float2 tw_sign(const float2* tw, int j, int sign) {
  const float2 w = tw[j];
  return make_float2(w.x, sign > 0 ? w.y : -w.y);
}

// one butterfly of a small prime radix R: direct R-point DFT with table twiddles
template <int R, int KCP>
AVX_D void small_dft(const float2* src, float2* dst, const float2* tw, int j, int nb, int k, int tws, int idxD,
                     int Ns, int kk, int W, int sign) {
  float2 v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const float2 s0 = src[(j + r * nb) * KCP + kk];
    v[r] = r ? cmul(s0, tw_sign(tw, r * k * tws, sign)) : s0;
  }
  // outputs one at a time: unrolling them all as well costs registers (and
  // spills) for the larger radices
#pragma unroll 1
  for (int q = 0; q < R; ++q) {
    float2 acc = v[0];
#pragma unroll
    for (int m = 1; m < R; ++m) cfma(acc, v[m], tw_sign(tw, ((m * q) % R) * nb, sign));
    dst[(idxD + q * Ns) * KCP + kk] = acc;
  }
}

// floor(j / d) for j < 2^16 and 1 <= d < 2^16 from m = ceil(2^32 / d) (m = 0 for d = 1):
// j m = j 2^32 / d + j e / d with e = m d - 2^32 < d, and j e < 2^32, so the
// high word is exact.
AVX_D unsigned div_magic(unsigned d) { return d == 1u ? 0u : 0xFFFFFFFFu / d + 1u; }
AVX_D int fast_div(int j, unsigned d, unsigned m) { return d == 1u ? j : (int)__umulhi((unsigned)j, m); }

// The radix plans live in the kernels' parameter structs.  Handing row_fft a
// pointer into one would make every thread copy the struct to local memory;
// instead thread 0 copies the plan to shared memory with constant indices.  A
// __syncthreads() must separate this from row_fft.
AVX_D void stage_plan(const int (&rad)[12], int* splan) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < 12; ++i) splan[i] = rad[i];
  }
}

// LARGE = false compiles the radix-2/3/4/5 passes only (the plans of sizes
// whose prime factors are at most 5), which keeps the register count down.
template <int KC, bool LARGE = true>
__device__ float2* row_fft(float2* src, float2* dst, const float2* tw, int W, int nrad, const int* rad, int sign) {
  constexpr int KCP = KC + 2;
  int Ns = 1;
  // kk is fixed per thread when the block size is a multiple of KC
  for (int p = 0; p < nrad; ++p) {
    const int R = rad[p];
    const int nb = W / R;
    const int tws = W / (Ns * R);  // r k tws < W for r < R, k < Ns: twiddle indices need no reduction
    const unsigned mNs = div_magic((unsigned)Ns);
    for (int e = threadIdx.x; e < nb * KC; e += blockDim.x) {
      const int kk = e % KC, j = e / KC;
      const int q = fast_div(j, (unsigned)Ns, mNs);
      const int k = j - q * Ns;
      const int idxD = q * Ns * R + k;
      if (R == 2) {
        const float2 v0 = src[j * KCP + kk];
        const float2 v1 = cmul(src[(j + nb) * KCP + kk], tw_sign(tw, k * tws, sign));
        dst[idxD * KCP + kk] = cadd(v0, v1);
        dst[(idxD + Ns) * KCP + kk] = csub(v0, v1);
      } else if (R == 4) {
        const float2 v0 = src[j * KCP + kk];
        const float2 v1 = cmul(src[(j + nb) * KCP + kk], tw_sign(tw, k * tws, sign));
        const float2 v2 = cmul(src[(j + 2 * nb) * KCP + kk], tw_sign(tw, 2 * k * tws, sign));
        const float2 v3 = cmul(src[(j + 3 * nb) * KCP + kk], tw_sign(tw, 3 * k * tws, sign));
        const float2 a0 = cadd(v0, v2), a1 = csub(v0, v2);
        const float2 b0 = cadd(v1, v3), b1 = csub(v1, v3);
        // i*sign*b1
        const float2 ib1 = sign > 0 ? make_float2(-b1.y, b1.x) : make_float2(b1.y, -b1.x);
        dst[idxD * KCP + kk] = cadd(a0, b0);
        dst[(idxD + Ns) * KCP + kk] = cadd(a1, ib1);
        dst[(idxD + 2 * Ns) * KCP + kk] = csub(a0, b0);
        dst[(idxD + 3 * Ns) * KCP + kk] = csub(a1, ib1);
      } else if (R == 3) {
        const float2 v0 = src[j * KCP + kk];
        const float2 v1 = cmul(src[(j + nb) * KCP + kk], tw_sign(tw, k * tws, sign));
        const float2 v2 = cmul(src[(j + 2 * nb) * KCP + kk], tw_sign(tw, 2 * k * tws, sign));
        const float2 t1 = cadd(v1, v2);
        const float2 t2 = make_float2(v0.x - 0.5f * t1.x, v0.y - 0.5f * t1.y);
        const float2 d = csub(v1, v2);
        const float h = 0.86602540378443864676f * (float)sign;
        const float2 id = make_float2(-h * d.y, h * d.x);  // i*sign*(sqrt(3)/2)*(v1 - v2)
        dst[idxD * KCP + kk] = cadd(v0, t1);
        dst[(idxD + Ns) * KCP + kk] = cadd(t2, id);
        dst[(idxD + 2 * Ns) * KCP + kk] = csub(t2, id);
      } else if (!LARGE || R == 5) {
        small_dft<5, KCP>(src, dst, tw, j, nb, k, tws, idxD, Ns, kk, W, sign);
      } else if (R == 7) {
        small_dft<7, KCP>(src, dst, tw, j, nb, k, tws, idxD, Ns, kk, W, sign);
      } else if (R == 11) {
        small_dft<11, KCP>(src, dst, tw, j, nb, k, tws, idxD, Ns, kk, W, sign);
      } else {
        small_dft<13, KCP>(src, dst, tw, j, nb, k, tws, idxD, Ns, kk, W, sign);
      }
    }
    __syncthreads();
    float2* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

