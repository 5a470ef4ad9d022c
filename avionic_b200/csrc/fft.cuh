// Shared-memory mixed-radix FFT of many short sequences (device code).
#pragma once

#include "common.cuh"

// Row pitch (in complex values) of the [x][pitch] sequence buffers: KC + 1.
// An odd pitch spreads the x-strided accesses (the transposing loads and
// stores around the passes) over all 32 banks.
#define AVX_FFT_PITCH(KC) ((KC) + 1)

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
  constexpr int KCP = AVX_FFT_PITCH(KC);
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


// ---------------------------------------------------------------------------
// Compile-time plans.  The same Stockham passes as row_fft with the radix
// sequence, the sequence length, the direction and the block size (NT
// threads) fixed at compile time, so that the index arithmetic folds to
// shifts and constants.  Plans exist for the lengths fft_plan_id() lists;
// row_fft_planned falls back to row_fft for the others.
// ---------------------------------------------------------------------------

template <int R, int SIGN>
AVX_D void butterfly_fixed(float2 (&v)[R], const float2* tw, int nb) {
  if constexpr (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
    const float2 ib1 = SIGN > 0 ? make_float2(-b1.y, b1.x) : make_float2(b1.y, -b1.x);  // i*sign*b1
    v[0] = cadd(a0, b0);
    v[1] = cadd(a1, ib1);
    v[2] = csub(a0, b0);
    v[3] = csub(a1, ib1);
  } else if constexpr (R == 8) {
    // two 4-point DFTs of the even and odd inputs, joined by the 8th roots of unity
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    butterfly_fixed<4, SIGN>(e, tw, nb);
    butterfly_fixed<4, SIGN>(o, tw, nb);
    constexpr float h = 0.70710678118654752440f;
    const float s = (float)SIGN;
    const float2 t1 = make_float2(h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x));    // o1 (1 + i s) / sqrt 2
    const float2 t2 = make_float2(-s * o[2].y, s * o[2].x);                                 // o2 i s
    const float2 t3 = make_float2(-h * (o[3].x + s * o[3].y), h * (s * o[3].x - o[3].y));  // o3 (-1 + i s) / sqrt 2
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);
    v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
  } else if constexpr (R == 3) {
    const float2 t1 = cadd(v[1], v[2]);
    const float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    const float2 d = csub(v[1], v[2]);
    const float h = 0.86602540378443864676f * (float)SIGN;
    const float2 id = make_float2(-h * d.y, h * d.x);  // i*sign*(sqrt(3)/2)*(v1 - v2)
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, id);
    v[2] = csub(t2, id);
  } else {
    // direct R-point DFT with the table's R-th roots of unity (index (m q mod R) nb)
    float2 o[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      float2 acc = v[0];
#pragma unroll
      for (int m = 1; m < R; ++m) {
        const float2 w = tw[((m * q) % R) * nb];
        cfma(acc, v[m], make_float2(w.x, SIGN > 0 ? w.y : -w.y));
      }
      o[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = o[q];
  }
}

template <int KC, int NT, int W, int SIGN, int NS, int R>
AVX_D void fft_pass_fixed(const float2* src, float2* dst, const float2* tw) {
  constexpr int KCP = AVX_FFT_PITCH(KC), NB = W / R, TWS = W / (NS * R), TOTAL = NB * KC;
#pragma unroll
  for (int e0 = 0; e0 < TOTAL; e0 += NT) {
    const int e = e0 + (int)threadIdx.x;
    if (TOTAL % NT != 0 && e >= TOTAL) break;
    const int kk = e % KC, j = e / KC;
    const int q = j / NS, k = j - q * NS;
    const int idxD = q * NS * R + k;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float2 s0 = src[(j + r * NB) * KCP + kk];
      if (r == 0) {
        v[r] = s0;
      } else {
        const float2 w = tw[r * k * TWS];
        v[r] = cmul(s0, make_float2(w.x, SIGN > 0 ? w.y : -w.y));
      }
    }
    butterfly_fixed<R, SIGN>(v, tw, NB);
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(idxD + r * NS) * KCP + kk] = v[r];
  }
}

template <int KC, int NT, int W, int SIGN, int NS>
AVX_D float2* fft_fixed_rec(float2* src, float2*, const float2*) {
  return src;
}

template <int KC, int NT, int W, int SIGN, int NS, int R, int... Rest>
AVX_D float2* fft_fixed_rec(float2* src, float2* dst, const float2* tw) {
  fft_pass_fixed<KC, NT, W, SIGN, NS, R>(src, dst, tw);
  __syncthreads();
  return fft_fixed_rec<KC, NT, W, SIGN, NS * R, Rest...>(dst, src, tw);
}

// Plan identifiers: a length with a compile-time plan is its own identifier;
// 1 = a run-time plan whose radices are at most 5, 0 = any run-time plan.
// The compile-time plans lead with radix-8 passes (one shared-memory round
// trip fewer than the run-time plans' radix-4 passes).
inline int fft_plan_id(int n, int nrad, const int* rad) {
  switch (n) {
    case 96: case 128: case 160: case 192: case 256: case 320: return n;
    default: break;
  }
  for (int i = 0; i < nrad; ++i)
    if (rad[i] > 5) return 0;
  return 1;
}

// The run-time plan of a length (what fft_plan_id gives a length without a
// compile-time plan): 1 when every radix is at most 5, else 0.
inline int fft_plan_id_runtime(int nrad, const int* rad) {
  for (int i = 0; i < nrad; ++i)
    if (rad[i] > 5) return 0;
  return 1;
}

// row_fft with a plan chosen at compile time; blockDim.x must be 256
template <int KC, int PLAN, int SIGN>
AVX_D float2* row_fft_planned(float2* src, float2* dst, const float2* tw, int W, int nrad, const int* rad) {
  if constexpr (PLAN == 96) return fft_fixed_rec<KC, 256, 96, SIGN, 1, 8, 4, 3>(src, dst, tw);
  else if constexpr (PLAN == 128) return fft_fixed_rec<KC, 256, 128, SIGN, 1, 8, 8, 2>(src, dst, tw);
  else if constexpr (PLAN == 160) return fft_fixed_rec<KC, 256, 160, SIGN, 1, 8, 4, 5>(src, dst, tw);
  else if constexpr (PLAN == 192) return fft_fixed_rec<KC, 256, 192, SIGN, 1, 8, 8, 3>(src, dst, tw);
  else if constexpr (PLAN == 256) return fft_fixed_rec<KC, 256, 256, SIGN, 1, 8, 8, 4>(src, dst, tw);
  else if constexpr (PLAN == 320) return fft_fixed_rec<KC, 256, 320, SIGN, 1, 8, 8, 5>(src, dst, tw);
  else return row_fft<KC, PLAN == 0>(src, dst, tw, W, nrad, rad, SIGN);
}

// calls CALL(id) with the compile-time plan identifier id
#define AVX_FFT_PLAN_DISPATCH(ID, CALL) \
  switch (ID) {                         \
    case 96: CALL(96); break;           \
    case 128: CALL(128); break;         \
    case 160: CALL(160); break;         \
    case 192: CALL(192); break;         \
    case 256: CALL(256); break;         \
    case 320: CALL(320); break;         \
    case 1: CALL(1); break;             \
    default: CALL(0); break;            \
  }
