// Split-BF16x3 tensor-core y-transform (tcgen05.mma kind::f16, sm_100a).
//
// For frame t the CTA computes a 128-row tile of
//   P[(c, x)][kk] = sum_y F[kk][y] b1[c, y, x] u[t, y, x]
// as the real GEMM D[m][n] = sum_k A[m][k] B[n][k], m = c W + x,
// k = 2 y + {re, im}, n = 2 kk + {re, im}; A is produced by the CTA's threads
// from b1 and u and split into three bf16 pieces, B is the precomputed
// coefficient table (tc_dft.cuh).  K runs in stages of 16 image rows through
// two A buffers in tensor memory and a three-slot coefficient ring in shared
// memory; one thread issues the 12 MMAs of a stage (2 K steps x 6 piece
// products) and commits them to the buffer's mbarrier, which the producers
// wait on before refilling that buffer.  The fp32 accumulator lives in tensor
// memory and is read back with tcgen05.ld.
#include <cuda_bf16.h>

#include <cmath>
#include <algorithm>
#include <cstring>
#include <vector>

#include "tc_dft.cuh"

namespace avx {

namespace {

constexpr int kLBO = 128;  // bytes between core matrices adjacent along K
constexpr int kSBO = 512;  // bytes between 8-row groups (TC_KS / 8 core matrices)
constexpr unsigned kWaitLimit = 1u << 22;  // mbarrier polls before giving up

AVX_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

AVX_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

AVX_D bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false when the phase did not complete within the limit
AVX_D bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (unsigned i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

AVX_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
AVX_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle, LBO = 128 B along K,
// SBO between 8-row groups, descriptor version 1 (sm_100)
AVX_D uint64_t smem_desc_sbo(uint32_t addr, int sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((kLBO >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
AVX_D uint64_t smem_desc(uint32_t addr) { return smem_desc_sbo(addr, kSBO); }

// kind::f16 instruction descriptor: bf16 x bf16 -> f32, both K-major, M = 128
AVX_HD uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

AVX_D void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

AVX_D void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

AVX_D void tmem_ld(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Three bf16 pieces of v by truncation, returned as fp32 bit patterns whose
// low 16 bits are zero: p0 = v with the low 16 bits cleared, p1 the same of
// v - p0, p2 the same of v - p0 - p1 (both differences are exact in fp32).
// Each piece carries 8 significant bits, 24 in all.
AVX_D void split3t(float v, uint32_t (&p)[3]) {
  const uint32_t b0 = __float_as_uint(v) & 0xFFFF0000u;
  const float r1 = v - __uint_as_float(b0);
  const uint32_t b1 = __float_as_uint(r1) & 0xFFFF0000u;
  const float r2 = r1 - __uint_as_float(b1);
  p[0] = b0;
  p[1] = b1;
  p[2] = __float_as_uint(r2);  // truncated by the packing
}

// two pieces (upper halves) -> one 32-bit word, lo in the low half
AVX_D uint32_t packhi(uint32_t lo, uint32_t hi) { return __byte_perm(lo, hi, 0x7632); }

}  // namespace

size_t tc_ytab_bytes(int H, int T, int np) { return (size_t)T * tc_nstage(H) * 3 * tc_piece_bytes(np); }

size_t tc_ydft_smem_bytes(int np) { return 3 * (size_t)3 * tc_piece_bytes(np) + 64; }

static unsigned short host_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even (finite inputs)
  return (unsigned short)(u >> 16);
}

static double host_bf16_value(unsigned short h) {
  const uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return (double)f;
}

void tc_build_ytab(int W, int H, int T, int sx, int sy, const int* rows, const int* row_off, int np,
                   unsigned short* out) {
  (void)W;
  (void)sx;
  const int nst = tc_nstage(H);
  const size_t piece = (size_t)tc_piece_bytes(np) / 2;  // in bf16 elements
  const double inv = 1.0 / std::sqrt((double)H);
  for (int t = 0; t < T; ++t) {
    const int r0 = row_off[t], S = row_off[t + 1] - r0;
    for (int s = 0; s < nst; ++s) {
      unsigned short* base = out + ((size_t)t * nst + s) * 3 * piece;
      for (int n = 0; n < np; ++n)
        for (int k = 0; k < TC_KS; ++k) {
          const int kk = n >> 1, y = (s * TC_KS + k) >> 1;
          double v = 0.0;
          if (kk < S && y < H) {
            const int ky = rows[r0 + kk];
            const long long a1 = ((ky - sy) % H + H) % H, a2 = ((y - sy) % H + H) % H;
            const double ang = 2.0 * M_PI * (double)((a1 * a2) % H) / H;
            const double fr = std::cos(ang) * inv, fi = std::sin(ang) * inv;
            const bool re_out = (n & 1) == 0, re_in = (k & 1) == 0;
            v = re_out ? (re_in ? fr : -fi) : (re_in ? fi : fr);
          }
          const size_t off = (size_t)(n / 8) * 256 + (k / 8) * 64 + (n % 8) * 8 + (k % 8);  // in elements
          double r = v;
          for (int p = 0; p < 3; ++p) {
            const unsigned short h = host_bf16((float)r);
            base[p * piece + off] = h;
            r -= host_bf16_value(h);
          }
        }
    }
  }
}

// A operand in tensor memory.  Warp w owns TMEM lane quadrant q = w % 4, so
// thread (w, lane) produces tile row m = 32 q + lane, image rows 8 kh .. 8 kh
// + 7 of every stage (kh = w / 4, the stage's K step kh), and writes the three
// bf16 pieces of its 16 K values with one tcgen05.st each: A never touches
// shared memory, and the MMAs read it from TMEM.  TMEM columns: the fp32
// accumulator [0, np), then per A buffer b, K step ks and piece p the 8
// columns (16 bf16 per lane) at np_al + ((2 b + ks) 3 + p) 8.  The
// coefficient pieces (B) run through a three-slot shared-memory ring filled
// one stage ahead by a bulk copy.  The MMAs of stage s are committed to
// bar[s % 2]; stage s + 2 waits on that barrier (one lane per warp polls it)
// before it overwrites the A buffer, and thread 0 before it loads the
// coefficients of stage s + 3 into the slot stage s used.
AVX_D void tmem_st8(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

// D (tmem) += A (tmem) x B (smem descriptor)^T, kind::f16
AVX_D void mma_bf16_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

AVX_D void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
AVX_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// one contiguous global -> shared copy on the bulk-copy engine, completion
// counted in bytes on bar; source in this GPU's memory, destination this CTA
AVX_D void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Stage hand-off on mbarriers, no CTA barrier in the loop: every thread
// arrives on afull[b] once its tcgen05.st of A buffer b completed; thread 0
// waits for the 256 arrivals and for the stage's coefficients, issues the
// stage's MMAs and commits them to bar[b], while the other warps go on to the
// next stage.  The coefficient stages come by one bulk copy each (thread 0,
// completion on bfull[s % 3]), so the producing threads only load, multiply,
// split and store A.  FULL: every tile row exists (C W a multiple of 128) and
// every stage lies inside the image (H a multiple of 16), so the loads carry
// no range tests.
template <bool U2, bool FULL>
__global__ void __launch_bounds__(TC_THREADS, 3) ydft_tc_kernel(KArgs a) {
  if (a.st && a.st->stop) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  const CartGeomDev& g = a.g;
  const int W = g.W, H = g.H, C = g.C;
  const int t = blockIdx.y;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const int S = r1 - r0;
  if (S == 0) return;
  const int np = a.tc_np;
  const int pieceB = tc_piece_bytes(np);
  const int stageB = 3 * pieceB;
  unsigned char* sB = smem;  // 3 stages
  uint64_t* bar = reinterpret_cast<uint64_t*>(sB + 3 * stageB);  // [2] MMAs of A buffer b done
  uint64_t* bfull = bar + 2;                                     // [3] coefficient stage landed
  uint64_t* afull = bar + 5;                                     // [2] A buffer b written
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 7);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3, kh = warp >> 2;
  const int m = 32 * q + lane;
  const int mg = blockIdx.x * TC_M + m;
  const int CW = C * W;
  const bool valid = mg < CW;
  const int c = valid ? mg / W : 0, x = valid ? mg - c * W : 0;
  const int HW = W * H;
  const int np_al = (np + 7) & ~7;
  const uint32_t ncols = np_al + 96 <= 128 ? 128u : 256u;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    for (int i = 0; i < 3; ++i) mbar_init(&bfull[i], 1);
    mbar_init(&afull[0], TC_THREADS);
    mbar_init(&afull[1], TC_THREADS);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = idesc_bf16(np);
  const uint32_t lane_base = (uint32_t)(q * 32) << 16;

  const float2* __restrict__ pb = a.b1 + (long long)c * HW + x;
  const float2* __restrict__ pu = a.in + (long long)t * HW + x;
  const float2* __restrict__ pw = U2 ? a.in2 + (long long)t * HW + x : nullptr;
  const int nst = tc_nstage(H);
  const unsigned char* __restrict__ btab =
      reinterpret_cast<const unsigned char*>(a.tc_ytab) + (size_t)t * nst * stageB;
  bool ok = true;

  auto issue_b = [&](int st) {  // thread 0
    uint64_t* fb = &bfull[st % 3];
    mbar_expect_tx(fb, (uint32_t)stageB);
    bulk_g2s(sB + (st % 3) * stageB, btab + (size_t)st * stageB, (uint32_t)stageB, fb);
  };

  float2 rb[8], ru[8], rw[U2 ? 8 : 1];
  auto load_stage = [&](int st) {
    const int y0 = st * (TC_KS / 2) + 8 * kh;
    if (FULL) {
      const long long o = (long long)y0 * W;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        rb[i] = __ldg(pb + o + i * W);
        ru[i] = pu[o + i * W];
        if (U2) rw[i] = pw[o + i * W];
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int y = y0 + i;
        const bool in = valid && y < H;
        const int off = y * W;
        rb[i] = in ? __ldg(pb + off) : czero();
        ru[i] = in ? pu[off] : czero();
        if (U2) rw[i] = in ? pw[off] : czero();
      }
    }
  };

  if (tid == 0) issue_b(0);
  load_stage(0);
  for (int s = 0; s < nst; ++s) {
    const int buf = s & 1;
    if (s >= 2) {
      // MMAs of stage s - 2 done: A buffer buf is free (and, for thread 0, the
      // coefficient slot of stage s + 1)
      bool w = true;
      if (lane == 0) w = mbar_wait(&bar[buf], (uint32_t)((s - 2) >> 1) & 1u);
      ok = __shfl_sync(0xffffffffu, w ? 1 : 0, 0) && ok;
    }
    if (tid == 0 && s + 1 < nst) issue_b(s + 1);
    float2 v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = cmul(rb[i], U2 ? csub(ru[i], rw[i]) : ru[i]);
    if (s + 1 < nst) load_stage(s + 1);
    uint32_t pw3[3][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      uint32_t re[3], im[3];
      split3t(v[i].x, re);
      split3t(v[i].y, im);
#pragma unroll
      for (int p = 0; p < 3; ++p) pw3[p][i] = packhi(re[p], im[p]);
    }
    const uint32_t acol = (uint32_t)(np_al + ((2 * buf + kh) * 3) * 8);
#pragma unroll
    for (int p = 0; p < 3; ++p) tmem_st8(tmem + lane_base + acol + (uint32_t)(p * 8), pw3[p]);
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    tc_fence_before();
    mbar_arrive(&afull[buf]);
    if (tid == 0) {
      bool w = mbar_wait(&afull[buf], (uint32_t)(s >> 1) & 1u);
      w = mbar_wait(&bfull[s % 3], (uint32_t)(s / 3) & 1u) && w;
      ok = ok && w;
      tc_fence_after();
      const uint32_t b0 = smem_u32(sB + (s % 3) * stageB);
#pragma unroll
      for (int ks = 0; ks < TC_KS / 16; ++ks) {
        const int pa[6] = {0, 0, 1, 0, 1, 2};
        const int pbk[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
        for (int pr = 0; pr < 6; ++pr) {
          const uint32_t ta = tmem + (uint32_t)(np_al + ((2 * buf + ks) * 3 + pa[pr]) * 8);
          const uint64_t db = smem_desc(b0 + pbk[pr] * pieceB + ks * 2 * kLBO);
          mma_bf16_ta(tmem, ta, db, idesc, (s | ks | pr) != 0);
        }
      }
      mma_commit(&bar[buf]);
    }
    __syncwarp();
  }
  const int last = nst - 1;
  ok = mbar_wait(&bar[last & 1], (uint32_t)(last >> 1) & 1u) && ok;
  if (nst >= 2) ok = mbar_wait(&bar[(last - 1) & 1], (uint32_t)((last - 1) >> 1) & 1u) && ok;
  tc_fence_after();
  if (!__all_sync(0xffffffffu, ok)) {
    if (a.st && lane == 0) atomicExch(&a.st->err, 2);
  } else {
    const int ncol_half = np / 2;
    float2* out = a.qp + kbase(g, t, c, r0, r1) + x;
    for (int cc = kh * ncol_half; cc < (kh + 1) * ncol_half; cc += 8) {
      float vv[8];
      tmem_ld(tmem + lane_base + (uint32_t)cc, vv);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int kk = (cc >> 1) + i;
        if (valid && kk < S) out[(long long)kk * W] = make_float2(vv[2 * i], vv[2 * i + 1]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---------------------------------------------------------------------------
// Column adjoint: CTA (x tile of 32 columns, y tile of 128 rows, frame t).
// For each coil c the GEMM
//   D[y][(x, part)] = sum_k A[y][k] B_c[(x, part)][k],  k = 2 kk + part'
// with A the conjugate coefficients (table) and B_c built from Q'_c:
//   B[(x,0)][(kk,0)] = Re Q, B[(x,0)][(kk,1)] = -Im Q, B[(x,1)][(kk,0)] = Im Q, B[(x,1)][(kk,1)] = Re Q
// gives D = G Q'_c (real and imaginary parts in adjacent columns).  Coil c's
// MMAs go to one of two TMEM buffers while the threads read coil c-1's result
// from the other, multiply it by conj(b1) and accumulate in registers.
// ---------------------------------------------------------------------------

size_t tc_ctab_bytes(int H, int T, int kc) { return (size_t)T * tc_ytiles(H) * 3 * TC_M * kc * 2; }

size_t tc_coladj_smem_bytes(int kc) { return (size_t)3 * TC_M * kc * 2 + (size_t)3 * 256 * kc * 2 + 64; }

void tc_build_ctab(int H, int T, int sy, const int* rows, const int* row_off, int kc, unsigned short* out) {
  const int nty = tc_ytiles(H);
  const size_t piece = (size_t)TC_M * kc;  // elements
  const size_t sbo = (size_t)kc / 8 * 64;  // elements between 8-row groups
  const double inv = 1.0 / std::sqrt((double)H);
  for (int t = 0; t < T; ++t) {
    const int r0 = row_off[t], S = row_off[t + 1] - r0;
    for (int ty = 0; ty < nty; ++ty) {
      unsigned short* base = out + ((size_t)t * nty + ty) * 3 * piece;
      for (int r = 0; r < TC_M; ++r)
        for (int k = 0; k < kc; ++k) {
          const int y = ty * TC_M + r, kk = k >> 1;
          double v = 0.0;
          if (kk < S && y < H) {
            const int ky = rows[r0 + kk];
            const long long a1 = ((ky - sy) % H + H) % H, a2 = ((y - sy) % H + H) % H;
            const double ang = 2.0 * M_PI * (double)((a1 * a2) % H) / H;
            v = (k & 1) ? -std::sin(ang) * inv : std::cos(ang) * inv;
          }
          const size_t off = (size_t)(r / 8) * sbo + (k / 8) * 64 + (r % 8) * 8 + (k % 8);
          double rr = v;
          for (int p = 0; p < 3; ++p) {
            const unsigned short h = host_bf16((float)rr);
            base[p * piece + off] = h;
            rr -= host_bf16_value(h);
          }
        }
    }
  }
}

AVX_D uint32_t tmem_base_addr(const uint32_t* tslot) { return *reinterpret_cast<const volatile uint32_t*>(tslot); }

AVX_D void tmem_ld(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

AVX_D void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(TC_THREADS, 2) coladj_tc_kernel(KArgs k, float2* img) {
  if (k.st && k.st->stop) return;
  constexpr int XT = CA_TC_XT;        // columns per tile
  constexpr int XH = XT / 2;          // columns per thread in the epilogue
  constexpr int CC = 256 / (2 * XT);  // coils per MMA (N = 2 XT CC <= 256)
  extern __shared__ __align__(1024) unsigned char smem[];
  const CartGeomDev& g = k.g;
  const int W = g.W, H = g.H, C = g.C;
  const int t = blockIdx.z;
  const int x0 = blockIdx.x * XT, y0 = blockIdx.y * TC_M;
  const int r0 = g.row_off[t], r1 = g.row_off[t + 1];
  const int S = r1 - r0;
  const int kc = k.tc_kc;
  const int cc_max = min(C, CC);
  const int nb = ((2 * XT * cc_max + 15) / 16) * 16;  // MMA N of a full chunk
  const int pieceA = TC_M * kc * 2, pieceB = nb * kc * 2;
  const int sbo = kc / 8 * 128;
  const uint32_t ncols = nb <= 32 ? 32u : (nb <= 64 ? 64u : (nb <= 128 ? 128u : 256u));
  unsigned char* sA = smem;
  unsigned char* sB = smem + 3 * pieceA;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 3 * pieceA + 3 * pieceB);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int half = tid >> 7;
  const int y = y0 + (tid & (TC_M - 1));
  const int xe = x0 + XH * half;  // first column of this thread's epilogue share
  const long long HW = (long long)W * H;
  float2 acc[XH];
#pragma unroll
  for (int i = 0; i < XH; ++i) acc[i] = make_float2(0.f, 0.f);

  if (S > 0) {
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                   "r"(ncols)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // A: this frame's coefficient pieces for the y tile
    const uint4* src = k.tc_ctab + ((size_t)t * tc_ytiles(H) + blockIdx.y) * 3 * (pieceA / 16);
    for (int e = tid; e < 3 * pieceA / 16; e += TC_THREADS)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sA + 16 * e)), "l"(src + e) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_addr(tslot);
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    bool ok = true;
    int phase = 0;

    // coil maps of four coils ahead of the combine, in registers (their L2
    // latency hides behind the split, the MMAs and three combines)
    float2 pb0[XH], pb1[XH], pb2[XH], pb3[XH];
    auto load_b1 = [&](int cc, int cend, float2 (&pb)[XH]) {
      // column-tile order: consecutive rows y of one column are adjacent
      const float2* bc = k.b1t + (((long long)blockIdx.x * C + cc) * XT + XH * half) * H + y;
#pragma unroll
      for (int i = 0; i < XH; ++i)
        pb[i] = (cc < cend && y < H) ? __ldg(bc + (long long)i * H) : make_float2(0.f, 0.f);
    };
    auto combine = [&](int cl, const float2 (&pb)[XH]) {
      float v[XT];
      static_assert(XT == 8 || XT == 16, "the epilogue reads 8 or 16 accumulator columns per thread");
      tmem_ld(tmem + lane_base + (uint32_t)(2 * XT * cl + half * XT), v);
#pragma unroll
      for (int i = 0; i < XH; ++i) acc[i] = cadd(acc[i], cmulc(pb[i], make_float2(v[2 * i], v[2 * i + 1])));
    };
    for (int c0 = 0; c0 < C; c0 += CC) {
      const int ncc = min(CC, C - c0);
      const int nbc = ((2 * XT * ncc + 15) / 16) * 16;
      const int cend = c0 + ncc;
      load_b1(c0, cend, pb0);
      load_b1(c0 + 1, cend, pb1);
      load_b1(c0 + 2, cend, pb2);
      load_b1(c0 + 3, cend, pb3);
      // B rows n = 16 cl + 2 xl + part for coil c0 + cl; items (coil, column, 4 compact rows)
      const int items = ncc * XT * (kc / 8);
      for (int it = tid; it < items; it += TC_THREADS) {
        const int xl = it % XT, rest = it / XT;
        const int jg = rest % (kc / 8), cl = rest / (kc / 8);
        const float2* q = k.qp + kbase(g, t, c0 + cl, r0, r1);
        float2 qv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int kk = 4 * jg + i;
          qv[i] = (kk < S && x0 + xl < W) ? q[(long long)kk * W + x0 + xl] : make_float2(0.f, 0.f);
        }
        // pieces of Re Q and Im Q; those of -Im Q are the same with the sign flipped
        uint32_t re[4][3], im[4][3];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          split3t(qv[i].x, re[i]);
          split3t(qv[i].y, im[i]);
        }
        const int n0 = 2 * XT * cl + 2 * xl, n1 = n0 + 1;
        const int off0 = (n0 >> 3) * sbo + jg * kLBO + (n0 & 7) * 16;
        const int off1 = (n1 >> 3) * sbo + jg * kLBO + (n1 & 7) * 16;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          // row (x, 0): Re Q, -Im Q;  row (x, 1): Im Q, Re Q
          *reinterpret_cast<uint4*>(sB + p * pieceB + off0) =
              make_uint4(packhi(re[0][p], im[0][p] ^ 0x80000000u), packhi(re[1][p], im[1][p] ^ 0x80000000u),
                         packhi(re[2][p], im[2][p] ^ 0x80000000u), packhi(re[3][p], im[3][p] ^ 0x80000000u));
          *reinterpret_cast<uint4*>(sB + p * pieceB + off1) =
              make_uint4(packhi(im[0][p], re[0][p]), packhi(im[1][p], re[1][p]), packhi(im[2][p], re[2][p]),
                         packhi(im[3][p], re[3][p]));
        }
      }
      // rows of a partly filled last 16-row group
      for (int n = 2 * XT * ncc + tid; n < nbc; n += TC_THREADS)
        for (int j = 0; j < kc / 8; ++j)
#pragma unroll
          for (int p = 0; p < 3; ++p)
            *reinterpret_cast<uint4*>(sB + p * pieceB + (n >> 3) * sbo + j * kLBO + (n & 7) * 16) =
                make_uint4(0u, 0u, 0u, 0u);
      asm volatile("cp.async.wait_all;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
        const uint32_t idesc = idesc_bf16(nbc);
        const int pa[6] = {0, 0, 1, 0, 1, 2};
        const int pbk[6] = {0, 1, 0, 2, 1, 0};
        for (int ks = 0; ks < kc / 16; ++ks) {
#pragma unroll
          for (int pr = 0; pr < 6; ++pr) {
            const uint64_t da = smem_desc_sbo(a0 + pa[pr] * pieceA + ks * 2 * kLBO, sbo);
            const uint64_t db = smem_desc_sbo(b0 + pbk[pr] * pieceB + ks * 2 * kLBO, sbo);
            mma_bf16(tmem, da, db, idesc, (ks | pr) != 0);
          }
        }
        mma_commit(&bar[0]);
      }
      {
        // one lane per warp polls the MMAs' barrier
        bool w = true;
        if ((tid & 31) == 0) w = mbar_wait(&bar[0], (uint32_t)phase);
        ok = __shfl_sync(0xffffffffu, w ? 1 : 0, 0) && ok;
      }
      phase ^= 1;
      tc_fence_after();
      for (int cl = 0; cl < ncc; cl += 4) {
        combine(cl, pb0);
        load_b1(c0 + cl + 4, cend, pb0);
        if (cl + 1 < ncc) combine(cl + 1, pb1);
        load_b1(c0 + cl + 5, cend, pb1);
        if (cl + 2 < ncc) combine(cl + 2, pb2);
        load_b1(c0 + cl + 6, cend, pb2);
        if (cl + 3 < ncc) combine(cl + 3, pb3);
        load_b1(c0 + cl + 7, cend, pb3);
      }
      tc_fence_before();
      __syncthreads();  // TMEM and B are reused by the next chunk
    }
    if (!ok && k.st && tid == 0) atomicExch(&k.st->err, 3);
    if (warp == 0)
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
  if (y < H) {
    float2* out = img + (long long)t * HW + (long long)y * W + xe;
#pragma unroll
    for (int i = 0; i < XH; ++i)
      if (xe + i < W) out[i] = acc[i];
  }
}

size_t b1t_count(int W, int H, int C) { return (size_t)((W + CA_TC_XT - 1) / CA_TC_XT) * C * CA_TC_XT * H; }

__global__ void b1_tile_transpose_kernel(const float2* __restrict__ b1, float2* __restrict__ b1t, int W, int H,
                                         int C, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(e % H);
    long long r = e / H;
    const int xs = (int)(r % CA_TC_XT);
    r /= CA_TC_XT;
    const int c = (int)(r % C);
    const int tx = (int)(r / C);
    const int x = tx * CA_TC_XT + xs;
    b1t[e] = x < W ? b1[((long long)c * H + y) * W + x] : make_float2(0.f, 0.f);
  }
}

void launch_b1_tile_transpose(const float2* b1, float2* b1t, int W, int H, int C, cudaStream_t s) {
  const long long n = (long long)b1t_count(W, H, C);
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
  b1_tile_transpose_kernel<<<blocks, 256, 0, s>>>(b1, b1t, W, H, C, n);
}

cudaError_t configure_tc_kernels() {
  const cudaFuncAttribute smem = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(ydft_tc_kernel<false, false>, smem, AVX_DYN_SMEM_MAX);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(ydft_tc_kernel<true, false>, smem, AVX_DYN_SMEM_MAX);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(ydft_tc_kernel<false, true>, smem, AVX_DYN_SMEM_MAX);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(ydft_tc_kernel<true, true>, smem, AVX_DYN_SMEM_MAX);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(coladj_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, AVX_DYN_SMEM_MAX);
}

void launch_coladj_tc(const KArgs& k, float2* img, cudaStream_t s) {
  dim3 gr((k.g.W + CA_TC_XT - 1) / CA_TC_XT, tc_ytiles(k.g.H), k.g.T);
  coladj_tc_kernel<<<gr, TC_THREADS, tc_coladj_smem_bytes(k.tc_kc), s>>>(k, img);
}

void launch_ydft_tc(const KArgs& k, cudaStream_t s) {
  dim3 gr((k.g.C * k.g.W + TC_M - 1) / TC_M, k.g.T);
  const size_t sm = tc_ydft_smem_bytes(k.tc_np);
  // every thread's tile row exists and every stage lies inside the image
  const bool full = (k.g.C * k.g.W) % TC_M == 0 && k.g.H % (TC_KS / 2) == 0;
  if (k.in2) {
    if (full)
      ydft_tc_kernel<true, true><<<gr, TC_THREADS, sm, s>>>(k);
    else
      ydft_tc_kernel<true, false><<<gr, TC_THREADS, sm, s>>>(k);
  } else {
    if (full)
      ydft_tc_kernel<false, true><<<gr, TC_THREADS, sm, s>>>(k);
    else
      ydft_tc_kernel<false, false><<<gr, TC_THREADS, sm, s>>>(k);
  }
}

}  // namespace avx
