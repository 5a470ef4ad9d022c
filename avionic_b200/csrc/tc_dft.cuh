// Tensor-core (tcgen05, sm_100a) partial DFTs in split-BF16x3 precision.
//
// A value v (fp32) is split into three bf16 pieces v0 + v1 + v2 (each the
// truncated bf16 of the remaining residual on the device, the rounded one in
// the host-built coefficient tables; 24 significant bits in all); a product
// a*b is formed from the six piece products with i + j <= 2, accumulated in
// fp32 in tensor memory.  The dropped terms are near 2^-24 relative, so the
// result carries fp32-level accuracy.
#pragma once

#include "pd_args.cuh"

#define TC_M 128        // MMA rows (tile of (coil, column) pairs or image rows)
#define TC_KS 32        // real K per pipeline stage (16 image rows of the y-transform)
#define TC_THREADS 256  // threads per CTA
#define TC_MAX_NP 96    // largest MMA N of the y-transform / K of the adjoint (48 sampled rows
                        // per frame): the adjoint's shared memory, 2304 kc bytes, stays within 227 KB
#define CA_TC_XT 8      // image columns per tile of the tensor-core column adjoint (16 coils per MMA)

namespace avx {

// bytes of one split piece of an operand tile with `rows` rows and TC_KS
// real K values, in the K-major no-swizzle core-matrix layout:
//   byte(r, k) = (r / 8) * 512 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
AVX_HD int tc_piece_bytes(int rows) { return rows * TC_KS * 2; }
AVX_HD int tc_nstage(int H) { return (2 * H + TC_KS - 1) / TC_KS; }  // stages of 16 image rows

// y-transform coefficient table of one operator: for frame t and stage s the
// three pieces of the [np x TC_KS] operand B, np = 2 * (rows per frame)
// rounded up to 16; rows n = 2 kk + part of the output, k = 2 (y - 16 s) + part'.
//   B[2kk][2y] = Re F, B[2kk][2y+1] = -Im F, B[2kk+1][2y] = Im F, B[2kk+1][2y+1] = Re F
// with F[kk][y] = exp(+2 pi i (ky_kk - sy)(y - sy) / H) / sqrt(H).
size_t tc_ytab_bytes(int H, int T, int np);
void tc_build_ytab(int W, int H, int T, int sx, int sy, const int* rows, const int* row_off, int np,
                   unsigned short* out);

size_t tc_ydft_smem_bytes(int np);
cudaError_t configure_tc_kernels();
void launch_ydft_tc(const KArgs& k, cudaStream_t s);

// Column-adjoint coefficient table: for frame t and 128-row tile ty the three
// pieces of the [128 x kc] operand A (K-major core-matrix layout with
// SBO = 16 kc bytes), rows y = 128 ty + r, k = 2 kk + part:
//   A[y][2kk] = Re G, A[y][2kk+1] = Im G,  G[y][kk] = exp(-2 pi i (ky_kk - sy)(y - sy) / H) / sqrt(H)
// kc = 2 x (rows per frame) rounded up to 16 (at most TC_MAX_NP).
AVX_HD int tc_ytiles(int H) { return (H + TC_M - 1) / TC_M; }
size_t tc_ctab_bytes(int H, int T, int kc);
void tc_build_ctab(int H, int T, int sy, const int* rows, const int* row_off, int kc, unsigned short* out);
size_t tc_coladj_smem_bytes(int kc);
// img[t] = sum_c conj(b1_c) column-IDFT(Q'_c), Q' (k.qp) split on the fly;
// needs k.b1t (below)
void launch_coladj_tc(const KArgs& k, float2* img, cudaStream_t s);

// b1 in column-tile order: b1t[((tx C + c) CA_TC_XT + xs) H + y] = b1[c][y][tx CA_TC_XT + xs]
// (zero past the last column), so that the adjoint's threads, one per image
// row, read consecutive addresses.  Elements: b1t_count(W, H, C).
size_t b1t_count(int W, int H, int C);
void launch_b1_tile_transpose(const float2* b1, float2* b1t, int W, int H, int C, cudaStream_t s);

}  // namespace avx
