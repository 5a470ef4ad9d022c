// Launch interface of the primal-dual kernels (pd_kernels.cu).
#pragma once

#include "pd_args.cuh"

#define KSPACE_KC 16  // compact k-space rows per chunk (y-transform and row kernels)
#ifndef ROWS_RB
#define ROWS_RB 4     // global loads a thread of the row kernel issues together
#endif
#define YD_XS 16      // image columns per CTA of the y-transform
#define YD_CG 16      // coil slots per CTA of the y-transform
#define CA_TX 16      // column-adjoint threads along x (two columns each, 16 apart)
#define CA_TY 8       // column-adjoint threads along y
#define CA_YP 8       // column-adjoint rows per thread
#define CA_KQ 32      // compact rows per coefficient chunk of the column adjoint
#define ADJ_TX 32     // tile width (x) of the primal / gap kernels
#define ADJ_TY 4      // thread rows per tile
#define ADJ_YP 4      // pixels per thread along y
#define ADJ_TH (ADJ_TY * ADJ_YP)
// Launch shapes the autotuner chooses from (PDArgs::primal_tile, dual_block):
// primal tiles (threads along x, threads along y, pixels per thread along y)
// and dual-kernel block sizes; index 0 of each is the untuned default.
#define AVX_PRIMAL_TILES 7  // 0-4: one pixel per thread; 5-6: pairs (TGV2 / ICTGV2 with even W)
#define AVX_DUAL_BLOCKS 6  // 0-2: one pixel per thread; 3-5: two (TGV2 / ICTGV2 with even W)

// timed stages of one iteration (avx_solver_kernel_times)
#define AVX_NSTAGE 5

namespace avx {

struct Ptr8 {
  float2* p[8];
};

struct GapConst {
  double lam, N, stop_gap;  // the data-energy constant is DevState::d_off
  double alpha0, alpha1, ic_a, ic_b;
  double stop_rel;          // > 0: also stop once gap <= stop_rel * first gap
};

size_t kspace_smem_bytes(int W, int H);  // largest dynamic shared memory of the transform kernels
int gap_img_blocks(int W, int H, int T);
cudaError_t configure_kernels();

// one Cartesian iteration: dual, y-transform, rows, column adjoint, primal;
// ev (optional) receives AVX_NSTAGE + 1 events around the stages
void launch_iteration(int method, const PDArgs& a, const KArgs& k, float2* khz, cudaStream_t s,
                      cudaEvent_t* ev = nullptr);
void launch_dual(int method, const PDArgs& a, cudaStream_t s);
void launch_primal(int method, const PDArgs& a, cudaStream_t s);
// the shape behind a tuning index: primal tile "TXxTYxYP", dual block "N threads"
const char* primal_tile_name(int i);
bool dual_pairs(int method, int W);  // the two-pixel dual and primal kernels apply
int dual_block_threads(int i);
void launch_ydft(const KArgs& k, cudaStream_t s);
void launch_rows(const KArgs& k, int mode, cudaStream_t s);
void launch_step_img(int method, const PDArgs& a, const Ptr8& e_dev, int P, double* pimg, cudaStream_t s);
void launch_step_finalize(const PDArgs& a, double* pimg, double* pk, int nk, double ratio, cudaStream_t s);
void launch_gap_tail(int method, const PDArgs& a, const KArgs& k_x, double* pimg, double* pk, int nk,
                     const GapConst& gc, double* hg, double* hn, double* hf, int cap, int init_only,
                     cudaStream_t s);
// y-transform followed by the row kernel in the given mode (0 PD step, 1 step-rule norm, 2 gap, 3 apply,
// 4 normal operator: Q' = row-IFFT(mask^2 X), for A^H A by the column adjoint)
void launch_kspace(const KArgs& k, int mode, cudaStream_t s);
// img[t] = sum_c conj(b1_c) column-IDFT of the compact rows in k.qp
void launch_adjoint(const KArgs& k, float2* img, cudaStream_t s);
void launch_step(int method, const PDArgs& a, const KArgs& k_e, const Ptr8& e_dev, int P,
                 double* pimg, double* pk, double ratio, cudaStream_t s);
void launch_gap(int method, const PDArgs& a, const KArgs& k_x, float2* khz, double* pimg, double* pk,
                const GapConst& gc, double* hg, double* hn, double* hf, int cap, int init_only, cudaStream_t s);
void launch_gather_rows(const CartGeomDev& g, const float2* dense, float2* compact, int apply_mask,
                        cudaStream_t s);
void launch_dense_rowidft(const CartGeomDev& g, float2* dense, float2* qp, const float* mask_dense,
                          cudaStream_t s);

}  // namespace avx
