// Launch interface of the primal-dual kernels (pd_kernels.cu).
#pragma once

#include "pd_args.cuh"

#define KSPACE_KC 16  // compact k-space rows per chunk in kspace_kernel
#define ADJ_TX 32     // tile width (x) of the column-adjoint / primal kernels
#define ADJ_TY 4      // thread rows per tile
#define ADJ_YP 4      // pixels per thread along y
#define ADJ_TH (ADJ_TY * ADJ_YP)
#define ADJ_KQ 32     // compact rows staged per chunk in the adjoint

namespace avx {

struct Ptr8 {
  float2* p[8];
};

struct GapConst {
  double lam, d_off_energy, N, stop_gap;
  double alpha0, alpha1, ic_a, ic_b;
};

size_t kspace_smem_bytes(int W, int H);
int gap_img_blocks(int W, int H, int T);
cudaError_t configure_kernels();

void launch_iteration(int method, const PDArgs& a, const KArgs& k, cudaStream_t s);
void launch_dual(int method, const PDArgs& a, cudaStream_t s);
void launch_primal(int method, const PDArgs& a, const KArgs& k, cudaStream_t s, bool cart = true);
void launch_step_img(int method, const PDArgs& a, const Ptr8& e_dev, int P, double* pimg, cudaStream_t s);
void launch_step_finalize(const PDArgs& a, double* pimg, double* pk, int nk, double ratio, cudaStream_t s);
void launch_gap_tail(int method, const PDArgs& a, const KArgs& k_x, double* pimg, double* pk, int nk,
                     const GapConst& gc, double* hg, double* hn, double* hf, int cap, int init_only, bool cart,
                     cudaStream_t s);
void launch_kspace(const KArgs& k, int mode, cudaStream_t s);
void launch_adjoint(const KArgs& k, float2* img, cudaStream_t s);
void launch_step(int method, const PDArgs& a, const KArgs& k_e, const Ptr8& e_dev, int P,
                 double* pimg, double* pk, double ratio, cudaStream_t s);
void launch_gap(int method, const PDArgs& a, const KArgs& k_x, double* pimg, double* pk, const GapConst& gc,
                double* hg, double* hn, double* hf, int cap, int init_only, cudaStream_t s);
void launch_gather_rows(const CartGeomDev& g, const float2* dense, float2* compact, int apply_mask,
                        cudaStream_t s);
void launch_dense_rowidft(const CartGeomDev& g, float2* dense, float2* qp, const float* mask_dense,
                          cudaStream_t s);

}  // namespace avx
