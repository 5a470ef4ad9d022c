// Kernel argument blocks for the primal-dual core.
#pragma once

#include "common.cuh"

// Geometry of one Cartesian operator.  k-space is stored compactly: for
// frame t only the rows ky that carry a non-zero mask value anywhere along x
// are kept, in ascending ky order.  Compact row r (global over all frames)
// belongs to frame t when row_off[t] <= r < row_off[t+1]; its ky is rows[r].
// A compact k-space array holds, for frame t and coil c, the block
//   base(t, c) = (row_off[t] * C + c * (row_off[t+1] - row_off[t])) * W
// of (row_off[t+1]-row_off[t]) x W complex values (row-major, kx fastest).
struct CartGeomDev {
  int W, H, C, T;
  int sx, sy;             // centring shifts (W/2, H/2) or 0
  const int* rows;        // [R] ky of each compact row
  const int* row_off;     // [T+1]
  const float* mrow;      // [R*W] mask value at each compact sample
  const float2* twx;      // [W] exp(+2 pi i j / W)
  const float2* twy;      // [H] exp(+2 pi i j / H)
  float inv_sqrt_w, inv_sqrt_h;
  int nrad;               // radix passes of the length-W row FFT (0: dense DFT)
  int rad[12];            // radices, first pass first
};

AVX_HD long long kbase(const CartGeomDev& g, int /* frame: implied by r0, r1 */, int c, int r0, int r1) {
  return ((long long)r0 * g.C + (long long)c * (r1 - r0)) * g.W;
}

// Finite-difference weights of one regulariser branch (1/dx, 1/dy, 1/dt).
struct Wts {
  float ix, iy, it;      // 1/dx, 1/dy, 1/dt
  float hx, hy, ht;      // 1/(2dx), 1/(2dy), 1/(2dt) for the symmetrised gradient
};

struct PDArgs {
  int W, H, T;
  long long N;
  float2* x[8];     // primal components
  float2* xb[8];    // extragradient components
  float2* y[18];    // dual components
  Wts w1, w2;       // branch weights (w2 used by ICTGV2 only)
  float r1, r2, r3, r4;  // prox scales (1/radius) of y1, y2, y3, y4
  float alpha0, alpha1, alpha;  // regulariser weights (norm evaluation)
  float ic_a, ic_b;             // ICTGV2 branch factors alpha/m, (1-alpha)/m
  const float2* khz;            // K^H z image when the operator supplies it (radial)
  DevState* st;
  int primal_tile, dual_block;  // launch shapes (indices into the tuning tables of pd_kernels.cu)
};

struct KArgs {
  CartGeomDev g;
  const float2* b1;     // [C*H*W]
  const float2* in;     // image input (T*H*W)
  const float2* in2;    // optional second image (in - in2 is transformed)
  float2* z;            // compact dual variable
  const float2* d;      // compact data
  float2* qp;           // compact row-inverse-transformed output
  float2* dense_out;    // dense k-space output (operator apply)
  float lam;            // data weight lambda
  int binary_mask;      // 1 when every mask value is 0 or 1
  DevState* st;
  double* partial;      // [slots * gridBlocks]
  // split-BF16x3 tensor-core y-transform (null: fp32 CUDA-core kernels)
  const uint4* tc_ytab; // coefficient pieces, tc_dft.cuh
  int tc_np;            // MMA N (2 x rows per frame, rounded up to 16)
  // split-BF16x3 tensor-core column adjoint (null: fp32 CUDA-core kernel)
  const uint4* tc_ctab; // conjugate coefficient pieces, tc_dft.cuh
  int tc_kc;            // MMA K (2 x rows per frame, rounded up to 16)
  const float2* b1t;    // b1 in column-tile order for the tensor-core adjoint (tc_dft.cuh)
  // row-FFT schedule of the row kernel (chosen by the autotuner): compact rows
  // per pass (8, 12 or 16; 0 = 16) and the radix plan (0: the compile-time
  // plan of the length when there is one, 1: the run-time plan)
  int rows_kc, rows_rt;
};
