// Radial (non-Cartesian) operator: geometry and launchers (radial.cu).
//
// K_f x = sqrt(w_f) NUFFT_f(b1_c x_f) / sqrt(HW) with a tapered Kaiser-Bessel
// gridding NUFFT on an oversampled grid (definition in oracle/radial.py);
// K^H its exact adjoint.  Grid layout [frame][coil][Gy][Gx];
// samples [frame][coil][S].
#pragma once

#include "pd_args.cuh"

struct RadialGeomDev {
  int W, H, C, T, S;        // image, coils, frames, samples per frame
  int Gx, Gy;               // oversampled grid
  int sw, nsx, nsy;         // sector width and sector counts
  int nw;                   // interpolation window points per axis (ceil(J) + 1)
  float J, beta, kb_norm;   // kernel width, shape, 1 / (I0(beta) - 1)
  float norm;               // 1 / sqrt(W H)
  const float* traj;        // [T][2][S] kx then ky, cycles/pixel in [-0.5, 0.5)
  const float* sqrt_w;      // [T][S]
  const float* inv_psi_x;   // [W] 1 / deapodisation
  const float* inv_psi_y;   // [H]
  const int* order;         // [T][S] sample indices sorted by sector (stable)
  const int* sec_start;     // [T][nsx*nsy + 1] offsets into order
  const int* spread_list;   // per (frame, sector): the samples whose window reaches the sector, in summation order
  const int* spread_off;    // [T*nsx*nsy + 1] offsets into spread_list, index f*nsx*nsy + sector
  const int* spread_blocks; // [T*nsx*nsy] f*nsx*nsy + sector, longest list first
  const int2* win0;         // [T][S] first grid cell (x, y) of each sample's window, unwrapped
  const float* winw;        // [T][S][2 nw] the window's weights, x then y
  const float2* twgx;       // [Gx] exp(+2 pi i j / Gx)
  const float2* twgy;       // [Gy]
  int nradx, radx[12];      // FFT plan along x
  int nrady, rady[12];      // FFT plan along y
};

struct RArgs {
  RadialGeomDev g;
  const float2* b1;       // [C][H][W]
  const float2* in;       // image input [T][H][W]
  const float2* in2;      // optional: in - in2 is transformed
  float2* grid;           // [T][C][Gy][Gx]
  float2* z;              // [T][C][S] dual variable
  const float2* d;        // [T][C][S] data (already sqrt(w)-weighted, as main.cpp does)
  float2* out;            // samples out (apply) or image out (adjoint)
  float lam;
  DevState* st;
  double* partial;
};

namespace avx {

size_t radial_fft_smem_bytes(int G);
size_t radial_adj_smem_bytes(int G, int W);
int radial_interp_blocks(const RadialGeomDev& g);
cudaError_t configure_radial_kernels();

// per-sample window starts and weights (g.win0, g.winw), once per operator
void launch_rad_windows(const RadialGeomDev& g, int2* win0, float* winw, cudaStream_t s);
// Per-sample tables of an operator, built on the device (stream-ordered, each
// call returns after its stream work when it reads a result back):
// flags bit 0: a trajectory value outside [-1/2, 1/2]; bit 1: a negative density
cudaError_t rad_validate(const float* traj, long long nt, const float* dens, long long nd, int* flags_host,
                         cudaStream_t s);
// sqrt(w), and the samples of every frame stably sorted by sector (order,
// [T][S]) with the sectors' offsets (sec_start, [T][nsx nsy + 1]); needs g.traj
cudaError_t rad_build_order(const RadialGeomDev& g, const float* dens, float* sqrt_w, int* order, int* sec_start,
                            cudaStream_t s);
// the spreading work lists' offsets (off, [T nsx nsy + 1]) and total length
cudaError_t rad_count_lists(const RadialGeomDev& g, const int* order, const int* sec_start, const int2* win0,
                            int* off, long long* total, cudaStream_t s);
// the work lists and the CTA order (longest list first)
cudaError_t rad_fill_lists(const RadialGeomDev& g, const int* order, const int* sec_start, const int2* win0,
                           const int* off, int* list, int* blocks, cudaStream_t s);
// grid -> samples; mode 0 z prox, 1 sum |K u|^2, 2 gap sums, 3 write samples to a.out
void launch_rad_interp(const RArgs& a, int mode, cudaStream_t s);
// forward image -> grid: the zero-padded, deapodised b1 (in - in2) and its
// unnormalised 2D DFT (sign -1) in two passes, the padding fused into the row pass
void launch_rad_forward_grid(const RArgs& a, cudaStream_t s);
// adjoint grid -> image: column DFT (sign +1), then the row DFT fused with
// the crop, deapodisation and coil combination with conj(b1) into img
void launch_rad_adjoint_image(const RArgs& a, float2* img, cudaStream_t s);
// samples (a.z, or a.in as samples when from_in) -> grid, by sector gather
void launch_rad_spread(const RArgs& a, const float2* samples, cudaStream_t s);

}  // namespace avx
