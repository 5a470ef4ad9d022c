/*
 * avionic.h -- C ABI of the AVIONIC B200 reconstruction core (libavionic_core.so).
 *
 * Drop-in boundary for the reference's reconstruction path.  Each entry point
 * replaces one piece of the reference's C++ interface (citations are paths in
 * the IMTtugraz/AVIONIC tree):
 *
 *   operators  <- BaseOperator / CartesianOperator
 *                 (CUDA/include/base_operator.h:24-112,
 *                  CUDA/include/cartesian_operator.h:22-125)
 *   solvers    <- PDRecon / TV / TVTEMP / TGV2 / ICTV / ICTGV2
 *                 (CUDA/include/pd_recon.h:88-185, tv.h, tv_temp.h, tgv2.h,
 *                  ictv.h, ictgv2.h)
 *   utils      <- namespace utils stencils, norms, proximal maps, Ellipke
 *                 (CUDA/include/utils.h, CUDA/src/utils.cpp)
 *   host path  <- the avionic CLI's load -> reconstruct -> store sequence
 *                 (CUDA/src/main.cpp:323-917)
 *
 * Conventions.  complex64 values are avx_cf32 {re, im} (the memory layout of
 * std::complex<float>, CUDA/include/types.h:16).  Layouts follow the reference:
 * image x + W*(y + H*t); k-space x + W*(y + H*(c + C*t)); coil maps
 * x + W*(y + H*c); mask float x + W*(y + H*t).  Pointers named d_* are CUDA
 * device pointers of the current device; h_* are host pointers.  Functions
 * return avx_status and never throw; avx_last_error() describes the last
 * failure of the calling thread.  Nothing here allocates on the host-visible
 * side beyond the opaque handles.
 */
#ifndef AVIONIC_H_
#define AVIONIC_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct avx_cf32 {
  float re, im;
} avx_cf32;

typedef enum avx_status {
  AVX_OK = 0,
  AVX_E_ARG = 1,         /* invalid argument or dimension mismatch */
  AVX_E_CUDA = 2,        /* CUDA runtime error */
  AVX_E_NOMEM = 3,       /* device allocation failed */
  AVX_E_IO = 4,          /* file could not be read or written */
  AVX_E_UNSUPPORTED = 5, /* method or mode not provided by this library */
  AVX_E_NUMERIC = 6      /* non-finite value detected in a result */
} avx_status;

/* Method numbers of the reference's Method enum (CUDA/include/options_parser.h,
 * parsed at CUDA/src/options_parser.cpp:5-48). */
enum {
  AVX_METHOD_TV = 0,
  AVX_METHOD_TVTEMP = 1,
  AVX_METHOD_TGV2 = 2,
  AVX_METHOD_TGV2_3D = 3,
  AVX_METHOD_ICTV = 4,
  AVX_METHOD_ICTGV2 = 5
};

/* Union of PDParams, TVtempParams, TGV2Params, ICTVParams and ICTGV2Params
 * (CUDA/include/pd_recon.h:20-74, tv_temp.h:14-16, tgv2.h:9-16, ictv.h:8-23,
 * ictgv2.h:9-21) plus the
 * AdaptLambdaParams (pd_recon.h:20-32).  Fields a method does not use are
 * ignored. */
typedef struct avx_pd_params {
  unsigned maxIt;
  float stopPDGap;
  float sigma, tau, sigmaTauRatio;
  float timeSpaceWeight;
  float lambda;
  float dx, dy, dt;          /* overwritten from timeSpaceWeight by a run, as in the reference
                                (TVtemp keeps them: its dt weights the temporal difference) */
  float alpha0, alpha1;      /* alpha0: TGV2 / ICTGV2; alpha1: TGV2 / ICTV / ICTGV2 */
  float alpha;               /* ICTV / ICTGV2 trade-off */
  float timeSpaceWeight2;    /* ICTV / ICTGV2 second branch */
  float dx2, dy2, dt2;       /* ICTV / ICTGV2 second branch (overwritten by a run) */
  int adaptLambda;           /* 1: lambda = AdaptLambda(adaptK, adaptD) at solver creation */
  float adaptK, adaptD;
} avx_pd_params;

typedef struct avx_run_stats {
  unsigned iterations;   /* PD iterations executed */
  float sigma, tau;      /* final step sizes */
  unsigned gap_count;    /* gap evaluations recorded */
  double last_gap;       /* last normalised gap (gap / N) */
  int stopped_by_gap;    /* 1 when stopPDGap ended the run early */
  float elapsed_ms;      /* device time of the iteration loop */
  unsigned kernel_launches; /* kernels this library launched in the loop */
} avx_run_stats;

typedef struct avx_operator avx_operator;
typedef struct avx_solver avx_solver;

/* Export callback: the reference's ResultExportCallback
 * (CUDA/include/pd_recon.h:76) with the data already on the host. */
typedef void (*avx_export_cb)(const char* output_dir, const char* name, const avx_cf32* values,
                              size_t n, void* user);

const char* avx_version(void);
const char* avx_last_error(void);

/* ------------------------------------------------------------------ */
/* Cartesian operator                                                  */
/* ------------------------------------------------------------------ */

/* CartesianOperator(width, height, coils, frames, mask, centered)
 * (CUDA/src/cartesian_operator.cpp:3-34).  d_mask may be NULL (the reference's
 * empty-mask constructors).  The mask is copied; the operator does not keep
 * d_mask. */
avx_status avx_cartesian_operator_create(unsigned width, unsigned height, unsigned coils, unsigned frames,
                                         const float* d_mask, int centered, avx_operator** op);

/* Arithmetic of the Cartesian operator's transform along y (no reference
 * counterpart; the reference applies cuFFT in fp32):
 *   AVX_DFT_FP32           fp32 CUDA-core partial DFT
 *   AVX_DFT_SPLIT_BF16X3   tcgen05 tensor-core partial DFT with operands split
 *                          into three bf16 pieces (six piece products, fp32
 *                          accumulation; fp32-level accuracy)
 * The split form needs at most 48 sampled rows per frame; otherwise
 * AVX_E_UNSUPPORTED is returned and the mode is unchanged.  New operators
 * use the split form when it applies.  The radial operator ignores this. */
typedef enum avx_dft_mode { AVX_DFT_FP32 = 0, AVX_DFT_SPLIT_BF16X3 = 1 } avx_dft_mode;
avx_status avx_operator_set_dft_mode(avx_operator* op, int mode);
avx_status avx_operator_get_dft_mode(const avx_operator* op, int* mode);

/* NoncartesianOperator(width, height, coils, frames, nSpokes, nFE,
 * spokesPerFrame, kTraj, dens, kernelWidth, sectorWidth, osf)
 * (CUDA/src/noncartesian_operator.cpp:3-86): the radial gridding operator.
 * d_traj holds per frame [kx(S) | ky(S)] in cycles/pixel, within [-0.5, 0.5]
 * (AVX_E_ARG otherwise)
 * (S = nFE * spokesPerFrame); d_dens the density compensation w per frame
 * and sample.  K x = sqrt(w) NUFFT(b1 x) / sqrt(W H) with a tapered
 * Kaiser-Bessel gridding of width kernelWidth on a grid oversampled by osf,
 * sector-sorted by sectorWidth; k-space layout [frame][coil][sample]
 * (noncartesian_operator.cpp:117-121).  The operator uses the coil maps of each
 * call (the reference bakes them into its gpuNUFFT operators). */
avx_status avx_radial_operator_create(unsigned width, unsigned height, unsigned coils, unsigned frames,
                                      unsigned nSpokes, unsigned nFE, unsigned spokesPerFrame, const float* d_traj,
                                      const float* d_dens, float kernelWidth, float sectorWidth, float osf,
                                      avx_operator** op);

/* Sector layout of a radial operator, for inspection: h_order [T*S] sample
 * indices sorted by sector (stable), h_start [T*(nsectors+1)] offsets, grid_xy
 * the oversampled grid size (Gx, Gy).  Any output may be NULL.  (No reference
 * counterpart: gpuNUFFT keeps its sector map internal.) */
avx_status avx_radial_sector_map(const avx_operator* op, int* h_order, int* h_start, int* grid_xy);

/* BackwardOperation(img -> k-space) (cartesian_operator.cpp:122-160):
 * d_k[t,c] = mask[t] * F(b1[c] * x[t]); d_k is dense (W*H*C*T). */
avx_status avx_operator_backward(avx_operator* op, const avx_cf32* d_x, avx_cf32* d_k, const avx_cf32* d_b1);

/* ForwardOperation(k-space -> img) (cartesian_operator.cpp:65-111):
 * d_x[t] = sum_c conj(b1[c]) F^-1(mask[t] * k[t,c]).  Like the reference, it
 * multiplies d_k by the mask in place. */
avx_status avx_operator_forward(avx_operator* op, avx_cf32* d_k, avx_cf32* d_x, const avx_cf32* d_b1);

/* AdaptLambda(k, d) (cartesian_operator.cpp:47-62). */
avx_status avx_operator_adapt_lambda(const avx_operator* op, float k, float d, float* lambda_out);

void avx_operator_destroy(avx_operator* op);

/* ------------------------------------------------------------------ */
/* Primal-dual solvers                                                 */
/* ------------------------------------------------------------------ */

/* InitParams() defaults of TV / TVTEMP / TGV2 / ICTV / ICTGV2 (tv.cpp:39-57,
 * tv_temp.cpp:39-54, tgv2.cpp:36-56, ictv.cpp:37-60, ictgv2.cpp:37-63), with
 * adaptLambda = 1 and the method's (k, d).  TVtemp's dx and dy, which its
 * InitParams leaves unset and only its gap's TV norm reads, are 1. */
avx_status avx_default_params(int method, avx_pd_params* params);

/* TV/TVTEMP/TGV2/ICTV/ICTGV2(width, height, coils, frames, params, mrOp)
 * (tv.cpp:13-19, tv_temp.cpp:13-19, tgv2.cpp:10-16, ictv.cpp:11-17,
 * ictgv2.cpp:11-17).  params == NULL uses
 * avx_default_params.  When params->adaptLambda is set, lambda is replaced
 * by AdaptLambda(adaptK, adaptD) here (InitLambda, tv.cpp:25-37).  The
 * solver keeps a pointer to op, which must outlive it. */
avx_status avx_solver_create(int method, unsigned width, unsigned height, unsigned coils, unsigned frames,
                             const avx_pd_params* params, avx_operator* op, avx_solver** solver);

avx_status avx_solver_get_params(const avx_solver* s, avx_pd_params* params); /* GetParams() */
avx_status avx_solver_set_params(avx_solver* s, const avx_pd_params* params);
avx_status avx_solver_set_verbose(avx_solver* s, int verbose);               /* SetVerbose */
avx_status avx_solver_set_debug(avx_solver* s, int debug, int debugstep);    /* SetDebug */
/* No reference counterpart (the reference stops on the absolute gap only,
 * tv.cpp:189, tgv2.cpp:325, ictgv2.cpp:478): rel > 0 also ends the run at the
 * first gap evaluation with gap <= rel * (the run's first gap).  Evaluations
 * then happen every 20 iterations, as with stopPDGap.  rel in [0, 1). */
avx_status avx_solver_set_relative_stop(avx_solver* s, double rel);
avx_status avx_solver_set_stream(avx_solver* s, void* cuda_stream);          /* cudaStream_t, 0 = default */

/* No reference counterpart (the reference's AGILE kernels have fixed launch
 * shapes).  Launch shapes of the dual and primal kernels: with autotune set
 * (the default) the first run of a (device, method, W, H, T) times each
 * candidate on the solver's own fields, keeps the fastest and reuses it for
 * later runs and solvers of that shape in the process; with autotune clear
 * the given indices are used.  primal_tile in [0, 7): 32x8x1, 32x4x2, 64x4x1,
 * 32x4x4, 32x16x1 (threads along x, threads along y, pixels per thread along
 * y), then 128 and 256 threads with two pixels per thread and 128-bit
 * accesses (TGV2 and ICTGV2 with an even width; otherwise tile 0); dual_block in [0, 6): 256, 128, 512 threads with one pixel per thread,
 * then 256, 128, 512 threads with two pixels per thread and 128-bit
 * accesses (TGV2 and ICTGV2 with an even width; otherwise the one-pixel
 * kernel of that block size).  Index 0 is the default shape.  The shapes change the schedule only: every pixel's arithmetic is
 * the same in all of them (results agree to rounding; the compiler may fuse
 * multiply-adds differently in each). */
avx_status avx_solver_set_tuning(avx_solver* s, int autotune, int primal_tile, int dual_block);
/* The shapes in use (chosen by the autotuner after the first run); any output may be NULL. */
avx_status avx_solver_get_tuning(const avx_solver* s, int* primal_tile, int* dual_block, const char** primal_name,
                                 int* dual_threads);
/* FFT schedule of the Cartesian operator's row kernel: compact rows per pass
 * (8, 12 or 16; 16 by default) and the radix plan (0: the compile-time plan
 * of the row length when it has one, leading with radix-8 passes; 1: the
 * run-time plan).  With autotune set (avx_solver_set_tuning) the first run of
 * a (device, method, W, H, T, C, sampled rows per frame) times the candidate
 * schedules on the solver's own fields and keeps the fastest, replacing what
 * is set here.  Rows per pass change the schedule only; the two radix plans
 * round differently (results agree to fp32 rounding). */
avx_status avx_solver_set_kspace_schedule(avx_solver* s, int rows_per_pass, int runtime_plan);
avx_status avx_solver_get_kspace_schedule(const avx_solver* s, int* rows_per_pass, int* runtime_plan);

/* IterativeReconstruction(data, x, b1) (pd_recon.h:134-135): d_data dense
 * k-space (W*H*C*T), d_x initial image in / result out (W*H*T), d_b1 coil maps
 * (W*H*C).  Runs asynchronously on the solver's stream until the final
 * stop-state read, then returns. */
avx_status avx_solver_run(avx_solver* s, const avx_cf32* d_data, avx_cf32* d_x, const avx_cf32* d_b1);

/* AdaptStepSize on given extragradient differences (tv.cpp:79-97,
 * tv_temp.cpp:80-95, tgv2.cpp:89-128, ictv.cpp:97-128, ictgv2.cpp:97-161).
 * d_diff holds P component pointers (TV, TVtemp 1: e; ICTV 2: e1, e3;
 * TGV2 4: e1, e2[3]; ICTGV2 8: e1, e2[3], e3, e4[3]).  ICTV's norm of K e
 * covers the data term alone: the reference's gradient sums land in a buffer
 * that it then overwrites (ictv.cpp:104-125). */
avx_status avx_solver_adapt_step_size(avx_solver* s, const avx_cf32* const* d_diff, const avx_cf32* d_b1);

/* ComputeGStar / ComputePDGap (tv.cpp:202-235, tv_temp.cpp:184-224,
 * tgv2.cpp:130-176, ictv.cpp:146-200, ictgv2.cpp:178-249) on given primal
 * components (P pointers, as above), dual components (D pointers: TV 3,
 * TVtemp 1, ICTV 6, TGV2 9, ICTGV2 18), dense z and data.  The
 * gap is returned un-normalised, as ComputePDGap returns it.  Uses the
 * solver's current params (dx.. as set, no time-space recomputation). */
avx_status avx_solver_compute_gap(avx_solver* s, const avx_cf32* const* d_x, const avx_cf32* const* d_y,
                                  const avx_cf32* d_z, const avx_cf32* d_data, const avx_cf32* d_b1,
                                  double* gstar, double* gap);

/* Operator-norm estimate by power iteration, getopnorm (matlab/getopnorm.m:1-17;
 * its call in matlab/ls_pd.m:43-56 passes the encoding operator):
 *   y = K^H K x0;  iters times: x = y / ||y|| (y when ||y|| = 0), y = K^H K x, l = y^H x;
 *   *opnorm = |l|, an estimate of ||K||^2 (the largest eigenvalue of K^H K).
 * avx_operator_opnorm: K is the encoding operator (coil maps d_b1, transform,
 * mask or gridding; image -> k-space), d_x0 the start image (W*H*T values;
 * the reference draws it from randn).
 * avx_solver_opnorm: K is the solver's whole primal-dual operator, the
 * method's regularisation part (with the time-space weights a run would use)
 * stacked on the encoding operator, K^H the map of its primal update; the
 * symmetrised gradient's off-diagonal entries count twice in the dual inner
 * product, as in the step rule.  d_x0 starts the image component; the
 * auxiliary primal components start at zero.  With set_steps nonzero the
 * solver's initial steps become sigma = r / sqrt(l), tau = 1 / (r sqrt(l))
 * (r = sigmaTauRatio: the reference's sig = s r, tau = s / r with
 * s = 1 / ||K|| in place of 1/3, matlab/tgv2_dmri.m:96-99); a run still adapts
 * them by AdaptStepSize.
 * Operator applications run in the operator's arithmetic (fp32, or the split
 * form), norms and inner products in FP64 on the device.  iters >= 1 (the
 * reference uses 10).  hist (optional) receives |y^H x| after each of the
 * iters + 1 applications. */
avx_status avx_operator_opnorm(avx_operator* op, const avx_cf32* d_x0, const avx_cf32* d_b1, unsigned iters,
                               double* opnorm, double* hist);
avx_status avx_solver_opnorm(avx_solver* s, const avx_cf32* d_x0, const avx_cf32* d_b1, unsigned iters,
                             int set_steps, double* opnorm, double* hist);

/* ExportAdditionalResults (tv.cpp:237-248, tv_temp.cpp:226-236,
 * tgv2.cpp:340-355, ictv.cpp:372-391, ictgv2.cpp:494-516): x3_component
 * (ICTV, ICTGV2), and with debug on PDGap, ICTGVnorm and DATAfidelity
 * (ICTGV2), ictvnorm and DATAfidelity (ICTV). */
avx_status avx_solver_export(avx_solver* s, const char* output_dir, avx_export_cb cb, void* user);
avx_status avx_solver_get_stats(const avx_solver* s, avx_run_stats* stats);

/* Per-stage timing: with timing on, a run launches its kernels directly
 * (not from CUDA graphs) with CUDA events between the five stages of every
 * iteration on the solver's stream.  avx_solver_kernel_times writes the mean
 * durations in ms of the last run to mean_ms[0..4]:
 *   [0] dual update
 *   [1] forward transform: y-DFT of b1 x onto the sampled rows (Cartesian),
 *       zero-pad + oversampled FFT (radial)
 *   [2] k-space: row FFT, data prox, inverse row FFT (Cartesian),
 *       interpolation + data prox (radial)
 *   [3] adjoint: column IDFT + coil combine (Cartesian), spreading + FFT +
 *       crop (radial)
 *   [4] primal update
 * and to *count how many iterations were timed. */
avx_status avx_solver_set_timing(avx_solver* s, int on);
avx_status avx_solver_kernel_times(const avx_solver* s, float* mean_ms, unsigned* count);
void avx_solver_destroy(avx_solver* s);

/* ------------------------------------------------------------------ */
/* utils: stencils, norms, proximal maps (device pointers, 3D W x H x T) */
/* ------------------------------------------------------------------ */

/* utils::Gradient (utils.cpp:99-118): d_g[0..2] = D+x u/dx, D+y u/dy, D+t u/dt */
avx_status avx_gradient(const avx_cf32* d_u, avx_cf32* const* d_g, unsigned W, unsigned H, unsigned T,
                        float dx, float dy, float dt);
/* utils::Divergence (utils.cpp:733-757) */
avx_status avx_divergence(const avx_cf32* const* d_y, avx_cf32* d_div, unsigned W, unsigned H, unsigned T,
                          float dx, float dy, float dt);
/* utils::SymmetricGradient, 7-argument form (utils.cpp:397-456) */
avx_status avx_sym_gradient(const avx_cf32* const* d_v, avx_cf32* const* d_e, unsigned W, unsigned H,
                            unsigned T, float dx, float dy, float dt);
/* utils::SymmetricDivergence, 8-argument form (utils.cpp:961-1012) */
avx_status avx_sym_divergence(const avx_cf32* const* d_w, avx_cf32* const* d_d, unsigned W, unsigned H,
                              unsigned T, float dx, float dy, float dt);
/* utils::ProximalMap3 / ProximalMap6 (utils.cpp:1341-1351), in place */
avx_status avx_prox3(avx_cf32* const* d_y, unsigned N, float scale);
avx_status avx_prox6(avx_cf32* const* d_y, unsigned N, float scale);
/* utils::GradientNorm / SymmetricGradientNorm (utils.cpp:209-222, 610-631): real norms */
avx_status avx_norm3(const avx_cf32* const* d_g, float* d_norm, unsigned N);
avx_status avx_norm6(const avx_cf32* const* d_g, float* d_norm, unsigned N);
/* utils::TVNorm / TGV2Norm / ICTGV2Norm (utils.cpp:1119-1287), FP64 sums */
avx_status avx_tv_norm(const avx_cf32* d_u, unsigned W, unsigned H, unsigned T, float dx, float dy, float dt,
                       double* out);
avx_status avx_tgv2_norm(const avx_cf32* d_x1, const avx_cf32* const* d_x2, float alpha0, float alpha1,
                         unsigned W, unsigned H, unsigned T, float dx, float dy, float dt, double* out);
avx_status avx_ictgv2_norm(const avx_cf32* d_x1, const avx_cf32* const* d_x2, const avx_cf32* d_x3,
                           const avx_cf32* const* d_x4, float alpha0, float alpha1, float alpha, unsigned W,
                           unsigned H, unsigned T, const float* w1 /*dx,dy,dt*/, const float* w2, double* out);
/* TV norm that allocates nothing (no counterpart in the reference).  Same
 * result as avx_tv_norm, for callers that cannot allocate device memory when
 * they need it: the partial sums live in a fixed 64 KiB __device__ array that
 * every GPU loading the library holds until exit.  W*H*T must not exceed
 * 2,097,152 pixels (AVX_E_ARG otherwise).  The first call on a device resolves
 * the array's address and should precede any stream capture; the address is
 * kept for the process, so the entry point must not be used on a device after
 * cudaDeviceReset.  Calls that overlap on the GPU race on the shared array.
 * Runs on the legacy default stream and returns after the result reached
 * *out. */
avx_status avx_tv_norm_noalloc(const avx_cf32* d_u, unsigned W, unsigned H, unsigned T, float dx, float dy,
                               float dt, double* out);

/* utils::Ellipke (utils.cpp:18-47); returns NaN outside [0, 1] */
float avx_ellipke(float m);
/* PDRecon::ComputeTimeSpaceWeights (pd_recon.cpp:72-98) */
avx_status avx_time_space_weights(float time_space_weight, float* ds, float* dt);

/* ------------------------------------------------------------------ */
/* Coil-sensitivity estimation (CoilConstruction,                       */
/* CUDA/src/coil_construction.cpp, cartesian_coil_construction.cpp)     */
/* ------------------------------------------------------------------ */

/* CoilConstructionParams (CUDA/include/coil_construction.h:19-41) */
typedef struct avx_coil_params {
  float uH1mu, uReg;
  unsigned uNrIt;
  float uTau, uSigma, uSigmaTauRatio, uAlpha0, uAlpha1;
  float b1Reg;
  unsigned b1NrIt;
  float b1Tau, b1Sigma, b1SigmaTauRatio, b1FinalReg;
  unsigned b1FinalNrIt;
} avx_coil_params;

/* CoilConstruction::InitParams (coil_construction.cpp:22-48) */
avx_status avx_coil_default_params(avx_coil_params* p);

/* CartesianCoilConstruction::TimeAveragedReconstruction
 * (cartesian_coil_construction.cpp:23-86), uncentred transform:
 * crec_c = F^-1(sum_t k_{t,c} / max(1, sum_t mask_t)); u = sqrt(sum_c
 * |crec_c|^2), times the phase of sum_c crec_c when apply_phase.
 * d_mask may be NULL (all ones).  d_u: W*H, d_crec: W*H*C. */
avx_status avx_coil_time_averaged(unsigned W, unsigned H, unsigned C, unsigned T, const avx_cf32* d_kdata,
                                  const float* d_mask, avx_cf32* d_u, avx_cf32* d_crec, int apply_phase);

/* B1FromUH1 (coil_construction.cpp:363-445): per coil the solution of
 * (uH1mu |u|^2 - Laplace_periodic) b = conj(u) uH1mu |crec_c|, normalised
 * over coils; returns |b1|.  Solved by FP64 conjugate gradients to a relative
 * residual of 1e-12 (the reference stops at 800 FP32 iterations). */
avx_status avx_coil_b1_from_u_h1(unsigned W, unsigned H, unsigned C, const avx_coil_params* p, const avx_cf32* d_u,
                                 const avx_cf32* d_crec, avx_cf32* d_absb1);

/* UTGV2Recon (coil_construction.cpp:75-215) on the coils listed in h_inds;
 * d_x1 (W*H) is the initial image and receives the result. */
avx_status avx_coil_utgv2(unsigned W, unsigned H, const avx_coil_params* p, const avx_cf32* d_b1,
                          const avx_cf32* d_crec, const int* h_inds, unsigned ninds, avx_cf32* d_x1);

/* B1Recon (coil_construction.cpp:217-361) for `coils` coil images. */
avx_status avx_coil_b1_recon(unsigned W, unsigned H, unsigned coils, unsigned max_it, float mu,
                             const avx_coil_params* p, const avx_cf32* d_u0, const avx_cf32* d_crec, avx_cf32* d_b1);

/* PerformCoilConstruction (coil_construction.cpp:447-556), Cartesian data:
 * d_u receives the C image estimates (W*H*C, the last is the initial image
 * the CLI uses, main.cpp:634), d_b1 the coil maps (W*H*C).  p may be NULL. */
avx_status avx_coil_construction(unsigned W, unsigned H, unsigned C, unsigned T, const avx_coil_params* p,
                                 const avx_cf32* d_kdata, const float* d_mask, avx_cf32* d_u, avx_cf32* d_b1);

/* NoncartesianCoilConstruction::TimeAveragedReconstruction
 * (noncartesian_coil_construction.cpp:21-127): all frames' samples through
 * one radial gridding adjoint (kernel width 3, sector width 8, osf 2) per
 * coil.  d_traj/d_dens/d_kdata as for avx_radial_operator_create and the
 * radial k-space layout; S samples per frame. */
avx_status avx_coil_time_averaged_radial(unsigned W, unsigned H, unsigned C, unsigned T, unsigned S,
                                         const float* d_traj, const float* d_dens, const avx_cf32* d_kdata,
                                         avx_cf32* d_u, avx_cf32* d_crec, int apply_phase);

/* PerformCoilConstruction for radial data (main.cpp:210-248). */
avx_status avx_coil_construction_radial(unsigned W, unsigned H, unsigned C, unsigned T, unsigned S,
                                        const avx_coil_params* p, const float* d_traj, const float* d_dens,
                                        const avx_cf32* d_kdata, avx_cf32* d_u, avx_cf32* d_b1);

/* Data normalisation of the CLI's -o switch (main.cpp:573-579 ->
 * RawDataPreparation::NormalizeData, raw_data_preparation.cpp:340-378).
 * Cartesian (S == 0; d_mask = W*H*T mask, d_dens unused): the time-averaged
 * coil combination |u| of the centred transform (NormalizeCartData,
 * :821-844), factor 255 / m.  Radial (S > 0 samples per frame; d_mask = the
 * trajectory, d_dens the density): |u| = sqrt(sum_c |crec_c|^2) of the radial
 * time average (NormalizeNonCartData, :742-786), factor 255 T / m.  m is
 * FindNormalizationFactor (:661-686): the median of the first maximum of |u|
 * and every later value >= 0.9 of it.  d_kdata (the CLI's masked or
 * sqrt(w)-weighted k-space) is scaled in place; *datanorm receives the
 * factor (written as datanorm_factor.bin by the CLI, main.cpp:793-796).
 * AVX_E_NUMERIC when |u| is zero everywhere. */
avx_status avx_normalize_data(unsigned W, unsigned H, unsigned C, unsigned T, unsigned S, const float* d_mask,
                              const float* d_dens, avx_cf32* d_kdata, float* datanorm);

/* ------------------------------------------------------------------ */
/* Batched and served reconstructions                                  */
/* ------------------------------------------------------------------ */

/* No reference counterpart: the reference runs one reconstruction per
 * process (main.cpp:789).  An engine batches reconstructions continuously, at
 * iteration granularity.  Submitted requests wait in a queue; set-up threads
 * admit the first one whose device workspace fits the engine's HBM budget (a
 * request that has waited 2 s blocks later ones until it fits) and build its
 * operator, solver, device state and iteration graphs on a stream of its own,
 * with memory from the device's stream-ordered pool.  One scheduler thread
 * advances up to `workers` admitted requests together, 20 iterations (one
 * gap cadence) at a time with two such slices in flight per request, reads
 * each request's device state after every slice without blocking, and
 * retires a request at its stop test (stopPDGap, the normalised gap of the
 * reference, tgv2.cpp:317-330, or stop_gap_rel) or at maxIt, which frees its
 * budget for the next admission.  Requests of any mix of sizes, methods and
 * operators share the GPU this way; each result equals avx_solver_run on the
 * same inputs and parameters, bit for bit.  Buffers are the caller's device
 * buffers and must stay valid until the request's completion is polled. */
typedef struct avx_request {
  int method;                /* AVX_METHOD_TV / _TVTEMP / _TGV2 / _ICTV / _ICTGV2 */
  int op_kind;               /* 0 Cartesian, 1 radial */
  unsigned width, height, coils, frames;
  avx_pd_params params;      /* as for avx_solver_create (lambda adapted when asked) */
  int dft_mode;              /* Cartesian: preferred AVX_DFT_*; fp32 when the split form does not apply */
  const float* d_mask;       /* Cartesian: T*H*W mask or NULL */
  int centered;              /* Cartesian: centred FFT */
  unsigned n_fe, spokes_per_frame;          /* radial: samples per spoke, spokes per frame */
  const float* d_traj;                      /* radial: T x 2 x S trajectory in [-0.5, 0.5) */
  const float* d_dens;                      /* radial: T x S density compensation */
  float kernel_width, sector_width, osf;    /* radial: gridding parameters */
  const avx_cf32* d_data;    /* k-space: Cartesian T*C*H*W (masked), radial T*C*S (sqrt(w)-weighted) */
  avx_cf32* d_x;             /* T*H*W initial image in, reconstruction out */
  const avx_cf32* d_b1;      /* C*H*W coil maps */
  unsigned long long tag;    /* returned with the completion */
  float stop_gap_rel;        /* > 0: avx_solver_set_relative_stop(stop_gap_rel) for this run */
} avx_request;

typedef struct avx_completion {
  unsigned long long tag;
  int status;                /* avx_status of the run */
  int dft_mode;              /* form the Cartesian operator used */
  avx_run_stats stats;
  double queue_ms;           /* submit -> start (host clock) */
  double run_ms;             /* admission -> finished, set-up included (host clock) */
  size_t workspace_bytes;    /* the admission estimate */
} avx_completion;

typedef struct avx_batch avx_batch;

/* Device bytes a request needs while it runs (operator, solver, tables): an
 * upper bound that counts the Cartesian k-space at every row, since the mask
 * is not read at submission; admission holds this much until the request's
 * operator is built and then only its exact footprint. */
avx_status avx_query_workspace(const avx_request* r, size_t* bytes);
/* device: CUDA ordinal; hbm_budget: bytes the admitted requests may hold
 * together; workers: requests advanced together at most (>= 1; 1 runs them
 * one after another, each set up while the previous one runs). */
avx_status avx_batch_create(int device, size_t hbm_budget, int workers, avx_batch** out);
/* Queues a copy of *r.  AVX_E_NOMEM when its workspace exceeds the whole budget. */
avx_status avx_batch_submit(avx_batch* b, const avx_request* r);
/* Moves up to max finished requests to out (*n of them), waiting up to
 * wait_ms for the first (0: do not wait, negative: until one finishes or
 * nothing is pending). */
avx_status avx_serve_poll(avx_batch* b, avx_completion* out, int max, int* n, int wait_ms);
/* Blocks until every submitted request has finished (completions stay queued). */
avx_status avx_batch_drain(avx_batch* b);
/* Requests submitted and not yet polled. */
int avx_batch_pending(const avx_batch* b);
/* Drops the queued requests, waits for the admitted ones and stops the engine's threads. */
void avx_batch_destroy(avx_batch* b);

/* ------------------------------------------------------------------ */
/* Host-buffer reconstruction (the CLI path, main.cpp:507-839)         */
/* ------------------------------------------------------------------ */

/* Copies the host inputs to the device, masks the data (main.cpp:507-519),
 * replicates u0 over the frames (main.cpp:775-779), runs the method and
 * copies the image back.  h_mask may be NULL (all ones); h_u0 is one frame
 * (W*H) or NULL (zeros).  debugstep > 0 enables the gap history
 * (options_parser.cpp:79).  stats may be NULL.  The operator, solver,
 * device buffers and CUDA graphs of the last call are kept and reused while
 * the device, method, sizes, parameters, debug step and mask contents stay
 * the same (calls are serialised by a lock); every call copies the data,
 * coil maps and u0 and starts from the given parameters.  No reference
 * counterpart: the reference's main builds everything per run. */
avx_status avx_reconstruct_host(int method, unsigned width, unsigned height, unsigned coils, unsigned frames,
                                const avx_pd_params* params, int debugstep, const avx_cf32* h_kdata,
                                const float* h_mask, const avx_cf32* h_b1, const avx_cf32* h_u0,
                                avx_cf32* h_x, avx_run_stats* stats);

/* Frees the state kept by avx_reconstruct_host (no reference counterpart). */
void avx_reconstruct_host_release(void);

#ifdef __cplusplus
}
#endif

#endif /* AVIONIC_H_ */
