// Host side of the AVIONIC B200 reconstruction core: the Cartesian operator,
// the TV / TGV2 / ICTGV2 solvers and the C ABI declared in include/avionic.h.
//
// A solver run follows TV/TGV2/ICTGV2::IterativeReconstruction of the
// reference (CUDA/src/tv.cpp:99-200, tgv2.cpp:180-338, ictgv2.cpp:294-492):
// time-space weights, zeroed duals, x and xbar from the initial image, then
// maxIt iterations with the step rule at k < 10 or k % 50 == 0 and the gap on
// the verbose/debug/stop cadence.  All scalars that steer the loop (sigma,
// tau, the gap, the stop flag) stay on the device, so iterations are
// enqueued without host synchronisation; each of the four iteration shapes
// (plain, +step, +gap, +step+gap) is captured once as a CUDA graph and
// replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/avionic.h"
#include "coils.cuh"
#include "fft.cuh"
#include "fft2d.cuh"
#include "opnorm.cuh"
#include "pd_kernels.cuh"
#include "radial.cuh"
#include "tc_dft.cuh"
#include "utils_kernels.cuh"



namespace {

thread_local std::string g_err;

avx_status fail(avx_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

#define AVX_CK(call)                                                                         \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? AVX_E_NOMEM : AVX_E_CUDA,                \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

// Set by the batch engine while it builds a request's operator and solver:
// their buffers come from the device's stream-ordered pool on that stream and
// go back to it with cudaFreeAsync, so that retiring a request never waits
// for the other requests' work (cudaFree would synchronise the device).
thread_local cudaStream_t t_pool_stream = nullptr;

// The library's own stream-ordered pool on the current device (created on
// first use).  It keeps up to kPoolKeep bytes of freed memory for the next
// allocations, so that repeated calls do not unmap and map memory; while a
// batch engine lives it keeps everything (pool_hold).  The attributes of the
// application's default pool are never changed.
constexpr unsigned long long kPoolKeep = 4ull << 30;
static cudaMemPool_t library_pool() {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  unsigned long long keep = kPoolKeep;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = pool;
  return pool;
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t pool_stream = nullptr;  // non-null: allocated from the stream-ordered pool
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p && pool_stream)
      cudaFreeAsync(p, pool_stream);
    else if (p)
      cudaFree(p);
    p = nullptr;
    n = 0;
    pool_stream = nullptr;
  }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    if (t_pool_stream) {
      cudaMemPool_t pool = library_pool();
      cudaError_t e = pool ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), bytes, pool, t_pool_stream)
                           : cudaErrorMemoryAllocation;
      // the set-up code fills some buffers with synchronous copies on the
      // legacy stream: make the allocation visible to every stream first
      if (e == cudaSuccess) e = cudaStreamSynchronize(t_pool_stream);
      if (e != cudaSuccess) {
        p = nullptr;
        return e;
      }
      n = count;
      pool_stream = t_pool_stream;
      return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = count;
    return e;
  }
};

// A private stream for one synchronous entry point, ordered after the legacy
// stream on entry; while it lives, DevBufs take their memory from the
// stream-ordered pool on it (no device-wide synchronisation in cudaFree).
// DevBufs declared after it release their memory on it before it syncs and
// goes away.
struct PoolScope {
  cudaStream_t s = nullptr, prev = nullptr;
  cudaError_t init() {
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      s = nullptr;
      return e;
    }
    cudaEvent_t ev;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) {
      e = cudaEventRecord(ev, 0);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
      cudaEventDestroy(ev);
    }
    prev = t_pool_stream;
    t_pool_stream = s;
    return e;
  }
  ~PoolScope() {
    if (!s) return;
    cudaStreamSynchronize(s);
    t_pool_stream = prev;
    cudaStreamDestroy(s);
  }
};

// Complete elliptic integral of the second kind by the AGM
// (utils::Ellipke, utils.cpp:18-47; Abramowitz & Stegun 17.6).
double ellipke_d(double m) {
  double a0 = 1.0, b0 = std::sqrt(1.0 - m), s0 = m, mm = 1.0, a1 = 1.0;
  int i1 = 0;
  while (mm > 1e-7) {
    a1 = (a0 + b0) / 2.0;
    const double b1 = std::sqrt(a0 * b0);
    const double c1 = (a0 - b0) / 2.0;
    ++i1;
    const double w1 = std::pow(2.0, i1) * c1 * c1;
    mm = w1;
    s0 += w1;
    a0 = a1;
    b0 = b1;
  }
  const double k = M_PI / (2.0 * a1);
  return k * (1.0 - s0 / 2.0);
}

// PDRecon::ComputeTimeSpaceWeights (pd_recon.cpp:72-98)
bool time_space_weights(double tsw, double* ds, double* dt) {
  double r = 1.0 / tsw, w1, w2;
  if (r > 0.0 && r <= 1.0) {
    w2 = M_PI / (2.0 * ellipke_d(1.0 - r * r));
    w1 = r * w2;
  } else if (r > 1.0) {
    r = 1.0 / r;
    w1 = M_PI / (2.0 * ellipke_d(1.0 - r * r));
    w2 = r * w1;
  } else {
    return false;
  }
  *ds = 1.0 / w1;
  *dt = 1.0 / w2;
  return true;
}

Wts make_wts(float dx, float dy, float dt) {
  Wts w;
  w.ix = (float)(1.0 / (double)dx);
  w.iy = (float)(1.0 / (double)dy);
  w.it = (float)(1.0 / (double)dt);
  w.hx = (float)(1.0 / (2.0 * (double)dx));
  w.hy = (float)(1.0 / (2.0 * (double)dy));
  w.ht = (float)(1.0 / (2.0 * (double)dt));
  return w;
}

// primal and dual component counts: TV 1 / 3, TVtemp 1 / 1, TGV2 4 / 9, ICTV 2 / 6, ICTGV2 8 / 18
int method_P(int m) {
  return m == AVX_METHOD_TV || m == AVX_METHOD_TVTEMP ? 1 : m == AVX_METHOD_ICTV ? 2 : m == AVX_METHOD_TGV2 ? 4 : 8;
}
int method_D(int m) {
  return m == AVX_METHOD_TVTEMP ? 1 : m == AVX_METHOD_TV ? 3 : m == AVX_METHOD_ICTV ? 6 : m == AVX_METHOD_TGV2 ? 9 : 18;
}
bool method_ok(int m) {
  return m == AVX_METHOD_TV || m == AVX_METHOD_TVTEMP || m == AVX_METHOD_TGV2 || m == AVX_METHOD_ICTV ||
         m == AVX_METHOD_ICTGV2;
}
// methods with a second TV branch (x3 component, second time-space weight, norm and fidelity histories)
bool method_ic(int m) { return m == AVX_METHOD_ICTV || m == AVX_METHOD_ICTGV2; }

__global__ void sumsq_kernel(const float2* v, long long n, double* partial) {
  __shared__ double red[32];
  double acc[1] = {0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc[0] += (double)cabs2(v[i]);
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc[0];
}

// FP64 sum of squared magnitudes (synchronous; used at set-up only)
avx_status sum_sq(const float2* v, long long n, cudaStream_t s, double* out) {
  DevBuf<double> part;
  AVX_CK(part.alloc(256));
  sumsq_kernel<<<256, 256, 0, s>>>(v, n, part.p);
  AVX_CK(cudaGetLastError());
  std::vector<double> h(256);
  AVX_CK(cudaMemcpyAsync(h.data(), part.p, 256 * sizeof(double), cudaMemcpyDeviceToHost, s));
  AVX_CK(cudaStreamSynchronize(s));
  double acc = 0.0;
  for (double x : h) acc += x;
  *out = acc;
  return AVX_OK;
}

// kernel attributes are per device: one bit per configured device
unsigned long long g_configured = 0;

avx_status configure_once() {
  int dev = 0;
  AVX_CK(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (g_configured & bit) return AVX_OK;
  AVX_CK(avx::configure_kernels());
  AVX_CK(avx::configure_radial_kernels());
  AVX_CK(avx::configure_fft2d_kernels());
  AVX_CK(avx::configure_tc_kernels());
  g_configured |= bit;
  return AVX_OK;
}

}  // namespace

void avx_internal_set_error(const char* msg) { g_err = msg; }

// ===========================================================================
// Cartesian operator
// ===========================================================================

// Radix passes of a length-n FFT (4s first, then 2, 3, 5, 7, 11, 13); empty
// when n has a larger prime factor, in which case the dense DFT is used.
static std::vector<int> fft_radices(int n) {
  std::vector<int> r;
  while (n % 4 == 0) { r.push_back(4); n /= 4; }
  for (int p : {2, 3, 5, 7, 11, 13})
    while (n % p == 0) { r.push_back(p); n /= p; }
  if (n != 1 || r.size() > 12) r.clear();
  return r;
}

struct avx_operator {
  int kind = 0;  // 0 Cartesian, 1 radial
  int W = 0, H = 0, C = 0, T = 0, centered = 0;
  std::vector<int> radx;
  // radial (gridding) operator
  int S = 0, spf = 0;
  RadialGeomDev rg{};
  DevBuf<float> r_traj, r_sqrtw, r_ipx, r_ipy;
  DevBuf<int> r_order, r_secstart, r_spread_list, r_spread_off, r_spread_blocks;
  DevBuf<int2> r_win0;
  DevBuf<float> r_winw;
  DevBuf<float2> r_twgx, r_twgy, r_grid;
  DevBuf<float2> r_khz;  // K^H z image (T x H x W), both operator kinds
  bool has_mask = false, binary = true;
  std::vector<int> rows, row_off;
  int R = 0;
  double mask_norm2 = 0.0;
  DevBuf<int> d_rows, d_row_off;
  DevBuf<float> d_mrow, d_mask;
  DevBuf<float2> d_twx, d_twy, d_qp;
  // split-BF16x3 tensor-core y-transform
  int dft_mode = AVX_DFT_FP32;
  int tc_np = 0;  // MMA N of the y-transform = MMA K of the column adjoint; 0: split form not available
  DevBuf<uint4> tc_ytab, tc_ctab;
  DevBuf<float2> tc_b1t;  // coil maps in column-tile order for operator applies

  CartGeomDev geom() const {
    CartGeomDev g;
    g.W = W; g.H = H; g.C = C; g.T = T;
    g.sx = centered ? W / 2 : 0;
    g.sy = centered ? H / 2 : 0;
    g.rows = d_rows.p;
    g.row_off = d_row_off.p;
    g.mrow = d_mrow.p;
    g.twx = d_twx.p;
    g.twy = d_twy.p;
    g.inv_sqrt_w = (float)(1.0 / std::sqrt((double)W));
    g.inv_sqrt_h = (float)(1.0 / std::sqrt((double)H));
    g.nrad = (int)radx.size();
    for (int i = 0; i < 12; ++i) g.rad[i] = i < g.nrad ? radx[i] : 0;
    return g;
  }
};

static avx_status build_operator(avx_operator* op, const float* h_mask) {
  const int W = op->W, H = op->H, T = op->T;
  op->has_mask = h_mask != nullptr;
  op->rows.clear();
  op->row_off.assign(T + 1, 0);
  std::vector<float> mrow;
  op->binary = true;
  op->mask_norm2 = 0.0;
  for (int t = 0; t < T; ++t) {
    op->row_off[t] = (int)op->rows.size();
    for (int y = 0; y < H; ++y) {
      bool keep = !op->has_mask;
      if (op->has_mask) {
        const float* m = h_mask + ((size_t)t * H + y) * W;
        for (int x = 0; x < W; ++x) {
          const float v = m[x];
          op->mask_norm2 += (double)v * v;
          if (v != 0.f) keep = true;
          if (v != 0.f && v != 1.f) op->binary = false;
        }
      }
      if (!keep) continue;
      op->rows.push_back(y);
      for (int x = 0; x < W; ++x) mrow.push_back(op->has_mask ? h_mask[((size_t)t * H + y) * W + x] : 1.f);
    }
  }
  op->row_off[T] = (int)op->rows.size();
  op->R = (int)op->rows.size();
  op->radx = fft_radices(W);
  std::vector<float2> twx(W), twy(H);
  for (int j = 0; j < W; ++j) twx[j] = make_float2((float)std::cos(2.0 * M_PI * j / W), (float)std::sin(2.0 * M_PI * j / W));
  for (int j = 0; j < H; ++j) twy[j] = make_float2((float)std::cos(2.0 * M_PI * j / H), (float)std::sin(2.0 * M_PI * j / H));
  AVX_CK(op->d_rows.alloc(std::max(op->R, 1)));
  AVX_CK(op->d_row_off.alloc(T + 1));
  AVX_CK(op->d_mrow.alloc(std::max<size_t>(mrow.size(), 1)));
  AVX_CK(op->d_twx.alloc(W));
  AVX_CK(op->d_twy.alloc(H));
  AVX_CK(op->d_qp.alloc((size_t)op->C * std::max(op->R, 1) * W));
  AVX_CK(op->r_khz.alloc((size_t)T * H * W));
  if (op->R) AVX_CK(cudaMemcpy(op->d_rows.p, op->rows.data(), op->R * sizeof(int), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(op->d_row_off.p, op->row_off.data(), (T + 1) * sizeof(int), cudaMemcpyHostToDevice));
  if (!mrow.empty()) AVX_CK(cudaMemcpy(op->d_mrow.p, mrow.data(), mrow.size() * sizeof(float), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(op->d_twx.p, twx.data(), W * sizeof(float2), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(op->d_twy.p, twy.data(), H * sizeof(float2), cudaMemcpyHostToDevice));
  if (op->has_mask) {
    AVX_CK(op->d_mask.alloc((size_t)T * H * W));
    AVX_CK(cudaMemcpy(op->d_mask.p, h_mask, (size_t)T * H * W * sizeof(float), cudaMemcpyHostToDevice));
  }
  // coefficient tables of the tensor-core transforms (at most 48 rows per frame)
  int max_rows = 0;
  for (int t = 0; t < T; ++t) max_rows = std::max(max_rows, op->row_off[t + 1] - op->row_off[t]);
  const int np = std::max(16, (2 * max_rows + 15) / 16 * 16);
  op->tc_np = 0;
  op->dft_mode = AVX_DFT_FP32;
  if (max_rows > 0 && np <= TC_MAX_NP) {
    std::vector<unsigned short> tab(avx::tc_ytab_bytes(H, T, np) / 2);
    avx::tc_build_ytab(W, H, T, op->centered ? W / 2 : 0, op->centered ? H / 2 : 0, op->rows.data(),
                       op->row_off.data(), np, tab.data());
    AVX_CK(op->tc_ytab.alloc(tab.size() * 2 / sizeof(uint4)));
    AVX_CK(cudaMemcpy(op->tc_ytab.p, tab.data(), tab.size() * 2, cudaMemcpyHostToDevice));
    std::vector<unsigned short> ctab(avx::tc_ctab_bytes(H, T, np) / 2);
    avx::tc_build_ctab(H, T, op->centered ? H / 2 : 0, op->rows.data(), op->row_off.data(), np, ctab.data());
    AVX_CK(op->tc_ctab.alloc(ctab.size() * 2 / sizeof(uint4)));
    AVX_CK(cudaMemcpy(op->tc_ctab.p, ctab.data(), ctab.size() * 2, cudaMemcpyHostToDevice));
    op->tc_np = np;
    op->dft_mode = AVX_DFT_SPLIT_BF16X3;
  }
  return AVX_OK;
}

// 64-point Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_n)
static void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      const double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-15) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

static double kb_weight(double u, double J, double beta) {
  if (!(std::fabs(u) < J / 2.0)) return 0.0;
  const double r = 2.0 * u / J;
  return (std::cyl_bessel_i(0.0, beta * std::sqrt(std::max(1.0 - r * r, 0.0))) - 1.0) /
         (std::cyl_bessel_i(0.0, beta) - 1.0);
}

static bool smooth13(int n) {
  for (int p : {2, 3, 5, 7, 11, 13})
    while (n % p == 0) n /= p;
  return n == 1;
}

// oversampled grid: the smallest even size >= osf * d whose prime factors are <= 13
static int radial_grid_size(int d, double osf) {
  int n = 2 * (int)std::ceil(osf * d / 2.0);
  while (!smooth13(n)) n += 2;
  return n;
}

// The gridding operator's tables.  d_traj [T][2][S] and d_dens [T][S] are
// device arrays; the per-sample tables (sector order, sqrt(w), windows,
// spreading work lists) are built on the device, the per-axis ones (twiddles,
// deapodisation) on the host.
static avx_status build_radial(avx_operator* op, const float* d_traj, const float* d_dens, float J, float sw, float osf) {
  const int W = op->W, H = op->H, T = op->T, S = op->S;
  if (!(J > 0.f && J <= 7.f)) return fail(AVX_E_ARG, "kernelWidth must lie in (0, 7]");
  if (!(osf > 1.0f)) return fail(AVX_E_ARG, "osf must exceed 1");
  const int isw = (int)sw;
  if (isw < 2 || isw > 32 || (float)isw != sw) return fail(AVX_E_ARG, "sectorWidth must be an integer in [2, 32]");
  RadialGeomDev& g = op->rg;
  g.W = W; g.H = H; g.C = op->C; g.T = T; g.S = S;
  g.Gx = radial_grid_size(W, osf);
  g.Gy = radial_grid_size(H, osf);
  g.sw = isw;
  g.nsx = (g.Gx + isw - 1) / isw;
  g.nsy = (g.Gy + isw - 1) / isw;
  const int lastx = g.Gx - (g.nsx - 1) * isw, lasty = g.Gy - (g.nsy - 1) * isw;
  if (J / 2.f > (float)std::min(lastx, lasty) || J / 2.f > (float)isw)
    return fail(AVX_E_ARG, "kernelWidth too wide for the sector layout");
  // the kernels wrap window offsets with one add or subtract, which needs the
  // trajectory in [-1/2, 1/2] and a grid wider than the window plus two cells
  if ((float)std::min(g.Gx, g.Gy) <= J + 2.f)
    return fail(AVX_E_ARG, "oversampled grid too small for the kernel width");
  {
    int flags = 0;
    AVX_CK(avx::rad_validate(d_traj, (long long)T * 2 * S, d_dens, (long long)T * S, &flags, 0));
    if (flags & 1) return fail(AVX_E_ARG, "trajectory values must lie in [-0.5, 0.5]");
    if (flags & 2) return fail(AVX_E_ARG, "density compensation must be non-negative");
  }
  g.nw = (int)std::ceil(J) + 1;
  g.J = J;
  const double beta = M_PI * std::sqrt((J / osf) * (J / osf) * (osf - 0.5) * (osf - 0.5) - 0.8);
  g.beta = (float)beta;
  g.kb_norm = (float)(1.0 / (std::cyl_bessel_i(0.0, beta) - 1.0));
  g.norm = (float)(1.0 / std::sqrt((double)W * H));
  // deapodisation psi(p) = int w(t) cos(2 pi t p / G) dt
  std::vector<double> gx, gw;
  gauss_legendre(64, gx, gw);
  auto deap = [&](int d, int G, std::vector<float>& inv) {
    inv.resize(d);
    for (int n = 0; n < d; ++n) {
      const double p = n - d / 2;
      double acc = 0.0;
      for (int i = 0; i < 64; ++i) {
        const double t = gx[i] * J / 2.0;
        acc += gw[i] * (J / 2.0) * kb_weight(t, J, beta) * std::cos(2.0 * M_PI * t * p / G);
      }
      inv[n] = (float)(1.0 / acc);
    }
  };
  std::vector<float> ipx, ipy;
  deap(W, g.Gx, ipx);
  deap(H, g.Gy, ipy);
  const int nsec = g.nsx * g.nsy;
  const std::vector<int> rx = fft_radices(g.Gx), ry = fft_radices(g.Gy);
  if (rx.empty() || ry.empty()) return fail(AVX_E_UNSUPPORTED, "grid size has no FFT plan");
  g.nradx = (int)rx.size();
  g.nrady = (int)ry.size();
  for (int i = 0; i < 12; ++i) {
    g.radx[i] = i < g.nradx ? rx[i] : 0;
    g.rady[i] = i < g.nrady ? ry[i] : 0;
  }
  if (avx::radial_fft_smem_bytes(std::max(g.Gx, g.Gy)) > AVX_DYN_SMEM_MAX ||
      avx::radial_adj_smem_bytes(g.Gx, W) > AVX_DYN_SMEM_MAX)
    return fail(AVX_E_UNSUPPORTED, "oversampled grid too large for the grid FFT tile");
  std::vector<float2> twx(g.Gx), twy(g.Gy);
  for (int j = 0; j < g.Gx; ++j) twx[j] = make_float2((float)std::cos(2.0 * M_PI * j / g.Gx), (float)std::sin(2.0 * M_PI * j / g.Gx));
  for (int j = 0; j < g.Gy; ++j) twy[j] = make_float2((float)std::cos(2.0 * M_PI * j / g.Gy), (float)std::sin(2.0 * M_PI * j / g.Gy));
  AVX_CK(op->r_traj.alloc((size_t)T * 2 * S));
  AVX_CK(op->r_sqrtw.alloc((size_t)T * S));
  AVX_CK(op->r_ipx.alloc(W));
  AVX_CK(op->r_ipy.alloc(H));
  AVX_CK(op->r_order.alloc((size_t)T * S));
  AVX_CK(op->r_secstart.alloc((size_t)T * (nsec + 1)));
  AVX_CK(op->r_twgx.alloc(g.Gx));
  AVX_CK(op->r_twgy.alloc(g.Gy));
  AVX_CK(op->r_grid.alloc((size_t)T * op->C * g.Gx * g.Gy));
  AVX_CK(op->r_khz.alloc((size_t)T * H * W));
  AVX_CK(cudaMemcpy(op->r_traj.p, d_traj, (size_t)T * 2 * S * sizeof(float), cudaMemcpyDeviceToDevice));
  AVX_CK(cudaMemcpy(op->r_ipx.p, ipx.data(), W * sizeof(float), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(op->r_ipy.p, ipy.data(), H * sizeof(float), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(op->r_twgx.p, twx.data(), g.Gx * sizeof(float2), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(op->r_twgy.p, twy.data(), g.Gy * sizeof(float2), cudaMemcpyHostToDevice));
  g.traj = op->r_traj.p;
  // sector of every sample in float32 arithmetic, then a stable sort by sector
  AVX_CK(avx::rad_build_order(g, d_dens, op->r_sqrtw.p, op->r_order.p, op->r_secstart.p, 0));
  g.sqrt_w = op->r_sqrtw.p;
  g.inv_psi_x = op->r_ipx.p;
  g.inv_psi_y = op->r_ipy.p;
  g.order = op->r_order.p;
  g.sec_start = op->r_secstart.p;
  g.twgx = op->r_twgx.p;
  g.twgy = op->r_twgy.p;
  // the samples' window starts and weights depend on the trajectory alone
  AVX_CK(op->r_win0.alloc((size_t)T * S));
  AVX_CK(op->r_winw.alloc((size_t)T * S * 2 * g.nw));
  avx::launch_rad_windows(g, op->r_win0.p, op->r_winw.p, 0);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(0));
  g.win0 = op->r_win0.p;
  g.winw = op->r_winw.p;
  // The spreading's work list.  Per (frame, sector), the samples whose window
  // reaches the sector's cells, in the order the sector sums them: the 3x3
  // neighbouring sectors in (dy, dx) order, each in sorted order (fewer than
  // three sectors along an axis wrap onto themselves and are taken once).
  // The CTAs are numbered heaviest list first, so that the central sectors,
  // which every spoke crosses, start in the first wave.
  {
    AVX_CK(op->r_spread_off.alloc((size_t)T * nsec + 1));
    long long total = 0;
    AVX_CK(avx::rad_count_lists(g, op->r_order.p, op->r_secstart.p, op->r_win0.p, op->r_spread_off.p, &total, 0));
    AVX_CK(op->r_spread_list.alloc(std::max<size_t>((size_t)total, 1)));
    AVX_CK(op->r_spread_blocks.alloc((size_t)T * nsec));
    AVX_CK(avx::rad_fill_lists(g, op->r_order.p, op->r_secstart.p, op->r_win0.p, op->r_spread_off.p,
                               op->r_spread_list.p, op->r_spread_blocks.p, 0));
    g.spread_list = op->r_spread_list.p;
    g.spread_off = op->r_spread_off.p;
    g.spread_blocks = op->r_spread_blocks.p;
  }
  return AVX_OK;
}

static RArgs make_rargs(avx_operator* op, const float2* b1, const float2* in, const float2* in2) {
  RArgs r;
  memset(&r, 0, sizeof(r));
  r.g = op->rg;
  r.b1 = b1;
  r.in = in;
  r.in2 = in2;
  r.grid = op->r_grid.p;
  return r;
}

static avx_status check_dims(unsigned W, unsigned H, unsigned C, unsigned T) {
  if (!W || !H || !C || !T) return fail(AVX_E_ARG, "dimensions must be positive");
  if (avx::kspace_smem_bytes((int)W, (int)H) > AVX_DYN_SMEM_MAX)
    return fail(AVX_E_UNSUPPORTED, "image size exceeds the k-space kernel's shared-memory tile");
  if ((double)W * H * T * C > 4.0e9) return fail(AVX_E_ARG, "problem too large for 32-bit row offsets");
  return AVX_OK;
}


// Cached device state of avx_reconstruct_host: the operator, solver, CUDA
// graphs and device buffers of the last call are reused while the problem
// (device, method, sizes, parameters, debug step and mask contents) is
// unchanged; the data, coil maps and initial image are copied every call.
struct avx_solver;
struct HostPlan {
  int device = -1, method = -1, debugstep = 0;
  unsigned W = 0, H = 0, C = 0, T = 0;
  avx_pd_params params{};      // as given by the caller
  avx_pd_params run_params{};  // as the solver holds them before its first run
  bool has_mask = false;
  std::vector<float> mask;
  DevBuf<float2> dk, db1, dx;
  DevBuf<float> dm;
  avx_operator* op = nullptr;
  avx_solver* s = nullptr;
  cudaStream_t stream = nullptr;
  bool matches(int dev, int m, unsigned w, unsigned h, unsigned c, unsigned t, int ds, const avx_pd_params* p,
               const float* h_mask) const {
    if (!s || dev != device || m != method || w != W || h != H || c != C || t != T || ds != debugstep) return false;
    if (memcmp(p, &params, sizeof(params)) != 0) return false;
    if ((h_mask != nullptr) != has_mask) return false;
    return !h_mask || memcmp(h_mask, mask.data(), mask.size() * sizeof(float)) == 0;
  }
  void release();
};
static std::mutex g_plan_mu;
static HostPlan g_plan;

// ===========================================================================
// Solver
// ===========================================================================

struct avx_solver {
  int method = 0;
  int W = 0, H = 0, C = 0, T = 0;
  avx_pd_params p{};
  avx_operator* op = nullptr;
  bool verbose = false, debug = false;
  int debugstep = 1;
  double stop_rel = 0.0;  // relative gap stop (avx_solver_set_relative_stop)
  // launch shapes of the dual and primal kernels (avx_solver_set_tuning)
  bool autotune = true, tuned = false;
  int primal_tile = 0, dual_block = 0;
  int rows_kc = KSPACE_KC, rows_rt = 0;  // row-FFT schedule (avx_solver_set_kspace_schedule)
  cudaStream_t user_stream = 0;
  cudaStream_t stream = 0;
  bool own_stream = false;  // stream created by solver_alloc (else lent by the batch engine)
  // device state
  DevBuf<float2> prim, ext, dual, escr, z, d;
  DevBuf<float2> b1t;  // coil maps in column-tile order (tensor-core adjoint)
  DevBuf<DevState> st;
  DevBuf<double> pimg, pk, hist;
  int cap = 0;
  double d_off_energy = 0.0;
  avx_run_stats stats{};
  DevState last{};
  // graphs of the four iteration shapes
  cudaGraphExec_t gexec[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t graph_key = 0;
  // timing mode
  bool timing = false;
  std::vector<cudaEvent_t> events;
  float kmean[AVX_NSTAGE] = {};
  unsigned kcount = 0;

  ~avx_solver() {
    drop_graphs();
    for (auto e : events) cudaEventDestroy(e);
    if (stream && own_stream) cudaStreamDestroy(stream);
  }
  void drop_graphs() {
    for (auto& g : gexec)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  long long N() const { return (long long)W * H * T; }
  float2* primc(int c) { return prim.p + (size_t)c * N(); }
  float2* extc(int c) { return ext.p + (size_t)c * N(); }
  float2* dualc(int c) { return dual.p + (size_t)c * N(); }
  float2* escrc(int c) { return escr.p + (size_t)c * N(); }
};

static avx_status solver_alloc(avx_solver* s) {
  const int P = method_P(s->method), D = method_D(s->method);
  const size_t N = (size_t)s->N();
  const size_t K = s->op->kind == 1 ? (size_t)s->C * s->T * s->op->S : (size_t)s->C * std::max(s->op->R, 1) * s->W;
  AVX_CK(s->prim.alloc(P * N));
  AVX_CK(s->ext.alloc(P * N));
  AVX_CK(s->dual.alloc(D * N));
  AVX_CK(s->escr.alloc(P * N));
  AVX_CK(s->z.alloc(K));
  AVX_CK(s->d.alloc(K));
  AVX_CK(s->st.alloc(1));
  AVX_CK(s->pimg.alloc((size_t)8 * std::max(AVX_RED_BLOCKS, avx::gap_img_blocks(s->W, s->H, s->T))));
  const int nk = s->op->kind == 1 ? avx::radial_interp_blocks(s->op->rg) : s->C * s->T;
  AVX_CK(s->pk.alloc((size_t)3 * std::max(nk, 1)));
  s->cap = (int)s->p.maxIt + 2;
  AVX_CK(s->hist.alloc((size_t)3 * (s->cap + 1)));
  if (!s->stream) {
    AVX_CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return AVX_OK;
}

static void solver_weights(avx_solver* s, Wts* w1, Wts* w2) {
  *w1 = make_wts(s->p.dx, s->p.dy, s->p.dt);
  *w2 = make_wts(s->p.dx2, s->p.dy2, s->p.dt2);
}

static PDArgs make_pdargs(avx_solver* s) {
  PDArgs a;
  memset(&a, 0, sizeof(a));
  a.W = s->W; a.H = s->H; a.T = s->T; a.N = s->N();
  const int P = method_P(s->method), D = method_D(s->method);
  for (int c = 0; c < P; ++c) {
    a.x[c] = s->primc(c);
    a.xb[c] = s->extc(c);
  }
  for (int c = 0; c < D; ++c) a.y[c] = s->dualc(c);
  solver_weights(s, &a.w1, &a.w2);
  const double alpha = s->p.alpha;
  const double m = std::min(alpha, 1.0 - alpha);
  if (s->method == AVX_METHOD_TV || s->method == AVX_METHOD_TVTEMP) {
    a.r1 = 1.0f;  // ProximalMap3(y, 1.0) (tv.cpp:157), ProximalMap1D(y, 1.0) (tv_temp.cpp:136)
  } else if (s->method == AVX_METHOD_ICTV) {
    // ictv.cpp:272-278
    a.r1 = (float)(1.0 / ((double)s->p.alpha1 * (alpha / m)));
    a.r3 = (float)(1.0 / ((double)s->p.alpha1 * ((1.0 - alpha) / m)));
  } else if (s->method == AVX_METHOD_TGV2) {
    a.r1 = (float)(1.0 / (double)s->p.alpha1);  // tgv2.cpp:258-259
    a.r2 = (float)(1.0 / (double)s->p.alpha0);
  } else {
    // ictgv2.cpp:366-381
    a.r1 = (float)(1.0 / ((double)s->p.alpha1 * (alpha / m)));
    a.r2 = (float)(1.0 / ((double)s->p.alpha0 * (alpha / m)));
    a.r3 = (float)(1.0 / ((double)s->p.alpha1 * ((1.0 - alpha) / m)));
    a.r4 = (float)(1.0 / ((double)s->p.alpha0 * ((1.0 - alpha) / m)));
  }
  a.alpha0 = s->p.alpha0;
  a.alpha1 = s->p.alpha1;
  a.alpha = s->p.alpha;
  a.ic_a = (float)(alpha / m);
  a.ic_b = (float)((1.0 - alpha) / m);
  a.khz = s->op->r_khz.p;
  a.st = s->st.p;
  a.primal_tile = s->primal_tile;
  a.dual_block = s->dual_block;
  return a;
}

// Autotuner of the field-streaming kernels' launch shapes and of the row
// kernel's FFT schedule.  The first run of a (device, method, W, H, T, C,
// sampled rows per frame) times every candidate on the solver's own fields
// (3 warm-up and 5 timed launches each, CUDA events on its stream) and keeps
// the fastest; later runs and solvers of that shape reuse it.  The trial
// launches overwrite the fields, so the caller prepares them again.
struct TuneKey {
  int dev, method, W, H, T, C, rows;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, method, W, H, T, C, rows) < std::tie(o.dev, o.method, o.W, o.H, o.T, o.C, o.rows);
  }
};
// one entry per shape: the map's lock covers lookups only, and each shape's
// own lock is held while that shape is tuned, so shapes tune in parallel and
// solvers of one shape on several threads all take the one choice
struct TuneEntry {
  std::mutex mu;
  bool done = false;
  int primal_tile = 0, dual_block = 0;
  int rows_kc = KSPACE_KC, rows_rt = 0;
};
static std::mutex g_tune_mu;
static std::map<TuneKey, std::unique_ptr<TuneEntry>> g_tune;

static avx_status time_launches(avx_solver* s, void (*launch)(int, const PDArgs&, cudaStream_t), const PDArgs& a,
                                float* ms) {
  cudaEvent_t e0, e1;
  AVX_CK(cudaEventCreate(&e0));
  AVX_CK(cudaEventCreate(&e1));
  for (int i = 0; i < 3; ++i) launch(s->method, a, s->stream);
  AVX_CK(cudaEventRecord(e0, s->stream));
  for (int i = 0; i < 5; ++i) launch(s->method, a, s->stream);
  AVX_CK(cudaEventRecord(e1, s->stream));
  AVX_CK(cudaEventSynchronize(e1));
  AVX_CK(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  AVX_CK(cudaGetLastError());
  return AVX_OK;
}

static KArgs make_kargs(avx_solver* s, const float2* b1, const float2* in, const float2* in2);

// Row-FFT schedules the tuner tries: rows per pass (8, 12, 16) with the
// compile-time radix plan of the length, and 16 rows per pass with the
// run-time plan when the length has a compile-time one.  Rows per pass
// change the schedule only (every sequence goes through the same passes); the
// two radix plans round differently.
static avx_status tune_rows(avx_solver* s, const float2* b1) {
  KArgs k = make_kargs(s, b1, s->extc(0), nullptr);
  const CartGeomDev& g = k.g;
  const bool has_fixed = fft_plan_id(g.W, g.nrad, g.rad) != fft_plan_id_runtime(g.nrad, g.rad);
  const int cand[4][2] = {{KSPACE_KC, 0}, {12, 0}, {8, 0}, {KSPACE_KC, 1}};
  const int ncand = has_fixed ? 4 : 3;
  avx::launch_ydft(k, s->stream);  // compact rows for the trial launches to transform
  cudaEvent_t e0, e1;
  AVX_CK(cudaEventCreate(&e0));
  AVX_CK(cudaEventCreate(&e1));
  float best = 0.f;
  for (int i = 0; i < ncand; ++i) {
    k.rows_kc = cand[i][0];
    k.rows_rt = cand[i][1];
    for (int w = 0; w < 3; ++w) avx::launch_rows(k, 0, s->stream);
    cudaEventRecord(e0, s->stream);
    for (int w = 0; w < 5; ++w) avx::launch_rows(k, 0, s->stream);
    cudaEventRecord(e1, s->stream);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    if (ce == cudaSuccess) ce = cudaGetLastError();
    if (ce != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(AVX_E_CUDA, std::string("row-schedule tuning: ") + cudaGetErrorString(ce));
    }
    if (i == 0 || ms < best) {
      best = ms;
      s->rows_kc = cand[i][0];
      s->rows_rt = cand[i][1];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return AVX_OK;
}

static int max_rows_per_frame(const avx_operator* op) {
  int m = 0;
  for (int t = 0; t + 1 < (int)op->row_off.size(); ++t) m = std::max(m, op->row_off[t + 1] - op->row_off[t]);
  return m;
}

static avx_status autotune(avx_solver* s, const float2* b1) {
  int dev = 0;
  AVX_CK(cudaGetDevice(&dev));
  const TuneKey key{dev, s->method, s->W, s->H, s->T, s->C, s->op->kind == 0 ? max_rows_per_frame(s->op) : -1};
  TuneEntry* ent;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::unique_ptr<TuneEntry>& slot = g_tune[key];
    if (!slot) slot.reset(new TuneEntry());
    ent = slot.get();
  }
  std::lock_guard<std::mutex> lk(ent->mu);
  if (ent->done) {
    s->primal_tile = ent->primal_tile;
    s->dual_block = ent->dual_block;
    s->rows_kc = ent->rows_kc;
    s->rows_rt = ent->rows_rt;
    s->tuned = true;
    return AVX_OK;
  }
  PDArgs a = make_pdargs(s);
  float best = 0.f;
  for (int i = 0; i < AVX_PRIMAL_TILES; ++i) {
    if (i >= 5 && !avx::dual_pairs(s->method, s->W)) break;
    a.primal_tile = i;
    float ms;
    avx_status r = time_launches(s, avx::launch_primal, a, &ms);
    if (r != AVX_OK) return r;
    if (i == 0 || ms < best) {
      best = ms;
      s->primal_tile = i;
    }
  }
  a.primal_tile = s->primal_tile;
  for (int i = 0; i < AVX_DUAL_BLOCKS; ++i) {
    if (i >= 3 && !avx::dual_pairs(s->method, s->W)) break;
    a.dual_block = i;
    float ms;
    avx_status r = time_launches(s, avx::launch_dual, a, &ms);
    if (r != AVX_OK) return r;
    if (i == 0 || ms < best) {
      best = ms;
      s->dual_block = i;
    }
  }
  if (s->op->kind == 0 && s->op->R) {
    avx_status r = tune_rows(s, b1);
    if (r != AVX_OK) return r;
  }
  s->tuned = true;
  ent->primal_tile = s->primal_tile;
  ent->dual_block = s->dual_block;
  ent->rows_kc = s->rows_kc;
  ent->rows_rt = s->rows_rt;
  ent->done = true;
  return AVX_OK;
}

static void set_tc(KArgs* k, const avx_operator* op) {
  const bool on = op->kind == 0 && op->dft_mode == AVX_DFT_SPLIT_BF16X3 && op->tc_np > 0;
  k->tc_ytab = on ? op->tc_ytab.p : nullptr;
  k->tc_np = on ? op->tc_np : 0;
  k->tc_ctab = on ? op->tc_ctab.p : nullptr;
  k->tc_kc = on ? op->tc_np : 0;
}

static KArgs make_kargs(avx_solver* s, const float2* b1, const float2* in, const float2* in2) {
  KArgs k;
  memset(&k, 0, sizeof(k));
  k.g = s->op->geom();
  k.b1 = b1;
  k.in = in;
  k.in2 = in2;
  k.z = s->z.p;
  k.d = s->d.p;
  k.qp = s->op->d_qp.p;
  k.lam = s->p.lambda;
  k.binary_mask = s->op->binary ? 1 : 0;
  k.st = s->st.p;
  k.partial = s->pk.p;
  set_tc(&k, s->op);
  k.b1t = s->b1t.p;
  k.rows_kc = s->rows_kc;
  k.rows_rt = s->rows_rt;
  return k;
}

// the tensor-core adjoint reads the coil maps in column-tile order
static avx_status prepare_b1t(avx_solver* s, const float2* b1) {
  if (s->op->kind != 0 || s->op->dft_mode != AVX_DFT_SPLIT_BF16X3 || s->op->tc_np == 0) return AVX_OK;
  AVX_CK(s->b1t.alloc(avx::b1t_count(s->W, s->H, s->C)));
  avx::launch_b1_tile_transpose(b1, s->b1t.p, s->W, s->H, s->C, s->stream);
  AVX_CK(cudaGetLastError());
  return AVX_OK;
}

static avx::GapConst make_gapconst(avx_solver* s) {
  avx::GapConst gc;
  const double alpha = s->p.alpha, m = std::min(alpha, 1.0 - alpha);
  gc.lam = s->p.lambda;
  gc.N = (double)s->N();
  gc.stop_gap = s->p.stopPDGap;
  gc.alpha0 = s->p.alpha0;
  gc.alpha1 = s->p.alpha1;
  gc.ic_a = alpha / m;
  gc.ic_b = (1.0 - alpha) / m;
  gc.stop_rel = s->stop_rel;
  return gc;
}

static bool step_due(unsigned k) { return k < 10 || k % 50 == 0; }
static bool stop_active(const avx_solver* s) { return s->p.stopPDGap > 0 || s->stop_rel > 0; }
static bool gap_due(const avx_solver* s, unsigned k) {
  return (s->verbose && (k < 10 || k % 50 == 0)) || (s->debug && s->debugstep > 0 && k % (unsigned)s->debugstep == 0) ||
         (stop_active(s) && k % 20 == 0);
}

static unsigned shape_launches(int kind, int shape) {
  if (kind == 1) return 10u + ((shape & 1) ? 7u : 0u) + ((shape & 2) ? 10u : 0u);
  return 5u + ((shape & 1) ? 5u : 0u) + ((shape & 2) ? 5u : 0u);
}

static RArgs solver_rargs(avx_solver* s, const float2* b1, const float2* in, const float2* in2) {
  RArgs r = make_rargs(s->op, b1, in, in2);
  r.z = s->z.p;
  r.d = s->d.p;
  r.lam = s->p.lambda;
  r.st = s->st.p;
  r.partial = s->pk.p;
  return r;
}

// radial operator pass: K u (mode 0 z prox, 1 norm, 2 gap sums) and, for modes
// 0 and 2, K^H z into the operator's K^H z image.  ev (optional) receives
// events after the forward FFT, the interpolation and the adjoint.
static void radial_pass(avx_solver* s, int mode, const float2* b1, const float2* in, const float2* in2,
                        cudaEvent_t* ev = nullptr) {
  RArgs r = solver_rargs(s, b1, in, in2);
  avx::launch_rad_forward_grid(r, s->stream);
  if (ev) cudaEventRecord(ev[0], s->stream);
  avx::launch_rad_interp(r, mode, s->stream);
  if (ev) cudaEventRecord(ev[1], s->stream);
  if (mode == 1) return;
  avx::launch_rad_spread(r, s->z.p, s->stream);
  avx::launch_rad_adjoint_image(r, s->op->r_khz.p, s->stream);
  if (ev) cudaEventRecord(ev[2], s->stream);
}

static void enqueue_shape_radial(avx_solver* s, int shape, const float2* b1, cudaEvent_t* ev) {
  const PDArgs a = make_pdargs(s);
  const KArgs kdummy = make_kargs(s, b1, s->extc(0), nullptr);
  if (ev) cudaEventRecord(ev[0], s->stream);
  avx::launch_dual(s->method, a, s->stream);
  if (ev) cudaEventRecord(ev[1], s->stream);
  radial_pass(s, 0, b1, s->extc(0), nullptr, ev ? ev + 2 : nullptr);
  avx::launch_primal(s->method, a, s->stream);
  if (ev) cudaEventRecord(ev[5], s->stream);
  const int nk = avx::radial_interp_blocks(s->op->rg);
  if (shape & 1) {
    avx::Ptr8 e;
    const int P = method_P(s->method);
    for (int c = 0; c < 8; ++c) e.p[c] = c < P ? s->escrc(c) : nullptr;
    avx::launch_step_img(s->method, a, e, P, s->pimg.p, s->stream);
    radial_pass(s, 1, b1, s->escrc(0), nullptr);
    avx::launch_step_finalize(a, s->pimg.p, s->pk.p, nk, s->p.sigmaTauRatio, s->stream);
  }
  if (shape & 2) {
    radial_pass(s, 2, b1, s->primc(0), nullptr);
    double* h = s->hist.p;
    const bool ic = method_ic(s->method);
    avx::launch_gap_tail(s->method, a, kdummy, s->pimg.p, s->pk.p, nk, make_gapconst(s), h,
                         ic ? h + (s->cap + 1) : nullptr, ic ? h + 2 * (s->cap + 1) : nullptr, s->cap, 0, s->stream);
  }
}

static void enqueue_shape(avx_solver* s, int shape, const float2* b1, cudaEvent_t* ev = nullptr) {
  if (s->op->kind == 1) {
    enqueue_shape_radial(s, shape, b1, ev);
    return;
  }
  const PDArgs a = make_pdargs(s);
  const KArgs ks = make_kargs(s, b1, s->extc(0), nullptr);
  avx::launch_iteration(s->method, a, ks, s->op->r_khz.p, s->stream, ev);
  if (shape & 1) {
    avx::Ptr8 e;
    const int P = method_P(s->method);
    for (int c = 0; c < 8; ++c) e.p[c] = c < P ? s->escrc(c) : nullptr;
    const KArgs ke = make_kargs(s, b1, s->escrc(0), nullptr);
    avx::launch_step(s->method, a, ke, e, P, s->pimg.p, s->pk.p, s->p.sigmaTauRatio, s->stream);
  }
  if (shape & 2) {
    const KArgs kx = make_kargs(s, b1, s->primc(0), nullptr);
    double* h = s->hist.p;
    const bool ic = method_ic(s->method);
    avx::launch_gap(s->method, a, kx, s->op->r_khz.p, s->pimg.p, s->pk.p, make_gapconst(s), h,
                    ic ? h + (s->cap + 1) : nullptr, ic ? h + 2 * (s->cap + 1) : nullptr, s->cap, 0, s->stream);
  }
}

static avx_status prepare_run(avx_solver* s, const float2* data, const float2* x0) {
  const int P = method_P(s->method), D = method_D(s->method);
  const size_t N = (size_t)s->N();
  AVX_CK(cudaMemsetAsync(s->dual.p, 0, D * N * sizeof(float2), s->stream));
  AVX_CK(cudaMemsetAsync(s->z.p, 0, s->z.n * sizeof(float2), s->stream));
  AVX_CK(cudaMemsetAsync(s->d.p, 0, s->d.n * sizeof(float2), s->stream));
  if (P > 1) {
    AVX_CK(cudaMemsetAsync(s->primc(1), 0, (P - 1) * N * sizeof(float2), s->stream));
    AVX_CK(cudaMemsetAsync(s->extc(1), 0, (P - 1) * N * sizeof(float2), s->stream));
  }
  if (x0) {
    AVX_CK(cudaMemcpyAsync(s->primc(0), x0, N * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
    AVX_CK(cudaMemcpyAsync(s->extc(0), x0, N * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
  }
  if (data && s->op->kind == 1) {
    AVX_CK(cudaMemcpyAsync(s->d.p, data, s->d.n * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
    s->d_off_energy = 0.0;
  } else if (data && s->op->R) {
    avx::launch_gather_rows(s->op->geom(), data, s->d.p, 0, s->stream);
    AVX_CK(cudaGetLastError());
    // energy of the data rows the operator never samples enters g1 as a constant
    double all = 0.0, kept = 0.0;
    avx_status r = sum_sq(data, (long long)s->C * N, s->stream, &all);
    if (r != AVX_OK) return r;
    r = sum_sq(s->d.p, (long long)s->d.n, s->stream, &kept);
    if (r != AVX_OK) return r;
    s->d_off_energy = std::max(0.0, all - kept);
  } else {
    s->d_off_energy = 0.0;
  }
  DevState h{};
  h.sigma = s->p.sigma;
  h.tau = s->p.tau;
  h.d_off = s->d_off_energy;
  AVX_CK(cudaMemcpyAsync(s->st.p, &h, sizeof(h), cudaMemcpyHostToDevice, s->stream));
  AVX_CK(cudaStreamSynchronize(s->stream));
  return AVX_OK;
}

// Set-up of a run (tv.cpp:103-135 and twins): time-space weights, zeroed
// duals and k-space, x and xbar from the initial image, the compact data,
// launch-shape tuning, the tile-ordered coil maps and, with the debug export
// of ICTGV2, the gap of the initial state.  Ends with the solver's stream
// ordered after the caller's.
// the reference overwrites dx, dy, dt (and dx2..dt2) from the weights (tv.cpp:103-104)
// (TVtemp uses its configured dt as it is, tv_temp.cpp:98-103)
static avx_status solver_run_weights(avx_solver* s) {
  double ds, dt;
  if (s->method != AVX_METHOD_TVTEMP) {
    if (!time_space_weights(s->p.timeSpaceWeight, &ds, &dt))
      return fail(AVX_E_ARG, "ComputeTimeSpaceWeights: invalid ratio");
    s->p.dx = (float)ds; s->p.dy = (float)ds; s->p.dt = (float)dt;
  }
  if (method_ic(s->method)) {
    if (!time_space_weights(s->p.timeSpaceWeight2, &ds, &dt)) return fail(AVX_E_ARG, "ComputeTimeSpaceWeights: invalid ratio");
    s->p.dx2 = (float)ds; s->p.dy2 = (float)ds; s->p.dt2 = (float)dt;
  }
  return AVX_OK;
}

static avx_status solver_begin(avx_solver* s, const float2* data, float2* x, const float2* b1) {
  avx_status r = solver_alloc(s);
  if (r != AVX_OK) return r;
  r = solver_run_weights(s);
  if (r != AVX_OK) return r;
  if (s->stream != s->user_stream) {
    // order the internal stream after the caller's stream
    cudaEvent_t evin;
    AVX_CK(cudaEventCreateWithFlags(&evin, cudaEventDisableTiming));
    AVX_CK(cudaEventRecord(evin, s->user_stream));
    AVX_CK(cudaStreamWaitEvent(s->stream, evin, 0));
    cudaEventDestroy(evin);
  }
  r = prepare_run(s, data, x);
  if (r != AVX_OK) return r;
  if (s->autotune && !s->tuned) {
    r = autotune(s, b1);
    if (r != AVX_OK) return r;
    r = prepare_run(s, data, x);  // the trial launches overwrote the fields
    if (r != AVX_OK) return r;
  }
  r = prepare_b1t(s, b1);
  if (r != AVX_OK) return r;
  if (s->method == AVX_METHOD_ICTGV2 && s->debug) {
    PDArgs a = make_pdargs(s);
    const KArgs kx = make_kargs(s, b1, s->primc(0), nullptr);
    double* h = s->hist.p;
    if (s->op->kind == 1) {
      a.khz = s->op->r_khz.p;
      radial_pass(s, 2, b1, s->primc(0), nullptr);
      avx::launch_gap_tail(s->method, a, kx, s->pimg.p, s->pk.p, avx::radial_interp_blocks(s->op->rg),
                           make_gapconst(s), h, h + (s->cap + 1), h + 2 * (s->cap + 1), s->cap, 1, s->stream);
    } else {
      avx::launch_gap(s->method, a, kx, s->op->r_khz.p, s->pimg.p, s->pk.p, make_gapconst(s), h, h + (s->cap + 1),
                      h + 2 * (s->cap + 1), s->cap, 1, s->stream);
    }
    AVX_CK(cudaGetLastError());
  }
  // graphs depend on every pointer and scalar baked into the launches; the
  // step sizes and the data-energy constant live in DevState and are not baked
  avx_pd_params pk = s->p;
  pk.sigma = pk.tau = 0.f;
  const size_t key = (size_t)b1 ^ ((size_t)s->prim.p << 1) ^ ((size_t)s->op << 2) ^
                     ((size_t)s->op->dft_mode << 7) ^ ((size_t)(s->primal_tile * 8 + s->dual_block) << 9) ^
                     ((size_t)(s->rows_kc * 2 + s->rows_rt) << 16) ^
                     std::hash<std::string>()(std::string((const char*)&pk, sizeof(pk)));
  if (key != s->graph_key) {
    s->drop_graphs();
    s->graph_key = key;
  }
  return AVX_OK;
}

// The CUDA graph of iteration shape `shape` (bit 0: step rule, bit 1: gap),
// captured on the solver's stream at first use.
static avx_status solver_graph(avx_solver* s, int shape, const float2* b1) {
  if (s->gexec[shape]) return AVX_OK;
  cudaGraph_t g;
  AVX_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  enqueue_shape(s, shape, b1);
  AVX_CK(cudaStreamEndCapture(s->stream, &g));
  const cudaError_t e = cudaGraphInstantiate(&s->gexec[shape], g, 0);
  cudaGraphDestroy(g);
  AVX_CK(e);
  return AVX_OK;
}

static int iter_shape(const avx_solver* s, unsigned k) { return (step_due(k) ? 1 : 0) | (gap_due(s, k) ? 2 : 0); }

// Enqueues iterations [k0, k1) from the graphs of their shapes (no host
// synchronisation); *launches receives the kernels they hold.
static avx_status solver_enqueue(avx_solver* s, const float2* b1, unsigned k0, unsigned k1, unsigned* launches) {
  for (unsigned k = k0; k < k1; ++k) {
    const int shape = iter_shape(s, k);
    avx_status r = solver_graph(s, shape, b1);
    if (r != AVX_OK) return r;
    AVX_CK(cudaGraphLaunch(s->gexec[shape], s->stream));
    if (launches) *launches += shape_launches(s->op->kind, shape);
  }
  return AVX_OK;
}

// Statistics of a finished run from the device state it left in s->last.
static avx_status solver_finish_stats(avx_solver* s, float ms, unsigned launches) {
  s->p.sigma = (float)s->last.sigma;
  s->p.tau = (float)s->last.tau;
  s->stats.iterations = (unsigned)s->last.iters;
  s->stats.sigma = (float)s->last.sigma;
  s->stats.tau = (float)s->last.tau;
  s->stats.gap_count = (unsigned)s->last.ngap;
  s->stats.last_gap = s->last.gap;
  s->stats.stopped_by_gap = s->last.stop;
  s->stats.elapsed_ms = ms;
  s->stats.kernel_launches = launches;
  if (s->last.err) return fail(AVX_E_NUMERIC, "device-side check failed");
  return AVX_OK;
}

static avx_status solver_run(avx_solver* s, const float2* data, float2* x, const float2* b1) {
  avx_status r = solver_begin(s, data, x, b1);
  if (r != AVX_OK) return r;
  cudaEvent_t ev0, ev1;
  AVX_CK(cudaEventCreate(&ev0));
  AVX_CK(cudaEventCreate(&ev1));
  constexpr size_t NEV = AVX_NSTAGE + 1;  // events per timed iteration
  if (s->timing && s->events.size() < NEV * s->p.maxIt) {
    const size_t need = NEV * s->p.maxIt;
    while (s->events.size() < need) {
      cudaEvent_t e;
      AVX_CK(cudaEventCreate(&e));
      s->events.push_back(e);
    }
  }
  unsigned launches = 0;
  AVX_CK(cudaEventRecord(ev0, s->stream));
  unsigned k = 0;
  for (; k < s->p.maxIt; ++k) {
    const int shape = iter_shape(s, k);
    if (s->timing) {
      launches += shape_launches(s->op->kind, shape);
      enqueue_shape(s, shape, b1, &s->events[NEV * k]);
      AVX_CK(cudaGetLastError());
      continue;
    }
    r = solver_enqueue(s, b1, k, k + 1, &launches);
    if (r != AVX_OK) return r;
    if (stop_active(s) && (shape & 2) && (k % 100 == 0)) {
      int stop = 0;
      AVX_CK(cudaMemcpyAsync(&stop, &s->st.p->stop, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
      AVX_CK(cudaStreamSynchronize(s->stream));
      if (stop) {
        ++k;
        break;
      }
    }
  }
  AVX_CK(cudaEventRecord(ev1, s->stream));
  AVX_CK(cudaMemcpyAsync(x, s->primc(0), (size_t)s->N() * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
  AVX_CK(cudaMemcpyAsync(&s->last, s->st.p, sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
  AVX_CK(cudaStreamSynchronize(s->stream));
  AVX_CK(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev0, ev1);
  s->kcount = 0;
  for (int j = 0; j < AVX_NSTAGE; ++j) s->kmean[j] = 0.f;
  if (s->timing) {
    double acc[AVX_NSTAGE] = {};
    for (unsigned i = 0; i < k; ++i)
      for (int j = 0; j < AVX_NSTAGE; ++j) {
        float t = 0.f;
        cudaEventElapsedTime(&t, s->events[NEV * i + j], s->events[NEV * i + j + 1]);
        acc[j] += t;
      }
    s->kcount = k;
    for (int j = 0; j < AVX_NSTAGE; ++j) s->kmean[j] = k ? (float)(acc[j] / k) : 0.f;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  return solver_finish_stats(s, ms, launches);
}

// ===========================================================================
// Coil-sensitivity estimation (CUDA/src/coil_construction.cpp:55-556)
// ===========================================================================

namespace {

struct Fft2dTables {
  DevBuf<float2> twx, twy;
  Fft2dPlan plan{};
};

avx_status make_fft2d(int W, int H, Fft2dTables& t) {
  const std::vector<int> rx = fft_radices(W), ry = fft_radices(H);
  if (rx.empty() || ry.empty()) return fail(AVX_E_UNSUPPORTED, "image size has no FFT plan (prime factor > 13)");
  if (avx::fft2d_smem_bytes(std::max(W, H)) > AVX_DYN_SMEM_MAX) return fail(AVX_E_UNSUPPORTED, "image too large for the FFT tile");
  std::vector<float2> hx(W), hy(H);
  for (int j = 0; j < W; ++j) hx[j] = make_float2((float)std::cos(2.0 * M_PI * j / W), (float)std::sin(2.0 * M_PI * j / W));
  for (int j = 0; j < H; ++j) hy[j] = make_float2((float)std::cos(2.0 * M_PI * j / H), (float)std::sin(2.0 * M_PI * j / H));
  AVX_CK(t.twx.alloc(W));
  AVX_CK(t.twy.alloc(H));
  AVX_CK(cudaMemcpy(t.twx.p, hx.data(), W * sizeof(float2), cudaMemcpyHostToDevice));
  AVX_CK(cudaMemcpy(t.twy.p, hy.data(), H * sizeof(float2), cudaMemcpyHostToDevice));
  t.plan.W = W;
  t.plan.H = H;
  t.plan.twx = t.twx.p;
  t.plan.twy = t.twy.p;
  t.plan.nradx = (int)rx.size();
  t.plan.nrady = (int)ry.size();
  for (int i = 0; i < 12; ++i) {
    t.plan.radx[i] = i < t.plan.nradx ? rx[i] : 0;
    t.plan.rady[i] = i < t.plan.nrady ? ry[i] : 0;
  }
  return AVX_OK;
}

avx_status coil_time_averaged(int W, int H, int C, int T, const float2* kdata, const float* mask, float2* u,
                              float2* crec, int apply_phase, cudaStream_t s) {
  Fft2dTables ft;
  avx_status r = make_fft2d(W, H, ft);
  if (r != AVX_OK) return r;
  const int HW = W * H;
  avx::launch_ta_sum(kdata, mask, crec, HW, C, T, s);
  avx::launch_fft2d(ft.plan, crec, C, -1, s);  // unitary k-space -> image (e^{-2 pi i}), scaled below
  avx::launch_ta_combine(crec, u, HW, C, (float)(1.0 / std::sqrt((double)HW)), apply_phase, s);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(s));
  return AVX_OK;
}

avx_status coil_b1_from_u_h1(int W, int H, int C, const avx_coil_params& p, const float2* u, const float2* crec,
                             float2* absb1, cudaStream_t s) {
  const int N = W * H;
  DevBuf<double2> work;
  DevBuf<double> muu;
  AVX_CK(work.alloc((size_t)C * 4 * N));
  AVX_CK(muu.alloc((size_t)C * N));
  // the exact solution of the H1 system: FP64 CG to a relative residual of 1e-12
  avx::launch_h1_cg(u, crec, p.uH1mu, W, H, C, 50000, 1e-12, work.p, muu.p, absb1, nullptr, s);
  avx::launch_h1_normalize(absb1, N, C, s);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(s));
  return AVX_OK;
}

// Buffers of one coil-construction loop (UTGV2Recon or B1Recon) and the CUDA
// graph of its iterations.  Held across the greedy steps of
// PerformCoilConstruction, which call the same loop with the same sizes
// eleven times: the buffers are allocated once, and the iterations, whose
// kernels read every input through the fixed buffers, are captured once and
// replayed.  A loop used once (the C-ABI entry points, the final B1Recon)
// launches its iterations directly.
struct CoilLoop {
  bool use_graph = false;
  int N = 0, coils = 0;
  unsigned iters = 0;
  DevBuf<float2> buf, xw, Ib;
  DevBuf<int> dind;
  DevBuf<unsigned> umax;
  cudaGraphExec_t g = nullptr;
  ~CoilLoop() {
    if (g) cudaGraphExecDestroy(g);
  }
};

// Runs `iters` iterations of the loop through `launch` on stream s: from the
// loop's graph when it keeps one (captured on the first call), else directly.
template <class F>
static avx_status coil_iterate(CoilLoop& l, unsigned iters, cudaStream_t s, F launch) {
  if (!l.use_graph || s == 0) {
    for (unsigned it = 0; it < iters; ++it) launch();
    AVX_CK(cudaGetLastError());
    return AVX_OK;
  }
  if (l.g && l.iters != iters) {
    cudaGraphExecDestroy(l.g);
    l.g = nullptr;
  }
  if (!l.g) {
    cudaGraph_t gr;
    AVX_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (unsigned it = 0; it < iters; ++it) launch();
    AVX_CK(cudaStreamEndCapture(s, &gr));
    const cudaError_t e = cudaGraphInstantiate(&l.g, gr, 0);
    cudaGraphDestroy(gr);
    AVX_CK(e);
    l.iters = iters;
  }
  AVX_CK(cudaGraphLaunch(l.g, s));
  return AVX_OK;
}

avx_status coil_utgv2(int W, int H, const avx_coil_params& p, const float2* b10, const float2* crec0,
                      const std::vector<int>& inds, float2* x1, cudaStream_t s, CoilLoop* loop = nullptr) {
  const int N = W * H;
  CoilLoop local;
  CoilLoop& l = loop ? *loop : local;
  // 11 N: ext1, x2 (2), ext2 (2), y1 (2), y2 (3), Lw; 8 N more: the second
  // set of the double-buffered ext1, ext2, y1, y2
  if (l.N != N) {
    AVX_CK(l.buf.alloc((size_t)19 * N));
    AVX_CK(l.xw.alloc(N));
    AVX_CK(l.Ib.alloc(N));
    l.N = N;
  }
  AVX_CK(l.dind.alloc(std::max<size_t>(inds.size(), 1)));
  AVX_CK(cudaMemcpyAsync(l.dind.p, inds.data(), inds.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  AVX_CK(cudaMemsetAsync(l.buf.p, 0, (size_t)19 * N * sizeof(float2), s));
  CoilPD a;
  memset(&a, 0, sizeof(a));
  a.W = W;
  a.H = H;
  a.sigma = p.uSigma;
  a.tau = p.uTau;
  a.s1 = (float)(1.0 / ((double)p.uAlpha1 * p.uReg));
  a.s2 = (float)(1.0 / ((double)p.uAlpha0 * p.uReg));
  a.x1 = l.xw.p;
  a.x1n = l.xw.p;
  a.ext1 = l.buf.p;
  a.ext1n = l.buf.p;
  for (int k = 0; k < 2; ++k) {
    a.x2[k] = l.buf.p + (size_t)(1 + k) * N;
    a.ext2[k] = l.buf.p + (size_t)(3 + k) * N;
    a.ext2n[k] = a.ext2[k];
    a.y1[k] = l.buf.p + (size_t)(5 + k) * N;
  }
  for (int k = 0; k < 3; ++k) a.y2[k] = l.buf.p + (size_t)(7 + k) * N;
  float2* Lw = l.buf.p + (size_t)10 * N;
  a.Lw = Lw;
  a.Ib = l.Ib.p;
  AVX_CK(cudaMemcpyAsync(l.xw.p, x1, N * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  AVX_CK(cudaMemcpyAsync(a.ext1, x1, N * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  avx::launch_utgv_prep(b10, crec0, l.dind.p, (int)inds.size(), p.uTau, N, Lw, l.Ib.p, s);
  // one kernel per iteration; ext1, ext2, y1, y2 alternate between the two
  // sets (the second at 11 N .. 19 N), x1 and x2 stay in place
  UtgvBuffers ub[2];
  float2* second = l.buf.p + (size_t)11 * N;
  for (int q = 0; q < 2; ++q) {
    const bool odd = q == 1;
    auto pick = [&](float2* first, int j) { return odd ? second + (size_t)j * N : first; };
    auto other = [&](float2* first, int j) { return odd ? first : second + (size_t)j * N; };
    ub[q].ext1_in = pick(a.ext1, 0);
    ub[q].ext1_out = other(a.ext1, 0);
    for (int k = 0; k < 2; ++k) {
      ub[q].ext2_in[k] = pick(a.ext2[k], 1 + k);
      ub[q].ext2_out[k] = other(a.ext2[k], 1 + k);
      ub[q].y1_in[k] = pick(a.y1[k], 3 + k);
      ub[q].y1_out[k] = other(a.y1[k], 3 + k);
    }
    for (int k = 0; k < 3; ++k) {
      ub[q].y2_in[k] = pick(a.y2[k], 5 + k);
      ub[q].y2_out[k] = other(a.y2[k], 5 + k);
    }
  }
  unsigned it = 0;
  avx_status r = coil_iterate(l, p.uNrIt, s, [&] { avx::launch_utgv_fused(a, ub[it++ & 1u], s); });
  if (r != AVX_OK) return r;
  AVX_CK(cudaMemcpyAsync(x1, l.xw.p, N * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(s));
  return AVX_OK;
}

avx_status coil_b1_recon(int W, int H, int coils, unsigned max_it, float mu, const avx_coil_params& p,
                         const float2* u0, const float2* crec, float2* out, cudaStream_t s,
                         CoilLoop* loop = nullptr) {
  const int N = W * H;
  const size_t CN = (size_t)coils * N;
  CoilLoop local;
  CoilLoop& l = loop ? *loop : local;
  if (l.N != N || l.coils != coils) {
    AVX_CK(l.buf.alloc(9 * CN));
    AVX_CK(l.umax.alloc(1));
    l.N = N;
    l.coils = coils;
  }
  AVX_CK(cudaMemsetAsync(l.buf.p, 0, 9 * CN * sizeof(float2), s));
  AVX_CK(cudaMemsetAsync(l.umax.p, 0, sizeof(unsigned), s));
  CoilPD a;
  memset(&a, 0, sizeof(a));
  a.W = W;
  a.H = H;
  a.sigma = p.b1Sigma;
  a.tau = p.b1Tau;
  a.mu = mu;
  a.x1 = a.x1n = l.buf.p;
  a.ext1 = a.ext1n = l.buf.p + CN;
  a.y1[0] = l.buf.p + 2 * CN;
  a.y1[1] = l.buf.p + 3 * CN;
  float2* Lw = l.buf.p + 4 * CN;
  float2* Iu = l.buf.p + 5 * CN;
  a.Lw = Lw;
  a.Ib = Iu;
  avx::launch_absmax(u0, N, l.umax.p, s);
  avx::launch_b1r_prep(u0, l.umax.p, crec, coils, N, p.b1Tau, Lw, Iu, s);
  // one kernel per iteration; the extragradient and the duals alternate
  // between two buffers (the second set at 6 CN .. 9 CN), x stays in place
  float2* ext2 = l.buf.p + 6 * CN;
  float2* y2[2] = {l.buf.p + 7 * CN, l.buf.p + 8 * CN};
  unsigned it = 0;
  avx_status r = coil_iterate(l, max_it, s, [&] {
    const bool odd = (it++ & 1u) != 0;
    B1Buffers b;
    b.ext_in = odd ? ext2 : a.ext1;
    b.ext_out = odd ? a.ext1 : ext2;
    b.y0_in = odd ? y2[0] : a.y1[0];
    b.y1_in = odd ? y2[1] : a.y1[1];
    b.y0_out = odd ? a.y1[0] : y2[0];
    b.y1_out = odd ? a.y1[1] : y2[1];
    avx::launch_b1r_fused(a, coils, b, s);
  });
  if (r != AVX_OK) return r;
  avx::launch_b1r_normalize(a.x1, out, N, coils, s);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(s));
  return AVX_OK;
}

// FP64 sums for the greedy coil order (coil_construction.cpp:55-73, 471-520):
// out[j] = sum_i |a_i| |crec_{ks[j]},i| (sum_i |crec_{ks[j]},i| when a is null),
// one reduction per coil into its own partials, one copy back for all of them.
avx_status abs_sums(const float2* a, const float2* crec, const std::vector<int>& ks, int N, DevBuf<double>& part,
                    cudaStream_t s, std::vector<double>& out) {
  constexpr int NB = 64;
  AVX_CK(part.alloc(std::max<size_t>(ks.size(), 1) * NB));
  for (size_t j = 0; j < ks.size(); ++j) {
    const float2* c = crec + (size_t)ks[j] * N;
    avx::launch_abs_sum(a ? a : c, a ? c : nullptr, N, part.p + j * NB, NB, s);
  }
  AVX_CK(cudaGetLastError());
  std::vector<double> h(ks.size() * NB);
  AVX_CK(cudaMemcpyAsync(h.data(), part.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  AVX_CK(cudaStreamSynchronize(s));
  out.assign(ks.size(), 0.0);
  for (size_t j = 0; j < ks.size(); ++j) {
    double acc = 0.0;
    for (int i = 0; i < NB; ++i) acc += h[j * NB + i];
    out[j] = acc;
  }
  return AVX_OK;
}

__global__ void abs_inplace_kernel(float2* v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = make_float2(sqrtf(cabs2(v[i])), 0.f);
}

// NoncartesianCoilConstruction::TimeAveragedReconstruction
// (noncartesian_coil_construction.cpp:21-127): every frame's samples in one
// gridding adjoint (kernel width 3, sector width 8, osf 2), per coil.
avx_status coil_time_averaged_radial(int W, int H, int C, int T, int S, const float* traj, const float* dens,
                                     const float2* kdata, float2* u, float2* crec, int apply_phase, cudaStream_t s) {
  const size_t TS = (size_t)T * S;
  // every frame's kx, then every frame's ky: [T][2][S] -> [1][2][T S] (the
  // densities [T][S] already read as one frame)
  DevBuf<float> t1;
  AVX_CK(t1.alloc(2 * TS));
  for (int a = 0; a < 2; ++a)
    AVX_CK(cudaMemcpy2DAsync(t1.p + (size_t)a * TS, S * sizeof(float), traj + (size_t)a * S, 2 * S * sizeof(float),
                             S * sizeof(float), T, cudaMemcpyDeviceToDevice, s));
  AVX_CK(cudaStreamSynchronize(s));
  // one frame holding every frame's samples; the spreading grid holds every
  // coil (one pass over the samples for all coils), the adjoint grid
  // transform and crop run per coil (no coil combination)
  avx_operator op;
  op.kind = 1;
  op.W = W; op.H = H; op.C = C; op.T = 1;
  op.S = (int)TS;
  op.spf = 1;
  avx_status r = build_radial(&op, t1.p, dens, 3.f, 8.f, 2.f);
  if (r != AVX_OK) return r;
  DevBuf<float2> ones, samp;
  AVX_CK(ones.alloc((size_t)W * H));
  AVX_CK(samp.alloc((size_t)C * TS));
  std::vector<float2> h1((size_t)W * H, make_float2(1.f, 0.f));
  AVX_CK(cudaMemcpy(ones.p, h1.data(), h1.size() * sizeof(float2), cudaMemcpyHostToDevice));
  // coil c's samples of all frames, frame after frame: [frame][coil][sample] -> [coil][frame][sample]
  for (int c = 0; c < C; ++c)
    AVX_CK(cudaMemcpy2DAsync(samp.p + (size_t)c * TS, S * sizeof(float2), kdata + (size_t)c * S,
                             (size_t)C * S * sizeof(float2), S * sizeof(float2), T, cudaMemcpyDeviceToDevice, s));
  RArgs ra = make_rargs(&op, ones.p, nullptr, nullptr);
  avx::launch_rad_spread(ra, samp.p, s);
  const size_t G2 = (size_t)op.rg.Gx * op.rg.Gy;
  for (int c = 0; c < C; ++c) {
    RArgs rc = ra;
    rc.g.C = 1;
    rc.grid = op.r_grid.p + (size_t)c * G2;
    avx::launch_rad_adjoint_image(rc, crec + (size_t)c * W * H, s);
  }
  avx::launch_ta_combine(crec, u, W * H, C, 1.f, apply_phase, s);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(s));
  return AVX_OK;
}

avx_status coil_estimate_on(int W, int H, int C, const avx_coil_params& p, float2* u0p, float2* crecp, float2* u,
                            float2* b1, cudaStream_t s) {
  const int N = W * H;
  DevBuf<float2> absb1, w, uin, cin, x1;
  DevBuf<double> part;
  AVX_CK(absb1.alloc((size_t)C * N));
  AVX_CK(w.alloc(N));
  AVX_CK(uin.alloc(N));
  AVX_CK(cin.alloc(N));
  AVX_CK(x1.alloc(N));
  CoilLoop lu, lb;  // the greedy steps' UTGV2 and single-coil B1 loops
  lu.use_graph = lb.use_graph = true;
  float2* u0 = u0p;
  const float2* crec = crecp;
  avx_status r;
  abs_inplace_kernel<<<(N + 255) / 256, 256, 0, s>>>(u0, N);
  r = coil_b1_from_u_h1(W, H, C, p, u0, crec, absb1.p, s);
  if (r != AVX_OK) return r;
  // FindMaximumSum (coil_construction.cpp:55-73)
  std::vector<int> inds, all(C);
  std::vector<double> sums;
  for (int c = 0; c < C; ++c) all[c] = c;
  r = abs_sums(nullptr, crec, all, N, part, s, sums);
  if (r != AVX_OK) return r;
  {
    double best = -1.0;
    int bi = 0;
    for (int c = 0; c < C; ++c)
      if (sums[c] > best) {
        best = sums[c];
        bi = c;
      }
    inds.push_back(bi);
  }
  AVX_CK(cudaMemsetAsync(b1, 0, (size_t)C * N * sizeof(float2), s));
  AVX_CK(cudaMemsetAsync(u, 0, (size_t)C * N * sizeof(float2), s));
  AVX_CK(cudaMemcpyAsync(b1 + (size_t)inds[0] * N, absb1.p + (size_t)inds[0] * N, N * sizeof(float2),
                         cudaMemcpyDeviceToDevice, s));
  r = coil_utgv2(W, H, p, b1, crec, inds, u, s, &lu);  // u[0] starts at zero
  if (r != AVX_OK) return r;
  AVX_CK(cudaMemsetAsync(w.p, 0, N * sizeof(float2), s));
  float2* uMax = u;
  for (int cnt = 1; cnt < C; ++cnt) {
    const int prev = inds[cnt - 1];
    avx::launch_weight_update(w.p, absb1.p + (size_t)prev * N, N, s);
    std::vector<int> cand;
    for (int k = 0; k < C; ++k)
      if (std::find(inds.begin(), inds.end(), k) == inds.end()) cand.push_back(k);
    r = abs_sums(crec + (size_t)prev * N, crec, cand, N, part, s, sums);
    if (r != AVX_OK) return r;
    double best = -1.0;
    int mi = -1;
    for (size_t j = 0; j < cand.size(); ++j)
      if (sums[j] > best) {
        best = sums[j];
        mi = cand[j];
      }
    inds.push_back(mi);
    avx::launch_greedy_inputs(absb1.p + (size_t)mi * N, u + (size_t)(cnt - 1) * N, w.p, crec + (size_t)mi * N,
                              uin.p, cin.p, N, s);
    r = coil_b1_recon(W, H, 1, p.b1NrIt, p.b1Reg, p, uin.p, cin.p, x1.p, s, &lb);
    if (r != AVX_OK) return r;
    avx::launch_phase_apply(absb1.p + (size_t)mi * N, x1.p, b1 + (size_t)mi * N, N, s);
    uMax = u + (size_t)cnt * N;
    AVX_CK(cudaMemcpyAsync(uMax, u + (size_t)(cnt - 1) * N, N * sizeof(float2), cudaMemcpyDeviceToDevice, s));
    r = coil_utgv2(W, H, p, b1, crec, inds, uMax, s, &lu);
    if (r != AVX_OK) return r;
  }
  // final correction of all coils (coil_construction.cpp:555); run once, so
  // its iterations launch directly (capturing them would cost more than it saves)
  r = coil_b1_recon(W, H, C, p.b1FinalNrIt, p.b1FinalReg, p, uMax, crec, b1, s);
  if (r != AVX_OK) return r;
  AVX_CK(cudaGetLastError());
  return AVX_OK;
}

// PerformCoilConstruction after the time-averaged reconstruction
// (coil_construction.cpp:447-556): u0 (W*H, replaced by |u0|) and crec
// (C*W*H).  Runs on a stream of its own (the loops' graphs need one), ordered
// after s, and returns when it is done.
avx_status coil_construction(int W, int H, int C, int T, const avx_coil_params& p, const float2* kdata,
                             const float* mask, float2* u, float2* b1, cudaStream_t s) {
  DevBuf<float2> u0, crec;
  AVX_CK(u0.alloc((size_t)W * H));
  AVX_CK(crec.alloc((size_t)C * W * H));
  avx_status r = coil_time_averaged(W, H, C, T, kdata, mask, u0.p, crec.p, 1, s);
  if (r != AVX_OK) return r;
  r = coil_estimate_on(W, H, C, p, u0.p, crec.p, u, b1, s);
  if (r != AVX_OK) return r;
  AVX_CK(cudaStreamSynchronize(s));
  return AVX_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char* avx_version(void) { return "avionic-b200 0.1 (sm_100a)"; }
const char* avx_last_error(void) { return g_err.c_str(); }

avx_status avx_cartesian_operator_create(unsigned width, unsigned height, unsigned coils, unsigned frames,
                                         const float* d_mask, int centered, avx_operator** out) {
  if (!out) return fail(AVX_E_ARG, "null output handle");
  avx_status r = check_dims(width, height, coils, frames);
  if (r != AVX_OK) return r;
  r = configure_once();
  if (r != AVX_OK) return r;
  std::vector<float> hm;
  if (d_mask) {
    hm.resize((size_t)width * height * frames);
    AVX_CK(cudaMemcpy(hm.data(), d_mask, hm.size() * sizeof(float), cudaMemcpyDeviceToHost));
  }
  avx_operator* op = new avx_operator();
  op->W = (int)width; op->H = (int)height; op->C = (int)coils; op->T = (int)frames;
  op->centered = centered ? 1 : 0;
  r = build_operator(op, d_mask ? hm.data() : nullptr);
  if (r != AVX_OK) {
    delete op;
    return r;
  }
  *out = op;
  return AVX_OK;
}

avx_status avx_operator_set_dft_mode(avx_operator* op, int mode) {
  if (!op) return fail(AVX_E_ARG, "null operator");
  if (mode != AVX_DFT_FP32 && mode != AVX_DFT_SPLIT_BF16X3) return fail(AVX_E_ARG, "unknown DFT mode");
  if (mode == AVX_DFT_SPLIT_BF16X3 && (op->kind != 0 || op->tc_np == 0))
    return fail(AVX_E_UNSUPPORTED, "split-BF16x3 transform needs a Cartesian operator with <= 48 rows per frame");
  op->dft_mode = mode;
  return AVX_OK;
}

avx_status avx_operator_get_dft_mode(const avx_operator* op, int* mode) {
  if (!op || !mode) return fail(AVX_E_ARG, "null argument");
  *mode = op->kind == 0 ? op->dft_mode : AVX_DFT_FP32;
  return AVX_OK;
}

avx_status avx_radial_operator_create(unsigned width, unsigned height, unsigned coils, unsigned frames,
                                      unsigned nSpokes, unsigned nFE, unsigned spokesPerFrame, const float* d_traj,
                                      const float* d_dens, float kernelWidth, float sectorWidth, float osf,
                                      avx_operator** out) {
  if (!out || !d_traj || !d_dens) return fail(AVX_E_ARG, "null argument");
  if (!width || !height || !coils || !frames || !nFE || !spokesPerFrame)
    return fail(AVX_E_ARG, "dimensions must be positive");
  if (nSpokes != spokesPerFrame * frames) return fail(AVX_E_ARG, "nSpokes must equal spokesPerFrame * frames");
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  const size_t S = (size_t)nFE * spokesPerFrame;
  avx_operator* op = new avx_operator();
  op->kind = 1;
  op->W = (int)width; op->H = (int)height; op->C = (int)coils; op->T = (int)frames;
  op->S = (int)S;
  op->spf = (int)spokesPerFrame;
  r = build_radial(op, d_traj, d_dens, kernelWidth, sectorWidth, osf);
  if (r != AVX_OK) {
    delete op;
    return r;
  }
  *out = op;
  return AVX_OK;
}

avx_status avx_radial_sector_map(const avx_operator* op, int* h_order, int* h_start, int* grid_xy) {
  if (!op || op->kind != 1) return fail(AVX_E_ARG, "not a radial operator");
  const RadialGeomDev& g = op->rg;
  if (grid_xy) {
    grid_xy[0] = g.Gx;
    grid_xy[1] = g.Gy;
  }
  if (h_order)
    AVX_CK(cudaMemcpy(h_order, op->r_order.p, (size_t)g.T * g.S * sizeof(int), cudaMemcpyDeviceToHost));
  if (h_start)
    AVX_CK(cudaMemcpy(h_start, op->r_secstart.p, (size_t)g.T * (g.nsx * g.nsy + 1) * sizeof(int),
                      cudaMemcpyDeviceToHost));
  return AVX_OK;
}

avx_status avx_operator_backward(avx_operator* op, const avx_cf32* d_x, avx_cf32* d_k, const avx_cf32* d_b1) {
  if (!op || !d_x || !d_k || !d_b1) return fail(AVX_E_ARG, "null argument");
  if (op->kind == 1) {
    RArgs ra = make_rargs(op, reinterpret_cast<const float2*>(d_b1), reinterpret_cast<const float2*>(d_x), nullptr);
    ra.out = reinterpret_cast<float2*>(d_k);
    avx::launch_rad_forward_grid(ra, 0);
    avx::launch_rad_interp(ra, 3, 0);
    AVX_CK(cudaGetLastError());
    AVX_CK(cudaDeviceSynchronize());
    return AVX_OK;
  }
  const size_t K = (size_t)op->W * op->H * op->C * op->T;
  AVX_CK(cudaMemset(d_k, 0, K * sizeof(float2)));
  KArgs k;
  memset(&k, 0, sizeof(k));
  k.g = op->geom();
  k.b1 = reinterpret_cast<const float2*>(d_b1);
  k.in = reinterpret_cast<const float2*>(d_x);
  k.dense_out = reinterpret_cast<float2*>(d_k);
  k.qp = op->d_qp.p;  // y-transformed rows between the two kernels
  set_tc(&k, op);
  if (op->R) avx::launch_kspace(k, 3, 0);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}

avx_status avx_operator_forward(avx_operator* op, avx_cf32* d_k, avx_cf32* d_x, const avx_cf32* d_b1) {
  if (!op || !d_x || !d_k || !d_b1) return fail(AVX_E_ARG, "null argument");
  if (op->kind == 1) {
    RArgs ra = make_rargs(op, reinterpret_cast<const float2*>(d_b1), nullptr, nullptr);
    avx::launch_rad_spread(ra, reinterpret_cast<const float2*>(d_k), 0);
    avx::launch_rad_adjoint_image(ra, reinterpret_cast<float2*>(d_x), 0);
    AVX_CK(cudaGetLastError());
    AVX_CK(cudaDeviceSynchronize());
    return AVX_OK;
  }
  KArgs k;
  memset(&k, 0, sizeof(k));
  k.g = op->geom();
  k.b1 = reinterpret_cast<const float2*>(d_b1);
  k.qp = op->d_qp.p;
  set_tc(&k, op);
  if (k.tc_ctab) {
    AVX_CK(op->tc_b1t.alloc(avx::b1t_count(op->W, op->H, op->C)));
    avx::launch_b1_tile_transpose(k.b1, op->tc_b1t.p, op->W, op->H, op->C, 0);
    k.b1t = op->tc_b1t.p;
  }
  avx::launch_dense_rowidft(k.g, reinterpret_cast<float2*>(d_k), op->d_qp.p, op->has_mask ? op->d_mask.p : nullptr, 0);
  avx::launch_adjoint(k, reinterpret_cast<float2*>(d_x), 0);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}

avx_status avx_operator_adapt_lambda(const avx_operator* op, float k, float d, float* lambda_out) {
  if (!op || !lambda_out) return fail(AVX_E_ARG, "null argument");
  if (op->kind == 1) {
    // NoncartesianOperator::AdaptLambda (noncartesian_operator.cpp:88-95)
    const double subfac = op->W / (op->spf * M_PI / 2.0);
    *lambda_out = (float)(subfac * k + d);
    return AVX_OK;
  }
  double subfac = (double)op->W * op->H * op->T;
  if (op->has_mask)
    subfac /= op->mask_norm2;
  else
    subfac /= (double)op->W * op->H * op->T;
  *lambda_out = (float)(subfac * k + d);
  return AVX_OK;
}

void avx_operator_destroy(avx_operator* op) { delete op; }

avx_status avx_default_params(int method, avx_pd_params* p) {
  if (!p) return fail(AVX_E_ARG, "null params");
  if (!method_ok(method)) return fail(AVX_E_UNSUPPORTED, "method not provided (TV, TVtemp, TGV2, ICTV, ICTGV2 are)");
  memset(p, 0, sizeof(*p));
  p->maxIt = 500;
  p->stopPDGap = 0.f;
  p->sigma = (float)(1.0 / 3.0);
  p->tau = (float)(1.0 / 3.0);
  p->sigmaTauRatio = 1.f;
  p->dx = p->dy = p->dt = 1.f;
  p->dx2 = p->dy2 = p->dt2 = 1.f;
  p->alpha0 = (float)std::sqrt(2.0);
  p->alpha1 = 1.f;
  p->adaptLambda = 1;
  if (method == AVX_METHOD_ICTGV2) {
    p->timeSpaceWeight = 6.5f;  // ictgv2.cpp:46-58
    p->timeSpaceWeight2 = 2.5f;
    p->alpha = 0.6423f;
    p->adaptK = (float)(0.4 / (5.1191 * 0.35));
    p->adaptD = (float)(10.0 / (5.1191 * 0.35));
  } else if (method == AVX_METHOD_ICTV) {
    p->timeSpaceWeight = 4.f;  // ictv.cpp:37-60
    p->timeSpaceWeight2 = 0.5f;
    p->alpha = 0.5f;
    p->adaptK = (float)(0.4 / (5.1191 * 0.35));
    p->adaptD = (float)(10.0 / (5.1191 * 0.35));
  } else {
    p->timeSpaceWeight = 5.f;  // tv.cpp:48, tgv2.cpp:45
    p->adaptK = (float)(0.4 * 0.2991);
    p->adaptD = (float)(10.0 * 0.2991);
  }
  p->lambda = 1.f;
  return AVX_OK;
}

avx_status avx_solver_create(int method, unsigned width, unsigned height, unsigned coils, unsigned frames,
                             const avx_pd_params* params, avx_operator* op, avx_solver** out) {
  if (!out || !op) return fail(AVX_E_ARG, "null argument");
  if (!method_ok(method)) return fail(AVX_E_UNSUPPORTED, "method not provided (TV, TVtemp, TGV2, ICTV, ICTGV2 are)");
  if ((int)width != op->W || (int)height != op->H || (int)coils != op->C || (int)frames != op->T)
    return fail(AVX_E_ARG, "solver dimensions differ from the operator's");
  avx_solver* s = new avx_solver();
  s->method = method;
  s->W = (int)width; s->H = (int)height; s->C = (int)coils; s->T = (int)frames;
  s->op = op;
  if (params)
    s->p = *params;
  else
    avx_default_params(method, &s->p);
  if (s->p.adaptLambda) avx_operator_adapt_lambda(op, s->p.adaptK, s->p.adaptD, &s->p.lambda);
  *out = s;
  return AVX_OK;
}

avx_status avx_solver_get_params(const avx_solver* s, avx_pd_params* p) {
  if (!s || !p) return fail(AVX_E_ARG, "null argument");
  *p = s->p;
  return AVX_OK;
}
avx_status avx_solver_set_params(avx_solver* s, const avx_pd_params* p) {
  if (!s || !p) return fail(AVX_E_ARG, "null argument");
  s->p = *p;
  return AVX_OK;
}
avx_status avx_solver_set_verbose(avx_solver* s, int v) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  s->verbose = v != 0;
  return AVX_OK;
}
avx_status avx_solver_set_relative_stop(avx_solver* s, double rel) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  if (!(rel >= 0.0) || rel >= 1.0) return fail(AVX_E_ARG, "relative stop must lie in [0, 1)");
  s->stop_rel = rel;
  s->drop_graphs();
  return AVX_OK;
}

avx_status avx_solver_set_tuning(avx_solver* s, int autotune, int primal_tile, int dual_block) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  if (primal_tile < 0 || primal_tile >= AVX_PRIMAL_TILES || dual_block < 0 || dual_block >= AVX_DUAL_BLOCKS)
    return fail(AVX_E_ARG, "tuning index out of range");
  s->autotune = autotune != 0;
  s->tuned = false;
  s->primal_tile = primal_tile;
  s->dual_block = dual_block;
  s->drop_graphs();
  return AVX_OK;
}

avx_status avx_solver_get_tuning(const avx_solver* s, int* primal_tile, int* dual_block, const char** primal_name,
                                 int* dual_threads) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  if (primal_tile) *primal_tile = s->primal_tile;
  if (dual_block) *dual_block = s->dual_block;
  if (primal_name) *primal_name = avx::primal_tile_name(s->primal_tile);
  if (dual_threads) *dual_threads = avx::dual_block_threads(s->dual_block);
  return AVX_OK;
}

avx_status avx_solver_set_kspace_schedule(avx_solver* s, int rows_per_pass, int runtime_plan) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  if (rows_per_pass != 8 && rows_per_pass != 12 && rows_per_pass != 16)
    return fail(AVX_E_ARG, "rows per pass must be 8, 12 or 16");
  s->rows_kc = rows_per_pass;
  s->rows_rt = runtime_plan ? 1 : 0;
  s->drop_graphs();
  return AVX_OK;
}

avx_status avx_solver_get_kspace_schedule(const avx_solver* s, int* rows_per_pass, int* runtime_plan) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  if (rows_per_pass) *rows_per_pass = s->rows_kc;
  if (runtime_plan) *runtime_plan = s->rows_rt;
  return AVX_OK;
}

avx_status avx_solver_set_debug(avx_solver* s, int debug, int debugstep) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  s->debug = debug != 0;
  s->debugstep = debugstep;
  return AVX_OK;
}
avx_status avx_solver_set_stream(avx_solver* s, void* st) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  s->user_stream = (cudaStream_t)st;
  return AVX_OK;
}

avx_status avx_solver_run(avx_solver* s, const avx_cf32* d_data, avx_cf32* d_x, const avx_cf32* d_b1) {
  if (!s || !d_data || !d_x || !d_b1) return fail(AVX_E_ARG, "null argument");
  return solver_run(s, reinterpret_cast<const float2*>(d_data), reinterpret_cast<float2*>(d_x),
                    reinterpret_cast<const float2*>(d_b1));
}

avx_status avx_solver_adapt_step_size(avx_solver* s, const avx_cf32* const* d_diff, const avx_cf32* d_b1) {
  if (!s || !d_diff || !d_b1) return fail(AVX_E_ARG, "null argument");
  avx_status r = solver_alloc(s);
  if (r != AVX_OK) return r;
  const int P = method_P(s->method);
  const size_t N = (size_t)s->N();
  r = prepare_run(s, nullptr, nullptr);
  if (r != AVX_OK) return r;
  // e = xbar - x with xbar = 0 gives -diff; the norms are sign-invariant
  for (int c = 0; c < P; ++c) {
    AVX_CK(cudaMemcpyAsync(s->primc(c), d_diff[c], N * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
    AVX_CK(cudaMemsetAsync(s->extc(c), 0, N * sizeof(float2), s->stream));
  }
  const PDArgs a = make_pdargs(s);
  avx::Ptr8 e;
  for (int c = 0; c < 8; ++c) e.p[c] = c < P ? s->escrc(c) : nullptr;
  const float2* b1 = reinterpret_cast<const float2*>(d_b1);
  if (s->op->kind == 1) {
    avx::launch_step_img(s->method, a, e, P, s->pimg.p, s->stream);
    radial_pass(s, 1, b1, s->escrc(0), nullptr);
    avx::launch_step_finalize(a, s->pimg.p, s->pk.p, avx::radial_interp_blocks(s->op->rg), s->p.sigmaTauRatio,
                              s->stream);
  } else {
    const KArgs ke = make_kargs(s, b1, s->escrc(0), nullptr);
    avx::launch_step(s->method, a, ke, e, P, s->pimg.p, s->pk.p, s->p.sigmaTauRatio, s->stream);
  }
  AVX_CK(cudaGetLastError());
  DevState h;
  AVX_CK(cudaMemcpyAsync(&h, s->st.p, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  AVX_CK(cudaStreamSynchronize(s->stream));
  s->p.sigma = (float)h.sigma;
  s->p.tau = (float)h.tau;
  return AVX_OK;
}

avx_status avx_solver_compute_gap(avx_solver* s, const avx_cf32* const* d_x, const avx_cf32* const* d_y,
                                  const avx_cf32* d_z, const avx_cf32* d_data, const avx_cf32* d_b1, double* gstar,
                                  double* gap) {
  if (!s || !d_x || !d_y || !d_z || !d_data || !d_b1) return fail(AVX_E_ARG, "null argument");
  avx_status r = solver_alloc(s);
  if (r != AVX_OK) return r;
  const int P = method_P(s->method), D = method_D(s->method);
  const size_t N = (size_t)s->N();
  r = prepare_run(s, reinterpret_cast<const float2*>(d_data), nullptr);
  if (r != AVX_OK) return r;
  r = prepare_b1t(s, reinterpret_cast<const float2*>(d_b1));
  if (r != AVX_OK) return r;
  for (int c = 0; c < P; ++c)
    AVX_CK(cudaMemcpyAsync(s->primc(c), d_x[c], N * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
  for (int c = 0; c < D; ++c)
    AVX_CK(cudaMemcpyAsync(s->dualc(c), d_y[c], N * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
  if (s->op->kind == 1)
    AVX_CK(cudaMemcpyAsync(s->z.p, d_z, s->z.n * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
  else if (s->op->R)
    avx::launch_gather_rows(s->op->geom(), reinterpret_cast<const float2*>(d_z), s->z.p, 0, s->stream);
  PDArgs a = make_pdargs(s);
  const KArgs kx = make_kargs(s, reinterpret_cast<const float2*>(d_b1), s->primc(0), nullptr);
  avx::GapConst gc = make_gapconst(s);
  gc.stop_gap = -1.0;
  gc.stop_rel = 0.0;
  double* h = s->hist.p;
  int nk = s->C * s->T;
  if (s->op->kind == 1) {
    a.khz = s->op->r_khz.p;
    nk = avx::radial_interp_blocks(s->op->rg);
    radial_pass(s, 2, reinterpret_cast<const float2*>(d_b1), s->primc(0), nullptr);
    avx::launch_gap_tail(s->method, a, kx, s->pimg.p, s->pk.p, nk, gc, h, h + (s->cap + 1), h + 2 * (s->cap + 1),
                         s->cap, 0, s->stream);
  } else {
    avx::launch_gap(s->method, a, kx, s->op->r_khz.p, s->pimg.p, s->pk.p, gc, h, h + (s->cap + 1),
                    h + 2 * (s->cap + 1), s->cap, 0, s->stream);
  }
  AVX_CK(cudaGetLastError());
  const int nimg = avx::gap_img_blocks(s->W, s->H, s->T);
  std::vector<double> pk(3 * nk), pi(8 * nimg);
  AVX_CK(cudaMemcpyAsync(pk.data(), s->pk.p, pk.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  AVX_CK(cudaMemcpyAsync(pi.data(), s->pimg.p, pi.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  AVX_CK(cudaStreamSynchronize(s->stream));
  double v[11] = {0};
  for (int i = 0; i < nk; ++i)
    for (int j = 0; j < 3; ++j) v[j] += pk[j * nk + i];
  for (int i = 0; i < nimg; ++i)
    for (int j = 0; j < 8; ++j) v[3 + j] += pi[j * nimg + i];
  const double lam = s->p.lambda;
  const double g = 0.5 * lam * (v[0] + s->d_off_energy) + v[1] + v[2] / (2.0 * lam) + v[3] + v[4] + v[5] + v[6];
  double reg;
  if (s->method == AVX_METHOD_TV || s->method == AVX_METHOD_TVTEMP)
    reg = v[7];
  else if (s->method == AVX_METHOD_ICTV)
    reg = s->p.alpha1 * gc.ic_a * v[7] + s->p.alpha1 * gc.ic_b * v[9];
  else if (s->method == AVX_METHOD_TGV2)
    reg = s->p.alpha1 * v[7] + s->p.alpha0 * v[8];
  else
    reg = gc.ic_a * (s->p.alpha1 * v[7] + s->p.alpha0 * v[8]) + gc.ic_b * (s->p.alpha1 * v[9] + s->p.alpha0 * v[10]);
  if (gstar) *gstar = g;
  if (gap) *gap = std::fabs(g + reg);
  return AVX_OK;
}

// ===========================================================================
// Operator-norm estimate: getopnorm (matlab/getopnorm.m:1-17)
// ===========================================================================

// A^H A u into img with the operator's own kernels: the compact sampled rows,
// in the operator's y-transform arithmetic, for the Cartesian operator
// (row mode 4 applies mask^2 between the transforms); gridding, interpolation,
// spreading and the adjoint grid transform for the radial one.
static avx_status encoding_normal(avx_operator* op, const float2* b1, const float2* b1t, const float2* u, float2* img,
                                  float2* kbuf, DevState* st, cudaStream_t s) {
  if (op->kind == 1) {
    RArgs r = make_rargs(op, b1, u, nullptr);
    r.st = st;
    r.out = kbuf;
    avx::launch_rad_forward_grid(r, s);
    avx::launch_rad_interp(r, 3, s);
    avx::launch_rad_spread(r, kbuf, s);
    avx::launch_rad_adjoint_image(r, img, s);
    return AVX_OK;
  }
  if (!op->R) {
    AVX_CK(cudaMemsetAsync(img, 0, (size_t)op->W * op->H * op->T * sizeof(float2), s));
    return AVX_OK;
  }
  KArgs k;
  memset(&k, 0, sizeof(k));
  k.g = op->geom();
  k.b1 = b1;
  k.in = u;
  k.qp = op->d_qp.p;
  k.st = st;
  set_tc(&k, op);
  k.b1t = b1t;
  avx::launch_kspace(k, 4, s);
  avx::launch_adjoint(k, img, s);
  return AVX_OK;
}

// Power iteration over K^H K, K = (K_reg, A) of `method` (AVX_M_ENCODING: A
// alone), as getopnorm.m runs it:
//   y = K^H K x0;  iters times: x = y / ||y|| (y when ||y|| = 0), y = K^H K x, l = y^H x
// and *opnorm = |l|.  x0 starts the image component, the auxiliary primal
// components start at zero.  The operator applications run in fp32 (the
// operator's own arithmetic), the norms and inner products in FP64 on the
// device; the iterate is normalised on the device, so the loop reads the
// device once, at its end.  hist (optional) receives |y^H x| after each of
// the iters + 1 applications.
static avx_status power_iteration(avx_operator* op, int method, const Wts& w1, const Wts& w2, const float2* b1,
                                  const float2* b1t, const float2* x0, unsigned iters, cudaStream_t s, double* opnorm,
                                  double* hist) {
  const int P = method == AVX_M_ENCODING ? 1 : method_P(method);
  const int D = method == AVX_M_ENCODING ? 0 : method_D(method);
  const size_t N = (size_t)op->W * op->H * op->T;
  DevBuf<float2> x, y, d, khk, kbuf;
  DevBuf<double> partial, sums;
  DevBuf<DevState> st;
  AVX_CK(x.alloc(P * N));
  AVX_CK(y.alloc(P * N));
  AVX_CK(d.alloc(std::max(D, 1) * N));
  AVX_CK(khk.alloc(N));
  AVX_CK(kbuf.alloc(op->kind == 1 ? (size_t)op->C * op->T * op->S : 1));
  AVX_CK(partial.alloc(3 * AVX_RED_BLOCKS));
  AVX_CK(sums.alloc(3 * ((size_t)iters + 1)));
  AVX_CK(st.alloc(1));
  AVX_CK(cudaMemsetAsync(st.p, 0, sizeof(DevState), s));
  AVX_CK(cudaMemcpyAsync(x.p, x0, N * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  if (P > 1) AVX_CK(cudaMemsetAsync(x.p + N, 0, (P - 1) * N * sizeof(float2), s));
  avx::OpnArgs a;
  memset(&a, 0, sizeof(a));
  a.W = op->W; a.H = op->H; a.T = op->T; a.N = (long long)N;
  float2* xs[8] = {};
  for (int c = 0; c < P; ++c) {
    xs[c] = x.p + c * N;
    a.x[c] = xs[c];
    a.y[c] = y.p + c * N;
  }
  for (int c = 0; c < D; ++c) a.d[c] = d.p + c * N;
  a.khk = khk.p;
  a.w1 = w1;
  a.w2 = w2;
  a.partial = partial.p;
  for (unsigned i = 0; i <= iters; ++i) {
    if (i > 0) avx::launch_opn_normalise(a, P, xs, sums.p + 3 * (i - 1), s);
    if (D) avx::launch_opn_dual(method, a, s);
    avx_status r = encoding_normal(op, b1, b1t, a.x[0], khk.p, kbuf.p, st.p, s);
    if (r != AVX_OK) return r;
    avx::launch_opn_primal(method, a, s);
    avx::launch_opn_finalize(partial.p, sums.p + 3 * i, s);
  }
  AVX_CK(cudaGetLastError());
  std::vector<double> h(3 * ((size_t)iters + 1));
  DevState hs;
  AVX_CK(cudaMemcpyAsync(h.data(), sums.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  AVX_CK(cudaMemcpyAsync(&hs, st.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
  AVX_CK(cudaStreamSynchronize(s));
  if (hs.err) return fail(AVX_E_NUMERIC, "tensor-core y-transform: a pipeline wait timed out");
  for (unsigned i = 0; i <= iters; ++i) {
    const double l = std::hypot(h[3 * i + 1], h[3 * i + 2]);
    if (hist) hist[i] = l;
    if (i == iters) *opnorm = l;
  }
  return AVX_OK;
}

avx_status avx_operator_opnorm(avx_operator* op, const avx_cf32* d_x0, const avx_cf32* d_b1, unsigned iters,
                               double* opnorm, double* hist) {
  if (!op || !d_x0 || !d_b1 || !opnorm) return fail(AVX_E_ARG, "null argument");
  if (iters < 1) return fail(AVX_E_ARG, "the power iteration needs at least one iteration");
  const float2* b1 = reinterpret_cast<const float2*>(d_b1);
  const float2* b1t = nullptr;
  if (op->kind == 0 && op->dft_mode == AVX_DFT_SPLIT_BF16X3 && op->tc_np > 0) {
    AVX_CK(op->tc_b1t.alloc(avx::b1t_count(op->W, op->H, op->C)));
    avx::launch_b1_tile_transpose(b1, op->tc_b1t.p, op->W, op->H, op->C, 0);
    b1t = op->tc_b1t.p;
  }
  const Wts w0 = make_wts(1.f, 1.f, 1.f);
  return power_iteration(op, AVX_M_ENCODING, w0, w0, b1, b1t, reinterpret_cast<const float2*>(d_x0), iters, 0,
                         opnorm, hist);
}

avx_status avx_solver_opnorm(avx_solver* s, const avx_cf32* d_x0, const avx_cf32* d_b1, unsigned iters, int set_steps,
                             double* opnorm, double* hist) {
  if (!s || !d_x0 || !d_b1 || !opnorm) return fail(AVX_E_ARG, "null argument");
  if (iters < 1) return fail(AVX_E_ARG, "the power iteration needs at least one iteration");
  avx_status r = solver_alloc(s);
  if (r != AVX_OK) return r;
  r = solver_run_weights(s);
  if (r != AVX_OK) return r;
  const float2* b1 = reinterpret_cast<const float2*>(d_b1);
  r = prepare_b1t(s, b1);
  if (r != AVX_OK) return r;
  Wts w1, w2;
  solver_weights(s, &w1, &w2);
  double l = 0.0;
  r = power_iteration(s->op, s->method, w1, w2, b1, s->b1t.p, reinterpret_cast<const float2*>(d_x0), iters, s->stream,
                      &l, hist);
  if (r != AVX_OK) return r;
  *opnorm = l;
  if (set_steps) {
    if (!(l > 0.0) || !std::isfinite(l)) return fail(AVX_E_NUMERIC, "operator-norm estimate is not positive");
    // sig = s r, tau = s / r with s = 1 / ||K|| in place of 1/3 (tgv2_dmri.m:96-99)
    const double L = std::sqrt(l), ratio = s->p.sigmaTauRatio;
    s->p.sigma = (float)(ratio / L);
    s->p.tau = (float)(1.0 / (ratio * L));
  }
  return AVX_OK;
}

avx_status avx_solver_export(avx_solver* s, const char* dir, avx_export_cb cb, void* user) {
  if (!s || !cb) return fail(AVX_E_ARG, "null argument");
  auto send = [&](const char* name, const std::vector<double>& v) {
    std::vector<avx_cf32> c(v.size());
    for (size_t i = 0; i < v.size(); ++i) c[i] = avx_cf32{(float)v[i], 0.f};
    cb(dir, name, c.data(), c.size(), user);
  };
  if (method_ic(s->method) && s->prim.p) {
    std::vector<avx_cf32> x3((size_t)s->N());
    AVX_CK(cudaMemcpy(x3.data(), s->primc(s->method == AVX_METHOD_ICTV ? 1 : 4), x3.size() * sizeof(avx_cf32),
                      cudaMemcpyDeviceToHost));
    cb(dir, "x3_component", x3.data(), x3.size(), user);
  }
  if (s->debug && s->hist.p) {
    const int ng = s->last.ngap;
    std::vector<double> h((size_t)3 * (s->cap + 1));
    AVX_CK(cudaMemcpy(h.data(), s->hist.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    send("PDGap", std::vector<double>(h.begin(), h.begin() + ng));
    if (s->method == AVX_METHOD_ICTGV2) {
      const size_t o = s->cap + 1;
      send("ICTGVnorm", std::vector<double>(h.begin() + o, h.begin() + o + ng + 1));
      send("DATAfidelity", std::vector<double>(h.begin() + 2 * o, h.begin() + 2 * o + ng + 1));
    } else if (s->method == AVX_METHOD_ICTV) {  // ictv.cpp:375-390, no pre-loop record
      const size_t o = s->cap + 1;
      send("ictvnorm", std::vector<double>(h.begin() + o, h.begin() + o + ng));
      send("DATAfidelity", std::vector<double>(h.begin() + 2 * o, h.begin() + 2 * o + ng));
    }
  }
  return AVX_OK;
}

avx_status avx_solver_get_stats(const avx_solver* s, avx_run_stats* st) {
  if (!s || !st) return fail(AVX_E_ARG, "null argument");
  *st = s->stats;
  return AVX_OK;
}

avx_status avx_solver_set_timing(avx_solver* s, int on) {
  if (!s) return fail(AVX_E_ARG, "null solver");
  s->timing = on != 0;
  return AVX_OK;
}

avx_status avx_solver_kernel_times(const avx_solver* s, float* mean_ms, unsigned* count) {
  if (!s || !mean_ms) return fail(AVX_E_ARG, "null argument");
  for (int j = 0; j < AVX_NSTAGE; ++j) mean_ms[j] = s->kmean[j];
  if (count) *count = s->kcount;
  return AVX_OK;
}

void avx_solver_destroy(avx_solver* s) { delete s; }

}  // extern "C"

void HostPlan::release() {
  if (s) avx_solver_destroy(s);
  if (op) avx_operator_destroy(op);
  if (stream) cudaStreamDestroy(stream);
  s = nullptr;
  op = nullptr;
  stream = nullptr;
  dk.release();
  db1.release();
  dx.release();
  dm.release();
  mask.clear();
  device = method = -1;
}

extern "C" {

// ---------------------------------------------------------------------------
// utils
// ---------------------------------------------------------------------------

static avx::Ptr18 ptrs(const avx_cf32* const* p, int n) {
  avx::Ptr18 r;
  for (int i = 0; i < 18; ++i) r.p[i] = i < n ? const_cast<float2*>(reinterpret_cast<const float2*>(p[i])) : nullptr;
  return r;
}

avx_status avx_gradient(const avx_cf32* d_u, avx_cf32* const* d_g, unsigned W, unsigned H, unsigned T, float dx,
                        float dy, float dt) {
  if (!d_u || !d_g) return fail(AVX_E_ARG, "null argument");
  avx::launch_gradient(reinterpret_cast<const float2*>(d_u), ptrs(d_g, 3), W, H, T, make_wts(dx, dy, dt), 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_divergence(const avx_cf32* const* d_y, avx_cf32* d_div, unsigned W, unsigned H, unsigned T, float dx,
                          float dy, float dt) {
  if (!d_y || !d_div) return fail(AVX_E_ARG, "null argument");
  avx::launch_divergence(ptrs(d_y, 3), reinterpret_cast<float2*>(d_div), W, H, T, make_wts(dx, dy, dt), 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_sym_gradient(const avx_cf32* const* d_v, avx_cf32* const* d_e, unsigned W, unsigned H, unsigned T,
                            float dx, float dy, float dt) {
  if (!d_v || !d_e) return fail(AVX_E_ARG, "null argument");
  avx::launch_symgrad(ptrs(d_v, 3), ptrs(d_e, 6), W, H, T, make_wts(dx, dy, dt), 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_sym_divergence(const avx_cf32* const* d_w, avx_cf32* const* d_d, unsigned W, unsigned H, unsigned T,
                              float dx, float dy, float dt) {
  if (!d_w || !d_d) return fail(AVX_E_ARG, "null argument");
  avx::launch_symdiv(ptrs(d_w, 6), ptrs(d_d, 3), W, H, T, make_wts(dx, dy, dt), 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_prox3(avx_cf32* const* d_y, unsigned N, float scale) {
  if (!d_y) return fail(AVX_E_ARG, "null argument");
  avx::launch_prox(ptrs(d_y, 3), 3, N, scale, 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_prox6(avx_cf32* const* d_y, unsigned N, float scale) {
  if (!d_y) return fail(AVX_E_ARG, "null argument");
  avx::launch_prox(ptrs(d_y, 6), 6, N, scale, 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_norm3(const avx_cf32* const* d_g, float* d_norm, unsigned N) {
  if (!d_g || !d_norm) return fail(AVX_E_ARG, "null argument");
  avx::launch_norm(ptrs(d_g, 3), 3, d_norm, N, 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}
avx_status avx_norm6(const avx_cf32* const* d_g, float* d_norm, unsigned N) {
  if (!d_g || !d_norm) return fail(AVX_E_ARG, "null argument");
  avx::launch_norm(ptrs(d_g, 6), 6, d_norm, N, 0);
  AVX_CK(cudaDeviceSynchronize());
  return AVX_OK;
}

static avx_status regnorm(const float2* u, const float2* u2, const avx_cf32* const* v, unsigned W, unsigned H,
                          unsigned T, Wts w, double* s1, double* s2) {
  const int nb = 256;
  DevBuf<double> part;
  AVX_CK(part.alloc(2 * nb));
  avx::launch_regnorm(u, u2, v ? ptrs(v, 3) : avx::Ptr18{}, v ? 1 : 0, W, H, T, w, part.p, nb, 0);
  std::vector<double> h(2 * nb);
  AVX_CK(cudaMemcpy(h.data(), part.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
  double a = 0, b = 0;
  for (int i = 0; i < nb; ++i) {
    a += h[i];
    b += h[nb + i];
  }
  *s1 = a;
  *s2 = b;
  return AVX_OK;
}

avx_status avx_tv_norm(const avx_cf32* d_u, unsigned W, unsigned H, unsigned T, float dx, float dy, float dt,
                       double* out) {
  if (!d_u || !out) return fail(AVX_E_ARG, "null argument");
  double a, b;
  avx_status r = regnorm(reinterpret_cast<const float2*>(d_u), nullptr, nullptr, W, H, T, make_wts(dx, dy, dt), &a, &b);
  *out = a;
  return r;
}
avx_status avx_tgv2_norm(const avx_cf32* d_x1, const avx_cf32* const* d_x2, float alpha0, float alpha1, unsigned W,
                         unsigned H, unsigned T, float dx, float dy, float dt, double* out) {
  if (!d_x1 || !d_x2 || !out) return fail(AVX_E_ARG, "null argument");
  double a, b;
  avx_status r = regnorm(reinterpret_cast<const float2*>(d_x1), nullptr, d_x2, W, H, T, make_wts(dx, dy, dt), &a, &b);
  *out = alpha1 * a + alpha0 * b;
  return r;
}
avx_status avx_ictgv2_norm(const avx_cf32* d_x1, const avx_cf32* const* d_x2, const avx_cf32* d_x3,
                           const avx_cf32* const* d_x4, float alpha0, float alpha1, float alpha, unsigned W, unsigned H,
                           unsigned T, const float* w1, const float* w2, double* out) {
  if (!d_x1 || !d_x2 || !d_x3 || !d_x4 || !w1 || !w2 || !out) return fail(AVX_E_ARG, "null argument");
  double a1, b1, a2, b2;
  avx_status r = regnorm(reinterpret_cast<const float2*>(d_x1), reinterpret_cast<const float2*>(d_x3), d_x2, W, H, T,
                         make_wts(w1[0], w1[1], w1[2]), &a1, &b1);
  if (r != AVX_OK) return r;
  r = regnorm(reinterpret_cast<const float2*>(d_x3), nullptr, d_x4, W, H, T, make_wts(w2[0], w2[1], w2[2]), &a2, &b2);
  const double m = std::min((double)alpha, 1.0 - alpha);
  *out = (alpha / m) * (alpha1 * a1 + alpha0 * b1) + ((1.0 - alpha) / m) * (alpha1 * a2 + alpha0 * b2);
  return r;
}

float avx_ellipke(float m) {
  if (!(m >= 0.f && m <= 1.f)) {
    g_err = "Ellipke: only values in the range of [0,1] are allowed";
    return NAN;
  }
  return (float)ellipke_d(m);
}

avx_status avx_time_space_weights(float tsw, float* ds, float* dt) {
  if (!ds || !dt) return fail(AVX_E_ARG, "null argument");
  double a, b;
  if (!time_space_weights(tsw, &a, &b)) return fail(AVX_E_ARG, "ComputeTimeSpaceWeights: invalid ratio");
  *ds = (float)a;
  *dt = (float)b;
  return AVX_OK;
}

// ---------------------------------------------------------------------------
// coil-sensitivity estimation
// ---------------------------------------------------------------------------

avx_status avx_coil_default_params(avx_coil_params* p) {
  if (!p) return fail(AVX_E_ARG, "null params");
  p->uH1mu = 1e-5f;
  p->uReg = 0.2f;
  p->uNrIt = 100;
  p->uSigmaTauRatio = 1.f;
  p->uSigma = (float)std::sqrt(1.0 / 12.0);
  p->uTau = (float)std::sqrt(1.0 / 12.0);
  p->uAlpha0 = (float)std::sqrt(2.0);
  p->uAlpha1 = 1.f;
  p->b1Reg = 2.f;
  p->b1NrIt = 500;
  p->b1SigmaTauRatio = 1.f;
  p->b1Sigma = (float)std::sqrt(1.0 / 8.0);
  p->b1Tau = (float)std::sqrt(1.0 / 8.0);
  p->b1FinalReg = 0.1f;
  p->b1FinalNrIt = 1000;
  return AVX_OK;
}

avx_status avx_coil_time_averaged(unsigned W, unsigned H, unsigned C, unsigned T, const avx_cf32* d_kdata,
                                  const float* d_mask, avx_cf32* d_u, avx_cf32* d_crec, int apply_phase) {
  if (!d_kdata || !d_u || !d_crec) return fail(AVX_E_ARG, "null argument");
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  return coil_time_averaged((int)W, (int)H, (int)C, (int)T, reinterpret_cast<const float2*>(d_kdata), d_mask,
                            reinterpret_cast<float2*>(d_u), reinterpret_cast<float2*>(d_crec), apply_phase, 0);
}

avx_status avx_coil_b1_from_u_h1(unsigned W, unsigned H, unsigned C, const avx_coil_params* p, const avx_cf32* d_u,
                                 const avx_cf32* d_crec, avx_cf32* d_absb1) {
  if (!p || !d_u || !d_crec || !d_absb1) return fail(AVX_E_ARG, "null argument");
  return coil_b1_from_u_h1((int)W, (int)H, (int)C, *p, reinterpret_cast<const float2*>(d_u),
                           reinterpret_cast<const float2*>(d_crec), reinterpret_cast<float2*>(d_absb1), 0);
}

avx_status avx_coil_utgv2(unsigned W, unsigned H, const avx_coil_params* p, const avx_cf32* d_b1,
                          const avx_cf32* d_crec, const int* h_inds, unsigned ninds, avx_cf32* d_x1) {
  if (!p || !d_b1 || !d_crec || !h_inds || !ninds || !d_x1) return fail(AVX_E_ARG, "null argument");
  std::vector<int> inds(h_inds, h_inds + ninds);
  return coil_utgv2((int)W, (int)H, *p, reinterpret_cast<const float2*>(d_b1), reinterpret_cast<const float2*>(d_crec),
                    inds, reinterpret_cast<float2*>(d_x1), 0);
}

avx_status avx_coil_b1_recon(unsigned W, unsigned H, unsigned coils, unsigned max_it, float mu,
                             const avx_coil_params* p, const avx_cf32* d_u0, const avx_cf32* d_crec, avx_cf32* d_b1) {
  if (!p || !d_u0 || !d_crec || !d_b1) return fail(AVX_E_ARG, "null argument");
  return coil_b1_recon((int)W, (int)H, (int)coils, max_it, mu, *p, reinterpret_cast<const float2*>(d_u0),
                       reinterpret_cast<const float2*>(d_crec), reinterpret_cast<float2*>(d_b1), 0);
}

avx_status avx_coil_time_averaged_radial(unsigned W, unsigned H, unsigned C, unsigned T, unsigned S,
                                         const float* d_traj, const float* d_dens, const avx_cf32* d_kdata,
                                         avx_cf32* d_u, avx_cf32* d_crec, int apply_phase) {
  if (!d_traj || !d_dens || !d_kdata || !d_u || !d_crec) return fail(AVX_E_ARG, "null argument");
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  return coil_time_averaged_radial((int)W, (int)H, (int)C, (int)T, (int)S, d_traj, d_dens,
                                   reinterpret_cast<const float2*>(d_kdata), reinterpret_cast<float2*>(d_u),
                                   reinterpret_cast<float2*>(d_crec), apply_phase, 0);
}

// FindNormalizationFactor (raw_data_preparation.cpp:661-686): the first
// largest value, then every later value >= 0.9 of it in scan order (values
// before the first maximum are not considered), and utils::Median of those
// (utils.cpp:1442-1462: the mean of the two middle values for an even count).
static float find_normalization_factor(const std::vector<float>& v) {
  size_t imax = 0;
  for (size_t i = 1; i < v.size(); ++i)
    if (v[i] > v[imax]) imax = i;
  const double thr = (double)v[imax] * 0.9;
  std::vector<float> big{v[imax]};
  for (size_t i = imax + 1; i < v.size(); ++i)
    if ((double)v[i] >= thr) big.push_back(v[i]);
  std::sort(big.begin(), big.end());
  const size_t ind = (size_t)(big.size() * 0.5);
  if (big.size() % 2 == 0) return (float)(0.5 * (double)(big[ind] + big[ind - 1]));
  return big[ind];
}

avx_status avx_normalize_data(unsigned W, unsigned H, unsigned C, unsigned T, unsigned S, const float* d_mask,
                              const float* d_dens, avx_cf32* d_kdata, float* datanorm) {
  if (!d_mask || !d_kdata || !datanorm || (S > 0 && !d_dens)) return fail(AVX_E_ARG, "null argument");
  if (!W || !H || !C || !T) return fail(AVX_E_ARG, "empty dimensions");
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  const size_t HW = (size_t)W * H;
  DevBuf<float2> u, crec;
  AVX_CK(u.alloc(HW));
  AVX_CK(crec.alloc((size_t)C * HW));
  float2* kd = reinterpret_cast<float2*>(d_kdata);
  // |u| = sqrt(sum_c |crec_c|^2) of the time-averaged reconstruction without phase
  r = S > 0 ? coil_time_averaged_radial((int)W, (int)H, (int)C, (int)T, (int)S, d_mask, d_dens, kd, u.p, crec.p, 0, 0)
            : coil_time_averaged((int)W, (int)H, (int)C, (int)T, kd, d_mask, u.p, crec.p, 0, 0);
  if (r != AVX_OK) return r;
  std::vector<float2> hu(HW);
  AVX_CK(cudaMemcpy(hu.data(), u.p, HW * sizeof(float2), cudaMemcpyDeviceToHost));
  // The Cartesian normalisation transforms with the centred FFT
  // (raw_data_preparation.cpp:372-373), whose image magnitude is the
  // uncentred one shifted by (W/2, H/2); the scan order below follows it.
  std::vector<float> mag(HW);
  for (unsigned y = 0; y < H; ++y)
    for (unsigned x = 0; x < W; ++x) {
      const size_t src = S > 0 ? (size_t)y * W + x : (size_t)((y + H - H / 2) % H) * W + (x + W - W / 2) % W;
      const float2 v = hu[src];
      mag[(size_t)y * W + x] = std::sqrt(v.x * v.x + v.y * v.y);
    }
  const float median = find_normalization_factor(mag);
  if (!(median > 0.f) || !std::isfinite(median))
    return fail(AVX_E_NUMERIC, "no valid normalisation factor (the time-averaged image is zero or not finite)");
  const float f = S > 0 ? 255.f * (float)T / median : 255.f / median;
  const long long n = S > 0 ? (long long)S * C * T : (long long)HW * C * T;
  avx::launch_cscale(kd, n, f, 0);
  AVX_CK(cudaGetLastError());
  AVX_CK(cudaStreamSynchronize(0));
  *datanorm = f;
  return AVX_OK;
}

avx_status avx_coil_construction_radial(unsigned W, unsigned H, unsigned C, unsigned T, unsigned S,
                                        const avx_coil_params* p, const float* d_traj, const float* d_dens,
                                        const avx_cf32* d_kdata, avx_cf32* d_u, avx_cf32* d_b1) {
  if (!d_traj || !d_dens || !d_kdata || !d_u || !d_b1) return fail(AVX_E_ARG, "null argument");
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  avx_coil_params dp;
  avx_coil_default_params(&dp);
  PoolScope ps;
  AVX_CK(ps.init());
  DevBuf<float2> u0, crec;
  AVX_CK(u0.alloc((size_t)W * H));
  AVX_CK(crec.alloc((size_t)C * W * H));
  r = coil_time_averaged_radial((int)W, (int)H, (int)C, (int)T, (int)S, d_traj, d_dens,
                                reinterpret_cast<const float2*>(d_kdata), u0.p, crec.p, 1, ps.s);
  if (r != AVX_OK) return r;
  r = coil_estimate_on((int)W, (int)H, (int)C, p ? *p : dp, u0.p, crec.p, reinterpret_cast<float2*>(d_u),
                       reinterpret_cast<float2*>(d_b1), ps.s);
  if (r != AVX_OK) return r;
  AVX_CK(cudaStreamSynchronize(ps.s));
  return AVX_OK;
}

avx_status avx_coil_construction(unsigned W, unsigned H, unsigned C, unsigned T, const avx_coil_params* p,
                                 const avx_cf32* d_kdata, const float* d_mask, avx_cf32* d_u, avx_cf32* d_b1) {
  if (!d_kdata || !d_u || !d_b1) return fail(AVX_E_ARG, "null argument");
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  avx_coil_params dp;
  avx_coil_default_params(&dp);
  PoolScope ps;
  AVX_CK(ps.init());
  return coil_construction((int)W, (int)H, (int)C, (int)T, p ? *p : dp, reinterpret_cast<const float2*>(d_kdata),
                           d_mask, reinterpret_cast<float2*>(d_u), reinterpret_cast<float2*>(d_b1), ps.s);
}

// ---------------------------------------------------------------------------
// host-buffer path
// ---------------------------------------------------------------------------

avx_status avx_reconstruct_host(int method, unsigned W, unsigned H, unsigned C, unsigned T, const avx_pd_params* params,
                                int debugstep, const avx_cf32* h_kdata, const float* h_mask, const avx_cf32* h_b1,
                                const avx_cf32* h_u0, avx_cf32* h_x, avx_run_stats* stats) {
  if (!h_kdata || !h_b1 || !h_x) return fail(AVX_E_ARG, "null argument");
  avx_status r = check_dims(W, H, C, T);
  if (r != AVX_OK) return r;
  avx_pd_params defaults;
  if (!params) {
    r = avx_default_params(method, &defaults);
    if (r != AVX_OK) return r;
    params = &defaults;
  }
  std::lock_guard<std::mutex> lock(g_plan_mu);
  HostPlan& pl = g_plan;
  const size_t N = (size_t)W * H * T, K = N * C, HW = (size_t)W * H;
  int dev = 0;
  AVX_CK(cudaGetDevice(&dev));
  if (!pl.matches(dev, method, W, H, C, T, debugstep, params, h_mask)) {
    pl.release();
    AVX_CK(pl.dk.alloc(K));
    AVX_CK(pl.db1.alloc(HW * C));
    AVX_CK(pl.dx.alloc(N));
    if (h_mask) {
      AVX_CK(pl.dm.alloc(N));
      AVX_CK(cudaMemcpy(pl.dm.p, h_mask, N * sizeof(float), cudaMemcpyHostToDevice));
      pl.mask.assign(h_mask, h_mask + N);
    }
    r = avx_cartesian_operator_create(W, H, C, T, h_mask ? pl.dm.p : nullptr, 0, &pl.op);
    if (r != AVX_OK) return r;
    r = avx_solver_create(method, W, H, C, T, params, pl.op, &pl.s);
    if (r != AVX_OK) {
      pl.release();
      return r;
    }
    AVX_CK(cudaStreamCreateWithFlags(&pl.stream, cudaStreamNonBlocking));
    avx_solver_set_stream(pl.s, pl.stream);
    avx_solver_set_debug(pl.s, debugstep > 0, debugstep);
    pl.device = dev;
    pl.method = method;
    pl.W = W; pl.H = H; pl.C = C; pl.T = T;
    pl.debugstep = debugstep;
    pl.params = *params;
    pl.has_mask = h_mask != nullptr;
    avx_solver_get_params(pl.s, &pl.run_params);  // lambda adapted by the solver, if asked
  }
  // every call restarts from the parameters of a fresh solver (a run adapts sigma and tau)
  avx_solver_set_params(pl.s, &pl.run_params);
  cudaStream_t st = pl.stream;
  AVX_CK(cudaMemcpyAsync(pl.dk.p, h_kdata, K * sizeof(float2), cudaMemcpyHostToDevice, st));
  AVX_CK(cudaMemcpyAsync(pl.db1.p, h_b1, HW * C * sizeof(float2), cudaMemcpyHostToDevice, st));
  for (unsigned t = 0; t < T; ++t) {
    if (h_u0)
      AVX_CK(cudaMemcpyAsync(pl.dx.p + t * HW, h_u0, HW * sizeof(float2), cudaMemcpyHostToDevice, st));
    else
      AVX_CK(cudaMemsetAsync(pl.dx.p + t * HW, 0, HW * sizeof(float2), st));
  }
  // zero the data outside the mask (main.cpp:507-519): the compact rows only
  // read sampled rows, and the rest enter the gap's data term as zeros.
  if (h_mask) avx::launch_dense_rowidft(pl.op->geom(), pl.dk.p, pl.op->d_qp.p, pl.dm.p, st);  // masks dk in place
  AVX_CK(cudaGetLastError());
  r = avx_solver_run(pl.s, reinterpret_cast<avx_cf32*>(pl.dk.p), reinterpret_cast<avx_cf32*>(pl.dx.p),
                     reinterpret_cast<avx_cf32*>(pl.db1.p));
  if (r == AVX_OK) {
    AVX_CK(cudaMemcpyAsync(h_x, pl.dx.p, N * sizeof(float2), cudaMemcpyDeviceToHost, st));
    AVX_CK(cudaStreamSynchronize(st));
    if (stats) *stats = pl.s->stats;
  }
  return r;
}

void avx_reconstruct_host_release(void) {
  std::lock_guard<std::mutex> lock(g_plan_mu);
  g_plan.release();
}

}  // extern "C"

// ===========================================================================
// Batched and served reconstructions: continuous batching at iteration
// granularity.  Set-up threads admit queued requests against the HBM budget
// and build each one's operator, solver, device state and iteration graphs on
// a stream of its own (memory from the device's stream-ordered pool); one
// scheduler thread advances every admitted request by slices of 20
// iterations (the gap cadence), keeps two slices in flight per request,
// reads each request's device state after every slice without blocking, and
// retires a request at its stop test or its last iteration, freeing its
// budget for the next admission.
// ===========================================================================

namespace {

constexpr unsigned kSlice = 20;     // iterations per slice (the stop test's gap cadence)
constexpr int kSetupThreads = 4;    // request set-up threads per engine
constexpr double kStarveMs = 2000;  // queue head waits at most this long before it blocks later admissions

// Device bytes of a request.  R < 0: no mask row count known yet, so the
// Cartesian k-space is counted at every row (an upper bound).
size_t request_workspace(const avx_request& r, long long R_known, int max_rows_known) {
  const size_t W = r.width, H = r.height, C = r.coils, T = r.frames, N = W * H * T;
  const size_t P = (size_t)method_P(r.method), D = (size_t)method_D(r.method);
  const size_t c8 = sizeof(float2);
  size_t b = 0;
  size_t kspace = 0;  // values of z (and of d)
  if (r.op_kind == 0) {
    const size_t R = R_known >= 0 ? (size_t)R_known : H * T;
    const size_t max_rows = R_known >= 0 ? (size_t)max_rows_known : H;
    const size_t Rk = std::max<size_t>(R, 1);
    kspace = C * Rk * W;
    b += R * 4 + (T + 1) * 4 + R * W * 4 + (W + H) * c8 + kspace * c8 + N * c8 + (r.d_mask ? N * 4 : 0);
    const size_t np = std::max<size_t>(16, (2 * max_rows + 15) / 16 * 16);
    if (max_rows > 0 && np <= TC_MAX_NP) {
      b += avx::tc_ytab_bytes((int)H, (int)T, (int)np) + avx::tc_ctab_bytes((int)H, (int)T, (int)np);
      b += avx::b1t_count((int)W, (int)H, (int)C) * c8;
    }
  } else {
    const size_t S = (size_t)r.n_fe * r.spokes_per_frame;
    const int isw = std::max(2, (int)r.sector_width);
    const size_t Gx = (size_t)radial_grid_size((int)W, r.osf), Gy = (size_t)radial_grid_size((int)H, r.osf);
    const size_t sectors = T * ((Gx + isw - 1) / isw) * ((Gy + isw - 1) / isw) + 1;
    kspace = C * T * S;
    b += T * S * (2 * 4 + 4 + 4) + (W + H) * 4 + sectors * 4 + (Gx + Gy) * c8 + T * C * Gx * Gy * c8 + N * c8;
    b += T * S * (8 + 2 * 8 * 4);  // window starts and Kaiser-Bessel weights
    b += T * S * 4 * 4 + 2 * sectors * 4;  // the spreading's work list, its offsets and order
  }
  // solver: primal, extragradient and step scratch (3P), duals (D), z and d, reductions, history
  b += (3 * P + D) * N * c8 + 2 * kspace * c8;
  b += 8 * (size_t)std::max(AVX_RED_BLOCKS, avx::gap_img_blocks((int)W, (int)H, (int)T)) * 8;
  b += 3 * (std::max(C * T, (kspace + 255) / 256) + 1) * 8;
  b += 3 * ((size_t)r.params.maxIt + 3) * 8 + 4096;
  return b + b / 20 + ((size_t)4 << 20);  // pool granularity and slack
}

double ms_since(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// One admitted request.
struct Job {
  avx_request r{};
  size_t ws = 0;  // bytes held against the budget
  std::chrono::steady_clock::time_point t_submit, t_start;
  int slot = -1;  // stream and pinned state slots
  avx_operator* op = nullptr;
  avx_solver* s = nullptr;
  cudaStream_t stream = nullptr;
  unsigned k = 0;          // iterations enqueued
  unsigned launches = 0;   // kernels enqueued
  int inflight = 0;        // slices in flight (0..2)
  int head = 0;            // oldest slice in flight: index into ev / hs
  cudaEvent_t ev[2] = {nullptr, nullptr};
  DevState* hs[2] = {nullptr, nullptr};  // pinned copies of the device state after each slice
  bool stopped = false;
  avx_completion c{};
};

// Operator, solver, device state and iteration graphs of a request, built on
// the job's stream (pool memory).  Returns the status of the set-up.
avx_status job_setup(Job* j) {
  const avx_request& r = j->r;
  avx_status e;
  t_pool_stream = j->stream;
  if (r.op_kind == 0) {
    e = avx_cartesian_operator_create(r.width, r.height, r.coils, r.frames, r.d_mask, r.centered, &j->op);
    if (e == AVX_OK && avx_operator_set_dft_mode(j->op, r.dft_mode) != AVX_OK) avx_operator_set_dft_mode(j->op, AVX_DFT_FP32);
    if (e == AVX_OK) avx_operator_get_dft_mode(j->op, &j->c.dft_mode);
  } else {
    e = avx_radial_operator_create(r.width, r.height, r.coils, r.frames, r.spokes_per_frame * r.frames, r.n_fe,
                                   r.spokes_per_frame, r.d_traj, r.d_dens, r.kernel_width, r.sector_width, r.osf,
                                   &j->op);
  }
  if (e == AVX_OK) e = avx_solver_create(r.method, r.width, r.height, r.coils, r.frames, &r.params, j->op, &j->s);
  if (e == AVX_OK) {
    j->s->stream = j->stream;  // lent: the solver does not own it
    j->s->user_stream = j->stream;
    if (r.stop_gap_rel > 0.f) e = avx_solver_set_relative_stop(j->s, r.stop_gap_rel);
  }
  if (e == AVX_OK)
    e = solver_begin(j->s, reinterpret_cast<const float2*>(r.d_data), reinterpret_cast<float2*>(r.d_x),
                     reinterpret_cast<const float2*>(r.d_b1));
  // the graphs of every iteration shape the run takes
  for (unsigned k = 0; e == AVX_OK && k < j->s->p.maxIt; ++k) e = solver_graph(j->s, iter_shape(j->s, k),
                                                                                reinterpret_cast<const float2*>(r.d_b1));
  if (e == AVX_OK) {
    const cudaError_t ce = cudaStreamSynchronize(j->stream);
    if (ce != cudaSuccess) e = fail(AVX_E_CUDA, std::string("request set-up: ") + cudaGetErrorString(ce));
  }
  t_pool_stream = nullptr;
  return e;
}

void job_release(Job* j) {
  delete j->s;  // buffers go back to the pool on the job's stream
  delete j->op;
  j->s = nullptr;
  j->op = nullptr;
}

}  // namespace

struct avx_batch {
  int device = 0;
  size_t budget = 0, used = 0;
  int max_active = 1;
  int admitted = 0;  // in set-up, ready or running
  int pending = 0;   // submitted and not yet polled
  bool stop = false;
  std::mutex mu;
  std::condition_variable cv_setup, cv_sched, cv_done;
  struct Item {
    avx_request r;
    size_t ws;
    std::chrono::steady_clock::time_point t_submit;
  };
  std::deque<Item> queue;
  std::deque<Job*> ready;
  std::deque<avx_completion> done;
  std::vector<int> free_slots;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;  // 2 per slot
  DevState* h_states = nullptr;     // 2 per slot, pinned
  std::vector<std::thread> setup_threads;
  std::thread sched;

  void complete(Job* j, avx_status st) {
    j->c.status = (int)st;
    j->c.workspace_bytes = j->ws;
    std::lock_guard<std::mutex> lk(mu);
    used -= j->ws;
    --admitted;
    free_slots.push_back(j->slot);
    done.push_back(j->c);
    delete j;
    cv_setup.notify_all();
    cv_done.notify_all();
  }

  // first queued request whose workspace fits; nothing while the head has
  // waited longer than kStarveMs without fitting (it then gets the memory next)
  int pick() const {
    if (queue.empty() || free_slots.empty() || admitted >= max_active + kSetupThreads) return -1;
    const auto now = std::chrono::steady_clock::now();
    for (size_t i = 0; i < queue.size(); ++i) {
      if (used + queue[i].ws <= budget) return (int)i;
      if (i == 0 && ms_since(queue[0].t_submit, now) > kStarveMs) return -1;
    }
    return -1;
  }

  void setup_loop() {
    cudaSetDevice(device);
    for (;;) {
      Job* j = new Job();
      {
        std::unique_lock<std::mutex> lk(mu);
        int i = -1;
        while (!stop && (i = pick()) < 0) cv_setup.wait_for(lk, std::chrono::milliseconds(50));
        if (stop) {
          delete j;
          break;
        }
        j->r = queue[i].r;
        j->ws = queue[i].ws;
        j->t_submit = queue[i].t_submit;
        queue.erase(queue.begin() + i);
        used += j->ws;
        ++admitted;
        j->slot = free_slots.back();
        free_slots.pop_back();
      }
      j->t_start = std::chrono::steady_clock::now();
      j->c.tag = j->r.tag;
      j->c.queue_ms = ms_since(j->t_submit, j->t_start);
      j->stream = streams[j->slot];
      for (int q = 0; q < 2; ++q) {
        j->ev[q] = events[2 * j->slot + q];
        j->hs[q] = h_states + 2 * j->slot + q;
      }
      avx_status st = job_setup(j);
      if (st == AVX_OK && j->op->kind == 0) {
        // the exact footprint now that the sampled rows are known
        int max_rows = 0;
        for (int t = 0; t < j->op->T; ++t) max_rows = std::max(max_rows, j->op->row_off[t + 1] - j->op->row_off[t]);
        const size_t exact = request_workspace(j->r, j->op->R, max_rows);
        if (exact < j->ws) {
          std::lock_guard<std::mutex> lk(mu);
          used -= j->ws - exact;
          j->ws = exact;
          cv_setup.notify_all();
        }
      }
      if (st != AVX_OK) {
        job_release(j);
        j->c.run_ms = ms_since(j->t_start, std::chrono::steady_clock::now());
        complete(j, st);
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        ready.push_back(j);
      }
      cv_sched.notify_all();
    }
  }

  // enqueue the next slice of j and a copy of its device state after it
  avx_status launch_slice(Job* j) {
    const unsigned k1 = std::min(j->s->p.maxIt, (j->k / kSlice + 1) * kSlice);
    avx_status r = solver_enqueue(j->s, reinterpret_cast<const float2*>(j->r.d_b1), j->k, k1, &j->launches);
    if (r != AVX_OK) return r;
    const int q = (j->head + j->inflight) & 1;
    AVX_CK(cudaMemcpyAsync(j->hs[q], j->s->st.p, sizeof(DevState), cudaMemcpyDeviceToHost, j->stream));
    AVX_CK(cudaEventRecord(j->ev[q], j->stream));
    j->k = k1;
    ++j->inflight;
    return AVX_OK;
  }

  avx_status retire(Job* j) {
    avx_solver* s = j->s;
    AVX_CK(cudaMemcpyAsync(j->r.d_x, s->primc(0), (size_t)s->N() * sizeof(float2), cudaMemcpyDeviceToDevice,
                           j->stream));
    AVX_CK(cudaMemcpyAsync(&s->last, s->st.p, sizeof(DevState), cudaMemcpyDeviceToHost, j->stream));
    AVX_CK(cudaStreamSynchronize(j->stream));
    const float ms = (float)ms_since(j->t_start, std::chrono::steady_clock::now());
    const avx_status st = solver_finish_stats(s, ms, j->launches);
    j->c.stats = s->stats;
    return st;
  }

  void sched_loop() {
    cudaSetDevice(device);
    std::vector<Job*> active;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        while (!ready.empty() && (int)active.size() < max_active) {
          active.push_back(ready.front());
          ready.pop_front();
        }
        if (stop && active.empty()) break;
        if (active.empty()) {
          cv_sched.wait_for(lk, std::chrono::milliseconds(20));
          continue;
        }
      }
      bool progressed = false;
      for (size_t i = 0; i < active.size();) {
        Job* j = active[i];
        avx_status st = AVX_OK;
        bool finished = false;
        // completed slices: read the device state they left
        while (j->inflight > 0) {
          const cudaError_t q = cudaEventQuery(j->ev[j->head]);
          if (q == cudaErrorNotReady) break;
          if (q != cudaSuccess) {
            st = fail(AVX_E_CUDA, std::string("request slice failed: ") + cudaGetErrorString(q));
            finished = true;
            break;
          }
          const DevState& h = *j->hs[j->head];
          if (h.stop || h.err) j->stopped = true;
          j->head ^= 1;
          --j->inflight;
          progressed = true;
        }
        // keep two slices in flight until the run ends
        while (!finished && !j->stopped && j->inflight < 2 && j->k < j->s->p.maxIt) {
          st = launch_slice(j);
          if (st != AVX_OK) finished = true;
          progressed = true;
        }
        if (!finished && j->inflight == 0 && (j->stopped || j->k >= j->s->p.maxIt)) finished = true;
        if (finished) {
          const avx_status rs = retire(j);
          if (st == AVX_OK) st = rs;
          job_release(j);
          j->c.run_ms = ms_since(j->t_start, std::chrono::steady_clock::now());
          complete(j, st);
          active.erase(active.begin() + i);
          progressed = true;
          continue;
        }
        ++i;
      }
      if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  }
};

extern "C" {

avx_status avx_query_workspace(const avx_request* r, size_t* bytes) {
  if (!r || !bytes) return fail(AVX_E_ARG, "null argument");
  if (!method_ok(r->method)) return fail(AVX_E_UNSUPPORTED, "method not provided (TV, TVtemp, TGV2, ICTV, ICTGV2 are)");
  if (r->op_kind != 0 && r->op_kind != 1) return fail(AVX_E_ARG, "op_kind must be 0 (Cartesian) or 1 (radial)");
  if (!r->width || !r->height || !r->coils || !r->frames) return fail(AVX_E_ARG, "dimensions must be positive");
  if (r->op_kind == 1 && (!r->d_traj || !r->d_dens || !r->n_fe || !r->spokes_per_frame))
    return fail(AVX_E_ARG, "radial request needs trajectory, density and sample counts");
  *bytes = request_workspace(*r, -1, 0);
  return AVX_OK;
}

// The device's default memory pool keeps freed memory (release threshold
// unlimited) while at least one engine lives on the device; when the last one
// goes, the previous threshold comes back and the unused memory is returned,
// so that later synchronous allocations of the process find it free.
static avx_status pool_hold(int device, bool acquire) {
  static std::mutex mu;
  static std::map<int, int> held;  // device -> live engines
  std::lock_guard<std::mutex> lk(mu);
  int cur = 0;
  AVX_CK(cudaGetDevice(&cur));
  AVX_CK(cudaSetDevice(device));
  cudaMemPool_t pool = library_pool();
  cudaSetDevice(cur);
  if (!pool) return fail(AVX_E_CUDA, "cannot create the library's memory pool");
  int& h = held[device];
  if (acquire) {
    if (h++ == 0) {
      unsigned long long keep = ~0ull;
      AVX_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return AVX_OK;
  }
  if (h > 0 && --h == 0) {
    unsigned long long keep = kPoolKeep;
    AVX_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    AVX_CK(cudaMemPoolTrimTo(pool, kPoolKeep));
  }
  return AVX_OK;
}

avx_status avx_batch_create(int device, size_t hbm_budget, int workers, avx_batch** out) {
  if (!out || workers < 1 || hbm_budget == 0) return fail(AVX_E_ARG, "invalid batch engine arguments");
  int n = 0;
  AVX_CK(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(AVX_E_ARG, "no such CUDA device");
  AVX_CK(cudaSetDevice(device));
  avx_status r = configure_once();
  if (r != AVX_OK) return r;
  // keep freed pool memory for the next requests instead of returning it to
  // the driver while an engine lives on the device (pool_hold)
  r = pool_hold(device, true);
  if (r != AVX_OK) return r;
  avx_batch* b = new avx_batch();
  b->device = device;
  b->budget = hbm_budget;
  b->max_active = workers;
  const int slots = workers + kSetupThreads;
  avx_status st = AVX_OK;
  for (int i = 0; i < slots && st == AVX_OK; ++i) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      st = fail(AVX_E_CUDA, "cannot create the engine's streams");
      break;
    }
    b->streams.push_back(s);
    b->free_slots.push_back(slots - 1 - i);
    for (int q = 0; q < 2; ++q) {
      cudaEvent_t e;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) st = fail(AVX_E_CUDA, "cannot create events");
      else b->events.push_back(e);
    }
  }
  if (st == AVX_OK && cudaMallocHost(reinterpret_cast<void**>(&b->h_states), sizeof(DevState) * 2 * slots) != cudaSuccess)
    st = fail(AVX_E_NOMEM, "cannot allocate pinned state slots");
  if (st != AVX_OK) {
    for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    delete b;
    pool_hold(device, false);
    return st;
  }
  memset(b->h_states, 0, sizeof(DevState) * 2 * slots);
  for (int i = 0; i < kSetupThreads; ++i) b->setup_threads.emplace_back([b] { b->setup_loop(); });
  b->sched = std::thread([b] { b->sched_loop(); });
  *out = b;
  return AVX_OK;
}

avx_status avx_batch_submit(avx_batch* b, const avx_request* r) {
  if (!b || !r) return fail(AVX_E_ARG, "null argument");
  if (!r->d_data || !r->d_x || !r->d_b1) return fail(AVX_E_ARG, "request without data, image or coil maps");
  size_t ws = 0;
  avx_status st = avx_query_workspace(r, &ws);
  if (st != AVX_OK) return st;
  if (ws > b->budget) return fail(AVX_E_NOMEM, "request workspace exceeds the engine's HBM budget");
  {
    std::lock_guard<std::mutex> lk(b->mu);
    b->queue.push_back({*r, ws, std::chrono::steady_clock::now()});
    ++b->pending;
  }
  b->cv_setup.notify_all();
  return AVX_OK;
}

avx_status avx_serve_poll(avx_batch* b, avx_completion* out, int max, int* n, int wait_ms) {
  if (!b || !n || (max > 0 && !out)) return fail(AVX_E_ARG, "null argument");
  std::unique_lock<std::mutex> lk(b->mu);
  auto ready = [&] { return !b->done.empty() || b->pending == 0; };
  if (wait_ms < 0)
    b->cv_done.wait(lk, ready);
  else if (wait_ms > 0)
    b->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  int k = 0;
  while (k < max && !b->done.empty()) {
    out[k++] = b->done.front();
    b->done.pop_front();
    --b->pending;
  }
  *n = k;
  return AVX_OK;
}

avx_status avx_batch_drain(avx_batch* b) {
  if (!b) return fail(AVX_E_ARG, "null engine");
  std::unique_lock<std::mutex> lk(b->mu);
  b->cv_done.wait(lk, [&] { return b->queue.empty() && b->admitted == 0; });
  return AVX_OK;
}

int avx_batch_pending(const avx_batch* b) {
  if (!b) return 0;
  std::lock_guard<std::mutex> lk(const_cast<avx_batch*>(b)->mu);
  return b->pending;
}

void avx_batch_destroy(avx_batch* b) {
  if (!b) return;
  {
    // queued requests are dropped; admitted ones run to their end
    std::unique_lock<std::mutex> lk(b->mu);
    b->queue.clear();
    b->cv_done.wait(lk, [&] { return b->admitted == 0; });
    b->stop = true;
  }
  b->cv_setup.notify_all();
  b->cv_sched.notify_all();
  for (std::thread& t : b->setup_threads) t.join();
  b->sched.join();
  for (cudaStream_t s : b->streams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : b->events) cudaEventDestroy(e);
  cudaFreeHost(b->h_states);
  const int dev = b->device;
  delete b;
  pool_hold(dev, false);
}

}  // extern "C"
