// avionic: command-line reconstruction of Cartesian 2D+t multi-coil data.
//
// Drop-in for the reference executable's Cartesian TV / TGV2 / ICTGV2 path
// (CUDA/src/main.cpp:323-917): same flags, configuration keys, .bin inputs
// and outputs, and export file names.  Sequence: parse options and the
// configuration file, load k-space and mask, zero the data outside the mask
// (main.cpp:507-519), load b1 (-s) and u0 (-u) or form u0 as the coil-combined
// time average, replicate u0 over the frames (main.cpp:775-779), run the
// method, write the image, and with -e write x3_component, PDGap, ICTGVnorm
// and DATAfidelity next to the output (main.cpp:915-917).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "avionic.h"
#include "binio.h"
#include "config.h"

using cd = std::complex<double>;
using cf = std::complex<float>;

namespace {

int die(const std::string& msg) {
  std::cerr << "avionic: " << msg << std::endl;
  return -1;
}

std::string exe_dir(const char* argv0) {
  std::string p = argv0;
  const size_t s = p.find_last_of('/');
  return s == std::string::npos ? "." : p.substr(0, s);
}

struct Dev {
  void* p = nullptr;
  ~Dev() {
    if (p) cudaFree(p);
  }
};

void export_cb(const char* dir, const char* name, const avx_cf32* v, size_t n, void*) {
  std::vector<cd> out(n);
  for (size_t i = 0; i < n; ++i) out[i] = cd(v[i].re, v[i].im);
  std::string err;
  const std::string path = std::string(dir) + "/" + name;
  if (!avcli::write_bin(path, out, true, &err))
    std::cerr << "avionic: " << err << std::endl;
  else
    std::cout << "exported " << path << std::endl;
}

// Cartesian time-averaged coil-combined initial image:
// u0 = sum_c conj(b1_c) F^-1( sum_t k_{t,c} / max(1, sum_t mask_t) )
// (cartesian_coil_construction.cpp:23-86 forms the same average per coil).
std::vector<cf> time_average_u0(const std::vector<cf>& k, const std::vector<float>& mask, const std::vector<cf>& b1,
                                unsigned W, unsigned H, unsigned C, unsigned T) {
  const size_t HW = (size_t)W * H;
  std::vector<double> cnt(HW, 0.0);
  for (unsigned t = 0; t < T; ++t)
    for (size_t i = 0; i < HW; ++i) cnt[i] += mask[t * HW + i];
  std::vector<cf> u(HW, cf(0, 0));
  std::vector<cd> avg(HW), tmp(HW);
  for (unsigned c = 0; c < C; ++c) {
    std::fill(avg.begin(), avg.end(), cd(0, 0));
    for (unsigned t = 0; t < T; ++t)
      for (size_t i = 0; i < HW; ++i) avg[i] += cd(k[((size_t)t * C + c) * HW + i]);
    for (size_t i = 0; i < HW; ++i) avg[i] /= std::max(1.0, cnt[i]);
    // unitary k-space -> image transform (e^{-2 pi i} kernel), separable DFT
    for (unsigned y = 0; y < H; ++y)
      for (unsigned x = 0; x < W; ++x) {
        cd s(0, 0);
        for (unsigned kx = 0; kx < W; ++kx)
          s += avg[(size_t)y * W + kx] * std::polar(1.0, -2.0 * M_PI * ((double)kx * x / W));
        tmp[(size_t)y * W + x] = s / std::sqrt((double)W);
      }
    for (unsigned x = 0; x < W; ++x)
      for (unsigned y = 0; y < H; ++y) {
        cd s(0, 0);
        for (unsigned ky = 0; ky < H; ++ky)
          s += tmp[(size_t)ky * W + x] * std::polar(1.0, -2.0 * M_PI * ((double)ky * y / H));
        s /= std::sqrt((double)H);
        u[(size_t)y * W + x] += cf(std::conj(cd(b1[c * HW + (size_t)y * W + x])) * s);
      }
  }
  return u;
}

}  // namespace

int main(int argc, char** argv) {
  const auto t_start = std::chrono::steady_clock::now();
  avcli::Options o;
  std::string err;
  if (!avcli::parse_command_line(argc, argv, o, err)) {
    std::cerr << "avionic: " << err << std::endl;
    avcli::print_usage();
    return -1;
  }
  const bool raw_ok = o.rawdata && !o.positional.empty();
  if (o.help || !((o.have_dims && o.positional.size() >= 3) || raw_ok)) {
    avcli::print_usage();
    return -1;
  }
  if (o.rawdata) return die("raw data import (-r) is not provided by this build; convert to .bin first");
  if (o.params_file.empty()) o.params_file = exe_dir(argv[0]) + "/config/default.cfg";
  bool found = false;
  if (!avcli::parse_config_file(o.params_file, o, err, &found)) return die(err);
  if (found)
    std::cout << "Parsing configuration file: " << o.params_file << std::endl;
  else
    std::cout << "Warning: no configuration file found in " << o.params_file << "\n         using default parameters... "
              << std::endl;
  const std::string mname = o.conf.count("method") ? o.conf["method"] : "ICTGV2";
  const int method = avcli::method_from_name(mname);
  if (method < 0) return die("invalid method selected");
  if (method != AVX_METHOD_TV && method != AVX_METHOD_TGV2 && method != AVX_METHOD_ICTGV2)
    return die("method " + mname + " is not provided by this build (TV, TGV2, ICTGV2 are)");
  if (o.nonuniform) return die("nonuniform (-n) data is not provided by this build");
  if (o.normalize) return die("data normalisation (-o) is not provided by this build");
  avx_pd_params p;
  if (!avcli::params_for_method(o, method, &p, err)) return die(err);

  const unsigned W = o.dims[0], H = o.dims[1], C = o.dims[6], T = o.dims[7];
  const size_t HW = (size_t)W * H, N = HW * T, K = N * C;
  const std::string kfile = o.positional[0], mfile = o.positional[1], outfile = o.positional[2];
  const std::string outdir = avcli::parent_directory(outfile);
  if (o.gpu >= 0 && cudaSetDevice(o.gpu) != cudaSuccess) return die("cannot select GPU " + std::to_string(o.gpu));

  std::vector<cd> buf;
  bool cplx = false;
  if (avcli::file_extension(kfile) != ".bin") return die("k-space data must be a .bin vector file");
  if (!avcli::read_bin(kfile, buf, &cplx, &err)) return die(err);
  if (buf.size() != K) return die("k-space data holds " + std::to_string(buf.size()) + " values, dims require " +
                                  std::to_string(K));
  std::cout << "Data File " << kfile << " successfully loaded." << std::endl;
  std::vector<cf> kdata(K);
  for (size_t i = 0; i < K; ++i) kdata[i] = cf(buf[i]);
  if (!avcli::read_bin(mfile, buf, &cplx, &err)) return die(err);
  if (buf.size() != N) return die("mask holds " + std::to_string(buf.size()) + " values, dims require " + std::to_string(N));
  std::cout << "Mask File " << mfile << " successfully loaded." << std::endl;
  std::vector<float> mask(N);
  for (size_t i = 0; i < N; ++i) mask[i] = (float)buf[i].real();
  // zero the data outside the mask, per frame and coil (main.cpp:507-519)
  for (unsigned t = 0; t < T; ++t)
    for (unsigned c = 0; c < C; ++c)
      for (size_t i = 0; i < HW; ++i) kdata[((size_t)t * C + c) * HW + i] *= mask[t * HW + i];

  std::vector<cf> b1(HW * C, cf(1, 0)), u0(HW, cf(0, 0));
  if (o.sens.empty()) return die("coil construction (no -s) is not provided by this build; pass -s b1.bin");
  if (!avcli::read_bin(o.sens, buf, &cplx, &err)) return die(err);
  if (buf.size() != HW * C) return die("coil sensitivities hold " + std::to_string(buf.size()) + " values");
  for (size_t i = 0; i < HW * C; ++i) b1[i] = cf(buf[i]);
  std::cout << "B1 File " << o.sens << " successfully loaded." << std::endl;
  if (!o.u0.empty() && avcli::read_bin(o.u0, buf, &cplx, &err) && buf.size() == HW) {
    for (size_t i = 0; i < HW; ++i) u0[i] = cf(buf[i]);
    std::cout << " initial solution (u0) file " << o.u0 << " successfully loaded." << std::endl;
  } else {
    std::cout << "no initial solution (u0) data provided! using the coil-combined time average" << std::endl;
    u0 = time_average_u0(kdata, mask, b1, W, H, C, T);
  }

  Dev dk, dm, db, dx;
  if (cudaMalloc(&dk.p, K * sizeof(cf)) != cudaSuccess || cudaMalloc(&dm.p, N * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&db.p, HW * C * sizeof(cf)) != cudaSuccess || cudaMalloc(&dx.p, N * sizeof(cf)) != cudaSuccess)
    return die("device allocation failed");
  cudaMemcpy(dk.p, kdata.data(), K * sizeof(cf), cudaMemcpyHostToDevice);
  cudaMemcpy(dm.p, mask.data(), N * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(db.p, b1.data(), HW * C * sizeof(cf), cudaMemcpyHostToDevice);
  for (unsigned t = 0; t < T; ++t)
    cudaMemcpy((cf*)dx.p + t * HW, u0.data(), HW * sizeof(cf), cudaMemcpyHostToDevice);

  avx_operator* op = nullptr;
  if (avx_cartesian_operator_create(W, H, C, T, (const float*)dm.p, 0, &op) != AVX_OK) return die(avx_last_error());
  avx_solver* s = nullptr;
  if (avx_solver_create(method, W, H, C, T, &p, op, &s) != AVX_OK) return die(avx_last_error());
  avx_pd_params q;
  avx_solver_get_params(s, &q);
  if (p.adaptLambda)
    std::cout << "Adapted lambda with (k,d) (" << p.adaptK << ", " << p.adaptD << ") to " << q.lambda << std::endl;
  else
    std::cout << "Using lambda: " << q.lambda << std::endl;
  avx_solver_set_verbose(s, o.verbose);
  avx_solver_set_debug(s, o.debugstep > 0, o.debugstep);
  const auto t_init = std::chrono::steady_clock::now();
  std::cout << "Initialization time: " << std::chrono::duration<double>(t_init - t_start).count() << "s" << std::endl;
  if (avx_solver_run(s, (const avx_cf32*)dk.p, (avx_cf32*)dx.p, (const avx_cf32*)db.p) != AVX_OK)
    return die(avx_last_error());
  avx_run_stats st;
  avx_solver_get_stats(s, &st);
  const auto t_run = std::chrono::steady_clock::now();
  std::cout << "Execution time: " << std::chrono::duration<double>(t_run - t_init).count() << "s (" << st.iterations
            << " iterations, " << st.elapsed_ms << " ms on the device)" << std::endl;

  std::vector<cf> x(N);
  cudaMemcpy(x.data(), dx.p, N * sizeof(cf), cudaMemcpyDeviceToHost);
  std::vector<cd> xo(N);
  for (size_t i = 0; i < N; ++i) xo[i] = cd(x[i]);
  const std::string ext = avcli::file_extension(outfile);
  if (ext == ".h5") return die("HDF5 output is not provided by this build; use .bin");
  std::cout << "writing output file to: " << outfile << std::endl;
  if (!avcli::write_bin(outfile, xo, true, &err)) return die(err);
  if (o.extradata && avx_solver_export(s, outdir.c_str(), export_cb, nullptr) != AVX_OK) return die(avx_last_error());
  avx_solver_destroy(s);
  avx_operator_destroy(op);
  return 0;
}
