// avionic: command-line reconstruction of Cartesian and radial 2D+t multi-coil data.
//
// Drop-in for the reference executable's Cartesian TV / TGV2 / ICTGV2 path
// (CUDA/src/main.cpp:323-917): same flags, configuration keys, .bin inputs
// and outputs, and export file names.  Sequence: parse options and the
// configuration file, load k-space and mask, zero the data outside the mask
// (main.cpp:507-519), load b1 (-s) and u0 (-u) or form u0 as the coil-combined
// time average, replicate u0 over the frames (main.cpp:775-779), run the
// method, write the image, and with -e write x3_component, PDGap, ICTGVnorm
// and DATAfidelity next to the output (main.cpp:915-917).  With -o the
// k-space is normalised first (main.cpp:573-579) and the factor is written
// to datanorm_factor.bin (main.cpp:793-796).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <random>
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

// u0 = 0.5 sum_c conj(b1_c) crec_c from the time-averaged reconstruction
// without phase (PerformInitalizationGivenB1, main.cpp:250-289)
std::vector<cf> given_b1_u0(const std::vector<cf>& crec, const std::vector<cf>& b1, size_t HW, unsigned C) {
  std::vector<cf> u(HW, cf(0, 0));
  for (unsigned c = 0; c < C; ++c)
    for (size_t i = 0; i < HW; ++i) u[i] += std::conj(b1[c * HW + i]) * crec[c * HW + i];
  for (auto& v : u) v *= 0.5f;
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
  if (method != AVX_METHOD_TV && method != AVX_METHOD_TVTEMP && method != AVX_METHOD_TGV2 &&
      method != AVX_METHOD_ICTV && method != AVX_METHOD_ICTGV2)
    return die("method " + mname + " is not provided by this build (TV, TVTEMP, TGV2, ICTV, ICTGV2 are)");
  avx_pd_params p;
  if (!avcli::params_for_method(o, method, &p, err)) return die(err);

  const unsigned W = o.dims[0], H = o.dims[1], C = o.dims[6], T = o.dims[7];
  const size_t HW = (size_t)W * H, N = HW * T;
  const std::string kfile = o.positional[0], mfile = o.positional[1], outfile = o.positional[2];
  const std::string outdir = avcli::parent_directory(outfile);
  if (o.gpu >= 0 && cudaSetDevice(o.gpu) != cudaSuccess) return die("cannot select GPU " + std::to_string(o.gpu));

  std::vector<cd> buf;
  bool cplx = false;
  const unsigned nRO = o.dims[3], spf = o.dims[4];
  const size_t S = (size_t)nRO * spf;                  // radial samples per frame
  const size_t K = o.nonuniform ? S * C * T : N * C;   // k-space values
  if (avcli::file_extension(kfile) != ".bin") return die("k-space data must be a .bin vector file");
  if (!avcli::read_bin(kfile, buf, &cplx, &err)) return die(err);
  if (buf.size() != K) return die("k-space data holds " + std::to_string(buf.size()) + " values, dims require " +
                                  std::to_string(K));
  std::cout << "Data File " << kfile << " successfully loaded." << std::endl;
  std::vector<cf> kdata(K);
  for (size_t i = 0; i < K; ++i) kdata[i] = cf(buf[i]);
  if (!avcli::read_bin(mfile, buf, &cplx, &err)) return die(err);
  const size_t MN = o.nonuniform ? 2 * S * T : N;
  if (buf.size() != MN)
    return die(std::string(o.nonuniform ? "trajectory" : "mask") + " holds " + std::to_string(buf.size()) +
               " values, dims require " + std::to_string(MN));
  std::cout << (o.nonuniform ? "Trajectory" : "Mask") << " File " << mfile << " successfully loaded." << std::endl;
  std::vector<float> mask(MN);
  for (size_t i = 0; i < MN; ++i) mask[i] = (float)buf[i].real();
  std::vector<float> dens;
  if (o.nonuniform) {
    if (o.dens.empty()) return die("Density compensation data could not be loaded!");
    if (!avcli::read_bin(o.dens, buf, &cplx, &err)) return die(err);
    if (buf.size() != S * T) return die("density compensation holds " + std::to_string(buf.size()) + " values");
    dens.resize(S * T);
    for (size_t i = 0; i < S * T; ++i) dens[i] = (float)buf[i].real();
    // data *= sqrt(w) per frame and sample (main.cpp:546-570; the operator applies sqrt(w) itself)
    for (unsigned t = 0; t < T; ++t)
      for (unsigned c = 0; c < C; ++c)
        for (size_t j = 0; j < S; ++j) kdata[((size_t)t * C + c) * S + j] *= std::sqrt(dens[(size_t)t * S + j]);
  } else {
    // zero the data outside the mask, per frame and coil (main.cpp:507-519)
    for (unsigned t = 0; t < T; ++t)
      for (unsigned c = 0; c < C; ++c)
        for (size_t i = 0; i < HW; ++i) kdata[((size_t)t * C + c) * HW + i] *= mask[t * HW + i];
  }

  Dev dk, dm, db, dx, dd, du, dc;
  if (cudaMalloc(&dk.p, K * sizeof(cf)) != cudaSuccess || cudaMalloc(&dm.p, MN * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&db.p, HW * C * sizeof(cf)) != cudaSuccess || cudaMalloc(&dx.p, N * sizeof(cf)) != cudaSuccess ||
      cudaMalloc(&du.p, HW * C * sizeof(cf)) != cudaSuccess || cudaMalloc(&dc.p, HW * C * sizeof(cf)) != cudaSuccess)
    return die("device allocation failed");
  cudaMemcpy(dk.p, kdata.data(), K * sizeof(cf), cudaMemcpyHostToDevice);
  cudaMemcpy(dm.p, mask.data(), MN * sizeof(float), cudaMemcpyHostToDevice);
  if (o.nonuniform) {
    if (cudaMalloc(&dd.p, S * T * sizeof(float)) != cudaSuccess) return die("device allocation failed");
    cudaMemcpy(dd.p, dens.data(), S * T * sizeof(float), cudaMemcpyHostToDevice);
  }

  // data normalisation (-o) before the coil maps and u0 (main.cpp:573-579)
  float datanorm = 1.f;
  if (o.normalize) {
    std::cout << "Normalize binary data." << std::endl;
    if (avx_normalize_data(W, H, C, T, o.nonuniform ? (unsigned)S : 0u, (const float*)dm.p, (const float*)dd.p,
                           (avx_cf32*)dk.p, &datanorm) != AVX_OK)
      return die(avx_last_error());
    std::cout << "datanorm factor (in):" << datanorm << std::endl;
  }

  std::vector<cf> b1(HW * C, cf(1, 0)), u0(HW, cf(0, 0));
  avx_coil_params cp;
  avx_coil_default_params(&cp);
  auto cfv = [&](const char* k, float def) { return o.conf.count(k) ? std::stof(o.conf[k]) : def; };
  cp.uH1mu = cfv("coil.uH1mu", cp.uH1mu);
  cp.uReg = cfv("coil.uReg", cp.uReg);
  cp.uNrIt = (unsigned)cfv("coil.uNrIt", (float)cp.uNrIt);
  cp.uTau = cfv("coil.uTau", cp.uTau);
  cp.uSigma = cfv("coil.uSigma", cp.uSigma);
  cp.uAlpha0 = cfv("coil.uAlpha0", cp.uAlpha0);
  cp.uAlpha1 = cfv("coil.uAlpha1", cp.uAlpha1);
  cp.b1Reg = cfv("coil.b1Reg", cp.b1Reg);
  cp.b1NrIt = (unsigned)cfv("coil.b1NrIt", (float)cp.b1NrIt);
  cp.b1Tau = cfv("coil.b1Tau", cp.b1Tau);
  cp.b1Sigma = cfv("coil.b1Sigma", cp.b1Sigma);
  cp.b1FinalReg = cfv("coil.b1FinalReg", cp.b1FinalReg);
  cp.b1FinalNrIt = (unsigned)cfv("coil.b1FinalNrIt", (float)cp.b1FinalNrIt);
  if (!o.sens.empty() && avcli::read_bin(o.sens, buf, &cplx, &err)) {
    if (buf.size() != HW * C) return die("coil sensitivities hold " + std::to_string(buf.size()) + " values");
    for (size_t i = 0; i < HW * C; ++i) b1[i] = cf(buf[i]);
    std::cout << "B1 File " << o.sens << " successfully loaded." << std::endl;
    if (!o.u0.empty() && avcli::read_bin(o.u0, buf, &cplx, &err) && buf.size() == HW) {
      for (size_t i = 0; i < HW; ++i) u0[i] = cf(buf[i]);
      std::cout << " initial solution (u0) file " << o.u0 << " successfully loaded." << std::endl;
    } else {
      std::cout << "no initial solution (u0) data provided!" << std::endl;
      Dev tu;
      cudaMalloc(&tu.p, HW * sizeof(cf));
      const avx_status st =
          o.nonuniform ? avx_coil_time_averaged_radial(W, H, C, T, (unsigned)S, (const float*)dm.p, (const float*)dd.p,
                                                       (const avx_cf32*)dk.p, (avx_cf32*)tu.p, (avx_cf32*)dc.p, 0)
                       : avx_coil_time_averaged(W, H, C, T, (const avx_cf32*)dk.p, (const float*)dm.p,
                                                (avx_cf32*)tu.p, (avx_cf32*)dc.p, 0);
      if (st != AVX_OK) return die(avx_last_error());
      std::vector<cf> crec(HW * C);
      cudaMemcpy(crec.data(), dc.p, HW * C * sizeof(cf), cudaMemcpyDeviceToHost);
      u0 = given_b1_u0(crec, b1, HW, C);
    }
  } else {
    std::cout << "Performing Coil Construction!" << std::endl;
    const avx_status st =
        o.nonuniform ? avx_coil_construction_radial(W, H, C, T, (unsigned)S, &cp, (const float*)dm.p,
                                                    (const float*)dd.p, (const avx_cf32*)dk.p, (avx_cf32*)du.p,
                                                    (avx_cf32*)db.p)
                     : avx_coil_construction(W, H, C, T, &cp, (const avx_cf32*)dk.p, (const float*)dm.p,
                                             (avx_cf32*)du.p, (avx_cf32*)db.p);
    if (st != AVX_OK) return die(avx_last_error());
    cudaMemcpy(b1.data(), db.p, HW * C * sizeof(cf), cudaMemcpyDeviceToHost);
    cudaMemcpy(u0.data(), (cf*)du.p + (size_t)(C - 1) * HW, HW * sizeof(cf), cudaMemcpyDeviceToHost);
    if (o.nonuniform)
      for (auto& v : u0) v /= (float)T;  // main.cpp:636-640
    std::vector<cd> e(HW);
    for (size_t i = 0; i < HW; ++i) e[i] = cd(u0[i]);
    avcli::write_bin(outdir + "/u0_reconstructed.bin", e, true, &err);
    e.resize(HW * C);
    for (size_t i = 0; i < HW * C; ++i) e[i] = cd(b1[i]);
    avcli::write_bin(outdir + "/b1_reconstructed.bin", e, true, &err);
  }
  cudaMemcpy(db.p, b1.data(), HW * C * sizeof(cf), cudaMemcpyHostToDevice);
  for (unsigned t = 0; t < T; ++t)
    cudaMemcpy((cf*)dx.p + t * HW, u0.data(), HW * sizeof(cf), cudaMemcpyHostToDevice);

  avx_operator* op = nullptr;
  if (o.nonuniform) {
    const float kw = o.conf.count("gpunufft.kernelWidth") ? std::stof(o.conf["gpunufft.kernelWidth"]) : 3.f;
    const float sw = o.conf.count("gpunufft.sectorWidth") ? std::stof(o.conf["gpunufft.sectorWidth"]) : 8.f;
    const float osf = o.conf.count("gpunufft.osf") ? std::stof(o.conf["gpunufft.osf"]) : 2.f;
    std::cout << "Init NonCartesian Operator using kernelWidth:" << kw << " sectorWidth:" << sw << " OSF:" << osf
              << std::endl;
    if (avx_radial_operator_create(W, H, C, T, spf * T, nRO, spf, (const float*)dm.p, (const float*)dd.p, kw, sw,
                                   osf, &op) != AVX_OK)
      return die(avx_last_error());
  } else if (avx_cartesian_operator_create(W, H, C, T, (const float*)dm.p, 0, &op) != AVX_OK) {
    return die(avx_last_error());
  }
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
  if (o.opnorm_steps) {
    // getopnorm (matlab/getopnorm.m) from a seeded Gaussian image, as the
    // reference starts it from randn
    std::mt19937 gen(0);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<cf> r(N);
    for (auto& v : r) v = cf(nd(gen), nd(gen));
    Dev dr;
    if (cudaMalloc(&dr.p, N * sizeof(cf)) != cudaSuccess) return die("cudaMalloc failed");
    cudaMemcpy(dr.p, r.data(), N * sizeof(cf), cudaMemcpyHostToDevice);
    double l = 0.0;
    if (avx_solver_opnorm(s, (const avx_cf32*)dr.p, (const avx_cf32*)db.p, o.opnorm_steps, 1, &l, nullptr) != AVX_OK)
      return die(avx_last_error());
    avx_solver_get_params(s, &q);
    std::cout << "Operator norm estimate ||K||^2: " << l << " -> sigma " << q.sigma << ", tau " << q.tau
              << std::endl;
  }
  const auto t_init = std::chrono::steady_clock::now();
  std::cout << "Initialization time: " << std::chrono::duration<double>(t_init - t_start).count() << "s" << std::endl;
  if (avx_solver_run(s, (const avx_cf32*)dk.p, (avx_cf32*)dx.p, (const avx_cf32*)db.p) != AVX_OK)
    return die(avx_last_error());
  avx_run_stats st;
  avx_solver_get_stats(s, &st);
  if (o.normalize) {  // main.cpp:793-796
    const std::vector<cd> dn{cd(datanorm, 0.0)};
    if (!avcli::write_bin(outdir + "/datanorm_factor.bin", dn, true, &err)) return die(err);
  }
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
