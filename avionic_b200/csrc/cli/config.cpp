#include "config.h"

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <set>
#include <sstream>

namespace avcli {

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// Every key the reference's parser declares (options_parser.cpp:128-324).
const std::set<std::string>& known_keys() {
  static const std::set<std::string> k = [] {
    std::set<std::string> s = {"method", "maxIt", "stopPDGap"};
    auto add = [&](const std::string& sec, std::initializer_list<const char*> keys) {
      for (auto* key : keys) s.insert(sec + "." + key);
    };
    add("coil", {"uH1mu", "uReg", "uNrIt", "uTau", "uSigma", "uSigmaTauRatio", "uAlpha0", "uAlpha1", "b1Reg",
                 "b1NrIt", "b1Tau", "b1Sigma", "b1SigmaTauRatio", "b1FinalReg", "b1FinalNrIt"});
    add("tv", {"dx", "dy", "dt", "sigma", "tau", "sigmaTauRatio", "timeSpaceWeight", "lambda"});
    add("tvtemp", {"dt", "sigma", "tau", "sigmaTauRatio", "lambda"});
    add("tgv2", {"dx", "dy", "dt", "sigma", "tau", "sigmaTauRatio", "timeSpaceWeight", "lambda", "alpha0", "alpha1"});
    add("tgv2_3D", {"dx", "dy", "dz", "sigma", "tau", "sigmaTauRatio", "lambda", "alpha0", "alpha1"});
    add("ictv", {"dx", "dy", "dt", "sigma", "tau", "sigmaTauRatio", "timeSpaceWeight", "lambda", "alpha1", "alpha",
                 "timeSpaceWeight2", "dx2", "dy2", "dt2"});
    add("ictgv2", {"dx", "dy", "dt", "sigma", "tau", "sigmaTauRatio", "timeSpaceWeight", "lambda", "alpha0",
                   "alpha1", "alpha", "timeSpaceWeight2", "dx2", "dy2", "dt2"});
    add("asltgv2recon4D", {"dx", "dy", "dz", "dt", "sigma", "tau", "sigmaTauRatio", "timeSpaceWeight", "lambda_l",
                           "lambda_c", "alpha0", "alpha1", "alpha"});
    add("gpunufft", {"kernelWidth", "sectorWidth", "osf"});
    add("h1", {"mu", "relTol", "absTol", "maxIt"});
    add("adaptlambda", {"k", "d"});
    return s;
  }();
  return k;
}

// short flag -> long name, and whether it takes a value
struct Flag {
  const char* name;
  bool value;
};
const std::map<char, Flag>& short_flags() {
  static const std::map<char, Flag> f = {
      {'h', {"help", false}},      {'g', {"debugstep", true}},  {'v', {"verbose", false}},
      {'d', {"dims", true}},       {'n', {"nonuniform", false}}, {'o', {"normalize", false}},
      {'e', {"extradata", false}}, {'a', {"adaptlambda", false}}, {'w', {"dens", true}},
      {'p', {"params", true}},     {'s', {"sens", true}},       {'u', {"uzero", true}},
      {'l', {"labeldata", true}},  {'r', {"rawdata", false}},   {'f', {"forceOSRemoval", false}},
      {'t', {"tpat", true}},       {'z', {"slice", true}},      {'b', {"gpudevice", true}},
      {'q', {"dataBS", true}},     {'x', {"maskBS", true}},     {'y', {"finalOutBS", true}},
      {'m', {"method", true}},     {'i', {"maxIt", true}},      {'j', {"stopPDGap", true}},
  };
  return f;
}

bool long_takes_value(const std::string& n) {
  if (n == "opnormSteps") return true;
  for (auto& kv : short_flags())
    if (n == kv.second.name) return kv.second.value;
  return known_keys().count(n) > 0;
}

bool set_option(Options& o, const std::string& name, const std::string& val, std::string& err) {
  try {
    if (name == "help") o.help = true;
    else if (name == "debugstep") o.debugstep = std::stoi(val);
    else if (name == "verbose") o.verbose = true;
    else if (name == "nonuniform") o.nonuniform = true;
    else if (name == "normalize") o.normalize = true;
    else if (name == "extradata") o.extradata = true;
    else if (name == "adaptlambda") o.adaptlambda = true;
    else if (name == "rawdata") o.rawdata = true;
    else if (name == "forceOSRemoval") o.force_os_removal = true;
    else if (name == "dens") o.dens = val;
    else if (name == "params") o.params_file = val;
    else if (name == "sens") o.sens = val;
    else if (name == "uzero") o.u0 = val;
    else if (name == "labeldata") o.labeldata = val;
    else if (name == "tpat") o.tpat = std::stoi(val);
    else if (name == "opnormSteps") o.opnorm_steps = (unsigned)std::stoul(val);
    else if (name == "slice") o.slice = (unsigned)std::stoul(val);
    else if (name == "gpudevice") o.gpu = std::stoi(val);
    else if (name == "dataBS") o.data_bs = val;
    else if (name == "maskBS") o.mask_bs = val;
    else if (name == "finalOutBS") o.final_bs = val;
    else if (name == "dims") {
      // w:h:d:nRO:nEnc1:nEnc2:coils:frames (options_parser.cpp:50-74)
      std::stringstream ss(val);
      std::string tok;
      int i = 0;
      while (std::getline(ss, tok, ':')) {
        if (i >= 8 || tok.empty() || !std::isdigit((unsigned char)tok[0])) {
          err = "invalid dimensions";
          return false;
        }
        o.dims[i++] = (unsigned)std::stoul(tok);
      }
      if (i != 8) {
        err = "invalid dimensions";
        return false;
      }
      o.have_dims = true;
    } else if (known_keys().count(name)) {
      if (!o.conf.count(name)) o.conf[name] = val;  // first stored value wins
    } else {
      err = "unrecognised option '" + name + "'";
      return false;
    }
  } catch (const std::exception&) {
    err = "invalid value '" + val + "' for option '" + name + "'";
    return false;
  }
  return true;
}

float conf_f(const Options& o, const std::string& key, float def) {
  auto it = o.conf.find(key);
  return it == o.conf.end() ? def : std::strtof(it->second.c_str(), nullptr);
}

}  // namespace

bool parse_command_line(int argc, char** argv, Options& o, std::string& err) {
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a.size() > 2 && a[0] == '-' && a[1] == '-') {
      std::string name = a.substr(2), val;
      const size_t eq = name.find('=');
      if (eq != std::string::npos) {
        val = name.substr(eq + 1);
        name = name.substr(0, eq);
      } else if (long_takes_value(name)) {
        if (i + 1 >= argc) {
          err = "missing value for --" + name;
          return false;
        }
        val = argv[++i];
      }
      if (!set_option(o, name, val, err)) return false;
    } else if (a.size() >= 2 && a[0] == '-' && !std::isdigit((unsigned char)a[1])) {
      // one or more short flags; the last may take a value
      for (size_t j = 1; j < a.size(); ++j) {
        auto it = short_flags().find(a[j]);
        if (it == short_flags().end()) {
          err = std::string("unrecognised option '-") + a[j] + "'";
          return false;
        }
        std::string val;
        if (it->second.value) {
          if (j + 1 < a.size())
            val = a.substr(j + 1);
          else if (i + 1 < argc)
            val = argv[++i];
          else {
            err = std::string("missing value for -") + a[j];
            return false;
          }
          if (!set_option(o, it->second.name, val, err)) return false;
          break;
        }
        if (!set_option(o, it->second.name, val, err)) return false;
      }
    } else {
      o.positional.push_back(a);
    }
  }
  return true;
}

bool parse_config_file(const std::string& path, Options& o, std::string& err, bool* found) {
  std::ifstream in(path);
  *found = (bool)in;
  if (!in) return true;
  std::string line, section;
  int ln = 0;
  while (std::getline(in, line)) {
    ++ln;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    if (line.front() == '[') {
      if (line.back() != ']') {
        err = path + ":" + std::to_string(ln) + ": malformed section header";
        return false;
      }
      section = trim(line.substr(1, line.size() - 2));
      continue;
    }
    const size_t eq = line.find('=');
    if (eq == std::string::npos) {
      err = path + ":" + std::to_string(ln) + ": expected key = value";
      return false;
    }
    const std::string key = trim(line.substr(0, eq));
    const std::string val = trim(line.substr(eq + 1));
    const std::string full = section.empty() ? key : section + "." + key;
    if (!known_keys().count(full)) {
      err = path + ":" + std::to_string(ln) + ": unrecognised option '" + full + "'";
      return false;
    }
    if (!o.conf.count(full)) o.conf[full] = val;
  }
  return true;
}

int method_from_name(const std::string& name) {
  const std::string u = upper(trim(name));
  if (u == "TV") return AVX_METHOD_TV;
  if (u == "TVTEMP") return AVX_METHOD_TVTEMP;
  if (u == "TGV2") return AVX_METHOD_TGV2;
  if (u == "TGV2_3D") return AVX_METHOD_TGV2_3D;
  if (u == "ICTV") return AVX_METHOD_ICTV;
  if (u == "ICTGV2") return AVX_METHOD_ICTGV2;
  if (u == "BS_RECON") return 6;
  if (u == "ASLTGV2RECON4D") return 7;
  return -1;
}

bool params_for_method(const Options& o, int method, avx_pd_params* p, std::string& err) {
  if (avx_default_params(method, p) != AVX_OK) {
    err = avx_last_error();
    return false;
  }
  const std::string sec = method == AVX_METHOD_TV       ? "tv"
                          : method == AVX_METHOD_TVTEMP ? "tvtemp"
                          : method == AVX_METHOD_TGV2   ? "tgv2"
                          : method == AVX_METHOD_ICTV   ? "ictv"
                                                        : "ictgv2";
  auto f = [&](const char* k, float def) { return conf_f(o, sec + "." + k, def); };
  // keys a section does not declare (options_parser.cpp:180-324) keep their defaults
  if (method != AVX_METHOD_TVTEMP) {
    p->dx = f("dx", p->dx);
    p->dy = f("dy", p->dy);
    p->timeSpaceWeight = f("timeSpaceWeight", p->timeSpaceWeight);
  }
  p->dt = f("dt", p->dt);
  p->sigma = f("sigma", p->sigma);
  p->tau = f("tau", p->tau);
  p->sigmaTauRatio = f("sigmaTauRatio", p->sigmaTauRatio);
  p->lambda = f("lambda", p->lambda);
  if (method == AVX_METHOD_TGV2 || method == AVX_METHOD_ICTGV2) p->alpha0 = f("alpha0", p->alpha0);
  if (method == AVX_METHOD_TGV2 || method == AVX_METHOD_ICTV || method == AVX_METHOD_ICTGV2)
    p->alpha1 = f("alpha1", p->alpha1);
  if (method == AVX_METHOD_ICTV || method == AVX_METHOD_ICTGV2) {
    p->alpha = f("alpha", p->alpha);
    p->timeSpaceWeight2 = f("timeSpaceWeight2", p->timeSpaceWeight2);
    p->dx2 = f("dx2", p->dx2);
    p->dy2 = f("dy2", p->dy2);
    p->dt2 = f("dt2", p->dt2);
  }
  // maxIt / stopPDGap are top-level and apply to every method (options_parser.cpp:326-355)
  p->maxIt = (unsigned)conf_f(o, "maxIt", 500.f);
  p->stopPDGap = conf_f(o, "stopPDGap", 0.f);
  // lambda is adapted only with -a, from [adaptlambda] k (default 0) and d (default 1)
  p->adaptLambda = o.adaptlambda ? 1 : 0;
  p->adaptK = conf_f(o, "adaptlambda.k", 0.f);
  p->adaptD = conf_f(o, "adaptlambda.d", 1.f);
  return true;
}

void print_usage() {
  std::cout << "Usage: avionic [options] [-d w:h:d:nRO:nEnc1:nEnc2:c:f <kdata> <mask/traj> | -r <rawdata>] <output>\n"
            << "\nAVIONIC: Accelerated Variational dynamic MRI Reconstruction (B200 core)\n\n"
            << "Required:\n  -d  problem dimensions  kdata  mask/traj  output\n\n"
            << "Options:\n"
            << "  -h [ --help ]              show help message\n"
            << "  -g [ --debugstep ] arg (=10)  PD gap every arg iterations (0: off), exported with -e\n"
            << "  -v [ --verbose ]           verbose console output\n"
            << "  -d [ --dims ] arg          width:height:depth:readouts:encodings_y:encodings_z:coils:frames\n"
            << "  -n [ --nonuniform ]        nonuniform (radial) data\n"
            << "  -o [ --normalize ]         normalise the data\n"
            << "  -e [ --extradata ]         export additional results\n"
            << "  -a [ --adaptlambda ]       adapt lambda from [adaptlambda] k, d\n"
            << "  -w [ --dens ] arg          density compensation data\n"
            << "  -p [ --params ] arg        configuration file\n"
            << "  -s [ --sens ] arg          coil sensitivity data\n"
            << "  -u [ --uzero ] arg         initial image u0\n"
            << "  -b [ --gpudevice ] arg (=-1)  GPU device number\n"
            << "  -m [ --method ] arg (=ICTGV2) TV, TVTEMP, TGV2, ICTV, ICTGV2\n"
            << "  -i [ --maxIt ] arg (=500)  maximum number of iterations\n"
            << "  -j [ --stopPDGap ] arg (=0) stop at this normalised PD gap\n"
            << "  --opnormSteps arg (=0)     initial steps from arg power iterations of ||K|| (0: the\n"
            << "                             configured sigma, tau)\n";
}

}  // namespace avcli
