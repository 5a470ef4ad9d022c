// Command line and INI configuration of the avionic executable.
//
// Accepts the reference's flags (CUDA/src/options_parser.cpp:76-150) and
// configuration keys (:173-324) with the same precedence: values given on the
// command line are stored first and a configuration file never overrides them
// (:357-411).  Configuration syntax: "[section]" headers, "key = value" lines,
// "#" comments; keys may also be given on the command line as
// --section.key=value or --section.key value.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "avionic.h"

namespace avcli {

struct Options {
  bool help = false, verbose = false, nonuniform = false, normalize = false, extradata = false;
  bool adaptlambda = false, rawdata = false, force_os_removal = false;
  int debugstep = 10;
  int gpu = -1;
  int tpat = 1;
  unsigned opnorm_steps = 0;  // --opnormSteps: power iterations of the initial-step estimate (0: off)
  unsigned slice = 0;
  std::string dens, params_file, sens, u0, labeldata, data_bs, mask_bs, final_bs;
  bool have_dims = false;
  unsigned dims[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // w:h:d:nRO:nEnc1:nEnc2:coils:frames
  std::vector<std::string> positional;            // kdata, mask/trajectory, output
  std::map<std::string, std::string> conf;        // "tv.lambda" -> "3.0", "method" -> ...
};

// Parses argv.  Returns false with err set on malformed input.
bool parse_command_line(int argc, char** argv, Options& o, std::string& err);
// Reads the configuration file; keys already present are kept.  found is set
// false when the file cannot be opened (the reference warns and continues).
bool parse_config_file(const std::string& path, Options& o, std::string& err, bool* found);
// Method number (AVX_METHOD_*) of a case-insensitive name, or -1.
int method_from_name(const std::string& name);
// The solver parameters of a method from the parsed configuration.
bool params_for_method(const Options& o, int method, avx_pd_params* p, std::string& err);
void print_usage();

}  // namespace avcli
