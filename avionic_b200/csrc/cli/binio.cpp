#include "binio.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

namespace avcli {

bool read_bin(const std::string& path, std::vector<std::complex<double>>& out, bool* is_complex, std::string* err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    if (err) *err = "cannot open " + path;
    return false;
  }
  unsigned char flag = 0;
  uint32_t n = 0;
  if (std::fread(&flag, 1, 1, f) != 1 || std::fread(&n, 4, 1, f) != 1) {
    std::fclose(f);
    if (err) *err = "truncated header in " + path;
    return false;
  }
  const bool cplx = (flag & 1) != 0;
  std::vector<double> re(n), im(cplx ? n : 0);
  bool ok = std::fread(re.data(), 8, n, f) == n;
  if (ok && cplx) ok = std::fread(im.data(), 8, n, f) == n;
  std::fclose(f);
  if (!ok) {
    if (err) *err = "truncated data in " + path + " (expected " + std::to_string(n) + " values)";
    return false;
  }
  out.resize(n);
  for (uint32_t i = 0; i < n; ++i) out[i] = std::complex<double>(re[i], cplx ? im[i] : 0.0);
  if (is_complex) *is_complex = cplx;
  return true;
}

bool write_bin(const std::string& path, const std::vector<std::complex<double>>& v, bool is_complex,
               std::string* err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    if (err) *err = "cannot create " + path;
    return false;
  }
  const unsigned char flag = is_complex ? 1 : 0;
  const uint32_t n = (uint32_t)v.size();
  bool ok = std::fwrite(&flag, 1, 1, f) == 1 && std::fwrite(&n, 4, 1, f) == 1;
  std::vector<double> buf(n);
  for (uint32_t i = 0; i < n; ++i) buf[i] = v[i].real();
  ok = ok && std::fwrite(buf.data(), 8, n, f) == n;
  if (is_complex) {
    for (uint32_t i = 0; i < n; ++i) buf[i] = v[i].imag();
    ok = ok && std::fwrite(buf.data(), 8, n, f) == n;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok && err) *err = "write failed for " + path;
  return ok;
}

std::string file_extension(const std::string& path) {
  const size_t slash = path.find_last_of('/');
  const size_t dot = path.find_last_of('.');
  if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return "";
  return path.substr(dot);
}

std::string parent_directory(const std::string& path) {
  const size_t slash = path.find_last_of('/');
  if (slash == std::string::npos) return ".";
  if (slash == 0) return "/";
  return path.substr(0, slash);
}

}  // namespace avcli
