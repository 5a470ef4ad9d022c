// Reference .bin vector files: uint8 is_complex, uint32 n (little-endian),
// n float64 real parts, then n float64 imaginary parts when is_complex
// (matlab/writebin_vector.m:35-44, matlab/readbin_vector.m:30-40).
#pragma once

#include <complex>
#include <string>
#include <vector>

namespace avcli {

// Reads a vector file.  Real files give zero imaginary parts.  Returns false
// (with a message in err) on a missing, truncated or malformed file.
bool read_bin(const std::string& path, std::vector<std::complex<double>>& out, bool* is_complex, std::string* err);
bool write_bin(const std::string& path, const std::vector<std::complex<double>>& v, bool is_complex, std::string* err);

std::string file_extension(const std::string& path);  // utils::GetFileExtension
std::string parent_directory(const std::string& path);  // utils::GetParentDirectory

}  // namespace avcli
