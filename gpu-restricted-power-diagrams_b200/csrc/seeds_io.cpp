// C ABI of the seed files: the reference's text .xyz format
// (Utils::loadSeedsFile, Utils.cpp:36-79) and its binary format
// (readBinarySeedsFile / saveBinarySeedsFile, Utils.cpp:81-113).  Host only.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rpd.h"

namespace {

// A count line, then "x y z" (or "x y z w" for 4D files) per line; blank
// lines are skipped and, as in the reference, no normalisation is applied
// (test_voronoi.cpp:88 passes normalize=false).  The count must match.
int load_text(const char *path, bool four_d, std::vector<float> &xyzw) {
  std::ifstream in(path);
  if (!in.is_open()) return RPD_ERR_IO;
  std::string line;
  bool first = true;
  long long npts = -1;
  while (std::getline(in, line)) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    std::istringstream iss(line);
    if (first) {
      if (!(iss >> npts) || npts < 0 || npts > (1ll << 31) - 1) return RPD_ERR_FORMAT;
      xyzw.reserve(4 * size_t(npts));
      first = false;
      continue;
    }
    float x = 0, y = 0, z = 0, w = 0;
    if (!(iss >> x >> y >> z)) return RPD_ERR_FORMAT;
    if (four_d && !(iss >> w)) return RPD_ERR_FORMAT;
    xyzw.insert(xyzw.end(), {x, y, z, w});
  }
  if (first || (long long)(xyzw.size() / 4) != npts) return RPD_ERR_FORMAT;
  return RPD_OK;
}

// A size_t count N, then N x y z w floats (the float build's `real`).
int load_binary(const char *path, std::vector<float> &xyzw) {
  std::ifstream in(path, std::ios::binary);
  if (!in.is_open()) return RPD_ERR_IO;
  uint64_t n = 0;
  in.read(reinterpret_cast<char *>(&n), sizeof(n));
  if (!in.good() || n == 0 || n > (1ull << 31) - 1) return RPD_ERR_FORMAT;
  xyzw.resize(4 * size_t(n));
  in.read(reinterpret_cast<char *>(xyzw.data()), std::streamsize(sizeof(float) * xyzw.size()));
  if (!in.good()) return RPD_ERR_FORMAT;
  return RPD_OK;
}

}  // namespace

extern "C" {

int rpd_seeds_load(const char *path, int four_d, int binary, float **xyzw, int *n) {
  if (!path || !xyzw || !n) return RPD_ERR_INVALID;
  *xyzw = nullptr;
  *n = 0;
  std::vector<float> v;
  const int rc = binary ? load_binary(path, v) : load_text(path, four_d != 0, v);
  if (rc != RPD_OK) return rc;
  // a NaN or infinite value is a malformed file here (the reference's loader
  // passes it on to the solve, whose bins it breaks)
  for (float f : v)
    if (!std::isfinite(f)) return RPD_ERR_FORMAT;
  const size_t count = v.size() / 4;
  float *out = static_cast<float *>(std::malloc(sizeof(float) * (v.empty() ? 4 : v.size())));
  if (!out) return RPD_ERR_INVALID;
  if (!v.empty()) std::memcpy(out, v.data(), sizeof(float) * v.size());
  *xyzw = out;
  *n = int(count);
  return RPD_OK;
}

void rpd_seeds_free(float *xyzw) { std::free(xyzw); }

int rpd_seeds_save_binary(const char *path, const float *xyzw, int n) {
  if (!path || !xyzw || n <= 0) return RPD_ERR_INVALID;
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  if (!out.is_open()) return RPD_ERR_IO;
  const uint64_t count = uint64_t(n);
  out.write(reinterpret_cast<const char *>(&count), sizeof(count));
  out.write(reinterpret_cast<const char *>(xyzw), std::streamsize(sizeof(float) * 4 * size_t(n)));
  return out.good() ? RPD_OK : RPD_ERR_IO;
}

}  // extern "C"
