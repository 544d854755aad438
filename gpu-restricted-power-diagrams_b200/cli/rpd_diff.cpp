// rpd_diff: compares two result files of moments (a count line, then
// "m*x m*y m*z m" per cell, as rpd_voronoi --output=mg writes them) with
// rpd_compare_moments, printing the reference diff tool's report
// (utils/diffResult/main.cpp:62-121), or one JSON object with --json.
//
//   rpd_diff [--json] a.xyzw b.xyzw
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rpd.h"

namespace {

bool load(const std::string &path, std::vector<double> &v) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  long long n = -1;
  while (std::getline(in, line)) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    std::istringstream is(line);
    if (n < 0) {
      if (!(is >> n) || n < 0) return false;
      v.reserve(4 * size_t(n));
      continue;
    }
    double x, y, z, w;
    if (!(is >> x >> y >> z >> w)) return false;
    v.insert(v.end(), {x, y, z, w});
  }
  return n >= 0 && (long long)(v.size() / 4) == n;
}

}  // namespace

int main(int argc, char **argv) {
  bool json = false;
  std::vector<std::string> files;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--json") json = true;
    else files.push_back(a);
  }
  std::vector<double> r[2];
  if (files.size() != 2 || !load(files[0], r[0]) || !load(files[1], r[1])) {
    std::cerr << "Error:" << argv[0] << " [--json] res1.xyzw res2.xyzw\n";
    return 1;
  }
  if (r[0].size() != r[1].size()) {
    std::cerr << "Error:" << argv[0] << " files " << files[0] << " and " << files[1]
              << " do not contain the same numbers of data\n";
    return 1;
  }
  rpd_moment_diff d;
  if (rpd_compare_moments(r[0].data(), r[1].data(), r[0].size() / 4, &d) != RPD_OK) return 1;
  const double *A = d.sum_a, *B = d.sum_b;
  std::cout.precision(20);
  if (json) {
    auto arr = [](const double *x, int k) {
      std::ostringstream o;
      o.precision(17);
      o << "[";
      for (int i = 0; i < k; ++i) o << (i ? ", " : "") << x[i];
      return o.str() + "]";
    };
    std::cout << "{\"cells\": " << d.cells << ", \"cells_both\": " << d.cells_both << ", \"sum_a\": " << arr(A, 4)
              << ", \"sum_b\": " << arr(B, 4) << ", \"max_mass\": " << d.max_mass
              << ", \"max_bary\": " << arr(d.max_bary, 3) << ", \"max_moment\": " << arr(d.max_moment, 3)
              << ", \"avg_mass\": " << d.avg_mass << ", \"avg_bary\": " << arr(d.avg_bary, 3)
              << ", \"avg_moment\": " << arr(d.avg_moment, 3) << "}\n";
    return 0;
  }
  std::cout << "------------------- intrinsic (sum) --------------------------\n";
  std::cout << "Volume : " << A[3] << "\t" << B[3] << "\t" << (B[3] - A[3]) << "\n";
  std::cout << "Barycenter : " << A[0] / A[3] << "x" << A[1] / A[3] << "x" << A[2] / A[3] << "\t" << B[0] / B[3] << "x"
            << B[1] / B[3] << "x" << B[2] / B[3] << "\t" << (B[0] / B[3] - A[0] / A[3]) << "x"
            << (B[1] / B[3] - A[1] / A[3]) << "x" << (B[2] / B[3] - A[2] / A[3]) << "\n";
  std::cout << "------------------- maximal difference by cells--------------------------\n";
  std::cout << "Volume : " << d.max_mass << "\n";
  std::cout << "Barycenter : " << d.max_bary[0] << "x" << d.max_bary[1] << "x" << d.max_bary[2] << "\n";
  std::cout << "Barycenter x volume : " << d.max_moment[0] << "x" << d.max_moment[1] << "x" << d.max_moment[2] << "\n";
  std::cout << "------------------- average difference by cells--------------------------\n";
  std::cout << "Volume : " << d.avg_mass << "\n";
  std::cout << "Barycenter : " << d.avg_bary[0] << "x" << d.avg_bary[1] << "x" << d.avg_bary[2] << "\n";
  std::cout << "Barycenter x volume : " << d.avg_moment[0] << "x" << d.avg_moment[1] << "x" << d.avg_moment[2] << "\n";
  return 0;
}
