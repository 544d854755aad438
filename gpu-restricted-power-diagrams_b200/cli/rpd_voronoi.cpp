// rpd_voronoi: command-line driver with the reference test_voronoi's options
// (test_voronoi.cpp:65-223, Options.cpp:70-92) over librpd.
//
//   rpd_voronoi [--K=k] [--P=p] [--V=v] [--T=t] [--grid=FILE] [--output=xyz|mg|volume|geogram]
//               [--points4D] [--loadBinaryPoints] [--saveBinaryPoints=FILE] [--keepVolume=v]
//               [--printInvariants] [--checkGrid] [--debug] seeds.xyz
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rpd.hpp"

namespace {

// Seeds through the library's loader: the reference's text format
// (Utils::loadSeedsFile, Utils.cpp:36-79, not normalised) or, with
// --loadBinaryPoints, its binary format (Utils.cpp:81-97).
bool load_seeds(const char *path, bool four_d, bool binary, std::vector<float> &xyzw) {
  float *p = nullptr;
  int n = 0;
  if (rpd_seeds_load(path, four_d ? 1 : 0, binary ? 1 : 0, &p, &n) != RPD_OK) return false;
  xyzw.assign(p, p + 4 * size_t(n));
  rpd_seeds_free(p);
  return n > 0;
}

// --output=geogram (Utils::dropXYZGeogram, Utils.cpp:146-170, as
// test_voronoi.cpp:162-167 calls it): every seed's barycentre as a vertex
// and its mass as the attribute "w", in geogram's ASCII layout.
void write_geogram(const char *path, const std::vector<double> &bary) {
  const size_t n = bary.size() / 4;
  std::ofstream f(path, std::ios::binary);
  f << "[HEAD]\n\"GEOGRAM\"\n\"1.0\"\n[ATTS]\n\"GEO::Mesh::vertices\"\n" << n << "\n";
  f << "[ATTR]\n\"GEO::Mesh::vertices\"\n\"point\"\n\"double\"\n8\n3\n";
  for (size_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) f << bary[4 * i + d] / bary[4 * i + 3] << "\n";
  f << "[ATTR]\n\"GEO::Mesh::vertices\"\n\"w\"\n\"double\"\n8\n1\n";
  for (size_t i = 0; i < n; ++i) f << bary[4 * i + 3] << "\n";
}

void usage(const char *argv0) {
  std::cerr << "Usage: " << argv0 << " [options] points.xyz\n"
            << "\t--K=k --P=p --V=v --T=t: first-pass caps (default 20/25/30/100)\n"
            << "\t--grid=FILE: volume domain in the --grid text format\n"
            << "\t--output=xyz|mg|volume|geogram (repeatable)\n"
            << "\t--points4D: the seed file has a weight column\n"
            << "\t--loadBinaryPoints: the seed file is a 4D binary file\n"
            << "\t--saveBinaryPoints=file: save the seeds in a 4D binary file\n"
            << "\t--keepVolume=v: cells with volume below v are empty (default 1)\n"
            << "\t--keepDist2=d: with --grid, keep the used cells and d rings around them (default 0; -1 all)\n"
            << "\t--hessian: compute the facet-area rows (--H=h facets per row, default 50; --HC=1|4)\n"
            << "\t--safeRadius: stop clipping on the weighted security-radius guard\n"
            << "\t--precision=fp64|mixed|fp32: arithmetic of the clipping loop (default fp64)\n"
            << "\t--printInvariants --checkGrid --debug\n";
}

}  // namespace

int main(int argc, char **argv) {
  int K = 20, P = 25, V = 30, T = 100;
  std::string grid_file, seeds_file;
  std::vector<std::string> outputs;
  bool points4d = false, invariants = false, check_grid = false, debug = false, load_binary = false;
  std::string save_binary;
  double keep_volume = 1;
  int keep_dist2 = 0;  // test_voronoi's final keep distance (Options.cpp:42, test_voronoi.cpp:38)
  bool hessian = false, safe_radius = false;
  int precision = RPD_PRECISION_FP64;
  int H = 50, HC = 1;  // Options.cpp:22-23
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i], val;
    const size_t eq = a.find('=');
    if (eq != std::string::npos) {
      val = a.substr(eq + 1);
      a = a.substr(0, eq);
    }
    auto need = [&]() -> std::string {
      if (!val.empty()) return val;
      if (i + 1 < argc) return argv[++i];
      usage(argv[0]);
      std::exit(1);
    };
    if (a == "--K") K = std::atoi(need().c_str());
    else if (a == "--P") P = std::atoi(need().c_str());
    else if (a == "--V") V = std::atoi(need().c_str());
    else if (a == "--T") T = std::atoi(need().c_str());
    else if (a == "--grid") grid_file = need();
    else if (a == "--output") outputs.push_back(need());
    else if (a == "--keepVolume") keep_volume = std::atof(need().c_str());
    else if (a == "--keepDist2") keep_dist2 = std::atoi(need().c_str());
    else if (a == "--keepDist") (void)need();  // distance of the passes before the last: no effect here
    else if (a == "--points4D") points4d = true;
    else if (a == "--loadBinaryPoints") load_binary = true;
    else if (a == "--saveBinaryPoints") save_binary = need();
    else if (a == "--hessian") hessian = true;
    else if (a == "--safeRadius") safe_radius = true;
    else if (a == "--precision") {
      const std::string v = need();
      precision = v == "mixed" ? RPD_PRECISION_MIXED : (v == "fp32" ? RPD_PRECISION_FP32 : RPD_PRECISION_FP64);
    }
    else if (a == "--H") H = std::atoi(need().c_str());
    else if (a == "--HC") HC = std::atoi(need().c_str());
    else if (a == "--printInvariants") invariants = true;
    else if (a == "--checkGrid") check_grid = true;
    else if (a == "--debug") debug = true;
    else if (a == "-h" || a == "--help") { usage(argv[0]); return 1; }
    else if (!a.empty() && a[0] == '-') { std::cerr << "ignored option " << a << "\n"; }
    else seeds_file = a;
  }
  if (seeds_file.empty()) {
    usage(argv[0]);
    return 1;
  }
  std::vector<float> pts;
  if (!load_seeds(seeds_file.c_str(), points4d, load_binary, pts)) {
    std::cerr << argv[0] << ": could not load file " << seeds_file << "\n";
    return 1;
  }
  if (!save_binary.empty() && rpd_seeds_save_binary(save_binary.c_str(), pts.data(), int(pts.size() / 4)) != RPD_OK)
    std::cerr << argv[0] << ": could not save " << save_binary << "\n";
  auto ctx = rpd::Context::create(0);
  if (!ctx) {
    std::cerr << argv[0] << ": no usable sm_100 device\n";
    return 1;
  }
  rpd::Grid grid(debug);
  const bool has_grid = !grid_file.empty() && grid.load(grid_file.c_str());
  if (!grid_file.empty() && !has_grid) std::cerr << argv[0] << ": could not load grid " << grid_file << "\n";
  if (has_grid && check_grid && !grid.valid()) std::cerr << argv[0] << ": the grid is invalid.\n";
  if (invariants) {
    if (has_grid) grid.printInvariants(std::cerr);
    else std::cerr << "Grid::load: volume=" << 1e9 << "\nGrid::load: bary=500x500x500\n";
  }
  rpd::VoroAlgo algo(ctx, debug);
  algo.m_K = K;
  algo.m_P = P;
  algo.m_V = V;
  algo.m_T = T;
  algo.m_keepDistance = keep_dist2;
  algo.m_keepVolume = keep_volume;
  algo.m_H = hessian ? H : 0;  // Options.cpp:269-270
  algo.m_HC = HC;
  algo.m_safeRadius = safe_radius;
  algo.m_precision = precision;
  algo.setInputPoints(pts);
  if (has_grid) algo.setGrid(grid);
  std::vector<double> bary;
  std::vector<rpd::VoroAlgoStat> stats;
  const bool ok = algo.launch(
      [&](rpd::VoroAlgo const &a) {
        // back to one row per user seed (zeros for the unused ones), as
        // test_voronoi.cpp:186-211 places them with getPermutationToUser
        const std::vector<double> b = a.getBarycenters();
        const std::vector<int> perm = a.getPermutationToUser();
        bary.assign(4 * (pts.size() / 4), 0.0);
        for (size_t i = 0; i < perm.size(); ++i)
          for (int d = 0; d < 4; ++d) bary[4 * size_t(perm[i]) + d] = b[4 * i + d];
        return true;
      },
      stats);
  if (!ok) {
    std::cerr << argv[0] << ": launch failed: " << ctx->error() << "\n";
    return 1;
  }
  std::cout << "GTime[\"stat\"] = [";
  for (size_t i = 0; i < stats.size(); ++i) {
    stats[i].pythonPrint(std::cout);
    if (i + 1 < stats.size()) std::cout << ",\n";
  }
  std::cout << "]\n";
  const size_t n = bary.size() / 4;
  if (invariants) {
    double vol = 0, b[3] = {0, 0, 0};
    for (size_t i = 0; i < n; ++i) {
      if (bary[4 * i + 3] <= keep_volume) continue;
      vol += bary[4 * i + 3];
      for (int d = 0; d < 3; ++d) b[d] += bary[4 * i + d];
    }
    std::cerr << "Sum of volumes: " << std::setprecision(20) << vol << "\n";
    if (vol > 0) std::cerr << "Cells barycenter=" << b[0] / vol << "x" << b[1] / vol << "x" << b[2] / vol << "\n";
  }
  for (const auto &o : outputs) {
    if (o == "xyz") {
      // barycentres of the cells with |m| >= keepVolume (test_voronoi.cpp:158-161)
      std::ofstream f("gridGPU.xyz");
      size_t k = 0;
      for (size_t i = 0; i < n; ++i)
        if (bary[4 * i + 3] > RPD_NO_CELL_LIMITS && std::abs(bary[4 * i + 3]) >= keep_volume) ++k;
      f << k << "\n";
      for (size_t i = 0; i < n; ++i) {
        const double m = bary[4 * i + 3];
        if (m > RPD_NO_CELL_LIMITS && std::abs(m) >= keep_volume)
          f << bary[4 * i] / m << "  " << bary[4 * i + 1] / m << "  " << bary[4 * i + 2] / m << "\n";
      }
    } else if (o == "mg") {
      // per user seed m*x m*y m*z m, or zeros (test_voronoi.cpp:186-211)
      std::ofstream f("gridGPU_mg.xyzw");
      f << n << "\n" << std::setprecision(20);
      for (size_t i = 0; i < n; ++i) {
        if (bary[4 * i + 3] <= keep_volume) f << "0 0 0 0\n";
        else f << bary[4 * i] << " " << bary[4 * i + 1] << " " << bary[4 * i + 2] << " " << bary[4 * i + 3] << "\n";
      }
    } else if (o == "geogram") {
      write_geogram("gridGPU.geogram_ascii", bary);
    } else if (o == "volume") {
      double vol = 0;
      for (size_t i = 0; i < n; ++i)
        if (bary[4 * i + 3] > keep_volume) vol += bary[4 * i + 3];
      std::cerr << "Sum of volumes: " << std::setprecision(20) << vol << "\n";
    } else {
      std::cerr << argv[0] << ": ignored output : " << o << "\n";
    }
  }
  return 0;
}
