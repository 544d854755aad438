// rpd.hpp -- C++ facade of librpd with the reference's class and method names
// (knearests.h:9-50, Grid.h:14-70, voronoi.h:60-256), header-only over the
// C ABI of rpd.h.  A user of the reference swaps its includes for this one
// and keeps the same calls:
//
//   rpd::Grid grid;  grid.load("domain.txt");
//   rpd::VoroAlgo algo(rpd::Context::create(0));
//   algo.m_K = 50; algo.m_P = 30; algo.m_V = 40;
//   algo.setInputPoints(xyzw);            // std::vector<float>, 4 per seed
//   algo.setGrid(grid);
//   std::vector<rpd::VoroAlgoStat> stats;
//   algo.launch([&](rpd::VoroAlgo const &a) { bary = a.getBarycenters(); return true; }, stats);
//
// Differences: there is no OpenCL context (rpd::Context wraps a CUDA device);
// results are doubles; getBarycenters is in user order, so
// getPermutationToUser is the identity.
#pragma once

#include <functional>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "rpd.h"

namespace rpd {

class Context {
 public:
  static std::shared_ptr<Context> create(int device = 0) {
    int err = 0;
    rpd_context *c = rpd_context_create(device, &err);
    if (!c) return nullptr;
    return std::shared_ptr<Context>(new Context(c));
  }
  ~Context() { rpd_context_destroy(h_); }
  rpd_context *handle() const { return h_; }
  std::string error() const { return rpd_context_error(h_); }

 private:
  explicit Context(rpd_context *h) : h_(h) {}
  rpd_context *h_;
};

// Grid (Grid.h:14-70) over rpd_grid.
struct Grid {
  explicit Grid(bool debug = false) : m_debug(debug) {}
  ~Grid() { reset(nullptr); }
  Grid(const Grid &) = delete;
  Grid &operator=(const Grid &) = delete;

  bool valid() const { return h_ && rpd_grid_valid(h_, nullptr, 0) == 1; }
  bool load(char const *filename) {
    int err = 0;
    rpd_grid *g = rpd_grid_load(filename, &err);
    if (!g) return false;
    reset(g);
    return true;
  }
  bool save(char const *filename) const { return h_ && rpd_grid_save(h_, filename) == RPD_OK; }
  double getVolume() const { return h_ ? rpd_grid_volume(h_) : 0.0; }
  void printInvariants(std::ostream &os) const {
    double inv[4] = {0, 0, 0, 0};
    if (h_) rpd_grid_invariants(h_, inv);
    os << "Grid::load: volume=" << inv[3] << "\n";
    if (inv[3] != 0)
      os << "Grid::load: bary=" << inv[0] / inv[3] << "x" << inv[1] / inv[3] << "x" << inv[2] / inv[3] << "\n";
  }
  static std::unique_ptr<Grid> blob(int size, int nellipsoids, uint64_t seed) {
    int err = 0;
    std::unique_ptr<Grid> g(new Grid());
    g->reset(rpd_grid_make_blob(size, nellipsoids, seed, &err));
    return g->h_ ? std::move(g) : nullptr;
  }
  rpd_grid *handle() const { return h_; }

 private:
  void reset(rpd_grid *g) {
    if (h_) rpd_grid_destroy(h_);
    h_ = g;
  }
  rpd_grid *h_ = nullptr;
  bool m_debug;
};

// KNearests (knearests.h:9-50): binning at construction, K nearest of every
// seed on demand (user ids).
class KNearests {
 public:
  KNearests(std::shared_ptr<Context> ctx, std::vector<float> const &xyzw) : ctx_(std::move(ctx)) {
    int err = 0;
    s_ = rpd_solver_create(ctx_->handle(), &err);
    if (!s_ || rpd_solver_set_points(s_, xyzw.data(), int(xyzw.size() / 4), RPD_HOST) != RPD_OK)
      throw std::runtime_error("KNearests: " + ctx_->error());
  }
  ~KNearests() { rpd_solver_destroy(s_); }
  KNearests(const KNearests &) = delete;
  KNearests &operator=(const KNearests &) = delete;
  int getNumPoints() const { return rpd_solver_num_points(s_); }
  bool buildKnearests(int K, double &totalTime) {
    nearest_.assign(size_t(getNumPoints()) * K, -1);
    float ms = 0;
    if (rpd_solver_knn(s_, K, nearest_.data(), RPD_HOST, &ms) != RPD_OK) return false;
    totalTime += ms / 1e3;
    return true;
  }
  std::vector<int> getPermutation() const {
    std::vector<int> p(getNumPoints());
    rpd_solver_get_permutation(s_, p.data(), RPD_HOST);
    return p;
  }
  std::vector<int> const &getNearests() const { return nearest_; }

 private:
  std::shared_ptr<Context> ctx_;
  rpd_solver *s_ = nullptr;
  std::vector<int> nearest_;
};

// VoroAlgoStat (voronoi.h:60-103).
struct VoroAlgoStat {
  explicit VoroAlgoStat(std::string name) : m_name(std::move(name)) {}
  void pythonPrint(std::ostream &output, std::string prefix = "") const {
    output << "{\"name\" : \"" << prefix << m_name << "\", \"knn\":" << m_times[0] << ", \"CC\":" << m_times[1]
           << ", \"time\":" << m_times[2] << ", ";
    if (m_numDone) output << "\"nbdone\":" << m_numDone << ",";
    output << "\"nbcells\":" << m_num << "}";
  }
  std::string m_name;
  int m_num = 0;
  int m_numDone = 0;
  double m_times[3] = {0, 0, 0};  // knn, cells, total (seconds, device time)
};

// VoroAlgo (voronoi.h:105-256).
class VoroAlgo {
 public:
  explicit VoroAlgo(std::shared_ptr<Context> ctx, bool debug = false) : ctx_(std::move(ctx)), m_debug(debug) {
    int err = 0;
    s_ = rpd_solver_create(ctx_->handle(), &err);
    if (!s_) throw std::runtime_error("VoroAlgo: no solver");
  }
  ~VoroAlgo() { rpd_solver_destroy(s_); }
  VoroAlgo(VoroAlgo const &) = delete;
  VoroAlgo &operator=(VoroAlgo const &) = delete;

  bool launch(std::function<bool(VoroAlgo const &)> saveData, std::vector<VoroAlgoStat> &stats) {
    rpd_params p;
    rpd_params_default(&p);
    p.K = m_K;
    p.P = m_P;
    p.V = m_V;
    p.T = m_T;
    p.keep_distance = m_keepDistance;
    p.keep_volume = m_keepVolume;
    p.hessian_h = m_H;
    p.hessian_hc = m_HC;
    p.precision = m_precision;
    if (m_safeRadius) p.flags |= RPD_FLAG_SAFE_RADIUS;
    if (rpd_solver_launch(s_, &p) != RPD_OK) {
      if (m_debug) fprintf(stderr, "VoroAlgo::launch: %s\n", ctx_->error().c_str());
      return false;
    }
    rpd_stats st;
    rpd_solver_get_stats(s_, &st);
    for (int i = 0; i < st.npasses && i < 8; ++i) {
      VoroAlgoStat v(i == 0 ? "first" : "extra");
      v.m_num = st.pass_cells[i];
      v.m_times[0] = st.pass_knn_ms[i] / 1e3;
      v.m_times[1] = st.pass_cell_ms[i] / 1e3;
      v.m_times[2] = v.m_times[0] + v.m_times[1];
      stats.push_back(v);
    }
    return saveData ? saveData(*this) : true;
  }
  void setGrid(Grid const &grid) { rpd_solver_set_grid(s_, grid.handle()); }
  void setInputPoints(std::vector<float> const &seeds) {
    rpd_solver_set_points(s_, seeds.data(), int(seeds.size() / 4), RPD_HOST);
  }
  // Weight-only re-solve (no counterpart in the reference): new weights,
  // one per seed in the order given to setInputPoints; bins and neighbours
  // are kept.
  void setWeights(std::vector<float> const &w) { rpd_solver_set_weights(s_, w.data(), RPD_HOST); }
  int getNumInputPoints() const { return rpd_solver_num_points(s_); }
  // With m_keepDistance >= 0 and a grid the outputs are the used cells
  // (VoroAlgoComputeData::compressResult, voronoi.cpp:513-691), in
  // ascending user order; otherwise every seed, in user order.
  int getNumOutputPoints() const {
    const int u = rpd_solver_used_count(s_);
    return u >= 0 ? u : rpd_solver_num_points(s_);
  }
  std::vector<double> getBarycenters() const {
    const int u = rpd_solver_used_count(s_);
    std::vector<double> r(4 * size_t(getNumOutputPoints()));
    if (u >= 0) {
      std::vector<int> ids(size_t(u) + 1);
      rpd_solver_get_used(s_, r.data(), ids.data(), RPD_HOST);
    } else {
      rpd_solver_get_moments(s_, r.data(), RPD_HOST);
    }
    return r;
  }
  std::vector<int> getPermutationToUser() const {
    const int u = rpd_solver_used_count(s_);
    std::vector<int> r(getNumOutputPoints());
    if (u >= 0) {
      std::vector<double> rows(4 * size_t(u) + 4);
      rpd_solver_get_used(s_, rows.data(), r.data(), RPD_HOST);
    } else {
      for (size_t i = 0; i < r.size(); ++i) r[i] = int(i);
    }
    return r;
  }
  // --hessian rows (m_H > 0): per output point m_H facets of m_HC values
  // (the area, or the area-weighted centroid and the area), and their
  // neighbours as output indices, -1 after a row's last facet.
  std::vector<double> getHessians() const {
    if (m_H <= 0) return {};
    std::vector<double> v(size_t(getNumOutputPoints()) * m_H * m_HC + 1);
    std::vector<int> ids(size_t(getNumOutputPoints()) * m_H + 1);
    rpd_solver_get_hessian(s_, v.data(), ids.data(), RPD_HOST);
    v.pop_back();
    return v;
  }
  std::vector<int> getHessianIds() const {
    if (m_H <= 0) return {};
    std::vector<double> v(size_t(getNumOutputPoints()) * m_H * m_HC + 1);
    std::vector<int> ids(size_t(getNumOutputPoints()) * m_H + 1);
    rpd_solver_get_hessian(s_, v.data(), ids.data(), RPD_HOST);
    ids.pop_back();
    return ids;
  }
  std::vector<int> getStatus() const {
    std::vector<int> r(getNumOutputPoints());
    rpd_solver_get_status(s_, r.data(), RPD_HOST);
    return r;
  }

  int m_K = 25;
  int m_P = 35;
  int m_T = 100;
  int m_V = 40;
  // used cells with a grid (voronoi.cpp:1052-1053 defaults): -1 every seed,
  // else the kept ring distance; the mass that makes a cell used
  float m_keepVolume = 1;
  int m_keepDistance = 1;
  // --hessian (voronoi.cpp:1048-1049 defaults): facets per row (0: off) and
  // values per facet (1 or 4)
  int m_H = 0;
  int m_HC = 1;
  // no counterparts in VoroAlgo: the clipping arithmetic (RPD_PRECISION_*, in
  // place of the compile-time VHSAlgo / USE_DOUBLE choice) and the weighted
  // security-radius guard (RPD_FLAG_SAFE_RADIUS)
  int m_precision = RPD_PRECISION_FP64;
  bool m_safeRadius = false;

 private:
  std::shared_ptr<Context> ctx_;
  rpd_solver *s_ = nullptr;
  bool m_debug;
};

}  // namespace rpd
