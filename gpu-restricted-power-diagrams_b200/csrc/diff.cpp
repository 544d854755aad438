// Comparison of two moment sets (m*x, m*y, m*z, m per cell): the figures of
// the reference's result-diff tool (utils/diffResult/main.cpp:62-121) as a
// host function of the C ABI.
#include <cmath>
#include <cstring>

#include "../../include/rpd.h"

extern "C" int rpd_compare_moments(const double *a, const double *b, size_t n, rpd_moment_diff *out) {
  if (!a || !b || !out) return RPD_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->cells = (long long)n;
  for (int f = 0; f < 2; ++f) {
    const double *r = f ? b : a;
    double *sum = f ? out->sum_b : out->sum_a;
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < 4; ++j) sum[j] += r[4 * i + j];
  }
  long long both = 0;
  double ave[4] = {0, 0, 0, 0}, mave[3] = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    const double *p = a + 4 * i, *q = b + 4 * i;
    const double dm = std::fabs(q[3] - p[3]);
    if (dm > out->max_mass) out->max_mass = dm;
    // barycentres only where both cells have a positive mass
    if (p[3] <= 0 || q[3] <= 0) continue;
    ++both;
    ave[3] += dm;
    for (int j = 0; j < 3; ++j) {
      const double db = std::fabs(q[j] / q[3] - p[j] / p[3]);
      ave[j] += db;
      if (db > out->max_bary[j]) out->max_bary[j] = db;
      const double dmj = std::fabs(q[j] - p[j]);
      mave[j] += dmj;
      if (dmj > out->max_moment[j]) out->max_moment[j] = dmj;
    }
  }
  out->cells_both = both;
  if (both > 0) {
    out->avg_mass = ave[3] / double(both);
    for (int j = 0; j < 3; ++j) {
      out->avg_bary[j] = ave[j] / double(both);
      out->avg_moment[j] = mave[j] / double(both);
    }
  }
  return RPD_OK;
}
