// nlb_geometry.cpp -- host-side cell geometry (see nlb_geometry.h).
// Must be compiled with -ffp-contract=off: every expression below follows the
// reference's f64 association order, with no fused multiply-add.
#include "nlb_geometry.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace nlb {

namespace {

inline void mv(const double* m, double v0, double v1, double v2, double* out) {
  for (int r = 0; r < 3; ++r) {
    const double t = m[3 * r] * v0 + m[3 * r + 1] * v1;
    out[r] = t + m[3 * r + 2] * v2;
  }
}

inline double sq3(double a, double b, double c) {
  const double t = a * a + b * b;
  return t + c * c;
}

inline uint64_t as_usize(double x) {
  if (!(x > 0.0)) return 0;
  if (x >= 18446744073709551616.0) return std::numeric_limits<uint64_t>::max();
  return static_cast<uint64_t>(x);
}

inline int32_t as_i32(double x) {
  if (std::isnan(x)) return 0;
  if (x >= 2147483647.0) return std::numeric_limits<int32_t>::max();
  if (x <= -2147483648.0) return std::numeric_limits<int32_t>::min();
  return static_cast<int32_t>(x);
}

}  // namespace

double fmax_nan_ignoring(double a, double b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a > b ? a : b;
}

double fmin_nan_ignoring(double a, double b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}

bool make_cell(const double* h9, const bool pbc[3], HostCell& c, std::string& err) {
  for (int i = 0; i < 9; ++i) c.h[i] = h9[i];
  for (int a = 0; a < 3; ++a) c.pbc[a] = pbc[a];
  // nalgebra Matrix3::try_inverse: cofactors of the first row, determinant
  // (m11*A - m12*B) + m13*C, every entry cofactor / det.
  const double m11 = h9[0], m12 = h9[1], m13 = h9[2];
  const double m21 = h9[3], m22 = h9[4], m23 = h9[5];
  const double m31 = h9[6], m32 = h9[7], m33 = h9[8];
  const double ca = m22 * m33 - m32 * m23;
  const double cb = m21 * m33 - m31 * m23;
  const double cc = m21 * m32 - m31 * m22;
  const double t = m11 * ca - m12 * cb;
  const double det = t + m13 * cc;
  if (det == 0.0) {
    err = "Cell matrix is not invertible";
    return false;
  }
  c.hinv[0] = ca / det;
  c.hinv[1] = (m13 * m32 - m33 * m12) / det;
  c.hinv[2] = (m12 * m23 - m22 * m13) / det;
  c.hinv[3] = -cb / det;
  c.hinv[4] = (m11 * m33 - m31 * m13) / det;
  c.hinv[5] = (m13 * m21 - m23 * m11) / det;
  c.hinv[6] = cc / det;
  c.hinv[7] = (m12 * m31 - m32 * m11) / det;
  c.hinv[8] = (m11 * m22 - m21 * m12) / det;
  return true;
}

bool auto_box(const double* pos, int64_t n, double rc_max, HostCell& c, std::string& err) {
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      const double v = pos[3 * i + a];
      if (v < lo[a]) lo[a] = v;
      if (v > hi[a]) hi[a] = v;
    }
  return auto_box_from_bounds(lo, hi, rc_max, c, err);
}

bool auto_box_from_bounds(const double* lo, const double* hi, double rc_max, HostCell& c,
                          std::string& err) {
  const double margin = rc_max + 1.0;
  double h9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < 3; ++a) h9[4 * a] = (hi[a] - lo[a]) + 2.0 * margin;
  const bool none[3] = {false, false, false};
  return make_cell(h9, none, c, err);
}

void perpendicular_widths(const HostCell& c, double w[3]) {
  for (int r = 0; r < 3; ++r)
    w[r] = 1.0 / std::sqrt(sq3(c.hinv[3 * r], c.hinv[3 * r + 1], c.hinv[3 * r + 2]));
}

Method choose_method(const HostCell& c, int64_t n, double rc_max, uint64_t bf_threshold,
                     bool multi) {
  double w[3];
  perpendicular_widths(c, w);
  const double min_w = fmin_nan_ignoring(fmin_nan_ignoring(w[0], w[1]), w[2]);
  const bool mic_safe = rc_max * 2.0 < min_w;
  if ((uint64_t)n < bf_threshold && mic_safe) {
    const bool isolated = !c.pbc[0] && !c.pbc[1] && !c.pbc[2];
    return (isolated && !multi) ? Method::kBruteIsolated : Method::kBruteMic;
  }
  return Method::kCellList;
}

void plan_grid(const HostCell& c, double rc, GridParams& g) {
  for (int i = 0; i < 9; ++i) {
    g.h[i] = c.h[i];
    g.hinv[i] = c.hinv[i];
  }
  double w[3];
  perpendicular_widths(c, w);
  int64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    const uint64_t b = as_usize(std::floor(w[a] / rc));
    const uint64_t nb = std::max<uint64_t>(b, 1);
    // Bins per axis fit in i32 for any grid whose bin table fits in memory;
    // larger values are clamped and rejected by the caller's size check.
    g.nb[a] = (int32_t)std::min<uint64_t>(nb, (uint64_t)std::numeric_limits<int32_t>::max());
    // Saturating product: total stays <= 2^40 (a clamped value only ever
    // means "too many bins" to the callers' size checks).
    constexpr int64_t kCap = (int64_t)1 << 40;
    total = total > kCap / (int64_t)g.nb[a] ? kCap : total * (int64_t)g.nb[a];
  }
  g.total_bins = total;
  for (int a = 0; a < 3; ++a) g.ns[a] = as_i32(std::ceil((rc * (double)g.nb[a]) / w[a]));

  double vb[3][3];
  mv(c.h, 1.0 / (double)g.nb[0], 0.0, 0.0, vb[0]);
  mv(c.h, 0.0, 1.0 / (double)g.nb[1], 0.0, vb[1]);
  mv(c.h, 0.0, 0.0, 1.0 / (double)g.nb[2], vb[2]);
  mv(c.h, 0.5 / (double)g.nb[0], 0.5 / (double)g.nb[1], 0.5 / (double)g.nb[2], g.origin);
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) g.basis[a][k] = vb[a][k];
  double d[4], t[3];
  for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] + vb[1][k]) + vb[2][k];
  d[0] = sq3(t[0], t[1], t[2]);
  for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] + vb[1][k]) - vb[2][k];
  d[1] = sq3(t[0], t[1], t[2]);
  for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] - vb[1][k]) + vb[2][k];
  d[2] = sq3(t[0], t[1], t[2]);
  for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] - vb[1][k]) - vb[2][k];
  d[3] = sq3(t[0], t[1], t[2]);
  const double mx =
      fmax_nan_ignoring(fmax_nan_ignoring(fmax_nan_ignoring(d[0], d[1]), d[2]), d[3]);
  const double radius = 0.5 * std::sqrt(mx);
  g.radius = radius;
  // prune_limit = sqrt(rc*rc) + R (src/search.rs:488-489): the square root of
  // the squared cutoff is taken, not rc itself.
  const double pl = std::sqrt(rc * rc) + radius;
  g.prune_sq = pl * pl;
}

std::vector<int32_t> cutoff_order(const double* cutoffs, int32_t k) {
  std::vector<int32_t> order(k);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t a, int32_t b) { return cutoffs[a] < cutoffs[b]; });
  return order;
}

}  // namespace nlb
