// nl_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the neighbour-list search path of solccp/neighborlist-rs
// (Rust crate v0.1.9).  It is the parity checker for the CUDA library and the
// timed CPU baseline of bench.py.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline legs load it; the product library never does.
//
// Build: g++ -O2 -std=c++17 -ffp-contract=off -fno-fast-math -fPIC -shared
// (see oracle/Makefile).  -ffp-contract=off matters: the reference's f64
// arithmetic (wide::f64x4 and scalar Rust) never fuses multiply and add.
//
// Reference files restated here (paths inside the reference project):
//   src/cell.rs:18-93        Cell::new / to_fractional / perpendicular_widths /
//                            wrap / get_shift_and_displacement
//   src/search.rs:92-264     CellList::build (Morton sort, bins, wrap shifts)
//   src/search.rs:35-57      OffsetList::prepare (per-axis stencil tables)
//   src/search.rs:448-727    count_atom_neighbors / fill_atom_neighbors
//   src/search.rs:729-1078   count/fill_atom_neighbors_multi
//   src/search.rs:1080-1159  search_atom_neighbors (serial; same set and order)
//   src/search.rs:1162-1185  div_mod, compute_z_order, interleave_3
//   src/search.rs:1187-1405  brute_force_search_simd / _full / _multi
//   src/single.rs:8-164      search_single / search_single_multi (auto-box,
//                            mic_safe, dispatch)
//   src/batch.rs:10-290      search_batch / search_batch_multi
//   src/config.rs:4-40       brute-force / parallel thresholds
//   spec.md:100-108, RUST_API.md:89-90
//                            directed list, displacement vectors, distances
//                            (orc_edge_extras; asked for by the spec, not
//                            implemented by the reference)
//
// Third-party arithmetic restated (no Cargo.lock in the reference; Cargo.toml
// pins nalgebra ^0.34.1, wide ^1.1.1):
//   * nalgebra Matrix3::try_inverse: 3x3 adjugate / first-row cofactor
//     determinant, inverse entries = cofactor / det.
//   * nalgebra Matrix3 * Vector3 (gemv as column axpys):
//       out[r] = (m[r][0]*v0 + m[r][1]*v1) + m[r][2]*v2
//   * nalgebra norm_squared of a 3-vector: (a*a + b*b) + c*c
//   * wide::f64x4: lane-wise IEEE mul/add/lt, no FMA.
// Bit-level parity of the 3x3 inverse for skewed cells rests on this
// restatement of nalgebra; edge sets are pinned by the reference's own golden
// counts and unit tests (tests/test_oracle_golden.py).
//
// Ties in the atom Morton key: the reference uses sort_unstable_by_key on the
// key alone (src/search.rs:115), whose order among equal keys is unspecified.
// This oracle breaks ties by original atom index (as does the CUDA library).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_err;

size_t g_bf_threshold = 1000;   // src/config.rs DEFAULT_BRUTE_FORCE_THRESHOLD
size_t g_par_threshold = 300;   // src/config.rs DEFAULT_PARALLEL_THRESHOLD

struct Mat3 {
  double m[3][3];  // m[row][col]; columns are the lattice vectors
};

// Rust `f as i32`: truncation toward zero, saturating, NaN -> 0.
inline int32_t sat_i32(double x) {
  if (std::isnan(x)) return 0;
  if (x >= 2147483647.0) return std::numeric_limits<int32_t>::max();
  if (x <= -2147483648.0) return std::numeric_limits<int32_t>::min();
  return static_cast<int32_t>(x);
}

// Rust `f as usize` (64-bit): truncation, negatives and NaN -> 0, saturating.
inline uint64_t sat_u64(double x) {
  if (!(x > 0.0)) return 0;
  if (x >= 18446744073709551616.0) return std::numeric_limits<uint64_t>::max();
  return static_cast<uint64_t>(x);
}

// Rust f64::min / f64::max: a NaN operand is ignored.
inline double fmin_rs(double a, double b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}
inline double fmax_rs(double a, double b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a > b ? a : b;
}

inline void matvec(const Mat3& a, double v0, double v1, double v2, double out[3]) {
  for (int r = 0; r < 3; ++r) {
    double t = a.m[r][0] * v0 + a.m[r][1] * v1;
    out[r] = t + a.m[r][2] * v2;
  }
}

inline double norm2(double a, double b, double c) {
  double t = a * a + b * b;
  return t + c * c;
}

// nalgebra try_inverse for a 3x3 matrix (cofactor expansion on the first row).
bool invert3(const Mat3& a, Mat3& inv) {
  const double m11 = a.m[0][0], m12 = a.m[0][1], m13 = a.m[0][2];
  const double m21 = a.m[1][0], m22 = a.m[1][1], m23 = a.m[1][2];
  const double m31 = a.m[2][0], m32 = a.m[2][1], m33 = a.m[2][2];
  const double c_a = m22 * m33 - m32 * m23;
  const double c_b = m21 * m33 - m31 * m23;
  const double c_c = m21 * m32 - m31 * m22;
  double det = m11 * c_a - m12 * c_b;
  det = det + m13 * c_c;
  if (det == 0.0) return false;
  inv.m[0][0] = c_a / det;
  inv.m[0][1] = (m13 * m32 - m33 * m12) / det;
  inv.m[0][2] = (m12 * m23 - m22 * m13) / det;
  inv.m[1][0] = -c_b / det;
  inv.m[1][1] = (m11 * m33 - m31 * m13) / det;
  inv.m[1][2] = (m13 * m21 - m23 * m11) / det;
  inv.m[2][0] = c_c / det;
  inv.m[2][1] = (m12 * m31 - m32 * m11) / det;
  inv.m[2][2] = (m11 * m22 - m21 * m12) / det;
  return true;
}

struct Cell {
  Mat3 h;
  Mat3 hinv;
  bool pbc[3];
};

bool make_cell(const double* h9, const bool pbc[3], Cell& c) {
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) c.h.m[r][k] = h9[3 * r + k];
  for (int a = 0; a < 3; ++a) c.pbc[a] = pbc[a];
  if (!invert3(c.h, c.hinv)) {
    g_err = "Cell matrix is not invertible";
    return false;
  }
  return true;
}

// src/cell.rs:45-50
void perp_widths(const Cell& c, double w[3]) {
  for (int r = 0; r < 3; ++r)
    w[r] = 1.0 / std::sqrt(norm2(c.hinv.m[r][0], c.hinv.m[r][1], c.hinv.m[r][2]));
}

// src/single.rs:21-58 (auto-box: origin at 0, no periodicity)
bool auto_box(const double* pos, size_t n, double cutoff, Cell& c) {
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) {
      double v = pos[3 * i + a];
      if (v < lo[a]) lo[a] = v;
      if (v > hi[a]) hi[a] = v;
    }
  const double margin = cutoff + 1.0;
  double h9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < 3; ++a) h9[4 * a] = (hi[a] - lo[a]) + 2.0 * margin;
  const bool nopbc[3] = {false, false, false};
  return make_cell(h9, nopbc, c);
}

inline uint64_t spread_bits3(uint64_t x) {
  x &= 0x1fffffULL;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

inline double clamp_rs(double v, double lo, double hi) {
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;  // NaN passes through
}

// src/search.rs:1169-1175
inline uint64_t morton_of_frac(const double f[3]) {
  const double scale = 2097152.0;  // 2^21
  uint64_t q[3];
  for (int a = 0; a < 3; ++a) q[a] = sat_u64(clamp_rs(f[a], 0.0, 0.999999) * scale);
  return spread_bits3(q[0]) | (spread_bits3(q[1]) << 1) | (spread_bits3(q[2]) << 2);
}

// Euclidean division (src/search.rs:1162-1166)
inline void div_mod(int32_t v, int32_t m, int32_t& rem, int32_t& quot) {
  int32_t q = v / m;
  int32_t r = v % m;
  if (r < 0) {
    r += m;
    q -= 1;
  }
  rem = r;
  quot = q;
}

struct Grid {
  int64_t nb[3];
  int32_t ns[3];
  std::vector<int64_t> bin_rank;    // linear bin -> Morton rank
  std::vector<int64_t> starts;      // rank -> first slot (size total+1)
  std::vector<int64_t> particles;   // slot -> original index
  std::vector<double> px, py, pz;   // wrapped positions per slot
  std::vector<int32_t> sx, sy, sz;  // wrap shifts per slot
  double basis[3][3];               // basis[a] = H * e_a / nb_a
  double origin[3];
  double radius;
};

// src/search.rs:92-264
void build_grid(const Cell& c, const double* pos, size_t n, double cutoff, Grid& g) {
  std::vector<std::pair<uint64_t, int64_t>> keyed(n);
  for (size_t i = 0; i < n; ++i) {
    double f[3];
    matvec(c.hinv, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], f);
    for (int a = 0; a < 3; ++a) f[a] = f[a] - std::floor(f[a]);
    keyed[i] = {morton_of_frac(f), (int64_t)i};
  }
  std::sort(keyed.begin(), keyed.end());  // key, then original index

  double w[3];
  perp_widths(c, w);
  for (int a = 0; a < 3; ++a) {
    uint64_t b = sat_u64(std::floor(w[a] / cutoff));
    g.nb[a] = (int64_t)std::max<uint64_t>(b, 1);
  }
  const int64_t total = g.nb[0] * g.nb[1] * g.nb[2];

  {
    std::vector<std::pair<uint64_t, int64_t>> bm(total);
    for (int64_t i = 0; i < total; ++i) {
      uint64_t bx = i % g.nb[0];
      uint64_t by = (i / g.nb[0]) % g.nb[1];
      uint64_t bz = i / (g.nb[0] * g.nb[1]);
      bm[i] = {spread_bits3(bx) | (spread_bits3(by) << 1) | (spread_bits3(bz) << 2), i};
    }
    std::sort(bm.begin(), bm.end());
    g.bin_rank.assign(total, 0);
    for (int64_t r = 0; r < total; ++r) g.bin_rank[bm[r].second] = r;
  }

  for (int a = 0; a < 3; ++a) g.ns[a] = sat_i32(std::ceil((cutoff * (double)g.nb[a]) / w[a]));

  auto bin_of = [&](const double u[3]) {
    int64_t b[3];
    for (int a = 0; a < 3; ++a) {
      uint64_t q = sat_u64(u[a] * (double)g.nb[a]);
      b[a] = (int64_t)std::min<uint64_t>(q, (uint64_t)(g.nb[a] - 1));
    }
    return g.bin_rank[b[0] + g.nb[0] * (b[1] + g.nb[1] * b[2])];
  };

  std::vector<int64_t> counts(total, 0);
  for (auto& kv : keyed) {
    const double* p = pos + 3 * kv.second;
    double f[3], u[3];
    matvec(c.hinv, p[0], p[1], p[2], f);
    for (int a = 0; a < 3; ++a) u[a] = f[a] - std::floor(f[a]);
    counts[bin_of(u)] += 1;
  }
  g.starts.assign(total + 1, 0);
  int64_t acc = 0;
  for (int64_t r = 0; r < total; ++r) {
    g.starts[r] = acc;
    acc += counts[r];
  }
  g.starts[total] = acc;

  g.px.assign(n + 8, 0.0);
  g.py.assign(n + 8, 0.0);
  g.pz.assign(n + 8, 0.0);
  g.sx.assign(n, 0);
  g.sy.assign(n, 0);
  g.sz.assign(n, 0);
  g.particles.assign(n, 0);
  std::vector<int64_t> fill(g.starts.begin(), g.starts.end() - 1);
  for (auto& kv : keyed) {
    const double* p = pos + 3 * kv.second;
    double f[3], fl[3], u[3];
    matvec(c.hinv, p[0], p[1], p[2], f);
    int32_t s[3];
    for (int a = 0; a < 3; ++a) {
      fl[a] = std::floor(f[a]);
      s[a] = sat_i32(-fl[a]);
    }
    double sv[3];
    matvec(c.h, (double)(-s[0]), (double)(-s[1]), (double)(-s[2]), sv);
    for (int a = 0; a < 3; ++a) u[a] = f[a] - fl[a];
    const int64_t slot = fill[bin_of(u)]++;
    g.px[slot] = p[0] - sv[0];
    g.py[slot] = p[1] - sv[1];
    g.pz[slot] = p[2] - sv[2];
    g.sx[slot] = s[0];
    g.sy[slot] = s[1];
    g.sz[slot] = s[2];
    g.particles[slot] = kv.second;
  }

  double vb[3][3];
  matvec(c.h, 1.0 / (double)g.nb[0], 0.0, 0.0, vb[0]);
  matvec(c.h, 0.0, 1.0 / (double)g.nb[1], 0.0, vb[1]);
  matvec(c.h, 0.0, 0.0, 1.0 / (double)g.nb[2], vb[2]);
  matvec(c.h, 0.5 / (double)g.nb[0], 0.5 / (double)g.nb[1], 0.5 / (double)g.nb[2], g.origin);
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) g.basis[a][k] = vb[a][k];
  double d[4];
  {
    double t[3];
    for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] + vb[1][k]) + vb[2][k];
    d[0] = norm2(t[0], t[1], t[2]);
    for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] + vb[1][k]) - vb[2][k];
    d[1] = norm2(t[0], t[1], t[2]);
    for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] - vb[1][k]) + vb[2][k];
    d[2] = norm2(t[0], t[1], t[2]);
    for (int k = 0; k < 3; ++k) t[k] = (vb[0][k] - vb[1][k]) - vb[2][k];
    d[3] = norm2(t[0], t[1], t[2]);
  }
  const double mx = fmax_rs(fmax_rs(fmax_rs(d[0], d[1]), d[2]), d[3]);
  g.radius = 0.5 * std::sqrt(mx);
}

struct AxisEntry {
  int32_t bin;
  int32_t shift;
  double vec[3];
};

// Visits, in the reference's canonical order, every (slot j, image shift) that
// passes the half-list predicate and d2 < max_sq for sorted atom p, calling
// hit(j_orig, s[3], d2).  src/search.rs:448-576 and :1080-1159.
template <class Hit>
void visit_atom(const Cell& c, const Grid& g, int64_t p, double max_sq, Hit&& hit) {
  const double pix = g.px[p], piy = g.py[p], piz = g.pz[p];
  const int32_t six = g.sx[p], siy = g.sy[p], siz = g.sz[p];
  double fi[3];
  matvec(c.hinv, pix, piy, piz, fi);
  int32_t home[3];
  for (int a = 0; a < 3; ++a) {
    int32_t b = sat_i32(fi[a] * (double)g.nb[a]);
    home[a] = std::min<int32_t>(b, (int32_t)g.nb[a] - 1);
  }
  const int64_t io = g.particles[p];

  // Per-axis stencil tables (OffsetList); a small inline buffer avoids a heap
  // allocation per atom in the common case.
  AxisEntry inline_buf[3][16];
  std::vector<AxisEntry> heap_buf[3];
  const AxisEntry* ax_begin[3];
  int32_t ax_len[3];
  for (int a = 0; a < 3; ++a) {
    const int32_t len = 2 * g.ns[a] + 1;
    AxisEntry* dst = inline_buf[a];
    if (len > 16) {
      heap_buf[a].resize(len);
      dst = heap_buf[a].data();
    }
    for (int32_t d = -g.ns[a]; d <= g.ns[a]; ++d) {
      AxisEntry& e = dst[d + g.ns[a]];
      div_mod(home[a] + d, (int32_t)g.nb[a], e.bin, e.shift);
      for (int k = 0; k < 3; ++k) e.vec[k] = c.h.m[k][a] * (double)e.shift;
    }
    ax_begin[a] = dst;
    ax_len[a] = len;
  }
  const double pl = std::sqrt(max_sq) + g.radius;
  const double pl2 = pl * pl;

  const double* gx = g.px.data();
  const double* gy = g.py.data();
  const double* gz = g.pz.data();
  const int64_t* gp = g.particles.data();
  for (int32_t ix = 0; ix < ax_len[0]; ++ix) {
    const AxisEntry& ex = ax_begin[0][ix];
    double cx[3];
    for (int k = 0; k < 3; ++k) cx[k] = g.origin[k] + g.basis[0][k] * (double)ex.bin;
    for (int32_t iy = 0; iy < ax_len[1]; ++iy) {
      const AxisEntry& ey = ax_begin[1][iy];
      double cxy[3];
      for (int k = 0; k < 3; ++k) cxy[k] = cx[k] + g.basis[1][k] * (double)ey.bin;
      for (int32_t iz = 0; iz < ax_len[2]; ++iz) {
        const AxisEntry& ez = ax_begin[2][iz];
        double off[3], cs[3];
        for (int k = 0; k < 3; ++k) {
          double tc = cxy[k] + g.basis[2][k] * (double)ez.bin;
          off[k] = (ex.vec[k] + ey.vec[k]) + ez.vec[k];
          cs[k] = tc + off[k];
        }
        if (norm2(cs[0] - pix, cs[1] - piy, cs[2] - piz) > pl2) continue;
        const int64_t lin = ex.bin + g.nb[0] * (ey.bin + g.nb[1] * (int64_t)ez.bin);
        const int64_t rk = g.bin_rank[lin];
        const int64_t b0 = g.starts[rk], b1 = g.starts[rk + 1];
        if (b0 == b1) continue;
        const bool shifted = ex.shift != 0 || ey.shift != 0 || ez.shift != 0;
        // Blocks of 8 candidates: the distance loop has no branch and
        // vectorises like the reference's f64x4 loop (the SoA arrays carry 8
        // padding entries, so the last block may read past b1 harmlessly).
        for (int64_t q0 = b0; q0 < b1; q0 += 8) {
          double d2v[8];
          for (int t = 0; t < 8; ++t) {
            const double dx = (gx[q0 + t] - pix) + off[0];
            const double dy = (gy[q0 + t] - piy) + off[1];
            const double dz = (gz[q0 + t] - piz) + off[2];
            d2v[t] = norm2(dx, dy, dz);
          }
          const int tn = (int)std::min<int64_t>(8, b1 - q0);
          unsigned mask = 0;
          for (int t = 0; t < 8; ++t) mask |= (unsigned)(d2v[t] < max_sq) << t;
          mask &= (1u << tn) - 1u;
          while (mask) {
            const int t = __builtin_ctz(mask);
            mask &= mask - 1u;
            const int64_t q = q0 + t;
            const int64_t jo = gp[q];
            if (io < jo || (io == jo && shifted)) {
              int32_t s[3] = {(g.sx[q] - six) + ex.shift, (g.sy[q] - siy) + ey.shift,
                              (g.sz[q] - siz) + ez.shift};
              hit(io, jo, s, d2v[t]);
            }
          }
        }
      }
    }
  }
}

struct Edges {
  std::vector<int64_t> ei, ej;
  std::vector<int32_t> sh;
  void push(int64_t i, int64_t j, const int32_t s[3]) {
    ei.push_back(i);
    ej.push_back(j);
    sh.push_back(s[0]);
    sh.push_back(s[1]);
    sh.push_back(s[2]);
  }
};

template <class F>
void parallel_for(int64_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 2) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  // Chunking like rayon's with_min_len(n / (threads * 64)) (src/search.rs:296-297).
  const int64_t chunk = std::max<int64_t>(1, n / ((int64_t)nthreads * 64));
  std::atomic<int64_t> next{0};
  auto worker = [&]() {
    for (;;) {
      int64_t b = next.fetch_add(chunk);
      if (b >= n) break;
      int64_t e = std::min(n, b + chunk);
      for (int64_t i = b; i < e; ++i) f(i);
    }
  };
  std::vector<std::thread> ts;
  for (int t = 1; t < nthreads; ++t) ts.emplace_back(worker);
  worker();
  for (auto& t : ts) t.join();
}

// Two-pass count / exclusive scan / fill over sorted atoms
// (src/search.rs:291-342 and :344-446); k lists at once.
void grid_search(const Cell& c, const Grid& g, const std::vector<double>& rc_sq_sorted,
                 bool disjoint, int nthreads, std::vector<Edges>& out_sorted) {
  const int64_t n = (int64_t)g.particles.size();
  const size_t k = rc_sq_sorted.size();
  const double max_sq = rc_sq_sorted.back();
  std::vector<uint32_t> counts((size_t)n * k, 0);
  parallel_for(n, nthreads, [&](int64_t p) {
    uint32_t* cnt = &counts[(size_t)p * k];
    visit_atom(c, g, p, max_sq, [&](int64_t, int64_t, const int32_t*, double d2) {
      for (size_t q = 0; q < k; ++q)
        if (d2 < rc_sq_sorted[q]) {
          cnt[q] += 1;
          if (disjoint) break;
        }
    });
  });
  std::vector<int64_t> offs((size_t)n * k);
  std::vector<int64_t> totals(k, 0);
  for (size_t q = 0; q < k; ++q) {
    int64_t acc = 0;
    for (int64_t p = 0; p < n; ++p) {
      offs[(size_t)p * k + q] = acc;
      acc += counts[(size_t)p * k + q];
    }
    totals[q] = acc;
  }
  out_sorted.assign(k, Edges());
  for (size_t q = 0; q < k; ++q) {
    out_sorted[q].ei.resize(totals[q]);
    out_sorted[q].ej.resize(totals[q]);
    out_sorted[q].sh.resize(3 * totals[q]);
  }
  parallel_for(n, nthreads, [&](int64_t p) {
    int64_t at_inline[16];
    std::vector<int64_t> at_heap;
    int64_t* at = at_inline;
    if (k > 16) {
      at_heap.resize(k);
      at = at_heap.data();
    }
    for (size_t q = 0; q < k; ++q) at[q] = offs[(size_t)p * k + q];
    visit_atom(c, g, p, max_sq, [&](int64_t io, int64_t jo, const int32_t* s, double d2) {
      for (size_t q = 0; q < k; ++q)
        if (d2 < rc_sq_sorted[q]) {
          const int64_t w = at[q]++;
          out_sorted[q].ei[w] = io;
          out_sorted[q].ej[w] = jo;
          out_sorted[q].sh[3 * w] = s[0];
          out_sorted[q].sh[3 * w + 1] = s[1];
          out_sorted[q].sh[3 * w + 2] = s[2];
          if (disjoint) break;
        }
    });
  });
}

// src/cell.rs:74-93
inline void mic(const Cell& c, const double* ri, const double* rj, int32_t s[3], double disp[3]) {
  double df[3];
  matvec(c.hinv, rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2], df);
  double sf[3];
  for (int a = 0; a < 3; ++a) sf[a] = c.pbc[a] ? -std::round(df[a]) : 0.0;
  for (int a = 0; a < 3; ++a) s[a] = sat_i32(sf[a]);
  double hv[3];
  matvec(c.h, sf[0], sf[1], sf[2], hv);
  for (int a = 0; a < 3; ++a) disp[a] = (rj[a] + hv[a]) - ri[a];
}

// src/search.rs:1187-1292 (isolated, raw positions) and :1319-1405 (MIC).
void brute_force(const Cell& c, const double* pos, size_t n,
                 const std::vector<double>& rc_sq_sorted, bool disjoint,
                 std::vector<Edges>& out_sorted) {
  const size_t k = rc_sq_sorted.size();
  const double max_sq = rc_sq_sorted.back();
  out_sorted.assign(k, Edges());
  const bool isolated = !c.pbc[0] && !c.pbc[1] && !c.pbc[2];
  const int32_t zero[3] = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    const double* ri = pos + 3 * i;
    for (size_t j = i + 1; j < n; ++j) {
      const double* rj = pos + 3 * j;
      int32_t s[3] = {0, 0, 0};
      double d2;
      if (isolated) {
        // brute_force_search_simd: d = p_j - p_i on the raw positions.  The
        // multi-cutoff brute force takes the MIC route instead, which for
        // pbc = (F,F,F) adds an exact zero image and gives the same d2.
        d2 = norm2(rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]);
      } else {
        double disp[3];
        mic(c, ri, rj, s, disp);
        d2 = norm2(disp[0], disp[1], disp[2]);
      }
      if (!(d2 < max_sq)) continue;
      for (size_t q = 0; q < k; ++q)
        if (d2 < rc_sq_sorted[q]) {
          out_sorted[q].push(i, j, isolated ? zero : s);
          if (disjoint) break;
        }
    }
  }
}

// One system, k cutoffs (k == 1 is the single-cutoff path).  `multi` selects
// the multi-cutoff driver (auto-box margin and mic_safe use the max cutoff).
bool search_system(const double* pos, size_t n, const double* h9, const bool* pbc,
                   const std::vector<double>& cutoffs, bool disjoint, int nthreads,
                   std::vector<Edges>& out) {
  const size_t k = cutoffs.size();
  out.assign(k, Edges());
  if (n == 0 || k == 0) return true;
  double max_rc = NAN;
  for (double r : cutoffs) max_rc = fmax_rs(max_rc, r);
  Cell c;
  if (h9) {
    if (!make_cell(h9, pbc, c)) return false;
  } else {
    if (!auto_box(pos, n, max_rc, c)) return false;
  }
  double w[3];
  perp_widths(c, w);
  const double min_w = fmin_rs(fmin_rs(w[0], w[1]), w[2]);
  const bool mic_safe = max_rc * 2.0 < min_w;

  // Stable ascending order of the cutoffs (src/search.rs:354-360).
  std::vector<size_t> order(k);
  for (size_t q = 0; q < k; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t a, size_t b) { return cutoffs[a] < cutoffs[b]; });
  std::vector<double> rc_sq(k);
  for (size_t q = 0; q < k; ++q) rc_sq[q] = cutoffs[order[q]] * cutoffs[order[q]];

  std::vector<Edges> sorted_out;
  if (n < g_bf_threshold && mic_safe) {
    brute_force(c, pos, n, rc_sq, disjoint, sorted_out);
  } else {
    Grid g;
    build_grid(c, pos, n, max_rc, g);
    grid_search(c, g, rc_sq, disjoint, nthreads, sorted_out);
  }
  for (size_t q = 0; q < k; ++q) out[order[q]] = std::move(sorted_out[q]);
  return true;
}

}  // namespace

extern "C" {

struct orc_edges {
  int64_t n_edges;
  int64_t* edge_i;
  int64_t* edge_j;
  int32_t* shift;
};

const char* orc_last_error(void) { return g_err.c_str(); }

void orc_set_thresholds(int64_t brute_force, int64_t parallel) {
  g_bf_threshold = (size_t)brute_force;
  g_par_threshold = (size_t)parallel;
}

void orc_edges_free(orc_edges* e) {
  if (!e) return;
  std::free(e->edge_i);
  std::free(e->edge_j);
  std::free(e->shift);
  e->edge_i = e->edge_j = nullptr;
  e->shift = nullptr;
  e->n_edges = 0;
}

static void export_edges(const Edges& src, int64_t offset, orc_edges* dst) {
  const size_t m = src.ei.size();
  dst->n_edges = (int64_t)m;
  dst->edge_i = (int64_t*)std::malloc(sizeof(int64_t) * (m ? m : 1));
  dst->edge_j = (int64_t*)std::malloc(sizeof(int64_t) * (m ? m : 1));
  dst->shift = (int32_t*)std::malloc(sizeof(int32_t) * 3 * (m ? m : 1));
  for (size_t e = 0; e < m; ++e) {
    dst->edge_i[e] = src.ei[e] + offset;
    dst->edge_j[e] = src.ej[e] + offset;
  }
  if (m) std::memcpy(dst->shift, src.sh.data(), sizeof(int32_t) * 3 * m);
}

int orc_cell_inverse(const double h9[9], double inv9[9]) {
  Mat3 a, b;
  for (int r = 0; r < 9; ++r) a.m[r / 3][r % 3] = h9[r];
  if (!invert3(a, b)) return 1;
  for (int r = 0; r < 9; ++r) inv9[r] = b.m[r / 3][r % 3];
  return 0;
}

int orc_perp_widths(const double h9[9], double w[3]) {
  Cell c;
  const bool p[3] = {true, true, true};
  if (!make_cell(h9, p, c)) return 1;
  perp_widths(c, w);
  return 0;
}

// src/cell.rs:52-72
int orc_wrap(const double h9[9], const uint8_t pbc[3], const double p[3], double out[3]) {
  Cell c;
  const bool pb[3] = {pbc[0] != 0, pbc[1] != 0, pbc[2] != 0};
  if (!make_cell(h9, pb, c)) return 1;
  double f[3];
  matvec(c.hinv, p[0], p[1], p[2], f);
  for (int a = 0; a < 3; ++a)
    if (pb[a]) f[a] = f[a] - std::floor(f[a]);
  matvec(c.h, f[0], f[1], f[2], out);
  return 0;
}

int orc_mic(const double h9[9], const uint8_t pbc[3], const double ri[3], const double rj[3],
            int32_t s[3], double disp[3]) {
  Cell c;
  const bool pb[3] = {pbc[0] != 0, pbc[1] != 0, pbc[2] != 0};
  if (!make_cell(h9, pb, c)) return 1;
  mic(c, ri, rj, s, disp);
  return 0;
}

uint64_t orc_zorder(const double f[3]) { return morton_of_frac(f); }

// Cell-list structure for tests: num_bins[3], n_search[3], bin of each
// original atom (as linear index bx + nx*(by + ny*bz)) and the slot order.
int orc_cell_list(const double* pos, int64_t n, const double h9[9], double cutoff,
                  int64_t num_bins[3], int32_t n_search[3], int64_t* particles,
                  int64_t* atom_bin_linear) {
  Cell c;
  const bool p[3] = {true, true, true};
  if (!make_cell(h9, p, c)) return 1;
  Grid g;
  build_grid(c, pos, (size_t)n, cutoff, g);
  for (int a = 0; a < 3; ++a) {
    num_bins[a] = g.nb[a];
    n_search[a] = g.ns[a];
  }
  std::vector<int64_t> rank_to_lin(g.bin_rank.size());
  for (size_t l = 0; l < g.bin_rank.size(); ++l) rank_to_lin[g.bin_rank[l]] = (int64_t)l;
  for (int64_t r = 0; r + 1 < (int64_t)g.starts.size(); ++r)
    for (int64_t s = g.starts[r]; s < g.starts[r + 1]; ++s)
      atom_bin_linear[g.particles[s]] = rank_to_lin[r];
  for (int64_t s = 0; s < n; ++s) particles[s] = g.particles[s];
  return 0;
}

// Single system.  h9 == NULL selects the auto-box (isolated) cell.
int orc_search_single(const double* pos, int64_t n, const double* h9, const uint8_t* pbc,
                      double cutoff, int nthreads, orc_edges* out) {
  const bool pb[3] = {pbc ? pbc[0] != 0 : false, pbc ? pbc[1] != 0 : false,
                      pbc ? pbc[2] != 0 : false};
  std::vector<Edges> r;
  if (!search_system(pos, (size_t)n, h9, pb, {cutoff}, false, nthreads, r)) return 1;
  export_edges(r[0], 0, out);
  return 0;
}

int orc_search_single_multi(const double* pos, int64_t n, const double* h9,
                            const uint8_t* pbc, const double* cutoffs, int32_t k,
                            int disjoint, int nthreads, orc_edges* outs) {
  const bool pb[3] = {pbc ? pbc[0] != 0 : false, pbc ? pbc[1] != 0 : false,
                      pbc ? pbc[2] != 0 : false};
  std::vector<double> cs(cutoffs, cutoffs + k);
  std::vector<Edges> r;
  if (!search_system(pos, (size_t)n, h9, pb, cs, disjoint != 0, nthreads, r)) return 1;
  for (int32_t q = 0; q < k; ++q) export_edges(r[q], 0, &outs[q]);
  return 0;
}

// Batched systems (src/batch.rs:10-290).  cells: n_cells x 9 (rows of H,
// columns = lattice vectors), pbcs: n_cells x 3, has_cell: n_cells flags
// (0 = auto-box).  cells == NULL means every system is auto-boxed.
int orc_search_batch(const double* pos, int64_t n, const int32_t* batch, int64_t n_batch,
                     const double* cells, const uint8_t* pbcs, const uint8_t* has_cell,
                     int64_t n_cells, const double* cutoffs, int32_t k, int disjoint,
                     int nthreads, orc_edges* outs) {
  if (n_batch != n) {
    g_err = "positions and batch must have the same length";
    return 1;
  }
  std::vector<std::pair<int64_t, int64_t>> sys;
  if (n > 0 && k > 0) {
    int64_t start = 0;
    for (int64_t i = 1; i < n; ++i)
      if (batch[i] != batch[i - 1]) {
        sys.push_back({start, i});
        start = i;
      }
    sys.push_back({start, n});
    const int64_t have = cells ? n_cells : (int64_t)sys.size();
    if (have < (int64_t)sys.size()) {
      g_err = "Expected at least " + std::to_string(sys.size()) + " cells, but got " +
              std::to_string(have);
      return 1;
    }
  }
  std::vector<double> cs(cutoffs, cutoffs + k);
  const int64_t ns = (int64_t)sys.size();
  std::vector<std::vector<Edges>> per(ns);
  std::vector<int> ok(ns, 1);
  std::vector<std::string> errs(ns);
  // Systems run in parallel, each with a serial inner search (rayon nests
  // both levels; the edge order does not depend on the scheduling).
  parallel_for(ns, nthreads, [&](int64_t s) {
    const int64_t b = sys[s].first, e = sys[s].second;
    const double* h9 = nullptr;
    bool pb[3] = {false, false, false};
    if (cells && has_cell[s]) {
      h9 = cells + 9 * s;
      for (int a = 0; a < 3; ++a) pb[a] = pbcs[3 * s + a] != 0;
    }
    if (!search_system(pos + 3 * b, (size_t)(e - b), h9, pb, cs, disjoint != 0, 1, per[s])) {
      ok[s] = 0;
      errs[s] = g_err;
    }
  });
  for (int64_t s = 0; s < ns; ++s)
    if (!ok[s]) {
      g_err = errs[s];
      return 1;
    }
  for (int32_t q = 0; q < k; ++q) {
    Edges all;
    for (int64_t s = 0; s < ns; ++s) {
      const Edges& x = per[s][q];
      for (size_t e = 0; e < x.ei.size(); ++e) {
        all.ei.push_back(x.ei[e] + sys[s].first);
        all.ej.push_back(x.ej[e] + sys[s].first);
      }
      all.sh.insert(all.sh.end(), x.sh.begin(), x.sh.end());
    }
    export_edges(all, 0, &outs[q]);
  }
  return 0;
}

// Output options beyond the reference's half list (spec.md:100-108 asks for
// a directed option; RUST_API.md:89-90 documents it as "double the edges and
// negate the shifts").  Half edge e = (i, j, S):
//   vector   d = (r_j - r_i) + H.S, component k: (r_j,k - r_i,k) +
//            ((H[k][0] S0 + H[k][1] S1) + H[k][2] S2)   (no H term when the
//            system has no cell: d = r_j - r_i)
//   distance sqrt((d0^2 + d1^2) + d2^2), correctly rounded
//   directed the m half edges, then their reverses (j, i, -S, -d, same distance)
// Outputs: ei_out [2 mo] ([src | dst]), sh_out [3 mo], vec [3 mo], dist [mo],
// mo = directed ? 2m : m; any output may be NULL.
void orc_edge_extras(const double* pos, const double* h9, const int64_t* ei, const int64_t* ej,
                     const int32_t* sh, int64_t m, int directed, int64_t* ei_out,
                     int32_t* sh_out, double* vec, double* dist) {
  const int64_t mo = directed ? 2 * m : m;
  for (int64_t e = 0; e < m; ++e) {
    const int64_t i = ei[e], j = ej[e];
    const int32_t* s = sh + 3 * e;
    double d[3];
    for (int k = 0; k < 3; ++k) {
      const double rel = pos[3 * j + k] - pos[3 * i + k];
      if (h9) {
        const double hs = (h9[3 * k] * (double)s[0] + h9[3 * k + 1] * (double)s[1]) +
                          h9[3 * k + 2] * (double)s[2];
        d[k] = rel + hs;
      } else {
        d[k] = rel;
      }
    }
    const double r = std::sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
    if (ei_out) {
      ei_out[e] = i;
      ei_out[mo + e] = j;
      if (directed) {
        ei_out[m + e] = j;
        ei_out[mo + m + e] = i;
      }
    }
    for (int k = 0; k < 3; ++k) {
      if (sh_out) {
        sh_out[3 * e + k] = s[k];
        if (directed) sh_out[3 * (m + e) + k] = -s[k];
      }
      if (vec) {
        vec[3 * e + k] = d[k];
        if (directed) vec[3 * (m + e) + k] = -d[k];
      }
    }
    if (dist) {
      dist[e] = r;
      if (directed) dist[m + e] = r;
    }
  }
}

}  // extern "C"
