// k_batch.cu -- many small systems per launch (src/batch.rs:10-290).
//
//   k_plan        one warp per system: auto-box bounds (when the system has no
//                 cell), H^-1, perpendicular widths, mic_safe and the
//                 brute-force / cell-list dispatch, and the grid (bins,
//                 stencil half-widths, prune geometry) -- the same f64
//                 expressions, in the same order, as the host planner
//                 (nlb_geometry.cpp) and the reference (src/single.rs:8-164,
//                 src/search.rs:119-246).
//   k_batch_count / k_batch_emit
//                 persistent CTAs pull systems from a work queue (largest
//                 first).  A CTA keeps its whole system in shared memory:
//                 for the cell list it sorts the atoms by (bin Morton code,
//                 atom Morton key, index) -- bin code order is bin rank
//                 order, so no rank table is needed -- and finds a stencil
//                 cell's atoms by binary search on the sorted codes.  Warps
//                 then walk one atom each, exactly like the single-system
//                 kernels, and count or emit through the shared sinks.
// Per-atom counts of all systems form one flat row per cutoff; one exclusive
// scan gives every system's global edge offsets, so the emit pass writes the
// concatenated, exact-sized output (systems in input order) directly.
#include <algorithm>
#include <cstring>
#include <vector>

#include "k_traverse.cuh"

namespace nlb {

namespace {

__device__ __forceinline__ double dfmin(double a, double b) {
  if (a != a) return b;
  if (b != b) return a;
  return a < b ? a : b;
}
__device__ __forceinline__ double dfmax(double a, double b) {
  if (a != a) return b;
  if (b != b) return a;
  return a > b ? a : b;
}

// Device mirror of make_cell (nalgebra 3x3 inverse).  Returns false if det == 0.
__device__ bool dev_make_cell(const double* h, double* hinv) {
  const double m11 = h[0], m12 = h[1], m13 = h[2];
  const double m21 = h[3], m22 = h[4], m23 = h[5];
  const double m31 = h[6], m32 = h[7], m33 = h[8];
  const double ca = dsub(dmul(m22, m33), dmul(m32, m23));
  const double cb = dsub(dmul(m21, m33), dmul(m31, m23));
  const double cc = dsub(dmul(m21, m32), dmul(m31, m22));
  const double det = dadd(dsub(dmul(m11, ca), dmul(m12, cb)), dmul(m13, cc));
  if (det == 0.0) return false;
  hinv[0] = __ddiv_rn(ca, det);
  hinv[1] = __ddiv_rn(dsub(dmul(m13, m32), dmul(m33, m12)), det);
  hinv[2] = __ddiv_rn(dsub(dmul(m12, m23), dmul(m22, m13)), det);
  hinv[3] = __ddiv_rn(-cb, det);
  hinv[4] = __ddiv_rn(dsub(dmul(m11, m33), dmul(m31, m13)), det);
  hinv[5] = __ddiv_rn(dsub(dmul(m13, m21), dmul(m23, m11)), det);
  hinv[6] = __ddiv_rn(cc, det);
  hinv[7] = __ddiv_rn(dsub(dmul(m12, m31), dmul(m32, m11)), det);
  hinv[8] = __ddiv_rn(dsub(dmul(m11, m22), dmul(m21, m12)), det);
  return true;
}

__device__ void dev_widths(const double* hinv, double* w) {
  for (int r = 0; r < 3; ++r)
    w[r] = __ddiv_rn(1.0, __dsqrt_rn(norm2(hinv[3 * r], hinv[3 * r + 1], hinv[3 * r + 2])));
}

__device__ __forceinline__ void mv_plain(const double* m, double v0, double v1, double v2,
                                         double* out) {
  matvec(m, v0, v1, v2, out);
}

// Device mirror of plan_grid (host) for cutoff rc.
__device__ void dev_plan_grid(const double* w, double rc, GridParams& g) {
  int64_t total = 1;
  for (int a = 0; a < 3; ++a) {
    uint64_t b = sat_u64(floor(__ddiv_rn(w[a], rc)));
    if (b < 1) b = 1;
    if (b > 2147483647ull) b = 2147483647ull;
    g.nb[a] = (int32_t)b;
    total *= (int64_t)g.nb[a];
    if (total > ((int64_t)1 << 40)) total = ((int64_t)1 << 40);
  }
  g.total_bins = total;
  for (int a = 0; a < 3; ++a) g.ns[a] = sat_i32(ceil(__ddiv_rn(dmul(rc, (double)g.nb[a]), w[a])));
  double vb[3][3];
  mv_plain(g.h, __ddiv_rn(1.0, (double)g.nb[0]), 0.0, 0.0, vb[0]);
  mv_plain(g.h, 0.0, __ddiv_rn(1.0, (double)g.nb[1]), 0.0, vb[1]);
  mv_plain(g.h, 0.0, 0.0, __ddiv_rn(1.0, (double)g.nb[2]), vb[2]);
  mv_plain(g.h, __ddiv_rn(0.5, (double)g.nb[0]), __ddiv_rn(0.5, (double)g.nb[1]),
           __ddiv_rn(0.5, (double)g.nb[2]), g.origin);
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) g.basis[a][k] = vb[a][k];
  double d[4], t[3];
  for (int k = 0; k < 3; ++k) t[k] = dadd(dadd(vb[0][k], vb[1][k]), vb[2][k]);
  d[0] = norm2(t[0], t[1], t[2]);
  for (int k = 0; k < 3; ++k) t[k] = dsub(dadd(vb[0][k], vb[1][k]), vb[2][k]);
  d[1] = norm2(t[0], t[1], t[2]);
  for (int k = 0; k < 3; ++k) t[k] = dadd(dsub(vb[0][k], vb[1][k]), vb[2][k]);
  d[2] = norm2(t[0], t[1], t[2]);
  for (int k = 0; k < 3; ++k) t[k] = dsub(dsub(vb[0][k], vb[1][k]), vb[2][k]);
  d[3] = norm2(t[0], t[1], t[2]);
  const double mx = dfmax(dfmax(dfmax(d[0], d[1]), d[2]), d[3]);
  const double radius = dmul(0.5, __dsqrt_rn(mx));
  g.radius = radius;
  const double pl = dadd(__dsqrt_rn(dmul(rc, rc)), radius);
  g.prune_sq = dmul(pl, pl);
}

__global__ void k_plan(const double* __restrict__ pos, const int64_t* __restrict__ starts,
                       int32_t s0, int32_t s1, const double* __restrict__ cells,
                       const uint8_t* __restrict__ pbcs, const uint8_t* __restrict__ has_cell,
                       double rc_max_all, uint64_t bf_threshold, int multi, int64_t run_start,
                       SysPlan* __restrict__ plans, int32_t* __restrict__ error_flag,
                       const double* __restrict__ sys_rc) {
  const int lane = threadIdx.x & 31;
  const int32_t s = s0 + blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (s >= s1) return;
  const double rc_max = sys_rc ? sys_rc[s] : rc_max_all;
  const int64_t b = starts[s], e = starts[s + 1];
  const bool own_cell = cells && has_cell && has_cell[s];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (!own_cell) {
    for (int64_t i = b + lane; i < e; i += 32)
      for (int a = 0; a < 3; ++a) {
        const double v = pos[3 * i + a];
        if (v < lo[a]) lo[a] = v;
        if (v > hi[a]) hi[a] = v;
      }
    for (int a = 0; a < 3; ++a)
      for (int o = 16; o > 0; o >>= 1) {
        const double l2 = __shfl_xor_sync(0xffffffffu, lo[a], o);
        const double h2 = __shfl_xor_sync(0xffffffffu, hi[a], o);
        if (l2 < lo[a]) lo[a] = l2;
        if (h2 > hi[a]) hi[a] = h2;
      }
  }
  if (lane != 0) return;
  SysPlan P;
  P.start = b;
  P.n = (int32_t)(e - b);
  P.slot = b - run_start;
  P.rc_sq = dmul(rc_max, rc_max);
  GridParams& g = P.g;
  for (int i = 0; i < 9; ++i) g.h[i] = 0.0;
  if (own_cell) {
    for (int i = 0; i < 9; ++i) g.h[i] = cells[9 * s + i];
    for (int a = 0; a < 3; ++a) P.pbc[a] = pbcs ? (pbcs[3 * s + a] != 0) : 1;
  } else {
    const double margin = dadd(rc_max, 1.0);
    for (int a = 0; a < 3; ++a) g.h[4 * a] = dadd(dsub(hi[a], lo[a]), dmul(2.0, margin));
    P.pbc[0] = P.pbc[1] = P.pbc[2] = 0;
  }
  if (!dev_make_cell(g.h, g.hinv)) {
    P.method = -1;
    atomicExch(error_flag, 1);
    plans[s - s0] = P;
    return;
  }
  double w[3];
  dev_widths(g.hinv, w);
  const double min_w = dfmin(dfmin(w[0], w[1]), w[2]);
  const bool mic_safe = dmul(rc_max, 2.0) < min_w;
  if ((uint64_t)P.n < bf_threshold && mic_safe) {
    const bool isolated = !P.pbc[0] && !P.pbc[1] && !P.pbc[2];
    P.method = (isolated && !multi) ? 0 : 1;
    g.total_bins = 0;
  } else {
    P.method = 2;
    dev_plan_grid(w, rc_max, g);
    for (int a = 0; a < 3; ++a)
      if (g.ns[a] < 0 || g.ns[a] > (1 << 20)) {
        atomicExch(error_flag, 2);
        P.method = -1;  // (the host reports it; the passes skip the system)
      }
  }
  plans[s - s0] = P;
}

// ------------------------------------------------------------------ shared memory

struct SmemView {
  uint64_t* bcode;  // [cap] sort key 1 (bin Morton code), sorted
  uint64_t* key;    // [cap] sort key 2 (atom Morton key); after the sort, the
                    // boxes of the 32-slot blocks (6 doubles each: cap >= 32)
  int32_t* idx;     // [cap] sort key 3 (local atom index)
  double* px;       // [cap] wrapped (cell list) or raw (brute) positions
  double* py;
  double* pz;
  SlotMeta* meta;   // [cap]
};

__device__ __forceinline__ SmemView smem_view(unsigned char* base, int cap) {
  SmemView v;
  v.bcode = reinterpret_cast<uint64_t*>(base);
  v.key = v.bcode + cap;
  v.px = reinterpret_cast<double*>(v.key + cap);
  v.py = v.px + cap;
  v.pz = v.py + cap;
  v.meta = reinterpret_cast<SlotMeta*>(v.pz + cap);
  v.idx = reinterpret_cast<int32_t*>(v.meta + cap);
  return v;
}

__device__ __forceinline__ bool triple_less(uint64_t a0, uint64_t a1, int32_t a2, uint64_t b0,
                                            uint64_t b1, int32_t b2) {
  if (a0 != b0) return a0 < b0;
  if (a1 != b1) return a1 < b1;
  return a2 < b2;
}

__device__ void sort_triples(const SmemView& v, int n) {
  int p = 1;
  while (p < n) p <<= 1;
  for (int i = n + threadIdx.x; i < p; i += blockDim.x) {
    v.bcode[i] = ~0ull;
    v.key[i] = ~0ull;
    v.idx[i] = 0x7fffffff;
  }
  __syncthreads();
  for (int size = 2; size <= p; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < p; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const bool gt = triple_less(v.bcode[j], v.key[j], v.idx[j], v.bcode[i], v.key[i], v.idx[i]);
          if (gt == up) {
            uint64_t t0 = v.bcode[i];
            v.bcode[i] = v.bcode[j];
            v.bcode[j] = t0;
            uint64_t t1 = v.key[i];
            v.key[i] = v.key[j];
            v.key[j] = t1;
            int32_t t2 = v.idx[i];
            v.idx[i] = v.idx[j];
            v.idx[j] = t2;
          }
        }
      }
      __syncthreads();
    }
}

__device__ __forceinline__ uint64_t bin_code(int32_t bx, int32_t by, int32_t bz) {
  return spread_bits3((uint64_t)bx) | (spread_bits3((uint64_t)by) << 1) |
         (spread_bits3((uint64_t)bz) << 2);
}

// Loads one system into shared memory.  Cell list: sorted SoA in canonical
// order (bin rank, Morton key, index).  Brute force: raw positions.
__device__ void load_system(const SysPlan& P, const double* __restrict__ pos, const SmemView& v) {
  const int n = P.n;
  const double* sp = pos + 3 * P.start;
  if (P.method != 2) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      v.px[i] = sp[3 * i];
      v.py[i] = sp[3 * i + 1];
      v.pz[i] = sp[3 * i + 2];
    }
    __syncthreads();
    return;
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const AtomWrap w = wrap_atom(P.g, sp[3 * i], sp[3 * i + 1], sp[3 * i + 2]);
    v.bcode[i] = bin_code(w.bin[0], w.bin[1], w.bin[2]);
    v.key[i] = w.key;
    v.idx[i] = i;
  }
  __syncthreads();
  sort_triples(v, n);
  for (int p = threadIdx.x; p < n; p += blockDim.x) {
    const int i = v.idx[p];
    const AtomWrap w = wrap_atom(P.g, sp[3 * i], sp[3 * i + 1], sp[3 * i + 2]);
    v.px[p] = w.wx;
    v.py[p] = w.wy;
    v.pz[p] = w.wz;
    SlotMeta m;
    m.sx = w.s[0];
    m.sy = w.s[1];
    m.sz = w.s[2];
    m.orig = i;
    v.meta[p] = m;
  }
  __syncthreads();
  // FP64 bounding box of each aligned block of 32 sorted slots (blocks are
  // Morton-contiguous, so the boxes are tight); a block with a non-finite
  // coordinate gets the infinite box (never pruned).
  double* box = reinterpret_cast<double*>(v.key);
  const int lane = threadIdx.x & 31;
  for (int a = threadIdx.x >> 5; a < (n + 31) >> 5; a += blockDim.x >> 5) {
    const int p = 32 * a + lane;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool bad = false;
    if (p < n) {
      const double c[3] = {v.px[p], v.py[p], v.pz[p]};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = hi[k] = c[k];
        bad = bad || !isfinite(c[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
      for (int o = 16; o > 0; o >>= 1) {
        const double l2 = __shfl_xor_sync(0xffffffffu, lo[k], o);
        const double h2 = __shfl_xor_sync(0xffffffffu, hi[k], o);
        lo[k] = l2 < lo[k] ? l2 : lo[k];
        hi[k] = h2 > hi[k] ? h2 : hi[k];
      }
    if (__any_sync(0xffffffffu, bad))
      for (int k = 0; k < 3; ++k) {
        lo[k] = -INFINITY;
        hi[k] = INFINITY;
      }
    if (lane < 6) box[6 * a + lane] = lane < 3 ? lo[lane] : hi[lane - 3];
  }
  __syncthreads();
}

// Whether the block's box may hold a candidate within the cutoff of the
// atom at t = (atom - image offset): the box distance, shortened per axis by
// a slack far above the rounding of the pair test's own differences, against
// max_sq (1 + 1e-12).  Only removes candidates that cannot hit.
__device__ __forceinline__ bool block_near(const double* __restrict__ box, int a, const double* t,
                                           double thr) {
  const double* B = box + 6 * a;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double lo = B[k], hi = B[3 + k];
    double d = dsub(lo, t[k]);
    const double d2 = dsub(t[k], hi);
    d = d2 > d ? d2 : d;
    const double slack = dmul(1e-14, dadd(fabs(t[k]), fmax(fabs(lo), fabs(hi))));
    d = d > slack ? dsub(d, slack) : 0.0;
    s = dadd(s, dmul(d, d));
  }
  return !(s > thr);
}

// First index in [0, n) whose code is >= c.
__device__ __forceinline__ int lower_bound_code(const uint64_t* codes, int n, uint64_t c) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (codes[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

template <class Sink>
__device__ __forceinline__ void visit_smem_grid_atom(const SysPlan& P, const SmemView& v, int p,
                                                     double max_sq, Sink& sink) {
  const GridParams& g = P.g;
  const int lane = threadIdx.x & 31;
  const int n = P.n;
  const double pix = v.px[p], piy = v.py[p], piz = v.pz[p];
  const SlotMeta mi = v.meta[p];
  double fi[3];
  matvec(g.hinv, pix, piy, piz, fi);
  int32_t home[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int32_t hb = sat_i32(dmul(fi[a], (double)g.nb[a]));
    home[a] = hb < g.nb[a] - 1 ? hb : g.nb[a] - 1;
  }
  const int32_t ny = 2 * g.ns[1] + 1, nz = 2 * g.ns[2] + 1;
  const int64_t n_cells = (int64_t)(2 * g.ns[0] + 1) * ny * nz;
  const double* box = reinterpret_cast<const double*>(v.key);
  const double thr = dmul(max_sq, 1.0 + 1e-12);
  for (int64_t c0 = 0; c0 < n_cells; c0 += 32) {
    const int64_t c = c0 + lane;
    bool ok = c < n_cells;
    int b0 = 0, b1 = 0;
    uint32_t cmask = 0;
    double off[3] = {0.0, 0.0, 0.0};
    int32_t sh[3] = {0, 0, 0};
    if (ok) {
      const int32_t ix = (int32_t)(c / ((int64_t)ny * nz));
      const int32_t rem = (int32_t)(c - (int64_t)ix * ny * nz);
      const int32_t iy = rem / nz, iz = rem - (rem / nz) * nz;
      int32_t bin[3];
      div_mod(home[0] + ix - g.ns[0], g.nb[0], bin[0], sh[0]);
      div_mod(home[1] + iy - g.ns[1], g.nb[1], bin[1], sh[1]);
      div_mod(home[2] + iz - g.ns[2], g.nb[2], bin[2], sh[2]);
      double cs[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        off[k] = dadd(dadd(dmul(g.h[3 * k], (double)sh[0]), dmul(g.h[3 * k + 1], (double)sh[1])),
                      dmul(g.h[3 * k + 2], (double)sh[2]));
        double t = dadd(g.origin[k], dmul(g.basis[0][k], (double)bin[0]));
        t = dadd(t, dmul(g.basis[1][k], (double)bin[1]));
        t = dadd(t, dmul(g.basis[2][k], (double)bin[2]));
        cs[k] = dadd(t, off[k]);
      }
      if (norm2(dsub(cs[0], pix), dsub(cs[1], piy), dsub(cs[2], piz)) > g.prune_sq) {
        ok = false;
      } else {
        if (g.total_bins == 1) {  // (one bin: every image cell holds all the atoms)
          b0 = 0;
          b1 = n;
        } else {
          const uint64_t code = bin_code(bin[0], bin[1], bin[2]);
          b0 = lower_bound_code(v.bcode, n, code);
          b1 = code == ~0ull ? n : lower_bound_code(v.bcode, n, code + 1);
        }
        ok = b1 > b0;
        if (ok) {
          // Candidate chunks [b0 + 32k, ...) of this cell whose slots' block
          // boxes may hold a hit (chunks from the 33rd on are always kept).
          const double t[3] = {dsub(pix, off[0]), dsub(piy, off[1]), dsub(piz, off[2])};
          const int nch = (b1 - b0 + 31) >> 5;
          const int lim = nch < 32 ? nch : 32;
          for (int k = 0; k < lim; ++k) {
            const int f = b0 + 32 * k;
            const int l = (f + 32 < b1 ? f + 32 : b1) - 1;
            if (block_near(box, f >> 5, t, thr) ||
                ((l >> 5) != (f >> 5) && block_near(box, l >> 5, t, thr)))
              cmask |= 1u << k;
          }
          ok = cmask != 0 || nch > 32;
        }
      }
    }
    unsigned cells = __ballot_sync(0xffffffffu, ok);
    while (cells) {
      const int src = __ffs(cells) - 1;
      cells &= cells - 1;
      const int j0 = __shfl_sync(0xffffffffu, b0, src);
      const int j1 = __shfl_sync(0xffffffffu, b1, src);
      const double ox = shfl_d(off[0], src), oy = shfl_d(off[1], src), oz = shfl_d(off[2], src);
      int32_t cshift[3];
      cshift[0] = __shfl_sync(0xffffffffu, sh[0], src);
      cshift[1] = __shfl_sync(0xffffffffu, sh[1], src);
      cshift[2] = __shfl_sync(0xffffffffu, sh[2], src);
      const bool shifted = (cshift[0] | cshift[1] | cshift[2]) != 0;
      const uint32_t ck = __shfl_sync(0xffffffffu, cmask, src);
      for (int jb = j0, k = 0; jb < j1; jb += 32, ++k) {
        if (k < 32 && !((ck >> k) & 1u)) continue;
        sink.at(jb, cshift);
        const int j = jb + lane;
        bool hit = false;
        double d2 = 0.0;
        int32_t jo = 0;
        int32_t s[3] = {0, 0, 0};
        if (j < j1) {
          const double dx = dadd(dsub(v.px[j], pix), ox);
          const double dy = dadd(dsub(v.py[j], piy), oy);
          const double dz = dadd(dsub(v.pz[j], piz), oz);
          d2 = norm2(dx, dy, dz);
          const SlotMeta mj = v.meta[j];
          jo = mj.orig;
          hit = d2 < max_sq && (mi.orig < jo || (mi.orig == jo && shifted));
          s[0] = (mj.sx - mi.sx) + cshift[0];
          s[1] = (mj.sy - mi.sy) + cshift[1];
          s[2] = (mj.sz - mi.sz) + cshift[2];
        }
        sink(hit, d2, mi.orig, jo, s);
      }
    }
  }
}

template <class Sink>
__device__ __forceinline__ void visit_smem_brute_atom(const SysPlan& P, const SmemView& v, int i,
                                                      double max_sq, Sink& sink) {
  const int lane = threadIdx.x & 31;
  const int n = P.n;
  const double xi = v.px[i], yi = v.py[i], zi = v.pz[i];
  const int32_t no_shift[3] = {0, 0, 0};
  for (int jb = i + 1; jb < n; jb += 32) {
    sink.at(jb, no_shift);
    const int j = jb + lane;
    bool hit = false;
    double d2 = 0.0;
    int32_t s[3] = {0, 0, 0};
    if (j < n) {
      const double xj = v.px[j], yj = v.py[j], zj = v.pz[j];
      if (P.method == 0) {
        d2 = norm2(dsub(xj, xi), dsub(yj, yi), dsub(zj, zi));
      } else {
        double df[3];
        matvec(P.g.hinv, dsub(xj, xi), dsub(yj, yi), dsub(zj, zi), df);
        double sf[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          sf[a] = P.pbc[a] ? -round(df[a]) : 0.0;
          s[a] = sat_i32(sf[a]);
        }
        double hv[3];
        matvec(P.g.h, sf[0], sf[1], sf[2], hv);
        d2 = norm2(dsub(dadd(xj, hv[0]), xi), dsub(dadd(yj, hv[1]), yi), dsub(dadd(zj, hv[2]), zi));
      }
      hit = d2 < max_sq;
    }
    sink(hit, d2, i, j, s);
  }
}

// Pulls the next work item (system, first atom) for the whole CTA; system -1
// when the queue is empty.
__device__ __forceinline__ int2 next_item(int* work, const int2* items, int n_items) {
  __shared__ int s_next;
  if (threadIdx.x == 0) s_next = atomicAdd(work, 1);
  __syncthreads();
  const int w = s_next;
  __syncthreads();
  return w < n_items ? items[w] : make_int2(-1, 0);
}

__device__ __forceinline__ void load_plan(const SysPlan* plans, int s, SysPlan& sp_smem) {
  const int words = (int)(sizeof(SysPlan) / sizeof(int32_t));
  const int32_t* src = reinterpret_cast<const int32_t*>(plans + s);
  int32_t* dst = reinterpret_cast<int32_t*>(&sp_smem);
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// Per-system cutoff (CutoffSet.k == 0): the pass's single cutoff is the
// system's own (SysPlan.rc_sq).
__device__ __forceinline__ void system_cutoff(const CutoffSet& cs, const SysPlan& P,
                                              CutoffSet& out) {
  out = cs;
  out.k = 1;
  out.rc_sq[0] = P.rc_sq;
  out.max_sq = P.rc_sq;
  out.lower_sq = -1.0;
  out.disjoint = 0;
}

// Record sink of the single-cutoff count pass: besides the count, every
// candidate step of the atom with at least one hit becomes a record {hit
// mask, first candidate, the cell's image shift in three signed 10-bit
// fields}.  Lane l buffers the atom's l-th pending record; 32 pending
// records (and the atom's last ones) are flushed as one segment whose header
// holds the atom's run slot, its edges in earlier segments, the record count
// and the system.  Each atom's first segment was reserved with its warp's
// other atoms of the work item (one atomic per warp and item: a global
// atomic per atom serialised the pass on the counter); it is written even
// when empty, and further segments (atoms with more than 32 records) are
// taken one by one.  A segment or a shift that does not fit sets the
// overflow flag: the emit pass then recomputes instead of expanding.
struct RecSink {
  const CutoffSet* cs;
  BatchRecords rb;
  uint32_t cnt = 0;  // lane 0: the atom's edge count
  uint32_t r_mask = 0, r_j = 0, r_sh = 0;  // lane l: pending record l
  int n_rec = 0, e_done = 0, e_buf = 0;  // warp-uniform
  int32_t p_abs = 0, sys = 0;
  int first_sg = -1;  // the atom's reserved segment (-1: used)
  uint32_t cur_j = 0, cur_sh = 0;
  bool sh_ok = true;

  __device__ __forceinline__ void at(int32_t jb, const int32_t* csh) {
    cur_j = (uint32_t)jb;
    sh_ok = csh[0] >= -511 && csh[0] <= 511 && csh[1] >= -511 && csh[1] <= 511 &&
            csh[2] >= -511 && csh[2] <= 511;
    cur_sh = ((uint32_t)csh[0] & 1023u) | (((uint32_t)csh[1] & 1023u) << 10) |
             (((uint32_t)csh[2] & 1023u) << 20);
  }
  __device__ __forceinline__ void flush(bool last) {
    if (n_rec == 0 && !(last && first_sg >= 0)) return;
    const int lane = threadIdx.x & 31;
    int sg = first_sg;
    if (sg >= 0) {
      first_sg = -1;
    } else {
      if (lane == 0) sg = atomicAdd(rb.seg_top, 1);
      sg = __shfl_sync(0xffffffffu, sg, 0);
    }
    if (sg < rb.seg_cap) {
      if (lane < n_rec) {
        uint32_t* r = rb.rec + ((size_t)sg * 32 + lane) * 3;
        r[0] = r_mask;
        r[1] = r_j;
        r[2] = r_sh;
      }
      if (lane == 0) rb.seg_hdr[sg] = make_int4(p_abs, e_done, n_rec, sys);
    } else if (lane == 0) {
      *rb.overflow = 1;
    }
    e_done += e_buf;
    e_buf = 0;
    n_rec = 0;
  }
  __device__ __forceinline__ void operator()(bool hit, double d2, int32_t, int32_t,
                                             const int32_t*) {
    const int lane = threadIdx.x & 31;
    const bool h = hit && d2 < cs->rc_sq[0] && !(cs->disjoint && d2 < cs->lower_sq);
    const unsigned m = __ballot_sync(0xffffffffu, h);
    if (!m) return;
    if (lane == 0) cnt += __popc(m);
    if (!sh_ok && lane == 0) *rb.overflow = 1;
    if (lane == n_rec) {
      r_mask = m;
      r_j = cur_j;
      r_sh = cur_sh;
    }
    ++n_rec;
    e_buf += __popc(m);
    if (n_rec == 32) flush(false);
  }
};

template <int THREADS, bool REC>
// 80 registers per thread for 64 / 128 / 256-thread CTAs.  The 512-thread count
// spills at the 64-register budget of two CTAs per SM; one CTA per SM with
// room for ~106 registers measured 7-8 % faster.
__global__ void __launch_bounds__(THREADS, THREADS >= 512 ? 1 : 768 / THREADS)
    k_batch_count(const SysPlan* __restrict__ plans, const int2* __restrict__ items, int n_items,
                  int chunk, const double* __restrict__ pos, int cap, CutoffSet cs,
                  uint32_t* __restrict__ counts, int64_t row, int* __restrict__ work,
                  BatchRecords rb) {
  constexpr int kWarps = THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ SysPlan P;
  __shared__ CutoffSet cs_sys;
  const SmemView v = smem_view(smem, cap);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    const int2 item = next_item(work, items, n_items);
    if (item.x < 0) break;
    load_plan(plans, item.x, P);
    if (P.method < 0) continue;
    const CutoffSet* csp = &cs;
    if (cs.k == 0) {
      if (threadIdx.x == 0) system_cutoff(cs, P, cs_sys);
      __syncthreads();
      csp = &cs_sys;
    }
    load_system(P, pos, v);
    const int p_end = min(P.n, item.y + chunk);
    if (REC) {
      // The sorted meta of this item's atoms (brute force: unsorted, no
      // wrap shifts) for the expansion pass.
      for (int p = item.y + threadIdx.x; p < p_end; p += blockDim.x) {
        SlotMeta m{0, 0, 0, p};
        if (P.method == 2) m = v.meta[p];
        rb.meta[P.slot + p] = m;
      }
    }
    // (REC: this warp's atoms of the item reserve their first segments)
    int seg_base = 0;
    if (REC) {
      const int mine = p_end - item.y > warp ? (p_end - item.y - warp + kWarps - 1) / kWarps : 0;
      if (lane == 0 && mine > 0) seg_base = atomicAdd(rb.seg_top, mine);
      seg_base = __shfl_sync(0xffffffffu, seg_base, 0);
    }
    for (int p = item.y + warp, q = 0; p < p_end; p += kWarps, ++q) {
      if (REC) {
        RecSink sink{csp, rb};
        sink.p_abs = P.slot + p;
        sink.sys = item.x;
        sink.first_sg = seg_base + q;
        if (P.method == 2)
          visit_smem_grid_atom(P, v, p, csp->max_sq, sink);
        else
          visit_smem_brute_atom(P, v, p, csp->max_sq, sink);
        sink.flush(true);
        if (lane == 0) counts[P.slot + p] = sink.cnt;
      } else {
        CountSink sink{csp, 0u};
        if (P.method == 2)
          visit_smem_grid_atom(P, v, p, csp->max_sq, sink);
        else
          visit_smem_brute_atom(P, v, p, csp->max_sq, sink);
        if (lane < csp->k) counts[(int64_t)lane * row + P.slot + p] = sink.cnt;
      }
    }
    __syncthreads();
  }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS)
    k_batch_emit(const SysPlan* __restrict__ plans, const int2* __restrict__ items, int n_items,
                 int chunk, const double* __restrict__ pos, int cap, CutoffSet cs,
                 const int64_t* __restrict__ offs, int64_t row, EmitTargets t,
                 int* __restrict__ work) {
  constexpr int kWarps = THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ SysPlan P;
  __shared__ CutoffSet cs_sys;
  __shared__ EmitTargets1 t_blk;
  const SmemView v = smem_view(smem, cap);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool blocks = t.system_blocks && cs.k == 0;
  // Device-sized outputs: nothing is written when the offsets scan gave up,
  // or when any list of this pass holds more edges than the arena (the host
  // grows the arena and emits again).
  if (t.scan_error && *t.scan_error != 0) return;
  if (t.capacity > 0) {
    for (int q = 0; q < cs.k; ++q)
      if (offs[(int64_t)(q + 1) * row] - offs[(int64_t)q * row] > t.capacity) return;
  }
  for (;;) {
    const int2 item = next_item(work, items, n_items);
    if (item.x < 0) break;
    load_plan(plans, item.x, P);
    if (P.method < 0) continue;
    const CutoffSet* csp = &cs;
    if (cs.k == 0) {
      if (threadIdx.x == 0) {
        system_cutoff(cs, P, cs_sys);
        if (blocks) {
          // This system's edges e in [b0, b0 + m): sources at 2 b0 + (e - b0),
          // destinations at 2 b0 + m + (e - b0).
          const int64_t b0 = offs[P.slot] - offs[0];
          const int64_t m = offs[P.slot + P.n] - offs[P.slot];
          t_blk.src[0] = t.src[0] + b0;
          t_blk.dst[0] = t.src[0] + b0 + m;
          t_blk.sh[0] = t.sh[0];
        }
      }
      __syncthreads();
      csp = &cs_sys;
    }
    load_system(P, pos, v);
    const int64_t idx_off = t.local_indices ? t.index_offset : P.start + t.index_offset;
    const int p_end = min(P.n, item.y + chunk);
    for (int p = item.y + warp; p < p_end; p += kWarps) {
      int64_t cur = 0;
      if (lane < csp->k) {
        const int64_t r = (int64_t)lane * row;
        cur = t.base[lane] + (offs[r + P.slot + p] - offs[r]);
      }
      if (blocks) {
        EmitSinkT<EmitTargets1> sink{csp, &t_blk, cur, idx_off};
        if (P.method == 2)
          visit_smem_grid_atom(P, v, p, csp->max_sq, sink);
        else
          visit_smem_brute_atom(P, v, p, csp->max_sq, sink);
      } else {
        EmitSink sink{csp, &t, cur, idx_off};
        if (P.method == 2)
          visit_smem_grid_atom(P, v, p, csp->max_sq, sink);
        else
          visit_smem_brute_atom(P, v, p, csp->max_sq, sink);
      }
    }
    __syncthreads();
  }
}

__global__ void k_sys_bounds(const SysPlan* __restrict__ plans, int n_sys,
                             const int64_t* __restrict__ offs, int64_t row,
                             int64_t* __restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n_sys) out[s] = offs[plans[s].slot] - offs[0];
  if (s == n_sys) out[s] = offs[row - 1] - offs[0];
}

// Position of the k-th (from 0) set bit of m (k < popc(m)).
__device__ __forceinline__ int select_bit(uint32_t m, int k) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w >= 1; w >>= 1) {
    const int c = __popc(m & ((1u << w) - 1u));
    if (k >= c) {
      k -= c;
      m >>= w;
      pos += w;
    }
  }
  return pos;
}

// Expansion of the count pass's records into the single-cutoff list: one
// warp per segment; each record's hit lanes write (i, j, shift) at the
// atom's next slots, in record order -- the order the recomputing emit pass
// writes.  Shifts: (s_j - s_i) + the cell's image shift (cell list; zero
// wrap shifts and image for raw brute force); the minimum-image systems
// recompute the pair's shift from the raw positions exactly as the count
// pass did.
__global__ void __launch_bounds__(256, 4)
    k_batch_expand(BatchRecords rb, const SysPlan* __restrict__ plans,
                   const double* __restrict__ pos, const int64_t* __restrict__ offs, int64_t row,
                   EmitTargets t) {
  if (t.scan_error && *t.scan_error != 0) return;
  if (t.capacity > 0 && offs[row] - offs[0] > t.capacity) return;
  if (*rb.overflow) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *rb.need_recompute = 1;
    return;
  }
  const int n_seg = min(*rb.seg_top, rb.seg_cap);
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  // (the next segment's header and records are loaded while this one is
  // written)
  int sg = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int4 hdr_next = make_int4(0, 0, 0, 0);
  uint32_t rec_next[3] = {0u, 0u, 0u};
  if (sg < n_seg) {
    hdr_next = rb.seg_hdr[sg];
    const uint32_t* r = rb.rec + ((size_t)sg * 32 + lane) * 3;
    rec_next[0] = r[0];
    rec_next[1] = r[1];
    rec_next[2] = r[2];
  }
  for (; sg < n_seg; sg += warps) {
    const int4 hdr = hdr_next;
    uint32_t my_mask = 0, my_j = 0, my_sh = 0;
    if (lane < hdr.z) {
      my_mask = rec_next[0];
      my_j = rec_next[1];
      my_sh = rec_next[2];
    }
    if (sg + warps < n_seg) {
      hdr_next = rb.seg_hdr[sg + warps];
      const uint32_t* r = rb.rec + ((size_t)(sg + warps) * 32 + lane) * 3;
      rec_next[0] = r[0];
      rec_next[1] = r[1];
      rec_next[2] = r[2];
    }
    const SysPlan* P = plans + hdr.w;
    const int32_t method = P->method;
    const int64_t start = P->start;
    const int32_t slot = P->slot;
    const SlotMeta mi = rb.meta[hdr.x];
    const int64_t cur = t.base[0] + (offs[hdr.x] - offs[0]) + hdr.y;
    const int64_t idx_off = t.local_indices ? t.index_offset : start + t.index_offset;
    int64_t* src = t.src[0];
    int64_t* dst = t.dst[0];
    if (t.system_blocks) {
      // This system's list is one [src | dst] block at src[0] + 2 b0.
      const int64_t b0 = offs[slot] - offs[0];
      const int64_t m_sys = offs[slot + P->n] - offs[slot];
      src = t.src[0] + b0;
      dst = t.src[0] + b0 + m_sys;
    }
    double xi = 0.0, yi = 0.0, zi = 0.0;
    if (method == 1) {
      const double* pi = pos + 3 * (start + mi.orig);
      xi = pi[0];
      yi = pi[1];
      zi = pi[2];
    }
    // The segment's hits are consecutive in the list: hit h (records in
    // order, bits in order) goes to slot cur + h.  Each lane takes hits h =
    // lane, lane + 32, ...: its record by a binary search over the records'
    // inclusive hit counts, its candidate as that record's (h - first)-th
    // set bit; the warp's stores are contiguous.
    const int c = __popc(my_mask);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - c;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
#pragma unroll 2
    for (int h0 = 0; h0 < total; h0 += 32) {
      const int h = h0 + lane;
      int r = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int v = __shfl_sync(0xffffffffu, incl, r + step - 1);
        if (v <= h) r += step;
      }
      const uint32_t mask = __shfl_sync(0xffffffffu, my_mask, r);
      const int32_t j0 = (int32_t)__shfl_sync(0xffffffffu, my_j, r);
      const uint32_t psh = __shfl_sync(0xffffffffu, my_sh, r);
      const int first = __shfl_sync(0xffffffffu, excl, r);
      if (h < total) {
        const int jj = select_bit(mask, h - first);
        const SlotMeta mj = rb.meta[slot + j0 + jj];
        int32_t s[3];
        if (method == 1) {
          const double* pj = pos + 3 * (start + mj.orig);
          double df[3];
          matvec(P->g.hinv, dsub(pj[0], xi), dsub(pj[1], yi), dsub(pj[2], zi), df);
#pragma unroll
          for (int a = 0; a < 3; ++a) s[a] = sat_i32(P->pbc[a] ? -round(df[a]) : 0.0);
        } else {
          s[0] = (mj.sx - mi.sx) + ((int32_t)(psh << 22) >> 22);
          s[1] = (mj.sy - mi.sy) + ((int32_t)(psh << 12) >> 22);
          s[2] = (mj.sz - mi.sz) + ((int32_t)(psh << 2) >> 22);
        }
        const int64_t e = cur + h;
        src[e] = (int64_t)mi.orig + idx_off;
        dst[e] = (int64_t)mj.orig + idx_off;
        int32_t* sp = t.sh[0] + 3 * e;
        sp[0] = s[0];
        sp[1] = s[1];
        sp[2] = s[2];
      }
    }
  }
}

int grid_for(const void* func, int threads, size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

}  // namespace

size_t batch_smem_bytes(int cap) {
  return (size_t)cap * (2 * sizeof(uint64_t) + 3 * sizeof(double) + sizeof(SlotMeta) +
                        sizeof(int32_t));
}

void launch_plan(const double* pos, const int64_t* starts, int32_t s0, int32_t s1,
                 const double* cells, const uint8_t* pbcs, const uint8_t* has_cell, double rc_max,
                 uint64_t bf_threshold, int multi, int64_t run_start, SysPlan* plans,
                 int32_t* error_flag, cudaStream_t s, const double* sys_rc) {
  const int per_block = 8;
  const unsigned blocks = (unsigned)((s1 - s0 + per_block - 1) / per_block);
  k_plan<<<blocks, per_block * 32, 0, s>>>(pos, starts, s0, s1, cells, pbcs, has_cell, rc_max,
                                           bf_threshold, multi, run_start, plans, error_flag,
                                           sys_rc);
  note_launches(1);
}

void launch_sys_bounds(const SysPlan* plans, int n_sys, const int64_t* offs, int64_t row,
                       int64_t* out, cudaStream_t s) {
  k_sys_bounds<<<(unsigned)((n_sys + 1 + 127) / 128), 128, 0, s>>>(plans, n_sys, offs, row, out);
  note_launches(1);
}

const BatchShape kBatchShapeTable[kBatchShapes] = {
    // small_threads, large_threads, chunk, large_atoms
    {256, 512, 256, 512},  // default
    {128, 512, 256, 512},  // more systems in flight per SM
    {256, 256, 128, 256},  // finer items for the mid-size systems
    {128, 256, 128, 256},
    {256, 512, 128, 512},
    {512, 512, 256, 1024},  // systems up to 1024 atoms whole
    {64, 512, 256, 512},    // two warps per system: tiny systems
};

namespace {

using CountFn = decltype(&k_batch_count<256, false>);
using EmitFn = decltype(&k_batch_emit<256>);

CountFn count_fn(int threads, bool rec = false) {
  if (rec)
    return threads <= 64    ? &k_batch_count<64, true>
           : threads <= 128 ? &k_batch_count<128, true>
           : threads <= 256 ? &k_batch_count<256, true>
                            : &k_batch_count<512, true>;
  return threads <= 64    ? &k_batch_count<64, false>
         : threads <= 128 ? &k_batch_count<128, false>
         : threads <= 256 ? &k_batch_count<256, false>
                          : &k_batch_count<512, false>;
}
EmitFn emit_fn(int threads) {
  return threads <= 64    ? &k_batch_emit<64>
         : threads <= 128 ? &k_batch_emit<128>
         : threads <= 256 ? &k_batch_emit<256>
                          : &k_batch_emit<512>;
}

}  // namespace

void preload_batch_kernels() {
  // Loading a kernel's module happens on its first launch unless something
  // asks for its attributes first (lazy loading): do it for every variant.
  cudaFuncAttributes a;
  for (int threads : {64, 128, 256, 512}) {
    cudaFuncGetAttributes(&a, (const void*)count_fn(threads));
    cudaFuncGetAttributes(&a, (const void*)count_fn(threads, true));
    cudaFuncGetAttributes(&a, (const void*)emit_fn(threads));
  }
  cudaGetLastError();
}

void launch_batch_count(const SysPlan* plans, const BatchItems& w, const double* pos,
                        const CutoffSet& cs, uint32_t* counts, int64_t row, int* work2,
                        cudaStream_t s, const BatchRecords* rec) {
  const BatchShape& sh = w.shape;
  BatchRecords rb;
  std::memset(&rb, 0, sizeof(rb));
  if (rec) rb = *rec;
  if (w.n_large > 0) {
    const size_t smem = batch_smem_bytes(w.cap_large);
    const CountFn k = count_fn(sh.large_threads, rec != nullptr);
    ensure_smem_attr((const void*)k, (int)smem);
    const int grid = std::min(grid_for((const void*)k, sh.large_threads, smem), w.n_large);
    k<<<grid, sh.large_threads, smem, s>>>(plans, w.items, w.n_large, sh.chunk, pos,
                                           w.cap_large, cs, counts, row, work2, rb);
    note_launches(1);
  }
  if (w.n_small > 0) {
    const size_t smem = batch_smem_bytes(w.cap_small);
    const CountFn k = count_fn(sh.small_threads, rec != nullptr);
    ensure_smem_attr((const void*)k, (int)smem);
    const int grid = std::min(grid_for((const void*)k, sh.small_threads, smem), w.n_small);
    k<<<grid, sh.small_threads, smem, s>>>(plans, w.items + w.n_large, w.n_small, 1 << 30, pos,
                                           w.cap_small, cs, counts, row, work2 + 1, rb);
    note_launches(1);
  }
}

void launch_batch_expand(const BatchRecords& rb, const SysPlan* plans, const double* pos,
                         const int64_t* offs, int64_t row, const EmitTargets& t, cudaStream_t s) {
  const int grid = grid_for((const void*)k_batch_expand, 256, 0);
  k_batch_expand<<<grid, 256, 0, s>>>(rb, plans, pos, offs, row, t);
  note_launches(1);
}

void launch_batch_emit(const SysPlan* plans, const BatchItems& w, const double* pos,
                       const CutoffSet& cs, const int64_t* offs, int64_t row,
                       const EmitTargets& t, int* work2, cudaStream_t s) {
  const BatchShape& sh = w.shape;
  if (w.n_large > 0) {
    const size_t smem = batch_smem_bytes(w.cap_large);
    const EmitFn k = emit_fn(sh.large_threads);
    ensure_smem_attr((const void*)k, (int)smem);
    const int grid = std::min(grid_for((const void*)k, sh.large_threads, smem), w.n_large);
    k<<<grid, sh.large_threads, smem, s>>>(plans, w.items, w.n_large, sh.chunk, pos,
                                           w.cap_large, cs, offs, row, t, work2);
    note_launches(1);
  }
  if (w.n_small > 0) {
    const size_t smem = batch_smem_bytes(w.cap_small);
    const EmitFn k = emit_fn(sh.small_threads);
    ensure_smem_attr((const void*)k, (int)smem);
    const int grid = std::min(grid_for((const void*)k, sh.small_threads, smem), w.n_small);
    k<<<grid, sh.small_threads, smem, s>>>(plans, w.items + w.n_large, w.n_small, 1 << 30, pos,
                                           w.cap_small, cs, offs, row, t, work2 + 1);
    note_launches(1);
  }
}

void plan_batch_items(const int64_t* sizes, int n_sys, const BatchShape& shape,
                      std::vector<int2>& items, BatchItems& w) {
  std::vector<int32_t> order(n_sys);
  for (int i = 0; i < n_sys; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t x, int32_t y) { return sizes[x] > sizes[y]; });
  items.clear();
  w = BatchItems{};
  w.shape = shape;
  int64_t max_large = 0, max_small = 0;
  for (int32_t i : order) {
    const int64_t n = sizes[i];
    if (n > shape.large_atoms) {
      for (int64_t a = 0; a < n; a += shape.chunk) items.push_back(make_int2(i, (int)a));
      max_large = std::max(max_large, n);
    }
  }
  w.n_large = (int)items.size();
  for (int32_t i : order) {
    const int64_t n = sizes[i];
    if (n <= shape.large_atoms) {
      items.push_back(make_int2(i, 0));
      max_small = std::max(max_small, n);
    }
  }
  w.n_small = (int)items.size() - w.n_large;
  w.cap_large = 32;
  while (w.cap_large < max_large) w.cap_large <<= 1;
  w.cap_small = 32;
  while (w.cap_small < max_small) w.cap_small <<= 1;
}

}  // namespace nlb
