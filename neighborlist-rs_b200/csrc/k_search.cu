// k_search.cu -- stencil pair search: count pass and emit pass.
//
// One warp per (sorted) atom i.  The warp walks i's stencil cells in the
// reference's order (x outer, y, z inner; src/search.rs:492-496): lanes first
// evaluate 32 stencil cells at a time (periodic bin, image shift, prune test
// of src/search.rs:500-505, bin range), then the warp visits the surviving
// cells in order and tests 32 candidates j per step in bin storage order.
// Hits are compacted with ballot/popc, so the emit pass writes each atom's
// edges contiguously and in canonical order at the offset produced by the
// exclusive scan of the count pass (src/search.rs:291-342).
//
// Pair test (exact f64, no FMA): d = (x_j - x_i) + off, d2 = (dx^2 + dy^2) +
// dz^2 < rc^2, with the half-list predicate i < j or (i == j and image != 0)
// (src/search.rs:540-553).  Multi-cutoff: lane q keeps the count / cursor of
// cutoff q of the pass (src/search.rs:729-1078).
//
// Brute force (src/search.rs:1187-1405): the same warp machinery with
// candidates j = i+1..n-1 in index order, on raw positions (isolated) or with
// the round-based minimum image (src/cell.rs:74-93).
#include "k_traverse.cuh"

namespace nlb {

namespace {

constexpr int kWarpsPerBlock = 8;

// Visits sorted atom p's candidates in canonical order; all 32 lanes call
// sink(hit, d2, i_orig, j_orig, shift) once per candidate step.
template <class Sink>
__device__ __forceinline__ void visit_grid_atom(const GridParams& g, const GridBuffers& b,
                                                int64_t p, double max_sq, Sink& sink) {
  const int lane = threadIdx.x & 31;
  const double pix = b.px[p], piy = b.py[p], piz = b.pz[p];
  const SlotMeta mi = b.meta[p];
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

  for (int64_t c0 = 0; c0 < n_cells; c0 += 32) {
    const int64_t c = c0 + lane;
    bool ok = c < n_cells;
    int64_t b0 = 0, b1 = 0;
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
        const int64_t lin = bin[0] + (int64_t)g.nb[0] * (bin[1] + (int64_t)g.nb[1] * bin[2]);
        const int32_t r = b.rank_of_bin[lin];
        b0 = b.bin_start[r];
        b1 = b.bin_start[r + 1];
        ok = b1 > b0;
      }
    }
    unsigned cells = __ballot_sync(0xffffffffu, ok);
    while (cells) {
      const int src = __ffs(cells) - 1;
      cells &= cells - 1;
      const int64_t j0 = __shfl_sync(0xffffffffu, b0, src);
      const int64_t j1 = __shfl_sync(0xffffffffu, b1, src);
      const double ox = shfl_d(off[0], src), oy = shfl_d(off[1], src), oz = shfl_d(off[2], src);
      int32_t cshift[3];
      cshift[0] = __shfl_sync(0xffffffffu, sh[0], src);
      cshift[1] = __shfl_sync(0xffffffffu, sh[1], src);
      cshift[2] = __shfl_sync(0xffffffffu, sh[2], src);
      const bool shifted = (cshift[0] | cshift[1] | cshift[2]) != 0;
      for (int64_t jb = j0; jb < j1; jb += 32) {
        const int64_t j = jb + lane;
        bool hit = false;
        double d2 = 0.0;
        int32_t jo = 0;
        int32_t s[3] = {0, 0, 0};
        if (j < j1) {
          const double dx = dadd(dsub(b.px[j], pix), ox);
          const double dy = dadd(dsub(b.py[j], piy), oy);
          const double dz = dadd(dsub(b.pz[j], piz), oz);
          d2 = norm2(dx, dy, dz);
          const SlotMeta mj = b.meta[j];
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

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    k_grid_count(GridParams g, GridBuffers b, int64_t n, CutoffSet cs, uint32_t* __restrict__ counts) {
  const int64_t p = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (p >= n) return;  // warp-uniform
  CountSink sink{&cs, 0u};
  visit_grid_atom(g, b, p, cs.max_sq, sink);
  const int lane = threadIdx.x & 31;
  if (lane < cs.k) counts[(int64_t)lane * (n + 1) + p] = sink.cnt;
  if (p == n - 1 && lane < cs.k) counts[(int64_t)lane * (n + 1) + n] = 0;
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    k_grid_emit(GridParams g, GridBuffers b, int64_t n, CutoffSet cs,
                const int64_t* __restrict__ offs, EmitTargets t) {
  const int64_t p = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (p >= n) return;
  const int lane = threadIdx.x & 31;
  int64_t cur = 0;
  if (lane < cs.k) {
    const int64_t row = (int64_t)lane * (n + 1);
    cur = t.base[lane] + (offs[row + p] - offs[row]);
  }
  EmitSink sink{&cs, &t, cur, t.index_offset};
  visit_grid_atom(g, b, p, cs.max_sq, sink);
}

// ---------------------------------------------------------------- brute force

template <class Sink>
__device__ __forceinline__ void visit_brute_atom(const BruteParams& bp, const double* pos,
                                                 int64_t n, int64_t i, double max_sq, Sink& sink) {
  const int lane = threadIdx.x & 31;
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  for (int64_t jb = i + 1; jb < n; jb += 32) {
    const int64_t j = jb + lane;
    bool hit = false;
    double d2 = 0.0;
    int32_t s[3] = {0, 0, 0};
    if (j < n) {
      const double xj = pos[3 * j], yj = pos[3 * j + 1], zj = pos[3 * j + 2];
      if (bp.mode == kBruteRaw) {
        d2 = norm2(dsub(xj, xi), dsub(yj, yi), dsub(zj, zi));
      } else {
        double df[3];
        matvec(bp.hinv, dsub(xj, xi), dsub(yj, yi), dsub(zj, zi), df);
        double sf[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          sf[a] = bp.pbc[a] ? -round(df[a]) : 0.0;
          s[a] = sat_i32(sf[a]);
        }
        double hv[3];
        matvec(bp.h, sf[0], sf[1], sf[2], hv);
        d2 = norm2(dsub(dadd(xj, hv[0]), xi), dsub(dadd(yj, hv[1]), yi), dsub(dadd(zj, hv[2]), zi));
      }
      hit = d2 < max_sq;
    }
    sink(hit, d2, (int32_t)i, (int32_t)j, s);
  }
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    k_brute_count(BruteParams bp, const double* __restrict__ pos, int64_t n, CutoffSet cs,
                  uint32_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (i >= n) return;
  CountSink sink{&cs, 0u};
  visit_brute_atom(bp, pos, n, i, cs.max_sq, sink);
  const int lane = threadIdx.x & 31;
  if (lane < cs.k) counts[(int64_t)lane * (n + 1) + i] = sink.cnt;
  if (i == n - 1 && lane < cs.k) counts[(int64_t)lane * (n + 1) + n] = 0;
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    k_brute_emit(BruteParams bp, const double* __restrict__ pos, int64_t n, CutoffSet cs,
                 const int64_t* __restrict__ offs, EmitTargets t) {
  const int64_t i = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (i >= n) return;
  const int lane = threadIdx.x & 31;
  int64_t cur = 0;
  if (lane < cs.k) {
    const int64_t row = (int64_t)lane * (n + 1);
    cur = t.base[lane] + (offs[row + i] - offs[row]);
  }
  EmitSink sink{&cs, &t, cur, t.index_offset};
  visit_brute_atom(bp, pos, n, i, cs.max_sq, sink);
}

inline unsigned blocks_for(int64_t n) {
  return (unsigned)((n + kWarpsPerBlock - 1) / kWarpsPerBlock);
}

}  // namespace

void launch_grid_count(const GridParams& g, const GridBuffers& b, int64_t n,
                       const CutoffSet& cs, uint32_t* counts, cudaStream_t s) {
  k_grid_count<<<blocks_for(n), kWarpsPerBlock * 32, 0, s>>>(g, b, n, cs, counts);
  note_launches(1);
}

void launch_grid_emit(const GridParams& g, const GridBuffers& b, int64_t n, const CutoffSet& cs,
                      const int64_t* offs, const EmitTargets& t, cudaStream_t s) {
  k_grid_emit<<<blocks_for(n), kWarpsPerBlock * 32, 0, s>>>(g, b, n, cs, offs, t);
  note_launches(1);
}

void launch_brute_count(const BruteParams& bp, const double* pos, int64_t n, const CutoffSet& cs,
                        uint32_t* counts, cudaStream_t s) {
  k_brute_count<<<blocks_for(n), kWarpsPerBlock * 32, 0, s>>>(bp, pos, n, cs, counts);
  note_launches(1);
}

void launch_brute_emit(const BruteParams& bp, const double* pos, int64_t n, const CutoffSet& cs,
                       const int64_t* offs, const EmitTargets& t, cudaStream_t s) {
  k_brute_emit<<<blocks_for(n), kWarpsPerBlock * 32, 0, s>>>(bp, pos, n, cs, offs, t);
  note_launches(1);
}

}  // namespace nlb
