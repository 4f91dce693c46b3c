// k_search2.cu -- stencil search for one to four cutoffs as (atom group,
// stencil cell) pair tasks, with an FP32 pair test and an exact FP64
// guard-band recheck.
//
// Same edges, same order as k_search.cu and the reference.  The canonical
// order is (sorted atom, stencil cell in x/y/z order, candidate in bin
// order), so per-(atom, cell) edge counts, scanned in that order, give every
// (atom, cell) its exact output offset and all tasks can run in parallel:
//
// * A task is one group of at most 32 atoms of one bin (lane = atom) and one
//   stencil cell.  The cell (periodic bin, image shift, FP64 image offset,
//   bin range) is shared by the group; each lane applies the reference's
//   FP64 prune test for its own atom (src/search.rs:500-505).
// * The cell's candidates are staged 32 at a time in shared memory as FP32
//   positions relative to their bin centre (original index in .w); each lane
//   tests them in bin order against its atom: dx = x_j + (T - x_i) with the
//   cell translation T = c_cell + off - c_bin formed in FP64 and rounded once.
// * Guard band (make_guard_band): d2_32 < rc^2 - delta is a certain hit,
//   d2_32 >= rc^2 + delta a certain miss; in between, the reference's exact
//   FP64 expression (x_j - x_i) + off on the FP64 wrapped positions decides
//   (src/search.rs:540-553).  Results are identical to the FP64 kernels.
// * Several cutoffs share one traversal of the grid built at the largest
//   (CellList::par_search_multi, src/search.rs:344-435, 729-893): each
//   pair's FP32 distance is compared with every cutoff's band and an
//   ambiguous pair is rechecked once in FP64 against all of them; list q
//   then has its edges in the same canonical order.  Disjoint shells give a
//   pair to the first cutoff it falls inside (src/search.rs:845-848), so
//   list q drops the pairs inside cutoff q - 1.
// * Atoms whose home stencil differs from their stored bin (the search
//   recomputes the home bin from the wrapped position, src/search.rs:454-457;
//   this differs only within rounding of a bin face) are skipped by the
//   tasks and handled by one warp each, in FP64, with the same outputs.
#include <cmath>
#include <cstring>

#include "k_traverse.cuh"

namespace nlb {

namespace {

constexpr int kPairWarps = 8;  // warps per CTA
// Emit pass: hits of one task staged per warp before the warp writes them out
// (dynamic shared memory, kPairWarps x stage_cap 16-bit entries: lane << 11 |
// candidate offset, for cells of at most kStageCell candidates).  Grids whose
// tasks hold at most ~kStageSmall hits get the small stage; denser ones the
// large (88 KB, so that two 256-thread CTAs still fit an SM beside their
// static shared memory), which the small-task grids would pay for in L1.
constexpr int kStageSmall = 1536;
constexpr int kStageLarge = 5632;
constexpr int kStageCell = 2048;
constexpr size_t stage_smem(int cap) { return sizeof(uint16_t) * kPairWarps * (size_t)cap; }

struct CellDesc {
  int32_t b0, b1;  // candidate slots
  int32_t sh[3];   // image shift
  double off[3];   // image offset (FP64, reference order)
  double cs[3];    // bin centre + offset (FP64), the prune test's target
};

// Stencil cell c of the stencil centred on bin `home`.
__device__ __forceinline__ CellDesc describe_cell(const GridParams& g, const GridBuffers& b,
                                                  const int32_t home[3], int32_t c) {
  const int32_t ny = 2 * g.ns[1] + 1, nz = 2 * g.ns[2] + 1;
  const int32_t ix = c / (ny * nz);
  const int32_t rem = c - ix * (ny * nz);
  const int32_t iy = rem / nz, iz = rem - (rem / nz) * nz;
  CellDesc d;
  int32_t bin[3];
  div_mod(home[0] + ix - g.ns[0], g.nb[0], bin[0], d.sh[0]);
  div_mod(home[1] + iy - g.ns[1], g.nb[1], bin[1], d.sh[1]);
  div_mod(home[2] + iz - g.ns[2], g.nb[2], bin[2], d.sh[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d.off[k] = dadd(dadd(dmul(g.h[3 * k], (double)d.sh[0]), dmul(g.h[3 * k + 1], (double)d.sh[1])),
                    dmul(g.h[3 * k + 2], (double)d.sh[2]));
    double t = dadd(g.origin[k], dmul(g.basis[0][k], (double)bin[0]));
    t = dadd(t, dmul(g.basis[1][k], (double)bin[1]));
    t = dadd(t, dmul(g.basis[2][k], (double)bin[2]));
    d.cs[k] = dadd(t, d.off[k]);
  }
  const int64_t lin = bin[0] + (int64_t)g.nb[0] * (bin[1] + (int64_t)g.nb[1] * bin[2]);
  const int32_t r = b.rank_of_bin[lin];
  d.b0 = (int32_t)b.bin_start[r];
  d.b1 = (int32_t)b.bin_start[r + 1];
  return d;
}

// One warp per irregular atom: every stencil cell of its own home stencil in
// order, candidates 32 at a time across lanes (FP64, like k_search.cu), each
// candidate tested against the K cutoffs.
template <bool EMIT, int K>
__device__ void pair_irregular(const GridParams& g, const GridBuffers& b, int32_t n_cells,
                               const PairBands& pb, uint32_t* __restrict__ counts,
                               const int64_t* __restrict__ offs, const EmitTargets& t,
                               int64_t* __restrict__ dst0, int64_t gwarp, int64_t nwarps) {
  const int lane = threadIdx.x & 31;
  const int32_t n_irr = b.counters[1];
  int64_t off0[K];
#pragma unroll
  for (int q = 0; q < K; ++q) off0[q] = EMIT ? offs[q * pb.row] : 0;
  for (int64_t w = gwarp; w < n_irr; w += nwarps) {
    const int32_t p = b.irr_list[w];
    const double xi = b.px[p], yi = b.py[p], zi = b.pz[p];
    const SlotMeta mi = b.meta[p];
    double fi[3];
    matvec(g.hinv, xi, yi, zi, fi);
    int32_t home[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int32_t v = sat_i32(dmul(fi[a], (double)g.nb[a]));
      home[a] = v < g.nb[a] - 1 ? v : g.nb[a] - 1;
    }
    for (int32_t c = 0; c < n_cells; ++c) {
      const CellDesc d = describe_cell(g, b, home, c);
      const bool live = !(norm2(dsub(d.cs[0], xi), dsub(d.cs[1], yi), dsub(d.cs[2], zi)) > g.prune_sq);
      const bool shifted = (d.sh[0] | d.sh[1] | d.sh[2]) != 0;
      uint32_t cnt[K];
      int64_t slot[K];
#pragma unroll
      for (int q = 0; q < K; ++q) {
        cnt[q] = 0;
        slot[q] = EMIT ? t.base[q] + (offs[q * pb.row + (int64_t)p * n_cells + c] - off0[q]) : 0;
      }
      if (live) {
        for (int32_t jb = d.b0; jb < d.b1; jb += 32) {
          const int32_t j = jb + lane;
          bool ord = false;
          double d2 = 0.0;
          int32_t jo = 0;
          SlotMeta mj{};
          if (j < d.b1) {
            const double ex = dadd(dsub(b.px[j], xi), d.off[0]);
            const double ey = dadd(dsub(b.py[j], yi), d.off[1]);
            const double ez = dadd(dsub(b.pz[j], zi), d.off[2]);
            mj = b.meta[j];
            jo = mj.orig;
            d2 = norm2(ex, ey, ez);
            ord = mi.orig < jo || (mi.orig == jo && shifted);
          }
#pragma unroll
          for (int q = 0; q < K; ++q) {
            const bool hit = ord && d2 < pb.q[q].rc_sq &&
                             !(q > 0 && pb.disjoint && d2 < pb.q[q > 0 ? q - 1 : 0].rc_sq);
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (!EMIT) {
              cnt[q] += __popc(m);
            } else {
              if (hit) {
                const int64_t e = slot[q] + __popc(m & lanemask_lt());
                t.src[q][e] = (int64_t)mi.orig + t.index_offset;
                (q == 0 ? dst0 : t.dst[q])[e] = (int64_t)jo + t.index_offset;
                int32_t* sp = t.sh[q] + 3 * e;
                sp[0] = (mj.sx - mi.sx) + d.sh[0];
                sp[1] = (mj.sy - mi.sy) + d.sh[1];
                sp[2] = (mj.sz - mi.sz) + d.sh[2];
              }
              slot[q] += __popc(m);
            }
          }
        }
      }
      if (!EMIT && lane == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) counts[q * pb.row + (int64_t)p * n_cells + c] = cnt[q];
      }
    }
  }
}

// Euclidean division with the common in-range cases first.
__device__ __forceinline__ void div_mod_fast(int32_t v, int32_t m, int32_t& rem, int32_t& quot) {
  if (v >= 0 && v < m) {
    rem = v;
    quot = 0;
  } else if (v < 0 && v >= -m) {
    rem = v + m;
    quot = -1;
  } else if (v >= m && v < 2 * m) {
    rem = v - m;
    quot = 1;
  } else {
    div_mod(v, m, rem, quot);
  }
}

// Register budgets measured best on B200: the single-cutoff passes at 3 CTAs
// per SM (80 registers, no spills); with several cutoffs, which keep more
// masks live, the count pass at 2 and the emit pass unbounded.
template <bool EMIT, int K>
__global__ void __launch_bounds__(kPairWarps * 32, EMIT ? (K == 1 ? 3 : 1) : (K == 1 ? 3 : 2))
    k_pair_tasks(GridParams g, GridBuffers b, int64_t n, int32_t n_cells, PairBands pb,
                 uint32_t* __restrict__ counts, const int64_t* __restrict__ offs, EmitTargets t,
                 int32_t stage_cap) {
  // Staged candidates as pairs (2m, 2m + 1): {x, x', y, y'}, {z, z'}, {idx, idx'}.
  __shared__ float4 stage_xy[kPairWarps][16];
  __shared__ float2 stage_z[kPairWarps][16];
  __shared__ int2 stage_w[kPairWarps][16];
  __shared__ SlotMeta stage_m[kPairWarps][32];
  __shared__ char4 stencil[kPairMaxCells];  // (dx, dy, dz) of each stencil cell, x outer
  // Emit pass: per warp, each lane's first output slot minus its stage offset,
  // each lane's atom meta, and the staged hits (lane << 11 | candidate offset
  // in the cell) of the current task.
  __shared__ int64_t lane_base[EMIT ? kPairWarps : 1][32];
  __shared__ SlotMeta lane_meta[EMIT ? kPairWarps : 1][32];
  extern __shared__ uint16_t stage_hits[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  {
    const int32_t ny = 2 * g.ns[1] + 1, nz = 2 * g.ns[2] + 1;
    for (int c = threadIdx.x; c < n_cells; c += blockDim.x) {
      const int32_t ix = c / (ny * nz);
      const int32_t rem = c - ix * (ny * nz);
      const int32_t iy = rem / nz;
      stencil[c] = make_char4((signed char)(ix - g.ns[0]), (signed char)(iy - g.ns[1]),
                              (signed char)(rem - iy * nz - g.ns[2]), 0);
    }
    __syncthreads();
  }
  float* sxy = reinterpret_cast<float*>(stage_xy[warp]);
  float* sz = reinterpret_cast<float*>(stage_z[warp]);
  int32_t* sw = reinterpret_cast<int32_t*>(stage_w[warp]);
  SlotMeta* smt = stage_m[warp];
  pdl_wait();
  if (EMIT && t.report && blockIdx.x == 0 && threadIdx.x == 0) {
    volatile int64_t* r = t.report;
    r[1] = t.total_dev ? *t.total_dev : 0;
    r[2] = (t.scan_error ? *t.scan_error : 0) | (t.grid_scan_error ? *t.grid_scan_error : 0);
    r[3] = t.mask_top ? (int64_t)*t.mask_top : 0;
    __threadfence_system();
    r[0] = 1;
  }
  int64_t* dst0 = EMIT ? t.dst[0] : nullptr;
  if (EMIT && t.scan_error && *t.scan_error != 0) return;  // offsets not valid
  if (EMIT && t.total_dev) {
    const int64_t m_total = *t.total_dev;
    if (m_total > t.capacity) return;  // the caller grows the arena and emits again
    dst0 = t.src[0] + m_total;
  }
  const uint32_t n_tasks = (uint32_t)b.counters[0] * (uint32_t)n_cells;
  const uint32_t step = gridDim.x * kPairWarps;
  // Emit on dense grids: tasks from a shared counter, so that warps that
  // drew cheap tasks take more (static striding leaves a long tail there).
  uint32_t* const queue = EMIT ? b.emit_queue : nullptr;
  auto next_task = [&](uint32_t cur) -> uint32_t {
    if (!queue) return cur + step;
    uint32_t v = 0;
    if (lane == 0) v = atomicAdd(queue, 1u);
    return __shfl_sync(0xffffffffu, v, 0);
  };
  int64_t off0[K];
  float lo[K], hi[K];
#pragma unroll
  for (int q = 0; q < K; ++q) {
    off0[q] = EMIT ? offs[q * pb.row] : 0;
    lo[q] = pb.q[q].lo;
    hi[q] = pb.q[q].hi;
  }

  for (uint32_t task = queue ? next_task(0) : blockIdx.x * kPairWarps + warp; task < n_tasks;
       task = next_task(task)) {
    const uint32_t gi = task / (uint32_t)n_cells;
    const int32_t c = (int32_t)(task - gi * (uint32_t)n_cells);
    const GroupRec grp = b.groups[gi];
    const int32_t len = grp.end - grp.first < 32 ? grp.end - grp.first : 32;
    const int32_t p = grp.first + (lane < len ? lane : 0);
    const bool mine = lane < len && !b.irr[p];
    if (EMIT && b.masks) {
      // Hits recorded by the count pass: expand the stored masks.
      const int4 hdr = b.task_hdr[task];
      // Loads that need no header, issued before its branch so that their
      // latency overlaps the header's.
      SlotMeta mi{};
      int64_t o_lo = 0, o_hi = 0;
      if (lane < len) {
        mi = b.meta[p];
        if (K == 1) {
          const int64_t idx = (int64_t)p * n_cells + c;
          o_lo = offs[idx];
          o_hi = offs[idx + 1];
        }
      }
      if (hdr.x == -2) continue;
      if (hdr.x >= 0) {
        const int32_t h0 = hdr.y, h1 = hdr.z;
        const int32_t words = ((h1 - h0 + 31) >> 5) * 32;  // one cutoff's masks
        const uint32_t pw = (uint32_t)hdr.w;  // three signed 10-bit shifts
        const int32_t s0 = (int32_t)(pw << 22) >> 22;
        const int32_t s1 = (int32_t)(pw << 12) >> 22;
        const int32_t s2 = (int32_t)(pw << 2) >> 22;
#pragma unroll 1
        for (int q = 0; q < K; ++q) {
          int64_t* __restrict__ srcq = t.src[q];
          int64_t* __restrict__ dstq = q == 0 ? dst0 : t.dst[q];
          int32_t* __restrict__ shq = t.sh[q];
          const uint32_t* mq = b.masks + (int64_t)hdr.x + (int64_t)q * words;
          int64_t slot = 0;
          int32_t cnt = 0;
          if (mine && K == 1) {
            slot = t.base[0] + (o_lo - off0[0]);
            cnt = (int32_t)(o_hi - o_lo);
          } else if (mine) {
            const int64_t idx = q * pb.row + (int64_t)p * n_cells + c;
            const int64_t o0 = offs[idx];
            slot = t.base[q] + (o0 - off0[q]);
            cnt = (int32_t)(offs[idx + 1] - o0);
          }
          // Stage the task's hits (lane's hits at [pre, pre + cnt)), then
          // write them with the whole warp in stage order: each lane's
          // (atom, cell) run is contiguous in the output, so consecutive
          // threads store to consecutive slots instead of 32 lanes storing to
          // 32 runs.
          int32_t pre = cnt;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= o) pre += y;
          }
          const int32_t total = __shfl_sync(0xffffffffu, pre, 31);
          pre -= cnt;
          if (total <= stage_cap && h1 - h0 <= kStageCell) {
            uint16_t* st = stage_hits + warp * stage_cap;
            lane_base[warp][lane] = slot - pre;
            lane_meta[warp][lane] = mi;
            int32_t r = pre;
            const int32_t r_end = pre + cnt;  // the lane's own stage range
            for (int32_t jb = h0; jb < h1; jb += 32) {
              uint32_t hits = mine ? mq[(jb - h0) + lane] : 0u;
              while (hits) {
                const int jj = __ffs(hits) - 1;
                hits &= hits - 1;
                if (r < r_end) st[r] = (uint16_t)((lane << 11) | (jb - h0 + jj));
                ++r;
              }
            }
            __syncwarp();
            // Four waves at a time: their candidate gathers are in flight
            // together before any of their stores.
            for (int32_t k0 = lane; k0 < total; k0 += 4 * 32) {
              uint32_t v[4];
              SlotMeta mj[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int32_t k = k0 + 32 * u;
                v[u] = k < total ? st[k] : 0u;
                if (k < total) mj[u] = b.meta[h0 + (int32_t)(v[u] & 2047u)];
              }
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int32_t k = k0 + 32 * u;
                if (k >= total) break;
                const int l = (int)(v[u] >> 11);
                const SlotMeta ml = lane_meta[warp][l];
                const int64_t e = lane_base[warp][l] + k;
                srcq[e] = (int64_t)ml.orig + t.index_offset;
                dstq[e] = (int64_t)mj[u].orig + t.index_offset;
                int32_t* sp = shq + 3 * e;
                sp[0] = (mj[u].sx - ml.sx) + s0;
                sp[1] = (mj[u].sy - ml.sy) + s1;
                sp[2] = (mj[u].sz - ml.sz) + s2;
              }
            }
            __syncwarp();
          } else {
            for (int32_t jb = h0; jb < h1; jb += 32) {
              uint32_t hits = mine ? mq[(jb - h0) + lane] : 0u;
              if (!__any_sync(0xffffffffu, hits != 0)) continue;
              if (jb + lane < h1) smt[lane] = b.meta[jb + lane];
              __syncwarp();
              while (hits) {
                const int jj = __ffs(hits) - 1;
                hits &= hits - 1;
                const SlotMeta mj = smt[jj];
                srcq[slot] = (int64_t)mi.orig + t.index_offset;
                dstq[slot] = (int64_t)mj.orig + t.index_offset;
                int32_t* sp = shq + 3 * slot;
                sp[0] = (mj.sx - mi.sx) + s0;
                sp[1] = (mj.sy - mi.sy) + s1;
                sp[2] = (mj.sz - mi.sz) + s2;
                ++slot;
              }
              __syncwarp();
            }
          }
        }
        continue;
      }
      // hdr.x == -1: the masks did not fit; recompute below.
    }

    // The stencil cell (shared by the group) and the group's bin centre.
    const char4 st = stencil[c];
    int32_t bin[3], sh[3];
    div_mod_fast(grp.bx + st.x, g.nb[0], bin[0], sh[0]);
    div_mod_fast(grp.by + st.y, g.nb[1], bin[1], sh[1]);
    div_mod_fast(grp.bz + st.z, g.nb[2], bin[2], sh[2]);
    double off[3], cs[3], cb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      off[k] = dadd(dadd(dmul(g.h[3 * k], (double)sh[0]), dmul(g.h[3 * k + 1], (double)sh[1])),
                    dmul(g.h[3 * k + 2], (double)sh[2]));
      double v = dadd(g.origin[k], dmul(g.basis[0][k], (double)bin[0]));
      v = dadd(v, dmul(g.basis[1][k], (double)bin[1]));
      v = dadd(v, dmul(g.basis[2][k], (double)bin[2]));
      cs[k] = dadd(v, off[k]);
      double w = dadd(g.origin[k], dmul(g.basis[0][k], (double)grp.bx));
      w = dadd(w, dmul(g.basis[1][k], (double)grp.by));
      cb[k] = dadd(w, dmul(g.basis[2][k], (double)grp.bz));
    }
    const int64_t lin = bin[0] + (int64_t)g.nb[0] * (bin[1] + (int64_t)g.nb[1] * bin[2]);
    const int32_t r = b.rank_of_bin[lin];
    const int32_t b0 = (int32_t)b.bin_start[r], b1 = (int32_t)b.bin_start[r + 1];

    const double xi = b.px[p], yi = b.py[p], zi = b.pz[p];
    const bool live =
        mine && !(norm2(dsub(cs[0], xi), dsub(cs[1], yi), dsub(cs[2], zi)) > g.prune_sq);
    uint32_t cnt[K];
    int64_t slot[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      cnt[q] = 0;
      slot[q] = 0;
      if (EMIT && mine) slot[q] = t.base[q] + (offs[q * pb.row + (int64_t)p * n_cells + c] - off0[q]);
    }
    const bool work = __any_sync(0xffffffffu, live) && b1 > b0;
    const int32_t words = ((b1 - b0 + 31) >> 5) * 32;  // one cutoff's masks
    // Count pass: reserve this task's hit masks (one word per lane per chunk
    // per cutoff).
    int32_t mbase = -2;
    if (!EMIT && b.masks) {
      if (work) {
        long long top = 0;
        if (lane == 0) top = (long long)atomicAdd(b.mask_top, (unsigned long long)(K * words));
        top = __shfl_sync(0xffffffffu, top, 0);
        const bool fits = top + K * words <= b.mask_cap && top + K * words < 0x7fffffffLL &&
                          sh[0] >= -511 && sh[0] <= 511 && sh[1] >= -511 && sh[1] <= 511 &&
                          sh[2] >= -511 && sh[2] <= 511;
        mbase = fits ? (int32_t)top : -1;
      }
      if (lane == 0)
        b.task_hdr[task] = make_int4(mbase, b0, b1,
                                     (sh[0] & 1023) | ((sh[1] & 1023) << 10) | ((sh[2] & 1023) << 20));
    }
    if (work) {
      const float4 a = b.p32[p];
      const int32_t io = __float_as_int(a.w);
      const float tx = __double2float_rn(dsub(cs[0], cb[0]));
      const float ty = __double2float_rn(dsub(cs[1], cb[1]));
      const float tz = __double2float_rn(dsub(cs[2], cb[2]));
      const float ux = tx - a.x;
      const float uy = ty - a.y;
      const float uz = tz - a.z;
      // Chunk pruning (count pass, dense grids): the group's box in its bin
      // frame; a candidate chunk whose box, moved by the cell translation,
      // stays farther than the band allows is skipped (its masks are zero).
      const bool prune = !EMIT && b.cbox != nullptr;
      float4 glo = make_float4(0.f, 0.f, 0.f, 0.f), ghi = glo;
      if (prune) {
        glo = b.cbox[2 * (int64_t)grp.first];
        ghi = b.cbox[2 * (int64_t)grp.first + 1];
      }
      const float skip_sq = hi[K - 1] + (hi[K - 1] - lo[K - 1]);
      const float2 ux2 = make_float2(ux, ux), uy2 = make_float2(uy, uy), uz2 = make_float2(uz, uz);
      const bool shifted = (sh[0] | sh[1] | sh[2]) != 0;
      // Half-list predicate io < jo || (io == jo && shifted) as one compare.
      const int32_t io_adj = shifted ? io - 1 : io;
      SlotMeta mi;
      if (EMIT) mi = b.meta[p];
      for (int32_t jb = b0; jb < b1; jb += 32) {
        const int32_t nj = b1 - jb < 32 ? b1 - jb : 32;
        if (prune) {
          const float4 clo = b.cbox[2 * (int64_t)jb], chi = b.cbox[2 * (int64_t)jb + 1];
          const float gx = fmaxf(fmaxf((clo.x + tx) - ghi.x, glo.x - (chi.x + tx)), 0.f);
          const float gy = fmaxf(fmaxf((clo.y + ty) - ghi.y, glo.y - (chi.y + ty)), 0.f);
          const float gz = fmaxf(fmaxf((clo.z + tz) - ghi.z, glo.z - (chi.z + tz)), 0.f);
          if (gx * gx + gy * gy + gz * gz > skip_sq) {
            if (mbase >= 0) {
#pragma unroll
              for (int q = 0; q < K; ++q)
                b.masks[(int64_t)mbase + (int64_t)q * words + (jb - b0) + lane] = 0u;
            }
            continue;
          }
        }
        // Stage 32 candidates; slots past the bin end hold a far sentinel.
        float4 qv = make_float4(1e30f, 1e30f, 1e30f, __int_as_float(-1));
        if (lane < nj) {
          qv = b.p32[jb + lane];
          if (EMIT) smt[lane] = b.meta[jb + lane];
        }
        {
          const int pr = lane >> 1, h = lane & 1;
          sxy[4 * pr + h] = qv.x;
          sxy[4 * pr + 2 + h] = qv.y;
          sz[2 * pr + h] = qv.z;
          sw[2 * pr + h] = __float_as_int(qv.w);
        }
        __syncwarp();
        // FP32 test of all 32 staged candidates into bit masks, two at a time
        // with the packed FP32 units (element-wise the same roundings as the
        // scalar dx = x_j + u, d2 = fma(dz, dz, fma(dy, dy, dx * dx))), one
        // squared distance per pair against every cutoff's band.
        // (candidates 31 down to 0: each predicate's sign bit appended, see
        // push_sign)
        uint32_t inside[K], maybe[K], order = 0;
#pragma unroll
        for (int q = 0; q < K; ++q) inside[q] = maybe[q] = 0;
#pragma unroll
        for (int pr = 15; pr >= 0; --pr) {
          const float4 xy = stage_xy[warp][pr];
          const float2 z = stage_z[warp][pr];
          const int2 w = stage_w[warp][pr];
          const float2 dx = __fadd2_rn(make_float2(xy.x, xy.y), ux2);
          const float2 dy = __fadd2_rn(make_float2(xy.z, xy.w), uy2);
          const float2 dz = __fadd2_rn(z, uz2);
          const float2 d2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
#pragma unroll
          for (int q = 0; q < K; ++q) {
            const float2 sl = __fadd2_rn(d2, make_float2(-lo[q], -lo[q]));
            const float2 sh = __fadd2_rn(d2, make_float2(-hi[q], -hi[q]));
            inside[q] = push_sign(push_sign(inside[q], __float_as_uint(sl.y)), __float_as_uint(sl.x));
            maybe[q] = push_sign(push_sign(maybe[q], __float_as_uint(sh.y)), __float_as_uint(sh.x));
          }
          order = push_sign(push_sign(order, (uint32_t)(io_adj - w.y)), (uint32_t)(io_adj - w.x));
        }
        if (!live) order = 0;
        // Guard bands: the reference's exact FP64 test decides (for every
        // cutoff at once; it agrees with the certain FP32 outcomes).
        uint32_t amb = 0;
#pragma unroll
        for (int q = 0; q < K; ++q) amb |= maybe[q] & ~inside[q];
        amb &= order;
        while (amb) {
          const int jj = __ffs(amb) - 1;
          amb &= amb - 1;
          const int32_t j = jb + jj;
          const double ex = dadd(dsub(b.px[j], xi), off[0]);
          const double ey = dadd(dsub(b.py[j], yi), off[1]);
          const double ez = dadd(dsub(b.pz[j], zi), off[2]);
          const double d2e = norm2(ex, ey, ez);
#pragma unroll
          for (int q = 0; q < K; ++q)
            if (d2e < pb.q[q].rc_sq) inside[q] |= 1u << jj;
        }
        uint32_t hits[K];
#pragma unroll
        for (int q = 0; q < K; ++q) hits[q] = inside[q] & order;
        // Disjoint shells: cutoff q keeps only the pairs outside cutoff q - 1.
        if (K > 1 && pb.disjoint) {
#pragma unroll
          for (int q = K - 1; q > 0; --q) hits[q] &= ~inside[q - 1];
        }
        if (!EMIT) {
#pragma unroll
          for (int q = 0; q < K; ++q) {
            cnt[q] += __popc(hits[q]);
            if (mbase >= 0) b.masks[(int64_t)mbase + (int64_t)q * words + (jb - b0) + lane] = hits[q];
          }
        } else {
#pragma unroll
          for (int q = 0; q < K; ++q) {
            int64_t* __restrict__ dstq = q == 0 ? dst0 : t.dst[q];
            while (hits[q]) {
              const int jj = __ffs(hits[q]) - 1;
              hits[q] &= hits[q] - 1;
              const SlotMeta mj = smt[jj];
              t.src[q][slot[q]] = (int64_t)io + t.index_offset;
              dstq[slot[q]] = (int64_t)mj.orig + t.index_offset;
              int32_t* sp = t.sh[q] + 3 * slot[q];
              sp[0] = (mj.sx - mi.sx) + sh[0];
              sp[1] = (mj.sy - mi.sy) + sh[1];
              sp[2] = (mj.sz - mi.sz) + sh[2];
              ++slot[q];
            }
          }
        }
        __syncwarp();
      }
    }
    if (!EMIT && mine) {
#pragma unroll
      for (int q = 0; q < K; ++q) counts[q * pb.row + (int64_t)p * n_cells + c] = cnt[q];
    }
  }
  // Atoms whose home stencil is not their stored bin (normally none).
  pair_irregular<EMIT, K>(g, b, n_cells, pb, counts, offs, t, dst0,
                          (int64_t)blockIdx.x * kPairWarps + warp, step);
  if (!EMIT && blockIdx.x == 0 && threadIdx.x < K) counts[threadIdx.x * pb.row + n * (int64_t)n_cells] = 0;
}

int pair_grid(const void* func, size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, kPairWarps * 32, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

inline int32_t stencil_cells(const GridParams& g) {
  return (2 * g.ns[0] + 1) * (2 * g.ns[1] + 1) * (2 * g.ns[2] + 1);
}

}  // namespace

bool make_guard_band(const GridParams& g, double rc, GuardBand& band) {
  // FP32 unit roundoff.  A task's candidates lie in a cell that is not pruned
  // for the lane's atom, so |c_cell + off - x_i| <= rc + R and
  // |T| = |c_cell + off - c_bin| <= rc + 2R; bin-relative coordinates satisfy
  // |x| <= R.  The FP32 roundings of x_j, x_i, T, T - x_i and x_j + (T - x_i)
  // bound each component's error by u (7R + 3rc) for pairs with |d| <= rc
  // (eps doubles it).  The FMA reduction adds at most 3u d2.  delta covers
  // 2 sqrt(3) eps |d| + 3 eps^2 + 3u d2 with a factor 2, plus the FP64
  // reference's own rounding.
  const double u = std::ldexp(1.0, -24);
  const double R = g.radius;
  if (!std::isfinite(R) || !std::isfinite(rc) || R <= 0.0) return false;
  const double eps = 2.0 * u * (7.0 * R + 3.0 * rc) + 1e-12;
  const double r = rc + eps;
  const double delta =
      2.0 * (2.0 * std::sqrt(3.0) * eps * r + 3.0 * eps * eps + 4.0 * u * r * r) + 1e-12 * r * r;
  const double rc2 = rc * rc;
  if (!(delta < 1e-3 * rc2)) return false;
  if (stencil_cells(g) > kPairMaxCells) return false;
  band.rc_sq = rc2;
  band.lo = std::nextafter((float)(rc2 - delta), -INFINITY);
  band.hi = std::nextafter((float)(rc2 + delta), INFINITY);
  return true;
}

namespace {

PairBands single_band(const GuardBand& band) {
  PairBands pb;
  std::memset(&pb, 0, sizeof(pb));
  pb.q[0] = band;
  pb.k = 1;
  return pb;
}

template <int K>
void pair_count_k(const GridParams& g, const GridBuffers& b, int64_t n, const PairBands& pb,
                  uint32_t* counts, cudaStream_t s) {
  EmitTargets t{};
  const int32_t cells = stencil_cells(g);
  launch_pdl(k_pair_tasks<false, K>, dim3(pair_grid((const void*)k_pair_tasks<false, K>, 0)),
             dim3(kPairWarps * 32), 0, s, g, b, n, cells, pb, counts, (const int64_t*)nullptr, t,
             (int32_t)0);
  note_launches(1);
}

template <int K>
void pair_emit_k(const GridParams& g, const GridBuffers& b, int64_t n, const PairBands& pb,
                 const int64_t* offs, const EmitTargets& t, cudaStream_t s) {
  const int32_t cells = stencil_cells(g);
  // A task's hits are at most 32 x (candidates of one cell); decide by the
  // mean bin occupancy.
  const double per_bin = g.total_bins > 0 ? (double)n / (double)g.total_bins : 0.0;
  const int32_t cap = 32.0 * per_bin > (double)kStageSmall ? kStageLarge : kStageSmall;
  GridBuffers bq = b;
  if (cap != kStageLarge) bq.emit_queue = nullptr;  // cheap, even tasks: static striding
  ensure_smem_attr((const void*)k_pair_tasks<true, K>, (int)stage_smem(kStageLarge));
  launch_pdl(k_pair_tasks<true, K>,
             dim3(pair_grid((const void*)k_pair_tasks<true, K>, stage_smem(cap))),
             dim3(kPairWarps * 32), stage_smem(cap), s, g, bq, n, cells, pb, (uint32_t*)nullptr,
             offs, t, cap);
  note_launches(1);
}

}  // namespace

void launch_pair_count(const GridParams& g, const GridBuffers& b, int64_t n,
                       const GuardBand& band, uint32_t* counts, cudaStream_t s) {
  pair_count_k<1>(g, b, n, single_band(band), counts, s);
}

void launch_pair_emit(const GridParams& g, const GridBuffers& b, int64_t n,
                      const GuardBand& band, const int64_t* offs, const EmitTargets& t,
                      cudaStream_t s) {
  pair_emit_k<1>(g, b, n, single_band(band), offs, t, s);
}

void launch_pair_count_multi(const GridParams& g, const GridBuffers& b, int64_t n,
                             const PairBands& pb, uint32_t* counts, cudaStream_t s) {
  switch (pb.k) {
    case 1: pair_count_k<1>(g, b, n, pb, counts, s); break;
    case 2: pair_count_k<2>(g, b, n, pb, counts, s); break;
    case 3: pair_count_k<3>(g, b, n, pb, counts, s); break;
    default: pair_count_k<4>(g, b, n, pb, counts, s); break;
  }
  static_assert(kFp32MaxCutoffs == 4, "one instantiation per cutoff count");
}

void launch_pair_emit_multi(const GridParams& g, const GridBuffers& b, int64_t n,
                            const PairBands& pb, const int64_t* offs, const EmitTargets& t,
                            cudaStream_t s) {
  switch (pb.k) {
    case 1: pair_emit_k<1>(g, b, n, pb, offs, t, s); break;
    case 2: pair_emit_k<2>(g, b, n, pb, offs, t, s); break;
    case 3: pair_emit_k<3>(g, b, n, pb, offs, t, s); break;
    default: pair_emit_k<4>(g, b, n, pb, offs, t, s); break;
  }
}

}  // namespace nlb
