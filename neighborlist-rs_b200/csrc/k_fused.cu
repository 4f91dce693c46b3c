// k_fused.cu -- single-cutoff cell-list search in ONE launch: count, offsets
// and emit of each 32-atom group by one CTA.
//
// The pair-task pipeline (k_search2.cu) runs three launches after the build:
// a count pass over (group, stencil cell) tasks, an exclusive scan of the
// per-(atom, cell) counts, and an emit pass.  On sparse grids (a few dozen
// atoms per bin, the common case) each launch is short and the chain is
// dominated by launch ramps, tails and dependent-load latency.  Here one CTA
// takes a group ticket (tickets are handed out in canonical group order:
// bins in rank order, 32-atom runs in slot order) and
//
//   1. describes the group's stencil cells (bin, image shift, FP64 offset,
//      FP32 translation into the group's bin frame) in shared memory;
//   2. counts: warp w tests cells w, w + 8, ... with the FP32 pair test and
//      the FP64 guard-band recheck of k_search2.cu (same predicate, same
//      roundings), keeping every lane's 32-bit hit mask per candidate chunk
//      in shared memory and its count per cell;
//   3. turns the counts into each atom's cell offsets and the group's total
//      E, and finds the group's first output slot G with a decoupled
//      look-back over the groups before it (bounded polls: a wait that runs
//      out records an error word and the group writes nothing);
//   4. writes the group's block [G, G + E) of the canonical list -- atoms in
//      slot order, cells in stencil order, candidates in bin order -- by
//      staging (lane, cell, candidate) entries in canonical order in shared
//      memory and storing them with consecutive threads on consecutive slots.
//
// Sources and shifts go to their arrays at slot e, destinations to a
// separate array (the total M is known only when the last group is done);
// for [src | dst] the CTAs then move the destinations behind the sources
// once every group is written.
// The last group writes M.  A group whose block does not fit the capacity
// writes nothing (the host grows the arrays and runs the launch again).
// Atoms whose home stencil differs from their stored bin ("irregular",
// within rounding of a bin face) are counted and written by one warp each in
// FP64 over their own stencil, exactly like the pair-task kernels.
#include <cmath>
#include <cstring>

#include "k_traverse.cuh"

namespace nlb {

namespace {

constexpr int kFThreads = 256;
constexpr int kFWarps = kFThreads / 32;
constexpr int kFStage = 4096;      // output entries staged per window
constexpr int kFJBits = 17;        // candidate offset bits of a stage entry

constexpr uint64_t kFStatusShift = 62;
constexpr uint64_t kFAggregate = 1ull << kFStatusShift;
constexpr uint64_t kFInclusive = 2ull << kFStatusShift;
constexpr uint64_t kFValueMask = (1ull << kFStatusShift) - 1;

__device__ __forceinline__ uint64_t f_load(const uint64_t* p) {
  return *reinterpret_cast<const volatile uint64_t*>(p);
}
__device__ __forceinline__ void f_store(uint64_t* p, uint64_t v) {
  __threadfence();
  *reinterpret_cast<volatile uint64_t*>(p) = v;
}

// {M, error word} to the host-mapped report, then its ready word.
__device__ __forceinline__ void f_report(const FusedOut& o, int64_t m, int64_t err) {
  if (!o.report) return;
  __threadfence();
  volatile int64_t* r = o.report;
  r[1] = m;
  r[2] = err;
  __threadfence_system();
  r[0] = 1;
}

struct FCell {
  double off[3];   // FP64 image offset (reference order)
  double cs[3];    // bin centre + offset: the prune test's target
  float t[3];      // FP32 translation into the group's bin frame
  int32_t b0, b1;  // candidate slots
  int32_t sh[3];   // image shift
  int32_t mbase;   // first mask word in shared memory (-1: masks not kept)
};
static_assert(sizeof(FCell) == 88, "fused_cells_bytes assumes 88-byte cell records");

// Euclidean division with the common in-range cases first.
__device__ __forceinline__ void f_div_mod(int32_t v, int32_t m, int32_t& rem, int32_t& quot) {
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

// Cell c of the stencil centred on bin (hx, hy, hz).
__device__ __forceinline__ void f_describe(const GridParams& g, const GridBuffers& b, int32_t hx,
                                           int32_t hy, int32_t hz, int32_t c, FCell& d,
                                           const double* cb) {
  const int32_t ny = 2 * g.ns[1] + 1, nz = 2 * g.ns[2] + 1;
  const int32_t ix = c / (ny * nz);
  const int32_t rem = c - ix * (ny * nz);
  const int32_t iy = rem / nz, iz = rem - (rem / nz) * nz;
  int32_t bin[3];
  f_div_mod(hx + ix - g.ns[0], g.nb[0], bin[0], d.sh[0]);
  f_div_mod(hy + iy - g.ns[1], g.nb[1], bin[1], d.sh[1]);
  f_div_mod(hz + iz - g.ns[2], g.nb[2], bin[2], d.sh[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d.off[k] = dadd(dadd(dmul(g.h[3 * k], (double)d.sh[0]), dmul(g.h[3 * k + 1], (double)d.sh[1])),
                    dmul(g.h[3 * k + 2], (double)d.sh[2]));
    double v = dadd(g.origin[k], dmul(g.basis[0][k], (double)bin[0]));
    v = dadd(v, dmul(g.basis[1][k], (double)bin[1]));
    v = dadd(v, dmul(g.basis[2][k], (double)bin[2]));
    d.cs[k] = dadd(v, d.off[k]);
    d.t[k] = cb ? __double2float_rn(dsub(d.cs[k], cb[k])) : 0.f;
  }
  const int64_t lin = bin[0] + (int64_t)g.nb[0] * (bin[1] + (int64_t)g.nb[1] * bin[2]);
  const int32_t r = b.rank_of_bin[lin];
  d.b0 = (int32_t)b.bin_start[r];
  d.b1 = (int32_t)b.bin_start[r + 1];
}

// One 32-candidate chunk of a cell for the warp's 32 atoms.  Candidates
// farther from the group's box (gbox: FP32, in the group's bin frame) than
// the band allows cannot be within the cutoff of any of its atoms and are
// dropped first; the kept ones are staged contiguously and go through the
// FP32 test of k_search2.cu on packed pairs, the guard band rechecked in
// FP64, the half-list predicate.  Returns the lane's hit mask over the
// chunk's candidate offsets.
__device__ __forceinline__ uint32_t f_chunk(const GridBuffers& b, const FCell& cell, int32_t jb,
                                            float ux, float uy, float uz, int32_t io_adj,
                                            bool live, double xi, double yi, double zi, float lo,
                                            float hi, double rc_sq, const float4* gbox,
                                            float4* sxy4, float2* sz2, int2* sw2,
                                            uint8_t* smap) {
  const int lane = threadIdx.x & 31;
  const int32_t nj = cell.b1 - jb < 32 ? cell.b1 - jb : 32;
  float4 qv = make_float4(1e30f, 1e30f, 1e30f, __int_as_float(-1));
  bool keep = false;
  if (lane < nj) {
    qv = b.p32[jb + lane];
    const float4 glo = gbox[0], ghi = gbox[1];
    const float cx = qv.x + cell.t[0], cy = qv.y + cell.t[1], cz = qv.z + cell.t[2];
    const float gx = fmaxf(fmaxf(cx - ghi.x, glo.x - cx), 0.f);
    const float gy = fmaxf(fmaxf(cy - ghi.y, glo.y - cy), 0.f);
    const float gz = fmaxf(fmaxf(cz - ghi.z, glo.z - cz), 0.f);
    // (margin: one band width, as the chunk pruning of k_search2.cu)
    keep = gx * gx + gy * gy + gz * gz <= hi + (hi - lo);
  }
  const uint32_t km = __ballot_sync(0xffffffffu, keep);
  if (km == 0) return 0;
  const int nk = __popc(km);
  float* sxy = reinterpret_cast<float*>(sxy4);
  float* sz = reinterpret_cast<float*>(sz2);
  int32_t* sw = reinterpret_cast<int32_t*>(sw2);
  __syncwarp();  // (the previous chunk's readers are done)
  if (keep) {
    const int k = __popc(km & lanemask_lt());
    const int pr = k >> 1, h = k & 1;
    sxy[4 * pr + h] = qv.x;
    sxy[4 * pr + 2 + h] = qv.y;
    sz[2 * pr + h] = qv.z;
    sw[2 * pr + h] = __float_as_int(qv.w);
    smap[k] = (uint8_t)lane;
  }
  if (lane == 0 && (nk & 1)) {
    // the odd slot of the last pair: a far sentinel
    const int pr = nk >> 1;
    sxy[4 * pr + 1] = 1e30f;
    sxy[4 * pr + 3] = 1e30f;
    sz[2 * pr + 1] = 1e30f;
    sw[2 * pr + 1] = -1;
  }
  __syncwarp();
  const float2 ux2 = make_float2(ux, ux), uy2 = make_float2(uy, uy), uz2 = make_float2(uz, uz);
  const float2 nlo2 = make_float2(-lo, -lo), nhi2 = make_float2(-hi, -hi);
  uint32_t inside = 0, maybe = 0, order = 0;
  // (kept candidates from the last down to 0: each predicate's sign bit
  // appended, see push_sign, leaves kept candidate k at bit k)
  for (int pr = ((nk + 1) >> 1) - 1; pr >= 0; --pr) {
    const float4 xy = sxy4[pr];
    const float2 z = sz2[pr];
    const int2 w = sw2[pr];
    const float2 dx = __fadd2_rn(make_float2(xy.x, xy.y), ux2);
    const float2 dy = __fadd2_rn(make_float2(xy.z, xy.w), uy2);
    const float2 dz = __fadd2_rn(z, uz2);
    const float2 d2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 sl = __fadd2_rn(d2, nlo2), sh = __fadd2_rn(d2, nhi2);
    inside = push_sign(push_sign(inside, __float_as_uint(sl.y)), __float_as_uint(sl.x));
    maybe = push_sign(push_sign(maybe, __float_as_uint(sh.y)), __float_as_uint(sh.x));
    order = push_sign(push_sign(order, (uint32_t)(io_adj - w.y)), (uint32_t)(io_adj - w.x));
  }
  if (!live) order = 0;
  uint32_t amb = maybe & ~inside & order;
  while (amb) {
    const int k = __ffs(amb) - 1;
    amb &= amb - 1;
    const int32_t j = jb + smap[k];
    const double ex = dadd(dsub(b.px[j], xi), cell.off[0]);
    const double ey = dadd(dsub(b.py[j], yi), cell.off[1]);
    const double ez = dadd(dsub(b.pz[j], zi), cell.off[2]);
    if (norm2(ex, ey, ez) < rc_sq) inside |= 1u << k;
  }
  uint32_t hk = inside & order;
  // Kept candidate k back to its offset in the chunk.
  if (km == (nj == 32 ? 0xffffffffu : (1u << nj) - 1u)) return hk;
  uint32_t hits = 0;
  while (hk) {
    const int k = __ffs(hk) - 1;
    hk &= hk - 1;
    hits |= 1u << smap[k];
  }
  return hits;
}

// Irregular atom p (its home stencil is not its stored bin): one warp walks
// its own stencil in FP64 exactly like pair_irregular in k_search2.cu.
// EMIT = false: cnt[c * 32] (stride 32) receives the count of cell c.
// EMIT = true: its edges go to slots [e0, ...) in canonical order.
template <bool EMIT>
__device__ void f_irregular(const GridParams& g, const GridBuffers& b, int32_t n_cells,
                            double rc_sq, int32_t p, uint32_t* cnt, int64_t e0,
                            const FusedOut& o) {
  const int lane = threadIdx.x & 31;
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
  int64_t slot = e0;
  for (int32_t c = 0; c < n_cells; ++c) {
    FCell d;
    f_describe(g, b, home[0], home[1], home[2], c, d, nullptr);
    const bool live =
        !(norm2(dsub(d.cs[0], xi), dsub(d.cs[1], yi), dsub(d.cs[2], zi)) > g.prune_sq);
    const bool shifted = (d.sh[0] | d.sh[1] | d.sh[2]) != 0;
    uint32_t count = 0;
    if (live) {
      for (int32_t jb = d.b0; jb < d.b1; jb += 32) {
        const int32_t j = jb + lane;
        bool hit = false;
        SlotMeta mj{};
        if (j < d.b1) {
          const double ex = dadd(dsub(b.px[j], xi), d.off[0]);
          const double ey = dadd(dsub(b.py[j], yi), d.off[1]);
          const double ez = dadd(dsub(b.pz[j], zi), d.off[2]);
          mj = b.meta[j];
          hit = norm2(ex, ey, ez) < rc_sq && (mi.orig < mj.orig || (mi.orig == mj.orig && shifted));
        }
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (EMIT && hit) {
          const int64_t e = slot + __popc(m & lanemask_lt());
          o.src[e] = (int64_t)mi.orig;
          o.dst[e] = (int64_t)mj.orig;
          int32_t* sp = o.sh + 3 * e;
          sp[0] = (mj.sx - mi.sx) + d.sh[0];
          sp[1] = (mj.sy - mi.sy) + d.sh[1];
          sp[2] = (mj.sz - mi.sz) + d.sh[2];
        }
        slot += __popc(m);
        count += __popc(m);
      }
    }
    if (!EMIT && lane == 0) cnt[c * 32] = count;
  }
}

// Four CTAs per SM (64 registers): every group of a ~10k-atom system is then
// in flight at once (with three per SM the last ~7 % of the groups waited
// for a second round).
__global__ void __launch_bounds__(kFThreads, 4)
    k_pair_fused(GridParams g, GridBuffers b, int32_t n_cells, GuardBand band, FusedOut o) {
  extern __shared__ __align__(16) unsigned char fsm[];
  FCell* cells = reinterpret_cast<FCell*>(fsm);
  uint32_t* pre = reinterpret_cast<uint32_t*>(fsm + fused_cells_bytes(n_cells));
  uint32_t* masks = pre + (n_cells + 1) * 32;
  uint32_t* stage = masks + o.mask_words;
  __shared__ float4 st_xy[kFWarps][16];
  __shared__ float2 st_z[kFWarps][16];
  __shared__ int2 st_w[kFWarps][16];
  __shared__ uint8_t st_map[kFWarps][32];
  __shared__ float4 s_gbox[2];  // the group's FP32 box in its bin frame
  __shared__ SlotMeta lmeta[32];
  __shared__ int64_t abase[33];
  __shared__ int32_t s_ticket, s_irr, s_big, s_skip, s_cell;
  __shared__ int64_t s_G;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float lo = band.lo, hi = band.hi;
  const double rc_sq = band.rc_sq;
  uint64_t* const gstate = o.state + 2;
  pdl_wait();
  const int32_t n_groups = b.counters[0];

  for (;;) {
    if (tid == 0) s_ticket = (int32_t)atomicAdd(reinterpret_cast<unsigned long long*>(o.state), 1ull);
    __syncthreads();
    const int32_t t = s_ticket;
    if (t >= n_groups) break;
    const GroupRec grp = b.groups[t];
    const int32_t len = grp.end - grp.first < 32 ? grp.end - grp.first : 32;
    const int32_t p = grp.first + (lane < len ? lane : 0);

    // 1. the group's stencil cells
    if (tid < 32) {
      s_irr = __ballot_sync(0xffffffffu, lane < len && b.irr[p] != 0) != 0;
      if (lane == 0) s_big = 0;
    }
    double cb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double w = dadd(g.origin[k], dmul(g.basis[0][k], (double)grp.bx));
      w = dadd(w, dmul(g.basis[1][k], (double)grp.by));
      cb[k] = dadd(w, dmul(g.basis[2][k], (double)grp.bz));
    }
    // (cell c on lane c / 8 of warp c % 8: the FP64 work spread over the warps)
    for (int c = (tid & 31) * kFWarps + (tid >> 5); c < n_cells; c += kFThreads) {
      FCell d;
      f_describe(g, b, grp.bx, grp.by, grp.bz, c, d, cb);
      d.mbase = -1;
      cells[c] = d;
    }
    if (warp == 1 && lane < len) lmeta[lane] = b.meta[p];
    if (warp == 2) {
      // The group's box (its atoms' packed FP32 positions; lanes past len
      // repeat the first atom).
      const float4 q = b.p32[p];
      float4 lo4 = q, hi4 = q;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo4.x = fminf(lo4.x, __shfl_xor_sync(0xffffffffu, lo4.x, o));
        lo4.y = fminf(lo4.y, __shfl_xor_sync(0xffffffffu, lo4.y, o));
        lo4.z = fminf(lo4.z, __shfl_xor_sync(0xffffffffu, lo4.z, o));
        hi4.x = fmaxf(hi4.x, __shfl_xor_sync(0xffffffffu, hi4.x, o));
        hi4.y = fmaxf(hi4.y, __shfl_xor_sync(0xffffffffu, hi4.y, o));
        hi4.z = fmaxf(hi4.z, __shfl_xor_sync(0xffffffffu, hi4.z, o));
      }
      if (lane == 0) {
        s_gbox[0] = lo4;
        s_gbox[1] = hi4;
      }
    }
    __syncthreads();
    if (tid == 0) {
      // Masks stay in shared memory while they fit, cell by cell.
      int32_t acc = 0, big = 0;
      for (int c = 0; c < n_cells; ++c) {
        const int32_t nc = cells[c].b1 - cells[c].b0;
        const int32_t words = ((nc + 31) >> 5) * 32;
        if (acc + words <= o.mask_words) {
          cells[c].mbase = acc;
          acc += words;
        }
        big |= nc >= (1 << kFJBits);
      }
      s_big = big;
      s_cell = 0;
    }
    __syncthreads();

    // 2. count (warp w: cells w, w + 8, ...)
    const bool mine = lane < len && !b.irr[p];
    const float4 a = b.p32[p];
    const int32_t io = __float_as_int(a.w);
    const double xi = b.px[p], yi = b.py[p], zi = b.pz[p];
    // (cells handed out one at a time: warps that drew cheap cells take more)
    for (;;) {
      int c = 0;
      if (lane == 0) c = atomicAdd(&s_cell, 1);
      c = __shfl_sync(0xffffffffu, c, 0);
      if (c >= n_cells) break;
      const FCell& cell = cells[c];
      const bool live = mine && !(norm2(dsub(cell.cs[0], xi), dsub(cell.cs[1], yi),
                                        dsub(cell.cs[2], zi)) > g.prune_sq);
      uint32_t cnt = 0;
      if (__any_sync(0xffffffffu, live) && cell.b1 > cell.b0) {
        const bool shifted = (cell.sh[0] | cell.sh[1] | cell.sh[2]) != 0;
        const int32_t io_adj = shifted ? io - 1 : io;
        const float ux = cell.t[0] - a.x, uy = cell.t[1] - a.y, uz = cell.t[2] - a.z;
        for (int32_t jb = cell.b0; jb < cell.b1; jb += 32) {
          const uint32_t hits = f_chunk(b, cell, jb, ux, uy, uz, io_adj, live, xi, yi, zi, lo, hi,
                                        rc_sq, s_gbox, st_xy[warp], st_z[warp], st_w[warp],
                                        st_map[warp]);
          cnt += __popc(hits);
          if (cell.mbase >= 0) masks[cell.mbase + (jb - cell.b0) + lane] = hits;
        }
      }
      pre[c * 32 + lane] = cnt;
    }
    __syncthreads();
    if (s_irr && warp == 0) {
      for (int l = 0; l < len; ++l)
        if (b.irr[grp.first + l])
          f_irregular<false>(g, b, n_cells, rc_sq, grp.first + l, pre + l, 0, o);
    }
    __syncthreads();

    // 3. offsets: cells within each atom and atoms within the group (warp 0),
    //    whose total E is published at once for the groups after this one
    const bool publish = t != o.withhold;  // false only under the test hook
    if (warp == 0) {
      uint32_t run = 0;
      for (int c = 0; c < n_cells; ++c) {
        const uint32_t v = pre[c * 32 + lane];
        pre[c * 32 + lane] = run;
        run += v;
      }
      pre[n_cells * 32 + lane] = run;
      int64_t x = run;
#pragma unroll
      for (int s = 1; s < 32; s <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, s);
        if (lane >= s) x += y;
      }
      abase[lane] = x - (int64_t)run;
      const int64_t E0 = __shfl_sync(0xffffffffu, x, 31);
      if (lane == 31) abase[32] = E0;
      if (lane == 0 && publish)
        f_store(&gstate[t], (t == 0 ? kFInclusive : kFAggregate) | ((uint64_t)E0 & kFValueMask));
    }
    if (tid == 0) s_cell = 0;
    __syncthreads();
    const int64_t E = abase[32];
    const bool staged = E > 0 && !s_irr && !s_big;

    // Stages the entries [w0, w1) of the group's block in canonical order
    // (every calling warp takes cells from s_cell).
    auto build_window = [&](int64_t w0, int64_t w1) {
      for (;;) {
        int c = 0;
        if (lane == 0) c = atomicAdd(&s_cell, 1);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= n_cells) break;
        const FCell& cell = cells[c];
        const int64_t start = abase[lane] + pre[c * 32 + lane];
        const int64_t cntc = (int64_t)pre[(c + 1) * 32 + lane] - pre[c * 32 + lane];
        const bool need = cntc > 0 && start < w1 && start + cntc > w0;
        if (!__any_sync(0xffffffffu, need)) continue;
        const bool shifted = (cell.sh[0] | cell.sh[1] | cell.sh[2]) != 0;
        const int32_t io_adj = shifted ? io - 1 : io;
        const float ux = cell.t[0] - a.x, uy = cell.t[1] - a.y, uz = cell.t[2] - a.z;
        const bool live = mine && !(norm2(dsub(cell.cs[0], xi), dsub(cell.cs[1], yi),
                                          dsub(cell.cs[2], zi)) > g.prune_sq);
        int64_t pos = start;
        for (int32_t jb = cell.b0; jb < cell.b1; jb += 32) {
          uint32_t hits;
          if (cell.mbase >= 0)
            hits = masks[cell.mbase + (jb - cell.b0) + lane];
          else
            hits = f_chunk(b, cell, jb, ux, uy, uz, io_adj, live, xi, yi, zi, lo, hi, rc_sq,
                           s_gbox, st_xy[warp], st_z[warp], st_w[warp], st_map[warp]);
          if (!need) hits = 0;
          while (hits) {
            const int jj = __ffs(hits) - 1;
            hits &= hits - 1;
            if (pos >= w0 && pos < w1)
              stage[pos - w0] = ((uint32_t)lane << 27) | ((uint32_t)c << kFJBits) |
                                (uint32_t)(jb - cell.b0 + jj);
            ++pos;
          }
        }
      }
    };

    // 3b. the group within the list: warp 0 walks back over the groups
    //     before it while the other warps stage the block's first window
    if (warp == 0) {
      int64_t prefix = 0;
      bool failed_any = false;
      if (t > 0) {
        int32_t tt = t - 1;
        for (;;) {
          const int32_t pred = tt - lane;
          uint64_t v = kFInclusive;
          bool failed = false;
          if (pred >= 0) {
            int spins = 0;
            v = f_load(&gstate[pred]);
            while ((v >> kFStatusShift) == 0 && spins < o.spin_limit) {
              __nanosleep(32);
              v = f_load(&gstate[pred]);
              ++spins;
            }
            failed = (v >> kFStatusShift) == 0;
          }
          if (__any_sync(0xffffffffu, failed)) {
            if (lane == 0) atomicExch(reinterpret_cast<unsigned long long*>(&o.state[1]), 1ull);
            failed_any = true;
            break;
          }
          const unsigned inc = __ballot_sync(0xffffffffu, (v >> kFStatusShift) == 2);
          const int stop = __ffs(inc) - 1;
          int64_t val = (pred >= 0 && lane <= (stop < 0 ? 31 : stop)) ? (int64_t)(v & kFValueMask) : 0;
#pragma unroll
          for (int s = 16; s > 0; s >>= 1) val += __shfl_xor_sync(0xffffffffu, val, s);
          prefix += val;
          if (stop >= 0) break;
          tt -= 32;
        }
        if (lane == 0 && publish)
          f_store(&gstate[t], kFInclusive | ((uint64_t)(prefix + E) & kFValueMask));
      }
      if (lane == 0) {
        s_G = prefix;
        s_skip = failed_any || prefix + E > o.capacity;
        if (t == n_groups - 1) *o.total = failed_any ? 0 : prefix + E;
      }
    } else if (staged) {
      build_window(0, E < kFStage ? E : kFStage);
    }
    __syncthreads();

    // 4. write the group's block [G, G + E)
    const int64_t G = s_G;
    if (!s_skip && staged) {
      for (int64_t w0 = 0; w0 < E; w0 += kFStage) {
        const int64_t w1 = E - w0 < kFStage ? E : w0 + kFStage;
        if (w0 > 0) {
          if (tid == 0) s_cell = 0;
          __syncthreads();
          build_window(w0, w1);
          __syncthreads();
        }
        for (int64_t k = w0 + tid; k < w1; k += kFThreads) {
          const uint32_t v = stage[k - w0];
          const int l = (int)(v >> 27);
          const int c = (int)((v >> kFJBits) & 1023u);
          const int32_t jj = (int32_t)(v & ((1u << kFJBits) - 1));
          const FCell& cell = cells[c];
          const SlotMeta mj = b.meta[cell.b0 + jj];
          const SlotMeta ml = lmeta[l];
          const int64_t e = G + k;
          o.src[e] = (int64_t)ml.orig;
          o.dst[e] = (int64_t)mj.orig;
          int32_t* sp = o.sh + 3 * e;
          sp[0] = (mj.sx - ml.sx) + cell.sh[0];
          sp[1] = (mj.sy - ml.sy) + cell.sh[1];
          sp[2] = (mj.sz - ml.sz) + cell.sh[2];
        }
        __syncthreads();
      }
    } else if (!s_skip && E > 0) {
      // Groups with an irregular atom or a huge cell: each lane writes its own
      // runs (regular atoms), then the irregular atoms one warp each.
      for (int c = warp; c < n_cells; c += kFWarps) {
        const FCell& cell = cells[c];
        const int64_t start = abase[lane] + pre[c * 32 + lane];
        const int64_t cntc = (int64_t)pre[(c + 1) * 32 + lane] - pre[c * 32 + lane];
        const bool need = mine && cntc > 0;
        if (!__any_sync(0xffffffffu, need)) continue;
        const bool shifted = (cell.sh[0] | cell.sh[1] | cell.sh[2]) != 0;
        const int32_t io_adj = shifted ? io - 1 : io;
        const float ux = cell.t[0] - a.x, uy = cell.t[1] - a.y, uz = cell.t[2] - a.z;
        const bool live = mine && !(norm2(dsub(cell.cs[0], xi), dsub(cell.cs[1], yi),
                                          dsub(cell.cs[2], zi)) > g.prune_sq);
        const SlotMeta mi = lmeta[lane < len ? lane : 0];
        int64_t e = G + start;
        for (int32_t jb = cell.b0; jb < cell.b1; jb += 32) {
          uint32_t hits;
          if (cell.mbase >= 0)
            hits = masks[cell.mbase + (jb - cell.b0) + lane];
          else
            hits = f_chunk(b, cell, jb, ux, uy, uz, io_adj, live, xi, yi, zi, lo, hi, rc_sq,
                           s_gbox, st_xy[warp], st_z[warp], st_w[warp], st_map[warp]);
          if (!need) hits = 0;
          while (hits) {
            const int jj = __ffs(hits) - 1;
            hits &= hits - 1;
            const SlotMeta mj = b.meta[jb + jj];
            o.src[e] = (int64_t)mi.orig;
            o.dst[e] = (int64_t)mj.orig;
            int32_t* sp = o.sh + 3 * e;
            sp[0] = (mj.sx - mi.sx) + cell.sh[0];
            sp[1] = (mj.sy - mi.sy) + cell.sh[1];
            sp[2] = (mj.sz - mi.sz) + cell.sh[2];
            ++e;
          }
        }
      }
      if (s_irr && warp == 0) {
        for (int l = 0; l < len; ++l)
          if (b.irr[grp.first + l])
            f_irregular<true>(g, b, n_cells, rc_sq, grp.first + l, nullptr, G + abase[l], o);
      }
    }
    __syncthreads();
    // One thread releases the group's writes (ordered before it by the
    // barrier) with the completion count; the last group to complete reports.
    if (tid == 0) {
      __threadfence();
      if (atomicAdd(o.done, 1ull) == (unsigned long long)n_groups - 1ull) {
        __threadfence();
        const int64_t m = *reinterpret_cast<volatile int64_t*>(o.total);
        const int64_t err = (int64_t)f_load(&o.state[1]);
        f_report(o, m, err);
      }
    }
  }
  // No groups at all: the list is empty.
  if (n_groups == 0 && blockIdx.x == 0 && tid == 0) {
    *o.total = 0;
    f_report(o, 0, 0);
  }
  if (!o.move || n_groups == 0) return;
  // [src | dst]: once every group is written (all tickets are taken by
  // running CTAs, so the wait ends; bounded all the same), each CTA moves
  // its stride of the destinations behind the M sources.
  if (tid == 0) {
    int spins = 0;
    unsigned long long d = *reinterpret_cast<volatile unsigned long long*>(o.done);
    while (d < (unsigned long long)n_groups && spins < o.spin_limit) {
      __nanosleep(64);
      d = *reinterpret_cast<volatile unsigned long long*>(o.done);
      ++spins;
    }
    s_skip = d >= (unsigned long long)n_groups ? 0 : 1;
    if (s_skip) atomicExch(reinterpret_cast<unsigned long long*>(&o.state[1]), 1ull);
  }
  __syncthreads();
  if (s_skip) return;
  __threadfence();
  const int64_t m = *reinterpret_cast<volatile int64_t*>(o.total);
  if (m > o.capacity) return;
  for (int64_t e = (int64_t)blockIdx.x * kFThreads + tid; e < m; e += (int64_t)gridDim.x * kFThreads)
    o.src[m + e] = __ldcg(&o.dst[e]);
}

}  // namespace

size_t fused_smem_bytes(int32_t n_cells, int32_t mask_words) {
  return fused_cells_bytes(n_cells) + sizeof(uint32_t) * (((size_t)n_cells + 1) * 32 + mask_words +
                                                           kFStage);
}

void launch_pair_fused(const GridParams& g, const GridBuffers& b, int32_t n_cells,
                       const GuardBand& band, const FusedOut& o, cudaStream_t s) {
  const size_t smem = fused_smem_bytes(n_cells, o.mask_words);
  ensure_smem_attr((const void*)k_pair_fused, (int)smem);
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_fused, kFThreads, smem);
  if (per_sm < 1) per_sm = 1;
  launch_pdl(k_pair_fused, dim3((unsigned)(sms * per_sm)), dim3(kFThreads), smem, s, g, b, n_cells,
             band, o);
  note_launches(1);
}

}  // namespace nlb
