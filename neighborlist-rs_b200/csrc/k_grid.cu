// k_grid.cu -- cell-list build on the device (src/search.rs:92-264).
//
// Order produced (identical to the reference): atoms grouped by bin in bin
// Morton-rank order; inside a bin by atom Morton key (ties: original index).
//
//   k_rank_table : Morton rank of every bin, counted analytically (no sort):
//                  rank(c) = #grid points whose 63-bit Morton code is < code(c).
//   k_prep       : per atom: fraction, wrap, Morton key, bin rank, bin histogram.
//   (scan)       : bin histogram -> bin starts.
//   k_scatter    : atoms -> bin segments (arbitrary order inside a segment).
//   k_place      : every atom to its slot (wrapped positions, wrap shifts,
//                  original indices, packed FP32 positions, group records):
//                  in bins of at most kRankSortMax atoms kPlaceSplit threads
//                  per atom count the bin's (key, index) pairs below its own
//                  (rank sort); larger bins are sorted by one CTA each -- bitonic in
//                  shared memory up to kSortCap, merge path through global
//                  scratch above it.
//   k_chunk_box  : bounding box of each 32-atom chunk (dense grids only).
#include "nlb_kernels.h"

namespace nlb {

namespace {

constexpr int kSortThreads = 128;
constexpr int kSortCap = 2048;  // elements sorted entirely in shared memory
constexpr int64_t kRankSortMax = 512;  // bins up to this size: rank placement
constexpr int kPlaceSplit = 8;         // threads per atom in the rank placement

// Grid points p (0 <= p_a < nb_a) whose Morton code is smaller than that of c.
__device__ int64_t morton_rank(const int32_t c[3], const int32_t nb[3]) {
  int64_t rank = 0;
  for (int l = 20; l >= 0; --l) {
    for (int a = 2; a >= 0; --a) {  // code bit 3l+a, most significant first
      if (!((c[a] >> l) & 1)) continue;
      int64_t cnt = 1;
      for (int b = 0; b < 3; ++b) {
        int64_t lo, len;
        if (b == a) {
          lo = ((int64_t)(c[b] >> (l + 1))) << (l + 1);
          len = (int64_t)1 << l;
        } else if (b < a) {
          lo = ((int64_t)(c[b] >> (l + 1))) << (l + 1);
          len = (int64_t)1 << (l + 1);
        } else {
          lo = ((int64_t)(c[b] >> l)) << l;
          len = (int64_t)1 << l;
        }
        int64_t hi = lo + len;
        if (hi > nb[b]) hi = nb[b];
        const int64_t w = hi - lo;
        if (w <= 0) {
          cnt = 0;
          break;
        }
        cnt *= w;
      }
      rank += cnt;
    }
  }
  return rank;
}

__global__ void k_rank_table(GridParams g, int32_t* __restrict__ rank_of_bin) {
  const int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (lin >= g.total_bins) return;
  int32_t c[3];
  c[0] = (int32_t)(lin % g.nb[0]);
  c[1] = (int32_t)((lin / g.nb[0]) % g.nb[1]);
  c[2] = (int32_t)(lin / ((int64_t)g.nb[0] * g.nb[1]));
  rank_of_bin[lin] = (int32_t)morton_rank(c, g.nb);
}

constexpr int kPrepThreads = 256;

// Exclusive scan of the bin histogram by one CTA (kPrepThreads threads):
// bin_start[b] = sum of counts below b, bin_start[nb] = total.  With
// group_start, also the exclusive scan of the 32-atom groups per bin
// (ceil(count / 32)): the canonical index of each bin's first group.
__device__ void cta_bin_scan(const int32_t* __restrict__ bin_count, int64_t nb,
                             int64_t* __restrict__ bin_start, int32_t* __restrict__ group_start) {
  __shared__ int64_t warp_tot[kPrepThreads / 32];
  __shared__ int64_t warp_grp[kPrepThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t per = (nb + kPrepThreads - 1) / kPrepThreads;
  const int64_t b0 = tid * per < nb ? tid * per : nb;
  const int64_t b1 = b0 + per < nb ? b0 + per : nb;
  int64_t sum = 0, gsum = 0;
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t v = __ldcg(&bin_count[b]);
    sum += v;
    gsum += (v + 31) / 32;
  }
  int64_t x = sum, gx = gsum;  // inclusive scans over the CTA
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    const int64_t gy = __shfl_up_sync(0xffffffffu, gx, o);
    if (lane >= o) {
      x += y;
      gx += gy;
    }
  }
  if (lane == 31) {
    warp_tot[warp] = x;
    warp_grp[warp] = gx;
  }
  __syncthreads();
  int64_t before = 0, gbefore = 0;
  for (int w = 0; w < warp; ++w) {
    before += warp_tot[w];
    gbefore += warp_grp[w];
  }
  int64_t run = before + x - sum, grun = gbefore + gx - gsum;
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t v = __ldcg(&bin_count[b]);
    bin_start[b] = run;
    run += v;
    if (group_start) group_start[b] = (int32_t)grun;
    grun += (v + 31) / 32;
  }
  if (tid == kPrepThreads - 1) bin_start[nb] = before + x;
}

// Per atom: wrap, Morton key, bin rank, histogram.  With `done`, the last
// CTA to finish also scans the histogram into bin_start.
__global__ void __launch_bounds__(kPrepThreads)
    k_prep(GridParams g, const double* __restrict__ pos, int64_t n,
           const int32_t* __restrict__ rank_of_bin, uint64_t* __restrict__ key,
           int32_t* __restrict__ rank, int32_t* __restrict__ bin_count,
           int64_t* __restrict__ bin_start, int32_t* __restrict__ done,
           int32_t* __restrict__ group_start, int32_t* __restrict__ fill) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const AtomWrap w = wrap_atom(g, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    const int64_t lin = w.bin[0] + (int64_t)g.nb[0] * (w.bin[1] + (int64_t)g.nb[1] * w.bin[2]);
    const int32_t r = rank_of_bin[lin];
    key[i] = w.key;
    rank[i] = r;
    // (the histogram's old value is the atom's place in its bin segment,
    // before the bin sort)
    const int32_t at = atomicAdd(&bin_count[r], 1);
    if (fill) fill[i] = at;
  }
  if (!done) return;
  __shared__ int last;
  // One thread releases the CTA's histogram updates (ordered before it by the
  // barrier) together with its completion count.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(done, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  cta_bin_scan(bin_count, g.total_bins, bin_start, group_start);
}

__global__ void k_scatter(const uint64_t* __restrict__ key, const int32_t* __restrict__ rank,
                          int64_t n, const int64_t* __restrict__ bin_start,
                          int32_t* __restrict__ bin_fill, uint64_t* __restrict__ skey,
                          int32_t* __restrict__ sidx, const int32_t* __restrict__ fill) {
  pdl_wait();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t r = rank[i];
  const int64_t slot = bin_start[r] + (fill ? fill[i] : atomicAdd(&bin_fill[r], 1));
  skey[slot] = key[i];
  sidx[slot] = (int32_t)i;
}

__device__ __forceinline__ bool pair_less(uint64_t ka, int32_t ia, uint64_t kb, int32_t ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Bitonic sort of cnt (<= kSortCap) pairs held in shared memory.
__device__ void smem_bitonic(uint64_t* k, int32_t* v, int cnt) {
  int p = 1;
  while (p < cnt) p <<= 1;
  for (int i = cnt + threadIdx.x; i < p; i += blockDim.x) {
    k[i] = ~0ull;
    v[i] = 0x7fffffff;
  }
  __syncthreads();
  for (int size = 2; size <= p; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < p; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const bool gt = pair_less(k[j], v[j], k[i], v[i]);
          if (gt == up) {
            const uint64_t tk = k[i];
            k[i] = k[j];
            k[j] = tk;
            const int32_t tv = v[i];
            v[i] = v[j];
            v[j] = tv;
          }
        }
      }
      __syncthreads();
    }
  }
}

// Slot p of the sorted order holds atom idx: wrapped position, wrap shifts,
// original index and, for the pair-task searches (p32 set), the packed FP32
// position in its bin's frame, the bin and the irregular flag.  Returns the
// packed position and the bin's index (zero without p32).
struct SlotOut {
  float4 q;
  int32_t lin;
};
__device__ __forceinline__ SlotOut store_slot(const GridParams& g, const double* __restrict__ pos,
                                             int64_t p, int32_t idx, double* __restrict__ px,
                                             double* __restrict__ py, double* __restrict__ pz,
                                             SlotMeta* __restrict__ meta,
                                             float4* __restrict__ p32, int32_t* __restrict__ sbin,
                                             int32_t* __restrict__ irr_list,
                                             uint8_t* __restrict__ irr,
                                             int32_t* __restrict__ counters) {
  const AtomWrap w = wrap_atom(g, pos[3 * (int64_t)idx], pos[3 * (int64_t)idx + 1],
                               pos[3 * (int64_t)idx + 2]);
  px[p] = w.wx;
  py[p] = w.wy;
  pz[p] = w.wz;
  SlotMeta mt;
  mt.sx = w.s[0];
  mt.sy = w.s[1];
  mt.sz = w.s[2];
  mt.orig = idx;
  meta[p] = mt;
  SlotOut so;
  so.q = make_float4(0.f, 0.f, 0.f, 0.f);
  so.lin = 0;
  if (p32) {
    // Bin centre of the stored bin (same expression as the prune test's
    // target centre, src/search.rs:493-497).
    double c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double t = dadd(g.origin[k], dmul(g.basis[0][k], (double)w.bin[0]));
      t = dadd(t, dmul(g.basis[1][k], (double)w.bin[1]));
      c[k] = dadd(t, dmul(g.basis[2][k], (double)w.bin[2]));
    }
    so.q = make_float4(__double2float_rn(dsub(w.wx, c[0])), __double2float_rn(dsub(w.wy, c[1])),
                       __double2float_rn(dsub(w.wz, c[2])), __int_as_float(idx));
    p32[p] = so.q;
    so.lin = w.bin[0] + g.nb[0] * (w.bin[1] + g.nb[1] * w.bin[2]);
    sbin[p] = so.lin;
    // Home stencil centre, recomputed from the wrapped position exactly as
    // the search does (src/search.rs:454-457).
    double fi[3];
    matvec(g.hinv, w.wx, w.wy, w.wz, fi);
    bool same = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int32_t v = sat_i32(dmul(fi[a], (double)g.nb[a]));
      const int32_t hb = v < g.nb[a] - 1 ? v : g.nb[a] - 1;
      same = same && hb == w.bin[a];
    }
    irr[p] = same ? 0 : 1;
    if (!same) irr_list[atomicAdd(&counters[1], 1)] = (int32_t)p;
  }
  return so;
}

// Bounding box of one 32-slot chunk held by a warp, one slot per lane
// (`valid`: the lane holds a slot); lane 0 stores it at box[0..1].
__device__ __forceinline__ void warp_box(float4 q, bool valid, float4* __restrict__ box) {
  float4 lo = q, hi = q;
  if (!valid) {
    lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o));
    lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
    lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o));
    hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
    hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o));
    hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
  }
  if ((threadIdx.x & 31) == 0) {
    box[0] = make_float4(lo.x, lo.y, lo.z, 0.f);
    box[1] = make_float4(hi.x, hi.y, hi.z, 0.f);
  }
}

// The group records of the bin of rank r (slots [s, e), bin index lin), at
// their canonical place when the group starts are known (bins in rank order,
// 32-atom runs in slot order), else where a counter puts them.
__device__ __forceinline__ void store_groups(const GridParams& g, int64_t r, int64_t s, int64_t e,
                                             int32_t lin, GroupRec* __restrict__ groups,
                                             int32_t* __restrict__ counters,
                                             const int32_t* __restrict__ group_start) {
  const int ng = (int)((e - s + 31) / 32);
  const int placed = atomicAdd(&counters[0], ng);
  const int base = group_start ? group_start[r] : placed;
  GroupRec gr;
  gr.end = (int32_t)e;
  gr.lin = lin;
  gr.bx = lin % g.nb[0];
  gr.by = (lin / g.nb[0]) % g.nb[1];
  gr.bz = lin / (g.nb[0] * g.nb[1]);
  for (int k = 0; k < ng; ++k) {
    gr.first = (int32_t)(s + 32 * k);
    groups[base + k] = gr;
  }
}

// Bins of more than kRankSortMax atoms: one CTA sorts the bin of rank r --
// bitonic in shared memory up to kSortCap, merge path through global scratch
// above it -- and gathers its slots.
__device__ void sort_bin(const GridParams& g, const double* __restrict__ pos, int64_t r,
                         const int64_t* __restrict__ bin_start, uint64_t* __restrict__ skey,
                         int32_t* __restrict__ sidx, uint64_t* __restrict__ skey2,
                         int32_t* __restrict__ sidx2, double* __restrict__ px,
                         double* __restrict__ py, double* __restrict__ pz,
                         SlotMeta* __restrict__ meta, float4* __restrict__ p32,
                         int32_t* __restrict__ sbin, GroupRec* __restrict__ groups,
                         int32_t* __restrict__ irr_list, uint8_t* __restrict__ irr,
                         int32_t* __restrict__ counters, float4* __restrict__ cbox,
                         const int32_t* __restrict__ group_start, uint64_t* sk, int32_t* sv) {
  const int64_t s = bin_start[r];
  const int64_t e = bin_start[r + 1];
  const int64_t cnt = e - s;
  const int32_t* final_idx = sidx;
  // Sort chunks of kSortCap in shared memory (the whole bin when it fits).
  for (int64_t c0 = 0; c0 < cnt; c0 += kSortCap) {
    const int m = (int)(cnt - c0 < kSortCap ? cnt - c0 : kSortCap);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      sk[i] = skey[s + c0 + i];
      sv[i] = sidx[s + c0 + i];
    }
    __syncthreads();
    smem_bitonic(sk, sv, m);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      skey[s + c0 + i] = sk[i];
      sidx[s + c0 + i] = sv[i];
    }
    __syncthreads();
  }
  if (cnt > kSortCap) {
    // Merge sorted runs pairwise (merge path per output element), ping-ponging
    // between the bin's range of (skey, sidx) and (skey2, sidx2).
    uint64_t* ak = skey + s;
    int32_t* av = sidx + s;
    uint64_t* bk = skey2 + s;
    int32_t* bv = sidx2 + s;
    for (int64_t w = kSortCap; w < cnt; w <<= 1) {
      for (int64_t d = threadIdx.x; d < cnt; d += blockDim.x) {
        const int64_t a0 = (d / (2 * w)) * (2 * w);
        const int64_t la = cnt - a0 < w ? cnt - a0 : w;
        const int64_t lb = cnt - a0 - la < w ? cnt - a0 - la : w;
        const int64_t dd = d - a0;
        const uint64_t* A = ak + a0;
        const int32_t* Av = av + a0;
        const uint64_t* B = ak + a0 + la;
        const int32_t* Bv = av + a0 + la;
        int64_t lo = dd > lb ? dd - lb : 0, hi = dd < la ? dd : la;
        while (lo < hi) {
          const int64_t mid = (lo + hi) >> 1;
          if (pair_less(A[mid], Av[mid], B[dd - mid - 1], Bv[dd - mid - 1]))
            lo = mid + 1;
          else
            hi = mid;
        }
        const int64_t ia = lo, ib = dd - lo;
        const bool take_a = ib >= lb || (ia < la && pair_less(A[ia], Av[ia], B[ib], Bv[ib]));
        bk[d] = take_a ? A[ia] : B[ib];
        bv[d] = take_a ? Av[ia] : Bv[ib];
      }
      __syncthreads();
      uint64_t* tk = ak;
      ak = bk;
      bk = tk;
      int32_t* tv = av;
      av = bv;
      bv = tv;
    }
    final_idx = av - s;
  }
  // Gather the sorted slots: wrapped positions, wrap shifts, original index.
  // Each warp pass covers one 32-slot chunk (offsets from s are multiples of
  // 32), whose box it reduces in registers.
  const int lane = threadIdx.x & 31;
  int32_t lin0 = 0;
  for (int64_t p0 = s + (threadIdx.x & ~31); p0 < e; p0 += blockDim.x) {
    const int64_t p = p0 + lane;
    SlotOut so;
    so.q = make_float4(0.f, 0.f, 0.f, 0.f);
    so.lin = 0;
    if (p < e)
      so = store_slot(g, pos, p, final_idx[p], px, py, pz, meta, p32, sbin, irr_list, irr,
                      counters);
    if (p == s) lin0 = so.lin;
    if (p32 && cbox) warp_box(so.q, p < e, cbox + 2 * p0);
  }
  if (p32 && threadIdx.x == 0) store_groups(g, r, s, e, lin0, groups, counters, group_start);
}

// Places every atom at its slot.  Blocks [0, atom_blocks): kPlaceSplit
// threads per entry p of the bin segments k_scatter wrote (arbitrary order
// inside a segment); for bins of at most kRankSortMax atoms the atom's place in its
// bin is the number of the bin's (key, index) pairs below its own (a rank
// sort: the bin's pairs are read by each of its atoms, from L1), and the
// thread writes the slot there directly; the atom placed first writes the
// bin's group records.  Blocks from atom_blocks on: block atom_blocks + r
// sorts bin r when it is larger (sort_bin).
__global__ void __launch_bounds__(kSortThreads)
    k_place(GridParams g, const double* __restrict__ pos, int64_t n,
            const int32_t* __restrict__ rank, const int64_t* __restrict__ bin_start,
            uint64_t* __restrict__ skey, int32_t* __restrict__ sidx,
            uint64_t* __restrict__ skey2, int32_t* __restrict__ sidx2,
            double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz,
            SlotMeta* __restrict__ meta, float4* __restrict__ p32, int32_t* __restrict__ sbin,
            GroupRec* __restrict__ groups, int32_t* __restrict__ irr_list,
            uint8_t* __restrict__ irr, int32_t* __restrict__ counters,
            float4* __restrict__ cbox, const int32_t* __restrict__ group_start,
            int32_t atom_blocks) {
  __shared__ uint64_t sk[kSortCap];
  __shared__ int32_t sv[kSortCap];
  pdl_wait();
  if ((int32_t)blockIdx.x >= atom_blocks) {
    const int64_t r = (int64_t)blockIdx.x - atom_blocks;
    if (bin_start[r + 1] - bin_start[r] <= kRankSortMax) return;
    sort_bin(g, pos, r, bin_start, skey, sidx, skey2, sidx2, px, py, pz, meta, p32, sbin, groups,
             irr_list, irr, counters, cbox, group_start, sk, sv);
    return;
  }
  // (kPlaceSplit consecutive threads per entry, each counting a strided
  // share of the bin: more loads in flight than one thread per atom)
  const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kPlaceSplit;
  const int part = (int)(threadIdx.x % kPlaceSplit);
  if (p >= n) return;  // (the same for the entry's threads, as below)
  const uint64_t k = skey[p];
  const int32_t i = sidx[p];
  const int32_t r = rank[i];
  const int64_t s = bin_start[r], e = bin_start[r + 1];
  if (e - s > kRankSortMax) return;
  int32_t below = 0;
  for (int64_t q = s + part; q < e; q += kPlaceSplit)
    below += pair_less(__ldg(&skey[q]), __ldg(&sidx[q]), k, i) ? 1 : 0;
  const unsigned group = ((1u << kPlaceSplit) - 1u) << (threadIdx.x & 31 & ~(kPlaceSplit - 1));
#pragma unroll
  for (int o = 1; o < kPlaceSplit; o <<= 1) below += __shfl_xor_sync(group, below, o);
  if (part != 0) return;
  const SlotOut so = store_slot(g, pos, s + below, i, px, py, pz, meta, p32, sbin, irr_list, irr,
                                counters);
  if (p32 && below == 0) store_groups(g, r, s, e, so.lin, groups, counters, group_start);
}

// Bounding box of every 32-atom group's chunk (one warp per group).
__global__ void k_chunk_box(const GroupRec* __restrict__ groups,
                            const int32_t* __restrict__ counters, const float4* __restrict__ p32,
                            float4* __restrict__ cbox) {
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t ng = counters[0];
  for (int64_t t = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ng; t += nw) {
    const GroupRec gr = groups[t];
    const int32_t end = gr.end - gr.first < 32 ? gr.end : gr.first + 32;
    const bool valid = gr.first + lane < end;
    const float4 q = valid ? p32[gr.first + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    warp_box(q, valid, cbox + 2 * (int64_t)gr.first);
  }
}

constexpr int kBoundsThreads = 1024;

__global__ void __launch_bounds__(kBoundsThreads)
    k_bounds(const double* __restrict__ pos, int64_t n, double* __restrict__ out) {
  __shared__ double red[6][kBoundsThreads / 32];
  double lo[3] = {INFINITY, INFINITY, INFINITY};
  double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double v = pos[3 * i + a];
      if (v < lo[a]) lo[a] = v;
      if (v > hi[a]) hi[a] = v;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      const double l2 = __shfl_xor_sync(0xffffffffu, lo[a], o);
      const double h2 = __shfl_xor_sync(0xffffffffu, hi[a], o);
      if (l2 < lo[a]) lo[a] = l2;
      if (h2 > hi[a]) hi[a] = h2;
    }
    if (lane == 0) {
      red[a][warp] = lo[a];
      red[3 + a][warp] = hi[a];
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double l = INFINITY, h = -INFINITY;
    for (int w = 0; w < kBoundsThreads / 32; ++w) {
      if (red[threadIdx.x][w] < l) l = red[threadIdx.x][w];
      if (red[3 + threadIdx.x][w] > h) h = red[3 + threadIdx.x][w];
    }
    out[threadIdx.x] = l;
    out[3 + threadIdx.x] = h;
  }
}

}  // namespace

void launch_bounds(const double* pos, int64_t n, double* out, cudaStream_t s) {
  k_bounds<<<1, kBoundsThreads, 0, s>>>(pos, n, out);
  note_launches(1);
}

void launch_grid_build(const GridParams& g, const double* pos, int64_t n, const GridBuffers& b,
                       cudaStream_t s, bool need_rank_table) {
  const int T = 256;
  if (need_rank_table) {
    k_rank_table<<<(unsigned)((g.total_bins + T - 1) / T), T, 0, s>>>(g, b.rank_of_bin);
    note_launches(1);
  }
  const bool fused = b.build_done != nullptr && g.total_bins <= kFusedBinScanMax;
  k_prep<<<(unsigned)((n + kPrepThreads - 1) / kPrepThreads), kPrepThreads, 0, s>>>(
      g, pos, n, b.rank_of_bin, b.key, b.rank, b.bin_count, b.bin_start,
      fused ? b.build_done : nullptr, fused ? b.group_start : nullptr, b.fill);
  if (!fused) exclusive_scan_i32(b.bin_count, g.total_bins, b.bin_start, b.scan_tmp, s);
  launch_pdl(k_scatter, dim3((unsigned)((n + T - 1) / T)), dim3(T), 0, s, b.key, b.rank, n,
             b.bin_start, b.bin_fill, b.skey, b.sidx, (const int32_t*)b.fill);
  const int32_t atom_blocks = (int32_t)((kPlaceSplit * n + kSortThreads - 1) / kSortThreads);
  launch_pdl(k_place, dim3((unsigned)(atom_blocks + g.total_bins)), dim3(kSortThreads), 0, s, g,
             pos, n, (const int32_t*)b.rank, (const int64_t*)b.bin_start, b.skey, b.sidx, b.skey2,
             b.sidx2, b.px, b.py, b.pz, b.meta, b.p32, b.sbin, b.groups, b.irr_list, b.irr,
             b.counters, b.cbox, fused ? (const int32_t*)b.group_start : nullptr, atom_blocks);
  note_launches(3);
  if (b.p32 && b.cbox) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    launch_pdl(k_chunk_box, dim3((unsigned)(2 * sms)), dim3(256), 0, s, (const GroupRec*)b.groups,
               (const int32_t*)b.counters, (const float4*)b.p32, b.cbox);
    note_launches(1);
  }
}

}  // namespace nlb
