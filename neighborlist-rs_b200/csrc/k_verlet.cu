// k_verlet.cu -- kernels of the Verlet (skin) list manager.
//
//   k_max_disp      max_i |r_i - r_i,ref|^2 over the atoms (FP64, exact
//                   squares and sums; the max of non-negative doubles is
//                   taken on their bit patterns, which order the same way)
//   k_verlet_compact  one pass over the stored edges (i, j, S): kept when
//                   |(r_j - r_i) + H.S|^2 < rc^2 with the current positions
//                   (the displacement expression of k_extras.cu), compacted
//                   in stored order by a decoupled look-back over tiles
//                   ([src | dst], shifts)
// Both are HBM-bound streaming kernels (24 B per atom; 28 B + two position
// gathers per stored edge and 28 B (+ 16 for the destinations' move) per
// kept edge).
#include <algorithm>
#include <atomic>

#include "nlb_kernels.h"

namespace nlb {

namespace {

__device__ __forceinline__ void edge_disp(const double* __restrict__ pos,
                                          const EdgeExtrasCell& cell, int64_t i, int64_t j,
                                          int32_t s0, int32_t s1, int32_t s2, double* d) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double rel = dsub(pos[3 * j + k], pos[3 * i + k]);
    if (cell.has_cell) {
      const double hs = dadd(dadd(dmul(cell.h[3 * k], (double)s0),
                                  dmul(cell.h[3 * k + 1], (double)s1)),
                             dmul(cell.h[3 * k + 2], (double)s2));
      d[k] = dadd(rel, hs);
    } else {
      d[k] = rel;
    }
  }
}

__global__ void k_max_disp(const double* __restrict__ pos, const double* __restrict__ ref,
                           int64_t n, unsigned long long* __restrict__ out) {
  double best = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double d = norm2(dsub(pos[3 * i], ref[3 * i]), dsub(pos[3 * i + 1], ref[3 * i + 1]),
                           dsub(pos[3 * i + 2], ref[3 * i + 2]));
    // NaN (a broken trajectory) must force a rebuild: map it to +inf.
    const double v = d != d ? INFINITY : d;
    best = v > best ? v : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other > best ? other : best;
  }
  if ((threadIdx.x & 31) == 0)
    atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

constexpr int kVcThreads = 256;
constexpr int kVcPer = 8;                          // stored edges per thread
constexpr int kVcTile = kVcThreads * kVcPer;       // stored edges per tile
constexpr uint64_t kVcShift = 62;
constexpr uint64_t kVcAggregate = 1ull << kVcShift;
constexpr uint64_t kVcInclusive = 2ull << kVcShift;
constexpr uint64_t kVcValue = (1ull << kVcShift) - 1;

// One pass over the stored list: CTAs take tiles of kVcTile stored edges in
// order (tickets), test them at rc with the current positions (each warp a
// run of 256 edges, lane-striped so that loads are coalesced), find the
// tile's first output slot by a decoupled look-back over the tiles before it
// (bounded polls; a wait that runs out sets state[1] and the tile writes
// nothing), and write the kept edges in stored order: sources and shifts in
// place, destinations to dst_tmp.  Once every tile is written (all tickets
// are held by running CTAs, so the wait ends; bounded all the same), the
// CTAs move the destinations behind the M sources.  state (zeroed): [0]
// ticket, [1] error, [2] tiles done, [3] M, [4 + t] tile t's look-back word.
__global__ void __launch_bounds__(kVcThreads)
    k_verlet_compact(const double* __restrict__ pos, EdgeExtrasCell cell,
                     const int64_t* __restrict__ ei, const int32_t* __restrict__ sh, int64_t m,
                     double rc_sq, int64_t* __restrict__ out_ei, int32_t* __restrict__ out_sh,
                     int64_t* __restrict__ dst_tmp, uint64_t* __restrict__ state,
                     int32_t spin_limit) {
  __shared__ int64_t s_tile, s_base;
  __shared__ int32_t warp_cnt[kVcThreads / 32];
  __shared__ int32_t s_skip;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t n_tiles = (m + kVcTile - 1) / kVcTile;
  uint64_t* const tiles = state + 4;
  for (;;) {
    if (tid == 0) s_tile = (int64_t)atomicAdd(reinterpret_cast<unsigned long long*>(state), 1ull);
    __syncthreads();
    const int64_t t = s_tile;
    if (t >= n_tiles) break;
    const int64_t wbase = t * kVcTile + (int64_t)warp * 32 * kVcPer;
    uint32_t kmask[kVcPer];
    int32_t wtot = 0;
#pragma unroll
    for (int k = 0; k < kVcPer; ++k) {
      const int64_t e = wbase + 32 * k + lane;
      bool keep = false;
      if (e < m) {
        double d[3];
        edge_disp(pos, cell, ei[e], ei[m + e], sh[3 * e], sh[3 * e + 1], sh[3 * e + 2], d);
        keep = norm2(d[0], d[1], d[2]) < rc_sq;
      }
      kmask[k] = __ballot_sync(0xffffffffu, keep);
      wtot += __popc(kmask[k]);
    }
    if (lane == 0) warp_cnt[warp] = wtot;
    __syncthreads();
    int32_t woff = 0, tile_tot = 0;
#pragma unroll
    for (int w = 0; w < kVcThreads / 32; ++w) {
      const int32_t v = warp_cnt[w];
      woff += w < warp ? v : 0;
      tile_tot += v;
    }
    if (warp == 0) {
      // Publish the tile's count at once, then walk back over the tiles
      // before it (32 at a time) to its first output slot.
      if (lane == 0) {
        __threadfence();
        *reinterpret_cast<volatile uint64_t*>(&tiles[t]) =
            (t == 0 ? kVcInclusive : kVcAggregate) | (uint64_t)tile_tot;
      }
      int64_t prefix = 0;
      bool failed_any = false;
      if (t > 0) {
        int64_t tt = t - 1;
        for (;;) {
          const int64_t pred = tt - lane;
          uint64_t v = kVcInclusive;
          bool failed = false;
          if (pred >= 0) {
            int spins = 0;
            v = *reinterpret_cast<const volatile uint64_t*>(&tiles[pred]);
            while ((v >> kVcShift) == 0 && spins < spin_limit) {
              __nanosleep(32);
              v = *reinterpret_cast<const volatile uint64_t*>(&tiles[pred]);
              ++spins;
            }
            failed = (v >> kVcShift) == 0;
          }
          if (__any_sync(0xffffffffu, failed)) {
            if (lane == 0) atomicExch(reinterpret_cast<unsigned long long*>(&state[1]), 1ull);
            failed_any = true;
            break;
          }
          const unsigned inc = __ballot_sync(0xffffffffu, (v >> kVcShift) == 2);
          const int stop = __ffs(inc) - 1;
          int64_t val = (pred >= 0 && lane <= (stop < 0 ? 31 : stop)) ? (int64_t)(v & kVcValue) : 0;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
          prefix += val;
          if (stop >= 0) break;
          tt -= 32;
        }
        if (lane == 0 && !failed_any) {
          __threadfence();
          *reinterpret_cast<volatile uint64_t*>(&tiles[t]) =
              kVcInclusive | (uint64_t)(prefix + tile_tot);
        }
      }
      if (lane == 0) {
        s_base = prefix;
        s_skip = failed_any ? 1 : 0;
        if (t == n_tiles - 1) state[3] = failed_any ? 0 : (uint64_t)(prefix + tile_tot);
      }
    }
    __syncthreads();
    if (!s_skip) {
      const int64_t g = s_base + woff;
      int32_t acc = 0;
#pragma unroll
      for (int k = 0; k < kVcPer; ++k) {
        const int64_t e = wbase + 32 * k + lane;
        if ((kmask[k] >> lane) & 1u) {
          const int64_t o = g + acc + __popc(kmask[k] & ((1u << lane) - 1u));
          out_ei[o] = ei[e];
          dst_tmp[o] = ei[m + e];
          out_sh[3 * o] = sh[3 * e];
          out_sh[3 * o + 1] = sh[3 * e + 1];
          out_sh[3 * o + 2] = sh[3 * e + 2];
        }
        acc += __popc(kmask[k]);
      }
    }
    // One thread releases the tile's writes (ordered before it by the
    // barrier) with the completion count.
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(reinterpret_cast<unsigned long long*>(&state[2]), 1ull);
    }
  }
  if (n_tiles == 0) return;
  if (tid == 0) {
    int spins = 0;
    unsigned long long d = *reinterpret_cast<volatile unsigned long long*>(&state[2]);
    while (d < (unsigned long long)n_tiles && spins < spin_limit) {
      __nanosleep(64);
      d = *reinterpret_cast<volatile unsigned long long*>(&state[2]);
      ++spins;
    }
    s_skip = d >= (unsigned long long)n_tiles ? 0 : 1;
    if (s_skip) atomicExch(reinterpret_cast<unsigned long long*>(&state[1]), 1ull);
  }
  __syncthreads();
  if (s_skip) return;
  __threadfence();
  const int64_t total = (int64_t)*reinterpret_cast<volatile uint64_t*>(&state[3]);
  for (int64_t k = (int64_t)blockIdx.x * kVcThreads + tid; k < total;
       k += (int64_t)gridDim.x * kVcThreads)
    out_ei[total + k] = __ldcg(&dst_tmp[k]);
}

int stream_grid(int64_t items) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (items + 255) / 256;
  const int64_t cap = (int64_t)sms * 8;
  return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

void launch_max_disp(const double* pos, const double* ref, int64_t n, unsigned long long* out,
                     cudaStream_t s) {
  cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
  if (n <= 0) return;
  k_max_disp<<<stream_grid(n), 256, 0, s>>>(pos, ref, n, out);
  note_launches(1);
}

int64_t verlet_compact_state_words(int64_t m) { return 4 + (m + kVcTile - 1) / kVcTile; }

void launch_verlet_compact(const double* pos, const EdgeExtrasCell& cell, const int64_t* ei,
                           const int32_t* sh, int64_t m, double rc_sq, int64_t* out_ei,
                           int32_t* out_sh, int64_t* dst_tmp, uint64_t* state,
                           int32_t spin_limit, cudaStream_t s) {
  cudaMemsetAsync(state, 0, sizeof(uint64_t) * (size_t)verlet_compact_state_words(m), s);
  if (m <= 0) return;
  // (SMs and resident CTAs per SM of each device, looked up once)
  static std::atomic<int> cached[64][2];
  int dev = 0;
  cudaGetDevice(&dev);
  const bool known = dev >= 0 && dev < 64;
  int sms = known ? cached[dev][0].load() : 0, per_sm = known ? cached[dev][1].load() : 0;
  if (sms <= 0 || per_sm <= 0) {
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_verlet_compact, kVcThreads, 0);
    sms = std::max(sms, 1);
    per_sm = std::max(per_sm, 1);
    if (known) {
      cached[dev][0].store(sms);
      cached[dev][1].store(per_sm);
    }
  }
  const int64_t n_tiles = (m + kVcTile - 1) / kVcTile;
  const int64_t grid = std::min<int64_t>((int64_t)sms * per_sm, std::max<int64_t>(n_tiles, sms));
  k_verlet_compact<<<(unsigned)grid, kVcThreads, 0, s>>>(pos, cell, ei, sh, m, rc_sq, out_ei,
                                                         out_sh, dst_tmp, state, spin_limit);
  note_launches(1);
}

}  // namespace nlb
