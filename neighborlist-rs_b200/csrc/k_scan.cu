// k_scan.cu -- exclusive prefix sums used by the count -> scan -> emit
// pipeline (per-atom edge counts -> int64 edge offsets) and by the bin
// histogram (bin counts -> bin starts).
//
// One tile = 1024 threads x 16 items.  Inputs up to one tile take a single
// launch; larger inputs take three (tile scans, scan of tile totals, add).
// Loads and stores are staged through shared memory so global accesses are
// coalesced.  HBM-bound: 4 B read + 8 B written per element.
#include "nlb_kernels.h"

namespace nlb {

namespace {

constexpr int kThreads = 1024;
constexpr int kItems = 16;
constexpr int64_t kTile = (int64_t)kThreads * kItems;

// Exclusive scan of one value per thread across the block; returns the
// exclusive prefix and writes the block total to *total.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
  __shared__ int64_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    int64_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  const int64_t warp_prefix = warp ? warp_sums[warp - 1] : 0;
  *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

template <class TIn>
__global__ void __launch_bounds__(kThreads) scan_tiles(const TIn* __restrict__ in, int64_t n,
                                                       int64_t* __restrict__ out,
                                                       int64_t* __restrict__ tile_totals) {
  extern __shared__ int64_t stage[];  // kTile items (128 KB, dynamic)
  const int64_t base = (int64_t)blockIdx.x * kTile;
  for (int k = 0; k < kItems; ++k) {
    const int64_t i = base + (int64_t)k * kThreads + threadIdx.x;
    stage[k * kThreads + threadIdx.x] = i < n ? (int64_t)in[i] : 0;
  }
  __syncthreads();
  int64_t loc[kItems];
  int64_t sum = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    loc[k] = sum;
    sum += stage[threadIdx.x * kItems + k];
  }
  int64_t total;
  const int64_t pre = block_exclusive_scan(sum, &total);
#pragma unroll
  for (int k = 0; k < kItems; ++k) stage[threadIdx.x * kItems + k] = pre + loc[k];
  __syncthreads();
  for (int k = 0; k < kItems; ++k) {
    const int64_t i = base + (int64_t)k * kThreads + threadIdx.x;
    if (i < n) out[i] = stage[k * kThreads + threadIdx.x];
  }
  if (threadIdx.x == 0) {
    if (tile_totals) tile_totals[blockIdx.x] = total;
    if (gridDim.x == 1) out[n] = total;
  }
}

__global__ void __launch_bounds__(kThreads) add_tile_bases(int64_t* __restrict__ out, int64_t n,
                                                           const int64_t* __restrict__ bases) {
  const int64_t base = (int64_t)blockIdx.x * kTile;
  const int64_t add = bases[blockIdx.x];
  for (int k = 0; k < kItems; ++k) {
    const int64_t i = base + (int64_t)k * kThreads + threadIdx.x;
    if (i < n) out[i] += add;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = bases[gridDim.x];
}

constexpr size_t kStageBytes = sizeof(int64_t) * kTile;

template <class TIn>
void scan_impl(const TIn* in, int64_t n, int64_t* out, int64_t* tmp, cudaStream_t s) {
  ensure_smem_attr((const void*)scan_tiles<TIn>, (int)kStageBytes);
  const int64_t tiles = (n + kTile - 1) / kTile;
  if (tiles <= 1) {
    scan_tiles<TIn><<<1, kThreads, kStageBytes, s>>>(in, n, out, nullptr);
    note_launches(1);
    return;
  }
  // tmp layout: [tile totals (tiles)] [scanned totals (tiles + 1)] [scratch...]
  int64_t* totals = tmp;
  int64_t* bases = tmp + tiles;
  scan_tiles<TIn><<<(unsigned)tiles, kThreads, kStageBytes, s>>>(in, n, out, totals);
  scan_impl<int64_t>(totals, tiles, bases, tmp + 2 * tiles + 1, s);
  add_tile_bases<<<(unsigned)tiles, kThreads, 0, s>>>(out, n, bases);
  note_launches(2);
}

}  // namespace

int64_t scan_tmp_elems(int64_t n) {
  int64_t need = 0;
  while (n > kTile) {
    const int64_t tiles = (n + kTile - 1) / kTile;
    need += 2 * tiles + 1;
    n = tiles;
  }
  return need + 1;
}

void exclusive_scan_u32(const uint32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                        cudaStream_t s) {
  scan_impl<uint32_t>(in, n, out, tmp, s);
}

void exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                        cudaStream_t s) {
  scan_impl<int32_t>(in, n, out, tmp, s);
}

}  // namespace nlb
