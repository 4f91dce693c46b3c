// k_scan.cu -- exclusive prefix sums (edge counts -> int64 edge offsets,
// bin histogram -> bin starts) in ONE launch of any size.
//
// Single-pass scan with decoupled look-back: each CTA takes the next tile
// ticket (so every tile it waits on belongs to a CTA that is already
// running), scans its tile in shared memory, publishes its aggregate, then a
// warp walks back over the predecessors' published aggregates / inclusive
// prefixes 32 at a time until it meets an inclusive prefix.  Every wait is
// bounded: after kSpinLimit polls the CTA records an error in the state
// buffer (word 1, read back by the host) and stops waiting.  A failure-
// detection hook (nlb_debug_scan_stall) makes one tile of the calling
// thread's next scan withhold its publication, with a short poll limit, so
// that the bounded wait and its error report can be exercised without any
// fault: the successors give up, record the error and finish.  HBM-bound:
// 4 B read + 8 B written per element.  The state buffer (tiles + 2 words) is
// zeroed by a memset node right before the kernel.
#include "nlb_kernels.h"

namespace nlb {

namespace {

constexpr int kThreads = 256;
constexpr int kTile = (int)kScanTile;
constexpr int kItems = kTile / kThreads;
static_assert(kItems * kThreads == kTile, "tile = threads x items");
constexpr int kPadShift = 5;              // one padding word per 32 elements
constexpr int kSpinLimit = 1 << 22;

// One-shot failure-detection hook of the calling host thread (see
// nlb_debug_scan_stall): tile to withhold in the next scan and its poll limit.
thread_local int32_t tl_withhold_tile = -1;
thread_local int32_t tl_withhold_spins = 0;

constexpr uint64_t kStatusShift = 62;
constexpr uint64_t kAggregate = 1ull << kStatusShift;
constexpr uint64_t kInclusive = 2ull << kStatusShift;
constexpr uint64_t kValueMask = (1ull << kStatusShift) - 1;

__device__ __forceinline__ int pad(int i) { return i + (i >> kPadShift); }

__device__ __forceinline__ uint64_t load_state(const uint64_t* p) {
  return *reinterpret_cast<const volatile uint64_t*>(p);
}

__device__ __forceinline__ void store_state(uint64_t* p, uint64_t v) {
  __threadfence();
  *reinterpret_cast<volatile uint64_t*>(p) = v;
}

template <class TIn>
__global__ void __launch_bounds__(kThreads)
    k_scan(const TIn* __restrict__ in, int64_t n, int64_t* __restrict__ out,
           uint64_t* __restrict__ state, int32_t withhold, int32_t spin_limit) {
  // state[0]: tile ticket counter; state[1]: error flag; state[2 + t]: tile t.
  __shared__ uint32_t stage_in[kTile + kTile / 32];
  __shared__ int64_t warp_sums[kThreads / 32];
  __shared__ int64_t s_prefix;
  __shared__ int s_tile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  pdl_wait();
  if (tid == 0) s_tile = (int)atomicAdd(reinterpret_cast<unsigned long long*>(&state[0]), 1ull);
  __syncthreads();
  const int tile = s_tile;
  const int64_t base = (int64_t)tile * kTile;

  // Coalesced load into padded shared memory; each thread then owns kItems
  // consecutive elements.
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    const int i = k * kThreads + tid;
    const int64_t g = base + i;
    stage_in[pad(i)] = g < n ? (uint32_t)in[g] : 0u;
  }
  __syncthreads();
  int64_t local[kItems];
  int64_t sum = 0;
#pragma unroll
  for (int k = 0; k < kItems; ++k) {
    local[k] = sum;
    sum += stage_in[pad(tid * kItems + k)];
  }
  // Block exclusive scan of the per-thread sums.
  int64_t x = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < kThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kThreads / 32) warp_sums[lane] = w;
  }
  __syncthreads();
  const int64_t aggregate = warp_sums[kThreads / 32 - 1];
  const int64_t thread_prefix = (warp ? warp_sums[warp - 1] : 0) + x - sum;

  // Decoupled look-back (warp 0).
  if (warp == 0) {
    uint64_t* tiles = state + 2;
    int64_t prefix = 0;
    const bool publish = tile != withhold;  // false only under the test hook
    if (tile == 0) {
      if (lane == 0 && publish)
        store_state(&tiles[0], kInclusive | ((uint64_t)aggregate & kValueMask));
    } else {
      if (lane == 0 && publish)
        store_state(&tiles[tile], kAggregate | ((uint64_t)aggregate & kValueMask));
      int t = tile - 1;
      for (;;) {
        const int pred = t - lane;  // lane 0 = nearest predecessor
        uint64_t v = kInclusive;    // lanes before tile 0 act as an empty prefix
        bool failed = false;
        if (pred >= 0) {
          int spins = 0;
          v = load_state(&tiles[pred]);
          while ((v >> kStatusShift) == 0 && spins < spin_limit) {
            __nanosleep(32);
            v = load_state(&tiles[pred]);
            ++spins;
          }
          failed = (v >> kStatusShift) == 0;
        }
        if (__any_sync(0xffffffffu, failed)) {
          if (lane == 0) atomicExch(reinterpret_cast<unsigned long long*>(&state[1]), 1ull);
          break;
        }
        const bool inc = (v >> kStatusShift) == 2;
        const unsigned inc_mask = __ballot_sync(0xffffffffu, inc);
        const int stop = __ffs(inc_mask) - 1;  // nearest inclusive prefix in this window
        int64_t val = (pred >= 0 && lane <= (stop < 0 ? 31 : stop)) ? (int64_t)(v & kValueMask) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
        prefix += val;
        if (stop >= 0) break;
        t -= 32;
      }
      if (lane == 0 && publish)
        store_state(&tiles[tile], kInclusive | ((uint64_t)(prefix + aggregate) & kValueMask));
    }
    if (lane == 0) s_prefix = prefix;
  }
  __syncthreads();
  const int64_t prefix = s_prefix;

  // Results go out through shared memory in two halves so the global stores
  // are coalesced (the int64 stage reuses the input stage's space).
  int64_t* stage_out = reinterpret_cast<int64_t*>(stage_in);
  constexpr int kHalf = kTile / 2;
  for (int h = 0; h < 2; ++h) {
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
      const int i = tid * kItems + k;
      if (i >= h * kHalf && i < (h + 1) * kHalf) {
        const int li = i - h * kHalf;
        stage_out[li + (li >> kPadShift)] = prefix + thread_prefix + local[k];
      }
    }
    __syncthreads();
    for (int li = tid; li < kHalf; li += kThreads) {
      const int64_t g = base + h * kHalf + li;
      if (g < n) out[g] = stage_out[li + (li >> kPadShift)];
    }
  }
  const int64_t last_tile = n > 0 ? (n - 1) / kTile : 0;
  if (tid == 0 && tile == last_tile) out[n] = prefix + aggregate;
}

static_assert(sizeof(int64_t) * ((kTile / 2) + (kTile / 2) / 32) <=
                  sizeof(uint32_t) * (kTile + kTile / 32),
              "the output stage must fit in the input stage");

template <class TIn>
void scan_impl(const TIn* in, int64_t n, int64_t* out, int64_t* tmp, cudaStream_t s,
               bool zero_state = true) {
  const int64_t tiles = n > 0 ? (n + kTile - 1) / kTile : 1;
  if (zero_state) cudaMemsetAsync(tmp, 0, sizeof(int64_t) * (size_t)(tiles + 2), s);
  const int32_t withhold = tl_withhold_tile;
  const int32_t spins = withhold >= 0 ? tl_withhold_spins : kSpinLimit;
  tl_withhold_tile = -1;
  launch_pdl(k_scan<TIn>, dim3((unsigned)tiles), dim3(kThreads), 0, s, in, n, out,
             reinterpret_cast<uint64_t*>(tmp), withhold, spins);
  note_launches(1);
}

}  // namespace

bool scan_stall_armed() { return tl_withhold_tile >= 0; }

bool take_scan_stall(int32_t* tile, int32_t* spin_limit) {
  if (tl_withhold_tile < 0) return false;
  *tile = tl_withhold_tile;
  *spin_limit = tl_withhold_spins;
  tl_withhold_tile = -1;
  return true;
}

void arm_scan_stall(int32_t tile, int32_t spin_limit) {
  tl_withhold_tile = tile;
  tl_withhold_spins = spin_limit;
}

int64_t scan_tmp_elems(int64_t n) { return (n > 0 ? (n + kTile - 1) / kTile : 1) + 2; }

void exclusive_scan_u32(const uint32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                        cudaStream_t s) {
  scan_impl<uint32_t>(in, n, out, tmp, s);
}

void exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                        cudaStream_t s) {
  scan_impl<int32_t>(in, n, out, tmp, s);
}

void exclusive_scan_u32_zeroed(const uint32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                               cudaStream_t s) {
  scan_impl<uint32_t>(in, n, out, tmp, s, false);
}

}  // namespace nlb
