// nlb_api.cpp -- C ABI, dispatch and device workspace management.
//
// Host-side counterpart of the reference's drivers (src/single.rs,
// src/batch.rs, src/api.rs): validation, cell construction, the brute-force
// / cell-list dispatch, and the count -> scan -> emit orchestration of the
// CUDA kernels on a per-thread stream.  Results come back in pinned host
// memory from a reuse pool, so the device-to-host copy of the edge arrays
// runs at full PCIe rate.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/neighborlist_b200.h"
#include "nlb_geometry.h"
#include "nlb_internal.h"
#include "nlb_kernels.h"

namespace nlb {

// ------------------------------------------------------------------ errors

thread_local std::string g_last_error;

Status fail(int code, const std::string& msg) {
  g_last_error = msg;
  return Status{code};
}

Status cuda_fail(cudaError_t e, const char* what) {
  return fail(NLB_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ config

std::atomic<uint64_t> g_bf_threshold{1000};   // src/config.rs DEFAULT_BRUTE_FORCE_THRESHOLD
std::atomic<uint64_t> g_par_threshold{300};   // DEFAULT_PARALLEL_THRESHOLD
std::atomic<uint64_t> g_stack_threshold{1000};  // DEFAULT_STACK_THRESHOLD

std::atomic<int64_t> g_launches{0};
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
std::atomic<int64_t> g_graph_replays{0};
void note_graph_replay() { g_graph_replays.fetch_add(1, std::memory_order_relaxed); }

thread_local cudaStream_t tl_user_stream = nullptr;

// FP32 guard-band search (k_search2.cu) on/off; NLB_FP64_SEARCH=1 selects the
// all-FP64 kernels (same results) for comparisons.
bool fp32_search_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("NLB_FP64_SEARCH");
    return !(v && v[0] == '1');
  }();
  return on;
}
thread_local bool tl_profile = false;

// ------------------------------------------------------------------ pinned pool

namespace {

struct PinnedPool {
  std::mutex mu;
  // Blocks up to 2^kMaxShift bytes: power-of-two classes carved from
  // kChunk-byte pinned chunks; a released block goes to its class's free
  // list and is never returned to the system.  cudaHostAlloc is slow (tens
  // of ms) and serialises with other CUDA calls, so steady-state traffic
  // must not reach it.
  static constexpr int kMinShift = 12;  // 4 KB: every block 4 KB aligned
  static constexpr int kMaxShift = 28;  // 256 MB
  static constexpr size_t kChunk = size_t(512) << 20;
  std::vector<void*> free_class[kMaxShift + 1];
  std::unordered_map<void*, int> class_of;  // class blocks handed out
  char* bump = nullptr;
  size_t bump_left = 0;
  // Larger blocks: dedicated allocations, cached by size (up to kMaxCached).
  std::multimap<size_t, void*> free_blocks;  // size -> block
  std::unordered_map<void*, size_t> sizes;   // every dedicated block
  size_t cached = 0;
  static constexpr size_t kMaxCached = size_t(16) << 30;
  // Counters (nlb_pinned_stats).
  int64_t n_host_alloc = 0, us_host_alloc = 0, bytes_host_alloc = 0;
  int64_t n_host_free = 0, us_host_free = 0, n_hits = 0;

  static int class_for(size_t bytes) {
    int k = kMinShift;
    while ((size_t(1) << k) < bytes) ++k;
    return k;
  }

  void* host_alloc(size_t bytes) {
    void* p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    const int64_t us = std::chrono::duration_cast<std::chrono::microseconds>(
                           std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> lk(mu);
    ++n_host_alloc;
    us_host_alloc += us;
    bytes_host_alloc += (int64_t)bytes;
    return p;
  }

  // Splits the rest of the current chunk into free class blocks, largest
  // first (every block size is a multiple of 4 KB, so all stay 4 KB aligned).
  void retire_chunk_locked() {
    for (int k = kMaxShift; k >= kMinShift && bump_left; --k) {
      const size_t b = size_t(1) << k;
      while (bump_left >= b) {
        free_class[k].push_back(bump);
        bump += b;
        bump_left -= b;
      }
    }
    bump = nullptr;
    bump_left = 0;
  }

  // Takes a class-k block from the free list, the current chunk, or by
  // splitting the smallest larger free block in halves (under mu); only when
  // all three fail does the caller pin a new chunk.
  void* take_class_locked(int k) {
    if (!free_class[k].empty()) {
      void* p = free_class[k].back();
      free_class[k].pop_back();
      ++n_hits;
      return p;
    }
    const size_t b = size_t(1) << k;
    if (bump_left >= b) {
      void* p = bump;
      bump += b;
      bump_left -= b;
      return p;
    }
    for (int j = k + 1; j <= kMaxShift; ++j) {
      if (free_class[j].empty()) continue;
      char* p = static_cast<char*>(free_class[j].back());
      free_class[j].pop_back();
      for (int i = j - 1; i >= k; --i) free_class[i].push_back(p + (size_t(1) << i));
      ++n_hits;
      return p;
    }
    return nullptr;
  }

  void* alloc(size_t bytes) {
    bytes = std::max<size_t>(bytes, 256);
    if (bytes <= (size_t(1) << kMaxShift)) {
      const int k = class_for(bytes);
      {
        std::lock_guard<std::mutex> lk(mu);
        if (void* p = take_class_locked(k)) {
          class_of[p] = k;
          return p;
        }
      }
      void* chunk = host_alloc(kChunk);
      if (!chunk) return nullptr;
      std::lock_guard<std::mutex> lk(mu);
      retire_chunk_locked();
      bump = static_cast<char*>(chunk);
      bump_left = kChunk;
      void* p = take_class_locked(k);
      class_of[p] = k;
      return p;
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = free_blocks.lower_bound(bytes);
      if (it != free_blocks.end() && it->first <= 2 * bytes + (size_t(1) << 20)) {
        void* p = it->second;
        cached -= it->first;
        free_blocks.erase(it);
        ++n_hits;
        return p;
      }
    }
    void* p = host_alloc(bytes);
    if (!p) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    sizes[p] = bytes;
    return p;
  }

  // Pre-carves chunks so that the first `bytes` of class traffic do not
  // wait for cudaHostAlloc.
  void reserve(size_t bytes) {
    size_t have = 0;
    {
      std::lock_guard<std::mutex> lk(mu);
      have = bump_left;
      for (int k = kMinShift; k <= kMaxShift; ++k) have += free_class[k].size() << k;
    }
    while (have < bytes) {
      void* chunk = host_alloc(kChunk);
      if (!chunk) return;
      std::lock_guard<std::mutex> lk(mu);
      retire_chunk_locked();
      bump = static_cast<char*>(chunk);
      bump_left = kChunk;
      have += kChunk;
    }
  }

  // Slices: results that point into a shared block (one device-to-host copy
  // for many results); the block returns to the pool with its last slice.
  std::unordered_map<void*, void*> slice_block;
  std::unordered_map<void*, int64_t> block_refs;

  void share(void* block, void* slice) {
    std::lock_guard<std::mutex> lk(mu);
    slice_block[slice] = block;
    ++block_refs[block];
  }

  void release(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu);
    auto sl = slice_block.find(p);
    if (sl != slice_block.end()) {
      void* block = sl->second;
      slice_block.erase(sl);
      if (--block_refs[block] > 0) return;
      block_refs.erase(block);
      p = block;
    }
    auto ck = class_of.find(p);
    if (ck != class_of.end()) {
      free_class[ck->second].push_back(p);
      class_of.erase(ck);
      return;
    }
    auto it = sizes.find(p);
    if (it == sizes.end()) return;  // not ours
    const size_t sz = it->second;
    while (cached + sz > kMaxCached && !free_blocks.empty()) {
      auto big = std::prev(free_blocks.end());
      cached -= big->first;
      sizes.erase(big->second);
      const auto t0 = std::chrono::steady_clock::now();
      cudaFreeHost(big->second);
      us_host_free += std::chrono::duration_cast<std::chrono::microseconds>(
                          std::chrono::steady_clock::now() - t0).count();
      ++n_host_free;
      free_blocks.erase(big);
    }
    free_blocks.emplace(sz, p);
    cached += sz;
  }
};

PinnedPool& pinned_pool() {
  static PinnedPool* pool = new PinnedPool();  // never destroyed (process lifetime)
  return *pool;
}

}  // namespace

void* pinned_alloc(size_t bytes) { return pinned_pool().alloc(bytes); }
void pinned_release(void* p) { pinned_pool().release(p); }
void pinned_share(void* block, void* slice) { pinned_pool().share(block, slice); }

void pinned_reserve(size_t bytes) { pinned_pool().reserve(bytes); }

void pinned_stats(int64_t* out) {
  PinnedPool& p = pinned_pool();
  std::lock_guard<std::mutex> lk(p.mu);
  out[0] = p.n_host_alloc;
  out[1] = p.us_host_alloc;
  out[2] = p.bytes_host_alloc;
  out[3] = p.n_host_free;
  out[4] = p.us_host_free;
  out[5] = p.n_hits;
  size_t cached = p.cached + p.bump_left;
  for (int k = PinnedPool::kMinShift; k <= PinnedPool::kMaxShift; ++k)
    cached += p.free_class[k].size() << k;
  out[6] = (int64_t)cached;
}

// ------------------------------------------------------------------ context

namespace {

// Per-device stream-ordered pool of the single-system result arrays, so that
// a build can hand its arrays to the caller (nlb_build_device_owned) and the
// next build gets fresh ones without cudaMalloc's device-wide cost.  Memory
// stays mapped in the pool (release threshold: unlimited).
struct ResultPool {
  std::mutex mu;
  cudaMemPool_t pool[64] = {};
  // Blocks handed to callers: pointer -> (device, bytes).
  std::unordered_map<void*, std::pair<int, size_t>> owned;
  int64_t handed = 0, returned = 0;
};

ResultPool& result_pool() {
  static ResultPool* p = new ResultPool();  // process lifetime
  return *p;
}

cudaMemPool_t result_pool_for(int dev) {
  ResultPool& rp = result_pool();
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(rp.mu);
  if (!rp.pool[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    rp.pool[dev] = pool;
  }
  return rp.pool[dev];
}

}  // namespace

void take_result_arrays(Ctx& c, int64_t** ei, int32_t** sh) {
  ResultPool& rp = result_pool();
  std::lock_guard<std::mutex> lk(rp.mu);
  Ctx::Buf* bs[2] = {&c.bufs[kSlotOutEi], &c.bufs[kSlotOutSh]};
  for (Ctx::Buf* b : bs) {
    if (b->p) {
      rp.owned[b->p] = {c.device, b->cap};
      ++rp.handed;
    }
  }
  *ei = static_cast<int64_t*>(bs[0]->p);
  *sh = static_cast<int32_t*>(bs[1]->p);
  *bs[0] = Ctx::Buf{};
  *bs[1] = Ctx::Buf{};
}

void warm_result_pool(int device, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = result_pool_for(device);
  void* p = nullptr;
  if (pool && bytes > 0 && cudaMallocFromPoolAsync(&p, bytes, pool, s) == cudaSuccess) {
    cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
  }
  cudaGetLastError();
}

void* alloc_owned_device(int device, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = result_pool_for(device);
  void* p = nullptr;
  if (!pool || cudaMallocFromPoolAsync(&p, std::max<size_t>(bytes, 256), pool, s) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  ResultPool& rp = result_pool();
  std::lock_guard<std::mutex> lk(rp.mu);
  rp.owned[p] = {device, bytes};
  ++rp.handed;
  return p;
}

void release_owned_device(void* p, cudaStream_t s) {
  if (!p) return;
  ResultPool& rp = result_pool();
  {
    std::lock_guard<std::mutex> lk(rp.mu);
    if (rp.owned.erase(p) == 0) return;
    ++rp.returned;
  }
  cudaFreeAsync(p, s);
}

void* Ctx::raw(int slot, size_t bytes) {
  Buf& b = bufs[slot];
  if (bytes > b.cap) {
    // Every slot comes from the stream-ordered pool (result arrays must, to
    // be handed over; the others so that a grown slot's old memory stays
    // mapped for the next allocation instead of being unmapped by cudaFree
    // and mapped again by cudaMalloc).  Growth waits for the device first
    // (the old array may still be in use on another stream, as a cudaFree
    // would).
    if (b.p) {
      cudaDeviceSynchronize();
      if (b.pooled)
        cudaFreeAsync(b.p, stream);
      else
        cudaFree(b.p);
    }
    b = Buf{};
    const size_t cap = std::max<size_t>(bytes + bytes / 4, 4096);
    cudaMemPool_t pool = result_pool_for(device);
    if (!pool || cudaMallocFromPoolAsync(&b.p, cap, pool, stream) != cudaSuccess) {
      cudaGetLastError();
      b = Buf{};
      return nullptr;
    }
    b.cap = cap;
    b.pooled = true;
    return b.p;
  }
  return b.p;
}

namespace {
thread_local std::unordered_map<int, Ctx*> tl_ctxs;
}  // namespace

void release_thread_ctx() {
  release_fast_states();
  release_batch_graphs();
  for (auto& kv : tl_ctxs) {
    Ctx* c = kv.second;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    for (Ctx::Buf& b : c->bufs) {
      if (b.p && b.pooled)
        cudaFreeAsync(b.p, c->own_stream);
      else if (b.p)
        cudaFree(b.p);
    }
    cudaStreamSynchronize(c->own_stream);
    for (Ctx::Buf& b : c->batch_out)
      if (b.p) cudaFree(b.p);
    for (cudaEvent_t ev : c->ev)
      if (ev) cudaEventDestroy(ev);
    tune_release(*c);
    if (c->h_small) cudaFreeHost(c->h_small);
    if (c->h_report) cudaFreeHost(c->h_report);
    if (c->early_ev) cudaEventDestroy(c->early_ev);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    cudaSetDevice(prev);
    delete c;
  }
  tl_ctxs.clear();
}

Status get_ctx(Ctx** out) {
  auto& ctxs = tl_ctxs;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice (is a CUDA device present?)");
  Ctx* c = nullptr;
  auto it = ctxs.find(dev);
  if (it != ctxs.end()) {
    c = it->second;
  } else {
    c = new Ctx();  // lives until release_thread_ctx (server workers) or process exit
    c->device = dev;
    e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
    e = cudaHostAlloc((void**)&c->h_small, sizeof(int64_t) * kSmallHost, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc");
    e = cudaHostAlloc((void**)&c->h_report, sizeof(int64_t) * 8, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&c->d_report, c->h_report, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc (mapped)");
    e = cudaEventCreateWithFlags(&c->early_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreate");
    for (int i = 0; i < 6; ++i) cudaEventCreate(&c->ev[i]);
    ctxs[dev] = c;
  }
  c->stream = tl_user_stream ? tl_user_stream : c->own_stream;
  if (c->early_stream && c->early_stream != c->stream) {
    // The last call returned early on another stream: this stream's work
    // follows it.
    e = cudaStreamWaitEvent(c->stream, c->early_ev, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
    c->early_stream = nullptr;
  }
  if (tl_profile != c->prof) {
    c->prof = tl_profile;
    c->prof_pending_count = c->prof_pending_emit = false;
  }
  *out = c;
  return Status{NLB_OK};
}

// Accumulates the phase times of completed (synchronized) profiled work.
void Ctx::harvest() {
  float ms = 0.f;
  if (prof_pending_count) {
    if (cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) prof_ms[0] += ms;
    if (cudaEventElapsedTime(&ms, ev[1], ev[2]) == cudaSuccess) prof_ms[1] += ms;
    if (cudaEventElapsedTime(&ms, ev[2], ev[3]) == cudaSuccess) prof_ms[2] += ms;
    prof_pending_count = false;
  }
  if (prof_pending_emit) {
    if (cudaEventElapsedTime(&ms, ev[4], ev[5]) == cudaSuccess) prof_ms[3] += ms;
    prof_pending_emit = false;
    prof_calls += 1;
  }
  cudaGetLastError();
}

void ensure_smem_attr(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;  // (func, device) -> bytes
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(func, dev);
  auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return;
  cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  done[key] = bytes;
}

// ------------------------------------------------------------------ one system

// Counts one system's edges per sorted cutoff.  Leaves the per-atom offsets
// in the context for emit_system().  Synchronizes once (to read the totals).
Status count_system(Ctx& c, SystemPlan& sp, const double* d_pos) {
  const int64_t n = sp.n;
  const int32_t k = (int32_t)sp.rc_sq.size();
  cudaStream_t s = c.stream;
  // Count layout: k rows of n + 1 per-atom counts, or (pair tasks) one row of
  // n * S per-(atom, stencil cell) counts plus a trailing zero.
  const int64_t cells = sp.fp32 ? (int64_t)(2 * sp.grid.ns[0] + 1) * (2 * sp.grid.ns[1] + 1) *
                                      (2 * sp.grid.ns[2] + 1)
                                : 0;
  const int64_t row = sp.fp32 ? n * cells + 1 : n + 1;
  sp.row = row;
  sp.counts = slot<uint32_t>(c, kSlotCounts, (size_t)k * row);
  sp.offs = slot<int64_t>(c, kSlotOffs, (size_t)k * row + 1);
  // Offsets-scan state, then a separate state for the bin scan of grids too
  // large for k_prep's own (so that each keeps its own error word).
  const int64_t offs_state = scan_tmp_elems((int64_t)k * row);
  int64_t* scan_tmp = slot<int64_t>(
      c, kSlotScanTmp, (size_t)(offs_state + scan_tmp_elems(sp.grid.total_bins)));
  if (!sp.counts || !sp.offs || !scan_tmp) return fail(NLB_ERR_NOMEM, "device allocation failed");

  c.mark(0);
  if (sp.method == Method::kCellList) {
    GridBuffers& b = sp.gb;
    const int64_t nb = sp.grid.total_bins;
    const size_t tab_cap_before = c.bufs[kSlotRankTab].cap;
    const void* tab_before = c.bufs[kSlotRankTab].p;
    b.rank_of_bin = slot<int32_t>(c, kSlotRankTab, nb);
    const bool same_tab = b.rank_of_bin == tab_before && tab_cap_before > 0 &&
                          c.rank_nb[0] == sp.grid.nb[0] && c.rank_nb[1] == sp.grid.nb[1] &&
                          c.rank_nb[2] == sp.grid.nb[2];
    // One zeroed block: bin histogram, scatter cursors, pair-task counters,
    // 64-bit hit-mask cursor (8-byte aligned: 2 nb + 2 is even), build
    // completion count, emit task counter.
    int32_t* zeroed = slot<int32_t>(c, kSlotBinCount, 2 * (size_t)nb + 6);
    b.bin_count = zeroed;
    b.bin_fill = zeroed ? zeroed + nb : nullptr;
    b.build_done = zeroed ? zeroed + 2 * nb + 4 : nullptr;
    b.emit_queue = zeroed ? reinterpret_cast<uint32_t*>(zeroed + 2 * nb + 5) : nullptr;
    b.bin_start = slot<int64_t>(c, kSlotBinStart, nb + 1);
    b.key = slot<uint64_t>(c, kSlotKey, n);
    b.rank = slot<int32_t>(c, kSlotRank, n);
    b.skey = slot<uint64_t>(c, kSlotSkey, n);
    b.sidx = slot<int32_t>(c, kSlotSidx, n);
    b.skey2 = slot<uint64_t>(c, kSlotSkey2, n);
    b.sidx2 = slot<int32_t>(c, kSlotSidx2, n);
    b.px = slot<double>(c, kSlotPx, n);
    b.py = slot<double>(c, kSlotPy, n);
    b.pz = slot<double>(c, kSlotPz, n);
    b.meta = slot<SlotMeta>(c, kSlotMeta, n);
    b.scan_tmp = scan_tmp + offs_state;
    b.p32 = nullptr;
    b.sbin = nullptr;
    b.groups = nullptr;
    b.irr_list = nullptr;
    b.irr = nullptr;
    b.counters = nullptr;
    if (sp.fp32) {
      b.p32 = slot<float4>(c, kSlotP32, n);
      b.sbin = slot<int32_t>(c, kSlotSbin, n);
      b.groups = slot<GroupRec>(c, kSlotGroups, n / 32 + std::min<int64_t>(n, nb) + 1);
      b.irr_list = slot<int32_t>(c, kSlotIrrList, n);
      b.irr = slot<uint8_t>(c, kSlotIrr, n);
      b.counters = zeroed ? zeroed + 2 * nb : nullptr;
      // Hit masks of all k cutoffs, recorded by the count pass for the emit
      // pass: the last run's need x 1.25, at least 64 words per atom and
      // cutoff (tasks that do not fit recompute their tests in the emit).
      const int64_t max_tasks = (n / 32 + std::min<int64_t>(n, nb) + 1) * cells;
      int64_t mask_cap = std::max<int64_t>((int64_t)k * 64 * n + 4096,
                                           c.pair_mask_words + c.pair_mask_words / 4);
      const int64_t mask_have = (int64_t)(c.bufs[kSlotMasks].cap / sizeof(uint32_t));
      if (mask_have > mask_cap) mask_cap = mask_have;
      b.task_hdr = slot<int4>(c, kSlotTaskHdr, max_tasks);
      b.masks = slot<uint32_t>(c, kSlotMasks, mask_cap);
      const bool chunk_boxes = (double)n / (double)nb >= kChunkPruneMinPerBin;
      b.cbox = chunk_boxes ? slot<float4>(c, kSlotCbox, 2 * (size_t)n) : nullptr;
      if (chunk_boxes && !b.cbox) return fail(NLB_ERR_NOMEM, "device allocation failed");
      b.mask_cap = mask_cap;
      b.mask_top = zeroed ? reinterpret_cast<unsigned long long*>(zeroed + 2 * nb + 2) : nullptr;
      if (!b.p32 || !b.sbin || !b.groups || !b.irr_list || !b.irr || !b.counters ||
          !b.task_hdr || !b.masks || !b.mask_top)
        return fail(NLB_ERR_NOMEM, "device allocation failed");
    }
    if (!b.rank_of_bin || !b.bin_count || !b.bin_fill || !b.bin_start || !b.key || !b.rank ||
        !b.skey || !b.sidx || !b.skey2 || !b.sidx2 || !b.px || !b.py || !b.pz || !b.meta)
      return fail(NLB_ERR_NOMEM, "device allocation failed");
    cudaMemsetAsync(zeroed, 0, sizeof(int32_t) * (2 * (size_t)nb + 6), s);
    launch_grid_build(sp.grid, d_pos, n, b, s, !same_tab);
    for (int a = 0; a < 3; ++a) c.rank_nb[a] = sp.grid.nb[a];
  }
  c.mark(1);
  const bool pair_tasks = sp.method == Method::kCellList && sp.fp32;
  if (pair_tasks) {
    sp.pbands.row = row;
    launch_pair_count_multi(sp.grid, sp.gb, n, sp.pbands, sp.counts, s);
  }
  for (int32_t g0 = 0; g0 < k && !pair_tasks; g0 += kMaxCutoffsPerPass) {
    CutoffSet cs = sp.pass(g0);
    uint32_t* rows = sp.counts + (size_t)g0 * row;
    if (sp.method == Method::kCellList)
      launch_grid_count(sp.grid, sp.gb, n, cs, rows, s);
    else
      launch_brute_count(sp.brute, d_pos, n, cs, rows, s);
  }
  c.mark(2);
  exclusive_scan_u32(sp.counts, (int64_t)k * row, sp.offs, scan_tmp, s);
  c.mark(3);
  // Row starts offs[q * row], q = 0..k, in one strided copy.
  if (k + 4 > kSmallHost) return fail(NLB_ERR_VALUE, "too many cutoffs");
  cudaError_t e = cudaMemcpy2DAsync(c.h_small, sizeof(int64_t), sp.offs, sizeof(int64_t) * row,
                                    sizeof(int64_t), (size_t)k + 1, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)  // the scan's bounded-wait error word
    e = cudaMemcpyAsync(c.h_small + k + 1, scan_tmp + 1, sizeof(int64_t), cudaMemcpyDeviceToHost,
                        s);
  if (e == cudaSuccess && pair_tasks)  // hit-mask words the count pass asked for
    e = cudaMemcpyAsync(c.h_small + k + 2, sp.gb.mask_top, sizeof(int64_t),
                        cudaMemcpyDeviceToHost, s);
  const bool bin_scan = sp.method == Method::kCellList &&
                        !(sp.gb.build_done && sp.grid.total_bins <= kFusedBinScanMax);
  c.h_small[k + 3] = 0;
  if (e == cudaSuccess && bin_scan)  // the separate bin scan's error word
    e = cudaMemcpyAsync(c.h_small + k + 3, sp.gb.scan_tmp + 1, sizeof(int64_t),
                        cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy2DAsync");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "count pass");
  if (c.h_small[k + 1] != 0 || c.h_small[k + 3] != 0)
    return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
  if (c.prof) {
    c.harvest();  // a previous emit on this stream is complete too
    c.prof_pending_count = true;
    c.harvest();
  }
  if (pair_tasks) c.pair_mask_words = c.h_small[k + 2];
  sp.m.resize(k);
  for (int32_t q = 0; q < k; ++q) sp.m[q] = c.h_small[q + 1] - c.h_small[q];
  return Status{NLB_OK};
}

// Emits one system's edges into the given device lists (per sorted cutoff).
Status emit_system(Ctx& c, SystemPlan& sp, const double* d_pos, const DevLists& L,
                   const int64_t* base, int64_t index_offset) {
  const int32_t k = (int32_t)sp.rc_sq.size();
  c.mark(4);
  const bool pair_tasks = sp.method == Method::kCellList && sp.fp32;
  if (pair_tasks) {
    EmitTargets t;
    std::memset(&t, 0, sizeof(t));
    for (int32_t q = 0; q < k; ++q) {
      t.src[q] = L.src[q];
      t.dst[q] = L.dst[q];
      t.sh[q] = L.sh[q];
      t.base[q] = base[q];
    }
    t.index_offset = index_offset;
    launch_pair_emit_multi(sp.grid, sp.gb, sp.n, sp.pbands, sp.offs, t, c.stream);
  }
  for (int32_t g0 = 0; g0 < k && !pair_tasks; g0 += kMaxCutoffsPerPass) {
    CutoffSet cs = sp.pass(g0);
    EmitTargets t;
    std::memset(&t, 0, sizeof(t));
    for (int32_t q = 0; q < cs.k; ++q) {
      t.src[q] = L.src[g0 + q];
      t.dst[q] = L.dst[g0 + q];
      t.sh[q] = L.sh[g0 + q];
      t.base[q] = base[g0 + q];
    }
    t.index_offset = index_offset;
    const int64_t* offs = sp.offs + (size_t)g0 * sp.row;
    if (sp.method == Method::kCellList)
      launch_grid_emit(sp.grid, sp.gb, sp.n, cs, offs, t, c.stream);
    else
      launch_brute_emit(sp.brute, d_pos, sp.n, cs, offs, t, c.stream);
  }
  c.mark(5);
  if (c.prof) c.prof_pending_emit = true;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "emit launch");
  return Status{NLB_OK};
}

CutoffSet SystemPlan::pass(int32_t g0) const {
  CutoffSet cs;
  std::memset(&cs, 0, sizeof(cs));
  const int32_t k = (int32_t)rc_sq.size();
  cs.k = std::min<int32_t>(kMaxCutoffsPerPass, k - g0);
  for (int32_t q = 0; q < cs.k; ++q) cs.rc_sq[q] = rc_sq[g0 + q];
  cs.disjoint = disjoint ? 1 : 0;
  cs.lower_sq = g0 > 0 ? rc_sq[g0 - 1] : -1.0;
  cs.max_sq = rc_sq.back();
  return cs;
}

// Validates and plans one system (cell or auto-box, dispatch, grid).
Status plan_system(const double* pos_host, int64_t n, const double* cell9, const bool pbc[3],
                   const std::vector<double>& cutoffs, bool disjoint, bool multi,
                   SystemPlan& sp, const double* bounds6) {
  sp.n = n;
  sp.disjoint = disjoint;
  const int32_t k = (int32_t)cutoffs.size();
  double rc_max = NAN;
  for (double r : cutoffs) rc_max = fmax_nan_ignoring(rc_max, r);
  std::string err;
  if (cell9) {
    if (!make_cell(cell9, pbc, sp.cell, err)) return fail(NLB_ERR_VALUE, err);
  } else if (bounds6) {
    if (!auto_box_from_bounds(bounds6, bounds6 + 3, rc_max, sp.cell, err))
      return fail(NLB_ERR_VALUE, err);
  } else {
    if (!auto_box(pos_host, n, rc_max, sp.cell, err)) return fail(NLB_ERR_VALUE, err);
  }
  sp.order = cutoff_order(cutoffs.data(), k);
  sp.rc_sq.resize(k);
  for (int32_t q = 0; q < k; ++q) sp.rc_sq[q] = cutoffs[sp.order[q]] * cutoffs[sp.order[q]];
  sp.method = choose_method(sp.cell, n, rc_max, g_bf_threshold.load(), multi);
  if (sp.method == Method::kCellList) {
    plan_grid(sp.cell, rc_max, sp.grid);
    for (int a = 0; a < 3; ++a)
      if (sp.grid.nb[a] >= (1 << 21))
        return fail(NLB_ERR_VALUE, "cell list needs more than 2^21 bins along one axis");
    if (sp.grid.total_bins > ((int64_t)1 << 31) - 2)
      return fail(NLB_ERR_VALUE, "cell list needs more than 2^31 bins");
    for (int a = 0; a < 3; ++a)
      if (sp.grid.ns[a] < 0 || sp.grid.ns[a] > (1 << 20))
        return fail(NLB_ERR_VALUE, "stencil too large for this cutoff and cell");
    // FP32 pair tasks with a guard band per cutoff, all cutoffs in one
    // traversal of the grid built at the largest.
    sp.fp32 = false;
    if (fp32_search_enabled() && k <= kFp32MaxCutoffs) {
      PairBands pb;
      std::memset(&pb, 0, sizeof(pb));
      pb.k = k;
      pb.disjoint = disjoint ? 1 : 0;
      bool ok = true;
      for (int32_t q = 0; q < k && ok; ++q)
        ok = make_guard_band(sp.grid, cutoffs[sp.order[q]], pb.q[q]);
      if (ok) {
        sp.pbands = pb;
        sp.band = pb.q[0];
        sp.fp32 = true;
      }
    }
  } else {
    std::memcpy(sp.brute.h, sp.cell.h, sizeof(sp.brute.h));
    std::memcpy(sp.brute.hinv, sp.cell.hinv, sizeof(sp.brute.hinv));
    for (int a = 0; a < 3; ++a) sp.brute.pbc[a] = sp.cell.pbc[a] ? 1 : 0;
    sp.brute.mode = sp.method == Method::kBruteIsolated ? kBruteRaw : kBruteMicMode;
  }
  if (n > (int64_t)INT32_MAX - 1) return fail(NLB_ERR_VALUE, "more than 2^31 atoms in one system");
  return Status{NLB_OK};
}

// ------------------------------------------------------------------ results

Status alloc_result(int64_t m, nlb_result* r) {
  r->n_edges = m;
  r->edge_index = static_cast<int64_t*>(pinned_alloc(sizeof(int64_t) * 2 * (size_t)m));
  r->shift = static_cast<int32_t*>(pinned_alloc(sizeof(int32_t) * 3 * (size_t)m));
  if (!r->edge_index || !r->shift) {
    pinned_release(r->edge_index);
    pinned_release(r->shift);
    r->edge_index = nullptr;
    r->shift = nullptr;
    return fail(NLB_ERR_NOMEM, "pinned host allocation failed");
  }
  return Status{NLB_OK};
}

void zero_results(nlb_result* outs, int32_t k) {
  for (int32_t q = 0; q < k; ++q) {
    outs[q].n_edges = 0;
    outs[q].edge_index = nullptr;
    outs[q].shift = nullptr;
  }
}

Status empty_results(nlb_result* outs, int32_t k) {
  for (int32_t q = 0; q < k; ++q) {
    Status st = alloc_result(0, &outs[q]);
    if (!st.ok()) return st;
  }
  return Status{NLB_OK};
}

// Device output workspace for k lists of sizes m[q], laid out exactly like
// the host results ([src | dst] per list) so each list downloads in one copy.
Status device_outputs(Ctx& c, const std::vector<int64_t>& m, DevLists& L) {
  int64_t tot = 0;
  for (int64_t x : m) tot += x;
  int64_t* ei_all = slot<int64_t>(c, kSlotOutEi, 2 * (size_t)tot);
  int32_t* sh_all = slot<int32_t>(c, kSlotOutSh, 3 * (size_t)tot);
  if (!ei_all || !sh_all) return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");
  L.src.resize(m.size());
  L.dst.resize(m.size());
  L.sh.resize(m.size());
  int64_t acc = 0;
  for (size_t q = 0; q < m.size(); ++q) {
    L.src[q] = ei_all + 2 * acc;
    L.dst[q] = ei_all + 2 * acc + m[q];
    L.sh[q] = sh_all + 3 * acc;
    acc += m[q];
  }
  return Status{NLB_OK};
}

// Copies contiguous device lists (sorted cutoff order) to pinned results in
// input cutoff order.
Status download_results(Ctx& c, const std::vector<int64_t>& m, const DevLists& L,
                        const std::vector<int32_t>& order, nlb_result* outs) {
  const int32_t k = (int32_t)m.size();
  for (int32_t q = 0; q < k; ++q) {
    nlb_result& r = outs[order[q]];
    Status st = alloc_result(m[q], &r);
    if (!st.ok()) return st;
    if (m[q] == 0) continue;
    // [src | dst] in one copy when the destinations follow the sources.
    const bool joined = L.dst[q] == L.src[q] + m[q];
    cudaError_t e = cudaMemcpyAsync(r.edge_index, L.src[q],
                                    sizeof(int64_t) * (joined ? 2 : 1) * m[q],
                                    cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess && !joined)
      e = cudaMemcpyAsync(r.edge_index + m[q], L.dst[q], sizeof(int64_t) * m[q],
                          cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(r.shift, L.sh[q], sizeof(int32_t) * 3 * m[q], cudaMemcpyDeviceToHost,
                          c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (results)");
  }
  cudaError_t e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return cuda_fail(e, "emit pass");
  if (c.prof) c.harvest();
  return Status{NLB_OK};
}

Status upload_positions(Ctx& c, const double* pos, int64_t n, double** d_pos) {
  *d_pos = slot<double>(c, kSlotPos, 3 * (size_t)n);
  if (!*d_pos) return fail(NLB_ERR_NOMEM, "device allocation failed");
  // (Staging large pageable inputs through a pinned block with host threads
  // measured slower than the driver's own pageable copy: 1.0 vs 0.7 ms for
  // the 13 MB of the 4096-system batch.)
  const size_t bytes = sizeof(double) * 3 * (size_t)n;
  cudaError_t e = cudaMemcpyAsync(*d_pos, pos, bytes, cudaMemcpyHostToDevice, c.stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (positions)");
  return Status{NLB_OK};
}

bool cutoffs_valid(const double* cs, int32_t k) {
  for (int32_t q = 0; q < k; ++q)
    if (!std::isfinite(cs[q]) || cs[q] <= 0.0) return false;
  return true;
}

// One system, k cutoffs, host in / host out.
Status run_single(const double* pos, int64_t n, const double* cell9, const uint8_t* pbc,
                  const double* cutoffs, int32_t k, bool disjoint, bool multi, nlb_result* outs) {
  zero_results(outs, k);
  if (k <= 0) return Status{NLB_OK};
  if (!cutoffs_valid(cutoffs, k))
    return fail(NLB_ERR_VALUE, multi ? "All cutoffs must be positive and finite"
                                     : "Cutoff must be positive and finite");
  if (n < 0) return fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
  if (n == 0) return empty_results(outs, k);
  if (!pos) return fail(NLB_ERR_VALUE, "positions is NULL");
  const bool pb[3] = {pbc ? pbc[0] != 0 : true, pbc ? pbc[1] != 0 : true,
                      pbc ? pbc[2] != 0 : true};
  SystemPlan sp;
  std::vector<double> cs(cutoffs, cutoffs + k);
  Status st = plan_system(pos, n, cell9, pb, cs, disjoint, multi, sp);
  if (!st.ok()) return st;
  Ctx* c = nullptr;
  st = get_ctx(&c);
  if (!st.ok()) return st;
  double* d_pos = nullptr;
  st = upload_positions(*c, pos, n, &d_pos);
  if (!st.ok()) return st;
  if (fast_eligible(sp)) {
    int64_t m = 0;
    // (host copies: no [src | dst] layout needed; the copies follow the
    // search on the stream, so the call goes on as soon as M is known)
    st = run_fast(*c, sp, d_pos, &m, false, true);
    if (!st.ok()) return st;
    DevLists L;
    L.src.assign(1, sp.out_src);
    L.dst.assign(1, sp.out_dst);
    L.sh.assign(1, sp.out_sh);
    st = download_results(*c, std::vector<int64_t>(1, m), L, sp.order, outs);
    if (!st.ok()) nlb_result_free(&outs[0]);
    return st;
  }
  st = count_system(*c, sp, d_pos);
  if (!st.ok()) return st;
  DevLists L;
  st = device_outputs(*c, sp.m, L);
  if (!st.ok()) return st;
  std::vector<int64_t> zeros(k, 0);
  st = emit_system(*c, sp, d_pos, L, zeros.data(), 0);
  if (!st.ok()) return st;
  st = download_results(*c, sp.m, L, sp.order, outs);
  if (!st.ok()) {
    for (int32_t q = 0; q < k; ++q) nlb_result_free(&outs[q]);
  }
  return st;
}

// One system, one cutoff: the half list on the device ([src | dst] *ei, *sh,
// *m edges), on c.stream.  pos_host (optional) serves the auto-box planner;
// without it the bounds come from the device positions.
Status half_list_device(Ctx& c, const double* pos_host, const double* d_pos, int64_t n,
                        const double* cell9, const uint8_t* pbc, double cutoff, int64_t** ei,
                        int32_t** sh, int64_t* m) {
  double bounds[6];
  const double* bptr = nullptr;
  if (!cell9 && !pos_host) {
    double* d_b = static_cast<double*>(c.raw(kSlotBatch0 + 31, sizeof(double) * 6));
    if (!d_b) return fail(NLB_ERR_NOMEM, "device allocation failed");
    launch_bounds(d_pos, n, d_b, c.stream);
    cudaError_t e = cudaMemcpyAsync(bounds, d_b, sizeof(bounds), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "bounds");
    bptr = bounds;
  }
  const bool pb[3] = {pbc ? pbc[0] != 0 : true, pbc ? pbc[1] != 0 : true,
                      pbc ? pbc[2] != 0 : true};
  SystemPlan sp;
  std::vector<double> cs(1, cutoff);
  Status st = plan_system(pos_host, n, cell9, pb, cs, false, false, sp, bptr);
  if (!st.ok()) return st;
  if (fast_eligible(sp)) {
    st = run_fast(c, sp, d_pos, m);
    if (!st.ok()) return st;
    *ei = sp.out_src;
    *sh = sp.out_sh;
    return Status{NLB_OK};
  }
  st = count_system(c, sp, d_pos);
  if (!st.ok()) return st;
  DevLists L;
  st = device_outputs(c, sp.m, L);
  if (!st.ok()) return st;
  const int64_t zero = 0;
  st = emit_system(c, sp, d_pos, L, &zero, 0);
  if (!st.ok()) return st;
  *m = sp.m[0];
  *ei = L.src[0];
  *sh = L.sh[0];
  return Status{NLB_OK};
}

// Output options applied to a device half list; results in workspace slots
// (or the half list itself when nothing changes it).
Status apply_extras(Ctx& c, const double* d_pos, const double* cell9, int flags, int64_t* ei,
                    int32_t* sh, int64_t m, nlb_result_ex* out) {
  const bool directed = (flags & NLB_DIRECTED) != 0;
  const int64_t mo = directed ? 2 * m : m;
  out->n_edges = mo;
  out->edge_index = ei;
  out->shift = sh;
  out->vectors = nullptr;
  out->distances = nullptr;
  if (directed) {
    out->edge_index = slot<int64_t>(c, kSlotBatch0 + 20, 2 * (size_t)mo);
    out->shift = slot<int32_t>(c, kSlotBatch0 + 21, 3 * (size_t)mo);
    if (!out->edge_index || !out->shift) return fail(NLB_ERR_NOMEM, "device allocation failed");
  }
  if (flags & NLB_VECTORS) {
    out->vectors = slot<double>(c, kSlotBatch0 + 22, 3 * (size_t)mo);
    if (!out->vectors) return fail(NLB_ERR_NOMEM, "device allocation failed");
  }
  if (flags & NLB_DISTANCES) {
    out->distances = slot<double>(c, kSlotBatch0 + 23, (size_t)mo);
    if (!out->distances) return fail(NLB_ERR_NOMEM, "device allocation failed");
  }
  if (!directed && !out->vectors && !out->distances) return Status{NLB_OK};
  EdgeExtrasCell cell{};
  if (cell9) {
    for (int k = 0; k < 9; ++k) cell.h[k] = cell9[k];
    cell.has_cell = 1;
  }
  launch_edge_extras(d_pos, cell, ei, sh, m, directed ? 1 : 0, directed ? out->edge_index : nullptr,
                     directed ? out->shift : nullptr, out->vectors, out->distances, c.stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "edge extras launch");
  return Status{NLB_OK};
}

bool extras_flags_valid(int flags) {
  return (flags & ~(NLB_DIRECTED | NLB_VECTORS | NLB_DISTANCES)) == 0;
}

// nlb_build_ex / nlb_build_device_ex: d_pos_in == nullptr means host
// positions (uploaded here) and pinned host results.
Status run_single_ex(const double* pos, const double* d_pos_in, int64_t n, const double* cell9,
                     const uint8_t* pbc, double cutoff, int flags, nlb_result_ex* out) {
  std::memset(out, 0, sizeof(*out));
  if (!extras_flags_valid(flags)) return fail(NLB_ERR_VALUE, "unknown output option flags");
  if (!cutoffs_valid(&cutoff, 1)) return fail(NLB_ERR_VALUE, "Cutoff must be positive and finite");
  if (n < 0) return fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
  const bool host = d_pos_in == nullptr;
  if (n > 0 && host && !pos) return fail(NLB_ERR_VALUE, "positions is NULL");
  Ctx* c = nullptr;
  Status st = get_ctx(&c);
  if (!st.ok()) return st;
  int64_t* ei = nullptr;
  int32_t* sh = nullptr;
  int64_t m = 0;
  const double* d_pos = d_pos_in;
  if (n > 0) {
    if (host) {
      double* up = nullptr;
      st = upload_positions(*c, pos, n, &up);
      if (!st.ok()) return st;
      d_pos = up;
    }
    st = half_list_device(*c, host ? pos : nullptr, d_pos, n, cell9, pbc, cutoff, &ei, &sh, &m);
    if (!st.ok()) return st;
  }
  nlb_result_ex dev;
  st = apply_extras(*c, d_pos, cell9, flags, ei, sh, m, &dev);
  if (!st.ok()) return st;
  if (!host) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "edge extras");
    if (c->prof) c->harvest();
    *out = dev;
    return Status{NLB_OK};
  }
  // Pinned host results.
  const int64_t mo = dev.n_edges;
  const size_t cnt = (size_t)std::max<int64_t>(mo, 1);
  out->n_edges = mo;
  out->edge_index = static_cast<int64_t*>(pinned_alloc(16 * cnt));
  out->shift = static_cast<int32_t*>(pinned_alloc(12 * cnt));
  if (flags & NLB_VECTORS) out->vectors = static_cast<double*>(pinned_alloc(24 * cnt));
  if (flags & NLB_DISTANCES) out->distances = static_cast<double*>(pinned_alloc(8 * cnt));
  if (!out->edge_index || !out->shift || ((flags & NLB_VECTORS) && !out->vectors) ||
      ((flags & NLB_DISTANCES) && !out->distances)) {
    nlb_result_ex_free(out);
    return fail(NLB_ERR_NOMEM, "pinned host allocation failed");
  }
  cudaError_t e = cudaSuccess;
  if (mo > 0) {
    e = cudaMemcpyAsync(out->edge_index, dev.edge_index, 16 * (size_t)mo, cudaMemcpyDeviceToHost,
                        c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out->shift, dev.shift, 12 * (size_t)mo, cudaMemcpyDeviceToHost,
                          c->stream);
    if (e == cudaSuccess && out->vectors)
      e = cudaMemcpyAsync(out->vectors, dev.vectors, 24 * (size_t)mo, cudaMemcpyDeviceToHost,
                          c->stream);
    if (e == cudaSuccess && out->distances)
      e = cudaMemcpyAsync(out->distances, dev.distances, 8 * (size_t)mo,
                          cudaMemcpyDeviceToHost, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    nlb_result_ex_free(out);
    return cuda_fail(e, "result copy");
  }
  if (c->prof) c->harvest();
  return Status{NLB_OK};
}

// One system, one cutoff, device in / device out (nlb_build_device).
Status run_single_device(const double* d_pos, int64_t n, const double* cell9, const uint8_t* pbc,
                         double cutoff, nlb_device_result* out) {
  out->n_edges = 0;
  out->edge_index = nullptr;
  out->shift = nullptr;
  if (!cutoffs_valid(&cutoff, 1)) return fail(NLB_ERR_VALUE, "Cutoff must be positive and finite");
  if (n < 0) return fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
  if (n == 0) return Status{NLB_OK};
  if (!d_pos) return fail(NLB_ERR_VALUE, "positions is NULL");
  Ctx* c = nullptr;
  Status st = get_ctx(&c);
  if (!st.ok()) return st;
  double bounds[6];
  const double* bptr = nullptr;
  if (!cell9) {
    double* d_b = static_cast<double*>(c->raw(kSlotBatch0 + 31, sizeof(double) * 6));
    if (!d_b) return fail(NLB_ERR_NOMEM, "device allocation failed");
    launch_bounds(d_pos, n, d_b, c->stream);
    cudaError_t e = cudaMemcpyAsync(bounds, d_b, sizeof(bounds), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "bounds");
    bptr = bounds;
  }
  const bool pb[3] = {pbc ? pbc[0] != 0 : true, pbc ? pbc[1] != 0 : true,
                      pbc ? pbc[2] != 0 : true};
  SystemPlan sp;
  std::vector<double> cs(1, cutoff);
  st = plan_system(nullptr, n, cell9, pb, cs, false, false, sp, bptr);
  if (!st.ok()) return st;
  if (fast_eligible(sp)) {
    int64_t m = 0;
    st = run_fast(*c, sp, d_pos, &m);
    if (!st.ok()) return st;
    out->n_edges = m;
    out->edge_index = sp.out_src;
    out->shift = sp.out_sh;
    return Status{NLB_OK};
  }
  st = count_system(*c, sp, d_pos);
  if (!st.ok()) return st;
  DevLists L;
  st = device_outputs(*c, sp.m, L);
  if (!st.ok()) return st;
  const int64_t zero = 0;
  st = emit_system(*c, sp, d_pos, L, &zero, 0);
  if (!st.ok()) return st;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "emit pass");
  if (c->prof) c->harvest();
  out->n_edges = sp.m[0];
  out->edge_index = L.src[0];
  out->shift = L.sh[0];
  return Status{NLB_OK};
}

Status run_single_device(const double* d_pos, int64_t n, const double* cell9, const uint8_t* pbc,
                         double cutoff, nlb_device_result* out, bool owned) {
  Status st = run_single_device(d_pos, n, cell9, pbc, cutoff, out);
  if (!st.ok() || !owned) return st;
  // Hand the arrays (the context's result slots) over to the caller.
  if (out->n_edges == 0) {
    out->edge_index = nullptr;
    out->shift = nullptr;
    return st;
  }
  Ctx* c = nullptr;
  st = get_ctx(&c);
  if (!st.ok()) return st;
  int64_t* ei = nullptr;
  int32_t* sh = nullptr;
  if (out->edge_index != c->bufs[kSlotOutEi].p || out->shift != c->bufs[kSlotOutSh].p)
    return fail(NLB_ERR_CUDA, "device result is not in the context's result arrays");
  take_result_arrays(*c, &ei, &sh);
  out->edge_index = ei;
  out->shift = sh;
  return st;
}

}  // namespace nlb

// ------------------------------------------------------------------ C ABI

using namespace nlb;

extern "C" {

const char* nlb_last_error(void) { return g_last_error.c_str(); }

const char* nlb_version(void) { return "neighborlist-b200 0.1.0 (sm_100a)"; }

int nlb_build(const double* positions, int64_t n_atoms, double cutoff, const double* cell,
              const uint8_t* pbc, int /*parallel*/, nlb_result* out) {
  if (!out) return fail(NLB_ERR_VALUE, "out is NULL").code;
  return run_single(positions, n_atoms, cell, pbc, &cutoff, 1, false, false, out).code;
}

int nlb_build_multi(const double* positions, int64_t n_atoms, const double* cutoffs,
                    int32_t n_cutoffs, const double* cell, const uint8_t* pbc, int disjoint,
                    nlb_result* outs) {
  if (n_cutoffs > 0 && (!outs || !cutoffs)) return fail(NLB_ERR_VALUE, "outs is NULL").code;
  return run_single(positions, n_atoms, cell, pbc, cutoffs, n_cutoffs, disjoint != 0, true, outs)
      .code;
}

int nlb_build_batch(const double* positions, int64_t n_atoms, const int32_t* batch,
                    int64_t n_batch, double cutoff, const double* cells, const uint8_t* pbcs,
                    const uint8_t* has_cell, int64_t n_cells, int /*parallel*/, nlb_result* out) {
  if (!out) return fail(NLB_ERR_VALUE, "out is NULL").code;
  return run_batch(positions, n_atoms, batch, n_batch, &cutoff, 1, cells, pbcs, has_cell, n_cells,
                   false, false, out)
      .code;
}

int nlb_build_batch_multi(const double* positions, int64_t n_atoms, const int32_t* batch,
                          int64_t n_batch, const double* cutoffs, int32_t n_cutoffs,
                          const double* cells, const uint8_t* pbcs, const uint8_t* has_cell,
                          int64_t n_cells, int disjoint, nlb_result* outs) {
  if (n_cutoffs > 0 && (!outs || !cutoffs)) return fail(NLB_ERR_VALUE, "outs is NULL").code;
  return run_batch(positions, n_atoms, batch, n_batch, cutoffs, n_cutoffs, cells, pbcs, has_cell,
                   n_cells, disjoint != 0, true, outs)
      .code;
}

int nlb_build_batch_ex(const double* positions, int64_t n_atoms, const int32_t* batch,
                       int64_t n_batch, const double* cutoffs, int32_t n_cutoffs,
                       const double* cells, const uint8_t* pbcs, const uint8_t* has_cell,
                       int64_t n_cells, int disjoint, int multi, nlb_result* outs,
                       int64_t* system_offsets) {
  if (n_cutoffs > 0 && (!outs || !cutoffs)) return fail(NLB_ERR_VALUE, "outs is NULL").code;
  return run_batch(positions, n_atoms, batch, n_batch, cutoffs, n_cutoffs, cells, pbcs, has_cell,
                   n_cells, disjoint != 0, multi != 0, outs, system_offsets)
      .code;
}

int nlb_build_ex(const double* positions, int64_t n_atoms, double cutoff, const double* cell,
                 const uint8_t* pbc, int flags, nlb_result_ex* out) {
  if (!out) return fail(NLB_ERR_VALUE, "out is NULL").code;
  return run_single_ex(positions, nullptr, n_atoms, cell, pbc, cutoff, flags, out).code;
}

int nlb_build_device_ex(const double* d_positions, int64_t n_atoms, double cutoff,
                        const double* cell, const uint8_t* pbc, int flags, nlb_result_ex* out) {
  if (!out) return fail(NLB_ERR_VALUE, "out is NULL").code;
  if (!d_positions && n_atoms > 0) {
    std::memset(out, 0, sizeof(*out));
    return fail(NLB_ERR_VALUE, "positions is NULL").code;
  }
  // A non-null placeholder selects the device-result path for empty input.
  static const double kNone = 0.0;
  return run_single_ex(nullptr, d_positions ? d_positions : &kNone, n_atoms, cell, pbc, cutoff,
                       flags, out)
      .code;
}

void nlb_result_ex_free(nlb_result_ex* r) {
  if (!r) return;
  pinned_release(r->edge_index);
  pinned_release(r->shift);
  pinned_release(r->vectors);
  pinned_release(r->distances);
  std::memset(r, 0, sizeof(*r));
}

void nlb_result_free(nlb_result* r) {
  if (!r) return;
  pinned_release(r->edge_index);
  pinned_release(r->shift);
  r->edge_index = nullptr;
  r->shift = nullptr;
  r->n_edges = 0;
}

void nlb_host_free(void* p) { pinned_release(p); }

void nlb_pinned_stats(int64_t* out) {
  if (out) pinned_stats(out);
}

int nlb_build_device(const double* d_positions, int64_t n_atoms, double cutoff,
                     const double* cell, const uint8_t* pbc, nlb_device_result* out) {
  if (!out) return fail(NLB_ERR_VALUE, "out is NULL").code;
  return run_single_device(d_positions, n_atoms, cell, pbc, cutoff, out).code;
}

int nlb_build_device_owned(const double* d_positions, int64_t n_atoms, double cutoff,
                           const double* cell, const uint8_t* pbc, nlb_device_result* out) {
  if (!out) return fail(NLB_ERR_VALUE, "out is NULL").code;
  return run_single_device(d_positions, n_atoms, cell, pbc, cutoff, out, true).code;
}

int nlb_device_free(void* p, void* stream) {
  if (!p) return NLB_OK;
  ResultPool& rp = result_pool();
  int dev = 0;
  {
    std::lock_guard<std::mutex> lk(rp.mu);
    auto it = rp.owned.find(p);
    if (it == rp.owned.end())
      return fail(NLB_ERR_VALUE, "nlb_device_free: not a block from nlb_build_device_owned").code;
    dev = it->second.first;
    rp.owned.erase(it);
    ++rp.returned;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != dev) cudaSetDevice(dev);
  cudaError_t e = cudaFreeAsync(p, static_cast<cudaStream_t>(stream));
  if (prev != dev) cudaSetDevice(prev);
  if (e != cudaSuccess) return cuda_fail(e, "nlb_device_free").code;
  return NLB_OK;
}

void nlb_device_blocks(int64_t* out3) {
  ResultPool& rp = result_pool();
  std::lock_guard<std::mutex> lk(rp.mu);
  int64_t bytes = 0;
  for (auto& kv : rp.owned) bytes += (int64_t)kv.second.second;
  out3[0] = rp.handed;
  out3[1] = rp.returned;
  out3[2] = bytes;
}

int nlb_copy_device(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return NLB_OK;
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice,
                                  static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "nlb_copy_device").code;
  return NLB_OK;
}

void nlb_set_stream(void* stream) { tl_user_stream = static_cast<cudaStream_t>(stream); }

int64_t nlb_kernel_launches(void) { return g_launches.load(); }

int64_t nlb_graph_replays(void) { return g_graph_replays.load(); }

int32_t nlb_last_single_pipeline(void) { return last_single_pipeline(); }

int32_t nlb_single_pipeline(int32_t mode) {
  if (mode < 0) return single_pipeline_mode();
  if (mode > 1) return -1;
  return set_single_pipeline_mode(mode);
}

int nlb_debug_scan_stall(int32_t tile, int32_t spin_limit) {
  if (tile < 0 || spin_limit < 1)
    return fail(NLB_ERR_VALUE, "nlb_debug_scan_stall: tile must be >= 0 and spin_limit >= 1")
        .code;
  arm_scan_stall(tile, spin_limit);
  return NLB_OK;
}

void nlb_profile(int enable) {
  tl_profile = enable != 0;
  Ctx* c = nullptr;
  if (get_ctx(&c).ok()) {
    c->prof_ms[0] = c->prof_ms[1] = c->prof_ms[2] = c->prof_ms[3] = 0.0;
    for (double& v : c->prof_host_ms) v = 0.0;
    c->prof_calls = 0;
    c->prof_pending_count = c->prof_pending_emit = false;
  }
}

int64_t nlb_profile_host(double* ms) {
  Ctx* c = nullptr;
  if (!get_ctx(&c).ok()) return -1;
  if (ms)
    for (int i = 0; i < 4; ++i) ms[i] = c->prof_host_ms[i];
  return c->prof_calls;
}

int64_t nlb_profile_read(double* ms) {
  Ctx* c = nullptr;
  if (!get_ctx(&c).ok()) return -1;
  if (ms)
    for (int i = 0; i < 4; ++i) ms[i] = c->prof_ms[i];
  return c->prof_calls;
}

int nlb_cell_check(const double* cell) {
  if (!cell) return fail(NLB_ERR_VALUE, "cell is NULL").code;
  HostCell c;
  std::string err;
  const bool pb[3] = {true, true, true};
  if (!make_cell(cell, pb, c, err)) return fail(NLB_ERR_VALUE, err).code;
  return NLB_OK;
}

void nlb_batch_cells(const double* ase_cells, int64_t n_cells, double* h9_out, uint8_t* has_out) {
  for (int64_t i = 0; i < n_cells; ++i) {
    const double* r = ase_cells + 9 * i;
    double* h = h9_out + 9 * i;
    bool any = false;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        h[3 * a + b] = r[3 * b + a];
        any = any || r[3 * b + a] != 0.0;
      }
    has_out[i] = any ? 1 : 0;
  }
}

int nlb_cell_wrap(const double* cell, const uint8_t* pbc, const double* p, double* out) {
  if (!cell || !p || !out) return fail(NLB_ERR_VALUE, "NULL argument").code;
  HostCell c;
  std::string err;
  const bool pb[3] = {pbc ? pbc[0] != 0 : true, pbc ? pbc[1] != 0 : true,
                      pbc ? pbc[2] != 0 : true};
  if (!make_cell(cell, pb, c, err)) return fail(NLB_ERR_VALUE, err).code;
  double f[3];
  for (int r = 0; r < 3; ++r) {
    const double t = c.hinv[3 * r] * p[0] + c.hinv[3 * r + 1] * p[1];
    f[r] = t + c.hinv[3 * r + 2] * p[2];
  }
  for (int a = 0; a < 3; ++a)
    if (pb[a]) f[a] = f[a] - std::floor(f[a]);
  for (int r = 0; r < 3; ++r) {
    const double t = c.h[3 * r] * f[0] + c.h[3 * r + 1] * f[1];
    out[r] = t + c.h[3 * r + 2] * f[2];
  }
  return NLB_OK;
}

size_t nlb_get_brute_force_threshold(void) { return (size_t)g_bf_threshold.load(); }
void nlb_set_brute_force_threshold(size_t v) { g_bf_threshold.store(v); }
size_t nlb_get_parallel_threshold(void) { return (size_t)g_par_threshold.load(); }
void nlb_set_parallel_threshold(size_t v) { g_par_threshold.store(v); }
size_t nlb_get_stack_threshold(void) { return (size_t)g_stack_threshold.load(); }
void nlb_set_stack_threshold(size_t v) { g_stack_threshold.store(std::min<size_t>(v, 1024)); }

}  // extern "C"
