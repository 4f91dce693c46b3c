// nlb_internal.h -- host-side internals shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/neighborlist_b200.h"
#include "nlb_geometry.h"
#include "nlb_kernels.h"

namespace nlb {

struct Status {
  int code;
  bool ok() const { return code == NLB_OK; }
};

Status fail(int code, const std::string& msg);
Status cuda_fail(cudaError_t e, const char* what);

extern thread_local std::string g_last_error;

// Device workspace slots (grow-only buffers, one set per host thread and device).
enum Slot : int {
  kSlotPos = 0,
  kSlotRankTab,
  kSlotBinCount,
  kSlotBinFill,
  kSlotBinStart,
  kSlotKey,
  kSlotRank,
  kSlotSkey,
  kSlotSidx,
  kSlotSkey2,
  kSlotSidx2,
  kSlotPx,
  kSlotPy,
  kSlotPz,
  kSlotMeta,
  kSlotScanTmp,
  kSlotCounts,
  kSlotOffs,
  kSlotOutEi,
  kSlotOutSh,
  kSlotP32,
  kSlotSbin,
  kSlotGroups,
  kSlotIrrList,
  kSlotIrr,
  kSlotCounters,
  kSlotTaskHdr,
  kSlotMasks,
  kSlotCbox,
  kSlotGroupStart,
  kSlotOutDst,
  kSlotFill,
  kSlotBatch0,  // first slot owned by the batched path
  kSlotCount = kSlotBatch0 + 32,
};

constexpr int kSmallHost = 4096;  // int64 slots of the per-context pinned scratch

// Kind of batch the launch-shape tuner keys on: cutoff count (0: one cutoff
// per system), and power-of-two buckets of the system count, the largest and
// the mean system, and a quarter-octave bucket of the largest cutoff.
struct TuneKey {
  int32_t device, k, n_sys_log2, max_log2, mean_log2, rc_bucket;
  bool operator<(const TuneKey& o) const;
};
TuneKey make_tune_key(int32_t device, int32_t k, const int64_t* sizes, int32_t n_sys,
                      double rc_max);

struct Ctx {
  struct Buf {
    void* p = nullptr;
    size_t cap = 0;
    bool pooled = false;  // from the result pool (stream-ordered), not cudaMalloc
  };
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;  // active stream: the caller's (nlb_set_stream) or own_stream
  int64_t* h_small = nullptr;     // pinned scratch for small device->host reads
  // Host-mapped pinned record a kernel fills when the edge count is known:
  // [0] ready (1), [1] M, [2] error word (h_report: host view, d_report:
  // device view).
  int64_t* h_report = nullptr;
  int64_t* d_report = nullptr;
  // A call on a caller's stream may return before its last kernels end (the
  // results are complete in that stream's order).  early_ev marks the end of
  // that work; a later call on another stream waits for it on the device.
  cudaEvent_t early_ev = nullptr;
  cudaStream_t early_stream = nullptr;
  Buf bufs[kSlotCount];
  // Batched outputs: [src, dst, shift] per cutoff, grow-only and kept across
  // calls (results are appended run by run, so growth preserves contents).
  std::vector<Buf> batch_out;
  // Phase timing (nlb_profile): events ev[0..3] bracket build / count / scan,
  // ev[4..5] the emit pass; harvested after the stream is synchronized.
  bool prof = false;
  bool prof_pending_count = false;
  bool prof_pending_emit = false;
  cudaEvent_t ev[6] = {};
  double prof_ms[4] = {0, 0, 0, 0};
  // Host wall time of batched builds while profiling (ms, accumulated):
  // input upload, issue-to-sync of the device work, result copies, whole call.
  double prof_host_ms[4] = {0, 0, 0, 0};
  // Bins per axis of the rank table currently in kSlotRankTab (-1: none).
  int32_t rank_nb[3] = {-1, -1, -1};
  // Hit-mask words the last multi-cutoff pair-task count pass needed.
  int64_t pair_mask_words = 0;
  // Events timing the candidate launch shapes of a new kind of batch
  // (nlb_tune.cpp), created on first use.
  cudaEvent_t tune_ev[kBatchShapes + 1] = {};
  int64_t prof_calls = 0;
  void mark(int i) {
    if (prof) cudaEventRecord(ev[i], stream);
  }
  void harvest();
  // Returns a device buffer of at least `bytes` for `slot` (contents are not
  // preserved on growth), or nullptr if the allocation failed.
  void* raw(int slot, size_t bytes);
};

Status get_ctx(Ctx** out);
// Hands the context's single-system result arrays (slots kSlotOutEi and
// kSlotOutSh, allocated from the per-device result pool) over to the caller:
// the context forgets them and its next build allocates fresh ones from the
// pool.  The caller returns each with nlb_device_free.
void take_result_arrays(Ctx& c, int64_t** ei, int32_t** sh);
// Frees the calling thread's contexts and fast-path graphs (threads that end
// before the process does, e.g. server workers).
void release_thread_ctx();
// A device block of the per-device stream-ordered result pool, allocated on
// stream s and registered as handed to a caller (nlb_device_free returns
// it); nullptr on failure.  release_owned_device takes one back that was
// never handed over after all.
void* alloc_owned_device(int device, size_t bytes, cudaStream_t s);
// Maps `bytes` of the device's stream-ordered pool (the one every workspace
// slot and result array comes from) now and leaves them free in it: later
// growth of a thread's workspace takes them without mapping device memory on
// its critical path.  The pool keeps them mapped (release threshold:
// unlimited).
void warm_result_pool(int device, size_t bytes, cudaStream_t s);
void release_owned_device(void* p, cudaStream_t s);
void release_fast_states();
void release_batch_graphs();
// Counts CUDA-graph replays of the fast paths (nlb_graph_replays).
void note_graph_replay();
bool fp32_search_enabled();

template <class T>
inline T* slot(Ctx& c, int s, size_t count) {
  return static_cast<T*>(c.raw(s, sizeof(T) * (count > 0 ? count : 1)));
}

void* pinned_alloc(size_t bytes);
void pinned_release(void* p);
// Registers `slice` (a pointer into pool block `block`, distinct from every
// other live slice) as a handle of its own: pinned_release(slice) drops it,
// and the block returns to the pool when its last slice is released.  The
// block itself must then not be released directly.
void pinned_share(void* block, void* slice);
void pinned_stats(int64_t* out);
void pinned_reserve(size_t bytes);

// One system after planning: cell, dispatch decision, grid or brute-force
// parameters, cutoffs in ascending order, and (after count_system) the
// per-cutoff edge totals and per-atom offsets on the device.
struct SystemPlan {
  int64_t n = 0;
  HostCell cell;
  Method method = Method::kCellList;
  GridParams grid{};
  BruteParams brute{};
  GridBuffers gb{};
  bool disjoint = false;
  std::vector<int32_t> order;   // sorted position q -> input cutoff index
  std::vector<double> rc_sq;    // ascending squared cutoffs
  std::vector<int64_t> m;       // edges per sorted cutoff (after count)
  bool fp32 = false;            // cell list, <= kFp32MaxCutoffs: FP32 guard-band kernels
  GuardBand band{};             // the first (or only) cutoff's band
  PairBands pbands{};           // every sorted cutoff's band (one traversal)
  uint32_t* counts = nullptr;
  int64_t* offs = nullptr;
  int64_t row = 0;              // length of one cutoff's count row
  bool rank_cached = false;     // fast path: rank table reusable
  int64_t* scan_state = nullptr;  // fast path: offsets-scan state (in the zeroed block)
  size_t zeroed_words = 0;        // fast path: int32 words cleared at the start of a run
  int64_t* out_src = nullptr;   // fast path: [src | dst] arena
  int32_t* out_sh = nullptr;    // fast path: shift arena
  int64_t* out_dst = nullptr;   // fast path: where the M destinations are after run_fast
  bool fused = false;           // fast path: one-launch count + offsets + emit (k_fused.cu)
  uint64_t* fused_state = nullptr;  // its ticket / error / look-back words (in the zeroed block)
  int64_t* fused_total = nullptr;   // its edge total (in the zeroed block)
  int64_t fused_words = 0;          // 64-bit words of fused_state + total
  CutoffSet pass(int32_t g0) const;
};

// Device destinations of k edge lists (sorted cutoff order).
struct DevLists {
  std::vector<int64_t*> src, dst;
  std::vector<int32_t*> sh;
};

// bounds6 (optional): per-axis min[3], max[3] of the positions for the
// auto-box when the positions are not on the host.
Status plan_system(const double* pos_host, int64_t n, const double* cell9, const bool pbc[3],
                   const std::vector<double>& cutoffs, bool disjoint, bool multi,
                   SystemPlan& sp, const double* bounds6 = nullptr);
Status count_system(Ctx& c, SystemPlan& sp, const double* d_pos);
Status emit_system(Ctx& c, SystemPlan& sp, const double* d_pos, const DevLists& L,
                   const int64_t* base, int64_t index_offset);

// Single-cutoff cell-list pipeline with no host round trip before M is
// known (the device reports M through host-mapped memory), replayed as a
// CUDA graph for repeated identical calls (nlb_fast.cpp).  Requires
// sp.method == kCellList and sp.fp32; leaves the M edges in sp.out_src
// (sources), sp.out_dst (destinations) and sp.out_sh.  contiguous = true
// puts the destinations right behind the sources (sp.out_dst = out_src + M,
// the [src | dst] layout); otherwise they may stay in a separate array.
// stream_ordered = true: the caller only queues further work on c.stream
// (e.g. the result copies) and synchronises it itself, so the call returns
// as soon as M is known even on the library's own stream.
Status run_fast(Ctx& c, SystemPlan& sp, const double* d_pos, int64_t* m_out,
                bool contiguous = true, bool stream_ordered = false);
// Single-system pipeline choice: 0 = automatic (the one-launch kernel on
// sparse grids), 1 = always the three-launch pair-task pipeline.
int32_t single_pipeline_mode();
int32_t set_single_pipeline_mode(int32_t mode);  // returns the previous mode
// Pipeline of the calling thread's last single-cutoff cell-list build:
// 0 = one launch, 1 = three launches, -1 = none yet.
int32_t last_single_pipeline();
inline bool fast_eligible(const SystemPlan& sp) {
  return sp.method == Method::kCellList && sp.fp32 && sp.rc_sq.size() == 1;
}

Status alloc_result(int64_t m, nlb_result* r);
void zero_results(nlb_result* outs, int32_t k);
Status empty_results(nlb_result* outs, int32_t k);
bool cutoffs_valid(const double* cs, int32_t k);
Status upload_positions(Ctx& c, const double* pos, int64_t n, double** d_pos);

// ---- launch-shape tuner for the batched kernels (nlb_tune.cpp)
// The work items of one batched run in every launch shape it tries: the
// chosen (or pinned) shape of its kind, or, for the first batch of a new
// kind, every candidate shape.  Usage: prepare() before the count pass; for
// each i < w.size(), mark(i) then that shape's count launches; mark(w.size());
// after the host has synchronised on the count pass, pick() returns the
// items for the emit pass (the fastest count, remembered for the kind).
struct ShapeTrials {
  TuneKey key{};
  std::vector<int32_t> shapes;
  std::vector<BatchItems> w;
  bool timed = false;
  Status prepare(Ctx& c, const TuneKey& k, const int64_t* sizes, int32_t n_sys, int items_slot);
  void mark(Ctx& c, size_t i);
  const BatchItems& pick(Ctx& c);
};
void tune_release(Ctx& c);

// sys_offsets (optional): k x (n_systems + 1) int64, row = input cutoff
// index; system i's edges of that list are [row[i], row[i + 1]).
Status run_batch(const double* pos, int64_t n, const int32_t* batch, int64_t n_batch,
                 const double* cutoffs, int32_t k, const double* cells, const uint8_t* pbcs,
                 const uint8_t* has_cell, int64_t n_cells, bool disjoint, bool multi,
                 nlb_result* outs, int64_t* sys_offsets = nullptr);

}  // namespace nlb
