// nlb_fast.cpp -- single-system, single-cutoff cell-list builds without a
// host round trip in the middle, replayed as a CUDA graph.
//
// The pipeline (bin histogram memset, atom prep, bin scan, scatter, per-bin
// sort + gather, pair-task count, offset scan, pair-task emit) is issued
// back to back on the caller's stream.  The emit pass reads the edge total
// from device memory and writes into a capacity-bounded arena (the previous
// total x 1.25, or a density estimate); the host synchronises once at the
// end, and only if the arena was too small does it grow it and run the emit
// pass again (the counts and offsets are still in place).
//
// On sparse grids (at most 64 atoms per bin on average, at most 125 stencil
// cells) the count, offsets scan and emit are one launch instead
// (k_fused.cu): the build stores the groups in canonical order, one CTA per
// group counts, finds its output offset by a look-back over the groups
// before it and writes its block; the edge total again comes from device
// memory, and an arena that was too small makes the host grow it and run the
// fused launch again.
//
// The first call with a given set of launch parameters runs the work
// directly; a repeated call with identical parameters (same positions
// buffer, cell, cutoff, sizes and workspace) captures the sequence into a
// CUDA graph and replays it from then on.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include "nlb_internal.h"

namespace nlb {

namespace {

// Everything the issued work depends on; compared bytewise.
struct FastKey {
  const double* d_pos;
  int64_t n;
  GridParams grid;
  GuardBand band;
  cudaStream_t stream;
  void* bufs[kSlotCount];
  int64_t capacity;
  int64_t mask_cap;
  int32_t need_rank;
  int32_t prof;
  int32_t fused;
  int32_t contiguous;
};

struct FastState {
  FastKey key;
  bool have_key = false;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;  // kernels per replay
  int64_t last_m = 0;
  int64_t last_mask_words = 0;
};

thread_local FastState tl_states[16];

FastState& state_for(Ctx& c) { return tl_states[c.device & 15]; }

int64_t stencil_cells_of(const GridParams& g) {
  return (int64_t)(2 * g.ns[0] + 1) * (2 * g.ns[1] + 1) * (2 * g.ns[2] + 1);
}

// Expected edges for sizing the first arena: half the pairs within rc at the
// system's mean density, plus one list entry per atom of slack.
int64_t estimate_edges(const SystemPlan& sp, double rc) {
  const double* h = sp.cell.h;
  const double det = h[0] * (h[4] * h[8] - h[7] * h[5]) - h[1] * (h[3] * h[8] - h[6] * h[5]) +
                     h[2] * (h[3] * h[7] - h[6] * h[4]);
  const double vol = std::fabs(det);
  const double rho = vol > 0 ? (double)sp.n / vol : 0.0;
  const double per_atom = 0.5 * rho * (4.0 / 3.0) * 3.141592653589793 * rc * rc * rc;
  const double est = (double)sp.n * (per_atom + 1.0);
  return (int64_t)std::min(est, 4.0e12);
}

std::atomic<int32_t> g_pipeline_mode{0};

}  // namespace

namespace {
thread_local int32_t tl_last_fused = -1;  // pipeline of this thread's last fast-path build
}  // namespace

int32_t single_pipeline_mode() { return g_pipeline_mode.load(); }
int32_t last_single_pipeline() { return tl_last_fused; }
int32_t set_single_pipeline_mode(int32_t mode) { return g_pipeline_mode.exchange(mode); }

void release_fast_states() {
  for (FastState& fs : tl_states) {
    if (fs.exec) cudaGraphExecDestroy(fs.exec);
    fs = FastState();
  }
}

// Sizes every workspace buffer of the fast pipeline (may allocate; never
// inside a capture).
Status prepare_fast(Ctx& c, SystemPlan& sp, int64_t capacity, int64_t mask_cap) {
  const int64_t n = sp.n;
  const int64_t nb = sp.grid.total_bins;
  const int64_t cells = stencil_cells_of(sp.grid);
  const int64_t row = n * cells + 1;
  sp.row = row;
  GridBuffers& b = sp.gb;
  const void* tab_before = c.bufs[kSlotRankTab].p;
  const size_t tab_cap = c.bufs[kSlotRankTab].cap;
  b.rank_of_bin = slot<int32_t>(c, kSlotRankTab, nb);
  sp.rank_cached = b.rank_of_bin == tab_before && tab_cap > 0 && c.rank_nb[0] == sp.grid.nb[0] &&
                   c.rank_nb[1] == sp.grid.nb[1] && c.rank_nb[2] == sp.grid.nb[2];
  // Zeroed block: bin histogram, scatter cursors, 2 task counters, 64-bit
  // mask cursor (8-byte aligned: 2 nb + 2 is even), build completion count,
  // emit task counter, then the offsets scan's state (8-byte aligned at
  // 2 nb + 6), so a single
  // memset at the start clears everything and the kernels follow each other
  // directly.
  // (Fused launch: its ticket, error and look-back words and its total take
  // the scan state's place.)
  const int64_t max_groups = n / 32 + std::min<int64_t>(n, nb) + 1;
  sp.fused_words = 2 + max_groups + 2;  // + total, completion count
  sp.zeroed_words = 2 * (size_t)nb + 6 +
                    2 * (size_t)(sp.fused ? sp.fused_words : scan_tmp_elems(row));
  int32_t* zeroed = slot<int32_t>(c, kSlotBinCount, sp.zeroed_words);
  sp.scan_state = zeroed ? reinterpret_cast<int64_t*>(zeroed + 2 * nb + 6) : nullptr;
  sp.fused_state = reinterpret_cast<uint64_t*>(sp.scan_state);
  sp.fused_total = sp.fused && zeroed ? sp.scan_state + 2 + max_groups : nullptr;
  b.group_start = sp.fused ? slot<int32_t>(c, kSlotGroupStart, nb) : nullptr;
  b.fill = slot<int32_t>(c, kSlotFill, n);
  b.bin_count = zeroed;
  b.bin_fill = zeroed ? zeroed + nb : nullptr;
  b.counters = zeroed ? zeroed + 2 * nb : nullptr;
  b.mask_top = zeroed ? reinterpret_cast<unsigned long long*>(zeroed + 2 * nb + 2) : nullptr;
  b.build_done = zeroed ? zeroed + 2 * nb + 4 : nullptr;
  b.emit_queue = zeroed ? reinterpret_cast<uint32_t*>(zeroed + 2 * nb + 5) : nullptr;
  const int64_t max_tasks = (n / 32 + std::min<int64_t>(n, nb) + 1) * cells;
  // (The fused launch needs no task headers, masks, counts or offsets.)
  b.task_hdr = slot<int4>(c, kSlotTaskHdr, sp.fused ? 1 : max_tasks);
  b.masks = slot<uint32_t>(c, kSlotMasks, sp.fused ? 1 : mask_cap);
  const bool chunk_boxes = nb > 0 && (double)n / (double)nb >= kChunkPruneMinPerBin;
  b.cbox = chunk_boxes ? slot<float4>(c, kSlotCbox, 2 * (size_t)n) : nullptr;
  b.mask_cap = sp.fused ? 0 : mask_cap;
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
  b.p32 = slot<float4>(c, kSlotP32, n);
  b.sbin = slot<int32_t>(c, kSlotSbin, n);
  b.groups = slot<GroupRec>(c, kSlotGroups, n / 32 + std::min<int64_t>(n, nb) + 1);
  b.irr_list = slot<int32_t>(c, kSlotIrrList, n);
  b.irr = slot<uint8_t>(c, kSlotIrr, n);
  b.scan_tmp = slot<int64_t>(c, kSlotScanTmp, scan_tmp_elems(std::max<int64_t>(row, nb)));
  sp.counts = slot<uint32_t>(c, kSlotCounts, sp.fused ? 1 : row);
  sp.offs = slot<int64_t>(c, kSlotOffs, sp.fused ? 1 : row + 1);
  sp.out_src = slot<int64_t>(c, kSlotOutEi, 2 * (size_t)capacity);
  sp.out_sh = slot<int32_t>(c, kSlotOutSh, 3 * (size_t)capacity);
  int64_t* dst_arena = sp.fused ? slot<int64_t>(c, kSlotOutDst, (size_t)capacity) : nullptr;
  if (sp.fused && (!dst_arena || !b.group_start))
    return fail(NLB_ERR_NOMEM, "device allocation failed");
  if (!b.rank_of_bin || !zeroed || !b.bin_start || !b.key || !b.rank || !b.skey || !b.sidx ||
      !b.skey2 || !b.sidx2 || !b.px || !b.py || !b.pz || !b.meta || !b.p32 || !b.sbin ||
      !b.groups || !b.irr_list || !b.irr || !b.scan_tmp || !sp.counts || !sp.offs ||
      !sp.out_src || !sp.out_sh || !b.task_hdr || !b.masks || (chunk_boxes && !b.cbox) ||
      !b.fill)
    return fail(NLB_ERR_NOMEM, "device allocation failed");
  return Status{NLB_OK};
}

FusedOut fused_targets(Ctx& c, const SystemPlan& sp, int64_t capacity) {
  FusedOut o;
  std::memset(&o, 0, sizeof(o));
  o.src = sp.out_src;
  o.dst = static_cast<int64_t*>(c.bufs[kSlotOutDst].p);
  o.sh = sp.out_sh;
  o.capacity = capacity;
  o.state = sp.fused_state;
  o.total = sp.fused_total;
  o.done = reinterpret_cast<unsigned long long*>(sp.fused_total + 1);
  o.report = c.prof ? nullptr : c.d_report;
  o.spin_limit = kFusedSpinLimit;
  o.withhold = -1;
  {
    const double per_bin = (double)sp.n / (double)std::max<int64_t>(sp.grid.total_bins, 1);
    const int64_t chunks = (int64_t)std::ceil(1.5 * per_bin / 32.0);
    const int64_t want = stencil_cells_of(sp.grid) * std::max<int64_t>(chunks, 1) * 32;
    o.mask_words = (int32_t)std::min<int64_t>(std::max<int64_t>(want, kFusedMaskMin), kFusedMaskMax);
  }
  int32_t tile = 0, spins = 0;
  if (take_scan_stall(&tile, &spins)) {  // failure-detection hook
    o.withhold = tile;
    o.spin_limit = spins;
  }
  return o;
}

// The fused launch (and the move of the destinations behind the sources).
void issue_fused(Ctx& c, SystemPlan& sp, int64_t capacity, bool contiguous) {
  FusedOut o = fused_targets(c, sp, capacity);
  o.move = contiguous ? 1 : 0;
  launch_pair_fused(sp.grid, sp.gb, (int32_t)stencil_cells_of(sp.grid), sp.band, o, c.stream);
}

EmitTargets fast_targets(const SystemPlan& sp, int64_t capacity, int64_t* report = nullptr) {
  EmitTargets t;
  std::memset(&t, 0, sizeof(t));
  t.src[0] = sp.out_src;
  t.sh[0] = sp.out_sh;
  t.total_dev = sp.offs + sp.row;
  t.capacity = capacity;
  t.scan_error = sp.scan_state + 1;
  t.report = report;
  t.mask_top = sp.gb.mask_top;
  // (grids too large for k_prep's own bin scan: the separate scan's error word)
  t.grid_scan_error = sp.grid.total_bins > kFusedBinScanMax ? sp.gb.scan_tmp + 1 : nullptr;
  return t;
}

// Issues the whole pipeline on c.stream (no host synchronisation).
void issue_fast(Ctx& c, SystemPlan& sp, const double* d_pos, int64_t capacity,
                bool contiguous) {
  cudaStream_t s = c.stream;
  const int64_t n = sp.n;
  c.mark(0);
  cudaMemsetAsync(sp.gb.bin_count, 0, sizeof(int32_t) * sp.zeroed_words, s);
  launch_grid_build(sp.grid, d_pos, n, sp.gb, s, !sp.rank_cached);
  c.mark(1);
  if (sp.fused) {
    // (Phases: counting and offsets are part of the one launch, timed with
    // the emit.)
    c.mark(2);
    c.mark(3);
    c.mark(4);
    issue_fused(c, sp, capacity, contiguous);
    c.mark(5);
    return;
  }
  launch_pair_count(sp.grid, sp.gb, n, sp.band, sp.counts, s);
  c.mark(2);
  exclusive_scan_u32_zeroed(sp.counts, sp.row, sp.offs, sp.scan_state, s);
  c.mark(3);
  c.mark(4);
  launch_pair_emit(sp.grid, sp.gb, n, sp.band, sp.offs,
                   fast_targets(sp, capacity, c.prof ? nullptr : c.d_report), s);
  c.mark(5);
}

// Waits until the launch just issued has filled the host-mapped report
// (c.h_report[0] = 1), polling the stream now and then: a stream that failed,
// or ended without a report, ends the wait with an error.
Status wait_report(Ctx& c) {
  volatile int64_t* r = c.h_report;
  for (uint32_t k = 1; r[0] == 0; ++k) {
    if ((k & 127) != 0) continue;
    const cudaError_t q = cudaStreamQuery(c.stream);
    if (q == cudaErrorNotReady) continue;
    if (q != cudaSuccess) return cuda_fail(q, "neighbour-list pipeline");
    if (r[0] == 0) {
      // (a launch that failed to start leaves its error with the runtime)
      const cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) return cuda_fail(le, "neighbour-list pipeline launch");
      return fail(NLB_ERR_CUDA, "the search ended without its report");
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return Status{NLB_OK};
}

// Runs the fast pipeline for a planned single-cutoff cell-list system and
// leaves M edges in sp.out_src ([src | dst]) / sp.out_sh.
//
// M reaches the host through host-mapped memory as soon as it is known: the
// one-launch search reports it when its last group is done, the three-launch
// pipeline when its emit pass starts.  On a caller's stream the call then
// returns at once: the remaining work (the emit, or the move of the
// destinations) is queued on that stream ahead of anything the caller queues
// there.  On the library's own stream it also waits for that work.
Status run_fast(Ctx& c, SystemPlan& sp, const double* d_pos, int64_t* m_out, bool contiguous,
                bool stream_ordered) {
  FastState& fs = state_for(c);
  const int64_t n_cells = stencil_cells_of(sp.grid);
  sp.fused = single_pipeline_mode() == 0 && n_cells <= kFusedMaxCells &&
             sp.grid.total_bins > 0 && sp.grid.total_bins <= kFusedBinScanMax &&
             (double)sp.n / (double)sp.grid.total_bins <= kFusedMaxPerBin;
  tl_last_fused = sp.fused ? 0 : 1;
  const double rc = std::sqrt(sp.rc_sq[0]);
  int64_t capacity = std::max<int64_t>(
      {4096, (int64_t)(1.25 * (double)fs.last_m), (int64_t)(1.5 * (double)estimate_edges(sp, rc))});
  // Keep the arena's current size if it is already large enough.
  const size_t have = c.bufs[kSlotOutSh].cap / (3 * sizeof(int32_t));
  if ((int64_t)have > capacity && c.bufs[kSlotOutEi].cap / (2 * sizeof(int64_t)) >= have)
    capacity = (int64_t)have;
  // Hit-mask arena: the last run's need x 1.25, at least 64 words per atom.
  int64_t mask_cap = std::max<int64_t>(64 * sp.n + 4096, fs.last_mask_words + fs.last_mask_words / 4);
  const int64_t mask_have = (int64_t)(c.bufs[kSlotMasks].cap / sizeof(uint32_t));
  if (mask_have > mask_cap) mask_cap = mask_have;
  Status st = prepare_fast(c, sp, capacity, mask_cap);
  if (!st.ok()) return st;

  FastKey key;
  std::memset(&key, 0, sizeof(key));
  key.d_pos = d_pos;
  key.n = sp.n;
  key.grid = sp.grid;
  key.band = sp.band;
  key.stream = c.stream;
  for (int i = 0; i < kSlotCount; ++i) key.bufs[i] = c.bufs[i].p;
  key.capacity = capacity;
  key.mask_cap = mask_cap;
  key.need_rank = sp.rank_cached ? 0 : 1;
  key.prof = c.prof ? 1 : 0;
  key.fused = sp.fused ? 1 : 0;
  key.contiguous = contiguous ? 1 : 0;

  const bool report = !c.prof;
  if (report) c.h_report[0] = 0;

  // (An armed failure-detection hook must reach a directly launched scan,
  // never a captured or replayed one.)
  const bool same = !scan_stall_armed() && fs.have_key &&
                    std::memcmp(&key, &fs.key, sizeof(key)) == 0;
  bool launched = false;
  if (same && fs.exec) {
    if (cudaGraphLaunch(fs.exec, c.stream) == cudaSuccess) {
      note_launches(fs.launches);
      note_graph_replay();
      launched = true;
    } else {
      cudaGetLastError();
    }
  } else if (same && c.stream != nullptr && !c.prof) {
    // (Profiling runs stay outside graphs: its per-phase events are timed on
    // directly launched kernels.)
    // Second identical call: capture the sequence once and replay it.
    if (fs.exec) {
      cudaGraphExecDestroy(fs.exec);
      fs.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    const int64_t l0 = nlb_kernel_launches();
    if (cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      issue_fast(c, sp, d_pos, capacity, contiguous);
      if (cudaStreamEndCapture(c.stream, &graph) == cudaSuccess && graph) {
        if (cudaGraphInstantiate(&fs.exec, graph, 0) != cudaSuccess) fs.exec = nullptr;
        cudaGraphDestroy(graph);
      }
    }
    cudaGetLastError();
    fs.launches = (int)(nlb_kernel_launches() - l0);
    if (fs.exec && cudaGraphLaunch(fs.exec, c.stream) == cudaSuccess) {
      note_graph_replay();
      launched = true;
    }
    cudaGetLastError();
  }
  if (!launched) {
    if (!same && fs.exec) {
      cudaGraphExecDestroy(fs.exec);
      fs.exec = nullptr;
    }
    issue_fast(c, sp, d_pos, capacity, contiguous);
  }
  fs.key = key;
  fs.have_key = true;
  for (int a = 0; a < 3; ++a) c.rank_nb[a] = sp.grid.nb[a];

  if (report) {
    Status rs = wait_report(c);
    if (!rs.ok()) return rs;
    const volatile int64_t* r = c.h_report;
    const int64_t m = r[1];
    if (r[2] != 0) return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
    if (m <= capacity) {
      if (c.stream == c.own_stream) {
        if (!stream_ordered) {
          const cudaError_t e = cudaStreamSynchronize(c.stream);
          if (e != cudaSuccess) return cuda_fail(e, "neighbour-list pipeline");
        }
      } else {
        const cudaError_t e = cudaEventRecord(c.early_ev, c.stream);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
        c.early_stream = c.stream;
      }
      sp.out_dst = sp.fused && !contiguous ? static_cast<int64_t*>(c.bufs[kSlotOutDst].p)
                                           : sp.out_src + m;
      fs.last_m = m;
      fs.last_mask_words = sp.fused ? 0 : r[3];
      *m_out = m;
      return Status{NLB_OK};
    }
    // (M above the capacity: the synchronous path below grows the arrays.)
  }

  // Without the report (phase profiling, or M above the capacity): one
  // synchronisation reads the total edges and the scan's wait-error word.
  cudaError_t e = cudaMemcpyAsync(c.h_small, sp.fused ? sp.fused_total : sp.offs + sp.row,
                                  sizeof(int64_t), cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess)  // the scan's (or the fused look-back's) wait-error word
    e = cudaMemcpyAsync(c.h_small + 1, sp.scan_state + 1, sizeof(int64_t),
                        cudaMemcpyDeviceToHost, c.stream);
  c.h_small[2] = 0;
  if (e == cudaSuccess && !sp.fused)
    e = cudaMemcpyAsync(c.h_small + 2, sp.gb.mask_top, sizeof(int64_t), cudaMemcpyDeviceToHost,
                        c.stream);
  // Grids too large for k_prep's own bin scan use a separate scan (state in
  // gb.scan_tmp): its error word too.
  c.h_small[3] = 0;
  if (e == cudaSuccess && sp.grid.total_bins > kFusedBinScanMax)
    e = cudaMemcpyAsync(c.h_small + 3, sp.gb.scan_tmp + 1, sizeof(int64_t),
                        cudaMemcpyDeviceToHost, c.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  if (e != cudaSuccess) return cuda_fail(e, "neighbour-list pipeline");
  if (c.h_small[1] != 0 || c.h_small[3] != 0)
    return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
  const int64_t m = c.h_small[0];
  if (c.prof) {
    c.prof_pending_count = true;
    c.prof_pending_emit = true;
    c.harvest();
  }
  if (m > capacity) {
    // Arena too small: grow it (outside any capture) and emit again.
    const int64_t cap2 = m + m / 8 + 1024;
    sp.out_src = slot<int64_t>(c, kSlotOutEi, 2 * (size_t)cap2);
    sp.out_sh = slot<int32_t>(c, kSlotOutSh, 3 * (size_t)cap2);
    if (!sp.out_src || !sp.out_sh) return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");
    if (sp.fused) {
      // The fused launch counts again: clear its ticket, look-back words and
      // total first.
      if (!slot<int64_t>(c, kSlotOutDst, (size_t)cap2))
        return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");
      cudaMemsetAsync(sp.fused_state, 0, sizeof(uint64_t) * (size_t)sp.fused_words, c.stream);
      issue_fused(c, sp, cap2, contiguous);
      e = cudaMemcpyAsync(c.h_small + 1, sp.scan_state + 1, sizeof(int64_t),
                          cudaMemcpyDeviceToHost, c.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
      if (e != cudaSuccess) return cuda_fail(e, "fused pass");
      if (c.h_small[1] != 0) return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
    } else {
      launch_pair_emit(sp.grid, sp.gb, sp.n, sp.band, sp.offs, fast_targets(sp, cap2), c.stream);
      e = cudaStreamSynchronize(c.stream);
      if (e != cudaSuccess) return cuda_fail(e, "emit pass");
    }
    fs.have_key = false;  // workspace pointers changed
  }
  sp.out_dst = sp.fused && !contiguous ? static_cast<int64_t*>(c.bufs[kSlotOutDst].p)
                                       : sp.out_src + m;
  fs.last_m = m;
  fs.last_mask_words = c.h_small[2];
  *m_out = m;
  return Status{NLB_OK};
}

}  // namespace nlb
