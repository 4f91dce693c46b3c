// nlb_kernels.h -- host launchers for the sm_100a kernels.
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "nlb_common.cuh"

namespace nlb {

// ---- k_scan.cu
// Exclusive scan of n values into out[0..n]; out[n] = total.  `tmp` needs
// scan_tmp_elems(n) = ceil(n / kScanTile) + 2 int64 elements.
constexpr int64_t kScanTile = 2048;  // elements per CTA (measured best of 1024-4096)
int64_t scan_tmp_elems(int64_t n);
// Failure-detection hook: the calling thread's next scan launch has `tile`
// withhold its publication and its successors poll at most spin_limit times
// (then record the error word and finish).  One-shot.
void arm_scan_stall(int32_t tile, int32_t spin_limit);
bool scan_stall_armed();
// Takes the armed hook for a launch that is not a scan (the fused search's
// look-back over groups); false when none is armed.
bool take_scan_stall(int32_t* tile, int32_t* spin_limit);
void exclusive_scan_u32(const uint32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                        cudaStream_t s);
void exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                        cudaStream_t s);
// As exclusive_scan_u32 with a state buffer (scan_tmp_elems(n) words) that
// the caller has already zeroed in stream order.
void exclusive_scan_u32_zeroed(const uint32_t* in, int64_t n, int64_t* out, int64_t* tmp,
                               cudaStream_t s);

// ---- k_grid.cu : cell-list build (src/search.rs:92-264)
// Buffers for one system's grid; all device pointers.
struct GridBuffers {
  int32_t* rank_of_bin;   // [total_bins] Morton rank of each linear bin
  int32_t* bin_count;     // [total_bins] atoms per bin rank (zeroed by caller)
  int32_t* bin_fill;      // [total_bins] scatter cursors (zeroed by caller)
  int64_t* bin_start;     // [total_bins + 1]
  uint64_t* key;          // [n] atom Morton keys (original order)
  int32_t* rank;          // [n] bin rank of each atom (original order)
  uint64_t* skey;         // [n] keys scattered by bin
  int32_t* sidx;          // [n] original indices scattered by bin
  uint64_t* skey2;        // [n] merge scratch for bins above the shared-memory capacity
  int32_t* sidx2;         // [n]
  double* px;             // [n] sorted wrapped positions (SoA)
  double* py;
  double* pz;
  SlotMeta* meta;         // [n] sorted wrap shifts + original index
  int64_t* scan_tmp;
  // Optional (nullptr = not produced): FP32 position of each sorted atom
  // relative to its own bin centre, with the original index in .w, and the
  // atom's linear bin index.  Used by the FP32 guard-band search kernels.
  float4* p32;
  int32_t* sbin;
  // Work lists for the pair-task search (k_search2.cu), filled by the build
  // when p32 is set: groups[g] = {first sorted slot, bin rank} of each run of
  // at most 32 atoms of one bin; irr_list = sorted slots of atoms whose home
  // stencil (recomputed from the wrapped position) differs from their stored
  // bin; irr[p] = 1 for those atoms; counters[0] = #groups, [1] = #irregular
  // (zeroed by the caller before the build).
  GroupRec* groups;
  int32_t* irr_list;
  uint8_t* irr;
  int32_t* counters;
  // Optional (zeroed by the caller before the build): completion counter of
  // k_prep, whose last CTA then scans the bin histogram into bin_start
  // itself (grids of at most kFusedBinScanMax bins); nullptr: separate scan.
  int32_t* build_done;
  // Optional (zeroed by the caller before the build): task counter of the
  // pair-task emit pass, which then hands tasks out dynamically on dense
  // grids (expensive, uneven tasks); nullptr: static assignment.
  uint32_t* emit_queue;
  // Optional (masks == nullptr: the emit pass recomputes every test): the
  // count pass stores, per pair task, the candidate range, image shift and a
  // 32-bit hit mask per lane per 32-candidate chunk per cutoff in `masks`
  // (bump-allocated through *mask_top, at most mask_cap words; cutoff q's
  // masks follow cutoff q - 1's); the emit pass then only expands bits.
  // task_hdr[task] = {mask base (-2: nothing to emit, -1: recompute), b0,
  // b1, packed shift}.
  int4* task_hdr;
  uint32_t* masks;
  unsigned long long* mask_top;
  int64_t mask_cap;
  // Optional (nullptr: no chunk pruning), set on grids dense enough that a
  // bin holds several 32-atom chunks: FP32 bounding box, in its bin's frame,
  // of the chunk of up to 32 sorted atoms starting at slot j (every chunk
  // starts at its bin's first slot + a multiple of 32): cbox[2j] = lower
  // corner, cbox[2j + 1] = upper corner.  Written by the build; the count
  // pass skips a (group, chunk) pair whose boxes are farther apart than the
  // guard band's upper bound by more than the band's width.
  float4* cbox;
  // Optional ([total_bins], written by k_prep's own bin scan): canonical
  // index of each bin's first group; the build then stores groups[] in
  // canonical order (bins in rank order, runs in slot order).
  int32_t* group_start;
  // Optional ([n]): each atom's place in its bin segment, taken by k_prep
  // from the histogram (k_scatter then needs no atomics); nullptr: k_scatter
  // takes places from bin_fill.
  int32_t* fill;
};

// Grids with at least this many atoms per bin on average get chunk boxes.
constexpr double kChunkPruneMinPerBin = 64.0;

constexpr int64_t kFusedBinScanMax = 65536;

// need_rank_table = false reuses rank_of_bin from a previous build with the
// same bins per axis.
void launch_grid_build(const GridParams& g, const double* pos, int64_t n, const GridBuffers& b,
                       cudaStream_t s, bool need_rank_table = true);

// ---- k_search.cu : count / emit (src/search.rs:291-446, :448-1078, :1187-1405)
struct CutoffSet {
  double rc_sq[kMaxCutoffsPerPass];  // ascending squared cutoffs of this pass
  int32_t k;                         // cutoffs in this pass (1..32)
  int32_t disjoint;                  // shells: first ascending cutoff only
  double lower_sq;                   // disjoint: squared cutoff just below this pass (or -1)
  double max_sq;                     // squared max cutoff of the whole call (pair filter)
};

struct EmitTargets {
  int64_t* src[kMaxCutoffsPerPass];  // edge sources per cutoff: [e]
  int64_t* dst[kMaxCutoffsPerPass];  // edge destinations per cutoff: [e]
  int32_t* sh[kMaxCutoffsPerPass];   // shifts per cutoff: [3e .. 3e+2]
  int64_t base[kMaxCutoffsPerPass];  // first edge slot of this system per cutoff
  int64_t index_offset;              // added to both atom indices (batched systems)
  // Pair-task emit only: when set, the list's total M is read from device
  // memory, destinations go to src[0] + M (the [src | dst] layout), and
  // nothing is written if M > capacity (the caller grows and re-emits).
  const int64_t* total_dev;
  int64_t capacity;
  // Pair-task emit only: when set and non-zero (the offsets scan gave up
  // waiting for a tile), nothing is written: the offsets are not valid.
  const int64_t* scan_error;
  // Pair-task emit only, optional: host-mapped report that block 0 fills as
  // the launch starts (the list's size is known then): [1] M, [2] the wait
  // error words (scan_error, grid_scan_error) or-ed, [3] *mask_top, then
  // [0] = 1.
  int64_t* report;
  const int64_t* grid_scan_error;
  const unsigned long long* mask_top;
  // Batched kernels: 1 = atom indices local to each system (served requests),
  // 0 = global indices (system start added).
  int32_t local_indices;
  // Batched kernels with per-system cutoffs: 1 = each system's list is one
  // contiguous [src | dst] block starting at src[0] + 2 * (its first edge
  // slot), with shifts at sh[0] + 3 * slot as usual (served requests).
  int32_t system_blocks;
};

// counts[q * (n + 1) + p] for sorted atom p; the trailing slot of each row is 0.
void launch_grid_count(const GridParams& g, const GridBuffers& b, int64_t n,
                       const CutoffSet& cs, uint32_t* counts, cudaStream_t s);
void launch_grid_emit(const GridParams& g, const GridBuffers& b, int64_t n, const CutoffSet& cs,
                      const int64_t* offs, const EmitTargets& t, cudaStream_t s);

// ---- k_search2.cu : stencil search as (atom group, stencil cell) tasks
// with an FP32 pair test and an exact FP64 recheck inside a guard band
// around each rc^2 (see k_search2.cu); one traversal serves up to
// kFp32MaxCutoffs cutoffs.
struct GuardBand {
  float lo;       // d2_32 < lo  => certainly inside (d2_64 < rc^2)
  float hi;       // d2_32 >= hi => certainly outside
  double rc_sq;   // exact test for d2_32 in [lo, hi)
};
// Cutoffs one pair-task traversal tests at once; more use the FP64 kernels.
constexpr int32_t kFp32MaxCutoffs = 4;
// The bands of k ascending cutoffs.  Counts and offsets hold one row of
// `row` = n * S + 1 entries per cutoff (S = stencil cells).
struct PairBands {
  GuardBand q[kFp32MaxCutoffs];
  int64_t row;
  int32_t k;
  int32_t disjoint;  // 1: list q leaves out the pairs inside cutoff q - 1
};
// Stencils above this many cells use the per-atom FP64 kernels.
constexpr int64_t kPairMaxCells = 1024;
// ---- k_fused.cu : count + offsets + emit of the single-cutoff list in one
// launch (one CTA per 32-atom group, decoupled look-back over the groups).
// Needs the groups in canonical order (GridBuffers::group_start set for the
// build) and at most kFusedMaxCells stencil cells.
constexpr int32_t kFusedMaxCells = 125;
// Grids with more atoms per bin than this keep the three-launch pipeline
// (measured at 370 atoms per bin, rc 14 on the cluster liquid: one launch
// 326 us against 189 us for count + scan + emit).
constexpr double kFusedMaxPerBin = 64.0;
// Hit-mask words a group keeps in shared memory: enough for every stencil
// cell at 1.5 x the mean bin occupancy, within these bounds (cells beyond
// the budget recompute their tests when the group writes).
constexpr int32_t kFusedMaskMin = 4096;
constexpr int32_t kFusedMaskMax = 12288;
struct FusedOut {
  int64_t* src;       // [capacity] sources
  int64_t* dst;       // [capacity] destinations (a separate array)
  int32_t* sh;        // [3 capacity] shifts
  int64_t capacity;   // a group whose block does not fit writes nothing
  uint64_t* state;    // zeroed: [0] group ticket, [1] error word, [2 + g] group g's look-back word
  int64_t* total;     // receives M
  // Zeroed completion count of the groups; the group that completes it
  // copies {M, error word} into `report` (host-mapped pinned memory, may be
  // null) and then sets report[0] = 1, so the host learns M without waiting
  // for the launch (or the ones queued after it) to end.
  unsigned long long* done;
  int64_t* report;
  // 1: after the last group, the CTAs move the M destinations behind the M
  // sources (src[M + e] = dst[e]: the [src | dst] layout of device results).
  int32_t move;
  int32_t spin_limit; // polls of one look-back wait before it gives up
  int32_t withhold;   // failure-detection hook: this group never publishes (-1: none)
  int32_t mask_words; // hit-mask words per group in shared memory
};
__host__ __device__ inline size_t fused_cells_bytes(int32_t n_cells) {
  return ((size_t)88 * (size_t)n_cells + 15) & ~(size_t)15;
}
size_t fused_smem_bytes(int32_t n_cells, int32_t mask_words);
constexpr int32_t kFusedSpinLimit = 1 << 22;
void launch_pair_fused(const GridParams& g, const GridBuffers& b, int32_t n_cells,
                       const GuardBand& band, const FusedOut& o, cudaStream_t s);

// Returns false when the FP32 test cannot be made safe for this grid (the
// band would be too wide); callers then use the FP64 kernels.
bool make_guard_band(const GridParams& g, double rc, GuardBand& band);
// counts[p * S + c] for every sorted atom p and cell c, plus counts[n * S] = 0.
void launch_pair_count(const GridParams& g, const GridBuffers& b, int64_t n,
                       const GuardBand& band, uint32_t* counts, cudaStream_t s);
// offs = exclusive scan of those counts; edges of (p, c) start at
// t.base[0] + offs[p * S + c] - offs[0].
void launch_pair_emit(const GridParams& g, const GridBuffers& b, int64_t n,
                      const GuardBand& band, const int64_t* offs, const EmitTargets& t,
                      cudaStream_t s);
// The same for bands.k cutoffs in one traversal: row q of counts / offs
// (counts + q * bands.row) belongs to cutoff q, whose edges of (p, c) start
// at t.base[q] + offs[q * row + p * S + c] - offs[q * row] in t.src[q] /
// t.dst[q] / t.sh[q].  With b.masks set, the count pass records its hit
// masks and the emit pass expands them.
void launch_pair_count_multi(const GridParams& g, const GridBuffers& b, int64_t n,
                             const PairBands& bands, uint32_t* counts, cudaStream_t s);
void launch_pair_emit_multi(const GridParams& g, const GridBuffers& b, int64_t n,
                            const PairBands& bands, const int64_t* offs, const EmitTargets& t,
                            cudaStream_t s);

enum BruteMode : int32_t { kBruteRaw = 0, kBruteMicMode = 1 };
struct BruteParams {
  double h[9];
  double hinv[9];
  int32_t pbc[3];
  int32_t mode;
};
void launch_brute_count(const BruteParams& bp, const double* pos, int64_t n, const CutoffSet& cs,
                        uint32_t* counts, cudaStream_t s);
void launch_brute_emit(const BruteParams& bp, const double* pos, int64_t n, const CutoffSet& cs,
                       const int64_t* offs, const EmitTargets& t, cudaStream_t s);

// ---- k_batch.cu : many small systems per launch (one CTA per system)
constexpr int kBatchMaxAtoms = 2048;  // larger systems take the single-system pipeline

struct SysPlan {
  GridParams g;      // h / hinv always; grid fields for the cell-list method
  int32_t pbc[3];
  int32_t method;    // 0 brute force (raw), 1 brute force (MIC), 2 cell list, -1 invalid cell
  int64_t start;     // first atom of the system (global index)
  int32_t n;         // atoms
  int32_t slot;      // first count slot of the system inside its run
  double rc_sq;      // the system's own squared cutoff (per-system cutoff runs)
};

size_t batch_smem_bytes(int cap);
// Plans systems [s0, s1): plans[s - s0].  error_flag: 1 = singular cell,
// 2 = stencil too large.
// sys_rc (optional, indexed like starts): a cutoff per system; the count /
// emit launches then take a CutoffSet with k == 0 and use each plan's rc_sq.
void launch_plan(const double* pos, const int64_t* starts, int32_t s0, int32_t s1,
                 const double* cells, const uint8_t* pbcs, const uint8_t* has_cell, double rc_max,
                 uint64_t bf_threshold, int multi, int64_t run_start, SysPlan* plans,
                 int32_t* error_flag, cudaStream_t s, const double* sys_rc = nullptr);
// out[s] = first edge of system s relative to the run (k == 1 rows), out[ns] = total.
void launch_sys_bounds(const SysPlan* plans, int n_sys, const int64_t* offs, int64_t row,
                       int64_t* out, cudaStream_t s);
// Launch shape of the batched kernels: the systems of at most large_atoms
// atoms are one work item each, run by CTAs of small_threads; larger systems
// are split into work items of `chunk` atoms run by CTAs of large_threads.
// Every shape gives the same results (counts per atom, offsets from one
// scan); which is fastest depends on the mix, so the tuner (nlb_tune.cpp)
// picks one per kind of batch.  Cell size is not a free parameter: the bins
// of the cell list fix the output order.
struct BatchShape {
  int small_threads;  // 64, 128, 256 or 512
  int large_threads;  // 256 or 512
  int chunk;          // atoms per work item of a large system
  int large_atoms;    // systems above this many atoms are split
};
constexpr int kBatchShapes = 7;
extern const BatchShape kBatchShapeTable[kBatchShapes];  // [0]: the default
// Loads every batched kernel variant into the current device's context, so
// that no variant's first launch pays for loading its module.
void preload_batch_kernels();
// Work items of one batched pass: (system, first atom) pairs, the split
// (large) systems first, then the others, each group largest first.
// cap_* = power of two >= the largest system of the group.
struct BatchItems {
  const int2* items = nullptr;  // device: [n_large | n_small]
  int n_large = 0, n_small = 0;
  int cap_large = 32, cap_small = 32;
  BatchShape shape{256, 512, 256, 512};
};
// Host: builds the item list (upload it and set w.items before launching).
void plan_batch_items(const int64_t* sizes, int n_sys, const BatchShape& shape,
                      std::vector<int2>& items, BatchItems& w);
// Hit records of a single-cutoff batched count pass, expanded into the list
// by launch_batch_expand instead of a recomputing emit pass.  seg_top,
// overflow and need_recompute must be zero on entry; capacity: seg_cap
// segments of 32 records (3 words each), meta: one per run slot.
struct BatchRecords {
  int4* seg_hdr;         // {run slot of the atom, its edges in earlier segments, records, system}
  uint32_t* rec;         // [seg_cap * 32 * 3]
  SlotMeta* meta;        // sorted meta per run slot (orig: index within the system)
  int* seg_top;          // segments used
  int* overflow;         // 1: records incomplete (the emit pass must recompute)
  int* need_recompute;   // set by the expansion when it found the overflow flag
  int seg_cap;
};

// counts[q * row + slot + p]; work2[0..1] must be zero on entry.  With rec
// (single-cutoff passes only) the pass also writes hit records.
void launch_batch_count(const SysPlan* plans, const BatchItems& w, const double* pos,
                        const CutoffSet& cs, uint32_t* counts, int64_t row, int* work2,
                        cudaStream_t s, const BatchRecords* rec = nullptr);
// Writes the single-cutoff list from the records (t: src/dst/sh[0], base[0],
// index options, capacity and scan_error as for launch_batch_emit).
void launch_batch_expand(const BatchRecords& rb, const SysPlan* plans, const double* pos,
                         const int64_t* offs, int64_t row, const EmitTargets& t, cudaStream_t s);
void launch_batch_emit(const SysPlan* plans, const BatchItems& w, const double* pos,
                       const CutoffSet& cs, const int64_t* offs, int64_t row,
                       const EmitTargets& t, int* work2, cudaStream_t s);

// Sets the dynamic shared-memory limit of a kernel once per device.
void ensure_smem_attr(const void* func, int bytes);

// Counts kernel launches issued by this library (reported by nlb_kernel_launches).
void note_launches(int n);

// ---- k_grid.cu : per-axis min / max of device positions (auto-box bounds)
// out[0..2] = min, out[3..5] = max (NaN coordinates are ignored, like the
// reference's `<` / `>` scan starting from +/-inf).
void launch_bounds(const double* pos, int64_t n, double* out, cudaStream_t s);

// Output options on a device half list ([src | dst] ei, shifts sh, m edges):
// directed list, displacement vectors, distances (k_extras.cu).  Outputs
// that are not wanted are NULL; with directed == 0 ei_out/sh_out may be NULL.
struct EdgeExtrasCell {
  double h[9];       // row-major H (columns = lattice vectors)
  int32_t has_cell;  // 0: no H term (vectors are r_j - r_i)
};
void launch_edge_extras(const double* pos, const EdgeExtrasCell& cell, const int64_t* ei,
                        const int32_t* sh, int64_t m, int directed, int64_t* ei_out,
                        int32_t* sh_out, double* vec, double* dist, cudaStream_t s);

// Verlet list manager (k_verlet.cu): largest squared displacement against
// the reference positions (as the bits of a double in *out); the stored
// edges kept at rc, compacted in stored order.
void launch_max_disp(const double* pos, const double* ref, int64_t n, unsigned long long* out,
                     cudaStream_t s);
// The kept edges in one pass (k_verlet_compact): out_ei [src | dst] of M
// edges and out_sh; dst_tmp has room for m destinations; state has
// verlet_compact_state_words(m) words (cleared here): [1] the look-back's
// error word, [3] M.
int64_t verlet_compact_state_words(int64_t m);
void launch_verlet_compact(const double* pos, const EdgeExtrasCell& cell, const int64_t* ei,
                           const int32_t* sh, int64_t m, double rc_sq, int64_t* out_ei,
                           int32_t* out_sh, int64_t* dst_tmp, uint64_t* state,
                           int32_t spin_limit, cudaStream_t s);

}  // namespace nlb
