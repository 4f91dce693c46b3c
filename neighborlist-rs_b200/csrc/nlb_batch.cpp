// nlb_batch.cpp -- batched systems (src/batch.rs:10-290).
//
// Splits the concatenated positions into systems wherever the batch id
// changes.  Consecutive systems of at most kBatchMaxAtoms atoms form a run
// that is planned, counted and emitted on the device by the batched kernels
// (k_batch.cu): four launches and one synchronisation per run, whatever the
// number of systems.  Larger systems take the single-system pipeline.  Lists
// are concatenated in system order with atom indices offset by each system's
// first atom, and each system is planned exactly like a single call (auto-box
// margin and mic_safe from the largest cutoff).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "nlb_internal.h"

namespace nlb {

extern std::atomic<uint64_t> g_bf_threshold;

namespace {

// Grows a context buffer to `need` bytes, keeping its first `used` bytes
// (a device-to-device copy and a free of the old block, only on growth).
bool grow_keep(Ctx::Buf& b, size_t need, size_t used, cudaStream_t s) {
  if (need <= b.cap) return true;
  const size_t cap = std::max<size_t>(need + need / 2, 1 << 16);
  void* q = nullptr;
  if (cudaMalloc(&q, cap) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (b.p) {
    if (used) cudaMemcpyAsync(q, b.p, used, cudaMemcpyDeviceToDevice, s);
    cudaStreamSynchronize(s);
    cudaFree(b.p);
  }
  b.p = q;
  b.cap = cap;
  return true;
}

// The k output lists of one batched call, in the context's persistent
// buffers (allocation only when a call needs more than any before it).
struct Outputs {
  Ctx& c;
  std::vector<int64_t> total;
  Outputs(Ctx& ctx, int32_t k) : c(ctx), total(k, 0) {
    if (c.batch_out.size() < 3 * (size_t)k) c.batch_out.resize(3 * (size_t)k);
  }
  void* src(int32_t q) const { return c.batch_out[3 * q].p; }
  void* dst(int32_t q) const { return c.batch_out[3 * q + 1].p; }
  void* shf(int32_t q) const { return c.batch_out[3 * q + 2].p; }
  bool reserve(const std::vector<int64_t>& add, cudaStream_t s) {
    for (size_t q = 0; q < total.size(); ++q) {
      const size_t used = (size_t)total[q], need = (size_t)(total[q] + add[q]);
      if (!grow_keep(c.batch_out[3 * q], 8 * need, 8 * used, s) ||
          !grow_keep(c.batch_out[3 * q + 1], 8 * need, 8 * used, s) ||
          !grow_keep(c.batch_out[3 * q + 2], 12 * need, 12 * used, s))
        return false;
    }
    return true;
  }
};

CutoffSet make_pass(const std::vector<double>& rc_sq, int32_t g0, bool disjoint) {
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

// One run [a, b) of small systems through the batched kernels.
// With sys_off (k rows of n_systems + 1, sorted cutoff order), also writes
// the first edge of each of systems [a, b) in every list.
Status run_small(Ctx& c, const double* d_pos, const std::vector<int64_t>& starts,
                 const int64_t* d_starts, const double* d_cells, const uint8_t* d_pbcs,
                 const uint8_t* d_has, int32_t a, int32_t b, double rc_max,
                 const std::vector<double>& rc_sq, bool disjoint, bool multi, Outputs& out,
                 std::vector<int64_t>* sys_off) {
  cudaStream_t s = c.stream;
  const int32_t ns = b - a;
  const int32_t k = (int32_t)rc_sq.size();
  const int64_t run_start = starts[a];
  const int64_t run_atoms = starts[b] - run_start;
  const int64_t row = run_atoms + 1;

  // Work items, largest systems first for load balance across the
  // persistent CTAs (larger systems split into chunks of atoms).
  std::vector<int64_t> sizes(ns);
  for (int32_t i = 0; i < ns; ++i) sizes[i] = starts[a + i + 1] - starts[a + i];
  // (every candidate launch shape when this kind of batch is new)
  ShapeTrials trials;
  Status st = trials.prepare(c, make_tune_key(c.device, k, sizes.data(), ns, rc_max),
                             sizes.data(), ns, kSlotBatch0 + 1);
  if (!st.ok()) return st;

  SysPlan* plans = slot<SysPlan>(c, kSlotBatch0 + 0, ns);
  int32_t* flags = slot<int32_t>(c, kSlotBatch0 + 2, 3);  // [0] plan error, [1..2] work counters
  uint32_t* counts = slot<uint32_t>(c, kSlotBatch0 + 3, (size_t)k * row);
  int64_t* offs = slot<int64_t>(c, kSlotBatch0 + 4, (size_t)k * row + 1);
  int64_t* scan_tmp = slot<int64_t>(c, kSlotBatch0 + 5, scan_tmp_elems((int64_t)k * row));
  if (!plans || !flags || !counts || !offs || !scan_tmp)
    return fail(NLB_ERR_NOMEM, "device allocation failed");

  cudaMemsetAsync(flags, 0, sizeof(int32_t) * 3, s);
  cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)k * row, s);
  c.mark(0);
  launch_plan(d_pos, d_starts, a, b, d_cells, d_pbcs, d_has, rc_max, g_bf_threshold.load(),
              multi ? 1 : 0, run_start, plans, flags, s);
  c.mark(1);
  // (The counts are the same in every shape: each trial writes all of them.)
  for (size_t t = 0; t < trials.w.size(); ++t) {
    trials.mark(c, t);
    for (int32_t g0 = 0; g0 < k; g0 += kMaxCutoffsPerPass) {
      const CutoffSet cs = make_pass(rc_sq, g0, disjoint);
      cudaMemsetAsync(flags + 1, 0, sizeof(int32_t) * 2, s);
      launch_batch_count(plans, trials.w[t], d_pos, cs, counts + (size_t)g0 * row, row,
                         flags + 1, s);
    }
  }
  trials.mark(c, trials.w.size());
  c.mark(2);
  exclusive_scan_u32(counts, (int64_t)k * row, offs, scan_tmp, s);
  c.mark(3);
  // Per-system edge offsets within this run, one row of ns + 1 per cutoff.
  std::vector<int64_t> run_bounds;
  if (sys_off) {
    int64_t* d_bounds = slot<int64_t>(c, kSlotBatch0 + 11, (size_t)k * (ns + 1));
    if (!d_bounds) return fail(NLB_ERR_NOMEM, "device allocation failed");
    for (int32_t q = 0; q < k; ++q)
      launch_sys_bounds(plans, ns, offs + (size_t)q * row, row, d_bounds + (size_t)q * (ns + 1), s);
    run_bounds.resize((size_t)k * (ns + 1));
    cudaMemcpyAsync(run_bounds.data(), d_bounds, sizeof(int64_t) * run_bounds.size(),
                    cudaMemcpyDeviceToHost, s);
  }
  if (k + 3 > kSmallHost) return fail(NLB_ERR_VALUE, "too many cutoffs");
  cudaError_t e = cudaMemcpy2DAsync(c.h_small, sizeof(int64_t), offs, sizeof(int64_t) * row,
                                    sizeof(int64_t), (size_t)k + 1, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(c.h_small + k + 1, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)  // the scan's bounded-wait error word
    e = cudaMemcpyAsync(c.h_small + k + 2, scan_tmp + 1, sizeof(int64_t), cudaMemcpyDeviceToHost,
                        s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "batched count pass");
  if (c.h_small[k + 2] != 0) return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
  if (c.prof) {
    c.harvest();
    c.prof_pending_count = true;
    c.harvest();
  }
  const int32_t plan_err = (int32_t)(c.h_small[k + 1] & 0xffffffff);
  if (plan_err == 1) return fail(NLB_ERR_VALUE, "Cell matrix is not invertible");
  if (plan_err == 2) return fail(NLB_ERR_VALUE, "stencil too large for this cutoff and cell");
  std::vector<int64_t> m(k);
  for (int32_t q = 0; q < k; ++q) m[q] = c.h_small[q + 1] - c.h_small[q];
  if (sys_off) {
    const size_t stride = starts.size();  // n_systems + 1
    for (int32_t q = 0; q < k; ++q)
      for (int32_t i = 0; i < ns; ++i)
        (*sys_off)[(size_t)q * stride + a + i] = out.total[q] + run_bounds[(size_t)q * (ns + 1) + i];
  }
  if (!out.reserve(m, s)) return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");

  const BatchItems& bw = trials.pick(c);
  c.mark(4);
  for (int32_t g0 = 0; g0 < k; g0 += kMaxCutoffsPerPass) {
    const CutoffSet cs = make_pass(rc_sq, g0, disjoint);
    EmitTargets t;
    std::memset(&t, 0, sizeof(t));
    for (int32_t q = 0; q < cs.k; ++q) {
      t.src[q] = static_cast<int64_t*>(out.src(g0 + q));
      t.dst[q] = static_cast<int64_t*>(out.dst(g0 + q));
      t.sh[q] = static_cast<int32_t*>(out.shf(g0 + q));
      t.base[q] = out.total[g0 + q];
    }
    cudaMemsetAsync(flags + 1, 0, sizeof(int32_t) * 2, s);
    launch_batch_emit(plans, bw, d_pos, cs, offs + (size_t)g0 * row, row, t, flags + 1, s);
  }
  c.mark(5);
  if (c.prof) c.prof_pending_emit = true;
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "batched emit launch");
  for (int32_t q = 0; q < k; ++q) out.total[q] += m[q];
  return Status{NLB_OK};
}

}  // namespace

Status run_batch(const double* pos, int64_t n, const int32_t* batch, int64_t n_batch,
                 const double* cutoffs, int32_t k, const double* cells, const uint8_t* pbcs,
                 const uint8_t* has_cell, int64_t n_cells, bool disjoint, bool multi,
                 nlb_result* outs, int64_t* sys_offsets) {
  zero_results(outs, k);
  if (n_batch != n) return fail(NLB_ERR_VALUE, "positions and batch must have the same length");
  if (k <= 0) return Status{NLB_OK};
  if (!cutoffs_valid(cutoffs, k))
    return fail(NLB_ERR_VALUE, multi ? "All cutoffs must be positive and finite"
                                     : "Cutoff must be positive and finite");
  if (n == 0) {
    if (sys_offsets) std::memset(sys_offsets, 0, sizeof(int64_t) * (size_t)k);  // no systems
    return empty_results(outs, k);
  }
  if (!pos || !batch) return fail(NLB_ERR_VALUE, "positions or batch is NULL");

  std::vector<int64_t> starts;
  starts.push_back(0);
  for (int64_t i = 1; i < n; ++i)
    if (batch[i] != batch[i - 1]) starts.push_back(i);
  starts.push_back(n);
  const int32_t n_sys = (int32_t)starts.size() - 1;
  const int64_t have = cells ? n_cells : (int64_t)n_sys;
  if (have < (int64_t)n_sys)
    return fail(NLB_ERR_VALUE, "Expected at least " + std::to_string(n_sys) +
                                   " cells, but got " + std::to_string(have));

  std::vector<double> cs(cutoffs, cutoffs + k);
  double rc_max = NAN;
  for (double r : cs) rc_max = fmax_nan_ignoring(rc_max, r);
  const std::vector<int32_t> order = cutoff_order(cutoffs, k);
  std::vector<double> rc_sq(k);
  for (int32_t q = 0; q < k; ++q) rc_sq[q] = cutoffs[order[q]] * cutoffs[order[q]];

  Ctx* c = nullptr;
  Status st = get_ctx(&c);
  if (!st.ok()) return st;
  cudaStream_t s = c->stream;
  double* d_pos = nullptr;
  st = upload_positions(*c, pos, n, &d_pos);
  if (!st.ok()) return st;
  int64_t* d_starts = slot<int64_t>(*c, kSlotBatch0 + 6, starts.size());
  double* d_cells = nullptr;
  uint8_t* d_pbcs = nullptr;
  uint8_t* d_has = nullptr;
  if (!d_starts) return fail(NLB_ERR_NOMEM, "device allocation failed");
  cudaMemcpyAsync(d_starts, starts.data(), sizeof(int64_t) * starts.size(),
                  cudaMemcpyHostToDevice, s);
  if (cells && n_sys > 0) {
    d_cells = slot<double>(*c, kSlotBatch0 + 7, 9 * (size_t)n_sys);
    d_pbcs = slot<uint8_t>(*c, kSlotBatch0 + 8, 3 * (size_t)n_sys);
    d_has = slot<uint8_t>(*c, kSlotBatch0 + 9, (size_t)n_sys);
    if (!d_cells || !d_pbcs || !d_has) return fail(NLB_ERR_NOMEM, "device allocation failed");
    cudaMemcpyAsync(d_cells, cells, sizeof(double) * 9 * n_sys, cudaMemcpyHostToDevice, s);
    if (pbcs)
      cudaMemcpyAsync(d_pbcs, pbcs, 3 * (size_t)n_sys, cudaMemcpyHostToDevice, s);
    else
      cudaMemsetAsync(d_pbcs, 1, 3 * (size_t)n_sys, s);
    if (has_cell)
      cudaMemcpyAsync(d_has, has_cell, (size_t)n_sys, cudaMemcpyHostToDevice, s);
    else
      cudaMemsetAsync(d_has, 1, (size_t)n_sys, s);
  }

  Outputs out(*c, k);
  // Per-system offsets in sorted cutoff order while the runs go by.
  std::vector<int64_t> sys_off;
  if (sys_offsets) sys_off.assign((size_t)k * starts.size(), 0);
  int32_t i = 0;
  while (i < n_sys) {
    const int64_t ni = starts[i + 1] - starts[i];
    if (ni <= kBatchMaxAtoms) {
      int32_t j = i;
      while (j < n_sys && starts[j + 1] - starts[j] <= kBatchMaxAtoms) ++j;
      st = run_small(*c, d_pos, starts, d_starts, d_cells, d_pbcs, d_has, i, j, rc_max, rc_sq,
                     disjoint, multi, out, sys_offsets ? &sys_off : nullptr);
      if (!st.ok()) return st;
      i = j;
      continue;
    }
    // A large system: the single-system pipeline.
    const double* h9 = nullptr;
    bool pb[3] = {false, false, false};
    if (cells && (!has_cell || has_cell[i])) {
      h9 = cells + 9 * (size_t)i;
      for (int a = 0; a < 3; ++a) pb[a] = pbcs ? pbcs[3 * (size_t)i + a] != 0 : true;
    }
    SystemPlan sp;
    st = plan_system(pos + 3 * starts[i], ni, h9, pb, cs, disjoint, multi, sp);
    if (!st.ok()) return st;
    st = count_system(*c, sp, d_pos + 3 * starts[i]);
    if (!st.ok()) return st;
    if (!out.reserve(sp.m, s)) return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");
    DevLists L;
    L.src.resize(k);
    L.dst.resize(k);
    L.sh.resize(k);
    for (int32_t q = 0; q < k; ++q) {
      L.src[q] = static_cast<int64_t*>(out.src(q));
      L.dst[q] = static_cast<int64_t*>(out.dst(q));
      L.sh[q] = static_cast<int32_t*>(out.shf(q));
    }
    st = emit_system(*c, sp, d_pos + 3 * starts[i], L, out.total.data(), starts[i]);
    if (!st.ok()) return st;
    for (int32_t q = 0; q < k; ++q) {
      if (sys_offsets) sys_off[(size_t)q * starts.size() + i] = out.total[q];
      out.total[q] += sp.m[q];
    }
    ++i;
  }

  for (int32_t q = 0; q < k; ++q) {
    nlb_result& r = outs[order[q]];
    st = alloc_result(out.total[q], &r);
    if (!st.ok()) return st;
    const int64_t m = out.total[q];
    if (m == 0) continue;
    cudaMemcpyAsync(r.edge_index, out.src(q), 8 * m, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(r.edge_index + m, out.dst(q), 8 * m, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(r.shift, out.shf(q), 12 * m, cudaMemcpyDeviceToHost, s);
  }
  if (sys_offsets) {
    const size_t stride = starts.size();
    for (int32_t q = 0; q < k; ++q) {
      sys_off[(size_t)q * stride + n_sys] = out.total[q];
      std::memcpy(sys_offsets + (size_t)order[q] * stride, sys_off.data() + (size_t)q * stride,
                  sizeof(int64_t) * stride);
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (c->prof) c->harvest();
  if (e != cudaSuccess) {
    for (int32_t q = 0; q < k; ++q) nlb_result_free(&outs[q]);
    return cuda_fail(e, "batched emit");
  }
  return Status{NLB_OK};
}

}  // namespace nlb
