// nlb_batch.cpp -- batched systems (src/batch.rs:10-290).
//
// Splits the concatenated positions into systems wherever the batch id
// changes, plans every system exactly like a single call (auto-box margin and
// mic_safe from the largest cutoff), and concatenates the per-system lists in
// system order with atom indices offset by each system's first atom.
#include <cstring>
#include <string>
#include <vector>

#include "nlb_internal.h"

namespace nlb {

namespace {

// Grow-only device array that keeps its contents when it grows.
struct GrowBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool reserve(size_t need, cudaStream_t s) {
    if (need <= bytes) return true;
    size_t cap = std::max<size_t>(need + need / 2, 1 << 16);
    void* q = nullptr;
    if (cudaMalloc(&q, cap) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (p) {
      cudaMemcpyAsync(q, p, bytes, cudaMemcpyDeviceToDevice, s);
      cudaStreamSynchronize(s);
      cudaFree(p);
    }
    p = q;
    bytes = cap;
    return true;
  }
  ~GrowBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

Status run_batch(const double* pos, int64_t n, const int32_t* batch, int64_t n_batch,
                 const double* cutoffs, int32_t k, const double* cells, const uint8_t* pbcs,
                 const uint8_t* has_cell, int64_t n_cells, bool disjoint, bool multi,
                 nlb_result* outs) {
  zero_results(outs, k);
  if (n_batch != n) return fail(NLB_ERR_VALUE, "positions and batch must have the same length");
  if (k <= 0) return Status{NLB_OK};
  if (!cutoffs_valid(cutoffs, k))
    return fail(NLB_ERR_VALUE, multi ? "All cutoffs must be positive and finite"
                                     : "Cutoff must be positive and finite");
  if (n == 0) return empty_results(outs, k);
  if (!pos || !batch) return fail(NLB_ERR_VALUE, "positions or batch is NULL");

  std::vector<std::pair<int64_t, int64_t>> sys;
  int64_t start = 0;
  for (int64_t i = 1; i < n; ++i)
    if (batch[i] != batch[i - 1]) {
      sys.push_back({start, i});
      start = i;
    }
  sys.push_back({start, n});
  const int64_t have = cells ? n_cells : (int64_t)sys.size();
  if (have < (int64_t)sys.size())
    return fail(NLB_ERR_VALUE, "Expected at least " + std::to_string(sys.size()) +
                                   " cells, but got " + std::to_string(have));

  std::vector<double> cs(cutoffs, cutoffs + k);
  Ctx* c = nullptr;
  Status st = get_ctx(&c);
  if (!st.ok()) return st;
  double* d_pos = nullptr;
  st = upload_positions(*c, pos, n, &d_pos);
  if (!st.ok()) return st;

  std::vector<GrowBuf> src(k), dst(k), shf(k);
  std::vector<int64_t> total(k, 0);
  std::vector<int32_t> order;
  for (size_t s = 0; s < sys.size(); ++s) {
    const int64_t b = sys[s].first, e = sys[s].second;
    const double* h9 = nullptr;
    bool pb[3] = {false, false, false};
    if (cells && has_cell && has_cell[s]) {
      h9 = cells + 9 * s;
      for (int a = 0; a < 3; ++a) pb[a] = pbcs ? pbcs[3 * s + a] != 0 : true;
    }
    SystemPlan sp;
    st = plan_system(pos + 3 * b, e - b, h9, pb, cs, disjoint, multi, sp);
    if (!st.ok()) return st;
    if (order.empty()) order = sp.order;
    st = count_system(*c, sp, d_pos + 3 * b);
    if (!st.ok()) return st;
    DevLists L;
    L.src.resize(k);
    L.dst.resize(k);
    L.sh.resize(k);
    for (int32_t q = 0; q < k; ++q) {
      const size_t need = (size_t)(total[q] + sp.m[q]);
      if (!src[q].reserve(8 * need, c->stream) || !dst[q].reserve(8 * need, c->stream) ||
          !shf[q].reserve(12 * need, c->stream))
        return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");
      L.src[q] = static_cast<int64_t*>(src[q].p);
      L.dst[q] = static_cast<int64_t*>(dst[q].p);
      L.sh[q] = static_cast<int32_t*>(shf[q].p);
    }
    st = emit_system(*c, sp, d_pos + 3 * b, L, total.data(), b);
    if (!st.ok()) return st;
    for (int32_t q = 0; q < k; ++q) total[q] += sp.m[q];
  }
  for (int32_t q = 0; q < k; ++q) {
    nlb_result& r = outs[order[q]];
    st = alloc_result(total[q], &r);
    if (!st.ok()) return st;
    if (total[q] == 0) continue;
    cudaMemcpyAsync(r.edge_index, src[q].p, 8 * total[q], cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(r.edge_index + total[q], dst[q].p, 8 * total[q], cudaMemcpyDeviceToHost,
                    c->stream);
    cudaMemcpyAsync(r.shift, shf[q].p, 12 * total[q], cudaMemcpyDeviceToHost, c->stream);
  }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    for (int32_t q = 0; q < k; ++q) nlb_result_free(&outs[q]);
    return cuda_fail(e, "batched emit");
  }
  return Status{NLB_OK};
}

}  // namespace nlb
