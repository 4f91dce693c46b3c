// nlb_server.cpp -- continuous-batching request loop.
//
// Clients submit structures of any size as they arrive; worker threads (each
// with its own CUDA stream and device workspace on the same GPU) repeatedly
// take the next work item from a shared FIFO:
//   * a batch: every queued small request (<= kBatchMaxAtoms atoms) that fits
//     the HBM budget, up to max_batch, planned/counted/emitted by the batched
//     kernels in one pass with a cutoff per system;
//   * or a single large request, run by the single-system pipeline.
// Requests that arrive while a batch runs join the next one, and work of
// different workers overlaps on the device.  Admission reserves a density-
// based estimate of each request's device footprint (positions, workspace,
// edges) against the budget; device-resident results keep their edge bytes
// reserved until the client releases them.  Each result is identical to the
// same request built alone (the kernels decide every edge per system).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "nlb_internal.h"

namespace nlb {

extern std::atomic<uint64_t> g_bf_threshold;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Req {
  int64_t id = 0;
  int64_t n = 0;
  double* pos = nullptr;  // pinned host copy
  bool has_cell = false;
  double h[9] = {0};
  uint8_t pbc[3] = {1, 1, 1};
  double rc = 0.0;
  bool device_result = false;
  size_t est_bytes = 0;     // reserved while queued / running
  size_t est_result = 0;    // estimated result bytes (28 per edge)
  size_t result_bytes = 0;  // stays reserved for device results until release
  double t_submit = 0, t_done = 0;
  int status = 0;  // 0 queued, 1 running, 2 done, <0 error code
  std::string err;
  int64_t m = 0;
  int64_t* ei = nullptr;  // [src | dst]
  int32_t* sh = nullptr;
  void* dev_block = nullptr;  // device result: the batch block ei/sh point into
  bool fail_staging = false;  // failure-detection hook: the staging of any batch holding it fails
};

// Result bytes one batch of small requests may produce (estimated): bounds
// the pinned block each batch copies its results into, so blocks are reused
// from the pool, and lets the workers overlap one batch's copies with the
// next batch's kernels.
constexpr size_t kBatchResultBytes = size_t(192) << 20;

// Pinned host memory pre-carved when a server starts: an eighth of its HBM
// budget, within [1, 4] GB (cudaHostAlloc pins ~1.7 GB/s here, far too slow
// to grow the pool on a request's critical path).
constexpr size_t kReservePinnedMin = size_t(1) << 30;
constexpr size_t kReservePinnedMax = size_t(4) << 30;
// Device-result pool memory mapped when a server starts (at most its budget).
constexpr size_t kPoolWarm = size_t(8) << 30;
// Workspace memory mapped at start (at most a quarter of the budget).
constexpr size_t kWorkspaceWarm = size_t(16) << 30;

// Pinned block size for `bytes`: the next power of two (at least 1 MB), so
// blocks of consecutive batches are interchangeable in the pool.
size_t block_class(size_t bytes) {
  size_t c = size_t(1) << 20;
  while (c < bytes) c <<= 1;
  return c;
}

// Returns the estimated device footprint; sets *result to the estimated
// result bytes.
size_t estimate_bytes(const Req& r, size_t* result) {
  *result = 0;
  if (r.n == 0) return 4096;
  // Density-based edge estimate: half the neighbours within rc at the mean
  // density of the system's box (its cell, or the auto-box of its span).
  double vol = 0.0;
  if (r.has_cell) {
    const double* h = r.h;
    vol = std::fabs(h[0] * (h[4] * h[8] - h[7] * h[5]) - h[1] * (h[3] * h[8] - h[6] * h[5]) +
                    h[2] * (h[3] * h[7] - h[6] * h[4]));
  } else {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < r.n; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], r.pos[3 * i + a]);
        hi[a] = std::max(hi[a], r.pos[3 * i + a]);
      }
    vol = 1.0;
    for (int a = 0; a < 3; ++a) vol *= (hi[a] - lo[a]) + 2.0 * (r.rc + 1.0);
  }
  const double rho = vol > 0 ? (double)r.n / vol : 0.0;
  // Boxes smaller than 2 rc see several images of every atom.
  const double per_atom = 0.5 * rho * (4.0 / 3.0) * 3.141592653589793 * r.rc * r.rc * r.rc + 1.0;
  const double edges = 1.3 * (double)r.n * per_atom + 64.0;
  const double work = 24.0 * r.n + 220.0 * r.n + 12.0 * 27.0 * r.n;
  *result = (size_t)std::min(edges * 28.0, 1e15);
  return (size_t)std::min(edges * 28.0 + work, 1e15);
}

}  // namespace

class Server {
 public:
  Server(int device, size_t budget, int n_workers, int max_batch)
      : device_(device), budget_(budget), max_batch_(std::max(1, max_batch)) {
    for (int w = 0; w < std::max(1, n_workers); ++w) threads_.emplace_back([this] { worker(); });
  }

  // Device results come from a server-owned stream-ordered pool (no
  // device-wide synchronisation per result); frees go to `free_stream_`.
  // Returns false (message set) if the pool cannot be created.
  bool init_device_pool() {
    cudaSetDevice(device_);
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    cudaError_t e = cudaMemPoolCreate(&pool_, &props);
    if (e == cudaSuccess) {
      uint64_t keep = budget_;
      e = cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&free_stream_, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      cuda_fail(e, "device result pool");
      return false;
    }
    // Map the pool's first kPoolWarm bytes now: growing it under load maps
    // fresh device memory on a worker's critical path and stalls the other
    // workers meanwhile (measured: a served run of device results at 7k
    // instead of ~100k systems/s).  The release threshold keeps it mapped.
    void* warm = nullptr;
    const size_t warm_bytes = std::min<size_t>(budget_, kPoolWarm);
    if (cudaMallocFromPoolAsync(&warm, warm_bytes, pool_, free_stream_) == cudaSuccess) {
      cudaFreeAsync(warm, free_stream_);
      cudaStreamSynchronize(free_stream_);
    }
    cudaGetLastError();
    // The same for the pool the workers' workspaces grow from: a worker
    // that first meets a request larger than any it has held maps several
    // GB (result arrays, hit masks) while the others wait.
    warm_result_pool(device_, std::min<size_t>(budget_ / 4, kWorkspaceWarm), free_stream_);
    // Pinned host blocks for request positions and host results, carved
    // before the first request rather than on its critical path.
    pinned_reserve(std::min(kReservePinnedMax, std::max(kReservePinnedMin, budget_ / 8)));
    return true;
  }

  ~Server() {
    {
      // Requests still queued are cancelled; running ones finish.
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      for (Req* r : queue_) {
        r->status = -NLB_ERR_VALUE;
        r->err = "server destroyed before the request ran";
      }
      queue_.clear();
    }
    cv_work_.notify_all();
    cv_done_.notify_all();
    for (auto& t : threads_) t.join();
    for (auto& kv : reqs_) free_req(kv.second);
    if (free_stream_) {
      cudaStreamSynchronize(free_stream_);
      cudaStreamDestroy(free_stream_);
    }
    if (pool_) cudaMemPoolDestroy(pool_);
  }

  int64_t submit(const double* pos, int64_t n, const double* cell, const uint8_t* pbc, double rc,
                 bool device_result) {
    if (!std::isfinite(rc) || rc <= 0.0) {
      fail(NLB_ERR_VALUE, "Cutoff must be positive and finite");
      return -NLB_ERR_VALUE;
    }
    if (n < 0 || (n > 0 && !pos)) {
      fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
      return -NLB_ERR_VALUE;
    }
    if (n > (int64_t)INT32_MAX - 1) {
      fail(NLB_ERR_VALUE, "more than 2^31 atoms in one system");
      return -NLB_ERR_VALUE;
    }
    if (cell) {
      HostCell hc;
      std::string err;
      const bool pb[3] = {true, true, true};
      if (!make_cell(cell, pb, hc, err)) {
        fail(NLB_ERR_VALUE, err);
        return -NLB_ERR_VALUE;
      }
    }
    Req* r = new Req();
    r->n = n;
    r->rc = rc;
    r->device_result = device_result;
    if (cell) {
      r->has_cell = true;
      std::memcpy(r->h, cell, sizeof(r->h));
      for (int a = 0; a < 3; ++a) r->pbc[a] = pbc ? pbc[a] : 1;
    }
    if (n > 0) {
      r->pos = static_cast<double*>(pinned_alloc(sizeof(double) * 3 * (size_t)n));
      if (!r->pos) {
        delete r;
        fail(NLB_ERR_NOMEM, "pinned host allocation failed");
        return -NLB_ERR_NOMEM;
      }
      std::memcpy(r->pos, pos, sizeof(double) * 3 * (size_t)n);
    }
    r->est_bytes = estimate_bytes(*r, &r->est_result);
    if (r->est_bytes > budget_) {
      free_req(r);
      fail(NLB_ERR_VALUE, "request exceeds the server's HBM budget");
      return -NLB_ERR_VALUE;
    }
    r->t_submit = now_s();
    std::lock_guard<std::mutex> lk(mu_);
    r->id = next_id_++;
    reqs_[r->id] = r;
    queue_.push_back(r);
    ++submitted_;
    cv_work_.notify_one();
    return r->id;
  }

  // NLB_OK = done (out filled), NLB_NOT_READY = not done within the timeout,
  // else the request's error code.
  int wait(int64_t id, double timeout_s, nlb_result* out, double* latency_ms) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return fail(NLB_ERR_VALUE, "unknown ticket").code;
    Req* r = it->second;
    const auto pred = [&] { return r->status == 2 || r->status < 0; };
    if (timeout_s < 0)
      cv_done_.wait(lk, pred);
    else if (!cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
      return NLB_NOT_READY;
    if (latency_ms) *latency_ms = 1e3 * (r->t_done - r->t_submit);
    if (r->status < 0) {
      // The error is reported once; the ticket is retired.
      const int code = -r->status;
      fail(code, r->err);
      reqs_.erase(it);
      free_req(r);
      return code;
    }
    if (out) {
      out->n_edges = r->m;
      out->edge_index = r->ei;
      out->shift = r->sh;
    }
    if (!r->device_result) {
      // Host results now belong to the caller (nlb_result_free); forget the ticket.
      r->ei = nullptr;
      r->sh = nullptr;
      reqs_.erase(it);
      free_req(r);
    }
    return NLB_OK;
  }

  // Workers take no new work while paused (requests queue up; running work
  // finishes).
  void pause(bool paused) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      paused_ = paused;
    }
    cv_work_.notify_all();
  }

  // Withdraws a request: a queued one leaves the queue, a finished one has
  // its result freed; either way the ticket is retired.  A running request
  // cannot be withdrawn (NLB_ERR_VALUE, "request still running").
  int cancel(int64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return fail(NLB_ERR_VALUE, "unknown ticket").code;
    Req* r = it->second;
    if (r->status == 1) return fail(NLB_ERR_VALUE, "request still running").code;
    if (r->status == 0) {
      queue_.erase(std::find(queue_.begin(), queue_.end(), r));
      ++cancelled_;
    }
    in_use_ -= r->result_bytes;
    r->result_bytes = 0;
    reqs_.erase(it);
    free_req(r);
    cv_work_.notify_all();
    return NLB_OK;
  }

  // Failure-detection hook: the staging of any batch that holds this queued
  // request fails (as if a CUDA call of the staging had returned an error),
  // so the worker reruns the batch one request at a time and only this
  // request fails.
  int debug_fail(int64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return fail(NLB_ERR_VALUE, "unknown ticket").code;
    if (it->second->status != 0) return fail(NLB_ERR_VALUE, "request not queued").code;
    it->second->fail_staging = true;
    return NLB_OK;
  }

  int release(int64_t id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return fail(NLB_ERR_VALUE, "unknown ticket").code;
    Req* r = it->second;
    if (r->status == 0 || r->status == 1) return fail(NLB_ERR_VALUE, "request still running").code;
    in_use_ -= r->result_bytes;
    r->result_bytes = 0;
    reqs_.erase(it);
    free_req(r);
    cv_work_.notify_all();
    return NLB_OK;
  }

  // Worker wall time (microseconds, all workers) by phase of the batched
  // path: host staging and launches up to the count synchronisation, the
  // wait for the count pass, result allocation/copies issue, the wait for
  // the emit pass and copies; and the time spent in large requests.
  std::atomic<int64_t> us_stage{0}, us_count_wait{0}, us_deliver{0}, us_emit_wait{0}, us_large{0};
  static int64_t us_since(double t0) { return (int64_t)(1e6 * (now_s() - t0)); }

  void stats(int64_t* s) {
    std::lock_guard<std::mutex> lk(mu_);
    s[0] = submitted_;
    s[1] = completed_;
    s[2] = failed_;
    s[3] = batches_;
    s[4] = (int64_t)in_use_;
    s[5] = (int64_t)queue_.size();
    s[6] = max_batch_seen_;
    s[7] = (int64_t)budget_;
    s[8] = us_stage.load();
    s[9] = us_count_wait.load();
    s[10] = us_deliver.load();
    s[11] = us_emit_wait.load();
    s[12] = us_large.load();
    s[13] = cancelled_;
    s[14] = us_queue_wait_;
    s[15] = max_queued_;
  }

 private:
  // Frees a request's result arrays (a failed or retried attempt).
  void discard(Req* r) {
    if (r->dev_block) {
      bool last = false;
      {
        std::lock_guard<std::mutex> lk(dev_mu_);
        auto it = dev_refs_.find(r->dev_block);
        last = it != dev_refs_.end() && --it->second == 0;
        if (last) dev_refs_.erase(it);
      }
      if (last) cudaFreeAsync(r->dev_block, free_stream_);
      r->dev_block = nullptr;
    } else if (r->device_result) {
      if (r->ei) cudaFreeAsync(r->ei, free_stream_);
      if (r->sh) cudaFreeAsync(r->sh, free_stream_);
    } else {
      pinned_release(r->ei);
      pinned_release(r->sh);
    }
    r->ei = nullptr;
    r->sh = nullptr;
    r->m = 0;
  }

  void free_req(Req* r) {
    if (!r) return;
    pinned_release(r->pos);
    discard(r);
    delete r;
  }

  // Takes the next work item under the lock: a batch of small requests or
  // one large request, within the HBM budget.  Empty when nothing fits yet.
  std::vector<Req*> take_work() {
    std::vector<Req*> items;
    size_t result_bytes = 0;
    auto it = queue_.begin();
    while (it != queue_.end()) {
      Req* r = *it;
      const bool small = r->n <= kBatchMaxAtoms;
      const bool fits = in_use_ + r->est_bytes <= budget_;
      if (!fits) break;  // FIFO: wait for memory rather than overtake
      if (!items.empty() && result_bytes + r->est_result > kBatchResultBytes) break;
      result_bytes += r->est_result;
      if (!small) {
        if (!items.empty()) break;
        items.push_back(r);
        in_use_ += r->est_bytes;
        it = queue_.erase(it);
        break;
      }
      items.push_back(r);
      in_use_ += r->est_bytes;
      it = queue_.erase(it);
      if ((int)items.size() >= max_batch_) break;
    }
    return items;
  }

  void worker() {
    cudaSetDevice(device_);
    for (;;) {
      std::vector<Req*> items;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] {
          if (stop_) return true;
          if (paused_ || queue_.empty()) return false;
          return in_use_ + queue_.front()->est_bytes <= budget_;
        });
        if (stop_) break;
        items = take_work();
        if (items.empty()) continue;
        const double t_start = now_s();
        for (Req* r : items) {
          r->status = 1;
          us_queue_wait_ += (int64_t)(1e6 * (t_start - r->t_submit));
        }
        max_queued_ = std::max<int64_t>(max_queued_, (int64_t)queue_.size() + (int64_t)items.size());
        ++batches_;
        max_batch_seen_ = std::max<int64_t>(max_batch_seen_, (int64_t)items.size());
      }
      std::vector<Status> st(items.size(), Status{NLB_OK});
      std::vector<std::string> msg(items.size());
      if (items.size() == 1 && items[0]->n > kBatchMaxAtoms) {
        const double t0 = now_s();
        st[0] = run_large(items[0]);
        us_large += us_since(t0);
        if (!st[0].ok()) msg[0] = g_last_error;
      } else {
        const Status all = run_batch_items(items);
        if (!all.ok() && items.size() > 1) {
          // Rerun one by one so that only the offending request fails.
          for (size_t i = 0; i < items.size(); ++i) {
            discard(items[i]);
            std::vector<Req*> one(1, items[i]);
            st[i] = run_batch_items(one);
            if (!st[i].ok()) msg[i] = g_last_error;
          }
        } else if (!all.ok()) {
          st[0] = all;
          msg[0] = g_last_error;
        }
      }
      const double t = now_s();
      {
        std::lock_guard<std::mutex> lk(mu_);
        for (size_t i = 0; i < items.size(); ++i) {
          Req* r = items[i];
          in_use_ -= r->est_bytes;
          r->t_done = t;
          if (st[i].ok()) {
            r->status = 2;
            ++completed_;
            if (r->device_result) {
              r->result_bytes = (size_t)r->m * 28;
              in_use_ += r->result_bytes;
            }
          } else {
            discard(r);
            r->status = -st[i].code;
            r->err = msg[i];
            ++failed_;
          }
        }
      }
      cv_done_.notify_all();
      cv_work_.notify_all();
    }
    pinned_release(staging_);
    staging_ = nullptr;
    staging_bytes_ = 0;
    release_thread_ctx();
  }

  // Allocates the request's own result and copies its [src | dst] block
  // (2m int64, contiguous on the device) and shifts into it.
  Status deliver(Ctx& c, Req* r, const int64_t* ei, const int32_t* sh, int64_t m) {
    r->m = m;
    const size_t bi = sizeof(int64_t) * 2 * (size_t)std::max<int64_t>(m, 1);
    const size_t bs = sizeof(int32_t) * 3 * (size_t)std::max<int64_t>(m, 1);
    const cudaMemcpyKind kind = r->device_result ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (r->device_result) {
      if (cudaMallocFromPoolAsync((void**)&r->ei, bi, pool_, c.stream) != cudaSuccess ||
          cudaMallocFromPoolAsync((void**)&r->sh, bs, pool_, c.stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(NLB_ERR_NOMEM, "device allocation for a served result failed");
      }
    } else {
      r->ei = static_cast<int64_t*>(pinned_alloc(bi));
      r->sh = static_cast<int32_t*>(pinned_alloc(bs));
      if (!r->ei || !r->sh) return fail(NLB_ERR_NOMEM, "pinned host allocation failed");
    }
    if (m == 0) return Status{NLB_OK};
    cudaError_t e = cudaMemcpyAsync(r->ei, ei, 16 * (size_t)m, kind, c.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r->sh, sh, 12 * (size_t)m, kind, c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "result copy");
    return Status{NLB_OK};
  }

  Status run_large(Req* r) {
    if (r->fail_staging) return fail(NLB_ERR_CUDA, "request staging failed (injected)");
    Ctx* c = nullptr;
    Status st = get_ctx(&c);
    if (!st.ok()) return st;
    double* d_pos = nullptr;
    st = upload_positions(*c, r->pos, r->n, &d_pos);
    if (!st.ok()) return st;
    SystemPlan sp;
    const bool pb[3] = {r->pbc[0] != 0, r->pbc[1] != 0, r->pbc[2] != 0};
    st = plan_system(r->pos, r->n, r->has_cell ? r->h : nullptr, pb, std::vector<double>(1, r->rc),
                     false, false, sp);
    if (!st.ok()) return st;
    if (fast_eligible(sp)) {
      int64_t m = 0;
      st = run_fast(*c, sp, d_pos, &m);
      if (!st.ok()) return st;
      st = deliver(*c, r, sp.out_src, sp.out_sh, m);
    } else {
      st = count_system(*c, sp, d_pos);
      if (!st.ok()) return st;
      DevLists L;
      L.src.resize(1);
      L.dst.resize(1);
      L.sh.resize(1);
      const int64_t m = sp.m[0];
      int64_t* a = slot<int64_t>(*c, kSlotOutEi, 2 * (size_t)std::max<int64_t>(m, 1));
      int32_t* b = slot<int32_t>(*c, kSlotOutSh, 3 * (size_t)std::max<int64_t>(m, 1));
      if (!a || !b) return fail(NLB_ERR_NOMEM, "device allocation failed");
      L.src[0] = a;
      L.dst[0] = a + m;
      L.sh[0] = b;
      const int64_t zero = 0;
      st = emit_system(*c, sp, d_pos, L, &zero, 0);
      if (!st.ok()) return st;
      st = deliver(*c, r, a, b, m);
    }
    if (!st.ok()) return st;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "served request");
    return Status{NLB_OK};
  }

  Status run_batch_items(std::vector<Req*>& items) {
    for (Req* r : items)
      if (r->fail_staging) return fail(NLB_ERR_CUDA, "batch staging failed (injected)");
    Ctx* c = nullptr;
    Status st = get_ctx(&c);
    if (!st.ok()) return st;
    // Zero-atom requests have no edges; the batched kernels take the rest.
    std::vector<Req*> work;
    for (Req* r : items) {
      if (r->n > 0) {
        work.push_back(r);
        continue;
      }
      st = deliver(*c, r, nullptr, nullptr, 0);
      if (!st.ok()) return st;
    }
    if (work.empty()) return Status{NLB_OK};
    return run_batch_nonempty(*c, work);
  }

  Status run_batch_nonempty(Ctx& cref, std::vector<Req*>& items) {
    double t_mark = now_s();
    Ctx* c = &cref;
    Status st{NLB_OK};
    cudaStream_t s = c->stream;
    const int32_t ns = (int32_t)items.size();
    std::vector<int64_t> starts(ns + 1, 0);
    for (int32_t i = 0; i < ns; ++i) starts[i + 1] = starts[i] + items[i]->n;
    const int64_t total_atoms = starts[ns];
    // Host staging (pinned, per worker) of positions and per-system tables.
    const size_t bytes_pos = sizeof(double) * 3 * (size_t)std::max<int64_t>(total_atoms, 1);
    const size_t bytes_tab =
        ((sizeof(int64_t) + 9 * sizeof(double) + 3 + 1 + sizeof(double)) * (size_t)(ns + 1) + 63) &
        ~(size_t)63;
    const size_t bytes_back = sizeof(int64_t) * (size_t)(ns + 4);
    if (staging_bytes_ < bytes_pos + bytes_tab + bytes_back) {
      pinned_release(staging_);
      staging_bytes_ = (bytes_pos + bytes_tab + bytes_back) * 2;
      staging_ = static_cast<unsigned char*>(pinned_alloc(staging_bytes_));
      if (!staging_) {
        staging_bytes_ = 0;
        return fail(NLB_ERR_NOMEM, "pinned host allocation failed");
      }
    }
    // Each worker thread owns its staging buffer (thread_local members).
    double* h_pos = reinterpret_cast<double*>(staging_);
    int64_t* h_starts = reinterpret_cast<int64_t*>(staging_ + bytes_pos);
    double* h_cells = reinterpret_cast<double*>(h_starts + ns + 1);
    double* h_rc = h_cells + 9 * (size_t)ns;
    uint8_t* h_pbc = reinterpret_cast<uint8_t*>(h_rc + ns);
    uint8_t* h_has = h_pbc + 3 * (size_t)ns;
    for (int32_t i = 0; i < ns; ++i) {
      Req* r = items[i];
      if (r->n) std::memcpy(h_pos + 3 * starts[i], r->pos, sizeof(double) * 3 * (size_t)r->n);
      h_starts[i] = starts[i];
      std::memcpy(h_cells + 9 * (size_t)i, r->h, 9 * sizeof(double));
      h_rc[i] = r->rc;
      for (int a = 0; a < 3; ++a) h_pbc[3 * i + a] = r->pbc[a];
      h_has[i] = r->has_cell ? 1 : 0;
    }
    h_starts[ns] = total_atoms;
    // Device copies.
    double* d_pos = slot<double>(*c, kSlotPos, 3 * (size_t)std::max<int64_t>(total_atoms, 1));
    unsigned char* d_tab = slot<unsigned char>(*c, kSlotBatch0 + 10, bytes_tab + 64);
    if (!d_pos || !d_tab) return fail(NLB_ERR_NOMEM, "device allocation failed");
    int64_t* d_starts = reinterpret_cast<int64_t*>(d_tab);
    double* d_cells = reinterpret_cast<double*>(d_starts + ns + 1);
    double* d_rc = d_cells + 9 * (size_t)ns;
    uint8_t* d_pbc = reinterpret_cast<uint8_t*>(d_rc + ns);
    uint8_t* d_has = d_pbc + 3 * (size_t)ns;
    cudaMemcpyAsync(d_pos, h_pos, sizeof(double) * 3 * (size_t)total_atoms, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_tab, h_starts, bytes_tab, cudaMemcpyHostToDevice, s);

    const int64_t row = total_atoms + 1;
    std::vector<int64_t> sizes(ns);
    double rc_max = 0.0;
    for (int32_t i = 0; i < ns; ++i) {
      sizes[i] = items[i]->n;
      rc_max = std::max(rc_max, items[i]->rc);
    }
    // (every candidate launch shape when this kind of batch is new)
    ShapeTrials trials;
    st = trials.prepare(*c, make_tune_key(c->device, 0, sizes.data(), ns, rc_max), sizes.data(),
                        ns, kSlotBatch0 + 1);
    if (!st.ok()) return st;
    SysPlan* plans = slot<SysPlan>(*c, kSlotBatch0 + 0, ns);
    int32_t* flags = slot<int32_t>(*c, kSlotBatch0 + 2, 3);
    uint32_t* counts = slot<uint32_t>(*c, kSlotBatch0 + 3, row);
    int64_t* offs = slot<int64_t>(*c, kSlotBatch0 + 4, row + 1);
    int64_t* scan_tmp = slot<int64_t>(*c, kSlotBatch0 + 5, scan_tmp_elems(row));
    int64_t* bounds = slot<int64_t>(*c, kSlotBatch0 + 11, ns + 1);
    if (!plans || !flags || !counts || !offs || !scan_tmp || !bounds)
      return fail(NLB_ERR_NOMEM, "device allocation failed");
    // Hit records for the expansion pass (a kind whose launch shape is
    // decided: one count pass), sized by the admission estimates; a batch
    // whose records do not fit recomputes in its emit pass instead.
    BatchRecords rb;
    std::memset(&rb, 0, sizeof(rb));
    const bool use_rec = !trials.timed;
    int32_t* rec_flags = nullptr;
    if (use_rec) {
      size_t est_edges = 0;
      for (Req* r : items) est_edges += r->est_result / 28;
      const int64_t segs = total_atoms + (int64_t)(est_edges / 32) + 1024;
      rb.seg_cap = (int)std::min<int64_t>(segs, INT32_MAX / 2);
      rb.seg_hdr = slot<int4>(*c, kSlotBatch0 + 13, (size_t)rb.seg_cap);
      rb.rec = slot<uint32_t>(*c, kSlotBatch0 + 14, (size_t)rb.seg_cap * 96);
      rb.meta = slot<SlotMeta>(*c, kSlotBatch0 + 15, (size_t)std::max<int64_t>(total_atoms, 1));
      rec_flags = slot<int32_t>(*c, kSlotBatch0 + 12, 3);
      if (!rb.seg_hdr || !rb.rec || !rb.meta || !rec_flags)
        return fail(NLB_ERR_NOMEM, "device allocation failed");
      rb.seg_top = rec_flags;
      rb.overflow = rec_flags + 1;
      rb.need_recompute = rec_flags + 2;
      cudaMemsetAsync(rec_flags, 0, sizeof(int32_t) * 3, s);
    }
    cudaMemsetAsync(flags, 0, sizeof(int32_t) * 3, s);
    cudaMemsetAsync(counts, 0, sizeof(uint32_t) * row, s);
    launch_plan(d_pos, d_starts, 0, ns, d_cells, d_pbc, d_has, 0.0, g_bf_threshold.load(), 0, 0,
                plans, flags, s, d_rc);
    CutoffSet cs;
    std::memset(&cs, 0, sizeof(cs));
    cs.k = 0;  // per-system cutoffs
    // (The counts are the same in every shape: each trial writes all of them.)
    for (size_t t = 0; t < trials.w.size(); ++t) {
      trials.mark(*c, t);
      if (t > 0) cudaMemsetAsync(flags + 1, 0, sizeof(int32_t) * 2, s);
      launch_batch_count(plans, trials.w[t], d_pos, cs, counts, row, flags + 1, s,
                         use_rec ? &rb : nullptr);
    }
    trials.mark(*c, trials.w.size());
    exclusive_scan_u32(counts, row, offs, scan_tmp, s);
    launch_sys_bounds(plans, ns, offs, row, bounds, s);
    // System bounds, the plan error word and the scan's bounded-wait error
    // word come back in the pinned staging area behind the tables.
    int64_t* hb = reinterpret_cast<int64_t*>(staging_ + bytes_pos + bytes_tab);
    int64_t* diag = hb + ns + 1;
    diag[0] = 0;
    diag[2] = 0;
    cudaError_t e = cudaMemcpyAsync(hb, bounds, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&diag[0], flags, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&diag[1], scan_tmp + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && use_rec)  // records complete?
      e = cudaMemcpyAsync(&diag[2], rb.overflow, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    us_stage += us_since(t_mark);
    t_mark = now_s();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    us_count_wait += us_since(t_mark);
    t_mark = now_s();
    if (e != cudaSuccess) return cuda_fail(e, "served batch count");
    const int32_t plan_err = (int32_t)(diag[0] & 0xffffffff);
    if (plan_err == 1) return fail(NLB_ERR_VALUE, "Cell matrix is not invertible");
    if (plan_err == 2) return fail(NLB_ERR_VALUE, "stencil too large for this cutoff and cell");
    if (diag[1] != 0) return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
    const int64_t m_total = hb[ns];
    // Device-resident results of the batch are slices of one block from the
    // server's pool that the emit pass writes directly; otherwise the edges
    // go to this worker's workspace and only come back to the host.
    bool any_dev = false;
    for (int32_t i = 0; i < ns; ++i) any_dev |= items[i]->device_result && hb[i + 1] > hb[i];
    void* dev_block = nullptr;
    int64_t* src = nullptr;
    int32_t* shf = nullptr;
    if (any_dev) {
      if (cudaMallocFromPoolAsync(&dev_block, 28 * (size_t)m_total, pool_, s) != cudaSuccess) {
        cudaGetLastError();
        return fail(NLB_ERR_NOMEM, "device allocation for served results failed");
      }
      src = static_cast<int64_t*>(dev_block);
      shf = reinterpret_cast<int32_t*>(src + 2 * m_total);
    } else {
      src = slot<int64_t>(*c, kSlotOutEi, 2 * (size_t)std::max<int64_t>(m_total, 1));
      shf = slot<int32_t>(*c, kSlotOutSh, 3 * (size_t)std::max<int64_t>(m_total, 1));
      if (!src || !shf) return fail(NLB_ERR_NOMEM, "device allocation for the edge lists failed");
    }
    EmitTargets t;
    std::memset(&t, 0, sizeof(t));
    t.src[0] = src;
    t.dst[0] = src + m_total;  // unused with system_blocks
    t.sh[0] = shf;
    t.local_indices = 1;
    t.system_blocks = 1;  // request i: [src | dst] at src + 2 hb[i]
    if (use_rec && (diag[2] & 0xffffffff) == 0) {
      launch_batch_expand(rb, plans, d_pos, offs, row, t, s);
    } else {
      cudaMemsetAsync(flags + 1, 0, sizeof(int32_t) * 2, s);
      launch_batch_emit(plans, trials.pick(*c), d_pos, cs, offs, row, t, flags + 1, s);
    }
    // Host results of the batch come back in two copies into shared pinned
    // blocks, each request holding slices of them.
    bool any_host = false;
    for (Req* r : items) any_host |= !r->device_result && r->n > 0;
    int64_t* blk_ei = nullptr;
    int32_t* blk_sh = nullptr;
    if (any_host && m_total > 0) {
      blk_ei = static_cast<int64_t*>(pinned_alloc(block_class(16 * (size_t)m_total)));
      blk_sh = static_cast<int32_t*>(pinned_alloc(block_class(12 * (size_t)m_total)));
      if (!blk_ei || !blk_sh) {
        pinned_release(blk_ei);
        pinned_release(blk_sh);
        return fail(NLB_ERR_NOMEM, "pinned host allocation failed");
      }
      e = cudaMemcpyAsync(blk_ei, src, 16 * (size_t)m_total, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(blk_sh, shf, 12 * (size_t)m_total, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) {
        pinned_release(blk_ei);
        pinned_release(blk_sh);
        if (dev_block) cudaFreeAsync(dev_block, s);
        return cuda_fail(e, "result copy");
      }
    }
    int shared = 0, dev_shared = 0;
    for (int32_t i = 0; i < ns && st.ok(); ++i) {
      Req* r = items[i];
      const int64_t b0 = hb[i], m = hb[i + 1] - hb[i];
      if (m == 0) {
        st = deliver(*c, r, src + 2 * b0, shf + 3 * b0, m);
        continue;
      }
      r->m = m;
      r->ei = (r->device_result ? src : blk_ei) + 2 * b0;
      r->sh = (r->device_result ? shf : blk_sh) + 3 * b0;
      if (r->device_result) {
        r->dev_block = dev_block;
        ++dev_shared;
      } else {
        pinned_share(blk_ei, r->ei);
        pinned_share(blk_sh, r->sh);
        ++shared;
      }
    }
    if (!shared) {
      pinned_release(blk_ei);
      pinned_release(blk_sh);
    }
    if (dev_block) {
      if (dev_shared) {
        std::lock_guard<std::mutex> lk(dev_mu_);
        dev_refs_[dev_block] = dev_shared;
      } else {
        cudaFreeAsync(dev_block, s);
      }
    }
    if (!st.ok()) return st;
    us_deliver += us_since(t_mark);
    t_mark = now_s();
    e = cudaStreamSynchronize(s);
    us_emit_wait += us_since(t_mark);
    if (e != cudaSuccess) return cuda_fail(e, "served batch emit");
    return Status{NLB_OK};
  }

  int device_;
  cudaMemPool_t pool_ = nullptr;
  std::mutex dev_mu_;
  std::unordered_map<void*, int64_t> dev_refs_;  // device block -> live result slices
  cudaStream_t free_stream_ = nullptr;
  size_t budget_;
  int max_batch_;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<Req*> queue_;
  std::unordered_map<int64_t, Req*> reqs_;
  size_t in_use_ = 0;
  bool stop_ = false;
  bool paused_ = false;
  int64_t cancelled_ = 0;
  int64_t us_queue_wait_ = 0;  // sum over started requests of submit -> start (admission wait)
  int64_t max_queued_ = 0;     // deepest queue seen when work was taken
  int64_t next_id_ = 1;
  int64_t submitted_ = 0, completed_ = 0, failed_ = 0, batches_ = 0, max_batch_seen_ = 0;
  std::vector<std::thread> threads_;
  static thread_local unsigned char* staging_;
  static thread_local size_t staging_bytes_;
};

thread_local unsigned char* Server::staging_ = nullptr;
thread_local size_t Server::staging_bytes_ = 0;

}  // namespace nlb

using nlb::Server;

extern "C" {

struct nlb_server {
  Server* impl;
};

nlb_server* nlb_server_create(int device, int64_t hbm_budget_bytes, int n_workers, int max_batch) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    nlb::fail(NLB_ERR_CUDA, "no such CUDA device");
    return nullptr;
  }
  if (hbm_budget_bytes <= 0) {
    nlb::fail(NLB_ERR_VALUE, "the HBM budget must be positive");
    return nullptr;
  }
  Server* impl = new Server(device, (size_t)hbm_budget_bytes, n_workers, max_batch);
  if (!impl->init_device_pool()) {
    const std::string msg = nlb::g_last_error;
    delete impl;
    nlb::fail(NLB_ERR_CUDA, msg);
    return nullptr;
  }
  nlb_server* s = new nlb_server();
  s->impl = impl;
  return s;
}

int64_t nlb_server_submit(nlb_server* s, const double* positions, int64_t n_atoms,
                          const double* cell, const uint8_t* pbc, double cutoff,
                          int device_result) {
  if (!s) return -nlb::fail(NLB_ERR_VALUE, "server is NULL").code;
  return s->impl->submit(positions, n_atoms, cell, pbc, cutoff, device_result != 0);
}

int nlb_server_wait(nlb_server* s, int64_t ticket, double timeout_s, nlb_result* out,
                    double* latency_ms) {
  if (!s) return nlb::fail(NLB_ERR_VALUE, "server is NULL").code;
  return s->impl->wait(ticket, timeout_s, out, latency_ms);
}

int nlb_server_release(nlb_server* s, int64_t ticket) {
  if (!s) return nlb::fail(NLB_ERR_VALUE, "server is NULL").code;
  return s->impl->release(ticket);
}

int nlb_server_pause(nlb_server* s, int paused) {
  if (!s) return nlb::fail(NLB_ERR_VALUE, "server is NULL").code;
  s->impl->pause(paused != 0);
  return NLB_OK;
}

int nlb_server_cancel(nlb_server* s, int64_t ticket) {
  if (!s) return nlb::fail(NLB_ERR_VALUE, "server is NULL").code;
  return s->impl->cancel(ticket);
}

int nlb_server_debug_fail(nlb_server* s, int64_t ticket) {
  if (!s) return nlb::fail(NLB_ERR_VALUE, "server is NULL").code;
  return s->impl->debug_fail(ticket);
}

void nlb_server_stats(nlb_server* s, int64_t* stats) {
  if (s && stats) s->impl->stats(stats);
}

void nlb_server_destroy(nlb_server* s) {
  if (!s) return;
  delete s->impl;
  delete s;
}

}  // extern "C"
