// nlb_tune.cpp -- launch-shape tuner for the batched kernels.
//
// The batched kernels (k_batch.cu) can run a batch in any of the launch
// shapes of kBatchShapeTable (CTA sizes, atoms per work item, the size above
// which a system is split), all with identical results.  Which shape is
// fastest depends on the batch: many tiny systems want more systems in flight
// per SM, a few mid-size ones want finer work items.  The tuner keys batches
// by kind (TuneKey) and decides each kind on its first batch:
//
//   * the candidates of a kind are the shapes that launch differently for
//     its largest system (shapes that split none of its systems differ only
//     in their CTA size for whole systems);
//   * the first batch of a kind runs its count pass once per candidate, back
//     to back on the stream with a CUDA event between the launches (counts
//     are the same in every shape, so running the pass again is harmless);
//     the host reads the events after the synchronisation the count pass
//     needs anyway, and the kind keeps the fastest shape for the rest of the
//     process -- its emit pass, which walks the same pairs, and every later
//     batch of the kind use it.
//
// A new kind therefore costs a few extra count passes once, and a batch of a
// known kind nothing.  Every kernel variant is loaded before the first timed
// launch, so no candidate pays for loading a module.  NLB_BATCH_SHAPE=i in
// the environment, or nlb_batch_shape(i), pins shape i for every batch.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "nlb_internal.h"

namespace nlb {

namespace {

struct TuneEntry {
  int32_t n_cand = 0;
  int32_t cand[kBatchShapes] = {};  // candidate shape indices
  int32_t best = -1;                // -1: not decided yet
  float ms[kBatchShapes] = {};      // count-pass time of each candidate
};

// One shape per distinct launch for batches whose largest system has at most
// max_atoms atoms.
void set_candidates(int64_t max_atoms, TuneEntry& e) {
  int32_t sig[kBatchShapes][4];
  e.n_cand = 0;
  for (int32_t i = 0; i < kBatchShapes; ++i) {
    const BatchShape& s = kBatchShapeTable[i];
    const bool split = max_atoms > s.large_atoms;
    const int32_t me[4] = {s.small_threads, split ? s.large_threads : 0, split ? s.chunk : 0,
                           split ? s.large_atoms : 0};
    bool seen = false;
    for (int32_t j = 0; j < e.n_cand && !seen; ++j)
      seen = std::equal(me, me + 4, sig[j]);
    if (seen) continue;
    std::copy(me, me + 4, sig[e.n_cand]);
    e.cand[e.n_cand++] = i;
  }
  if (e.n_cand == 1) e.best = e.cand[0];
}

// Devices whose kernel variants are loaded (under g_preload_mu, so that no
// thread times a candidate while another is still loading them).
std::mutex g_preload_mu;
bool g_preloaded[16] = {};

std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;

int32_t initial_pin() {
  const char* v = std::getenv("NLB_BATCH_SHAPE");
  if (!v || !*v) return -1;
  const int i = std::atoi(v);
  return i >= 0 && i < kBatchShapes ? i : -1;
}
int32_t g_pinned = initial_pin();

int32_t log2_bucket(int64_t v) {
  int32_t b = 0;
  while (v > 1) {
    v >>= 1;
    ++b;
  }
  return b;
}

}  // namespace

bool TuneKey::operator<(const TuneKey& o) const {
  return std::tie(device, k, n_sys_log2, max_log2, mean_log2, rc_bucket) <
         std::tie(o.device, o.k, o.n_sys_log2, o.max_log2, o.mean_log2, o.rc_bucket);
}

TuneKey make_tune_key(int32_t device, int32_t k, const int64_t* sizes, int32_t n_sys,
                      double rc_max) {
  TuneKey key;
  int64_t mx = 0, total = 0;
  for (int32_t i = 0; i < n_sys; ++i) {
    mx = std::max(mx, sizes[i]);
    total += sizes[i];
  }
  key.device = device;
  key.k = k;
  key.n_sys_log2 = log2_bucket(n_sys);
  key.max_log2 = log2_bucket(mx);
  key.mean_log2 = log2_bucket(n_sys > 0 ? total / n_sys : 0);
  key.rc_bucket = rc_max > 0.0 && std::isfinite(rc_max) ? (int32_t)std::floor(4.0 * std::log2(rc_max))
                                                         : 0;
  return key;
}

Status ShapeTrials::prepare(Ctx& c, const TuneKey& k, const int64_t* sizes, int32_t n_sys,
                           int items_slot) {
  key = k;
  shapes.clear();
  timed = false;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_pinned >= 0) {
      shapes.push_back(g_pinned);
    } else {
      auto it = g_tune.find(key);
      if (it == g_tune.end()) {
        it = g_tune.emplace(key, TuneEntry()).first;
        set_candidates(((int64_t)2 << key.max_log2) - 1, it->second);
      }
      const TuneEntry& e = it->second;
      if (e.best >= 0 || c.prof)  // (phase profiling owns the stream's event timeline)
        shapes.push_back(e.best >= 0 ? e.best : e.cand[0]);
      else
        shapes.assign(e.cand, e.cand + e.n_cand);
    }
  }
  timed = shapes.size() > 1;
  if (timed) {
    if (c.device >= 0 && c.device < 16) {
      std::lock_guard<std::mutex> lk(g_preload_mu);
      if (!g_preloaded[c.device]) {
        preload_batch_kernels();
        g_preloaded[c.device] = true;
      }
    }
    for (cudaEvent_t& ev : c.tune_ev)
      if (!ev && cudaEventCreate(&ev) != cudaSuccess) {
        cudaGetLastError();
        ev = nullptr;
        timed = false;
      }
    if (!timed) shapes.resize(1);
  }
  // Every trial's work items in one upload.
  w.assign(shapes.size(), BatchItems());
  std::vector<int2> all, one;
  std::vector<size_t> off(shapes.size());
  for (size_t i = 0; i < shapes.size(); ++i) {
    plan_batch_items(sizes, n_sys, kBatchShapeTable[shapes[i]], one, w[i]);
    off[i] = all.size();
    all.insert(all.end(), one.begin(), one.end());
  }
  int2* d = slot<int2>(c, items_slot, std::max<size_t>(all.size(), 1));
  if (!d) return fail(NLB_ERR_NOMEM, "device allocation failed");
  if (!all.empty())
    cudaMemcpyAsync(d, all.data(), sizeof(int2) * all.size(), cudaMemcpyHostToDevice, c.stream);
  for (size_t i = 0; i < shapes.size(); ++i) w[i].items = d + off[i];
  return Status{NLB_OK};
}

void ShapeTrials::mark(Ctx& c, size_t i) {
  if (timed && i <= shapes.size()) cudaEventRecord(c.tune_ev[i], c.stream);
}

const BatchItems& ShapeTrials::pick(Ctx& c) {
  if (!timed) return w[0];
  size_t best = 0;
  float best_ms = 0.0f;
  float ms[kBatchShapes] = {};
  bool ok = true;
  for (size_t i = 0; i < shapes.size() && ok; ++i) {
    ok = cudaEventElapsedTime(&ms[i], c.tune_ev[i], c.tune_ev[i + 1]) == cudaSuccess;
    if (ok && (i == 0 || ms[i] < best_ms)) {
      best = i;
      best_ms = ms[i];
    }
  }
  if (!ok) {
    cudaGetLastError();
    return w[0];
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(key);  // (gone after a concurrent reset)
  if (it != g_tune.end() && it->second.best < 0) {
    it->second.best = shapes[best];
    for (size_t i = 0; i < shapes.size(); ++i) it->second.ms[shapes[i]] = ms[i];
  }
  return w[best];
}

void tune_release(Ctx& c) {
  for (cudaEvent_t& ev : c.tune_ev) {
    if (ev) cudaEventDestroy(ev);
    ev = nullptr;
  }
}

}  // namespace nlb

using namespace nlb;

extern "C" {

int32_t nlb_batch_shape(int32_t shape) {
  if (shape < -1 || shape >= kBatchShapes) return -1;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_pinned = shape;
  return kBatchShapes;
}

int32_t nlb_batch_shape_info(int32_t shape, int32_t* out4) {
  if (shape < 0 || shape >= kBatchShapes || !out4) return -1;
  const BatchShape& s = kBatchShapeTable[shape];
  out4[0] = s.small_threads;
  out4[1] = s.large_threads;
  out4[2] = s.chunk;
  out4[3] = s.large_atoms;
  return 0;
}

int32_t nlb_batch_tuner_state(int64_t* out, int32_t cap) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  int32_t i = 0;
  for (const auto& kv : g_tune) {
    if (out && i < cap) {
      int64_t* r = out + 8 * (size_t)i;
      const TuneKey& k = kv.first;
      r[0] = k.device;
      r[1] = k.k;
      r[2] = k.n_sys_log2;
      r[3] = k.max_log2;
      r[4] = k.mean_log2;
      r[5] = k.rc_bucket;
      r[6] = kv.second.best;
      r[7] = kv.second.n_cand;
    }
    ++i;
  }
  return i;
}

void nlb_batch_tuner_reset(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
}

}  // extern "C"
