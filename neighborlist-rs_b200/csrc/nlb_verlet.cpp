// nlb_verlet.cpp -- Verlet (skin) list manager for MD-style callers.
//
// The reference's specification asks for it (spec.md:41-48, 64-67, 209-222:
// r_list = r_cut + r_skin, reference positions, rebuild when
// max_i |r_i - r_i,ref| > r_skin / 2, update / needs_rebuild / get); the
// reference does not implement it.  Each update:
//   1. if a list exists for the same atom count, cell and pbc, one kernel
//      takes the largest displacement since the last rebuild (one sync);
//   2. if there is no list, the system changed, or that displacement is
//      above skin / 2: rebuild -- the exact half list at rc + skin (the same
//      search as nlb_build), kept in the manager's device buffers, and the
//      current positions become the reference;
//   3. filter the stored list with the current positions at rc (keep flags,
//      one scan, compaction in stored order; one sync for the total).
// As long as no atom moved more than skin / 2, every pair now closer than rc
// was closer than rc + skin at the rebuild, so the filtered list holds
// exactly the pairs (i, j, S) with |(r_j - r_i) + H.S| < rc -- the set a
// fresh build at rc would give (pairs within rounding of rc aside), in the
// stored order.  Positions are taken as continuous trajectories: re-wrapping
// an atom into the box moves it by a lattice vector and forces a rebuild.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "nlb_internal.h"

namespace nlb {

// Polls of one look-back wait in the Verlet compaction before it gives up.
constexpr int32_t kVerletSpinLimit = 1 << 22;

// Search pieces shared with nlb_api.cpp.
Status half_list_device(Ctx& c, const double* pos_host, const double* d_pos, int64_t n,
                        const double* cell9, const uint8_t* pbc, double cutoff, int64_t** ei,
                        int32_t** sh, int64_t* m);

namespace {

// Grow-only device buffer owned by one manager (contents not kept on growth).
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  void* get(size_t bytes) {
    bytes = bytes ? bytes : 16;
    if (bytes > cap) {
      if (p) cudaFree(p);
      p = nullptr;
      cap = 0;
      if (cudaMalloc(&p, bytes + bytes / 4) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
      }
      cap = bytes + bytes / 4;
    }
    return p;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

class Verlet {
 public:
  Verlet(double rc, double skin) : rc_(rc), skin_(skin) {}

  // Device positions (d_pos) are used in place; host positions are uploaded
  // first.  Results stay in the manager's buffers until the next update.
  Status update(const double* pos_host, const double* d_pos_in, int64_t n, const double* cell9,
                const uint8_t* pbc, int* rebuilt, int64_t* m_out, int64_t** ei_out,
                int32_t** sh_out, bool owned = false) {
    std::lock_guard<std::mutex> lk(mu_);
    *rebuilt = 0;
    *m_out = 0;
    *ei_out = nullptr;
    *sh_out = nullptr;
    if (n < 0) return fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
    if (n > 0 && !pos_host && !d_pos_in) return fail(NLB_ERR_VALUE, "positions is NULL");
    Ctx* c = nullptr;
    Status st = get_ctx(&c);
    if (!st.ok()) return st;
    cudaStream_t s = c->stream;
    const double* d_pos = d_pos_in;
    if (n > 0 && pos_host) {
      double* up = static_cast<double*>(pos_up_.get(24 * (size_t)n));
      if (!up) return fail(NLB_ERR_NOMEM, "device allocation failed");
      cudaError_t e = cudaMemcpyAsync(up, pos_host, 24 * (size_t)n, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (positions)");
      d_pos = up;
    }
    ++updates_;
    bool rebuild = !same_system(n, cell9, pbc);
    if (!rebuild && n > 0) {
      // The displacement check and the filter of the stored list go out
      // together (the filter only reads the positions and the list) and one
      // synchronisation reads both; a rebuild, when due, discards the filter.
      auto* d = static_cast<unsigned long long*>(disp_.get(sizeof(unsigned long long)));
      if (!d) return fail(NLB_ERR_NOMEM, "device allocation failed");
      launch_max_disp(d_pos, static_cast<const double*>(ref_.p), n, d, s);
      cudaError_t e = cudaMemcpyAsync(c->h_small + 2, d, sizeof(unsigned long long),
                                      cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) return cuda_fail(e, "displacement check");
      st = filter(*c, d_pos, m_out, ei_out, sh_out, owned);
      if (!st.ok()) return st;
      if (m_list_ == 0) {  // (the filter had nothing to do and did not synchronise)
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "displacement check");
      }
      double d2 = 0.0;
      std::memcpy(&d2, c->h_small + 2, sizeof(double));
      last_disp_ = std::sqrt(d2);
      rebuild = last_disp_ > 0.5 * skin_;
      if (!rebuild) return Status{NLB_OK};
      if (owned) {
        release_owned_device(*ei_out, s);
        release_owned_device(*sh_out, s);
      }
      *m_out = 0;
      *ei_out = nullptr;
      *sh_out = nullptr;
    }
    if (rebuild) {
      st = rebuild_list(*c, pos_host, d_pos, n, cell9, pbc);
      if (!st.ok()) {
        have_ = false;
        return st;
      }
      *rebuilt = 1;
      ++rebuilds_;
    }
    return filter(*c, d_pos, m_out, ei_out, sh_out, owned);
  }

  // Largest displacement since the last rebuild (+inf when there is no list
  // for this atom count, cell and pbc); *needs = it exceeds skin / 2.
  Status needs_rebuild(const double* pos_host, const double* d_pos_in, int64_t n,
                       const double* cell9, const uint8_t* pbc, int* needs, double* disp) {
    std::lock_guard<std::mutex> lk(mu_);
    *needs = 1;
    *disp = INFINITY;
    if (n < 0) return fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
    if (!same_system(n, cell9, pbc)) return Status{NLB_OK};
    if (n == 0) {
      *needs = 0;
      *disp = 0.0;
      return Status{NLB_OK};
    }
    if (!pos_host && !d_pos_in) return fail(NLB_ERR_VALUE, "positions is NULL");
    Ctx* c = nullptr;
    Status st = get_ctx(&c);
    if (!st.ok()) return st;
    const double* d_pos = d_pos_in;
    if (pos_host) {
      double* up = static_cast<double*>(pos_up_.get(24 * (size_t)n));
      if (!up) return fail(NLB_ERR_NOMEM, "device allocation failed");
      cudaError_t e =
          cudaMemcpyAsync(up, pos_host, 24 * (size_t)n, cudaMemcpyHostToDevice, c->stream);
      if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (positions)");
      d_pos = up;
    }
    double d2 = 0.0;
    st = max_disp_sq(*c, d_pos, n, &d2);
    if (!st.ok()) return st;
    *disp = std::sqrt(d2);
    *needs = *disp > 0.5 * skin_ ? 1 : 0;
    return Status{NLB_OK};
  }

  void stats(int64_t* out) {
    std::lock_guard<std::mutex> lk(mu_);
    out[0] = updates_;
    out[1] = rebuilds_;
    out[2] = m_list_;
    out[3] = m_last_;
  }

  double cutoff() const { return rc_; }
  double skin() const { return skin_; }

 private:
  bool same_system(int64_t n, const double* cell9, const uint8_t* pbc) const {
    if (!have_ || n != n_ || (cell9 != nullptr) != has_cell_) return false;
    if (cell9) {
      for (int k = 0; k < 9; ++k)
        if (!(cell9[k] == h_[k])) return false;
    }
    for (int a = 0; a < 3; ++a)
      if ((pbc ? pbc[a] != 0 : true) != (pbc_[a] != 0)) return false;
    return true;
  }

  Status max_disp_sq(Ctx& c, const double* d_pos, int64_t n, double* d2) {
    auto* d = static_cast<unsigned long long*>(disp_.get(sizeof(unsigned long long)));
    if (!d) return fail(NLB_ERR_NOMEM, "device allocation failed");
    launch_max_disp(d_pos, static_cast<const double*>(ref_.p), n, d, c.stream);
    cudaError_t e = cudaMemcpyAsync(c.h_small, d, sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "displacement check");
    std::memcpy(d2, c.h_small, sizeof(double));
    return Status{NLB_OK};
  }

  Status rebuild_list(Ctx& c, const double* pos_host, const double* d_pos, int64_t n,
                      const double* cell9, const uint8_t* pbc) {
    int64_t* ei = nullptr;
    int32_t* sh = nullptr;
    int64_t m = 0;
    if (n > 0) {
      Status st = half_list_device(c, pos_host, d_pos, n, cell9, pbc, rc_ + skin_, &ei, &sh, &m);
      if (!st.ok()) return st;
    }
    int64_t* vei = static_cast<int64_t*>(list_ei_.get(16 * (size_t)m));
    int32_t* vsh = static_cast<int32_t*>(list_sh_.get(12 * (size_t)m));
    double* ref = static_cast<double*>(ref_.get(24 * (size_t)n));
    if (!vei || !vsh || !ref) return fail(NLB_ERR_NOMEM, "device allocation failed");
    cudaError_t e = cudaSuccess;
    if (m > 0) {
      e = cudaMemcpyAsync(vei, ei, 16 * (size_t)m, cudaMemcpyDeviceToDevice, c.stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(vsh, sh, 12 * (size_t)m, cudaMemcpyDeviceToDevice, c.stream);
    }
    if (e == cudaSuccess && n > 0)
      e = cudaMemcpyAsync(ref, d_pos, 24 * (size_t)n, cudaMemcpyDeviceToDevice, c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (Verlet list)");
    m_list_ = m;
    n_ = n;
    has_cell_ = cell9 != nullptr;
    std::memset(h_, 0, sizeof(h_));
    if (cell9) std::memcpy(h_, cell9, sizeof(h_));
    for (int a = 0; a < 3; ++a) pbc_[a] = pbc ? (pbc[a] != 0) : 1;
    have_ = true;
    last_disp_ = 0.0;
    return Status{NLB_OK};
  }

  // owned: the kept edges go to blocks of the result pool sized for the
  // whole stored list, handed to the caller (released again on failure).
  Status filter(Ctx& c, const double* d_pos, int64_t* m_out, int64_t** ei_out,
                int32_t** sh_out, bool owned = false) {
    const int64_t m = m_list_;
    int64_t* out_ei = nullptr;
    int32_t* out_sh = nullptr;
    if (owned) {
      if (m > 0) {
        out_ei = static_cast<int64_t*>(alloc_owned_device(c.device, 16 * (size_t)m, c.stream));
        out_sh = static_cast<int32_t*>(alloc_owned_device(c.device, 12 * (size_t)m, c.stream));
        if (!out_ei || !out_sh) {
          release_owned_device(out_ei, c.stream);
          release_owned_device(out_sh, c.stream);
          return fail(NLB_ERR_NOMEM, "device allocation failed");
        }
      }
    } else {
      out_ei = static_cast<int64_t*>(out_ei_.get(16 * (size_t)m));
      out_sh = static_cast<int32_t*>(out_sh_.get(12 * (size_t)m));
      if (!out_ei || !out_sh) return fail(NLB_ERR_NOMEM, "device allocation failed");
    }
    int64_t* dst_tmp = static_cast<int64_t*>(dst_tmp_.get(8 * (size_t)m));
    uint64_t* state =
        static_cast<uint64_t*>(state_.get(8 * (size_t)verlet_compact_state_words(m)));
    if (!dst_tmp || !state) {
      if (owned) {
        release_owned_device(out_ei, c.stream);
        release_owned_device(out_sh, c.stream);
      }
      return fail(NLB_ERR_NOMEM, "device allocation failed");
    }
    *ei_out = out_ei;
    *sh_out = out_sh;
    if (m == 0) {
      m_last_ = 0;
      return Status{NLB_OK};
    }
    EdgeExtrasCell cell{};
    if (has_cell_) {
      std::memcpy(cell.h, h_, sizeof(h_));
      cell.has_cell = 1;
    }
    const int64_t* vei = static_cast<const int64_t*>(list_ei_.p);
    const int32_t* vsh = static_cast<const int32_t*>(list_sh_.p);
    launch_verlet_compact(d_pos, cell, vei, vsh, m, rc_ * rc_, out_ei, out_sh, dst_tmp, state,
                          kVerletSpinLimit, c.stream);
    // M and the look-back's bounded-wait error word
    cudaError_t e = cudaMemcpyAsync(c.h_small, state + 3, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                    c.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c.h_small + 1, state + 1, sizeof(int64_t), cudaMemcpyDeviceToHost,
                          c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess || c.h_small[1] != 0) {
      if (owned) {
        release_owned_device(out_ei, c.stream);
        release_owned_device(out_sh, c.stream);
        *ei_out = nullptr;
        *sh_out = nullptr;
      }
      if (e != cudaSuccess) return cuda_fail(e, "Verlet filter");
      return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
    }
    m_last_ = c.h_small[0];
    *m_out = m_last_;
    return Status{NLB_OK};
  }

  std::mutex mu_;
  double rc_, skin_;
  bool have_ = false;
  int64_t n_ = 0;
  bool has_cell_ = false;
  double h_[9] = {0};
  uint8_t pbc_[3] = {1, 1, 1};
  int64_t m_list_ = 0, m_last_ = 0;
  int64_t updates_ = 0, rebuilds_ = 0;
  double last_disp_ = 0.0;
  DevBuf pos_up_, ref_, disp_, list_ei_, list_sh_, out_ei_, out_sh_, dst_tmp_, state_;
};

}  // namespace nlb

using nlb::Verlet;

extern "C" {

struct nlb_verlet {
  Verlet* impl;
};

nlb_verlet* nlb_verlet_create(double cutoff, double skin) {
  if (!std::isfinite(cutoff) || cutoff <= 0.0) {
    nlb::fail(NLB_ERR_VALUE, "Cutoff must be positive and finite");
    return nullptr;
  }
  if (!std::isfinite(skin) || skin < 0.0) {
    nlb::fail(NLB_ERR_VALUE, "Skin must be non-negative and finite");
    return nullptr;
  }
  nlb_verlet* v = new nlb_verlet();
  v->impl = new Verlet(cutoff, skin);
  return v;
}

int nlb_verlet_update(nlb_verlet* v, const double* positions, int64_t n_atoms, const double* cell,
                      const uint8_t* pbc, int* rebuilt, nlb_result* out) {
  if (!v || !out || !rebuilt) return nlb::fail(NLB_ERR_VALUE, "NULL argument").code;
  out->n_edges = 0;
  out->edge_index = nullptr;
  out->shift = nullptr;
  if (n_atoms > 0 && !positions) return nlb::fail(NLB_ERR_VALUE, "positions is NULL").code;
  int64_t m = 0;
  int64_t* ei = nullptr;
  int32_t* sh = nullptr;
  static const double kNone = 0.0;
  nlb::Status st = v->impl->update(positions ? positions : &kNone, nullptr, n_atoms, cell, pbc,
                                   rebuilt, &m, &ei, &sh);
  if (!st.ok()) return st.code;
  st = nlb::alloc_result(m, out);
  if (!st.ok()) return st.code;
  nlb::Ctx* c = nullptr;
  st = nlb::get_ctx(&c);
  if (!st.ok()) return st.code;
  cudaError_t e = cudaSuccess;
  if (m > 0) {
    e = cudaMemcpyAsync(out->edge_index, ei, 16 * (size_t)m, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out->shift, sh, 12 * (size_t)m, cudaMemcpyDeviceToHost, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    nlb_result_free(out);
    return nlb::cuda_fail(e, "result copy").code;
  }
  return NLB_OK;
}

int nlb_verlet_update_device(nlb_verlet* v, const double* d_positions, int64_t n_atoms,
                             const double* cell, const uint8_t* pbc, int* rebuilt,
                             nlb_device_result* out) {
  if (!v || !out || !rebuilt) return nlb::fail(NLB_ERR_VALUE, "NULL argument").code;
  out->n_edges = 0;
  out->edge_index = nullptr;
  out->shift = nullptr;
  if (n_atoms > 0 && !d_positions) return nlb::fail(NLB_ERR_VALUE, "positions is NULL").code;
  int64_t m = 0;
  int64_t* ei = nullptr;
  int32_t* sh = nullptr;
  static const double kNone = 0.0;
  nlb::Status st = v->impl->update(nullptr, d_positions ? d_positions : &kNone, n_atoms, cell,
                                   pbc, rebuilt, &m, &ei, &sh);
  if (!st.ok()) return st.code;
  out->n_edges = m;
  out->edge_index = ei;
  out->shift = sh;
  return NLB_OK;
}

int nlb_verlet_update_device_owned(nlb_verlet* v, const double* d_positions, int64_t n_atoms,
                                   const double* cell, const uint8_t* pbc, int* rebuilt,
                                   nlb_device_result* out) {
  if (!v || !out || !rebuilt) return nlb::fail(NLB_ERR_VALUE, "NULL argument").code;
  out->n_edges = 0;
  out->edge_index = nullptr;
  out->shift = nullptr;
  if (n_atoms > 0 && !d_positions) return nlb::fail(NLB_ERR_VALUE, "positions is NULL").code;
  int64_t m = 0;
  int64_t* ei = nullptr;
  int32_t* sh = nullptr;
  static const double kNone = 0.0;
  nlb::Status st = v->impl->update(nullptr, d_positions ? d_positions : &kNone, n_atoms, cell,
                                   pbc, rebuilt, &m, &ei, &sh, true);
  if (!st.ok()) return st.code;
  if (m == 0) {
    // (blocks sized for a non-empty stored list, but nothing was kept)
    nlb::Ctx* c = nullptr;
    if (nlb::get_ctx(&c).ok()) {
      nlb::release_owned_device(ei, c->stream);
      nlb::release_owned_device(sh, c->stream);
    }
    return NLB_OK;
  }
  out->n_edges = m;
  out->edge_index = ei;
  out->shift = sh;
  return NLB_OK;
}

int nlb_verlet_needs_rebuild(nlb_verlet* v, const double* positions, int64_t n_atoms,
                             const double* cell, const uint8_t* pbc, int positions_on_device,
                             int* needs, double* max_displacement) {
  if (!v || !needs || !max_displacement) return nlb::fail(NLB_ERR_VALUE, "NULL argument").code;
  return v->impl
      ->needs_rebuild(positions_on_device ? nullptr : positions,
                      positions_on_device ? positions : nullptr, n_atoms, cell, pbc, needs,
                      max_displacement)
      .code;
}

void nlb_verlet_stats(nlb_verlet* v, int64_t* stats) {
  if (v && stats) v->impl->stats(stats);
}

void nlb_verlet_destroy(nlb_verlet* v) {
  if (!v) return;
  delete v->impl;
  delete v;
}

}  // extern "C"
