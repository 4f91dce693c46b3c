// k_traverse.cuh -- warp-level hit sinks shared by the single-system and the
// batched search kernels.
//
// A traversal visits one atom's candidates 32 at a time; after each step all
// 32 lanes call sink(hit, d2, i, j, shift).  Lane q of the warp owns cutoff q
// of the pass: it accumulates that cutoff's count (count pass) or holds its
// next write slot (emit pass).  Hits are compacted with ballot/popc, so each
// atom's edges are written contiguously in candidate order.
#pragma once

#include "nlb_kernels.h"

namespace nlb {

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ double shfl_d(double v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// Hit sink for the count pass: lane q accumulates cutoff q's count.
// (Sinks also take at(first candidate of the step, the cell's image shift)
// before each step; only the batched record sink uses it.)
struct CountSink {
  const CutoffSet* cs;
  uint32_t cnt;  // lane q: count of cutoff q
  __device__ __forceinline__ void at(int32_t, const int32_t*) {}
  __device__ __forceinline__ void operator()(bool hit, double d2, int32_t, int32_t, const int32_t*) {
    const int lane = threadIdx.x & 31;
    const int k = cs->k;
    double prev = cs->lower_sq;
    for (int q = 0; q < k; ++q) {
      const double rq = cs->rc_sq[q];
      const bool h = hit && d2 < rq && !(cs->disjoint && d2 < prev);
      const unsigned m = __ballot_sync(0xffffffffu, h);
      if (lane == q) cnt += __popc(m);
      prev = rq;
    }
  }
};

// Destinations of one list (served requests: one system's [src | dst] block).
struct EmitTargets1 {
  int64_t* src[1];
  int64_t* dst[1];
  int32_t* sh[1];
};

// Hit sink for the emit pass: lane q holds cutoff q's next write slot.
template <class Targets>
struct EmitSinkT {
  const CutoffSet* cs;
  const Targets* t;
  int64_t cursor;  // lane q: next slot of cutoff q
  int64_t idx_off = 0;  // added to both atom indices
  __device__ __forceinline__ void at(int32_t, const int32_t*) {}
  __device__ __forceinline__ void operator()(bool hit, double d2, int32_t io, int32_t jo,
                                             const int32_t* s) {
    const int lane = threadIdx.x & 31;
    const int k = cs->k;
    double prev = cs->lower_sq;
    for (int q = 0; q < k; ++q) {
      const double rq = cs->rc_sq[q];
      const bool h = hit && d2 < rq && !(cs->disjoint && d2 < prev);
      const unsigned m = __ballot_sync(0xffffffffu, h);
      if (m) {
        const int64_t c = __shfl_sync(0xffffffffu, cursor, q);
        if (h) {
          const int64_t e = c + __popc(m & lanemask_lt());
          t->src[q][e] = (int64_t)io + idx_off;
          t->dst[q][e] = (int64_t)jo + idx_off;
          int32_t* sh = t->sh[q] + 3 * e;
          sh[0] = s[0];
          sh[1] = s[1];
          sh[2] = s[2];
        }
        if (lane == q) cursor += __popc(m);
      }
      prev = rq;
    }
  }
};
using EmitSink = EmitSinkT<EmitTargets>;

}  // namespace nlb
