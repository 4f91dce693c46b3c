// k_verlet.cu -- kernels of the Verlet (skin) list manager.
//
//   k_max_disp      max_i |r_i - r_i,ref|^2 over the atoms (FP64, exact
//                   squares and sums; the max of non-negative doubles is
//                   taken on their bit patterns, which order the same way)
//   k_verlet_keep   per stored edge (i, j, S): keep[e] = |(r_j - r_i) + H.S|^2
//                   < rc^2 with the current positions (the displacement
//                   expression of k_extras.cu)
//   k_verlet_emit   the kept edges, compacted in stored order through the
//                   exclusive scan of keep[] ([src | dst] with the device-side
//                   total, shifts)
// All three are HBM-bound streaming kernels (24 B per atom; 28 B + two
// position gathers per stored edge; 28 B per kept edge).
#include "nlb_kernels.h"

namespace nlb {

namespace {

__device__ __forceinline__ void edge_disp(const double* __restrict__ pos,
                                          const EdgeExtrasCell& cell, int64_t i, int64_t j,
                                          int32_t s0, int32_t s1, int32_t s2, double* d) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double rel = dsub(pos[3 * j + k], pos[3 * i + k]);
    if (cell.has_cell) {
      const double hs = dadd(dadd(dmul(cell.h[3 * k], (double)s0),
                                  dmul(cell.h[3 * k + 1], (double)s1)),
                             dmul(cell.h[3 * k + 2], (double)s2));
      d[k] = dadd(rel, hs);
    } else {
      d[k] = rel;
    }
  }
}

__global__ void k_max_disp(const double* __restrict__ pos, const double* __restrict__ ref,
                           int64_t n, unsigned long long* __restrict__ out) {
  double best = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double d = norm2(dsub(pos[3 * i], ref[3 * i]), dsub(pos[3 * i + 1], ref[3 * i + 1]),
                           dsub(pos[3 * i + 2], ref[3 * i + 2]));
    // NaN (a broken trajectory) must force a rebuild: map it to +inf.
    const double v = d != d ? INFINITY : d;
    best = v > best ? v : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other > best ? other : best;
  }
  if ((threadIdx.x & 31) == 0)
    atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

__global__ void k_verlet_keep(const double* __restrict__ pos, EdgeExtrasCell cell,
                              const int64_t* __restrict__ ei, const int32_t* __restrict__ sh,
                              int64_t m, double rc_sq, uint32_t* __restrict__ keep) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x) {
    double d[3];
    edge_disp(pos, cell, ei[e], ei[m + e], sh[3 * e], sh[3 * e + 1], sh[3 * e + 2], d);
    keep[e] = norm2(d[0], d[1], d[2]) < rc_sq ? 1u : 0u;
  }
}

__global__ void k_verlet_emit(const int64_t* __restrict__ ei, const int32_t* __restrict__ sh,
                              int64_t m, const uint32_t* __restrict__ keep,
                              const int64_t* __restrict__ offs, int64_t* __restrict__ out_ei,
                              int32_t* __restrict__ out_sh) {
  const int64_t total = offs[m];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (!keep[e]) continue;
    const int64_t o = offs[e];
    out_ei[o] = ei[e];
    out_ei[total + o] = ei[m + e];
    out_sh[3 * o] = sh[3 * e];
    out_sh[3 * o + 1] = sh[3 * e + 1];
    out_sh[3 * o + 2] = sh[3 * e + 2];
  }
}

int stream_grid(int64_t items) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (items + 255) / 256;
  const int64_t cap = (int64_t)sms * 8;
  return (int)(want < 1 ? 1 : (want < cap ? want : cap));
}

}  // namespace

void launch_max_disp(const double* pos, const double* ref, int64_t n, unsigned long long* out,
                     cudaStream_t s) {
  cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
  if (n <= 0) return;
  k_max_disp<<<stream_grid(n), 256, 0, s>>>(pos, ref, n, out);
  note_launches(1);
}

void launch_verlet_keep(const double* pos, const EdgeExtrasCell& cell, const int64_t* ei,
                        const int32_t* sh, int64_t m, double rc_sq, uint32_t* keep,
                        cudaStream_t s) {
  if (m <= 0) return;
  k_verlet_keep<<<stream_grid(m), 256, 0, s>>>(pos, cell, ei, sh, m, rc_sq, keep);
  note_launches(1);
}

void launch_verlet_emit(const int64_t* ei, const int32_t* sh, int64_t m, const uint32_t* keep,
                        const int64_t* offs, int64_t* out_ei, int32_t* out_sh, cudaStream_t s) {
  if (m <= 0) return;
  k_verlet_emit<<<stream_grid(m), 256, 0, s>>>(ei, sh, m, keep, offs, out_ei, out_sh);
  note_launches(1);
}

}  // namespace nlb
