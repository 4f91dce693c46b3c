// k_extras.cu -- output options on a device half list: the directed list
// ((i, j, S) followed by the reverses (j, i, -S)), displacement vectors
// d = (r_j - r_i) + H.S and distances |d|.
//
// One thread per half edge; it reads (i, j, S) and the two positions once and
// writes the forward entry at e and, when directed, the reverse entry at
// m + e.  The FP64 expression order is fixed (component k:
// (r_j,k - r_i,k) + ((H[k][0] S0 + H[k][1] S1) + H[k][2] S2); no H term for
// a system without a cell) and the distance is the correctly rounded square
// root of (d0^2 + d1^2) + d2^2, so results are reproducible bit for bit.
// HBM-bound: 28 B in + (28 + 24 + 8) B out per edge (x2 when directed), plus
// two 24 B position gathers that mostly hit L2.
#include "nlb_kernels.h"

namespace nlb {

namespace {

__global__ void k_edge_extras(const double* __restrict__ pos, EdgeExtrasCell cell,
                              const int64_t* __restrict__ ei, const int32_t* __restrict__ sh,
                              int64_t m, int directed, int64_t* __restrict__ ei_out,
                              int32_t* __restrict__ sh_out, double* __restrict__ vec,
                              double* __restrict__ dist) {
  const int64_t mo = directed ? 2 * m : m;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = ei[e], j = ei[m + e];
    const int32_t s0 = sh[3 * e], s1 = sh[3 * e + 1], s2 = sh[3 * e + 2];
    if (ei_out) {
      ei_out[e] = i;
      ei_out[mo + e] = j;
      if (directed) {
        ei_out[m + e] = j;
        ei_out[mo + m + e] = i;
      }
    }
    if (sh_out) {
      sh_out[3 * e] = s0;
      sh_out[3 * e + 1] = s1;
      sh_out[3 * e + 2] = s2;
      if (directed) {
        sh_out[3 * (m + e)] = -s0;
        sh_out[3 * (m + e) + 1] = -s1;
        sh_out[3 * (m + e) + 2] = -s2;
      }
    }
    if (!vec && !dist) continue;
    double d[3];
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
    if (vec) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        vec[3 * e + k] = d[k];
        if (directed) vec[3 * (m + e) + k] = -d[k];
      }
    }
    if (dist) {
      const double r = __dsqrt_rn(norm2(d[0], d[1], d[2]));
      dist[e] = r;
      if (directed) dist[m + e] = r;
    }
  }
}

}  // namespace

void launch_edge_extras(const double* pos, const EdgeExtrasCell& cell, const int64_t* ei,
                        const int32_t* sh, int64_t m, int directed, int64_t* ei_out,
                        int32_t* sh_out, double* vec, double* dist, cudaStream_t s) {
  if (m <= 0) return;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (m + 255) / 256;
  const int grid = (int)(want < (int64_t)sms * 8 ? want : (int64_t)sms * 8);
  k_edge_extras<<<grid, 256, 0, s>>>(pos, cell, ei, sh, m, directed, ei_out, sh_out, vec, dist);
  note_launches(1);
}

}  // namespace nlb
