// nlb_common.cuh -- shared types and exact-FP64 helpers for the neighbour-list
// kernels (sm_100a).
//
// Every floating-point expression that decides an edge, a bin or a shift is
// evaluated with explicitly rounded intrinsics (__dmul_rn/__dadd_rn/...) in
// the same association order as the reference's f64 code, so no multiply-add
// is ever contracted into an FMA.  The library is additionally compiled with
// -fmad=false.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nlb {

// Cutoffs handled by one multi-cutoff pass (one warp lane per cutoff).
constexpr int kMaxCutoffsPerPass = 32;

// Per-system grid description; mirrors the CellList fields of the reference
// (src/search.rs:68-89) that the search needs.
struct GridParams {
  double h[9];       // H, row-major; columns are the lattice vectors
  double hinv[9];    // H^-1 (row-major)
  int32_t nb[3];     // bins per axis: max(1, floor(w_a / rc))
  int32_t ns[3];     // stencil half-width per axis: ceil(rc * nb_a / w_a)
  double basis[3][3];  // basis[a] = H e_a / nb_a
  double origin[3];    // H (0.5/nb)
  double prune_sq;     // (sqrt(rc_max^2) + bin_bounding_radius)^2
  int64_t total_bins;
  double radius;       // bin bounding radius (half the largest bin diagonal)
};

// A run of at most 32 atoms of one bin (a pair-task group).
struct alignas(8) GroupRec {
  int32_t first, end;  // sorted slots [first, min(first + 32, end)); end = bin end
  int32_t bx, by, bz;  // the bin's coordinates
  int32_t lin;         // its linear index
};

// Sorted-slot payload that travels with a candidate: wrap shift and the
// original atom index, loaded as one 16-byte vector.
struct alignas(16) SlotMeta {
  int32_t sx, sy, sz;
  int32_t orig;
};

#if defined(__CUDACC__)
// ---------------------------------------------------------------- device only

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// nalgebra Matrix3 * Vector3 order: (m0*v0 + m1*v1) + m2*v2 per row.
__device__ __forceinline__ void matvec(const double* m, double v0, double v1, double v2,
                                       double* out) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
    out[r] = dadd(dadd(dmul(m[3 * r], v0), dmul(m[3 * r + 1], v1)), dmul(m[3 * r + 2], v2));
}

// (a*a + b*b) + c*c
__device__ __forceinline__ double norm2(double a, double b, double c) {
  return dadd(dadd(dmul(a, a), dmul(b, b)), dmul(c, c));
}

// Rust `f as i32`: truncate toward zero, saturate, NaN -> 0.
// acc << 1 with the sign bit of v as the new lowest bit.  Appending, for
// candidates 31 down to 0, the sign of (d2 - bound) (FP32, exactly rounded:
// negative iff d2 < bound for finite or infinite d2) or of (io - j) (no
// overflow for indices below 2^31 - 1) leaves candidate k's predicate at bit
// k: one funnel shift per predicate.
__device__ __forceinline__ uint32_t push_sign(uint32_t acc, uint32_t v) {
  return __funnelshift_l(v, acc, 1);
}

__device__ __forceinline__ int32_t sat_i32(double x) {
  if (x != x) return 0;
  if (x >= 2147483647.0) return 2147483647;
  if (x <= -2147483648.0) return (-2147483647 - 1);
  return (int32_t)x;
}

// Rust `f as usize`: truncate, negative/NaN -> 0, saturate.
__device__ __forceinline__ uint64_t sat_u64(double x) {
  if (!(x > 0.0)) return 0ull;
  if (x >= 18446744073709551616.0) return ~0ull;
  return (uint64_t)x;
}

__device__ __forceinline__ uint64_t spread_bits3(uint64_t x) {
  x &= 0x1fffffULL;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

// compute_z_order (src/search.rs:1169-1175) of a wrapped fraction.
__device__ __forceinline__ uint64_t morton_of_frac(double f0, double f1, double f2) {
  const double scale = 2097152.0;  // 2^21
  double c[3] = {f0, f1, f2};
  uint64_t q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double v = c[a];
    if (v < 0.0) v = 0.0;
    if (v > 0.999999) v = 0.999999;  // NaN passes through, like f64::clamp
    q[a] = sat_u64(dmul(v, scale));
  }
  return spread_bits3(q[0]) | (spread_bits3(q[1]) << 1) | (spread_bits3(q[2]) << 2);
}

// Euclidean division (i32::rem_euclid / div_euclid for a positive divisor).
__device__ __forceinline__ void div_mod(int32_t v, int32_t m, int32_t& rem, int32_t& quot) {
  int32_t q = v / m;
  int32_t r = v - q * m;
  if (r < 0) {
    r += m;
    q -= 1;
  }
  rem = r;
  quot = q;
}

// Per-atom wrap (src/search.rs:192-215): fraction, floor, wrap shift
// s = -floor(frac) as i32, wrapped position pos - H * (-s), and the bin
// coordinates of the wrapped fraction u = frac - floor(frac).
struct AtomWrap {
  double wx, wy, wz;
  int32_t s[3];
  int32_t bin[3];
  uint64_t key;
};

__device__ __forceinline__ AtomWrap wrap_atom(const GridParams& g, double px, double py,
                                              double pz) {
  AtomWrap w;
  double f[3];
  matvec(g.hinv, px, py, pz, f);
  double fl[3], u[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    fl[a] = floor(f[a]);
    u[a] = dsub(f[a], fl[a]);
    w.s[a] = sat_i32(-fl[a]);
    uint64_t b = sat_u64(dmul(u[a], (double)g.nb[a]));
    uint64_t cap = (uint64_t)(g.nb[a] - 1);
    w.bin[a] = (int32_t)(b < cap ? b : cap);
  }
  w.key = morton_of_frac(u[0], u[1], u[2]);
  // (-s) as f64, with i32 wrapping negation like the reference's release build.
  double sv[3];
  matvec(g.h, (double)(int32_t)(0u - (uint32_t)w.s[0]), (double)(int32_t)(0u - (uint32_t)w.s[1]),
         (double)(int32_t)(0u - (uint32_t)w.s[2]), sv);
  w.wx = dsub(px, sv[0]);
  w.wy = dsub(py, sv[1]);
  w.wz = dsub(pz, sv[2]);
  return w;
}

// Programmatic dependent launch: a kernel launched with launch_pdl may start
// while its predecessor in the stream drains; pdl_wait() blocks until the
// predecessor grid has completed and its writes are visible (a no-op when
// the kernel was launched normally).  Every kernel launched with launch_pdl
// calls pdl_wait() before it reads anything its predecessors wrote.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

#endif  // __CUDACC__

}  // namespace nlb
