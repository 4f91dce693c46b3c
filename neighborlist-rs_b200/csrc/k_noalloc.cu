// k_noalloc.cu -- a neighbour-list build that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they need a
// neighbour list:
//   * processes whose GPU memory is already claimed by a framework's caching
//     allocator (PyTorch, JAX/XLA preallocation), where a fresh cudaMalloc
//     fails or fragments the pool;
//   * code that runs between other stream-ordered work and must not stall it:
//     cudaFree (and a growing cudaMalloc) synchronises the whole device;
//   * long-running or real-time loops (MD engines, servers) that allocate
//     everything once at start-up and forbid allocation afterwards.
// nlb_build_noalloc serves them: the caller passes the device positions and
// fixed-capacity device output arrays, and every intermediate array of the
// cell-list / brute-force pipeline (bin tables, sorted atoms, per-atom edge
// counts and offsets) lives in ONE file-scope __device__ array,
// g_noalloc_scratch, sized for kNoAllocMaxAtoms atoms and kNoAllocMaxBins
// bins (about 1.8 MB).  Like any __device__ variable it is part of the
// library image: every GPU that loads the library holds it until the process
// exits.
//
// The kernels are the library's regular ones; only where their scratch comes
// from differs.  Host code cannot use the array's name as a device address
// (it is a host-side stand-in), so the first call on each device, with that
// device current, asks the runtime for the address with cudaGetSymbolAddress
// and caches it.  That first call should therefore happen before any stream
// capture begins.  The cached address belongs to the device's current
// context: after a cudaDeviceReset of that device the process must not call
// this entry point again.  Each call synchronises its stream (after the count
// pass and after the emit pass) before it returns.
//
// All calls share the one array: calls that overlap on the GPU (two host
// threads, or two streams, at once on the same device) race on it and must be
// serialised by the caller.  Each call re-zeroes the parts that must start at
// zero (bin histogram and scatter cursors); everything else is fully
// overwritten before it is read.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "nlb_internal.h"

namespace nlb {

namespace {

constexpr int64_t kNoAllocMaxAtoms = 16384;
constexpr int64_t kNoAllocMaxBins = 16384;
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Scan states for the largest scans here: the n + 1 counts in the first
// half, the bin histogram in the second (each keeps its own error word).
constexpr int64_t kNoAllocScanWords = 64;
constexpr int64_t kNoAllocBinScan = kNoAllocScanWords / 2;
static_assert((kNoAllocMaxAtoms + 1 + kScanTile - 1) / kScanTile + 2 <= kNoAllocBinScan &&
                  (kNoAllocMaxBins + kScanTile - 1) / kScanTile + 2 <= kNoAllocBinScan,
              "scan state of the scratch array too small for the scan tile");

// Byte layout of the scratch array (each piece 256-byte aligned).
struct Layout {
  size_t rank_of_bin, bin_count, bin_fill, bin_start, key, rank, skey, sidx, skey2, sidx2, px,
      py, pz, meta, counts, offs, scan_tmp, bounds, total;
};

constexpr Layout make_layout() {
  Layout L{};
  size_t o = 0;
  L.rank_of_bin = o; o += align256(sizeof(int32_t) * kNoAllocMaxBins);
  L.bin_count = o; o += align256(sizeof(int32_t) * kNoAllocMaxBins);
  L.bin_fill = o; o += align256(sizeof(int32_t) * kNoAllocMaxBins);
  L.bin_start = o; o += align256(sizeof(int64_t) * (kNoAllocMaxBins + 1));
  L.key = o; o += align256(sizeof(uint64_t) * kNoAllocMaxAtoms);
  L.rank = o; o += align256(sizeof(int32_t) * kNoAllocMaxAtoms);
  L.skey = o; o += align256(sizeof(uint64_t) * kNoAllocMaxAtoms);
  L.sidx = o; o += align256(sizeof(int32_t) * kNoAllocMaxAtoms);
  L.skey2 = o; o += align256(sizeof(uint64_t) * kNoAllocMaxAtoms);
  L.sidx2 = o; o += align256(sizeof(int32_t) * kNoAllocMaxAtoms);
  L.px = o; o += align256(sizeof(double) * kNoAllocMaxAtoms);
  L.py = o; o += align256(sizeof(double) * kNoAllocMaxAtoms);
  L.pz = o; o += align256(sizeof(double) * kNoAllocMaxAtoms);
  L.meta = o; o += align256(sizeof(SlotMeta) * kNoAllocMaxAtoms);
  L.counts = o; o += align256(sizeof(uint32_t) * (kNoAllocMaxAtoms + 1));
  L.offs = o; o += align256(sizeof(int64_t) * (kNoAllocMaxAtoms + 2));
  L.scan_tmp = o; o += align256(sizeof(int64_t) * kNoAllocScanWords);
  L.bounds = o; o += align256(sizeof(double) * 6);
  L.total = o;
  return L;
}

constexpr Layout kLayout = make_layout();

// The only scratch memory of nlb_build_noalloc.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kLayout.total];

// Device address of g_noalloc_scratch per device, filled by the first call
// made with that device current.
unsigned char* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mu;

Status scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(NLB_ERR_VALUE, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return Status{NLB_OK};
}

template <class T>
T* at(unsigned char* base, size_t off) {
  return reinterpret_cast<T*>(base + off);
}

}  // namespace

Status run_noalloc(const double* d_pos, int64_t n, double cutoff, const double* cell9,
                   const uint8_t* pbc, int64_t* d_edge_index, int32_t* d_shift,
                   int64_t max_edges, int64_t* n_edges, cudaStream_t s) {
  if (n_edges) *n_edges = 0;
  if (!n_edges) return fail(NLB_ERR_VALUE, "n_edges is NULL");
  if (!std::isfinite(cutoff) || cutoff <= 0.0)
    return fail(NLB_ERR_VALUE, "Cutoff must be positive and finite");
  if (n < 0) return fail(NLB_ERR_VALUE, "Positions must be (N, 3)");
  if (n > kNoAllocMaxAtoms)
    return fail(NLB_ERR_VALUE, "nlb_build_noalloc: " + std::to_string(n) +
                                   " atoms exceed its fixed capacity of " +
                                   std::to_string(kNoAllocMaxAtoms));
  if (max_edges < 0) return fail(NLB_ERR_VALUE, "max_edges must be >= 0");
  if (n == 0) return Status{NLB_OK};
  if (!d_pos || (max_edges > 0 && (!d_edge_index || !d_shift)))
    return fail(NLB_ERR_VALUE, "NULL positions or output pointer");

  unsigned char* base = nullptr;
  Status st = scratch_for_current_device(&base);
  if (!st.ok()) return st;

  // ---- plan (host, fixed-size arrays only)
  HostCell cell;
  std::string err;
  const bool pb[3] = {pbc ? pbc[0] != 0 : true, pbc ? pbc[1] != 0 : true,
                      pbc ? pbc[2] != 0 : true};
  if (cell9) {
    if (!make_cell(cell9, pb, cell, err)) return fail(NLB_ERR_VALUE, err);
  } else {
    double* d_b = at<double>(base, kLayout.bounds);
    double hb[6];
    launch_bounds(d_pos, n, d_b, s);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(hb, d_b, sizeof(hb), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "bounds");
    if (!auto_box_from_bounds(hb, hb + 3, cutoff, cell, err)) return fail(NLB_ERR_VALUE, err);
  }
  const Method method = choose_method(cell, n, cutoff, nlb_get_brute_force_threshold(), false);
  GridParams g{};
  BruteParams bp{};
  GridBuffers b{};
  if (method == Method::kCellList) {
    plan_grid(cell, cutoff, g);
    // Every size check happens here, before anything is launched into the
    // fixed scratch array.
    for (int a = 0; a < 3; ++a)
      if (g.nb[a] < 1 || g.nb[a] >= (1 << 21))
        return fail(NLB_ERR_VALUE, "cell list needs more than 2^21 bins along one axis");
    for (int a = 0; a < 3; ++a)
      if (g.ns[a] < 0 || g.ns[a] > (1 << 20))
        return fail(NLB_ERR_VALUE, "stencil too large for this cutoff and cell");
    if (g.total_bins < 1 || g.total_bins > kNoAllocMaxBins)
      return fail(NLB_ERR_VALUE, "nlb_build_noalloc: " + std::to_string(g.total_bins) +
                                     " cell-list bins exceed its fixed capacity of " +
                                     std::to_string(kNoAllocMaxBins));
    b.rank_of_bin = at<int32_t>(base, kLayout.rank_of_bin);
    b.bin_count = at<int32_t>(base, kLayout.bin_count);
    b.bin_fill = at<int32_t>(base, kLayout.bin_fill);
    b.bin_start = at<int64_t>(base, kLayout.bin_start);
    b.key = at<uint64_t>(base, kLayout.key);
    b.rank = at<int32_t>(base, kLayout.rank);
    b.skey = at<uint64_t>(base, kLayout.skey);
    b.sidx = at<int32_t>(base, kLayout.sidx);
    b.skey2 = at<uint64_t>(base, kLayout.skey2);
    b.sidx2 = at<int32_t>(base, kLayout.sidx2);
    b.px = at<double>(base, kLayout.px);
    b.py = at<double>(base, kLayout.py);
    b.pz = at<double>(base, kLayout.pz);
    b.meta = at<SlotMeta>(base, kLayout.meta);
    b.scan_tmp = at<int64_t>(base, kLayout.scan_tmp) + kNoAllocBinScan;
  } else {
    std::memcpy(bp.h, cell.h, sizeof(bp.h));
    std::memcpy(bp.hinv, cell.hinv, sizeof(bp.hinv));
    for (int a = 0; a < 3; ++a) bp.pbc[a] = cell.pbc[a] ? 1 : 0;
    bp.mode = method == Method::kBruteIsolated ? kBruteRaw : kBruteMicMode;
  }
  CutoffSet cs{};
  cs.k = 1;
  cs.rc_sq[0] = cutoff * cutoff;
  cs.disjoint = 0;
  cs.lower_sq = -1.0;
  cs.max_sq = cs.rc_sq[0];
  uint32_t* counts = at<uint32_t>(base, kLayout.counts);
  int64_t* offs = at<int64_t>(base, kLayout.offs);
  int64_t* scan_tmp = at<int64_t>(base, kLayout.scan_tmp);

  // ---- count pass (scratch re-zeroed where it must start at zero)
  cudaError_t e = cudaSuccess;
  if (method == Method::kCellList) {
    e = cudaMemsetAsync(b.bin_count, 0, sizeof(int32_t) * g.total_bins, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b.bin_fill, 0, sizeof(int32_t) * g.total_bins, s);
    if (e != cudaSuccess) return cuda_fail(e, "nlb_build_noalloc: clearing the bin tables");
    launch_grid_build(g, d_pos, n, b, s);
    launch_grid_count(g, b, n, cs, counts, s);
  } else {
    launch_brute_count(bp, d_pos, n, cs, counts, s);
  }
  exclusive_scan_u32(counts, n + 1, offs, scan_tmp, s);
  // Launch-configuration errors are not sticky and a later synchronisation
  // does not report them: ask for them right after the launches.
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "nlb_build_noalloc count pass launch");
  // The edge total and the scans' bounded-wait error words, in one sync.
  int64_t h_tail[3] = {0, 0, 0};
  e = cudaMemcpyAsync(&h_tail[0], offs + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h_tail[1], scan_tmp + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && method == Method::kCellList)
    e = cudaMemcpyAsync(&h_tail[2], b.scan_tmp + 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "nlb_build_noalloc count pass");
  if (h_tail[1] != 0 || h_tail[2] != 0)
    return fail(NLB_ERR_CUDA, "prefix scan gave up waiting for a tile");
  const int64_t total = h_tail[0];
  *n_edges = total;
  if (total > max_edges)
    return fail(NLB_ERR_VALUE, "nlb_build_noalloc: " + std::to_string(total) +
                                   " edges exceed the output capacity max_edges = " +
                                   std::to_string(max_edges));
  if (total == 0) return Status{NLB_OK};

  // ---- emit pass into the caller's (2, max_edges) / (max_edges, 3) arrays
  EmitTargets t;
  std::memset(&t, 0, sizeof(t));
  t.src[0] = d_edge_index;
  t.dst[0] = d_edge_index + max_edges;
  t.sh[0] = d_shift;
  t.base[0] = 0;
  t.index_offset = 0;
  if (method == Method::kCellList)
    launch_grid_emit(g, b, n, cs, offs, t, s);
  else
    launch_brute_emit(bp, d_pos, n, cs, offs, t, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "nlb_build_noalloc emit pass launch");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "nlb_build_noalloc emit pass");
  return Status{NLB_OK};
}

}  // namespace nlb

extern "C" int nlb_build_noalloc(const double* d_positions, int64_t n_atoms, double cutoff,
                                 const double* cell, const uint8_t* pbc, int64_t* d_edge_index,
                                 int32_t* d_shift, int64_t max_edges, int64_t* n_edges,
                                 void* stream) {
  return nlb::run_noalloc(d_positions, n_atoms, cutoff, cell, pbc, d_edge_index, d_shift,
                          max_edges, n_edges, static_cast<cudaStream_t>(stream))
      .code;
}
