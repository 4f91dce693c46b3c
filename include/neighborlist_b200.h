/* neighborlist_b200.h -- C ABI of the B200 neighbour-list library.
 *
 * Drop-in boundary for the search path of solccp/neighborlist-rs.  Each entry
 * point names the reference interface it replaces (paths inside that
 * project).  Conventions:
 *   - positions: n x 3 float64, row-major (x0 y0 z0 x1 ...), host memory;
 *   - cell: 9 float64, row-major H whose COLUMNS are the lattice vectors
 *     (Matrix3::new argument order, src/api.rs:93-98); NULL = no cell
 *     (auto-box: orthorhombic, origin 0, no periodicity, src/single.rs:21-58);
 *   - pbc: 3 bytes (0/1); honoured by the brute-force minimum-image path only,
 *     exactly like the reference (the cell-list path images every axis);
 *   - results: exact-sized, library-owned pinned host arrays,
 *     edge_index = [src_0..src_{M-1}, dst_0..dst_{M-1}] int64 (the layout of
 *     NeighborList::edge_index, src/api.rs:10-17) and shift = [x0 y0 z0 x1 ...]
 *     int32; release them with nlb_result_free.
 * Every function returns NLB_OK or an error code; nlb_last_error() gives the
 * calling thread's last message (the reference's Err(String) texts).
 * All entry points are thread-safe: each host thread gets its own CUDA stream
 * and device workspace on the current device.  Workspaces and result arrays
 * come from one stream-ordered memory pool per device, which keeps the
 * memory it has mapped for the life of the process (a thread's workspace
 * goes back to the pool, not to the driver, when the thread ends).
 */
#ifndef NEIGHBORLIST_B200_H
#define NEIGHBORLIST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NLB_OK 0
#define NLB_ERR_VALUE 1 /* invalid input; message from nlb_last_error() */
#define NLB_ERR_CUDA 2  /* CUDA failure (no device, launch or copy error) */
#define NLB_ERR_NOMEM 3 /* device or pinned-host allocation failed */
#define NLB_NOT_READY 4 /* nlb_server_wait: the request did not finish in time */

typedef struct nlb_result {
  int64_t n_edges;     /* M */
  int64_t* edge_index; /* 2*M int64: sources then destinations */
  int32_t* shift;      /* 3*M int32 */
} nlb_result;

/* Message of the calling thread's last failed call ("" if none). */
const char* nlb_last_error(void);

/* Single system, one cutoff.
 * Replaces neighborlist_rs::build_neighborlists (src/api.rs:20-38) and the
 * search behind the Python build_neighborlists (src/python_api.rs:141-186,
 * src/single.rs:8-90).  `parallel` is accepted for signature parity and does
 * not change the result (the reference's serial and parallel paths produce
 * the same edges in the same order). */
int nlb_build(const double* positions, int64_t n_atoms, double cutoff, const double* cell,
              const uint8_t* pbc, int parallel, nlb_result* out);

/* Single system, k cutoffs in one traversal (grid at the largest cutoff);
 * outs[q] receives the list of cutoffs[q].  disjoint != 0 puts each pair in
 * the first ascending shell only.
 * Replaces neighborlist_rs::single::search_single_multi (src/single.rs:92-164)
 * behind build_neighborlists_multi (src/python_api.rs:237-309). */
int nlb_build_multi(const double* positions, int64_t n_atoms, const double* cutoffs,
                    int32_t n_cutoffs, const double* cell, const uint8_t* pbc, int disjoint,
                    nlb_result* outs);

/* Batched systems: batch[i] is atom i's system id; a new system starts
 * wherever the id changes (src/batch.rs:25-38); ids must not decrease
 * (NLB_ERR_VALUE "Batch IDs must be monotonic (non-decreasing)", the check of
 * src/python_api.rs:315-423).  cells: n_cells x 9 (rows of H as above) or
 * NULL (every system auto-boxed); pbcs: n_cells x 3, or NULL for all
 * periodic; has_cell: n_cells flags, 0 = None (auto-box), or NULL for all
 * set.  Atom indices in the output are global (offset by each system's first
 * atom).
 * Replaces neighborlist_rs::build_neighborlists_batch (src/api.rs:43-84) and
 * batch::search_batch (src/batch.rs:10-147). */
int nlb_build_batch(const double* positions, int64_t n_atoms, const int32_t* batch,
                    int64_t n_batch, double cutoff, const double* cells, const uint8_t* pbcs,
                    const uint8_t* has_cell, int64_t n_cells, int parallel, nlb_result* out);

/* Batched systems, k cutoffs.
 * Replaces neighborlist_rs::batch::search_batch_multi (src/batch.rs:149-290). */
int nlb_build_batch_multi(const double* positions, int64_t n_atoms, const int32_t* batch,
                          int64_t n_batch, const double* cutoffs, int32_t n_cutoffs,
                          const double* cells, const uint8_t* pbcs, const uint8_t* has_cell,
                          int64_t n_cells, int disjoint, nlb_result* outs);

/* The batched build with a per-system offset table on the output (no
 * counterpart in the reference, whose batched result is the concatenated
 * list only).  Arguments as nlb_build_batch_multi; multi = 0 gives the
 * single-cutoff semantics of nlb_build_batch (n_cutoffs = 1).  When
 * system_offsets is not NULL it receives n_cutoffs rows of n_systems + 1
 * int64 (row = input cutoff index; n_systems counts the batch-id runs, 0 for
 * an empty input): system i's edges of that list are [row[i], row[i + 1]).
 * The table comes from the device's count pass at no extra synchronisation. */
int nlb_build_batch_ex(const double* positions, int64_t n_atoms, const int32_t* batch,
                       int64_t n_batch, const double* cutoffs, int32_t n_cutoffs,
                       const double* cells, const uint8_t* pbcs, const uint8_t* has_cell,
                       int64_t n_cells, int disjoint, int multi, nlb_result* outs,
                       int64_t* system_offsets);

/* Releases both arrays of a result (safe on a zeroed struct). */
void nlb_result_free(nlb_result* r);
/* Releases one array obtained from a result (for callers that hand the two
 * arrays to separate owners, e.g. two numpy arrays). */
void nlb_host_free(void* p);

/* Pinned host pool behind every host result (no counterpart in the
 * reference): fills 7 counters: cudaHostAlloc calls, microseconds spent in
 * them, bytes they allocated, cudaFreeHost calls, microseconds spent in
 * them, requests served from cached blocks, bytes cached now. */
void nlb_pinned_stats(int64_t* out);

/* Dispatch thresholds (src/config.rs:4-40).  The brute-force threshold decides
 * brute force vs cell list and therefore the output order; the parallel
 * threshold selects the reference's serial/parallel CPU variant and has no
 * effect on the result; the stack threshold is kept for API parity and is
 * clamped to 1024 like the reference. */
size_t nlb_get_brute_force_threshold(void);
void nlb_set_brute_force_threshold(size_t v);
size_t nlb_get_parallel_threshold(void);
void nlb_set_parallel_threshold(size_t v);
size_t nlb_get_stack_threshold(void);
void nlb_set_stack_threshold(size_t v);

/* ---- Device-resident path (positions and results stay in HBM). ----
 * nlb_build_device: like nlb_build, but `d_positions` is a device pointer and
 * the result arrays are device pointers into the calling thread's workspace,
 * valid until that thread's next build call (copy them out to keep them).
 * Layout is the same as nlb_result (edge_index = [src | dst], shift xyz).
 * Used by GNN pipelines that consume edge_index on the GPU (e.g. through
 * DLPack / torch) and by bench.py's device-resident measurement.
 * Ordering: on the library's own stream the call returns when the arrays are
 * complete.  On a stream set with nlb_set_stream it returns as soon as M is
 * known (the device reports it through host-mapped memory); the arrays are
 * complete in that stream's order -- work queued on it afterwards sees them,
 * work on other streams must wait for it (an event).  The same holds for
 * nlb_build_device_owned. */
typedef struct nlb_device_result {
  int64_t n_edges;
  int64_t* edge_index; /* device, 2*M int64 */
  int32_t* shift;      /* device, 3*M int32 */
} nlb_device_result;

int nlb_build_device(const double* d_positions, int64_t n_atoms, double cutoff,
                     const double* cell, const uint8_t* pbc, nlb_device_result* out);

/* Zero-copy device results (no counterpart in the reference, whose results
 * are host Vecs; its consumer is a GNN that takes edge_index on the GPU,
 * spec.md:13).  As nlb_build_device, but the two result arrays are handed
 * over to the caller: they are device blocks of the library's stream-ordered
 * result pool, written in place by the build (no copy), and stay valid until
 * the caller returns each one with nlb_device_free.  Both are NULL when
 * M = 0.  The blocks may be larger than 16 M and 12 M bytes; edge_index is
 * [src | dst] in its first 2 M entries.
 * nlb_device_free: returns such a block to the pool after the work queued so
 * far on `stream` (a cudaStream_t; NULL = legacy default stream): pass the
 * stream whose work last used the block.  NLB_ERR_VALUE for a pointer that is
 * not an outstanding block.
 * nlb_device_blocks: out3 = {blocks handed out, blocks returned, bytes of the
 * blocks still outstanding}. */
int nlb_build_device_owned(const double* d_positions, int64_t n_atoms, double cutoff,
                           const double* cell, const uint8_t* pbc, nlb_device_result* out);
int nlb_device_free(void* p, void* stream);
void nlb_device_blocks(int64_t* out3);

/* Device-to-device copy on `stream` (a cudaStream_t): lets callers move a
 * device result into memory they own before the next build. */
int nlb_copy_device(void* dst, const void* src, size_t bytes, void* stream);

/* Stream for the calling thread's subsequent calls (a cudaStream_t); NULL
 * restores the library's own non-blocking stream. */
void nlb_set_stream(void* stream);

/* Kernel launches issued by this library since load (all threads). */
int64_t nlb_kernel_launches(void);
/* CUDA-graph replays since load (all threads): a repeated identical
 * single-system build (same sizes, cell, cutoff, buffers, stream) and a
 * repeated batched build of the same shape (same system sizes, cutoffs,
 * decided launch shape, buffers, stream) replay their captured graphs. */
int64_t nlb_graph_replays(void);

/* Single-system, single-cutoff pipeline choice (no counterpart in the
 * reference).  mode 0 (the default): sparse grids (at most 64 atoms per bin
 * on average, at most 125 stencil cells) count, place and write their edges
 * in one launch, denser ones in three (count, offsets scan, emit); mode 1:
 * always the three-launch pipeline.  Both give identical results.  mode < 0
 * only queries.  Returns the previous mode, or -1 for an unknown mode. */
int32_t nlb_single_pipeline(int32_t mode);
/* The pipeline the calling thread's last single-cutoff cell-list build took:
 * 0 = one launch, 1 = three launches, -1 = none yet. */
int32_t nlb_last_single_pipeline(void);

/* Failure-detection hook (no counterpart in the reference, which has no
 * device waits).  The device prefix scans wait on their predecessor tiles
 * with bounded polls; when a wait runs out, the scan records an error word,
 * finishes without waiting further, the emit pass writes nothing, and the
 * build returns NLB_ERR_CUDA ("prefix scan gave up waiting for a tile") with
 * the device and the library still usable.  This call makes the calling
 * thread's next scan launch exercise that path: its tile `tile` withholds
 * its publication, and its successors poll at most spin_limit times.  One
 * shot; builds whose scan has fewer tiles are unaffected.  Returns NLB_OK,
 * or NLB_ERR_VALUE for tile < 0 or spin_limit < 1. */
int nlb_debug_scan_stall(int32_t tile, int32_t spin_limit);

/* Per-thread phase timing with CUDA events on the launching stream.
 * enable != 0 starts (and resets) it.  nlb_profile_read fills ms[0..3] with
 * the accumulated device time of: grid build, count pass, offset scan, emit
 * pass, and returns the number of profiled calls. */
void nlb_profile(int enable);
int64_t nlb_profile_read(double* ms);
/* Host wall time of profiled batched builds of small systems (ms, summed):
 * input upload, device work from issue to its synchronisation, result
 * copies, the whole call; returns the number of profiled calls. */
int64_t nlb_profile_host(double* ms);

/* Launch shapes of the batched kernels (no counterpart in the reference,
 * whose batch path has no launch configuration).  Batches are tuned per kind
 * (cutoff count, power-of-two buckets of the system count, the largest and
 * the mean system, quarter-octave bucket of the largest cutoff): the first
 * batch of a kind runs its count pass once in every candidate shape, timed
 * with CUDA events, and the kind keeps the fastest.  Every shape gives
 * identical results.
 *
 * nlb_batch_shape(i) pins shape i (0 = the default) for every batched
 * launch of the process, -1 returns to tuning; it returns the number of
 * shapes, or -1 if i is out of range.  NLB_BATCH_SHAPE=i in the environment
 * pins from the start.  nlb_batch_shape_info fills {threads per CTA for
 * whole systems, threads per CTA for split systems, atoms per work item of a
 * split system, size above which a system is split}.  nlb_batch_tuner_state
 * writes up to cap rows of 8 int64 {device, cutoffs (0: one per system),
 * log2 systems, log2 largest, log2 mean, cutoff bucket, chosen shape (-1:
 * not decided), candidate shapes} and returns the number of kinds seen;
 * nlb_batch_tuner_reset forgets them. */
int32_t nlb_batch_shape(int32_t shape);
int32_t nlb_batch_shape_info(int32_t shape, int32_t* out4);
int32_t nlb_batch_tuner_state(int64_t* out, int32_t cap);
void nlb_batch_tuner_reset(void);

/* ---- Output options (asked for by the reference's spec.md:100-108 and
 * RUST_API.md:89-90, not implemented by the reference). ----
 * nlb_build_ex: the nlb_build search, then on the device:
 *   NLB_DIRECTED   the M half edges followed by their reverses (j, i, -S):
 *                  2M edges ("double the edges and negate the shifts");
 *   NLB_VECTORS    d = (r_j - r_i) + H.S per edge, float64 x3 (component k
 *                  evaluated as (r_j,k - r_i,k) + ((H[k][0] S0 + H[k][1] S1)
 *                  + H[k][2] S2); r_j - r_i when cell is NULL); reverses get -d;
 *   NLB_DISTANCES  |d| = sqrt((d0^2 + d1^2) + d2^2), correctly rounded.
 * Arrays not asked for are NULL.  Free with nlb_result_ex_free.
 * nlb_build_device_ex: device positions in, device pointers into the calling
 * thread's workspace out (valid until its next build call). */
#define NLB_DIRECTED 1
#define NLB_VECTORS 2
#define NLB_DISTANCES 4
typedef struct nlb_result_ex {
  int64_t n_edges;     /* M, or 2M when directed */
  int64_t* edge_index; /* 2 * n_edges int64: sources then destinations */
  int32_t* shift;      /* 3 * n_edges int32 */
  double* vectors;     /* 3 * n_edges float64, or NULL */
  double* distances;   /* n_edges float64, or NULL */
} nlb_result_ex;
int nlb_build_ex(const double* positions, int64_t n_atoms, double cutoff, const double* cell,
                 const uint8_t* pbc, int flags, nlb_result_ex* out);
int nlb_build_device_ex(const double* d_positions, int64_t n_atoms, double cutoff,
                        const double* cell, const uint8_t* pbc, int flags, nlb_result_ex* out);
void nlb_result_ex_free(nlb_result_ex* r);

/* ---- Verlet (skin) list manager for MD (asked for by the reference's
 * spec.md:41-48, 64-67, 209-222 as DynamicNeighborManager; not implemented
 * by the reference). ----
 * nlb_verlet_create: cutoff rc, skin >= 0; the stored list is the exact half
 *   list at rc + skin (the nlb_build search) of the reference positions.
 * nlb_verlet_update: host positions in, host result out (free with
 *   nlb_result_free).  Rebuilds (*rebuilt = 1) when there is no list, the
 *   atom count, cell or pbc changed, or max_i |r_i - r_i,ref| > skin / 2;
 *   then returns the stored edges (i, j, S) with |(r_j - r_i) + H.S| < rc for
 *   the given positions, in stored order (the pairs a fresh nlb_build at rc
 *   finds, as long as positions are continuous; re-wrapped atoms force a
 *   rebuild).  One synchronisation per update without a rebuild.
 * nlb_verlet_update_device: device positions in; the result arrays are
 *   device pointers owned by the manager, valid until its next update.
 * nlb_verlet_update_device_owned: as nlb_verlet_update_device, but the two
 *   result arrays are written in place into blocks of the library's
 *   stream-ordered result pool and handed over, exactly like
 *   nlb_build_device_owned's (edge_index [src | dst] in the first 2 M
 *   entries; return each with nlb_device_free; both NULL when M = 0).
 * nlb_verlet_needs_rebuild: *needs and the current max displacement (+inf
 *   when the next update rebuilds anyway); positions_on_device selects the
 *   pointer kind.
 * nlb_verlet_stats: updates, rebuilds, stored edges, edges last returned.
 * A manager is used by one thread at a time (calls are serialised). */
typedef struct nlb_verlet nlb_verlet;
nlb_verlet* nlb_verlet_create(double cutoff, double skin);
int nlb_verlet_update(nlb_verlet* v, const double* positions, int64_t n_atoms, const double* cell,
                      const uint8_t* pbc, int* rebuilt, nlb_result* out);
int nlb_verlet_update_device(nlb_verlet* v, const double* d_positions, int64_t n_atoms,
                             const double* cell, const uint8_t* pbc, int* rebuilt,
                             nlb_device_result* out);
int nlb_verlet_update_device_owned(nlb_verlet* v, const double* d_positions, int64_t n_atoms,
                                   const double* cell, const uint8_t* pbc, int* rebuilt,
                                   nlb_device_result* out);
int nlb_verlet_needs_rebuild(nlb_verlet* v, const double* positions, int64_t n_atoms,
                             const double* cell, const uint8_t* pbc, int positions_on_device,
                             int* needs, double* max_displacement);
void nlb_verlet_stats(nlb_verlet* v, int64_t* stats);
void nlb_verlet_destroy(nlb_verlet* v);

/* ---- Build without allocating (no counterpart in the reference). ----
 * For callers that must not allocate GPU memory when they ask for a list:
 * processes whose HBM is held by a framework's caching allocator, code that
 * cannot afford cudaFree's device-wide synchronisation, and loops that only
 * allocate at start-up.  Single system, one cutoff, same edges in the same
 * order as nlb_build / nlb_build_device.  The caller passes device positions
 * (n x 3 float64) and device outputs: d_edge_index with room for
 * 2 x max_edges int64 (sources in [0, M), destinations in
 * [max_edges, max_edges + M)) and d_shift with room for max_edges x 3 int32;
 * *n_edges (host) receives M.  All scratch lives in one fixed __device__
 * array inside the library (about 1.8 MB per device, held until exit), so
 * systems are limited to 16384 atoms and 16384 cell-list bins; larger inputs
 * and M > max_edges are rejected with NLB_ERR_VALUE (outputs untouched when
 * M > max_edges; *n_edges still reports M).  The first call on each device
 * looks up the array's device address (make it before any stream capture);
 * after a cudaDeviceReset of that device, do not call it again in the same
 * process.  Calls share the array: calls that overlap on one device race and
 * must be serialised.  Runs on `stream` (a cudaStream_t, NULL = legacy
 * default), synchronises that stream twice (after the count pass and after
 * the emit pass) and returns after the results are complete. */
int nlb_build_noalloc(const double* d_positions, int64_t n_atoms, double cutoff,
                      const double* cell, const uint8_t* pbc, int64_t* d_edge_index,
                      int32_t* d_shift, int64_t max_edges, int64_t* n_edges, void* stream);

/* ---- Served request loop (continuous batching). ----
 * No single counterpart in the reference: it replaces the caller-side loop
 * that calls search_single (src/single.rs:8-89) once per arriving structure.
 * Worker threads (n_workers, each with its own stream and workspace on
 * `device`) take queued requests in arrival order; small requests
 * (<= 2048 atoms) that fit the HBM budget are run together by the batched
 * kernels, each with its own cutoff, and larger ones by the single-system
 * pipeline.  Every result equals nlb_build of the same request.
 *
 * nlb_server_create: hbm_budget_bytes bounds the estimated device footprint
 *   of admitted requests (positions, workspace, edges; device-resident
 *   results stay counted until released); max_batch bounds the systems per
 *   batch.  NULL on error (nlb_last_error).
 * nlb_server_submit: copies the positions; cell/pbc as in nlb_build.
 *   device_result != 0 keeps the result in HBM (nlb_result then holds device
 *   pointers).  Returns a ticket > 0, or -code on a rejected request (invalid
 *   input, or an estimate larger than the whole budget).
 * nlb_server_wait: timeout_s < 0 waits for good.  Returns NLB_OK and fills
 *   *out (and *latency_ms, submit -> done) when the request finished,
 *   NLB_NOT_READY on timeout, or the request's error code (nlb_last_error
 *   has its message).  Host results then belong to the caller (nlb_result_free) and
 *   the ticket is retired; device results stay owned by the server until
 *   nlb_server_release, which the caller issues once its own work reading
 *   them has completed.
 * nlb_server_stats: fills 16 counters: submitted, completed, failed, batches,
 *   HBM bytes reserved, queued requests, largest batch, budget, then worker
 *   wall time in microseconds (all workers) spent in: batch staging and
 *   launches, waiting for the count pass, issuing result copies, waiting
 *   for the emit pass and copies, large requests; then cancelled requests,
 *   the summed admission wait of started requests (submit -> taken by a
 *   worker, microseconds) and the deepest queue seen.
 * nlb_server_pause: paused != 0 stops the workers from taking new work
 *   (requests queue up, running work finishes); 0 resumes.
 * nlb_server_cancel: withdraws a queued request (it never runs) or frees a
 *   finished request's result; the ticket is retired either way.  A running
 *   request cannot be cancelled (NLB_ERR_VALUE, "request still running").
 * nlb_server_debug_fail: failure-detection hook for tests: the staging of
 *   any batch holding this queued request fails as if a CUDA call had
 *   returned an error; the worker reruns that batch one request at a time,
 *   so only this request fails (NLB_ERR_CUDA) and the others complete.
 * nlb_server_create also maps a quarter of the budget (at most 16 GB) of
 *   the workspace pool, so that workers grow into mapped memory.
 * nlb_server_destroy: cancels queued requests, lets running ones finish,
 *   joins the workers (returning their workspaces to the pool) and frees
 *   every result that was not handed over.  No thread may be inside nlb_server_wait then. */
typedef struct nlb_server nlb_server;
nlb_server* nlb_server_create(int device, int64_t hbm_budget_bytes, int n_workers, int max_batch);
int64_t nlb_server_submit(nlb_server* server, const double* positions, int64_t n_atoms,
                          const double* cell, const uint8_t* pbc, double cutoff,
                          int device_result);
int nlb_server_wait(nlb_server* server, int64_t ticket, double timeout_s, nlb_result* out,
                    double* latency_ms);
int nlb_server_release(nlb_server* server, int64_t ticket);
int nlb_server_pause(nlb_server* server, int paused);
int nlb_server_cancel(nlb_server* server, int64_t ticket);
int nlb_server_debug_fail(nlb_server* server, int64_t ticket);
void nlb_server_stats(nlb_server* server, int64_t* stats);
void nlb_server_destroy(nlb_server* server);

/* Cell helpers behind the Python PyCell class (src/python_api.rs:15-99).
 * nlb_cell_check: 0 if H is invertible, NLB_ERR_VALUE ("Cell matrix is not
 * invertible", src/cell.rs:18-21) otherwise.
 * nlb_cell_wrap: Cell::wrap (src/cell.rs:52-72): fractional wrap on the
 * periodic axes only. */
int nlb_cell_check(const double* cell);
int nlb_cell_wrap(const double* cell, const uint8_t* pbc, const double* position, double* out);
/* The batched calls' cell arrays from a (B, 3, 3) stack of ASE cells (rows
 * = lattice vectors; src/python_api.rs:353-407): h9_out (B x 9) receives
 * each cell transposed (columns = lattice vectors, the cells argument of
 * nlb_build_batch), has_out (B) 1 for a cell with a non-zero entry, 0 for an
 * all-zero one (isolated system, auto-box). */
void nlb_batch_cells(const double* ase_cells, int64_t n_cells, double* h9_out, uint8_t* has_out);

/* Library version string. */
const char* nlb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* NEIGHBORLIST_B200_H */
