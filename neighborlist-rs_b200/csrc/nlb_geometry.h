// nlb_geometry.h -- host-side cell geometry and grid planning (C++).
//
// Computes, in the reference's exact f64 operation order, everything the
// kernels take as parameters: H^-1 (nalgebra's 3x3 cofactor inverse),
// perpendicular widths (src/cell.rs:45-50), the auto-box (src/single.rs:21-58),
// mic_safe and the dispatch (src/single.rs:60-89), bins per axis, stencil
// half-widths and the bin geometry used for pruning (src/search.rs:119-152,
// :229-246).  Compiled with -ffp-contract=off.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "nlb_common.cuh"

namespace nlb {

struct HostCell {
  double h[9];
  double hinv[9];
  bool pbc[3];
};

// Returns false (and sets err) when det(H) == 0: "Cell matrix is not invertible".
bool make_cell(const double* h9, const bool pbc[3], HostCell& c, std::string& err);

// Orthorhombic box diag(span + 2 (rc + 1)), origin 0, no periodicity.
bool auto_box(const double* pos, int64_t n, double rc_max, HostCell& c, std::string& err);
// Same, from precomputed per-axis bounds lo[3], hi[3].
bool auto_box_from_bounds(const double* lo, const double* hi, double rc_max, HostCell& c,
                          std::string& err);

void perpendicular_widths(const HostCell& c, double w[3]);

enum class Method : int32_t {
  kBruteIsolated = 0,  // brute_force_search_simd (raw positions, zero shifts)
  kBruteMic = 1,       // brute_force_search_full / _multi (round-based MIC)
  kCellList = 2,       // CellList::build + search
};

// Dispatch of src/single.rs:60-89 / :149-163 (and src/batch.rs:100-124).
// `multi` selects the multi-cutoff brute force, which always takes the MIC
// route (identical distances for an isolated cell).
Method choose_method(const HostCell& c, int64_t n, double rc_max, uint64_t bf_threshold,
                     bool multi);

// Grid for the cell-list path at cutoff rc_max.
void plan_grid(const HostCell& c, double rc_max, GridParams& g);

// Stable ascending order of cutoffs (src/search.rs:354-360).
std::vector<int32_t> cutoff_order(const double* cutoffs, int32_t k);

double fmax_nan_ignoring(double a, double b);
double fmin_nan_ignoring(double a, double b);

}  // namespace nlb
