// Internal host/device interface of the B200 kriging engine: the parameter
// blocks the kernels take by value and the launchers the C ABI calls.
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "boitata_b200.h"

namespace btk {

constexpr int kMaxN = 64;       // most samples per system of the warp kernels (kernel.rs:11)
constexpr int kMaxLU = 128;     // most samples per system of the dense LU with its matrix in shared memory
constexpr int kMaxLUGlobal = 1024;  // most samples per system of the dense LU (krige.rs:127-201), the matrix in global memory
constexpr int kMaxSlots = 64;   // most list entries per search lane
constexpr double kPivot = 1e-12;  // kernel.rs:17
constexpr double kEps = 1e-6;     // coincident.rs:11

// Variogram with everything the kernels need precomputed on the host.
struct VgDev {
  double nugget, c0;
  int nstruct;
  int model[BTK_MAX_STRUCT];
  double param[BTK_MAX_STRUCT], sill[BTK_MAX_STRUCT], inv_range[BTK_MAX_STRUCT];
  int has_frame;
  double frame[9];  // diag(1/major, 1/semi, 1/minor) * rotation (aniso.rs:88-94)
  int stationary;   // no power structure (composite.rs:64-66)
};

// Search parameters in the form the search kernel uses.
struct SearchDev {
  double radius2;
  int min_samples, max_samples;
  int nsec;  // 1 without balancing, 4 quadrants, 8 octants
  int cap;   // per-sector list length: min(sector cap, max_samples)
  int planar;
  double axes[9];   // block_frame of the search ellipsoid (octant signs)
  double frame[9];  // projection into the search space
  double origin[3];  // first sample (search.rs:704-745)
  // Sector bit k of a sample is (approximately) bit_sign[k] * dp[bit_axis[k]] >= 0
  // for its offset dp from the target in the search frame: sectors are
  // orthants of the grid axes, which lets the search prune cells by sector.
  int nbits;
  int bit_axis[3], bit_sign[3];
  unsigned bit_mask[3];  // sectors whose index has bit k set
  // Hole and sector rules (search.rs:476-577). When `rules` is set the
  // search runs the reference's greedy selection over each target's nearest
  // candidates (k_search_rules) instead of the per-sector lists.
  int rules;
  int64_t max_per_hole;                            // -1: none
  int min_sectors, max_empty_sectors, min_holes;   // -1: none
  int plane;     // plane sector count (2..360), 0: octants / quadrants or none
  int balances;  // octants or plane sectors
  int rsec;      // sector count when balancing
  int rcap;      // samples per sector when balancing
  const uint32_t* hole;        // hole code per sample, original order; null: each sample its own hole
  const double *sx, *sy, *sz;  // sample world coordinates, original order
  // Sequential simulation (btk_sgs_simulate): samples from sgs_node0 on are
  // grid nodes in simulation order, and target t is node sgs_node0 + t. A
  // target sees the data and the earlier nodes already simulated (sgs_done);
  // an earlier node not yet simulated within the search's reach makes the
  // target stale (kStStale), to be searched again once that node is done.
  int sgs;
  uint32_t sgs_node0;
  const uint8_t* sgs_done;
  // Hard domains (search.rs:269-288 with no soft boundary): a target of
  // domain tdom[t] takes only samples of its own domain sdom[i] (codes >= 0;
  // a target code < 0, a domain without samples, takes none). Run by
  // k_search_rules. Null: no domains.
  const int32_t* sdom;
  const int32_t* tdom;
};

// Internal per-target status of a simulation search: searched too early.
constexpr int8_t kStStale = 5;

// Uniform grid over the projected samples, which are stored sorted by cell.
struct GridDev {
  double lo[3];
  double h;
  int dims[3];
  int64_t ncells;
  double slack;  // absolute margin on cell-face distances
  const uint32_t* start;  // ncells + 1
  const double *px, *py, *pz;  // projected, cell order
  const double *wx, *wy, *wz;  // world, cell order
  const uint32_t* idx;         // original sample index, cell order
};

// Everything a solve launch reads and writes.
struct SolveDev {
  VgDev vg;
  int kind;
  double kparam;
  const int8_t* kinds;  // per-target kind (ordinary / simple / indicator), or null for `kind`
  int max_samples;
  const double *sx, *sy, *sz, *sv, *se;  // samples, original order; se may be null
  const uint8_t* twin;                    // 1 where another sample lies within 1e-6 m
  const double *tx, *ty, *tz;            // targets, by target index
  const uint32_t* nbr;                   // [target][max_samples]
  const int32_t* count;
  const int8_t* sstatus;
  // Caller-supplied lists (btk_solve_noalloc): > 0, the number of samples;
  // the pair-testing kernels then check every neighbour index against it and
  // every count against max_samples, and fail the system (BTK_ST_INVALID)
  // instead of reading past the caller's buffers. 0: lists from the search.
  int64_t nsamples;
  const int64_t* list;      // systems of this bucket (target indices), or null for 0..m-1
  const int64_t* list_len;  // device count of `list`
  int64_t m;
  double *value, *variance, *lagrange;
  int32_t* n_used;
  int8_t* status;
  // Block support (block kriging): sup_n discretization offsets (x, y, z
  // triples, world frame) around each target, and the block's mean
  // covariance C(B,B) on the device; sup_n == 0 for point support.
  const double* sup;
  int sup_n;
  const double* sup_cbb;
  // Dense LU path: systems of more than 64 samples go to `lu` (count at
  // *lu_len); the LU kernel over every target walks `perm` (work slots, -1
  // padding) when it is set, else targets 0 .. m-1.
  int64_t *lu, *lu_len;
  const int64_t* perm;
  int64_t nwork;
  double* lu_scratch;  // systems beyond kMaxLU samples: lu_scratch_doubles() for the LU's matrices
  // Diagnostics pass (the LU kernel's `diag` form): per-target columns, and
  // the fitted samples' hole codes (null: every sample untagged).
  double *negw, *mdist;
  int32_t* nholes;
  const uint32_t* hole;
  // The same pass's kriging weights, [target][max_samples] in list order and
  // spread over coincident clusters as the estimate spreads them (null: not
  // wanted); rows of targets it does not estimate are left as they are.
  double* wout;
};

// Tile-shared solve (btk_tile.cu): the systems of kTileTargets consecutive
// work slots share one covariance table over the union of their samples.
constexpr int kTileTargets = 16;
struct TileDev {
  SolveDev s;           // system inputs and outputs (s.list unused)
  const int64_t* perm;  // work slot -> target index, -1 for padding; null: identity
  int64_t nwork;
  int umax;             // most distinct samples a tile's table holds
  int stride;           // row stride of the table, in doubles
  int64_t *small, *small_len;  // n <= 32 systems left to the per-system kernels
  int64_t *large, *large_len;  // n > 32
  int64_t *redo, *redo_len;    // mixed form: systems left to the FP64 re-solve
};

// A kriging objective and its gradient over frozen neighbourhoods
// (btk_adjoint.cu): the leave-one-out loss (system i is the fitted sample
// first + i, kriged from its leave-one-out list) or the mean estimate of a
// block model (system i is the target first + i).
struct GradDev {
  VgDev vg;         // the variogram at theta; vg.frame = M(theta), always set
  double dM[5][9];  // dM/d(semi, minor, azimuth, dip, rake), degrees for angles
  const double *sx, *sy, *sz, *sv, *se;
  const uint8_t* twin;
  const double *tx, *ty, *tz;  // mean objective: the targets; null: leave-one-out
  const uint32_t* nbr;
  const int32_t* count;
  const int8_t* sstatus;
  int max_samples;
  int64_t first;  // systems first .. first + n - 1
  int64_t n;
  const int64_t* list;      // FP64 pass over the systems the mixed pass left (offsets i), or null: all n
  const int64_t* list_len;
  int64_t *redo, *redo_len;  // mixed pass: systems left to the FP64 pass
  int want_grad;
  int stride;     // 2 + number of parameters
  double* part;   // [n][stride]: objective term, valid flag, gradient terms
  double* value;  // the systems' estimates (indexed first + i), or null
};

// ---- launchers (each returns the launch's error, if any) ----
// Tunables the autotuner picks (btk_tuning).
struct Tuning {
  int tile[3] = {4, 4, 2};       // block-model tile of one search warp (product 32)
  int search_warps = 0;          // warps per search CTA; 0: 4 (2 with 64 list slots)
  int solve_blocks_per_sm = 0;   // resident solve CTAs per SM; 0: as many as fit
  int tile_union = 64;           // tile-shared solve: most distinct samples per tile; 0: per-system solve
                                 // (64 lets four mixed-form CTAs share an SM; a tile above it is split)
  int host_chunk = 0;            // host-buffer calls: targets per pipelined chunk; 0: one chunk
  int tile_tensor = 0;           // mixed tile solve: 1 = trailing updates on the tensor pipe (split TF32)
  int mixed_large = 0;           // mixed form: 1 = systems above 32 samples by the FP64 per-system kernel
};

struct Launch {
  cudaStream_t stream;
  int sm_count;
  int64_t* counter;  // launches issued, for btk_launch_count
  Tuning tuning;
};

struct Frame9 {
  double m[9];
};

cudaError_t launch_project(const Launch& L, int64_t n, const double* x, const double* y, const double* z,
                           const double* frame, const double* origin, double* px, double* py, double* pz);
cudaError_t launch_bounds(const Launch& L, int64_t n, const double* px, const double* py, const double* pz,
                          double* partial /* 6 * 1024 */, double* out6);
// Temporary bytes of the grid build's stable sort of the samples by cell.
size_t grid_sort_temp_bytes(int64_t n, int64_t ncells);
cudaError_t launch_grid_build(const Launch& L, int64_t n, const double* x, const double* y, const double* z,
                              const double* px, const double* py, const double* pz, GridDev g, uint32_t* count,
                              uint32_t* start, uint32_t* cell_of, double* spx, double* spy, double* spz,
                              double* swx, double* swy, double* swz, uint32_t* sidx, uint32_t* sort_keys,
                              uint32_t* sort_vals, void* temp, size_t temp_bytes);
cudaError_t launch_twins(const Launch& L, int64_t n, GridDev g, int reach, const double* x, const double* y,
                         const double* z, uint8_t* twin);
cudaError_t launch_centroids(const Launch& L, btk_geometry g, Frame9 frame_t, int64_t first, int64_t m,
                             double* tx, double* ty, double* tz, int64_t* perm_tiles);
cudaError_t launch_search(const Launch& L, const SearchDev& sp, const GridDev& g, const double* tx,
                          const double* ty, const double* tz, const int64_t* perm, int64_t m, int loo,
                          uint32_t* nbr, int32_t* count, int8_t* status);
cudaError_t launch_bucket(const Launch& L, int64_t m, const int32_t* count, const int8_t* sstatus, int64_t* lists,
                          int64_t* lens);
// FP64 form; rows 32 (a warp per system) or 64 (a warp pair).
cudaError_t launch_solve(const Launch& L, const SolveDev& a, int rows);
// Mixed form; systems it leaves to FP64 are appended to redo / *redo_len.
cudaError_t launch_solve_mixed(const Launch& L, const SolveDev& a, int rows, int64_t* redo, int64_t* redo_len);
// FP64 re-solve of the redo list (a.list / a.list_len point at it).
cudaError_t launch_solve_redo(const Launch& L, const SolveDev& a, int rows);

// As launch_solve_mixed / launch_solve_redo for n <= 32, testing each
// system's own sample pairs for coincidence instead of reading a.twin.
cudaError_t launch_solve_mixed_pairs(const Launch& L, const SolveDev& a, int64_t* redo, int64_t* redo_len);
cudaError_t launch_solve_redo_pairs(const Launch& L, const SolveDev& a);

// Tile-shared solve of every work slot's system with n <= 32 (mixed: FP32
// factor with FP64 refinement, else FP64); the others go to a.small / a.large
// (and, mixed, a.redo) for the per-system kernels. Counts must start at 0.
cudaError_t launch_tile(const Launch& L, const TileDev& a, bool mixed);

// Work-slot permutation of m caller-supplied targets in Hilbert order of
// their positions, axis d weighted by w[d] (btk_order.cu). keys and vals
// hold 2m entries each; temp holds morton_temp_bytes(m). *perm points into
// vals on return.
size_t morton_temp_bytes(int64_t m);
// lat: 4 scratch words (the lattice steps and its off flag): targets on an
// axis-aligned lattice take the block-model path's order, tiles of
// L.tuning.tile in Hilbert order.
cudaError_t launch_morton_order(const Launch& L, int64_t m, const double* x, const double* y, const double* z,
                                const double w[3], double* partial, double* b6, unsigned long long* lat,
                                uint64_t* keys, int64_t* vals, void* temp, size_t temp_bytes, const int64_t** perm);

// C(B,B) of a block discretized by nd offsets (x, y, z triples) into *cbb:
// the mean over pairs of point covariances with the nugget left out at zero
// lag; the total sill for one point (btk_support.cu).
cudaError_t launch_support_cbb(const Launch& L, const VgDev& vg, const double* off, int nd, double* cbb);

// FP64 dense LU of the bordered system (btk_lu.cu) for the systems of
// a.list (or every target, through a.perm / a.nwork when a.list is null),
// at most kmax (<= kMaxLU) samples each.
// Search calibration (btk_calibrate.cu): cuts each target's count to the
// fewest leading samples that reach the target quality, after reordering the
// list round-robin over the sectors when `balance` is set.
struct CalDev {
  int32_t* count;
  uint32_t* nbr;
  int8_t* met;      // 1 met, 0 not met, -1 not calibrated (search failed)
  int calibration;  // 1 slope of regression, 2 kriging efficiency
  double target;
  int min_samples;
  int balance;
};
cudaError_t launch_calibrate(const Launch& L, const SolveDev& a, const SearchDev& sp, const CalDev& c, int kmax);

// Sequential simulation (btk_sgs.cu): the window's nodes still to simulate,
// in order, and the commit of a round's kriged nodes.
cudaError_t launch_sgs_pending(const Launch& L, int64_t first, int64_t last, uint32_t node0, const uint8_t* done,
                               int64_t* list, int64_t* len);
cudaError_t launch_sgs_commit(const Launch& L, int64_t nwork, const int64_t* list, const double* mean,
                              const double* var, const int8_t* status, const double* z, uint32_t node0, double* sv,
                              uint8_t* done, double* score, int8_t* how, int64_t* failed);

// With `diag`, the estimated systems (status OK) are solved again for their
// weights and only a.negw / a.mdist / a.nholes are written.
cudaError_t launch_solve_lu(const Launch& L, const SolveDev& a, int kmax, bool diag = false);
// Doubles of global scratch launch_solve_lu needs for systems of kmax samples (0 up to kMaxLU).
size_t lu_scratch_doubles(int sm_count, int kmax);

// Objective and gradient of systems of at most `rows` (32 or 64) samples,
// FP64 or mixed (FP32 factorisation with FP64 refinement; the systems it
// does not converge on are redone in FP64, so a.redo must hold a.n entries
// and a.redo_len one); sums[stride] receives the column sums of a.part.
cudaError_t launch_grad(const Launch& L, const GradDev& a, double* sums, int rows, bool mixed);

// Checks a variogram as btk_fit does and fills its device form; on failure
// returns a BTK_E* code with the reason in *why.
int prepare_variogram(const btk_variogram* vg, VgDev* out, std::string* why);

// FLOP/s of a CUDA-core FMA loop (fp64 != 0: double, else float).
double measure_fma_flops(cudaStream_t s, int sm_count, int fp64, int64_t* counter);

}  // namespace btk
