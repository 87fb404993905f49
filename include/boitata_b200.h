/* boitata_b200 — C ABI of the B200 kriging engine.
 *
 * Plain C, plain pointers and sizes; no CUDA or torch types in the
 * signatures (streams travel as `void*` holding a cudaStream_t). Every
 * entry point returns 0 on success or a negative BTK_E* code; the message of
 * the last failure on a context is btk_last_error(ctx). Nothing here exits,
 * throws or falls back to the CPU: without a usable CUDA device btk_create
 * fails with BTK_ECUDA.
 *
 * The entry points replace the kriging path of gstvschlz/boitata, whose
 * only interface today is the pyo3 estimator (no C ABI exists there):
 *   - btk_fit         crates/py/src/estimation.rs:1244-1311 (`store`) and
 *                     crates/estimation/src/search.rs:759-776 (SearchTree::new)
 *   - btk_predict*    crates/py/src/estimation.rs:1600-1742 (`predict`) ->
 *                     crates/estimation/src/batch.rs:15-38 (estimate_many) ->
 *                     crates/estimation/src/krige.rs:83-95 (krige)
 *   - btk_cross_validate  crates/py/src/estimation.rs:1811-1843 ->
 *                     crates/estimation/src/batch.rs:165-190 (leave_one_out_at)
 *   - btk_neighbors   crates/estimation/src/search.rs:944-982 (neighbors_in)
 *   - btk_centroids   crates/core/src/block_model.rs:76-86, 431-445
 * The parameter structs mirror crates/variogram/src/{composite,model,aniso}.rs
 * and crates/estimation/src/search.rs:31-81.
 */
#ifndef BOITATA_B200_H
#define BOITATA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---- */
#define BTK_OK 0
#define BTK_EINVAL (-1)       /* invalid parameter (reference: InvalidParameters) */
#define BTK_EUNSUPPORTED (-2) /* a reference option this engine does not run */
#define BTK_ECUDA (-3)        /* CUDA error; message in btk_last_error */
#define BTK_ENOTFITTED (-4)   /* predict before fit */
#define BTK_ENOMEM (-5)       /* device allocation failed */

/* ---- per-target status (one int8 per target) ---- */
#define BTK_ST_OK 0
#define BTK_ST_SEARCH_FAILED 1 /* fewer than min_samples (EstimError::SearchFailed) */
#define BTK_ST_SINGULAR 2      /* pivot <= 1e-12 * C(0) (kernel.rs:61) */
#define BTK_ST_UNSUPPORTED 3   /* more samples than the solve path holds */
#define BTK_ST_INVALID 4       /* simple kriging with a power structure (EstimError::InvalidParameters, krige.rs:117-124),
                                  or a caller's neighbour list out of bounds (btk_solve_noalloc) */
#define BTK_RULES_CANDIDATES 512 /* candidates a hole / sector rule search sorts per round */
#define BTK_ST_FP64_FALLBACK 0x10 /* flag: the mixed form re-solved this system in FP64 */

/* ---- variogram models (crates/variogram/src/model.rs:11-30) ---- */
#define BTK_SPHERICAL 0
#define BTK_EXPONENTIAL 1
#define BTK_GAUSSIAN 2
#define BTK_CUBIC 3
#define BTK_PENTASPHERICAL 4
#define BTK_CIRCULAR 5
#define BTK_SINEHOLE 6
#define BTK_MATERN 7 /* param = order */
#define BTK_POWER 8  /* param = exponent; not stationary: solved by the dense LU */
#define BTK_MAX_STRUCT 4

/* ---- kriging kinds (crates/estimation/src/krige.rs:20-27) ---- */
#define BTK_ORDINARY 0
#define BTK_SIMPLE 1    /* kparam = mean */
#define BTK_INDICATOR 2 /* kparam = threshold */

/* ---- precision forms ---- */
#define BTK_FP64 0  /* FP64 throughout */
#define BTK_MIXED 1 /* FP32 factorisation, FP64 residual refinement, Lagrange and variance */

/* Azimuth/dip/rake (degrees) and ranges of an anisotropy
 * (crates/variogram/src/aniso.rs:18-26); on = 0 means none. */
typedef struct {
  int32_t on;
  double azimuth, dip, rake, major, semi, minor;
} btk_aniso;

typedef struct { /* crates/variogram/src/model.rs:33-40 */
  int32_t model;
  double param; /* Matérn order or power exponent, else ignored */
  double sill;
  double range;
} btk_structure;

typedef struct { /* crates/variogram/src/composite.rs:13-18 */
  double nugget;
  int32_t nstruct;
  btk_structure s[BTK_MAX_STRUCT];
  btk_aniso aniso; /* shared by every structure */
} btk_variogram;

/* crates/estimation/src/search.rs:31-81; optional counts are -1 for None. */
typedef struct {
  int64_t min_samples, max_samples;
  double radius;
  int64_t max_per_hole;      /* -1: none; holes from btk_fit */
  int64_t octant;            /* 0/1 */
  int64_t sectors;           /* plane sectors (2..360), 0: none */
  int64_t max_per_sector;    /* plane sectors: samples per sector */
  int64_t max_per_octant;    /* -1: ceil(max_samples / sector count) */
  int64_t min_sectors;       /* -1: none */
  int64_t max_empty_sectors; /* -1: none */
  int64_t min_holes;         /* -1: none; a sample without a hole counts as its own */
  btk_aniso aniso;           /* search ellipsoid; on = 0: the variogram's */
  /* Calibration (search.rs:94-100, crates/py/src/estimation.rs:846-895): each
   * target keeps the fewest leading samples, from min_samples, whose slope of
   * regression (1) or kriging efficiency (2) reaches calibration_target; all
   * of them where none does. With octants or sectors the samples are first
   * taken round-robin over the sectors (search.rs:913-936). 0: none. */
  int64_t calibration;
  double calibration_target;
} btk_search;

/* Block-model parent grid (crates/core/src/block_model.rs:19-26): corner
 * origin, cell size, cell count, azimuth/dip/rake; cells run x fastest. */
typedef struct {
  double origin[3];
  double size[3];
  int64_t count[3];
  double rotation[3];
} btk_geometry;

/* Outputs of a prediction; any pointer but `value` may be NULL. */
typedef struct {
  double* value;
  double* variance;
  double* lagrange;
  int32_t* n_used;
  int8_t* status;
} btk_outputs;

/* Launch tunables (no counterpart in the reference): grid cell size in
 * samples per cell, the block-model tile one search warp serves (product
 * 32), warps per search CTA, resident solve CTAs per SM (0: defaults), and
 * the most distinct samples the tile-shared solve tabulates for 16
 * consecutive targets (32..255; 0: every system assembles its own matrix),
 * for calls with host buffers the targets per chunk of the copy/compute
 * pipeline (0: the whole call at once; at most 8 chunks), and for the mixed
 * form's tile-shared solve whether the factorisation's trailing updates run
 * on the tensor pipe (1: 8-column panels on the CUDA cores, the updates as
 * split-TF32 mma; 0: the unblocked FP32 elimination), and for the mixed
 * form's systems of more than 32 samples which per-system kernel solves them
 * (0: FP32 factorisation with FP64 refinement; 1: the FP64 kernel). */
typedef struct {
  double samples_per_cell;
  int32_t tile[3];
  int32_t search_warps;
  int32_t solve_blocks_per_sm;
  int32_t tile_union;
  int32_t host_chunk;
  int32_t tile_tensor;
  int32_t mixed_large;
} btk_tuning;

typedef struct btk_ctx btk_ctx;

const char* btk_version(void);

/* A context on CUDA device `device` with its own stream and device buffers.
 * One context per host thread. NULL on failure, with the reason in `err`. */
btk_ctx* btk_create(int device, char* err, size_t errlen);
void btk_destroy(btk_ctx* ctx);
const char* btk_last_error(const btk_ctx* ctx);

/* Stores the samples on the device and indexes them for `search`: the
 * projections into the search frame (origin at the first sample) and the
 * uniform grid over them. xyz is n x 3 row-major; err_var and holes may be
 * NULL. The caller has already dropped exact duplicates (the fit rule of
 * crates/py/src/args.rs:318-376). Replaces any earlier fit. */
int btk_fit(btk_ctx* ctx, int64_t n, const double* xyz, const double* values, const double* err_var,
            const int64_t* holes, const btk_search* search, const btk_variogram* vg);

/* A new search (a later pass) over the fitted samples; re-indexes them when
 * its ellipsoid differs. */
int btk_set_search(btk_ctx* ctx, const btk_search* search);

/* The per-target columns of the diagnostics table (crates/py/src/estimation.rs:
 * 1046-1105) that need the samples used or the weights: host arrays of m
 * entries, any of them NULL; NaN (n_holes 0) where a target is not estimated. */
typedef struct btk_diagnostics {
  double* negative_weight_sum; /* sum of the negative weights (Estimate::negative_weight_sum, krige.rs:70-75) */
  double* mean_distance;       /* mean Euclidean distance to the samples used (neighborhood.rs:94-98) */
  int32_t* n_holes;            /* distinct holes among the samples used; an untagged sample counts one
                                  (neighborhood.rs:84-93) */
  int8_t* target_met;          /* calibrated search: 1 where the samples used reach the target, 0 where
                                  even max_samples fall short; -1 without a calibration or estimate */
} btk_diagnostics;

/* Kriging at m targets given as host arrays (xyz m x 3 row-major); outputs
 * are host arrays of m entries. Host-device copies are part of the call. */
int btk_predict(btk_ctx* ctx, int64_t m, const double* xyz, int32_t kind, double kparam, int32_t precision,
                const btk_outputs* out);

/* Sequential Gaussian simulation of grid nodes (crates/simulation/src/sgs.rs:
 * 586-760, `sequential`): the fitted samples are the n_data conditioning data
 * (values = normal scores) followed by the grid nodes in simulation-path
 * order (their fitted values are overwritten). Node j, in that order, is
 * simple-kriged (mean 0, the fitted variogram, which the caller scales to a
 * unit sill) from the data and the nodes before it, and draws
 * score = mean + sqrt(variance) * z[j]; a node whose search finds fewer than
 * min_samples draws z[j]. Nodes run in parallel windows of `batch` (0: sized
 * from the data) whose nodes are searched again when an earlier node of the
 * window was still unsimulated within their reach, so the result is the
 * sequential one for any batch. Outputs (host, one per node): score, and
 * how (1 kriged, 2 marginal; may be NULL); *rounds (may be NULL) counts the
 * parallel rounds. Nodes on a datum (they take its value and draw nothing)
 * and the normal-score transform and its back-transform are the caller's. */
int btk_sgs_simulate(btk_ctx* ctx, int64_t n_data, const double* z, int64_t batch, double* score, int8_t* how,
                     int64_t* rounds);

/* btk_predict plus the diagnostics columns (the estimator's predict with
 * diagnostics=True, crates/py/src/estimation.rs:1734-1737). out->status is
 * required: a second pass re-solves each estimated system for its weights by
 * the dense LU (the weights of every solve form agree to rounding). */
int btk_predict_diagnostics(btk_ctx* ctx, int64_t m, const double* xyz, int32_t kind, double kparam,
                            int32_t precision, const btk_outputs* out, const btk_diagnostics* diag);

/* As btk_predict, with device pointers: d_xyz is 3 arrays (x, y, z) of m
 * doubles laid out back to back; outputs are device arrays; the work is
 * queued on `stream` (a cudaStream_t, NULL for the context's own). */
int btk_predict_device(btk_ctx* ctx, int64_t m, const double* d_xyz, int32_t kind, double kparam,
                       int32_t precision, const btk_outputs* d_out, void* stream);

/* Kriging at the centroids of every cell of `g`, generated on the device;
 * outputs are device arrays of count[0]*count[1]*count[2] entries in cell
 * order, queued on `stream`. */
int btk_predict_geometry_device(btk_ctx* ctx, const btk_geometry* g, int32_t kind, double kparam,
                                int32_t precision, const btk_outputs* d_out, void* stream);

/* As btk_predict / btk_predict_device with a kriging kind per target
 * (BTK_ORDINARY, BTK_SIMPLE or BTK_INDICATOR, one int8 each; host or device
 * array like the coordinates) sharing `kparam` (the simple-kriging mean or
 * the indicator threshold), so ordinary and simple kriging run in one launch.
 * No counterpart in the reference, whose estimator has one kind. */
int btk_predict_kinds(btk_ctx* ctx, int64_t m, const double* xyz, const int8_t* kinds, double kparam,
                      int32_t precision, const btk_outputs* out);
int btk_predict_kinds_device(btk_ctx* ctx, int64_t m, const double* d_xyz, const int8_t* d_kinds, double kparam,
                             int32_t precision, const btk_outputs* d_out, void* stream);

/* Leave-one-out at every fitted sample (host outputs of n entries). */
int btk_cross_validate(btk_ctx* ctx, int32_t kind, double kparam, int32_t precision, const btk_outputs* out);

/* Neighbour lists of m host targets: `idx` (m x max_samples, -1 padded) in
 * selection order, `count` per target, `ok` 1 where the search succeeds.
 * With `loo` set the targets are the n fitted samples themselves (xyz and m
 * ignored), each searched as if it were absent (search.rs:951-982).
 * `domains`: the targets' domain codes when the samples have domains
 * (btk_set_domains), else NULL; ignored with `loo`. */
int btk_neighbors(btk_ctx* ctx, int64_t m, const double* xyz, int32_t loo, const int32_t* domains, int64_t* idx,
                  int32_t* count, int8_t* ok);

/* Hard domains (crates/estimation/src/search.rs:269-288 with no soft
 * boundary; batch.rs:15-38 `domains`): after btk_fit, `codes` gives each
 * fitted sample's domain (n codes >= 0, host; NULL removes the domains).
 * Every later search of a target of domain d then takes only samples of
 * domain d, and leave-one-out takes each sample's own domain. Predictions
 * must then give each target's domain code (btk_predict_ex), a code < 0
 * (a domain without samples) leaving the target unestimated (status
 * BTK_ST_SEARCH_FAILED); the calls without target domains return BTK_EINVAL,
 * as the reference refuses them. The caller drops exact duplicates within a
 * domain only (crates/py/src/estimation.rs:1273-1308); samples of different
 * domains at one location never meet in a search. The gradients and the
 * simulation take samples without domains. */
int btk_set_domains(btk_ctx* ctx, const int32_t* codes);

/* Prediction at m host targets with every option of the reference's
 * estimator call: `kinds` (one int8 kind per target, or NULL for `kind`),
 * `domains` (one domain code per target, required exactly when the samples
 * have domains), outputs as btk_predict and, when `diag` is given (out->status
 * then required), the diagnostics columns as btk_predict_diagnostics. */
int btk_predict_ex(btk_ctx* ctx, int64_t m, const double* xyz, const int8_t* kinds, const int32_t* domains,
                   int32_t kind, double kparam, int32_t precision, const btk_outputs* out,
                   const btk_diagnostics* diag);
/* Kriging weights (weights_many, crates/estimation/src/batch.rs:76-95, as
 * the estimator's weight declustering calls it, crates/py/src/estimation.rs:
 * 1509-1585): btk_predict_ex's outputs at m host targets (out->value and
 * out->status required; `domains` as btk_predict_ex), and for each target
 * estimated its list (idx, m x max_samples, -1 past the samples used) and
 * the weight of each listed sample (weights, m x max_samples, 0 past them;
 * spread over coincident clusters as the estimate spreads them). Rows of
 * targets not estimated are -1 and 0. The weights come from the dense-LU
 * diagnostics pass in FP64, whatever `precision` the estimates take. */
int btk_predict_weights(btk_ctx* ctx, int64_t m, const double* xyz, int32_t kind, double kparam, int32_t precision,
                        const int32_t* domains, const btk_outputs* out, int64_t* idx, double* weights);
/* The same with device arrays (d_xyz as btk_predict_device), queued on `stream`. */
int btk_predict_ex_device(btk_ctx* ctx, int64_t m, const double* d_xyz, const int8_t* d_kinds,
                          const int32_t* d_domains, int32_t kind, double kparam, int32_t precision,
                          const btk_outputs* d_out, void* stream);

/* Centroids of cells [first, first + m) of `g` into host xyz (m x 3). */
int btk_centroids(btk_ctx* ctx, const btk_geometry* g, int64_t first, int64_t m, double* xyz);

/* Leave-one-out loss and its gradient with respect to the variogram. This
 * has no counterpart in the reference, which computes leave-one-out
 * estimates (batch.rs:165-190) but no gradient of them.
 * btk_loo_freeze runs the leave-one-out search of the fitted samples once
 * and keeps each sample's neighbour list (at most 64), so every later loss
 * and gradient uses those neighbourhoods, whatever variogram it is given.
 * btk_loo_gradient evaluates, for the variogram `vg` (same structure count
 * and models as needed, any parameters), the mean squared leave-one-out
 * error of ordinary kriging over the samples whose system is solvable and
 * holds no coincident samples (*n_valid of them), and, when want_grad is
 * set, its gradient in the order: nugget, sill of each structure, major
 * range of each structure, semi/major ratio, minor/major ratio, azimuth,
 * dip, rake (degrees); 1 + 2 nstruct + 5 values. A variogram without
 * anisotropy is taken as ratios 1, 1 and angles 0. `values` (n, or NULL)
 * receives the leave-one-out estimates. `precision`: BTK_FP64 (FP64
 * factorisation), or BTK_MIXED (FP32 factorisation refined in FP64 until the
 * solutions are good to about 1e-8, FP64 gradient accumulation; systems
 * whose refinement does not converge are solved in FP64). */
int btk_loo_freeze(btk_ctx* ctx);
int btk_loo_gradient(btk_ctx* ctx, const btk_variogram* vg, int32_t want_grad, int32_t precision, double* loss,
                     double* grad, int64_t* n_valid, double* values);

/* The same over the left-out samples first .. first + count - 1 only, as
 * sums for a reduction across ranks: sums[0] = sum of squared errors,
 * sums[1] = systems in the loss, sums[2 + k] = gradient sum of parameter k
 * (zero without want_grad); 2 + 1 + 2 nstruct + 5 values. The loss over a
 * partition of the samples is sum(sums[0]) / sum(sums[1]), and the gradient
 * sum(sums[2 + k]) / sum(sums[1]). */
int btk_loo_gradient_range(btk_ctx* ctx, const btk_variogram* vg, int64_t first, int64_t count, int32_t want_grad,
                           int32_t precision, double* sums);

/* The mean ordinary-kriging estimate of a block model and its gradient with
 * respect to the variogram; no counterpart in the reference. btk_mean_freeze
 * runs the search at every centroid of `g` (cell order, as
 * btk_predict_geometry_device) once and keeps each list (at most 64
 * samples), so later calls krige from those neighbourhoods whatever
 * variogram they are given. btk_mean_gradient gives the mean of the point
 * estimates over the centroids whose system is solvable and holds no
 * coincident samples (*n_valid), its gradient (the parameter order of
 * btk_loo_gradient) when want_grad is set, and the estimates themselves in
 * `values` (one per cell, NaN where none, or NULL). The FP64 objective
 * equals the mean of btk_predict_geometry_device's FP64 values to the bit.
 * btk_mean_gradient_range gives the sums over cells first .. first + count
 * - 1, as btk_loo_gradient_range does (sums[0] = sum of the estimates). */
int btk_mean_freeze(btk_ctx* ctx, const btk_geometry* g);
int btk_mean_gradient(btk_ctx* ctx, const btk_variogram* vg, int32_t want_grad, int32_t precision, double* mean,
                      double* grad, int64_t* n_valid, double* values);
int btk_mean_gradient_range(btk_ctx* ctx, const btk_variogram* vg, int64_t first, int64_t count, int32_t want_grad,
                            int32_t precision, double* sums);

/* Kernel launches issued by this context since it was created. */
int64_t btk_launch_count(const btk_ctx* ctx);

/* Block support for this context's later predictions (block kriging,
 * replacing BlockKriging / Method::Block: crates/py/src/estimation.rs:
 * 1414-1439 and 775-784, crates/estimation/src/block.rs:40-198). Each
 * target is then a block centre: the block of `size` (along the axes turned
 * by `rotation`, azimuth/dip/rake in degrees, NULL for none) is discretized
 * into disc[0] x disc[1] x disc[2] points, each sample's covariance with
 * the target is its mean covariance with those points (nugget left out at
 * zero lag), and the variance is C(B,B) - sum w C(x, B) - mu. One point is
 * point kriging. size NULL returns to point support. Cross-validation stays
 * at point support. At most BTK_MAX_SUPPORT_POINTS points. */
#define BTK_MAX_SUPPORT_POINTS 4096
int btk_set_support(btk_ctx* ctx, const double* size, const int32_t* disc, const double* rotation);
/* C(B,B) of the current support for the fitted variogram (C(0) for point
 * support): the reference's support_variance. */
int btk_support_variance(btk_ctx* ctx, double* out);

/* Tunables of this context; setting samples_per_cell re-indexes the fitted
 * samples. boitata_b200/autotune.py picks them by timing candidates. */
int btk_get_tuning(const btk_ctx* ctx, btk_tuning* out);
int btk_set_tuning(btk_ctx* ctx, const btk_tuning* tuning);

/* Captures btk_predict_geometry_device(g, ...) (centroids, search,
 * bucketing, solves, FP64 re-solves) into one CUDA graph held by the context;
 * btk_graph_launch replays it on `stream` (NULL: the context's stream),
 * writing the same d_out. No counterpart in the reference. */
int btk_graph_capture_geometry(btk_ctx* ctx, const btk_geometry* g, int32_t kind, double kparam,
                               int32_t precision, const btk_outputs* d_out);
/* The same for m device targets d_xyz (as btk_predict_device): with d_kinds
 * (one int8 kind per target, device) btk_predict_kinds_device is captured,
 * else btk_predict_device with `kind`. The graph reads d_xyz and d_kinds on
 * every replay, so the caller may change their contents between replays. */
int btk_graph_capture_device(btk_ctx* ctx, int64_t m, const double* d_xyz, const int8_t* d_kinds, int32_t kind,
                             double kparam, int32_t precision, const btk_outputs* d_out);
int btk_graph_launch(btk_ctx* ctx, void* stream);

/* Kriging without any allocation. This entry point has no counterpart in the
 * reference. It is for callers that cannot call cudaMalloc: a host that owns
 * every device allocation (its own arena or pool allocator, a fixed device
 * memory budget) or a plugin running inside another program's CUDA context.
 * The caller passes device buffers for every input and output:
 *   - n_samples samples d_x, d_y, d_z, d_values and d_err (NULL: no
 *     measurement error);
 *   - m targets d_tx, d_ty, d_tz;
 *   - each target's neighbour list d_nbr (m x max_samples sample indices, as
 *     btk_neighbors gives them), its length d_count and its search status
 *     d_status (BTK_ST_OK, or BTK_ST_SEARCH_FAILED);
 *   - outputs d_out, as for btk_predict_device.
 * It solves the systems in the mixed form (BTK_MIXED, FP64 re-solve where
 * needed) on `stream`, with the results of btk_predict_device; coincident
 * samples are detected within each system. The lists are checked on the
 * device: a count above max_samples, or an index at or past n_samples, fails
 * that target with BTK_ST_INVALID and nothing past the buffers is read.
 * Its only scratch is a static device array of BTK_NOALLOC_MAX_SYSTEMS + 1
 * int64 (2 MiB), held by every GPU that loads the library until the process
 * exits. Limits: at most BTK_NOALLOC_MAX_SYSTEMS systems per call (more
 * return BTK_EINVAL: split the call) and at most 32 samples per system. Each
 * call looks the array's address up in the current CUDA context
 * (cudaGetSymbolAddress); the first lookup in a context loads the module, so
 * make the first call there before capturing a stream. Every call shares the
 * array, so calls that overlap on the GPU race: serialise them on one stream.
 * `device` is made current for the call and the caller's device restored
 * afterwards; `err` (may be NULL) receives the reason of a failure. */
#define BTK_NOALLOC_MAX_SYSTEMS 262144
int btk_solve_noalloc(int device, const btk_variogram* vg, int32_t kind, double kparam, const double* d_x,
                      const double* d_y, const double* d_z, const double* d_values, const double* d_err,
                      int64_t n_samples, int64_t m, const double* d_tx, const double* d_ty, const double* d_tz,
                      const uint32_t* d_nbr, int32_t max_samples, const int32_t* d_count,
                      const int8_t* d_status, const btk_outputs* d_out, void* stream, char* err,
                      size_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* BOITATA_B200_H */
