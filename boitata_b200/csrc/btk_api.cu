// C ABI of the B200 kriging engine: contexts, device buffers, parameter
// checks and the fit / predict / cross-validate pipelines.
//
// Host-side math here is the one-off frame set-up of a call (3x3 matrices);
// every per-sample and per-target step runs in the CUDA kernels. There is no
// CPU path for the kriging itself.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "boitata_b200_measure.h"
#include "btk_internal.h"

namespace {

using namespace btk;

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr, n = 0;
  }
  cudaError_t grow(size_t want) {
    if (want <= n) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, sizeof(T) * (want > 0 ? want : 1));
    if (e == cudaSuccess) n = want;
    return e;
  }
};

// ---- 3x3 frames (crates/core/src/rotation.rs:8-43, aniso.rs:88-94) ----
// Products accumulate column by column as nalgebra's gemv does, so the
// search frame is the reference's to the last bit.
struct M3 {
  double m[3][3];
};

M3 eye() {
  M3 r{};
  r.m[0][0] = r.m[1][1] = r.m[2][2] = 1.0;
  return r;
}

M3 mul(const M3& a, const M3& b) {
  M3 r{};
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      double y = a.m[i][0] * b.m[0][j];
      y = a.m[i][1] * b.m[1][j] + y;
      y = a.m[i][2] * b.m[2][j] + y;
      r.m[i][j] = y;
    }
  return r;
}

M3 rows(double a, double b, double c, double d, double e, double f, double g, double h, double i) {
  M3 r;
  r.m[0][0] = a, r.m[0][1] = b, r.m[0][2] = c, r.m[1][0] = d, r.m[1][1] = e, r.m[1][2] = f;
  r.m[2][0] = g, r.m[2][1] = h, r.m[2][2] = i;
  return r;
}

M3 rotation(double az, double dip, double rake) {
  const double k = 3.14159265358979323846 / 180.0;  // f64::to_radians
  double sa = std::sin(az * k), ca = std::cos(az * k), sd = std::sin(dip * k), cd = std::cos(dip * k);
  double sr = std::sin(rake * k), cr = std::cos(rake * k);
  M3 r1 = rows(sa, ca, 0.0, -ca, sa, 0.0, 0.0, 0.0, 1.0);
  M3 r2 = rows(cd, 0.0, -sd, 0.0, 1.0, 0.0, sd, 0.0, cd);
  M3 r3 = rows(1.0, 0.0, 0.0, 0.0, cr, sr, 0.0, -sr, cr);
  return mul(mul(r3, r2), r1);
}

M3 block_frame(double az, double dip, double rake) {
  M3 r = rotation(az, dip, rake);
  return rows(-r.m[1][0], -r.m[1][1], -r.m[1][2], r.m[0][0], r.m[0][1], r.m[0][2], r.m[2][0], r.m[2][1], r.m[2][2]);
}

M3 aniso_matrix(const btk_aniso& a) {
  M3 d{};
  d.m[0][0] = 1.0 / a.major, d.m[1][1] = 1.0 / a.semi, d.m[2][2] = 1.0 / a.minor;
  return mul(d, rotation(a.azimuth, a.dip, a.rake));
}

void put9(const M3& m, double* out) {
  for (int i = 0; i < 9; ++i) out[i] = m.m[i / 3][i % 3];
}

// block_frame(rotation)^T of a geometry (crates/core/src/block_model.rs:84).
btk::Frame9 transposed_frame(const btk_geometry& g) {
  M3 f = block_frame(g.rotation[0], g.rotation[1], g.rotation[2]);
  btk::Frame9 out;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out.m[3 * i + j] = f.m[j][i];
  return out;
}

// Discretization offsets of a block (crates/estimation/src/block.rs:40-72:
// Discretization::points centred at the origin, i outer and k inner, then
// block_frame(rotation)^T * p in nalgebra's column order).
std::vector<double> block_offsets(const double size[3], const int32_t nd[3], const double rot[3]) {
  const M3 f = block_frame(rot[0], rot[1], rot[2]);
  const double dx = size[0] / double(nd[0]), dy = size[1] / double(nd[1]), dz = size[2] / double(nd[2]);
  const double x0 = 0.0 - size[0] / 2.0 + dx / 2.0, y0 = 0.0 - size[1] / 2.0 + dy / 2.0,
               z0 = 0.0 - size[2] / 2.0 + dz / 2.0;
  std::vector<double> out;
  out.reserve(3 * size_t(nd[0]) * nd[1] * nd[2]);
  for (int i = 0; i < nd[0]; ++i)
    for (int j = 0; j < nd[1]; ++j)
      for (int k = 0; k < nd[2]; ++k) {
        const double p[3] = {x0 + double(i) * dx, y0 + double(j) * dy, z0 + double(k) * dz};
        for (int r = 0; r < 3; ++r) {  // (f^T p)_r = sum_c f[c][r] p_c, column by column
          double y = f.m[0][r] * p[0];
          y = f.m[1][r] * p[1] + y;
          y = f.m[2][r] * p[2] + y;
          out.push_back(y);
        }
      }
  return out;
}

}  // namespace

struct btk_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  int64_t launches = 0;
  std::string err;
  double ppc = 2.0;  // samples per grid cell

  bool fitted = false;
  int64_t n = 0;
  bool has_err = false, planar = false;
  btk_search search{};
  btk_variogram vg{};
  VgDev vgd{};
  SearchDev spd{};
  GridDev gd{};
  std::vector<double> host_z;  // sample elevations, for the planar test

  DevBuf<double> x, y, z, v, e, px, py, pz, spx, spy, spz, swx, swy, swz, bpart, b6, frame9, origin3;
  DevBuf<uint32_t> sidx, start, cell_count, cell_of;
  DevBuf<uint8_t> twin;
  DevBuf<int64_t> loo_perm;
  DevBuf<uint32_t> gsort_keys, gsort_vals;  // stable sort of the samples by cell
  DevBuf<unsigned char> gsort_temp;

  // per-call scratch, grown on demand
  DevBuf<double> txyz, aos;
  DevBuf<double> wts;  // btk_predict_weights: [target][max_samples] kriging weights
  DevBuf<int64_t> perm, lists, lens, redo, redo_len;
  DevBuf<uint32_t> nbr;
  DevBuf<int32_t> cnt, o_nused;
  DevBuf<int8_t> sst, o_status, kinds;
  DevBuf<double> o_value, o_var, o_lag, o_negw, o_mdist;
  DevBuf<int32_t> o_nholes;
  DevBuf<int8_t> met, o_met;  // calibration: target met per work slot target
  // sequential simulation
  DevBuf<double> sg_z, sg_score;
  DevBuf<uint8_t> sg_done;
  DevBuf<int8_t> sg_how;
  DevBuf<int64_t> sg_list, sg_ctl;  // ctl: pending count, first failed node

  bool timing = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  // leave-one-out neighbourhoods frozen for the gradient
  bool frozen = false;
  DevBuf<uint32_t> loo_nbr;
  DevBuf<int32_t> loo_cnt;
  DevBuf<int8_t> loo_sst;
  DevBuf<double> g_part, g_sums, g_val;
  DevBuf<int64_t> g_redo;  // mixed form: systems left to the FP64 pass, and their count
  // block-model neighbourhoods frozen for the mean-estimate gradient
  int64_t mean_m = 0;
  DevBuf<double> mean_txyz;
  DevBuf<uint32_t> mean_nbr;
  DevBuf<int32_t> mean_cnt;
  DevBuf<int8_t> mean_sst;

  // pipelined host calls: copies in and out on their own streams
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t cev[16] = {};

  // spatial order of caller-supplied targets (btk_order.cu)
  DevBuf<uint64_t> ord_keys;
  DevBuf<int64_t> ord_vals;
  DevBuf<uint8_t> ord_temp;
  DevBuf<double> ord_part, ord_b6;
  DevBuf<unsigned long long> ord_lat;  // lattice steps of caller targets and their off flag

  // hole codes of the fitted samples (btk_fit), for the search's hole rules
  DevBuf<uint32_t> hole;
  bool has_hole = false;

  // the dense LU's matrices for systems beyond 128 samples
  DevBuf<double> lu_scratch;

  // domain codes of the fitted samples (btk_set_domains) and of a call's targets
  DevBuf<int32_t> dom, tdom;
  bool has_dom = false;

  // block support (btk_set_support): discretization offsets, C(B,B)
  DevBuf<double> sup, sup_cbb;
  int sup_n = 0;

  Tuning tuning;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int64_t graph_kernels = 0;

  Launch launch(cudaStream_t s) { return Launch{s ? s : stream, sm_count, &launches, tuning}; }
  void mark(int k, cudaStream_t s) {
    if (timing) cudaEventRecord(ev[k], s);
  }
};

namespace {

int fail(btk_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(ctx, BTK_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

bool fin(double v) { return std::isfinite(v); }

// crates/variogram/src/{composite,model,aniso}.rs validate(). A power
// structure has no sill; its systems go to the dense LU (krige.rs:127-201).
int check_vg(btk_ctx* ctx, const btk_variogram* vg) {
  if (!vg) return fail(ctx, BTK_EINVAL, "variogram is required");
  if (!(vg->nugget >= 0.0 && fin(vg->nugget))) return fail(ctx, BTK_EINVAL, "nugget must be finite and >= 0");
  if (vg->nstruct < 0 || vg->nstruct > BTK_MAX_STRUCT)
    return fail(ctx, BTK_EUNSUPPORTED, "at most 4 nested structures");
  for (int k = 0; k < vg->nstruct; ++k) {
    const btk_structure& s = vg->s[k];
    if (!(s.sill >= 0.0 && fin(s.sill) && s.range > 0.0 && fin(s.range)))
      return fail(ctx, BTK_EINVAL, "structure sill must be finite and >= 0, range finite and > 0");
    if (s.model < BTK_SPHERICAL || s.model > BTK_POWER) return fail(ctx, BTK_EINVAL, "unknown variogram model");
  }
  const btk_aniso& a = vg->aniso;
  if (a.on && (!(a.major > 0 && a.semi > 0 && a.minor > 0) || !fin(a.major) || !fin(a.semi) ||
               !fin(a.minor) || !fin(a.azimuth) || !fin(a.dip) || !fin(a.rake)))
    return fail(ctx, BTK_EINVAL, "anisotropy ranges must be finite and > 0, angles finite");
  return BTK_OK;
}

// The samples a system can hold: max_samples, or the fitted samples when there
// are fewer (but never below min_samples or min_holes, which keep their meaning).
int64_t held_samples(const btk_search& s, int64_t n) {
  return std::min(s.max_samples, std::max(n, std::max(s.min_samples, s.min_holes)));
}

// crates/estimation/src/search.rs:214-264, plus the options not run here. The
// support limits apply to what a system can hold with n fitted samples.
int check_search(btk_ctx* ctx, const btk_search* s, int64_t n = INT64_MAX) {
  if (!s) return fail(ctx, BTK_EINVAL, "search is required");
  if (std::isnan(s->radius) || s->radius <= 0.0 || s->max_samples <= 0 || s->min_samples < 0 ||
      s->min_samples > s->max_samples)
    return fail(ctx, BTK_EINVAL, "need radius > 0 and 1 <= min_samples <= max_samples");
  if (s->sectors > 0 && s->octant) return fail(ctx, BTK_EINVAL, "give octant or sectors, not both");
  if (s->max_per_octant >= 0 && !s->octant) return fail(ctx, BTK_EINVAL, "max_per_octant needs octant");
  if (s->max_per_octant == 0) return fail(ctx, BTK_EINVAL, "max_per_sector must be >= 1");
  const int64_t most = held_samples(*s, n);
  if (most > kMaxLUGlobal)
    return fail(ctx, BTK_EUNSUPPORTED, "more than 1024 samples per system (the dense LU's limit)");
  if (s->calibration && most > kMaxLU)
    return fail(ctx, BTK_EUNSUPPORTED, "a calibrated search of more than 128 samples (its Cholesky's shared-memory limit)");
  if (s->sectors > 0 && (s->sectors < 2 || s->sectors > 360 || s->max_per_sector < 1))
    return fail(ctx, BTK_EINVAL, "sectors need 2 <= count <= 360 and max_per_sector >= 1");
  const bool balances = s->octant || s->sectors > 0;
  if ((s->min_sectors >= 0 || s->max_empty_sectors >= 0) && !balances)
    return fail(ctx, BTK_EINVAL, "min_sectors and max_empty_sectors need octant or sectors");
  if (s->min_holes == 0 || s->min_holes > s->max_samples)
    return fail(ctx, BTK_EINVAL, "min_holes must be at least 1 and at most max_samples");
  if (s->calibration < 0 || s->calibration > 2) return fail(ctx, BTK_EINVAL, "unknown calibration");
  if (s->calibration == 1 && !(std::isfinite(s->calibration_target) && s->calibration_target > 0.0))
    return fail(ctx, BTK_EINVAL, "target_slope must be finite and > 0");
  if (s->calibration == 2 && !(std::isfinite(s->calibration_target) && s->calibration_target <= 1.0))
    return fail(ctx, BTK_EINVAL, "target_efficiency must be finite and <= 1");
  if (s->calibration && s->sectors > 360) return fail(ctx, BTK_EINVAL, "at most 360 sectors");
  const btk_aniso& a = s->aniso;
  if (a.on && (!(a.major > 0 && a.semi > 0 && a.minor > 0) || !fin(a.azimuth) || !fin(a.dip) ||
               !fin(a.rake)))
    return fail(ctx, BTK_EINVAL, "search anisotropy ranges must be finite and > 0, angles finite");
  return BTK_OK;
}

// The search as stored: a max_samples above what a system can hold (fewer
// fitted samples, e.g. the reference's "all of them" idiom) becomes that
// count, with the per-octant cap the original implies made explicit (the
// reference derives it from max_samples, search.rs:488-512), so every target
// selects the same samples and the tables are sized by what a system holds.
btk_search effective_search(const btk_search& s, int64_t n, bool planar) {
  btk_search e = s;
  const int64_t most = held_samples(s, n);
  if (most < s.max_samples) {
    if (e.octant && e.max_per_octant < 0) {
      const int64_t nsec = planar ? 4 : 8;
      e.max_per_octant = std::min(s.max_samples / nsec + (s.max_samples % nsec ? 1 : 0), most);
    }
    e.max_samples = most;
  }
  return e;
}

void make_vgdev(const btk_variogram& vg, VgDev& d) {
  d = VgDev{};
  d.nugget = vg.nugget;
  double sum = 0.0;
  for (int k = 0; k < vg.nstruct; ++k) sum += vg.s[k].sill;  // composite.rs:50-52
  d.c0 = vg.nugget + sum;
  d.nstruct = vg.nstruct;
  for (int k = 0; k < vg.nstruct; ++k) {
    d.model[k] = vg.s[k].model;
    d.param[k] = vg.s[k].param;
    d.sill[k] = vg.s[k].sill;
    d.inv_range[k] = 1.0 / std::fmax(vg.s[k].range, 2.2250738585072014e-308);
  }
  d.has_frame = vg.aniso.on ? 1 : 0;
  put9(vg.aniso.on ? aniso_matrix(vg.aniso) : eye(), d.frame);
  d.stationary = 1;
  for (int k = 0; k < vg.nstruct; ++k)
    if (vg.s[k].model == BTK_POWER) d.stationary = 0;
}

// Search frame and sector set-up (search.rs:343-348, 395-425, 488-512).
void make_searchdev(btk_ctx* ctx) {
  const btk_search& s = ctx->search;
  SearchDev& d = ctx->spd;
  const btk_aniso* metric = s.aniso.on ? &s.aniso : (ctx->vg.aniso.on ? &ctx->vg.aniso : nullptr);
  d.radius2 = s.radius * s.radius;
  d.min_samples = int(s.min_samples);
  d.max_samples = int(s.max_samples);
  d.planar = ctx->planar ? 1 : 0;
  d.nsec = s.octant ? (ctx->planar ? 4 : 8) : 1;
  int64_t cap = s.octant ? (s.max_per_octant >= 0 ? s.max_per_octant : (s.max_samples + d.nsec - 1) / d.nsec)
                         : s.max_samples;
  if (cap > s.max_samples) cap = s.max_samples;
  d.cap = int(cap);
  put9(metric ? block_frame(metric->azimuth, metric->dip, metric->rake) : eye(), d.axes);
  put9(metric ? aniso_matrix(*metric) : eye(), d.frame);
  // With a metric M = diag(1, 1/semi, 1/minor) R the octant frame is rows
  // (-R1, R0, R2), so its x, y, z are -semi dp1, dp0, minor dp2; without one
  // both frames are the identity.
  const int ax_x = metric ? 1 : 0, sg_x = metric ? -1 : 1, ax_y = metric ? 0 : 1;
  d.nbits = d.nsec == 8 ? 3 : (d.nsec == 4 ? 2 : 0);
  // Hole and sector rules (search.rs:476-577): the greedy selection kernel.
  d.plane = s.sectors > 0 ? int(s.sectors) : 0;
  d.balances = (s.octant || s.sectors > 0) ? 1 : 0;
  // More than 64 samples also take this kernel: its candidate buffer, not a
  // per-lane heap, holds the list; so do sector caps whose lists would not fit
  // a lane's 64 heap slots (e.g. 16 a sector over 8 octants).
  d.rules = (s.max_per_hole >= 0 || s.sectors > 0 || s.min_sectors >= 0 || s.max_empty_sectors >= 0 ||
             s.min_holes >= 0 || s.max_samples > kMaxN || int64_t(d.nsec) * cap > kMaxSlots) ? 1 : 0;
  d.max_per_hole = s.max_per_hole;
  d.min_sectors = int(s.min_sectors), d.max_empty_sectors = int(s.max_empty_sectors), d.min_holes = int(s.min_holes);
  d.rsec = d.plane ? d.plane : (s.octant ? d.nsec : 0);
  d.rcap = d.plane ? int(s.max_per_sector) : (s.octant ? int(cap) : INT32_MAX);
  d.hole = ctx->has_hole ? ctx->hole.p : nullptr;
  d.sx = ctx->x.p, d.sy = ctx->y.p, d.sz = ctx->z.p;
  d.sgs = 0, d.sgs_node0 = 0, d.sgs_done = nullptr;
  if (d.nsec == 8) {  // index bx << 2 | by << 1 | bz
    d.bit_axis[2] = ax_x, d.bit_sign[2] = sg_x, d.bit_mask[2] = 0xF0;
    d.bit_axis[1] = ax_y, d.bit_sign[1] = 1, d.bit_mask[1] = 0xCC;
    d.bit_axis[0] = 2, d.bit_sign[0] = 1, d.bit_mask[0] = 0xAA;
  } else if (d.nsec == 4) {  // index bx << 1 | by
    d.bit_axis[1] = ax_x, d.bit_sign[1] = sg_x, d.bit_mask[1] = 0xC;
    d.bit_axis[0] = ax_y, d.bit_sign[0] = 1, d.bit_mask[0] = 0xA;
  }
}

double frobenius(const double* m) {
  double s = 0.0;
  for (int i = 0; i < 9; ++i) s += m[i] * m[i];
  return std::sqrt(s);
}

// Projection and grid over the fitted samples for the current search.
int index_samples(btk_ctx* ctx) {
  const int64_t n = ctx->n;
  make_searchdev(ctx);
  Launch L = ctx->launch(nullptr);
  CK(ctx->frame9.grow(9));
  CK(ctx->origin3.grow(3));
  CK(cudaMemcpyAsync(ctx->frame9.p, ctx->spd.frame, 9 * sizeof(double), cudaMemcpyHostToDevice, L.stream));
  CK(cudaMemcpyAsync(ctx->origin3.p, ctx->spd.origin, 3 * sizeof(double), cudaMemcpyHostToDevice, L.stream));
  CK(ctx->px.grow(n));
  CK(ctx->py.grow(n));
  CK(ctx->pz.grow(n));
  CK(launch_project(L, n, ctx->x.p, ctx->y.p, ctx->z.p, ctx->frame9.p, ctx->origin3.p, ctx->px.p, ctx->py.p,
                    ctx->pz.p));
  CK(ctx->bpart.grow(6 * 1024));
  CK(ctx->b6.grow(6));
  CK(launch_bounds(L, n, ctx->px.p, ctx->py.p, ctx->pz.p, ctx->bpart.p, ctx->b6.p));
  double b[6];
  CK(cudaMemcpyAsync(b, ctx->b6.p, sizeof b, cudaMemcpyDeviceToHost, L.stream));
  CK(cudaStreamSynchronize(L.stream));

  GridDev& g = ctx->gd;
  double ext[3], longest = 0.0, prod = 1.0;
  int spanned = 0;
  for (int d = 0; d < 3; ++d) ext[d] = b[3 + d] - b[d], longest = std::fmax(longest, ext[d]);
  for (int d = 0; d < 3; ++d)
    if (ext[d] > longest * 1e-9) prod *= ext[d], ++spanned;
  const double target_cells = std::fmax(double(n) / ctx->ppc, 1.0);
  double h = longest > 0.0 ? std::pow(prod / target_cells, 1.0 / spanned) : 1.0;
  auto cells = [&](double hh) {
    double c = 1.0;
    for (double e : ext) c *= std::floor(e / hh) + 1.0;
    return c;
  };
  while (cells(h) > 4.0 * target_cells + 64.0) h *= 2.0;
  g.h = h;
  double scale = 0.0;
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = b[d];
    g.dims[d] = int(std::floor(ext[d] / h)) + 1;
    scale = std::fmax(scale, std::fmax(std::fabs(b[d]), std::fabs(b[3 + d])));
  }
  g.slack = 1e-9 * (scale + h);
  g.ncells = int64_t(g.dims[0]) * g.dims[1] * g.dims[2];
  CK(ctx->cell_count.grow(g.ncells));
  CK(ctx->start.grow(g.ncells + 1));
  CK(ctx->cell_of.grow(n));
  CK(ctx->spx.grow(n));
  CK(ctx->spy.grow(n));
  CK(ctx->spz.grow(n));
  CK(ctx->swx.grow(n));
  CK(ctx->swy.grow(n));
  CK(ctx->swz.grow(n));
  CK(ctx->sidx.grow(n));
  const size_t gtb = grid_sort_temp_bytes(n, g.ncells);
  if (n > 0 && gtb == 0) return fail(ctx, BTK_ECUDA, "grid sort sizing failed");
  CK(ctx->gsort_keys.grow(2 * size_t(n > 0 ? n : 1)));
  CK(ctx->gsort_vals.grow(2 * size_t(n > 0 ? n : 1)));
  CK(ctx->gsort_temp.grow(gtb > 0 ? gtb : 1));
  CK(launch_grid_build(L, n, ctx->x.p, ctx->y.p, ctx->z.p, ctx->px.p, ctx->py.p, ctx->pz.p, g, ctx->cell_count.p,
                       ctx->start.p, ctx->cell_of.p, ctx->spx.p, ctx->spy.p, ctx->spz.p, ctx->swx.p, ctx->swy.p,
                       ctx->swz.p, ctx->sidx.p, ctx->gsort_keys.p, ctx->gsort_vals.p,
                       ctx->gsort_temp.p, gtb));
  g.start = ctx->start.p;
  g.px = ctx->spx.p, g.py = ctx->spy.p, g.pz = ctx->spz.p;
  g.wx = ctx->swx.p, g.wy = ctx->swy.p, g.wz = ctx->swz.p;
  g.idx = ctx->sidx.p;
  const int reach = 1 + int(std::ceil(kEps * frobenius(ctx->spd.frame) / h));
  CK(ctx->twin.grow(n));
  CK(launch_twins(L, n, g, reach, ctx->x.p, ctx->y.p, ctx->z.p, ctx->twin.p));
  // Leave-one-out walks the samples in cell order, so a tile's targets are near.
  std::vector<uint32_t> order(n);
  CK(cudaMemcpyAsync(order.data(), ctx->sidx.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, L.stream));
  CK(cudaStreamSynchronize(L.stream));
  std::vector<int64_t> perm(order.begin(), order.end());
  CK(ctx->loo_perm.grow(n));
  CK(cudaMemcpy(ctx->loo_perm.p, perm.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice));
  return BTK_OK;
}

int ensure_scratch(btk_ctx* ctx, int64_t m) {
  const size_t mm = size_t(m > 0 ? m : 1);
  CK(ctx->nbr.grow(mm * size_t(ctx->search.max_samples)));
  CK(ctx->cnt.grow(mm));
  CK(ctx->sst.grow(mm));
  CK(ctx->lists.grow(3 * mm));  // n <= 32, 32 < n <= 64, dense LU
  CK(ctx->lens.grow(3));
  CK(ctx->redo.grow(2 * mm));
  CK(ctx->redo_len.grow(2));
  return BTK_OK;
}

// Fewest caller-supplied targets that are put in spatial order first.
constexpr int64_t kOrderMin = 2048;

// Search then solve for m targets whose coordinates are device SoA arrays.
// The fitted search, restricted by hard domains when the samples have them:
// the rules kernel then takes each target's own domain only, tdom[t] for a
// prediction and the left-out sample's for leave-one-out (loo).
SearchDev search_for(const btk_ctx* ctx, const int32_t* tdom, bool loo) {
  SearchDev sp = ctx->spd;
  if (ctx->has_dom) {
    sp.rules = 1;
    sp.sdom = ctx->dom.p;
    sp.tdom = loo ? ctx->dom.p : tdom;
  }
  return sp;
}

// A call's target domains against the fit's: both or neither.
int check_domains(btk_ctx* ctx, const int32_t* tdom, bool loo) {
  if (loo) return BTK_OK;
  if (ctx->has_dom && !tdom) return fail(ctx, BTK_EINVAL, "fitted with domains; predict needs domains too");
  if (!ctx->has_dom && tdom) return fail(ctx, BTK_EINVAL, "fitted without domains; predict takes none");
  return BTK_OK;
}

int run_path(btk_ctx* ctx, cudaStream_t s, int64_t m, const double* tx, const double* ty, const double* tz,
             const int64_t* perm, int64_t nwork, int loo, int32_t kind, double kparam, int32_t precision,
             const btk_outputs* o, const int8_t* kinds = nullptr, const btk_diagnostics* dg = nullptr,
             const int32_t* tdom = nullptr, double* wout = nullptr) {
  if (int rc = check_domains(ctx, tdom, loo != 0)) return rc;
  if (kind < BTK_ORDINARY || kind > BTK_INDICATOR) return fail(ctx, BTK_EINVAL, "unknown kriging kind");
  if (precision != BTK_FP64 && precision != BTK_MIXED) return fail(ctx, BTK_EINVAL, "unknown precision");
  if (kind == BTK_SIMPLE && !std::isfinite(kparam)) return fail(ctx, BTK_EINVAL, "simple kriging needs a finite mean");
  if (!o || !o->value) return fail(ctx, BTK_EINVAL, "outputs need a value array");
  if ((dg || wout) && !o->status) return fail(ctx, BTK_EINVAL, "diagnostics and weights need the status output");
  const btk_search& srch = ctx->search;
  if (srch.calibration == 1 && kind == BTK_SIMPLE && !kinds)
    return fail(ctx, BTK_EINVAL, "simple kriging has a slope of regression of 1; calibrate it with target_efficiency");
  int rc = ensure_scratch(ctx, m);
  if (rc) return rc;
  Launch L = ctx->launch(s);
  if (!perm && m >= kOrderMin) {  // caller's order: sort into Hilbert order so warps and tiles are compact
    const size_t tb = morton_temp_bytes(m);
    if (tb == 0) return fail(ctx, BTK_ECUDA, "radix sort sizing failed");
    CK(ctx->ord_keys.grow(2 * size_t(m)));
    CK(ctx->ord_vals.grow(2 * size_t(m)));
    CK(ctx->ord_temp.grow(tb));
    CK(ctx->ord_part.grow(6 * 1024));
    CK(ctx->ord_b6.grow(6));
    CK(ctx->ord_lat.grow(4));
    // World axes weighted by the search metric's stretch along each (column
    // norms of the search frame): key cells stay aligned with a block lattice
    // but are as long, in search distance, along every axis.
    double wgt[3];
    for (int d = 0; d < 3; ++d)
      wgt[d] = std::sqrt(ctx->spd.frame[d] * ctx->spd.frame[d] + ctx->spd.frame[3 + d] * ctx->spd.frame[3 + d] +
                         ctx->spd.frame[6 + d] * ctx->spd.frame[6 + d]);
    CK(launch_morton_order(L, m, tx, ty, tz, wgt, ctx->ord_part.p, ctx->ord_b6.p, ctx->ord_lat.p, ctx->ord_keys.p,
                           ctx->ord_vals.p, ctx->ord_temp.p, tb, &perm));
    nwork = m;
  }
  ctx->mark(0, L.stream);
  CK(launch_search(L, search_for(ctx, tdom, loo != 0), ctx->gd, tx, ty, tz, perm, nwork, loo, ctx->nbr.p, ctx->cnt.p,
                   ctx->sst.p));
  ctx->mark(1, L.stream);
  SolveDev a{};
  a.vg = ctx->vgd;
  a.kind = kind;
  a.kparam = kparam;
  a.kinds = kinds;
  a.max_samples = int(ctx->search.max_samples);
  a.sx = ctx->x.p, a.sy = ctx->y.p, a.sz = ctx->z.p, a.sv = ctx->v.p, a.se = ctx->has_err ? ctx->e.p : nullptr;
  a.twin = ctx->twin.p;
  a.tx = tx, a.ty = ty, a.tz = tz;
  a.nbr = ctx->nbr.p, a.count = ctx->cnt.p, a.sstatus = ctx->sst.p;
  a.m = m;
  a.value = o->value, a.variance = o->variance, a.lagrange = o->lagrange, a.n_used = o->n_used, a.status = o->status;
  if (const size_t lu = lu_scratch_doubles(ctx->sm_count, int(srch.max_samples))) {
    CK(ctx->lu_scratch.grow(lu));
    a.lu_scratch = ctx->lu_scratch.p;
  }
  if (ctx->sup_n > 0 && !loo) {  // block support; cross-validation stays at point support
    CK(launch_support_cbb(L, ctx->vgd, ctx->sup.p, ctx->sup_n, ctx->sup_cbb.p));
    a.sup = ctx->sup.p, a.sup_n = ctx->sup_n, a.sup_cbb = ctx->sup_cbb.p;
  }
  if (srch.calibration) {  // the fewest leading samples that reach the target quality
    CK(ctx->met.grow(size_t(m > 0 ? m : 1)));
    SolveDev ac = a;
    ac.perm = perm, ac.nwork = perm ? nwork : m;
    CalDev cd{};
    cd.count = ctx->cnt.p, cd.nbr = ctx->nbr.p, cd.met = ctx->met.p;
    cd.calibration = int(srch.calibration), cd.target = srch.calibration_target;
    cd.min_samples = int(srch.min_samples);
    cd.balance = ctx->spd.balances;
    CK(launch_calibrate(L, ac, ctx->spd, cd, int(srch.max_samples)));
  }
  // The diagnostics pass over every work slot, after the solve has set each status.
  // With `wout`, the same pass writes each estimated system's weights.
  auto diagnose = [&]() -> int {
    if (!dg && !wout) return BTK_OK;
    SolveDev ad = a;
    ad.perm = perm, ad.nwork = perm ? nwork : m;
    if (dg) {
      ad.negw = dg->negative_weight_sum, ad.mdist = dg->mean_distance, ad.nholes = dg->n_holes;
      ad.hole = ctx->has_hole ? ctx->hole.p : nullptr;
    }
    ad.wout = wout;
    CK(launch_solve_lu(L, ad, int(ctx->search.max_samples), true));
    if (dg && dg->target_met) {
      if (srch.calibration)
        CK(cudaMemcpyAsync(dg->target_met, ctx->met.p, size_t(m), cudaMemcpyDeviceToDevice, L.stream));
      else
        CK(cudaMemsetAsync(dg->target_met, 0xFF, size_t(m), L.stream));
    }
    return BTK_OK;
  };
  if (!ctx->vgd.stationary) {
    // A power structure: every system through the dense LU, as the reference
    // sends every non-stationary system to krige_lu (kernel.rs:31).
    SolveDev al = a;
    al.perm = perm, al.nwork = perm ? nwork : m;
    ctx->mark(2, L.stream);
    CK(launch_solve_lu(L, al, int(ctx->search.max_samples)));
    ctx->mark(3, L.stream);
    return diagnose();
  }
  const bool big = ctx->search.max_samples > kMaxN;
  if (big) {
    CK(cudaMemsetAsync(ctx->lens.p + 2, 0, sizeof(int64_t), L.stream));
    a.lu = ctx->lists.p + 2 * m, a.lu_len = ctx->lens.p + 2;
  }
  const bool two = ctx->search.max_samples > 32;
  const bool tiled = ctx->tuning.tile_union > 0;
  const int nb = two ? 2 : 1;
  if (precision == BTK_MIXED) CK(cudaMemsetAsync(ctx->redo_len.p, 0, 2 * sizeof(int64_t), L.stream));
  if (tiled) {
    // Tile-shared solve of the n <= 32 systems; the rest go to the lists.
    CK(cudaMemsetAsync(ctx->lens.p, 0, 2 * sizeof(int64_t), L.stream));
    TileDev td{};
    td.s = a;
    td.perm = perm;
    td.nwork = nwork;
    td.umax = ctx->tuning.tile_union;
    td.small = ctx->lists.p, td.small_len = ctx->lens.p;
    td.large = ctx->lists.p + m, td.large_len = ctx->lens.p + 1;
    td.redo = ctx->redo.p, td.redo_len = ctx->redo_len.p;
    CK(launch_tile(L, td, precision == BTK_MIXED));
  } else if (two) {
    CK(launch_bucket(L, m, ctx->cnt.p, ctx->sst.p, ctx->lists.p, ctx->lens.p));
  }
  for (int b = 0; b < nb; ++b) {
    SolveDev ab = a;
    if (two || tiled) ab.list = ctx->lists.p + b * m, ab.list_len = ctx->lens.p + b;
    const int rows = b == 0 ? 32 : 64;
    // The mixed form's systems above 32 samples take the FP64 kernel when the
    // tuning says so: per-pivot barriers, not arithmetic, bound those
    // kernels, so FP32 saves little there and its refinement adds sweeps.
    if (precision == BTK_FP64 || (b == 1 && ctx->tuning.mixed_large))
      CK(launch_solve(L, ab, rows));
    else
      CK(launch_solve_mixed(L, ab, rows, ctx->redo.p + b * m, ctx->redo_len.p + b));
  }
  ctx->mark(2, L.stream);
  if (precision == BTK_MIXED)
    for (int b = 0; b < nb; ++b) {  // systems the FP32 factorisation left to FP64
      SolveDev ar = a;
      ar.list = ctx->redo.p + b * m, ar.list_len = ctx->redo_len.p + b;
      CK(launch_solve_redo(L, ar, b == 0 ? 32 : 64));
    }
  if (big) {  // systems of more than 64 samples (FP64 in both precisions)
    SolveDev al = a;
    al.list = a.lu, al.list_len = a.lu_len;
    CK(launch_solve_lu(L, al, int(ctx->search.max_samples)));
  }
  ctx->mark(3, L.stream);
  return diagnose();
}

int need_fit(btk_ctx* ctx) {
  if (!ctx) return BTK_EINVAL;
  if (!ctx->fitted) return fail(ctx, BTK_ENOTFITTED, "estimator is not fitted; call fit first");
  return BTK_OK;
}

// Device outputs for a host call: value (+ optional arrays).
int host_outputs(btk_ctx* ctx, int64_t m, const btk_outputs* out, btk_outputs* d) {
  const size_t mm = size_t(m > 0 ? m : 1);
  CK(ctx->o_value.grow(mm));
  CK(ctx->o_var.grow(mm));
  CK(ctx->o_lag.grow(mm));
  CK(ctx->o_nused.grow(mm));
  CK(ctx->o_status.grow(mm));
  d->value = ctx->o_value.p;
  d->variance = ctx->o_var.p;
  d->lagrange = ctx->o_lag.p;
  d->n_used = ctx->o_nused.p;
  d->status = ctx->o_status.p;
  (void)out;
  return BTK_OK;
}

int copy_out(btk_ctx* ctx, int64_t m, const btk_outputs* d, const btk_outputs* out) {
  cudaStream_t s = ctx->stream;
  const size_t mm = size_t(m);
  if (m > 0) {
    CK(cudaMemcpyAsync(out->value, d->value, mm * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (out->variance) CK(cudaMemcpyAsync(out->variance, d->variance, mm * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (out->lagrange) CK(cudaMemcpyAsync(out->lagrange, d->lagrange, mm * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (out->n_used) CK(cudaMemcpyAsync(out->n_used, d->n_used, mm * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (out->status) CK(cudaMemcpyAsync(out->status, d->status, mm * sizeof(int8_t), cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  return BTK_OK;
}

__global__ void k_split_xyz(int64_t m, const double* aos, double* x, double* y, double* z) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < m; i += int64_t(gridDim.x) * blockDim.x) {
    x[i] = aos[3 * i], y[i] = aos[3 * i + 1], z[i] = aos[3 * i + 2];
  }
}

// Host m x 3 row-major coordinates to device x, y, z arrays in ctx->txyz.
int upload_targets(btk_ctx* ctx, int64_t m, const double* xyz) {
  const size_t mm = size_t(m > 0 ? m : 1);
  CK(ctx->aos.grow(3 * mm));
  CK(ctx->txyz.grow(3 * mm));
  if (m == 0) return BTK_OK;
  CK(cudaMemcpyAsync(ctx->aos.p, xyz, 3 * size_t(m) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  int64_t b = (m + 255) / 256;
  if (b > int64_t(ctx->sm_count) * 8) b = int64_t(ctx->sm_count) * 8;
  k_split_xyz<<<int(b), 256, 0, ctx->stream>>>(m, ctx->aos.p, ctx->txyz.p, ctx->txyz.p + m, ctx->txyz.p + 2 * m);
  ++ctx->launches;
  CK(cudaGetLastError());
  return BTK_OK;
}

}  // namespace

namespace {

// dM/dphi for M = diag(1, 1/semi, 1/minor) r3(rake) r2(dip) r1(az), angles in
// degrees (crates/core/src/rotation.rs:8-16, aniso.rs:88-94).
void aniso_derivatives(const btk_aniso& a, double dM[5][9]) {
  const double k = 3.14159265358979323846 / 180.0;
  const double sa = std::sin(a.azimuth * k), ca = std::cos(a.azimuth * k);
  const double sd = std::sin(a.dip * k), cd = std::cos(a.dip * k);
  const double sr = std::sin(a.rake * k), cr = std::cos(a.rake * k);
  M3 r1 = rows(sa, ca, 0.0, -ca, sa, 0.0, 0.0, 0.0, 1.0);
  M3 r2 = rows(cd, 0.0, -sd, 0.0, 1.0, 0.0, sd, 0.0, cd);
  M3 r3 = rows(1.0, 0.0, 0.0, 0.0, cr, sr, 0.0, -sr, cr);
  M3 d1 = rows(ca * k, -sa * k, 0.0, sa * k, ca * k, 0.0, 0.0, 0.0, 0.0);
  M3 d2 = rows(-sd * k, 0.0, -cd * k, 0.0, 0.0, 0.0, cd * k, 0.0, -sd * k);
  M3 d3 = rows(0.0, 0.0, 0.0, 0.0, -sr * k, cr * k, 0.0, -cr * k, -sr * k);
  M3 D{};
  D.m[0][0] = 1.0, D.m[1][1] = 1.0 / a.semi, D.m[2][2] = 1.0 / a.minor;
  M3 R = mul(mul(r3, r2), r1);
  M3 ds{}, dm{};
  ds.m[1][1] = -1.0 / (a.semi * a.semi);
  dm.m[2][2] = -1.0 / (a.minor * a.minor);
  put9(mul(ds, R), dM[0]);
  put9(mul(dm, R), dM[1]);
  put9(mul(D, mul(mul(r3, r2), d1)), dM[2]);
  put9(mul(D, mul(mul(r3, d2), r1)), dM[3]);
  put9(mul(D, mul(mul(d3, r2), r1)), dM[4]);
}

}  // namespace

namespace btk {

int prepare_variogram(const btk_variogram* vg, VgDev* out, std::string* why) {
  btk_ctx tmp;  // host-side only: its device buffers stay empty
  int rc = check_vg(&tmp, vg);
  if (rc != BTK_OK) {
    *why = tmp.err;
    return rc;
  }
  make_vgdev(*vg, *out);
  return BTK_OK;
}

}  // namespace btk

extern "C" {

const char* btk_version(void) { return "boitata_b200 0.1.0 (sm_100a)"; }

btk_ctx* btk_create(int device, char* err, size_t errlen) {
  auto say = [&](const std::string& m) {
    if (err && errlen) std::snprintf(err, errlen, "%s", m.c_str());
  };
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    say(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
    return nullptr;
  }
  if (device < 0 || device >= count) {
    say("device index out of range");
    return nullptr;
  }
  if ((e = cudaSetDevice(device)) != cudaSuccess) {
    say(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return nullptr;
  }
  btk_ctx* c = new btk_ctx;
  c->device = device;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
    say(std::string("stream/attribute: ") + cudaGetErrorString(e));
    delete c;
    return nullptr;
  }
  if (const char* p = std::getenv("BTK_SAMPLES_PER_CELL")) {
    double v = std::atof(p);
    if (v > 0.0) c->ppc = v;
  }
  return c;
}

void btk_destroy(btk_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream), cudaStreamDestroy(ctx->stream);
  for (cudaEvent_t e : ctx->ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->cev)
    if (e) cudaEventDestroy(e);
  if (ctx->up) cudaStreamSynchronize(ctx->up), cudaStreamDestroy(ctx->up);
  if (ctx->down) cudaStreamSynchronize(ctx->down), cudaStreamDestroy(ctx->down);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  delete ctx;
}

int btk_set_support(btk_ctx* ctx, const double* size, const int32_t* disc, const double* rotation) {
  if (!ctx) return BTK_EINVAL;
  if (!size) {
    ctx->sup_n = 0;
    return BTK_OK;
  }
  if (!disc) return fail(ctx, BTK_EINVAL, "a block size needs a discretization");
  for (int d = 0; d < 3; ++d) {
    if (disc[d] < 1)
      return fail(ctx, BTK_EINVAL, "discretization must be at least 1 per axis, got (" + std::to_string(disc[0]) +
                                       ", " + std::to_string(disc[1]) + ", " + std::to_string(disc[2]) + ")");
    if (!(std::isfinite(size[d]) && size[d] > 0.0)) return fail(ctx, BTK_EINVAL, "size must be finite and > 0");
    if (rotation && !std::isfinite(rotation[d])) return fail(ctx, BTK_EINVAL, "rotation must be finite");
  }
  const int64_t nd = int64_t(disc[0]) * disc[1] * disc[2];
  if (nd > BTK_MAX_SUPPORT_POINTS) return fail(ctx, BTK_EINVAL, "block discretization has more than 4096 points");
  const double zero[3] = {0.0, 0.0, 0.0};
  const std::vector<double> off = block_offsets(size, disc, rotation ? rotation : zero);
  CK(cudaSetDevice(ctx->device));
  CK(ctx->sup.grow(off.size()));
  CK(ctx->sup_cbb.grow(1));
  CK(cudaMemcpyAsync(ctx->sup.p, off.data(), off.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->sup_n = int(nd);
  return BTK_OK;
}

int btk_support_variance(btk_ctx* ctx, double* out) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out) return fail(ctx, BTK_EINVAL, "out is required");
  if (ctx->sup_n == 0) {
    *out = ctx->vgd.c0;
    return BTK_OK;
  }
  CK(cudaSetDevice(ctx->device));
  Launch L = ctx->launch(nullptr);
  CK(launch_support_cbb(L, ctx->vgd, ctx->sup.p, ctx->sup_n, ctx->sup_cbb.p));
  CK(cudaMemcpyAsync(out, ctx->sup_cbb.p, sizeof(double), cudaMemcpyDeviceToHost, L.stream));
  CK(cudaStreamSynchronize(L.stream));
  return BTK_OK;
}

int btk_get_tuning(const btk_ctx* ctx, btk_tuning* out) {
  if (!ctx || !out) return BTK_EINVAL;
  out->samples_per_cell = ctx->ppc;
  for (int a = 0; a < 3; ++a) out->tile[a] = ctx->tuning.tile[a];
  out->search_warps = ctx->tuning.search_warps;
  out->solve_blocks_per_sm = ctx->tuning.solve_blocks_per_sm;
  out->tile_union = ctx->tuning.tile_union;
  out->host_chunk = ctx->tuning.host_chunk;
  out->tile_tensor = ctx->tuning.tile_tensor;
  out->mixed_large = ctx->tuning.mixed_large;
  return BTK_OK;
}

int btk_set_tuning(btk_ctx* ctx, const btk_tuning* t) {
  if (!ctx || !t) return BTK_EINVAL;
  const int prod = t->tile[0] * t->tile[1] * t->tile[2];
  if (t->tile[0] < 1 || t->tile[1] < 1 || t->tile[2] < 1 || prod != 32)
    return fail(ctx, BTK_EINVAL, "the tile must hold 32 cells");
  if (!(t->search_warps == 0 || t->search_warps == 1 || t->search_warps == 2 || t->search_warps == 4 ||
        t->search_warps == 8))
    return fail(ctx, BTK_EINVAL, "search_warps must be 0, 1, 2, 4 or 8");
  if (t->solve_blocks_per_sm < 0) return fail(ctx, BTK_EINVAL, "solve_blocks_per_sm must be >= 0");
  if (t->tile_union != 0 && (t->tile_union < 32 || t->tile_union > 255))
    return fail(ctx, BTK_EINVAL, "tile_union must be 0 or in 32..255");
  if (t->host_chunk < 0) return fail(ctx, BTK_EINVAL, "host_chunk must be >= 0");
  if (t->tile_tensor != 0 && t->tile_tensor != 1) return fail(ctx, BTK_EINVAL, "tile_tensor must be 0 or 1");
  if (t->mixed_large != 0 && t->mixed_large != 1) return fail(ctx, BTK_EINVAL, "mixed_large must be 0 or 1");
  if (!(t->samples_per_cell > 0.0 && t->samples_per_cell <= 1e6))
    return fail(ctx, BTK_EINVAL, "samples_per_cell must be > 0");
  for (int a = 0; a < 3; ++a) ctx->tuning.tile[a] = t->tile[a];
  ctx->tuning.search_warps = t->search_warps;
  ctx->tuning.solve_blocks_per_sm = t->solve_blocks_per_sm;
  ctx->tuning.tile_union = t->tile_union;
  ctx->tuning.host_chunk = t->host_chunk;
  ctx->tuning.tile_tensor = t->tile_tensor;
  ctx->tuning.mixed_large = t->mixed_large;
  if (t->samples_per_cell != ctx->ppc) {
    ctx->ppc = t->samples_per_cell;
    if (ctx->fitted) {
      CK(cudaSetDevice(ctx->device));
      ctx->frozen = false;
      ctx->mean_m = 0;
      int rc = index_samples(ctx);
      if (rc) return rc;
      CK(cudaStreamSynchronize(ctx->stream));
    }
  }
  return BTK_OK;
}

}  // extern "C"

namespace {

// Captures `call(stream)` (one prediction on the context's stream) into the
// context's CUDA graph, replacing any earlier one. One plain call first sizes
// every buffer and sets every kernel attribute, so the captured call
// allocates nothing.
template <class Call>
int capture_graph(btk_ctx* ctx, Call call) {
  CK(cudaSetDevice(ctx->device));
  int rc = call(ctx->stream);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->graph_exec) {
    CK(cudaGraphExecDestroy(ctx->graph_exec));
    ctx->graph_exec = nullptr;
  }
  if (ctx->graph) {
    CK(cudaGraphDestroy(ctx->graph));
    ctx->graph = nullptr;
  }
  const bool timing = ctx->timing;
  ctx->timing = false;
  const int64_t before = ctx->launches;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
  rc = call(ctx->stream);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
  ctx->timing = timing;
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  CK(e);
  ctx->graph = graph;
  ctx->graph_kernels = ctx->launches - before;
  ctx->launches = before;
  CK(cudaGraphInstantiate(&ctx->graph_exec, graph, 0));
  return BTK_OK;
}

}  // namespace

extern "C" {

int btk_graph_capture_geometry(btk_ctx* ctx, const btk_geometry* g, int32_t kind, double kparam,
                               int32_t precision, const btk_outputs* d_out) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  return capture_graph(ctx, [&](cudaStream_t s) {
    return btk_predict_geometry_device(ctx, g, kind, kparam, precision, d_out, s);
  });
}

int btk_graph_capture_device(btk_ctx* ctx, int64_t m, const double* d_xyz, const int8_t* d_kinds, int32_t kind,
                             double kparam, int32_t precision, const btk_outputs* d_out) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (m <= 0 || !d_xyz) return fail(ctx, BTK_EINVAL, "a captured prediction needs targets");
  return capture_graph(ctx, [&](cudaStream_t s) {
    return d_kinds ? btk_predict_kinds_device(ctx, m, d_xyz, d_kinds, kparam, precision, d_out, s)
                   : btk_predict_device(ctx, m, d_xyz, kind, kparam, precision, d_out, s);
  });
}

int btk_graph_launch(btk_ctx* ctx, void* stream) {
  if (!ctx) return BTK_EINVAL;
  if (!ctx->graph_exec) return fail(ctx, BTK_EINVAL, "no captured graph; call btk_graph_capture_geometry first");
  CK(cudaSetDevice(ctx->device));
  CK(cudaGraphLaunch(ctx->graph_exec, stream ? static_cast<cudaStream_t>(stream) : ctx->stream));
  ctx->launches += ctx->graph_kernels;
  return BTK_OK;
}

int btk_set_timing(btk_ctx* ctx, int32_t on) {
  if (!ctx) return BTK_EINVAL;
  CK(cudaSetDevice(ctx->device));
  for (cudaEvent_t& e : ctx->ev)
    if (!e) CK(cudaEventCreate(&e));
  ctx->timing = on != 0;
  return BTK_OK;
}

int btk_phase_ms(btk_ctx* ctx, float* out3) {
  if (!ctx || !out3) return BTK_EINVAL;
  if (!ctx->timing) return fail(ctx, BTK_EINVAL, "timing is off; call btk_set_timing first");
  CK(cudaEventSynchronize(ctx->ev[3]));
  for (int k = 0; k < 3; ++k) CK(cudaEventElapsedTime(&out3[k], ctx->ev[k], ctx->ev[k + 1]));
  return BTK_OK;
}

double btk_peak_flops(btk_ctx* ctx, int32_t fp64) {
  if (!ctx) return -1.0;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return -1.0;
  return measure_fma_flops(ctx->stream, ctx->sm_count, fp64, &ctx->launches);
}

const char* btk_last_error(const btk_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t btk_launch_count(const btk_ctx* ctx) { return ctx ? ctx->launches : 0; }

int btk_fit(btk_ctx* ctx, int64_t n, const double* xyz, const double* values, const double* err_var,
            const int64_t* holes, const btk_search* search, const btk_variogram* vg) {
  if (!ctx) return BTK_EINVAL;
  ctx->fitted = false;
  ctx->has_dom = false;
  if (n <= 0 || !xyz || !values) return fail(ctx, BTK_EINVAL, "fit needs at least one sample with coordinates and values");
  if (n >= int64_t(0xffffffffu)) return fail(ctx, BTK_EINVAL, "too many samples");
  int rc = check_vg(ctx, vg);
  if (rc) return rc;
  if ((rc = check_search(ctx, search, n))) return rc;
  std::vector<double> hx(n), hy(n), hz(n);
  for (int64_t i = 0; i < n; ++i) {
    hx[i] = xyz[3 * i], hy[i] = xyz[3 * i + 1], hz[i] = xyz[3 * i + 2];
    if (!fin(hx[i]) || !fin(hy[i]) || !fin(hz[i])) return fail(ctx, BTK_EINVAL, "coordinates must be finite");
    if (!fin(values[i])) return fail(ctx, BTK_EINVAL, "values must be finite; drop missing values first");
    if (err_var && (!fin(err_var[i]) || err_var[i] < 0.0))
      return fail(ctx, BTK_EINVAL, "error_variance must be finite and >= 0");
  }
  CK(cudaSetDevice(ctx->device));
  ctx->n = n;
  ctx->frozen = false;
  ctx->mean_m = 0;
  ctx->vg = *vg;
  ctx->has_err = err_var != nullptr;
  bool planar = true;  // search.rs:470-473
  for (int64_t i = 1; i < n && planar; ++i) planar = hz[i] == hz[0];
  ctx->planar = planar;
  ctx->search = effective_search(*search, n, planar);
  ctx->spd.origin[0] = hx[0], ctx->spd.origin[1] = hy[0], ctx->spd.origin[2] = hz[0];
  make_vgdev(*vg, ctx->vgd);
  for (auto* b : {&ctx->x, &ctx->y, &ctx->z, &ctx->v, &ctx->e}) CK(b->grow(n));
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(ctx->x.p, hx.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->y.p, hy.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->z.p, hz.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->v.p, values, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (err_var) CK(cudaMemcpyAsync(ctx->e.p, err_var, n * sizeof(double), cudaMemcpyHostToDevice, s));
  ctx->has_hole = holes != nullptr;
  if (holes) {  // hole codes (crates/py/src/args.rs:276-292), equal codes = one hole
    std::vector<uint32_t> hc(n);
    for (int64_t i = 0; i < n; ++i) {
      if (holes[i] < 0 || holes[i] >= int64_t(0xffffffffu)) return fail(ctx, BTK_EINVAL, "hole codes must be in 0 .. 2^32 - 2");
      hc[i] = uint32_t(holes[i]);
    }
    CK(ctx->hole.grow(n));
    CK(cudaMemcpyAsync(ctx->hole.p, hc.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
  }
  if ((rc = index_samples(ctx))) return rc;
  CK(cudaStreamSynchronize(s));
  ctx->fitted = true;
  return BTK_OK;
}

int btk_set_search(btk_ctx* ctx, const btk_search* search) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if ((rc = check_search(ctx, search, ctx->n))) return rc;
  CK(cudaSetDevice(ctx->device));
  ctx->search = effective_search(*search, ctx->n, ctx->planar);
  ctx->frozen = false;
  ctx->mean_m = 0;
  if ((rc = index_samples(ctx))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  return BTK_OK;
}

int btk_predict_device(btk_ctx* ctx, int64_t m, const double* d_xyz, int32_t kind, double kparam, int32_t precision,
                       const btk_outputs* d_out, void* stream) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (m < 0 || (m > 0 && !d_xyz)) return fail(ctx, BTK_EINVAL, "targets are required");
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return run_path(ctx, static_cast<cudaStream_t>(stream), m, d_xyz, d_xyz + m, d_xyz + 2 * m, nullptr, m, 0, kind,
                  kparam, precision, d_out);
}

namespace {

// Host targets in, host outputs out, in chunks of tuning.host_chunk targets
// (at most 8 chunks; 0: one): the copy of chunk c + 1 in and of chunk c - 1
// out overlap chunk c's search and solve. Each chunk is a run_path of its own over the
// context's scratch, which the compute stream serialises; chunks write
// disjoint slices of the staged inputs and outputs.
int predict_host(btk_ctx* ctx, int64_t m, const double* xyz, const int8_t* kinds, int32_t kind, double kparam,
                 int32_t precision, const btk_outputs* out, const btk_diagnostics* diag = nullptr,
                 const int32_t* domains = nullptr) {
  if (int rc = check_domains(ctx, domains, false)) return rc;
  int64_t chunk = ctx->tuning.host_chunk > 0 ? int64_t(ctx->tuning.host_chunk) : m;
  if ((m + chunk - 1) / chunk > 8) chunk = (m + 7) / 8;
  const int64_t nc = (m + chunk - 1) / chunk;
  const size_t mm = size_t(m);
  CK(ctx->aos.grow(3 * mm));
  CK(ctx->txyz.grow(3 * mm));
  if (kinds) CK(ctx->kinds.grow(mm));
  if (domains) CK(ctx->tdom.grow(mm));
  btk_outputs d{};
  int rc = host_outputs(ctx, m, out, &d);
  if (rc) return rc;
  if (diag) {
    CK(ctx->o_negw.grow(mm));
    CK(ctx->o_mdist.grow(mm));
    CK(ctx->o_nholes.grow(mm));
    CK(ctx->o_met.grow(mm));
  }
  if (!ctx->up) CK(cudaStreamCreateWithFlags(&ctx->up, cudaStreamNonBlocking));
  if (!ctx->down) CK(cudaStreamCreateWithFlags(&ctx->down, cudaStreamNonBlocking));
  for (cudaEvent_t& e : ctx->cev)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t* in_done = ctx->cev;
  cudaEvent_t* out_ready = ctx->cev + 8;
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t off = c * chunk, mc = std::min(chunk, m - off);
    CK(cudaMemcpyAsync(ctx->aos.p + 3 * off, xyz + 3 * off, 3 * size_t(mc) * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->up));
    if (kinds) CK(cudaMemcpyAsync(ctx->kinds.p + off, kinds + off, size_t(mc), cudaMemcpyHostToDevice, ctx->up));
    if (domains)
      CK(cudaMemcpyAsync(ctx->tdom.p + off, domains + off, size_t(mc) * sizeof(int32_t), cudaMemcpyHostToDevice,
                         ctx->up));
    CK(cudaEventRecord(in_done[c], ctx->up));
  }
  double* t = ctx->txyz.p;
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t off = c * chunk, mc = std::min(chunk, m - off);
    CK(cudaStreamWaitEvent(ctx->stream, in_done[c], 0));
    int64_t b = (mc + 255) / 256;
    if (b > int64_t(ctx->sm_count) * 8) b = int64_t(ctx->sm_count) * 8;
    k_split_xyz<<<int(b), 256, 0, ctx->stream>>>(mc, ctx->aos.p + 3 * off, t + off, t + m + off, t + 2 * m + off);
    ++ctx->launches;
    CK(cudaGetLastError());
    btk_outputs dc{d.value + off, d.variance + off, d.lagrange + off, d.n_used + off, d.status + off};
    btk_diagnostics dd{ctx->o_negw.p + off, ctx->o_mdist.p + off, ctx->o_nholes.p + off, ctx->o_met.p + off};
    if ((rc = run_path(ctx, ctx->stream, mc, t + off, t + m + off, t + 2 * m + off, nullptr, mc, 0, kind, kparam,
                       precision, &dc, kinds ? ctx->kinds.p + off : nullptr, diag ? &dd : nullptr,
                       domains ? ctx->tdom.p + off : nullptr)))
      return rc;
    CK(cudaEventRecord(out_ready[c], ctx->stream));
    CK(cudaStreamWaitEvent(ctx->down, out_ready[c], 0));
    const size_t n = size_t(mc);
    CK(cudaMemcpyAsync(out->value + off, dc.value, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->down));
    if (out->variance)
      CK(cudaMemcpyAsync(out->variance + off, dc.variance, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->down));
    if (out->lagrange)
      CK(cudaMemcpyAsync(out->lagrange + off, dc.lagrange, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->down));
    if (out->n_used)
      CK(cudaMemcpyAsync(out->n_used + off, dc.n_used, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->down));
    if (out->status)
      CK(cudaMemcpyAsync(out->status + off, dc.status, n * sizeof(int8_t), cudaMemcpyDeviceToHost, ctx->down));
    if (diag && diag->negative_weight_sum)
      CK(cudaMemcpyAsync(diag->negative_weight_sum + off, dd.negative_weight_sum, n * sizeof(double),
                         cudaMemcpyDeviceToHost, ctx->down));
    if (diag && diag->mean_distance)
      CK(cudaMemcpyAsync(diag->mean_distance + off, dd.mean_distance, n * sizeof(double), cudaMemcpyDeviceToHost,
                         ctx->down));
    if (diag && diag->n_holes)
      CK(cudaMemcpyAsync(diag->n_holes + off, dd.n_holes, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->down));
    if (diag && diag->target_met)
      CK(cudaMemcpyAsync(diag->target_met + off, dd.target_met, n, cudaMemcpyDeviceToHost, ctx->down));
  }
  CK(cudaStreamSynchronize(ctx->down));
  CK(cudaStreamSynchronize(ctx->stream));
  return BTK_OK;
}

}  // namespace

int btk_predict(btk_ctx* ctx, int64_t m, const double* xyz, int32_t kind, double kparam, int32_t precision,
                const btk_outputs* out) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out || !out->value) return fail(ctx, BTK_EINVAL, "outputs need a value array");
  if (m < 0 || (m > 0 && !xyz)) return fail(ctx, BTK_EINVAL, "targets are required");
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return predict_host(ctx, m, xyz, nullptr, kind, kparam, precision, out);
}

int btk_predict_diagnostics(btk_ctx* ctx, int64_t m, const double* xyz, int32_t kind, double kparam,
                            int32_t precision, const btk_outputs* out, const btk_diagnostics* diag) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out || !out->value || !out->status) return fail(ctx, BTK_EINVAL, "outputs need value and status arrays");
  if (!diag) return fail(ctx, BTK_EINVAL, "diagnostics outputs are required");
  if (m < 0 || (m > 0 && !xyz)) return fail(ctx, BTK_EINVAL, "targets are required");
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return predict_host(ctx, m, xyz, nullptr, kind, kparam, precision, out, diag);
}

int btk_predict_kinds_device(btk_ctx* ctx, int64_t m, const double* d_xyz, const int8_t* d_kinds, double kparam,
                             int32_t precision, const btk_outputs* d_out, void* stream) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (m < 0 || (m > 0 && (!d_xyz || !d_kinds))) return fail(ctx, BTK_EINVAL, "targets and kinds are required");
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return run_path(ctx, static_cast<cudaStream_t>(stream), m, d_xyz, d_xyz + m, d_xyz + 2 * m, nullptr, m, 0,
                  BTK_ORDINARY, kparam, precision, d_out, d_kinds);
}

int btk_predict_kinds(btk_ctx* ctx, int64_t m, const double* xyz, const int8_t* kinds, double kparam,
                      int32_t precision, const btk_outputs* out) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out || !out->value) return fail(ctx, BTK_EINVAL, "outputs need a value array");
  if (m < 0 || (m > 0 && (!xyz || !kinds))) return fail(ctx, BTK_EINVAL, "targets and kinds are required");
  for (int64_t i = 0; i < m; ++i)
    if (kinds[i] < BTK_ORDINARY || kinds[i] > BTK_INDICATOR) return fail(ctx, BTK_EINVAL, "unknown kriging kind");
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return predict_host(ctx, m, xyz, kinds, BTK_ORDINARY, kparam, precision, out);
}

int btk_set_domains(btk_ctx* ctx, const int32_t* codes) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  ctx->frozen = false;
  ctx->mean_m = 0;
  if (!codes) {
    ctx->has_dom = false;
    return BTK_OK;
  }
  for (int64_t i = 0; i < ctx->n; ++i)
    if (codes[i] < 0) return fail(ctx, BTK_EINVAL, "every sample needs a domain code (>= 0)");
  CK(cudaSetDevice(ctx->device));
  CK(ctx->dom.grow(size_t(ctx->n)));
  CK(cudaMemcpy(ctx->dom.p, codes, size_t(ctx->n) * sizeof(int32_t), cudaMemcpyHostToDevice));
  ctx->has_dom = true;
  return BTK_OK;
}

int btk_predict_ex(btk_ctx* ctx, int64_t m, const double* xyz, const int8_t* kinds, const int32_t* domains,
                   int32_t kind, double kparam, int32_t precision, const btk_outputs* out,
                   const btk_diagnostics* diag) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out || !out->value) return fail(ctx, BTK_EINVAL, "outputs need a value array");
  if (diag && !out->status) return fail(ctx, BTK_EINVAL, "diagnostics need the status output");
  if (m < 0 || (m > 0 && !xyz)) return fail(ctx, BTK_EINVAL, "targets are required");
  if (kinds)
    for (int64_t i = 0; i < m; ++i)
      if (kinds[i] < BTK_ORDINARY || kinds[i] > BTK_INDICATOR) return fail(ctx, BTK_EINVAL, "unknown kriging kind");
  if ((rc = check_domains(ctx, domains, false))) return rc;
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return predict_host(ctx, m, xyz, kinds, kinds ? BTK_ORDINARY : kind, kparam, precision, out, diag, domains);
}

int btk_predict_weights(btk_ctx* ctx, int64_t m, const double* xyz, int32_t kind, double kparam, int32_t precision,
                        const int32_t* domains, const btk_outputs* out, int64_t* idx, double* weights) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out || !out->value || !out->status) return fail(ctx, BTK_EINVAL, "weights need the value and status outputs");
  if (m < 0 || (m > 0 && (!xyz || !idx || !weights)))
    return fail(ctx, BTK_EINVAL, "targets, idx and weights are required");
  if ((rc = check_domains(ctx, domains, false))) return rc;
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  if ((rc = upload_targets(ctx, m, xyz))) return rc;
  const size_t k = size_t(ctx->search.max_samples), mk = size_t(m) * k;
  CK(ctx->wts.grow(mk));
  CK(cudaMemsetAsync(ctx->wts.p, 0, mk * sizeof(double), ctx->stream));  // no row keeps an earlier call's weights
  if (domains) {
    CK(ctx->tdom.grow(size_t(m)));
    CK(cudaMemcpyAsync(ctx->tdom.p, domains, size_t(m) * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  }
  btk_outputs d{};
  if ((rc = host_outputs(ctx, m, out, &d))) return rc;
  const double* t = ctx->txyz.p;
  if ((rc = run_path(ctx, ctx->stream, m, t, t + m, t + 2 * m, nullptr, m, 0, kind, kparam, precision, &d, nullptr,
                     nullptr, domains ? ctx->tdom.p : nullptr, ctx->wts.p)))
    return rc;
  std::vector<uint32_t> nb(mk);
  std::vector<int32_t> cnt(static_cast<size_t>(m));
  CK(cudaMemcpyAsync(nb.data(), ctx->nbr.p, mk * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(cnt.data(), ctx->cnt.p, size_t(m) * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(weights, ctx->wts.p, mk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if ((rc = copy_out(ctx, m, &d, out))) return rc;  // synchronises the stream
  for (int64_t t0 = 0; t0 < m; ++t0) {
    const bool est = (out->status[t0] & 0x0F) == BTK_ST_OK;
    const size_t n = est ? size_t(std::max(cnt[t0], 0)) : 0;
    for (size_t r = 0; r < k; ++r) {
      const size_t e = size_t(t0) * k + r;
      const bool used = r < n;
      idx[e] = used ? int64_t(nb[e]) : -1;
      if (!used) weights[e] = 0.0;
    }
  }
  return BTK_OK;
}
int btk_predict_ex_device(btk_ctx* ctx, int64_t m, const double* d_xyz, const int8_t* d_kinds,
                          const int32_t* d_domains, int32_t kind, double kparam, int32_t precision,
                          const btk_outputs* d_out, void* stream) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (m < 0 || (m > 0 && !d_xyz)) return fail(ctx, BTK_EINVAL, "targets are required");
  if ((rc = check_domains(ctx, d_domains, false))) return rc;
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  return run_path(ctx, static_cast<cudaStream_t>(stream), m, d_xyz, d_xyz + m, d_xyz + 2 * m, nullptr, m, 0,
                  d_kinds ? BTK_ORDINARY : kind, kparam, precision, d_out, d_kinds, nullptr, d_domains);
}

int btk_predict_geometry_device(btk_ctx* ctx, const btk_geometry* g, int32_t kind, double kparam, int32_t precision,
                                const btk_outputs* d_out, void* stream) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!g) return fail(ctx, BTK_EINVAL, "geometry is required");
  for (int a = 0; a < 3; ++a) {
    if (!(g->size[a] > 0.0 && fin(g->size[a]))) return fail(ctx, BTK_EINVAL, "cell sizes must be positive");
    if (g->count[a] <= 0) return fail(ctx, BTK_EINVAL, "cell counts must be positive");
    if (!fin(g->origin[a]) || !fin(g->rotation[a])) return fail(ctx, BTK_EINVAL, "origin and rotation must be finite");
  }
  CK(cudaSetDevice(ctx->device));
  const int64_t m = g->count[0] * g->count[1] * g->count[2];
  const int* tw = ctx->tuning.tile;
  const int64_t tiles = ((g->count[0] + tw[0] - 1) / tw[0]) * ((g->count[1] + tw[1] - 1) / tw[1]) *
                        ((g->count[2] + tw[2] - 1) / tw[2]);
  const int64_t nwork = tiles * 32;
  CK(ctx->txyz.grow(3 * size_t(m)));
  CK(ctx->perm.grow(size_t(nwork)));
  Launch L = ctx->launch(static_cast<cudaStream_t>(stream));
  double* t = ctx->txyz.p;
  CK(launch_centroids(L, *g, transposed_frame(*g), 0, nwork, t, t + m, t + 2 * m, ctx->perm.p));
  return run_path(ctx, L.stream, m, t, t + m, t + 2 * m, ctx->perm.p, nwork, 0, kind, kparam, precision, d_out);
}

int btk_sgs_simulate(btk_ctx* ctx, int64_t n_data, const double* z, int64_t batch, double* score, int8_t* how,
                     int64_t* rounds) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (n_data < 1 || n_data > ctx->n) return fail(ctx, BTK_EINVAL, "n_data must be between 1 and the fitted samples");
  if (!score || (ctx->n > n_data && !z)) return fail(ctx, BTK_EINVAL, "z and score arrays are required");
  if (batch < 0) return fail(ctx, BTK_EINVAL, "batch must be >= 0 (0: automatic)");
  if (ctx->search.calibration)
    return fail(ctx, BTK_EINVAL, "SGS does not take target_slope or target_efficiency");
  if (!ctx->vgd.stationary)
    return fail(ctx, BTK_EINVAL, "simple kriging needs a variogram with a sill: every structure must be stationary");
  if (ctx->sup_n > 0) return fail(ctx, BTK_EINVAL, "SGS simulates points: clear the block support first");
  const int64_t m = ctx->n - n_data;
  if (rounds) *rounds = 0;
  if (m == 0) return BTK_OK;
  if (ctx->n > int64_t(0xffffffffu)) return fail(ctx, BTK_EINVAL, "too many samples and nodes");
  CK(cudaSetDevice(ctx->device));
  Launch L = ctx->launch(nullptr);
  const size_t mm = size_t(m);
  CK(ctx->sg_z.grow(mm));
  CK(ctx->sg_score.grow(mm));
  CK(ctx->sg_how.grow(mm));
  CK(ctx->sg_list.grow(mm));
  CK(ctx->sg_ctl.grow(2));
  CK(ctx->sg_done.grow(size_t(ctx->n)));
  btk_outputs d{};
  if ((rc = host_outputs(ctx, m, nullptr, &d))) return rc;
  CK(cudaMemcpyAsync(ctx->sg_z.p, z, mm * sizeof(double), cudaMemcpyHostToDevice, L.stream));
  CK(cudaMemsetAsync(ctx->sg_done.p, 0, size_t(ctx->n), L.stream));
  CK(cudaMemsetAsync(ctx->sg_how.p, 0, mm, L.stream));
  CK(cudaMemsetAsync(ctx->sg_ctl.p, 0xFF, 2 * sizeof(int64_t), L.stream));
  const SearchDev saved = ctx->spd;
  // One warp per node (the rules kernel): a window's nodes lie anywhere on the
  // path, so the tile search, which grows one box around 32 targets, does not
  // fit them.
  ctx->spd.rules = 1;
  ctx->spd.sgs = 1, ctx->spd.sgs_node0 = uint32_t(n_data), ctx->spd.sgs_done = ctx->sg_done.p;
  const uint32_t node0 = uint32_t(n_data);
  const int64_t most = ctx->search.max_samples;
  int64_t total_rounds = 0;
  int64_t ctl[2] = {0, -1};
  for (int64_t start = 0; start < m && rc == BTK_OK;) {
    // A window of the path is kriged in parallel against the nodes before it;
    // about window * most / (2 known) of its nodes go stale (sgs.rs:679-683).
    const int64_t known = n_data + start;
    int64_t size = batch > 0 ? batch : known / (most > 0 ? most : 1);
    size = std::max<int64_t>(batch > 0 ? 1 : 1024, std::min<int64_t>(size, batch > 0 ? 65536 : 8192));
    const int64_t end = std::min(m, start + size);
    for (int64_t round = 0; round <= size; ++round) {
      if ((rc = [&]() -> int {
             CK(launch_sgs_pending(L, start, end, node0, ctx->sg_done.p, ctx->sg_list.p, ctx->sg_ctl.p));
             CK(cudaMemcpyAsync(ctl, ctx->sg_ctl.p, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, L.stream));
             CK(cudaStreamSynchronize(L.stream));
             return BTK_OK;
           }()))
        break;
      if (ctl[1] >= 0) {
        rc = fail(ctx, BTK_EINVAL, "kriging failed at node " + std::to_string(ctl[1]) + " of the path (singular system)");
        break;
      }
      if (ctl[0] == 0) break;
      ++total_rounds;
      if ((rc = run_path(ctx, L.stream, m, ctx->x.p + n_data, ctx->y.p + n_data, ctx->z.p + n_data, ctx->sg_list.p,
                         ctl[0], 0, BTK_SIMPLE, 0.0, BTK_FP64, &d)))
        break;
      cudaError_t e = launch_sgs_commit(L, ctl[0], ctx->sg_list.p, d.value, d.variance, d.status, ctx->sg_z.p, node0,
                                        ctx->v.p, ctx->sg_done.p, ctx->sg_score.p, ctx->sg_how.p, ctx->sg_ctl.p + 1);
      if (e != cudaSuccess) {
        rc = fail(ctx, BTK_ECUDA, cudaGetErrorString(e));
        break;
      }
    }
    if (rc == BTK_OK && ctl[0] != 0) rc = fail(ctx, BTK_ECUDA, "simulation window did not finish");
    start = end;
  }
  ctx->spd = saved;
  if (rc) return rc;
  CK(cudaMemcpyAsync(score, ctx->sg_score.p, mm * sizeof(double), cudaMemcpyDeviceToHost, L.stream));
  if (how) CK(cudaMemcpyAsync(how, ctx->sg_how.p, mm, cudaMemcpyDeviceToHost, L.stream));
  CK(cudaStreamSynchronize(L.stream));
  if (rounds) *rounds = total_rounds;
  return BTK_OK;
}

int btk_cross_validate(btk_ctx* ctx, int32_t kind, double kparam, int32_t precision, const btk_outputs* out) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!out || !out->value) return fail(ctx, BTK_EINVAL, "outputs need a value array");
  CK(cudaSetDevice(ctx->device));
  btk_outputs d{};
  if ((rc = host_outputs(ctx, ctx->n, out, &d))) return rc;
  if ((rc = run_path(ctx, nullptr, ctx->n, ctx->x.p, ctx->y.p, ctx->z.p, ctx->loo_perm.p, ctx->n, 1, kind, kparam,
                     precision, &d)))
    return rc;
  return copy_out(ctx, ctx->n, &d, out);
}

int btk_neighbors(btk_ctx* ctx, int64_t m, const double* xyz, int32_t loo, const int32_t* domains, int64_t* idx,
                  int32_t* count, int8_t* ok) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if ((rc = check_domains(ctx, domains, loo != 0))) return rc;
  CK(cudaSetDevice(ctx->device));
  const double* t;
  const int64_t* perm = nullptr;
  if (loo) {
    m = ctx->n;
    t = ctx->x.p;
    perm = ctx->loo_perm.p;
  } else {
    if (m <= 0 || !xyz) return fail(ctx, BTK_EINVAL, "targets are required");
    if ((rc = upload_targets(ctx, m, xyz))) return rc;
    t = ctx->txyz.p;
  }
  if ((rc = ensure_scratch(ctx, m))) return rc;
  Launch L = ctx->launch(nullptr);
  const double *tx = loo ? ctx->x.p : t, *ty = loo ? ctx->y.p : t + m, *tz = loo ? ctx->z.p : t + 2 * m;
  if (domains && !loo) {
    CK(ctx->tdom.grow(size_t(m)));
    CK(cudaMemcpyAsync(ctx->tdom.p, domains, size_t(m) * sizeof(int32_t), cudaMemcpyHostToDevice, L.stream));
  }
  CK(launch_search(L, search_for(ctx, domains ? ctx->tdom.p : nullptr, loo != 0), ctx->gd, tx, ty, tz, perm, m,
                   loo ? 1 : 0, ctx->nbr.p, ctx->cnt.p, ctx->sst.p));
  const size_t k = size_t(ctx->search.max_samples);
  std::vector<uint32_t> nb(size_t(m) * k);
  std::vector<int8_t> st(m);
  CK(cudaMemcpyAsync(nb.data(), ctx->nbr.p, nb.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, L.stream));
  CK(cudaMemcpyAsync(count, ctx->cnt.p, size_t(m) * sizeof(int32_t), cudaMemcpyDeviceToHost, L.stream));
  CK(cudaMemcpyAsync(st.data(), ctx->sst.p, size_t(m) * sizeof(int8_t), cudaMemcpyDeviceToHost, L.stream));
  CK(cudaStreamSynchronize(L.stream));
  for (size_t i = 0; i < nb.size(); ++i) idx[i] = nb[i] == 0xffffffffu ? -1 : int64_t(nb[i]);
  for (int64_t i = 0; i < m; ++i) ok[i] = st[i] == BTK_ST_OK ? 1 : 0;
  return BTK_OK;
}

int btk_loo_freeze(btk_ctx* ctx) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (ctx->search.max_samples > kMaxN)
    return fail(ctx, BTK_EUNSUPPORTED, "the leave-one-out gradient takes at most 64 samples per system");
  if (ctx->search.calibration)
    return fail(ctx, BTK_EUNSUPPORTED, "the leave-one-out gradient takes an uncalibrated search");
  if (ctx->has_dom) return fail(ctx, BTK_EUNSUPPORTED, "the leave-one-out gradient takes samples without domains");
  CK(cudaSetDevice(ctx->device));
  const int64_t n = ctx->n;
  CK(ctx->loo_nbr.grow(size_t(n) * size_t(ctx->search.max_samples)));
  CK(ctx->loo_cnt.grow(size_t(n)));
  CK(ctx->loo_sst.grow(size_t(n)));
  Launch L = ctx->launch(nullptr);
  CK(launch_search(L, ctx->spd, ctx->gd, ctx->x.p, ctx->y.p, ctx->z.p, ctx->loo_perm.p, n, 1, ctx->loo_nbr.p,
                   ctx->loo_cnt.p, ctx->loo_sst.p));
  CK(cudaStreamSynchronize(L.stream));
  ctx->frozen = true;
  return BTK_OK;
}

namespace {

enum Objective { kLeaveOneOut = 0, kBlockMean = 1 };

// Sums over the frozen systems first .. first + count - 1 of an objective
// (leave-one-out loss or block-model mean estimate): sums[0] = objective sum,
// sums[1] = systems in it, sums[2 + k] = gradient sum of parameter k.
// values (full length, or null) gets the range's estimates.
int objective_sums(btk_ctx* ctx, Objective which, const btk_variogram* vg, int64_t first, int64_t count,
                   int32_t want_grad, int32_t precision, std::vector<double>& sums, double* values) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  const bool mean = which == kBlockMean;
  const char* what = mean ? "the mean-estimate gradient" : "the leave-one-out gradient";
  if (mean ? ctx->mean_m <= 0 : !ctx->frozen)
    return fail(ctx, BTK_EINVAL, mean ? "call btk_mean_freeze first" : "call btk_loo_freeze first");
  if (precision != BTK_FP64 && precision != BTK_MIXED) return fail(ctx, BTK_EINVAL, "unknown precision");
  if ((rc = check_vg(ctx, vg))) return rc;
  for (int k = 0; k < vg->nstruct; ++k)
    if (vg->s[k].model == BTK_POWER)
      return fail(ctx, BTK_EUNSUPPORTED, std::string(what) + " takes stationary variograms (no power structure)");
  const int64_t total = mean ? ctx->mean_m : ctx->n;
  if (first < 0 || count < 0 || first + count > total)
    return fail(ctx, BTK_EINVAL, mean ? "the range must lie within the frozen targets"
                                      : "the range must lie within the fitted samples");
  CK(cudaSetDevice(ctx->device));
  btk_variogram v = *vg;
  if (!v.aniso.on) v.aniso = btk_aniso{1, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0};  // isotropic, as a point of theta
  GradDev a{};
  make_vgdev(v, a.vg);
  // At unit ratios and zero angles (a variogram without anisotropy, as the
  // prediction path takes it) the lags are the plain Euclidean ones of
  // lag_world without a frame: the frame, rotation(0, 0, 0), is orthogonal
  // there, and it still gives the angle and ratio derivatives.
  const btk_aniso& an = v.aniso;
  a.vg.has_frame = (an.semi == an.major && an.minor == an.major && an.azimuth == 0.0 && an.dip == 0.0 &&
                    an.rake == 0.0) ? 0 : 1;
  aniso_derivatives(v.aniso, a.dM);
  const int ntheta = 1 + 2 * v.nstruct + 5;
  a.sx = ctx->x.p, a.sy = ctx->y.p, a.sz = ctx->z.p, a.sv = ctx->v.p, a.se = ctx->has_err ? ctx->e.p : nullptr;
  a.twin = ctx->twin.p;
  if (mean) {
    a.tx = ctx->mean_txyz.p, a.ty = ctx->mean_txyz.p + total, a.tz = ctx->mean_txyz.p + 2 * total;
    a.nbr = ctx->mean_nbr.p, a.count = ctx->mean_cnt.p, a.sstatus = ctx->mean_sst.p;
  } else {
    a.nbr = ctx->loo_nbr.p, a.count = ctx->loo_cnt.p, a.sstatus = ctx->loo_sst.p;
  }
  a.max_samples = int(ctx->search.max_samples);
  a.first = first;
  a.n = count;
  a.want_grad = want_grad ? 1 : 0;
  a.stride = 2 + ntheta;
  sums.assign(size_t(a.stride), 0.0);
  if (count == 0) return BTK_OK;
  CK(ctx->g_part.grow(size_t(count) * size_t(a.stride)));
  CK(ctx->g_sums.grow(size_t(a.stride)));
  a.part = ctx->g_part.p;
  if (precision == BTK_MIXED) {
    CK(ctx->g_redo.grow(size_t(count) + 1));
    a.redo_len = ctx->g_redo.p, a.redo = ctx->g_redo.p + 1;
  }
  if (values) {
    CK(ctx->g_val.grow(size_t(total)));
    a.value = ctx->g_val.p;
  }
  Launch L = ctx->launch(nullptr);
  ctx->mark(0, L.stream);
  // The mixed form's systems above 32 samples take the FP64 kernel when the
  // tuning says so, as in the prediction path (tuning.mixed_large).
  const int rows = ctx->search.max_samples > 32 ? 64 : 32;
  CK(launch_grad(L, a, ctx->g_sums.p, rows, precision == BTK_MIXED && !(rows > 32 && ctx->tuning.mixed_large)));
  ctx->mark(1, L.stream);
  ctx->mark(2, L.stream);
  ctx->mark(3, L.stream);
  CK(cudaMemcpyAsync(sums.data(), ctx->g_sums.p, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, L.stream));
  if (values)
    CK(cudaMemcpyAsync(values + first, a.value + first, size_t(count) * sizeof(double), cudaMemcpyDeviceToHost,
                       L.stream));
  CK(cudaStreamSynchronize(L.stream));
  return BTK_OK;
}

int finish_objective(const std::vector<double>& sums, int32_t want_grad, double* obj, double* grad,
                     int64_t* n_valid) {
  const int ntheta = int(sums.size()) - 2;
  const double cnt = sums[1];
  *obj = cnt > 0 ? sums[0] / cnt : NAN;
  if (n_valid) *n_valid = int64_t(cnt);
  if (grad && want_grad)
    for (int k = 0; k < ntheta; ++k) grad[k] = cnt > 0 ? sums[2 + k] / cnt : NAN;
  return BTK_OK;
}

}  // namespace

int btk_loo_gradient(btk_ctx* ctx, const btk_variogram* vg, int32_t want_grad, int32_t precision, double* loss,
                     double* grad, int64_t* n_valid, double* values) {
  if (!loss) return fail(ctx, BTK_EINVAL, "loss is required");
  std::vector<double> sums;
  const int rc = objective_sums(ctx, kLeaveOneOut, vg, 0, ctx ? ctx->n : 0, want_grad, precision, sums, values);
  if (rc) return rc;
  return finish_objective(sums, want_grad, loss, grad, n_valid);
}

int btk_loo_gradient_range(btk_ctx* ctx, const btk_variogram* vg, int64_t first, int64_t count, int32_t want_grad,
                           int32_t precision, double* sums) {
  if (!sums) return fail(ctx, BTK_EINVAL, "sums is required");
  std::vector<double> s;
  const int rc = objective_sums(ctx, kLeaveOneOut, vg, first, count, want_grad, precision, s, nullptr);
  if (rc) return rc;
  for (size_t k = 0; k < s.size(); ++k) sums[k] = (k < 2 || want_grad) ? s[k] : 0.0;
  return BTK_OK;
}

int btk_mean_freeze(btk_ctx* ctx, const btk_geometry* g) {
  int rc = need_fit(ctx);
  if (rc) return rc;
  if (!g) return fail(ctx, BTK_EINVAL, "geometry is required");
  for (int a = 0; a < 3; ++a) {
    if (!(g->size[a] > 0.0 && fin(g->size[a]))) return fail(ctx, BTK_EINVAL, "cell sizes must be positive");
    if (g->count[a] <= 0) return fail(ctx, BTK_EINVAL, "cell counts must be positive");
    if (!fin(g->origin[a]) || !fin(g->rotation[a])) return fail(ctx, BTK_EINVAL, "origin and rotation must be finite");
  }
  if (ctx->search.max_samples > kMaxN)
    return fail(ctx, BTK_EUNSUPPORTED, "the mean-estimate gradient takes at most 64 samples per system");
  if (ctx->search.calibration)
    return fail(ctx, BTK_EUNSUPPORTED, "the mean-estimate gradient takes an uncalibrated search");
  if (ctx->has_dom) return fail(ctx, BTK_EUNSUPPORTED, "the mean-estimate gradient takes samples without domains");
  CK(cudaSetDevice(ctx->device));
  const int64_t m = g->count[0] * g->count[1] * g->count[2];
  const int* tw = ctx->tuning.tile;
  const int64_t tiles = ((g->count[0] + tw[0] - 1) / tw[0]) * ((g->count[1] + tw[1] - 1) / tw[1]) *
                        ((g->count[2] + tw[2] - 1) / tw[2]);
  const int64_t nwork = tiles * 32;
  ctx->mean_m = 0;
  CK(ctx->mean_txyz.grow(3 * size_t(m)));
  CK(ctx->mean_nbr.grow(size_t(m) * size_t(ctx->search.max_samples)));
  CK(ctx->mean_cnt.grow(size_t(m)));
  CK(ctx->mean_sst.grow(size_t(m)));
  CK(ctx->perm.grow(size_t(nwork)));
  Launch L = ctx->launch(nullptr);
  double* t = ctx->mean_txyz.p;
  CK(launch_centroids(L, *g, transposed_frame(*g), 0, nwork, t, t + m, t + 2 * m, ctx->perm.p));
  CK(launch_search(L, ctx->spd, ctx->gd, t, t + m, t + 2 * m, ctx->perm.p, nwork, 0, ctx->mean_nbr.p,
                   ctx->mean_cnt.p, ctx->mean_sst.p));
  CK(cudaStreamSynchronize(L.stream));
  ctx->mean_m = m;
  return BTK_OK;
}

int btk_mean_gradient(btk_ctx* ctx, const btk_variogram* vg, int32_t want_grad, int32_t precision, double* mean,
                      double* grad, int64_t* n_valid, double* values) {
  if (!mean) return fail(ctx, BTK_EINVAL, "mean is required");
  std::vector<double> sums;
  const int rc =
      objective_sums(ctx, kBlockMean, vg, 0, ctx ? ctx->mean_m : 0, want_grad, precision, sums, values);
  if (rc) return rc;
  return finish_objective(sums, want_grad, mean, grad, n_valid);
}

int btk_mean_gradient_range(btk_ctx* ctx, const btk_variogram* vg, int64_t first, int64_t count, int32_t want_grad,
                            int32_t precision, double* sums) {
  if (!sums) return fail(ctx, BTK_EINVAL, "sums is required");
  std::vector<double> s;
  const int rc = objective_sums(ctx, kBlockMean, vg, first, count, want_grad, precision, s, nullptr);
  if (rc) return rc;
  for (size_t k = 0; k < s.size(); ++k) sums[k] = (k < 2 || want_grad) ? s[k] : 0.0;
  return BTK_OK;
}

int btk_centroids(btk_ctx* ctx, const btk_geometry* g, int64_t first, int64_t m, double* xyz) {
  if (!ctx || !g || m < 0) return fail(ctx, BTK_EINVAL, "geometry and a non-negative count are required");
  if (m == 0) return BTK_OK;
  CK(cudaSetDevice(ctx->device));
  CK(ctx->txyz.grow(3 * size_t(m)));
  Launch L = ctx->launch(nullptr);
  double* t = ctx->txyz.p;
  CK(launch_centroids(L, *g, transposed_frame(*g), first, m, t, t + m, t + 2 * m, nullptr));
  std::vector<double> a(3 * size_t(m));
  CK(cudaMemcpyAsync(a.data(), t, a.size() * sizeof(double), cudaMemcpyDeviceToHost, L.stream));
  CK(cudaStreamSynchronize(L.stream));
  for (int64_t i = 0; i < m; ++i) xyz[3 * i] = a[i], xyz[3 * i + 1] = a[m + i], xyz[3 * i + 2] = a[2 * m + i];
  return BTK_OK;
}

}  // extern "C"
