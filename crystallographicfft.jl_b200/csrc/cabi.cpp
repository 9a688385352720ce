// extern "C" entry points of libcfft_b200 (declared in include/cfft_b200.h).
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/cfft_b200.h"
#include "exec.h"
#include "fast_api.h"
#include "scft.h"
#include "sno.h"
#include "fractal_tree.h"

using cfft::Status;

namespace {

thread_local std::string g_last_error;

cfft_status ret(Status s, const std::string& msg = std::string()) {
  if (s != Status::kOk) g_last_error = msg;
  return static_cast<cfft_status>(static_cast<int>(s));
}

bool read_ops(int dim, int n_ops, const int32_t* R, const int32_t* t, std::vector<cfft::SymOp>* ops,
              std::string* err) {
  if (dim != 2 && dim != 3) { *err = "dim must be 2 or 3"; return false; }
  if (n_ops < 1 || !R || !t) { *err = "empty or null operation list"; return false; }
  ops->resize(n_ops);
  for (int k = 0; k < n_ops; ++k) {
    cfft::SymOp& op = (*ops)[k];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) op.R[i][j] = R[9 * k + 3 * i + j];
    for (int i = 0; i < 3; ++i) op.t[i] = t[3 * k + i];
    for (int d = dim; d < 3; ++d) {
      op.t[d] = 0;
      for (int j = 0; j < 3; ++j) op.R[d][j] = op.R[j][d] = (d == j);
    }
  }
  return true;
}

bool read_N(int dim, const int* N, int* out, std::string* err) {
  if (!N) { *err = "null grid"; return false; }
  for (int d = 0; d < 3; ++d) out[d] = d < dim ? N[d] : 1;
  for (int d = 0; d < dim; ++d)
    if (out[d] < 1) { *err = "grid edges must be positive"; return false; }
  return true;
}

}  // namespace

extern "C" {

cfft_status cfft_get_ops(int sg, int dim, const int* N, int cap, int* n_ops, int32_t* R, int32_t* t) {
  std::string err;
  int n[3];
  if (!n_ops || !read_N(dim, N, n, &err)) return ret(Status::kInvalid, err.empty() ? "null argument" : err);
  std::vector<cfft::SymOp> ops;
  Status s = cfft::get_ops(sg, dim, n, &ops, &err);
  if (s != Status::kOk) return ret(s, err);
  *n_ops = static_cast<int>(ops.size());
  if (!R || !t) return CFFT_OK;
  if (cap < *n_ops) return ret(Status::kInvalid, "capacity too small for the operation list");
  for (size_t k = 0; k < ops.size(); ++k) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) R[9 * k + 3 * i + j] = ops[k].R[i][j];
    for (int i = 0; i < 3; ++i) t[3 * k + i] = ops[k].t[i];
  }
  return CFFT_OK;
}

int cfft_list_groups(int dim, int* out, int cap) { return cfft::list_groups(dim, out, cap); }

cfft_status cfft_find_optimal_shift(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t,
                                    double* shift, int32_t* t_shifted) {
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(dim, N, n, &err) || !read_ops(dim, n_ops, R, t, &ops, &err)) return ret(Status::kInvalid, err);
  if (!shift || !t_shifted) return ret(Status::kInvalid, "null output");
  double sh[3];
  std::vector<cfft::SymOp> out;
  cfft::find_optimal_shift(ops, n, dim, sh, &out);
  for (int d = 0; d < dim; ++d) shift[d] = sh[d];
  for (int k = 0; k < n_ops; ++k)
    for (int i = 0; i < 3; ++i) t_shifted[3 * k + i] = out[k].t[i];
  return CFFT_OK;
}

int cfft_count_special_positions(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t) {
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(dim, N, n, &err) || !read_ops(dim, n_ops, R, t, &ops, &err)) { ret(Status::kInvalid, err); return -1; }
  return cfft::count_special_positions_fast(n, dim, ops);
}

cfft_status cfft_auto_L(int dim, int n_ops, const int32_t* R, const int32_t* t, int* L) {
  std::string err;
  std::vector<cfft::SymOp> ops;
  if (!read_ops(dim, n_ops, R, t, &ops, &err) || !L) return ret(Status::kInvalid, err.empty() ? "null output" : err);
  auto l = cfft::auto_L(ops, dim);
  for (int d = 0; d < 3; ++d) L[d] = l[d];
  return CFFT_OK;
}

int cfft_detect_centering(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t) {
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(dim, N, n, &err) || !read_ops(dim, n_ops, R, t, &ops, &err)) { ret(Status::kInvalid, err); return -1; }
  return static_cast<int>(cfft::detect_centering_type(ops, n, dim));
}

cfft_status cfft_spectral_asu(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t, int cap,
                              int* n_spec, int32_t* idx, int32_t* mult) {
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(dim, N, n, &err) || !read_ops(dim, n_ops, R, t, &ops, &err) || !n_spec)
    return ret(Status::kInvalid, err.empty() ? "null output" : err);
  if (static_cast<long>(n[0]) * n[1] * n[2] > (1L << 28)) return ret(Status::kUnsupported, "grid too large");
  auto pts = cfft::calc_spectral_asu(ops, n, dim);
  *n_spec = static_cast<int>(pts.size());
  if (!idx && !mult) return CFFT_OK;
  if (cap < *n_spec) return ret(Status::kInvalid, "capacity too small for the spectral ASU");
  for (size_t s = 0; s < pts.size(); ++s) {
    if (idx)
      for (int d = 0; d < 3; ++d) idx[3 * s + d] = pts[s].h[d];
    if (mult) mult[s] = pts[s].mult;
  }
  return CFFT_OK;
}

static cfft_status plan_create_impl(const cfft_desc* desc, cfft_plan* plan, bool device,
                                    const cfft_tuning* tuning = nullptr) {
  if (!desc || !plan) return ret(Status::kInvalid, "null argument");
  *plan = nullptr;
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(desc->dim, desc->N, n, &err) || !read_ops(desc->dim, desc->n_ops, desc->R, desc->t, &ops, &err))
    return ret(Status::kInvalid, err);
  if (desc->precision != 4 && desc->precision != 8) return ret(Status::kInvalid, "precision must be 4 or 8");
  if (desc->max_batch < 1) return ret(Status::kInvalid, "max_batch must be positive");
  if (desc->path < 0 || desc->path > 5) return ret(Status::kInvalid, "unknown path");
  auto* p = new (std::nothrow) cfft::Plan();
  if (!p) return ret(Status::kAlloc, "host allocation failed");
  p->precision = desc->precision;
  p->max_batch = desc->max_batch;
  if (tuning) {
    p->tune.chunk_bytes = tuning->chunk_bytes;
    p->tune.lanes = tuning->lanes;
    p->tune.zr_slots = tuning->zr_slots;
    p->tune.wide = tuning->wide;
    p->tune.tma = tuning->tma;
    p->tune.cluster = tuning->cluster;
  }
  p->ds = desc->ds;
  std::memcpy(p->lattice, desc->lattice, sizeof(p->lattice));
  const bool plain = desc->path == CFFT_PATH_M2 || desc->path == CFFT_PATH_M2Q;
  Status s = cfft::build_tables(ops, n, desc->dim, !plain, &p->T, &err, desc->path == CFFT_PATH_FULLGRID);
  if (s == Status::kOk && (desc->path == CFFT_PATH_M2Q || desc->path == CFFT_PATH_M7)) {
    // plan_m7_scft (src/q_fused_krfft.jl:822-850) refuses P lattices and odd subgrids;
    // the centred plan exists exactly when neither holds.
    if (desc->path == CFFT_PATH_M7 && !p->T.centered) {
      s = Status::kInvalid;
      err = "M7 SCFT requires a centred lattice (I/F/C/A) with L = 2 and even M; use M2Q";
    } else {
      p->qmode = desc->path;
      s = cfft::build_q_tables(p->T, p->lattice, p->ds, &p->q_host, &p->q_gather, &err);
    }
  }
  if (s == Status::kOk && device) s = cfft::plan_device_init(p, &err);
  if (s == Status::kOk && !device) cfft::compute_kernel(p->T, p->lattice, p->ds, &p->T.K);
  if (s != Status::kOk) {
    cfft::plan_device_free(p);
    delete p;
    return ret(s, err);
  }
  *plan = reinterpret_cast<cfft_plan>(p);
  return CFFT_OK;
}

cfft_status cfft_plan_create(const cfft_desc* desc, cfft_plan* plan) { return plan_create_impl(desc, plan, true); }
cfft_status cfft_plan_create_tuned(const cfft_desc* desc, const cfft_tuning* tuning, cfft_plan* plan) {
  if (tuning && (tuning->lanes < 0 || tuning->lanes > 4 || (tuning->zr_slots && tuning->zr_slots != 2 &&
                 tuning->zr_slots != 4) || tuning->wide < -1 || tuning->wide > 1 || tuning->tma < -1 ||
                 tuning->tma > 3 || (tuning->cluster > 0 && tuning->cluster != 8 && tuning->cluster != 16) ||
                 tuning->cluster < -1 || tuning->chunk_bytes < 0))
    return ret(Status::kInvalid, "invalid tuning value");
  return plan_create_impl(desc, plan, true, tuning);
}
cfft_status cfft_plan_create_host(const cfft_desc* desc, cfft_plan* plan) { return plan_create_impl(desc, plan, false); }

cfft_status cfft_plan_destroy(cfft_plan plan) {
  if (!plan) return CFFT_OK;
  auto* p = reinterpret_cast<cfft::Plan*>(plan);
  cfft::plan_device_free(p);
  delete p;
  return CFFT_OK;
}

cfft_status cfft_plan_info(cfft_plan plan, cfft_info* info) {
  if (!plan || !info) return ret(Status::kInvalid, "null argument");
  const auto* p = reinterpret_cast<cfft::Plan*>(plan);
  const auto& T = p->T;
  for (int d = 0; d < 3; ++d) { info->N[d] = T.N[d]; info->L[d] = T.L[d]; info->M[d] = T.M[d]; info->H[d] = T.H[d]; }
  info->n_spec = static_cast<int>(T.spec.size());
  info->n_ops = static_cast<int>(T.ops.size());
  info->n_rep = T.d;
  info->centering = static_cast<int>(T.centering);
  info->centered = T.centered ? 1 : 0;
  info->n_channels = T.n_ch;
  info->n_orbits = static_cast<int>(T.orbit_rep.size());
  info->n_rem_ops = static_cast<int>(T.rem_ops.size());
  info->precision = p->precision;
  info->max_batch = p->max_batch;
  info->P = T.P;
  info->workspace_bytes = static_cast<int64_t>(p->workspace_bytes);
  int tma = 0;
  if (p->fast_h > 0 && !p->cluster && p->d_geom) {
    bool fw = false, fwe = false, bw = false;
    if (p->precision == 8) cfft::fast_tma_planes_f64(p->fast_h, p->cent_type, p->tune.tma, &fw, &fwe, &bw);
    else cfft::fast_tma_planes_f32(p->fast_h, p->cent_type, p->tune.tma, &fw, &fwe, &bw);
    tma = (fw ? 8 : 0) | (bw ? 16 : 0);
  }
  info->exec_path = (p->fast_h > 0 ? 1 : 0) | (p->reps_quad ? 2 : 0) | (p->cluster ? 4 : 0) | tma |
                    (p->reps_wide && !p->cluster ? 32 : 0) | (p->qsep ? 64 : 0);
  info->chunk = p->chunk;
  info->lanes = p->lanes;
  return CFFT_OK;
}

cfft_status cfft_block_plan_create(int n_blocks, const int32_t* dims, int precision, cfft_block_plan* plan) {
  if (!plan) return ret(Status::kInvalid, "null argument");
  *plan = nullptr;
  std::string err;
  cfft::BlockPlan* bp = nullptr;
  const Status s = cfft::block_plan_create(n_blocks, dims, precision, &bp, &err);
  if (s != Status::kOk) return ret(s, err);
  *plan = reinterpret_cast<cfft_block_plan>(bp);
  return CFFT_OK;
}

cfft_status cfft_block_plan_destroy(cfft_block_plan plan) {
  cfft::block_plan_destroy(reinterpret_cast<cfft::BlockPlan*>(plan));
  return CFFT_OK;
}

cfft_status cfft_block_forward(cfft_block_plan plan, const void* in, void* out, void* stream) {
  std::string err;
  return ret(cfft::block_execute(reinterpret_cast<cfft::BlockPlan*>(plan), in, out, false, stream, &err), err);
}

cfft_status cfft_block_backward(cfft_block_plan plan, const void* in, void* out, void* stream) {
  std::string err;
  return ret(cfft::block_execute(reinterpret_cast<cfft::BlockPlan*>(plan), in, out, true, stream, &err), err);
}

cfft_status cfft_calc_asu(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t, int cap,
                          int* n_points, int32_t* idx, int32_t* depth, int32_t* mult) {
  if (!n_points) return ret(Status::kInvalid, "null argument");
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(dim, N, n, &err) || !read_ops(dim, n_ops, R, t, &ops, &err)) return ret(Status::kInvalid, err);
  for (auto& op : ops)
    for (int d = dim; d < 3; ++d) {
      op.t[d] = 0;
      for (int j = 0; j < 3; ++j) op.R[d][j] = op.R[j][d] = (d == j);
    }
  const auto pts = cfft::calc_asu(ops, n, dim);
  *n_points = static_cast<int>(pts.size());
  if (!idx && !depth && !mult) return CFFT_OK;
  if (cap < *n_points) return ret(Status::kInvalid, "capacity too small for the ASU");
  for (size_t k = 0; k < pts.size(); ++k) {
    for (int d = 0; d < 3; ++d) {
      if (idx) idx[3 * k + d] = pts[k].idx[d];
      if (depth) depth[3 * k + d] = pts[k].depth[d];
    }
    if (mult) mult[k] = pts[k].mult;
  }
  return CFFT_OK;
}

cfft_status cfft_fractal_tree(int dim, const int* N, int n_ops, const int32_t* R, const int32_t* t, int flags, int cap,
                              int* n_leaves, int* n_inner, int32_t* leaves) {
  if (!n_leaves || !n_inner) return ret(Status::kInvalid, "null argument");
  std::string err;
  int n[3];
  std::vector<cfft::SymOp> ops;
  if (!read_N(dim, N, n, &err) || !read_ops(dim, n_ops, R, t, &ops, &err)) return ret(Status::kInvalid, err);
  if (flags < 0 || flags > 3) return ret(Status::kInvalid, "flags must be 0..3");
  std::vector<cfft::TreeLeaf> lv;
  cfft::fractal_tree(ops, n, dim, flags, &lv, n_inner);
  *n_leaves = static_cast<int>(lv.size());
  if (!leaves) return CFFT_OK;
  if (cap < *n_leaves) return ret(Status::kInvalid, "capacity too small for the tree's leaves");
  for (size_t k = 0; k < lv.size(); ++k) {
    for (int d = 0; d < 3; ++d) {
      leaves[10 * k + d] = lv[k].n[d];
      leaves[10 * k + 3 + d] = lv[k].scale[d];
      leaves[10 * k + 6 + d] = lv[k].offset[d];
    }
    leaves[10 * k + 9] = lv[k].depth;
  }
  return CFFT_OK;
}

cfft_status cfft_plan_q_tables(cfft_plan plan, double* Q, int32_t* gather) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  const auto* p = reinterpret_cast<cfft::Plan*>(plan);
  if (!p->qmode) return ret(Status::kUnsupported, "not an M2Q / M7 plan");
  if (Q) std::memcpy(Q, p->q_host.data(), p->q_host.size() * sizeof(double));
  if (gather) std::memcpy(gather, p->q_gather.data(), p->q_gather.size() * sizeof(int32_t));
  return CFFT_OK;
}

cfft_status cfft_plan_spectral_asu(cfft_plan plan, int32_t* idx, int32_t* mult) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  const auto& T = reinterpret_cast<cfft::Plan*>(plan)->T;
  for (size_t s = 0; s < T.spec.size(); ++s) {
    if (idx)
      for (int d = 0; d < 3; ++d) idx[3 * s + d] = T.spec[s].h[d];
    if (mult) mult[s] = T.spec[s].mult;
  }
  return CFFT_OK;
}

cfft_status cfft_plan_rep_ops(cfft_plan plan, int32_t* R, int32_t* t) {
  if (!plan || !R || !t) return ret(Status::kInvalid, "null argument");
  const auto& T = reinterpret_cast<cfft::Plan*>(plan)->T;
  for (size_t k = 0; k < T.rep_ops.size(); ++k) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) R[9 * k + 3 * i + j] = T.rep_ops[k].R[i][j];
    for (int i = 0; i < 3; ++i) t[3 * k + i] = T.rep_ops[k].t[i];
  }
  return CFFT_OK;
}

cfft_status cfft_plan_backward_tables(cfft_plan plan, int32_t* orbit_rep, int32_t* inv_spec, int32_t* inv_phase) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  const auto& T = reinterpret_cast<cfft::Plan*>(plan)->T;
  if (orbit_rep) std::memcpy(orbit_rep, T.orbit_rep.data(), T.orbit_rep.size() * 4);
  if (inv_spec) std::memcpy(inv_spec, T.inv_spec.data(), T.inv_spec.size() * 4);
  if (inv_phase) std::memcpy(inv_phase, T.inv_phase.data(), T.inv_phase.size() * 4);
  return CFFT_OK;
}

cfft_status cfft_plan_kernel(cfft_plan plan, double* K) {
  if (!plan || !K) return ret(Status::kInvalid, "null argument");
  const auto& T = reinterpret_cast<cfft::Plan*>(plan)->T;
  std::memcpy(K, T.K.data(), T.K.size() * sizeof(double));
  return CFFT_OK;
}

cfft_status cfft_update_kernel(cfft_plan plan, double ds, const double* lattice) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  auto* p = reinterpret_cast<cfft::Plan*>(plan);
  p->ds = ds;
  if (lattice) std::memcpy(p->lattice, lattice, sizeof(p->lattice));
  std::string err;
  if (p->qmode) {  // update_m2_kernel! rebuilds the Q matrices (src/q_fused_krfft.jl:1036-1052)
    Status s = cfft::build_q_tables(p->T, p->lattice, p->ds, &p->q_host, &p->q_gather, &err);
    if (s != Status::kOk) return ret(s, err);
  }
  if (!p->d_geom) {
    cfft::compute_kernel(p->T, p->lattice, p->ds, &p->T.K);
    return CFFT_OK;
  }
  return ret(cfft::plan_upload_kernel(p, &err), err);
}

#define CFFT_EXEC(expr)                                               \
  do {                                                                \
    if (!plan) return ret(Status::kInvalid, "null plan");            \
    auto* p = reinterpret_cast<cfft::Plan*>(plan);                    \
    if (!p->d_geom) return ret(Status::kInvalid, "plan has no device state (created with cfft_plan_create_host)"); \
    std::string err;                                                  \
    Status s_ = (expr);                                               \
    return ret(s_, err);                                              \
  } while (0)

cfft_status cfft_scft_create(cfft_plan plan, const cfft_scft_params* params, cfft_scft* scft) {
  if (!plan || !params || !scft) return ret(Status::kInvalid, "null argument");
  cfft::ScftParams prm;
  prm.f = params->f;
  prm.chiN = params->chiN;
  prm.Ns = params->Ns;
  prm.history = params->history;
  prm.tol = params->tol;
  prm.max_iter = params->max_iter;
  prm.lam_simple = params->lam_simple;
  prm.lam_anderson = params->lam_anderson;
  prm.anderson_start = params->anderson_start;
  prm.min_simple = params->min_simple;
  std::string err;
  cfft::Scft* s = nullptr;
  const Status st = cfft::scft_create(reinterpret_cast<cfft::Plan*>(plan), prm, &s, &err);
  if (st == Status::kOk) *scft = reinterpret_cast<cfft_scft>(s);
  return ret(st, err);
}

int64_t cfft_sno_param_count(void) { return cfft::SnoLayout::total; }

cfft_status cfft_sno_create(const cfft_sno_config* cfg, cfft_sno* model) {
  if (!model) return ret(Status::kInvalid, "null argument");
  cfft::SnoConfig c;
  if (cfg) {
    c.lr = cfg->lr;
    c.beta1 = cfg->beta1;
    c.beta2 = cfg->beta2;
    c.eps = cfg->eps;
    c.weight_decay = cfg->weight_decay;
  }
  std::string err;
  cfft::SnoModel* m = nullptr;
  const Status st = cfft::sno_model_create(c, &m, &err);
  if (st == Status::kOk) *model = reinterpret_cast<cfft_sno>(m);
  return ret(st, err);
}

cfft_status cfft_sno_destroy(cfft_sno model) {
  cfft::sno_model_destroy(reinterpret_cast<cfft::SnoModel*>(model));
  return CFFT_OK;
}

cfft_status cfft_sno_set_params(cfft_sno model, const float* host) {
  if (!model || !host) return ret(Status::kInvalid, "null argument");
  std::string err;
  return ret(cfft::sno_set_params(reinterpret_cast<cfft::SnoModel*>(model), host, &err), err);
}

cfft_status cfft_sno_get_params(cfft_sno model, float* host) {
  if (!model || !host) return ret(Status::kInvalid, "null argument");
  std::string err;
  return ret(cfft::sno_get_params(reinterpret_cast<cfft::SnoModel*>(model), host, &err), err);
}

cfft_status cfft_sno_get_grads(cfft_sno model, float* host) {
  if (!model || !host) return ret(Status::kInvalid, "null argument");
  std::string err;
  return ret(cfft::sno_get_grads(reinterpret_cast<cfft::SnoModel*>(model), host, &err), err);
}

cfft_status cfft_sno_grads_device(cfft_sno model, void* dst, void* stream) {
  if (!model || !dst) return ret(Status::kInvalid, "null argument");
  std::string err;
  return ret(cfft::sno_grads_device(reinterpret_cast<cfft::SnoModel*>(model), dst, stream, &err), err);
}

cfft_status cfft_sno_apply_grads(cfft_sno model, const void* grads, double lr, void* stream) {
  if (!model) return ret(Status::kInvalid, "null argument");
  std::string err;
  return ret(cfft::sno_apply_grads(reinterpret_cast<cfft::SnoModel*>(model), grads, lr, stream, &err), err);
}

cfft_status cfft_sno_bind(cfft_sno model, cfft_plan plan, int group_slot, const double* shift, int max_samples,
                          cfft_sno_ctx* ctx) {
  if (!model || !plan || !shift || !ctx) return ret(Status::kInvalid, "null argument");
  std::string err;
  cfft::SnoCtx* c = nullptr;
  const Status st = cfft::sno_bind(reinterpret_cast<cfft::SnoModel*>(model), reinterpret_cast<cfft::Plan*>(plan),
                                   group_slot, shift, max_samples, &c, &err);
  if (st == Status::kOk) *ctx = reinterpret_cast<cfft_sno_ctx>(c);
  return ret(st, err);
}

cfft_status cfft_sno_unbind(cfft_sno_ctx ctx) {
  cfft::sno_unbind(reinterpret_cast<cfft::SnoCtx*>(ctx));
  return CFFT_OK;
}

cfft_status cfft_sno_predict(cfft_sno_ctx ctx, const double* params, int n_samples, void* w_out, void* stream) {
  std::string err;
  return ret(cfft::sno_predict(reinterpret_cast<cfft::SnoCtx*>(ctx), params, n_samples, w_out, stream, &err), err);
}

cfft_status cfft_sno_train(cfft_sno_ctx ctx, const double* params, int n_samples, const void* w_target, double lr,
                           int step, double* loss, void* stream) {
  std::string err;
  return ret(cfft::sno_train(reinterpret_cast<cfft::SnoCtx*>(ctx), params, n_samples, w_target, lr, step, loss, stream,
                             &err),
             err);
}

cfft_status cfft_scft_destroy(cfft_scft scft) {
  cfft::scft_destroy(reinterpret_cast<cfft::Scft*>(scft));
  return CFFT_OK;
}

static void to_c_state(const cfft::ScftState& s, cfft_scft_state* out) {
  out->Q = s.Q;
  out->F = s.F;
  out->err = s.err;
  out->iterations = s.iterations;
  out->converged = s.converged;
}

cfft_status cfft_scft_evaluate(cfft_scft scft, const void* w, void* phi, void* d, cfft_scft_state* state,
                               void* stream) {
  if (!scft || !state) return ret(Status::kInvalid, "null argument");
  std::string err;
  cfft::ScftState s;
  const Status st = cfft::scft_evaluate(reinterpret_cast<cfft::Scft*>(scft), w, phi, d, &s, stream, &err);
  to_c_state(s, state);
  return ret(st, err);
}

cfft_status cfft_scft_solve(cfft_scft scft, void* w, cfft_scft_state* state, void* stream) {
  if (!scft || !state) return ret(Status::kInvalid, "null argument");
  std::string err;
  cfft::ScftState s;
  const Status st = cfft::scft_solve(reinterpret_cast<cfft::Scft*>(scft), w, &s, stream, &err);
  to_c_state(s, state);
  return ret(st, err);
}

cfft_status cfft_scft_densities(cfft_scft scft, void* phi, void* stream) {
  if (!scft || !phi) return ret(Status::kInvalid, "null argument");
  std::string err;
  return ret(cfft::scft_densities(reinterpret_cast<cfft::Scft*>(scft), phi, stream, &err), err);
}

cfft_status cfft_plan_device_status(cfft_plan plan, int clear) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  std::string err;
  const Status s = cfft::plan_device_status(reinterpret_cast<cfft::Plan*>(plan), clear != 0, &err);
  return ret(s, err);
}

cfft_status cfft_wait_selftest(cfft_plan plan, unsigned long long timeout_ns, void* stream) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  std::string err;
  const Status s = cfft::plan_wait_selftest(reinterpret_cast<cfft::Plan*>(plan), timeout_ns, stream, &err);
  return ret(s, err);
}

cfft_status cfft_forward(cfft_plan plan, const void* f0, void* F, int batch, void* stream) {
  CFFT_EXEC(cfft::exec_forward(p, f0, F, batch, stream, &err));
}
cfft_status cfft_backward(cfft_plan plan, const void* F, void* f0, int batch, void* stream) {
  CFFT_EXEC(cfft::exec_backward(p, F, f0, batch, stream, &err));
}
cfft_status cfft_scft_step(cfft_plan plan, void* f0, int batch, void* stream) {
  CFFT_EXEC(cfft::exec_scft_step(p, f0, batch, stream, &err));
}

cfft_status cfft_forward_plans(int n_plans, const cfft_plan* plans, const void* const* f0, void* const* F,
                               const int* batch, void* stream) {
  if (n_plans < 1 || !plans || !f0 || !F || !batch) return ret(Status::kInvalid, "invalid plan array arguments");
  for (int i = 0; i < n_plans; ++i) {
    const cfft_status st = cfft_forward(plans[i], f0[i], F[i], batch[i], stream);
    if (st != CFFT_OK) {
      g_last_error = "plan " + std::to_string(i) + ": " + g_last_error;
      return st;
    }
  }
  return CFFT_OK;
}

cfft_status cfft_backward_plans(int n_plans, const cfft_plan* plans, const void* const* F, void* const* f0,
                                const int* batch, void* stream) {
  if (n_plans < 1 || !plans || !F || !f0 || !batch) return ret(Status::kInvalid, "invalid plan array arguments");
  for (int i = 0; i < n_plans; ++i) {
    const cfft_status st = cfft_backward(plans[i], F[i], f0[i], batch[i], stream);
    if (st != CFFT_OK) {
      g_last_error = "plan " + std::to_string(i) + ": " + g_last_error;
      return st;
    }
  }
  return CFFT_OK;
}
cfft_status cfft_step_diffusion(cfft_plan plan, void* q, const void* w, double dt, int n_steps, int batch,
                                void* stream) {
  CFFT_EXEC(cfft::exec_step_diffusion(p, q, w, dt, n_steps, batch, stream, &err));
}
cfft_status cfft_fullgrid_to_subgrid(cfft_plan plan, const void* u, void* f0, int batch, void* stream) {
  CFFT_EXEC(cfft::exec_full_to_sub(p, u, f0, batch, stream, &err));
}
cfft_status cfft_subgrid_to_fullgrid(cfft_plan plan, const void* f0, void* u, int batch, void* stream) {
  CFFT_EXEC(cfft::exec_sub_to_full(p, f0, u, batch, stream, &err));
}
cfft_status cfft_subgrid_spectrum(cfft_plan plan, const void* f0, void* G0, int batch, void* stream) {
  CFFT_EXEC(cfft::exec_subgrid_spectrum(p, f0, G0, batch, stream, &err));
}
cfft_status cfft_forward_host(cfft_plan plan, const void* f0_host, void* F_host, int batch) {
  CFFT_EXEC(cfft::exec_host(p, 0, f0_host, F_host, batch, &err));
}
cfft_status cfft_backward_host(cfft_plan plan, const void* F_host, void* f0_host, int batch) {
  CFFT_EXEC(cfft::exec_host(p, 1, F_host, f0_host, batch, &err));
}
cfft_status cfft_scft_step_host(cfft_plan plan, void* f0_host, int batch) {
  CFFT_EXEC(cfft::exec_host(p, 2, nullptr, f0_host, batch, &err));
}

cfft_status cfft_profile_roundtrip(cfft_plan plan, const void* f0, void* F, void* f0_out, int batch, void* stream,
                                   float* stage_ms, int* n_stages) {
  CFFT_EXEC(cfft::exec_profile_roundtrip(p, f0, F, f0_out, batch, stream, stage_ms, n_stages, &err));
}

cfft_status cfft_forward_noalloc(cfft_plan plan, const void* f0, void* F, int batch, void* stream) {
  if (!plan) return ret(Status::kInvalid, "null plan");
  std::string err;
  return ret(cfft::exec_forward_noalloc(reinterpret_cast<cfft::Plan*>(plan), f0, F, batch, stream, &err), err);
}

const char* cfft_status_string(cfft_status s) {
  switch (s) {
    case CFFT_OK: return "ok";
    case CFFT_ERR_INVALID: return "invalid argument";
    case CFFT_ERR_CUDA: return "CUDA error";
    case CFFT_ERR_NOT_COMMENSURATE: return "operation not commensurate with the grid";
    case CFFT_ERR_UNSUPPORTED: return "unsupported size or group";
    case CFFT_ERR_TIMEOUT: return "device wait timed out";
    case CFFT_ERR_ALLOC: return "allocation failed";
    case CFFT_ERR_NOT_REACHABLE: return "subgrid parity class not reachable";
  }
  return "unknown status";
}

const char* cfft_last_error(void) { return g_last_error.c_str(); }

int cfft_version(void) { return 110; }

int64_t cfft_launch_count(int reset) { return cfft::launch_count(reset != 0); }

}  // extern "C"
