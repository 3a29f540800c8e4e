// C ABI of the B200 Peridigm hot path (declarations and reference citations in
// include/pd_b200.h). Host-side orchestration only: argument checks, uploads,
// kernel sequencing on the context's stream, status and error reporting.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bc_expr.cuh"
#include "pd_internal.cuh"

using namespace pdb;

namespace {

const char* kVersion = "pd_b200 0.1 (sm_100a)";

int fail(pd_ctx* c, int code, const std::string& msg) {
  c->err = msg;
  return code;
}

#define CHECK_CTX(c) \
  if (!(c)) return PD_ERR_ARG

#define TRY(expr)                 \
  do {                            \
    int rc_ = (expr);             \
    if (rc_ != PD_OK) return rc_; \
  } while (0)

int ensure_device(pd_ctx* c) {
  PD_CUDA_TRY(c, cudaSetDevice(c->device));
  return PD_OK;
}

// Per-point material arrays from block tables and per-point overrides.
int upload_material(pd_ctx* c) {
  const int64_t n = c->n;
  std::vector<double4> pt(n);
  std::vector<double> sc(n), hp(n);
  c->any_damage = false;
  for (int64_t i = 0; i < n; ++i) {
    const int b = c->hblock.empty() ? 0 : c->hblock[i];
    const double K = c->field_K.empty() ? c->block_K[b] : c->field_K[i];
    const double mu = c->field_mu.empty() ? c->block_mu[b] : c->field_mu[i];
    pt[i] = make_double4(0.0, K, mu, c->block_rho[b]);
    sc[i] = c->field_sc.empty() ? c->block_sc[b] : c->field_sc[i];
    if (sc[i] >= 0.0) c->any_damage = true;
    hp[i] = c->block_h[b];
  }
  PD_CUDA_TRY(c, c->pt.alloc(n));
  PD_CUDA_TRY(c, c->sc.alloc(n));
  PD_CUDA_TRY(c, h2d(c, c->pt.p, pt.data(), n * sizeof(double4)));
  PD_CUDA_TRY(c, h2d(c, c->sc.p, sc.data(), n * sizeof(double)));
  PD_CUDA_TRY(c, h2d(c, c->hp.p, hp.data(), n * sizeof(double)));
  c->sc_min = INFINITY;
  {
    double m = INFINITY;
    for (int64_t i = 0; i < n; ++i)
      if (sc[i] >= 0.0) m = std::min(m, sc[i]);
    c->sc_gate64 = m * (1.0 - 1e-12);
  }
  if (c->precision == PD_SPLIT_FP32) {
    PD_CUDA_TRY(c, c->own.alloc(n));
    std::vector<float> scf(n);
    for (int64_t i = 0; i < n; ++i) {
      scf[i] = (float)sc[i];
      if (scf[i] >= 0.0f) c->sc_min = std::min(c->sc_min, scf[i]);
    }
    PD_CUDA_TRY(c, c->scf.alloc(n));
    PD_CUDA_TRY(c, h2d(c, c->scf.p, scf.data(), n * sizeof(float)));
  }
  return check_sc_pairs(c);
}

int upload_horizons(pd_ctx* c) {
  std::vector<double> hp(c->n);
  for (int64_t i = 0; i < c->n; ++i) hp[i] = c->block_h[c->hblock.empty() ? 0 : c->hblock[i]];
  PD_CUDA_TRY(c, c->hp.alloc(c->n));
  PD_CUDA_TRY(c, h2d(c, c->hp.p, hp.data(), c->n * sizeof(double)));
  return PD_OK;
}

int alloc_state(pd_ctx* c) {
  if (c->u.count >= (size_t)(3 * c->n) && c->n > 0) return PD_OK;
  const int64_t n = c->n;
  for (int k = 0; k < 2; ++k) {
    if (c->precision == PD_SPLIT_FP32) {
      PD_CUDA_TRY(c, c->ur[k].alloc(n));
      PD_CUDA_TRY(c, dzero(c, c->ur[k].p, c->ur[k].bytes()));
    } else {
      PD_CUDA_TRY(c, c->st[k].alloc(n));
      PD_CUDA_TRY(c, dzero(c, c->st[k].p, c->st[k].bytes()));
    }
  }
  PD_CUDA_TRY(c, c->ab64.alloc(c->precision != PD_SPLIT_FP32 ? n : 1));
  PD_CUDA_TRY(c, c->u.alloc(3 * n));
  PD_CUDA_TRY(c, c->v.alloc(3 * n));
  PD_CUDA_TRY(c, c->a.alloc(3 * n));
  PD_CUDA_TRY(c, c->f.alloc(3 * n));
  PD_CUDA_TRY(c, c->fc.alloc(3 * n));
  PD_CUDA_TRY(c, c->theta.alloc(n));
  PD_CUDA_TRY(c, c->node_damage.alloc(n));
  for (auto* b : {&c->u, &c->v, &c->a, &c->f, &c->fc, &c->theta, &c->node_damage})
    PD_CUDA_TRY(c, dzero(c, b->p, b->bytes()));
  c->cur = 0;
  c->state_init = false;
  return PD_OK;
}

// Everything a model evaluation needs: bonds, material, weighted volume, state buffers.
int ensure_ready(pd_ctx* c) {
  TRY(ensure_device(c));
  if (c->n == 0 || !c->row.p) return fail(c, PD_ERR_STATE, "points and bonds must be set first");
  if (!c->have_material)
    return fail(c, PD_ERR_STATE, "no material: call pd_material_lps, pd_material_linear_lps or pd_material_bond_based first");
  {
    int model = -1;
    for (int m : c->block_model) {
      if (m < 0) continue;
      if (model >= 0 && m != model)
        return fail(c, PD_ERR_UNSUPPORTED, "all blocks of a context must use one material model");
      model = m;
    }
    if (model >= 0 && model != c->material_model) {
      c->material_model = model;
      c->wv_done = false;
    }
  }
  if (c->material_model == PD_MATERIAL_LINEAR_LPS && c->precision != PD_FP64 && c->tpo_split != 4)
    return fail(c, PD_ERR_UNSUPPORTED, "the split-FP32 Linear LPS passes run at 4 lanes per point (the sliced bond "
                                       "stream); use threads_per_point 0 or 4, or PD_FP64");
  if (c->precision == PD_FP64_SLICED &&
      (c->material_model != PD_MATERIAL_LPS || c->influence != PD_INFLUENCE_ONE))
    return fail(c, PD_ERR_UNSUPPORTED, "PD_FP64_SLICED runs the LPS elastic material with the \"One\" influence "
                                       "function; use PD_FP64 for other materials and influence functions");
  if (c->precision == PD_SPLIT_FP32 && c->influence != PD_INFLUENCE_ONE &&
      c->material_model != PD_MATERIAL_BOND_BASED) {
    // The split passes weight both halves of a bond, t_ij and t_ji, with the
    // owner's omega(|X|, h_i); that equals the neighbor's omega(|X|, h_j) only
    // when every point has the same horizon.
    const double* h = c->block_h.data();
    for (size_t b = 1; b < c->block_h.size(); ++b)
      if (h[b] != h[0])
        return fail(c, PD_ERR_UNSUPPORTED,
                    "the split-FP32 passes support the Parabolic Decay and Gaussian influence functions only when all "
                    "blocks have one horizon; use PD_FP64 or the \"One\" influence function");
  }
  if (!c->symmetric)  // (the bond set-up adds the missing reverse halves)
    return fail(c, PD_ERR_STATE, "bond families are not symmetric after the bond set-up");
  TRY(alloc_state(c));
  if (!c->wv_done) {
    TRY(upload_material(c));
    PD_CUDA_TRY(c, launch_weighted_volume(c));
    PD_CUDA_TRY(c, launch_pack_owner(c));
    PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->wv_done = true;
  }
  if (c->bc_dirty) {
    const int64_t n = c->n;
    c->has_bc = false;
    for (uint8_t m : c->h_bc_mask) c->has_bc |= (m != 0);
    if (c->has_bc) {
      PD_CUDA_TRY(c, c->bc_mask.alloc(n));
      PD_CUDA_TRY(c, c->bc_a.alloc(3 * n));
      PD_CUDA_TRY(c, c->bc_b.alloc(3 * n));
      PD_CUDA_TRY(c, h2d(c, c->bc_mask.p, c->h_bc_mask.data(), n));
      PD_CUDA_TRY(c, h2d(c, c->bc_a.p, c->h_bc_a.data(), 3 * n * sizeof(double)));
      PD_CUDA_TRY(c, h2d(c, c->bc_b.p, c->h_bc_b.data(), 3 * n * sizeof(double)));
    }
    // prescribed functions: the dofs that use one and the programs
    std::vector<int32_t> dofs, starts;
    for (int64_t k = 0; k < 3 * n; ++k)
      if (c->h_bc_prog[k] >= 0 && ((c->h_bc_mask[k / 3] >> (k % 3 + 3)) & 1)) {
        dofs.push_back((int32_t)k);
        starts.push_back((int32_t)c->h_bc_prog[k]);
      }
    c->n_bc_expr = (int64_t)dofs.size();
    if (c->n_bc_expr) {
      PD_CUDA_TRY(c, c->bc_dofs.alloc(dofs.size()));
      PD_CUDA_TRY(c, c->bc_start.alloc(starts.size()));
      PD_CUDA_TRY(c, c->bc_code.alloc(c->h_bc_code.size()));
      PD_CUDA_TRY(c, c->bc_konst.alloc(std::max<size_t>(c->h_bc_konst.size(), 1)));
      PD_CUDA_TRY(c, c->bc_cp.alloc(3 * n));
      PD_CUDA_TRY(c, dzero(c, c->bc_cp.p, c->bc_cp.bytes()));
      PD_CUDA_TRY(c, h2d(c, c->bc_dofs.p, dofs.data(), dofs.size() * sizeof(int32_t)));
      PD_CUDA_TRY(c, h2d(c, c->bc_start.p, starts.data(), starts.size() * sizeof(int32_t)));
      PD_CUDA_TRY(c, h2d(c, c->bc_code.p, c->h_bc_code.data(), c->h_bc_code.size() * sizeof(int32_t)));
      if (!c->h_bc_konst.empty())
        PD_CUDA_TRY(c, h2d(c, c->bc_konst.p, c->h_bc_konst.data(), c->h_bc_konst.size() * sizeof(double)));
    }
    c->bc_dirty = false;
  }
  return PD_OK;
}

int check_status(pd_ctx* c) {
  int st = 0;
  PD_CUDA_TRY(c, cudaMemcpyAsync(&st, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (st) PD_CUDA_TRY(c, cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  // a non-finite prescribed value first: it makes the next forces non-finite too
  if (st & ST_NONFINITE_BC) return fail(c, PD_ERR_NONFINITE, "NaN returned by dirichlet increment BC evaluation");
  if (st & ST_NONFINITE_FORCE) return fail(c, PD_ERR_NONFINITE, "NaN returned by force evaluation");
  if (st & ST_NONFINITE_CONTACT) return fail(c, PD_ERR_NONFINITE, "NaN returned by contact force evaluation");
  if (st & ST_TIMEOUT) return fail(c, PD_ERR_TIMEOUT, "a bounded device wait ran out");
  if (st & ST_BAD_INDEX) return fail(c, PD_ERR_ARG, "a point index was outside the context (ignored)");
  return PD_OK;
}

// evalModel on the configuration already in st[cur]; trial damage on dmg_trial.
// f_host (may be null): where the force density also goes on the host; *host_done
// tells whether the evaluation copied it there.
int eval_trial(pd_ctx* c, double* f_dev, double* f_host = nullptr, bool* host_done = nullptr,
               const double* y_host = nullptr) {
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->dmg_trial.p, c->dmg.p, (size_t)c->nb, cudaMemcpyDeviceToDevice, c->stream));
  note_damage_copy(c, c->dmg_trial.p, c->dmg.p);
  StepParams sp{};
  sp.mode = EVAL_ONLY;
  sp.damage_on = c->any_damage ? 1 : 0;
  sp.f_out = f_dev;
  sp.f_host = f_host;
  sp.y_host = y_host;
  PD_CUDA_TRY(c, launch_eval(c, sp, c->dmg_trial.p, host_done));
  c->trial_valid = true;
  return check_status(c);
}

}  // namespace

namespace pdb {
int ensure_ready_internal(pd_ctx* c) { return ensure_ready(c); }
}  // namespace pdb

extern "C" {

const char* pd_version(void) { return kVersion; }

const char* pd_last_error(const pd_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int pd_create(const pd_config* cfg, pd_ctx** out) {
  if (!out) return PD_ERR_ARG;
  *out = nullptr;
  pd_ctx* c = new pd_ctx();
  if (cfg) {
    c->device = cfg->device;
    c->precision = cfg->precision;
    c->influence = cfg->influence;
    if (cfg->threads_per_point) c->tpo = c->tpo_split = cfg->threads_per_point;
  }
  if (c->precision != PD_FP64 && c->precision != PD_SPLIT_FP32 && c->precision != PD_FP64_SLICED) {
    delete c;
    return PD_ERR_ARG;
  }
  if (c->influence < 0 || c->influence > 2 || !(c->tpo == 4 || c->tpo == 8 || c->tpo == 16 || c->tpo == 32)) {
    delete c;
    return PD_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || c->device < 0 || c->device >= ndev) {
    delete c;
    return PD_ERR_CUDA;
  }
  if (cudaSetDevice(c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      c->status.alloc(1) != cudaSuccess || dzero(c, c->status.p, sizeof(int)) != cudaSuccess) {
    delete c;
    return PD_ERR_CUDA;
  }
  c->block_h.assign(1, 0.0);
  c->block_K.assign(1, 0.0);
  c->block_mu.assign(1, 0.0);
  c->block_rho.assign(1, 0.0);
  c->block_sc.assign(1, -1.0);
  c->block_model.assign(1, -1);
  *out = c;
  return PD_OK;
}

int pd_destroy(pd_ctx* c) {
  if (!c) return PD_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  contact_release(c);
  qs_release(c);
  mpnn_release(c);
  coarse_release(c);
  for (cudaEvent_t e : c->kev) cudaEventDestroy(e);
  if (c->vbeg) cudaEventDestroy(c->vbeg);
  for (cudaEvent_t e : c->up_ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : c->chunk_ev)
    if (e) cudaEventDestroy(e);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  cudaStream_t s = c->stream;
  delete c;
  if (s) cudaStreamDestroy(s);
  return PD_OK;
}

int pd_set_points(pd_ctx* c, int64_t n, const double* x, const double* vol, const int32_t* block) {
  CHECK_CTX(c);
  if (n <= 0 || n >= (int64_t(1) << 31) || !x || !vol) return fail(c, PD_ERR_ARG, "pd_set_points: bad arguments");
  TRY(ensure_device(c));
  coarse_release(c);
  c->blk_dev.release();
  c->n = n;
  c->hx.assign(x, x + 3 * n);
  c->hvol.assign(vol, vol + n);
  int32_t nblk = 1;
  if (block) {
    c->hblock.assign(block, block + n);
    for (int64_t i = 0; i < n; ++i) {
      if (block[i] < 0) return fail(c, PD_ERR_ARG, "pd_set_points: negative block id");
      nblk = std::max(nblk, block[i] + 1);
    }
  } else {
    c->hblock.clear();
  }
  c->n_blocks = nblk;
  c->block_h.resize(nblk, c->block_h.empty() ? 0.0 : c->block_h[0]);
  c->block_K.resize(nblk, 0.0);
  c->block_mu.resize(nblk, 0.0);
  c->block_rho.resize(nblk, 0.0);
  c->block_sc.resize(nblk, -1.0);
  c->block_model.resize(nblk, -1);
  std::vector<double4> xv(n);
  for (int64_t i = 0; i < n; ++i) xv[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], vol[i]);
  PD_CUDA_TRY(c, c->xv.alloc(n));
  PD_CUDA_TRY(c, h2d(c, c->xv.p, xv.data(), n * sizeof(double4)));
  c->row.release();
  c->col.release();
  c->nb = 0;
  c->wv_done = false;
  coarse_release(c);
  c->h_bc_mask.assign(n, 0);
  c->h_bc_a.assign(3 * n, 0.0);
  c->h_bc_b.assign(3 * n, 0.0);
  c->h_bc_prog.assign(3 * n, -1);
  c->h_bc_code.clear();
  c->h_bc_konst.clear();
  c->bc_dirty = true;
  coarse_invalidate(c);
  c->field_K.clear();
  c->field_mu.clear();
  c->field_sc.clear();
  for (int k = 0; k < 2; ++k) {
    c->st[k].release();
    c->ur[k].release();
  }
  c->u.release();
  c->state_init = false;
  return PD_OK;
}

int pd_set_block_horizons(pd_ctx* c, int32_t n_blocks, const double* horizon) {
  CHECK_CTX(c);
  if (n_blocks <= 0 || !horizon) return fail(c, PD_ERR_ARG, "pd_set_block_horizons: bad arguments");
  if (n_blocks > (int32_t)c->block_h.size()) {
    c->block_h.resize(n_blocks, 0.0);
    c->block_K.resize(n_blocks, 0.0);
    c->block_mu.resize(n_blocks, 0.0);
    c->block_rho.resize(n_blocks, 0.0);
    c->block_sc.resize(n_blocks, -1.0);
  }
  for (int b = 0; b < n_blocks; ++b) {
    if (!(horizon[b] > 0.0)) return fail(c, PD_ERR_ARG, "horizon must be positive");
    c->block_h[b] = horizon[b];
  }
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_build_bonds(pd_ctx* c, const pd_plane_filter* filters, int32_t n_filters) {
  CHECK_CTX(c);
  if (c->n == 0) return fail(c, PD_ERR_STATE, "pd_build_bonds: points not set");
  if (n_filters > 0 && !filters) return fail(c, PD_ERR_ARG, "pd_build_bonds: null filters");
  for (int32_t b = 0; b < c->n_blocks; ++b)
    if (!(c->block_h[b] > 0.0)) return fail(c, PD_ERR_STATE, "pd_build_bonds: horizon of every block must be set");
  TRY(ensure_device(c));
  TRY(upload_horizons(c));
  TRY(build_bonds_device(c, filters, n_filters));
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_set_bonds(pd_ctx* c, const int32_t* nl, int64_t len) {
  CHECK_CTX(c);
  if (c->n == 0) return fail(c, PD_ERR_STATE, "pd_set_bonds: points not set");
  if (!nl || len < c->n) return fail(c, PD_ERR_ARG, "pd_set_bonds: neighbor list too short");
  TRY(ensure_device(c));
  std::vector<int64_t> row(c->n + 1);
  std::vector<int32_t> col;
  col.reserve(len - c->n);
  int64_t k = 0;
  for (int64_t i = 0; i < c->n; ++i) {
    if (k >= len) return fail(c, PD_ERR_ARG, "pd_set_bonds: neighbor list ends early");
    const int32_t cnt = nl[k++];
    if (cnt < 0 || k + cnt > len) return fail(c, PD_ERR_ARG, "pd_set_bonds: bad neighbor count");
    row[i] = (int64_t)col.size();
    for (int32_t q = 0; q < cnt; ++q) {
      const int32_t j = nl[k++];
      if (j < 0 || j >= c->n || j == i) return fail(c, PD_ERR_ARG, "pd_set_bonds: neighbor id out of range or self");
      col.push_back(j);
    }
  }
  if (k != len) return fail(c, PD_ERR_ARG, "pd_set_bonds: trailing entries in neighbor list");
  row[c->n] = (int64_t)col.size();
  c->nb = (int64_t)col.size();
  PD_CUDA_TRY(c, c->row.alloc(c->n + 1));
  PD_CUDA_TRY(c, c->col.alloc(std::max<int64_t>(c->nb, 1)));
  PD_CUDA_TRY(c, h2d(c, c->row.p, row.data(), (c->n + 1) * sizeof(int64_t)));
  if (c->nb) PD_CUDA_TRY(c, h2d(c, c->col.p, col.data(), c->nb * sizeof(int32_t)));
  if (c->hp.count < (size_t)c->n) TRY(upload_horizons(c));
  TRY(finalize_bonds(c, false));
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_num_bonds(const pd_ctx* c, int64_t* nb) {
  if (!c || !nb) return PD_ERR_ARG;
  *nb = c->nb_user;  // the families' bonds (the device rows may also hold phantom halves)
  return PD_OK;
}

int pd_get_bonds(pd_ctx* c, int32_t* nl, int64_t cap, int64_t* len) {
  CHECK_CTX(c);
  if (!len) return fail(c, PD_ERR_ARG, "pd_get_bonds: null len");
  *len = c->n + c->nb_user;
  if (cap == 0) return PD_OK;
  if (!nl || cap < *len) return fail(c, PD_ERR_ARG, "pd_get_bonds: buffer too small");
  TRY(ensure_device(c));
  std::vector<int64_t> row(c->n + 1);
  std::vector<int32_t> col(std::max<int64_t>(c->nb, 1));
  PD_CUDA_TRY(c, d2h(c, row.data(), c->row.p, (c->n + 1) * sizeof(int64_t)));
  if (c->nb) PD_CUDA_TRY(c, d2h(c, col.data(), c->col.p, c->nb * sizeof(int32_t)));
  int64_t k = 0;
  for (int64_t i = 0; i < c->n; ++i) {  // the families as given or built (no phantom halves)
    const int64_t head = k++;
    for (int64_t b = row[i]; b < row[i + 1]; ++b)
      if (!c->phantoms || c->h_orig[b]) nl[k++] = col[b];
    nl[head] = (int32_t)(k - head - 1);
  }
  return PD_OK;
}

int pd_material_lps(pd_ctx* c, int32_t block, double K, double mu, double rho) {
  CHECK_CTX(c);
  if (block < 0 || block >= (int32_t)c->block_K.size()) return fail(c, PD_ERR_ARG, "pd_material_lps: bad block");
  if (!(K > 0.0) || !(mu > 0.0) || !(rho > 0.0)) return fail(c, PD_ERR_ARG, "pd_material_lps: moduli and density must be positive");
  c->block_K[block] = K;
  c->block_mu[block] = mu;
  c->block_rho[block] = rho;
  c->block_model[block] = PD_MATERIAL_LPS;
  c->have_material = true;
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_material_bond_based(pd_ctx* c, int32_t block, double K, double rho, int32_t plane, double height) {
  CHECK_CTX(c);
  if (block < 0 || block >= (int32_t)c->block_K.size()) return fail(c, PD_ERR_ARG, "pd_material_bond_based: bad block");
  if (!(K > 0.0) || !(rho > 0.0)) return fail(c, PD_ERR_ARG, "pd_material_bond_based: modulus and density must be positive");
  if (plane != 0 && !(height > 0.0))
    return fail(c, PD_ERR_ARG, "pd_material_bond_based: in case of plane strain or plane stress the height must be given");
  c->block_K[block] = K;
  c->block_mu[block] = 0.0;
  c->block_rho[block] = rho;
  c->block_model[block] = PD_MATERIAL_BOND_BASED;
  c->bb_plane = plane != 0;
  c->bb_height = plane != 0 ? height : 0.0;
  c->have_material = true;
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_material_linear_lps(pd_ctx* c, int32_t block, double K, double mu, double rho) {
  CHECK_CTX(c);
  if (block < 0 || block >= (int32_t)c->block_K.size()) return fail(c, PD_ERR_ARG, "pd_material_linear_lps: bad block");
  if (!(K > 0.0) || !(mu > 0.0) || !(rho > 0.0))
    return fail(c, PD_ERR_ARG, "pd_material_linear_lps: moduli and density must be positive");
  c->block_K[block] = K;
  c->block_mu[block] = mu;
  c->block_rho[block] = rho;
  c->block_model[block] = PD_MATERIAL_LINEAR_LPS;
  c->have_material = true;
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_material_lps_field(pd_ctx* c, const double* K, const double* mu) {
  CHECK_CTX(c);
  if (c->n == 0 || !K || !mu) return fail(c, PD_ERR_ARG, "pd_material_lps_field: bad arguments");
  for (int64_t i = 0; i < c->n; ++i)
    if (!(K[i] > 0.0) || !(mu[i] > 0.0)) return fail(c, PD_ERR_ARG, "pd_material_lps_field: moduli must be positive");
  c->field_K.assign(K, K + c->n);
  c->field_mu.assign(mu, mu + c->n);
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_damage_critical_stretch(pd_ctx* c, int32_t block, double s_c) {
  CHECK_CTX(c);
  if (block < 0 || block >= (int32_t)c->block_sc.size()) return fail(c, PD_ERR_ARG, "pd_damage_critical_stretch: bad block");
  c->block_sc[block] = s_c;
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_damage_critical_stretch_field(pd_ctx* c, const double* s_c) {
  CHECK_CTX(c);
  if (c->n == 0 || !s_c) return fail(c, PD_ERR_ARG, "pd_damage_critical_stretch_field: bad arguments");
  c->field_sc.assign(s_c, s_c + c->n);
  c->wv_done = false;
  coarse_release(c);
  return PD_OK;
}

int pd_weighted_volume(pd_ctx* c, double* m_out) {
  CHECK_CTX(c);
  TRY(ensure_ready(c));
  if (m_out) {
    std::vector<double4> pt(c->n);
    PD_CUDA_TRY(c, d2h(c, pt.data(), c->pt.p, c->n * sizeof(double4)));
    for (int64_t i = 0; i < c->n; ++i) m_out[i] = pt[i].x;
  }
  return PD_OK;
}

int pd_compute_force_device(pd_ctx* c, const double* y_dev, double* f_dev) {
  CHECK_CTX(c);
  if (!y_dev) return fail(c, PD_ERR_ARG, "pd_compute_force_device: null coordinates");
  TRY(ensure_ready(c));
  PD_CUDA_TRY(c, launch_state_from_y(c, y_dev));
  return eval_trial(c, f_dev);
}

int pd_compute_force(pd_ctx* c, const double* y, double* f_out) {
  CHECK_CTX(c);
  if (!y) return fail(c, PD_ERR_ARG, "pd_compute_force: null coordinates");
  TRY(ensure_ready(c));
  const size_t bytes = 3 * (size_t)c->n * sizeof(double);
  // y is uploaded (in chunks, beside the dilatation, where the path allows)
  // through the force buffer, then f is written there
  bool copied = false;
  TRY(eval_trial(c, c->f.p, f_out, &copied, y));
  if (f_out && !copied) {
    PD_CUDA_TRY(c, cudaMemcpyAsync(f_out, c->f.p, bytes, cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  return PD_OK;
}

int pd_compute_damage(pd_ctx* c, const double* y) { return pd_compute_force(c, y, nullptr); }

int pd_update_state(pd_ctx* c) {
  CHECK_CTX(c);
  TRY(ensure_device(c));
  if (c->trial_valid) {
    // commit by exchanging the buffers: the trial's damage becomes the
    // committed one (the evaluation has completed: its call synchronised);
    // the next trial starts from a copy of it. The sliced mirror's source is
    // tracked by address, which moves with the buffer.
    std::swap(c->dmg.p, c->dmg_trial.p);
    std::swap(c->dmg.count, c->dmg_trial.count);
    c->trial_valid = false;
  }
  return PD_OK;
}

int pd_set_bond_damage(pd_ctx* c, const double* bd) {
  CHECK_CTX(c);
  if (!bd || !c->dmg.p) return fail(c, PD_ERR_STATE, "pd_set_bond_damage: bonds not set");
  std::vector<uint8_t> h((size_t)std::max<int64_t>(c->nb, 1));
  for (int64_t b = 0, u = 0; b < c->nb; ++b) {
    if (c->phantoms && !c->h_orig[b]) {  // a phantom half: its own half does not exist
      h[b] = (uint8_t)(1 | kPhantomOwn);
      continue;
    }
    const double v = bd[u++];
    if (v == 0.0) h[b] = 0;
    else if (v == 1.0) h[b] = 1;
    else return fail(c, PD_ERR_UNSUPPORTED, "bond damage must be 0 or 1 (critical-stretch values)");
  }
  TRY(ensure_device(c));
  // the rows' own halves, then each bond's partner half (bit 1) from the partner's row
  PD_CUDA_TRY(c, h2d(c, c->dmg_trial.p, h.data(), (size_t)c->nb));
  TRY(mirror_damage(c, c->dmg_trial.p, c->dmg.p));
  c->dmg_gen++;
  c->trial_valid = false;
  coarse_invalidate(c);
  return PD_OK;
}

int pd_critical_time_step(pd_ctx* c, double* dt_out) {
  CHECK_CTX(c);
  if (!dt_out) return fail(c, PD_ERR_ARG, "pd_critical_time_step: null output");
  TRY(ensure_ready(c));
  DBuf<double> d;
  PD_CUDA_TRY(c, d.alloc(1));
  PD_CUDA_TRY(c, launch_critical_dt(c, d.p));
  PD_CUDA_TRY(c, cudaMemcpyAsync(dt_out, d.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return PD_OK;
}

int pd_set_state(pd_ctx* c, const double* u, const double* v) {
  CHECK_CTX(c);
  TRY(ensure_ready(c));
  const size_t bytes = 3 * (size_t)c->n * sizeof(double);
  if (u) PD_CUDA_TRY(c, h2d(c, c->u.p, u, bytes));
  else if (!c->state_init) PD_CUDA_TRY(c, dzero(c, c->u.p, bytes));
  if (v) PD_CUDA_TRY(c, h2d(c, c->v.p, v, bytes));
  else if (!c->state_init) PD_CUDA_TRY(c, dzero(c, c->v.p, bytes));
  if (u || !c->state_init) {
    c->cur = 0;
    PD_CUDA_TRY(c, launch_sync_state(c));
    PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  c->state_init = true;
  return PD_OK;
}

int pd_add_prescribed_displacement(pd_ctx* c, int64_t np, const int64_t* pts, int32_t coord, double a, double b) {
  CHECK_CTX(c);
  if (c->n == 0) return fail(c, PD_ERR_STATE, "points not set");
  if (coord < 0 || coord > 2 || np < 0 || (np > 0 && !pts)) return fail(c, PD_ERR_ARG, "bad boundary condition");
  for (int64_t k = 0; k < np; ++k) {
    const int64_t i = pts[k];
    if (i < 0 || i >= c->n) return fail(c, PD_ERR_ARG, "boundary-condition point out of range");
    c->h_bc_mask[i] |= (uint8_t)(1u << coord);
    c->h_bc_mask[i] &= (uint8_t)~(1u << (coord + 3));
    c->h_bc_a[3 * i + coord] = a;
    c->h_bc_b[3 * i + coord] = b;
    c->h_bc_prog[3 * i + coord] = -1;
  }
  c->bc_dirty = true;
  coarse_invalidate(c);
  return PD_OK;
}

int pd_add_prescribed_displacement_function(pd_ctx* c, int64_t np, const int64_t* pts, int32_t coord,
                                            const char* function) {
  CHECK_CTX(c);
  if (c->n == 0) return fail(c, PD_ERR_STATE, "points not set");
  if (coord < 0 || coord > 2 || np < 0 || (np > 0 && !pts) || !function)
    return fail(c, PD_ERR_ARG, "bad boundary condition");
  for (int64_t k = 0; k < np; ++k)
    if (pts[k] < 0 || pts[k] >= c->n) return fail(c, PD_ERR_ARG, "boundary-condition point out of range");
  int64_t start = 0;
  std::string err;
  if (!expr_compile(function, c->h_bc_code, c->h_bc_konst, &start, &err)) return fail(c, PD_ERR_ARG, err);
  for (int64_t k = 0; k < np; ++k) {
    const int64_t i = pts[k];
    c->h_bc_mask[i] |= (uint8_t)((1u << coord) | (1u << (coord + 3)));
    c->h_bc_prog[3 * i + coord] = start;
  }
  c->bc_dirty = true;
  coarse_invalidate(c);
  return PD_OK;
}

int pd_clear_boundary_conditions(pd_ctx* c) {
  CHECK_CTX(c);
  std::fill(c->h_bc_mask.begin(), c->h_bc_mask.end(), 0);
  std::fill(c->h_bc_prog.begin(), c->h_bc_prog.end(), -1);
  c->h_bc_code.clear();
  c->h_bc_konst.clear();
  c->bc_dirty = true;
  coarse_invalidate(c);
  return PD_OK;
}

int pd_verlet_run(pd_ctx* c, double dt, double t0, int64_t nsteps, pd_stats* stats) {
  CHECK_CTX(c);
  if (!(dt > 0.0) || nsteps < 0) return fail(c, PD_ERR_ARG, "pd_verlet_run: dt must be positive and nsteps >= 0");
  TRY(ensure_ready(c));
  if (!c->state_init) TRY(pd_set_state(c, nullptr, nullptr));
  const bool contact = c->contact != nullptr;
  cudaEvent_t e0, e1;
  PD_CUDA_TRY(c, cudaEventCreate(&e0));
  PD_CUDA_TRY(c, cudaEventCreate(&e1));
  StepParams sp{};
  sp.dt = dt;
  sp.t0 = t0;
  sp.damage_on = c->any_damage ? 1 : 0;
  sp.has_bc = c->has_bc ? 1 : 0;
  sp.has_contact = contact ? 1 : 0;
  // initial evaluation (Peridigm.cpp:1393-1423): its damage is not committed
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->dmg_trial.p, c->dmg.p, (size_t)c->nb, cudaMemcpyDeviceToDevice, c->stream));
  note_damage_copy(c, c->dmg_trial.p, c->dmg.p);
  if (contact) {
    TRY(contact_prepare(c, 0));
    TRY(contact_eval(c));
  }
  sp.step = 0;
  sp.mode = nsteps == 0 ? EVAL_LAST : EVAL_ADVANCE;
  sp.f_out = nsteps == 0 ? c->f.p : nullptr;
  PD_CUDA_TRY(c, cudaEventRecord(e0, c->stream));
  PD_CUDA_TRY(c, launch_eval(c, sp, c->dmg_trial.p));
  if (nsteps > 0) c->cur ^= 1;
  for (int64_t s = 1; s <= nsteps; ++s) {
    sp.step = s;
    const bool last = s == nsteps;
    sp.mode = last ? EVAL_LAST : EVAL_ADVANCE;
    sp.f_out = last ? c->f.p : nullptr;
    if (contact) {
      TRY(contact_prepare(c, s));
      TRY(contact_eval(c));
    }
    PD_CUDA_TRY(c, launch_eval(c, sp, c->dmg.p));
    if (!last) c->cur ^= 1;
  }
  PD_CUDA_TRY(c, cudaEventRecord(e1, c->stream));
  PD_CUDA_TRY(c, cudaEventSynchronize(e1));
  if (c->ktime) PD_CUDA_TRY(c, collect_kernel_times(c));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->trial_valid = false;
  int rc = check_status(c);
  if (stats) {
    stats->steps = nsteps;
    stats->bonds = c->nb_user;
    stats->device_ms = ms;
    TRY(count_broken(c, &stats->broken_bonds));
    stats->contact_pairs = contact_pairs(c);
  }
  return rc;
}

// ---- stepping form: begin + step(n - 1) + finish == pd_verlet_run(n) ------
static StepParams verlet_params(const pd_ctx* c, double dt, double t0) {
  StepParams sp{};
  sp.dt = dt;
  sp.t0 = t0;
  sp.damage_on = c->any_damage ? 1 : 0;
  sp.has_bc = c->has_bc ? 1 : 0;
  sp.has_contact = c->contact != nullptr ? 1 : 0;
  return sp;
}

int pd_verlet_begin(pd_ctx* c, double dt, double t0) {
  CHECK_CTX(c);
  if (!(dt > 0.0)) return fail(c, PD_ERR_ARG, "pd_verlet_begin: dt must be positive");
  TRY(ensure_ready(c));
  if (!c->state_init) TRY(pd_set_state(c, nullptr, nullptr));
  StepParams sp = verlet_params(c, dt, t0);
  if (!c->vbeg) PD_CUDA_TRY(c, cudaEventCreate(&c->vbeg));
  PD_CUDA_TRY(c, cudaEventRecord(c->vbeg, c->stream));
  // initial evaluation (Peridigm.cpp:1393-1423): its damage is not committed
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->dmg_trial.p, c->dmg.p, (size_t)c->nb, cudaMemcpyDeviceToDevice, c->stream));
  note_damage_copy(c, c->dmg_trial.p, c->dmg.p);
  if (sp.has_contact) {
    TRY(contact_prepare(c, 0));
    TRY(contact_eval(c));
  }
  sp.step = 0;
  sp.mode = EVAL_ADVANCE;
  PD_CUDA_TRY(c, launch_eval(c, sp, c->dmg_trial.p));
  c->cur ^= 1;
  c->vrun = true;
  c->vdt = dt;
  c->vt0 = t0;
  c->vstep = 0;
  c->trial_valid = false;
  return check_status(c);
}

int pd_verlet_step(pd_ctx* c, int64_t nsteps) {
  CHECK_CTX(c);
  if (!c->vrun) return fail(c, PD_ERR_STATE, "pd_verlet_step: call pd_verlet_begin first");
  if (nsteps < 0) return fail(c, PD_ERR_ARG, "pd_verlet_step: nsteps must be >= 0");
  StepParams sp = verlet_params(c, c->vdt, c->vt0);
  for (int64_t k = 0; k < nsteps; ++k) {
    sp.step = ++c->vstep;
    sp.mode = EVAL_ADVANCE;
    if (sp.has_contact) {
      TRY(contact_prepare(c, sp.step));
      TRY(contact_eval(c));
    }
    PD_CUDA_TRY(c, launch_eval(c, sp, c->dmg.p));
    c->cur ^= 1;
  }
  return check_status(c);
}

int pd_verlet_finish(pd_ctx* c, pd_stats* stats) {
  CHECK_CTX(c);
  if (!c->vrun) return fail(c, PD_ERR_STATE, "pd_verlet_finish: call pd_verlet_begin first");
  StepParams sp = verlet_params(c, c->vdt, c->vt0);
  sp.step = ++c->vstep;
  sp.mode = EVAL_LAST;
  sp.f_out = c->f.p;
  if (sp.has_contact) {
    TRY(contact_prepare(c, sp.step));
    TRY(contact_eval(c));
  }
  PD_CUDA_TRY(c, launch_eval(c, sp, c->dmg.p));
  cudaEvent_t e1;
  PD_CUDA_TRY(c, cudaEventCreate(&e1));
  PD_CUDA_TRY(c, cudaEventRecord(e1, c->stream));
  PD_CUDA_TRY(c, cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->vbeg, e1);
  cudaEventDestroy(e1);
  c->vrun = false;
  const int rc = check_status(c);
  if (stats) {
    stats->steps = c->vstep;
    stats->bonds = c->nb_user;
    stats->device_ms = ms;
    TRY(count_broken(c, &stats->broken_bonds));
    stats->contact_pairs = contact_pairs(c);
  }
  return rc;
}

int pd_pack_state_device(pd_ctx* c, int64_t n_idx, const int32_t* idx_dev, double* out_dev) {
  CHECK_CTX(c);
  if (n_idx < 0 || (n_idx > 0 && (!idx_dev || !out_dev))) return fail(c, PD_ERR_ARG, "pd_pack_state_device: bad arguments");
  if (!c->vrun) return fail(c, PD_ERR_STATE, "pd_pack_state_device: only between pd_verlet_begin and pd_verlet_finish");
  PD_CUDA_TRY(c, launch_pack_state(c, n_idx, idx_dev, out_dev));
  return check_status(c);
}

int pd_unpack_state_device(pd_ctx* c, int64_t n_idx, const int32_t* idx_dev, const double* in_dev) {
  CHECK_CTX(c);
  if (n_idx < 0 || (n_idx > 0 && (!idx_dev || !in_dev))) return fail(c, PD_ERR_ARG, "pd_unpack_state_device: bad arguments");
  if (!c->vrun) return fail(c, PD_ERR_STATE, "pd_unpack_state_device: only between pd_verlet_begin and pd_verlet_finish");
  PD_CUDA_TRY(c, launch_unpack_state(c, n_idx, idx_dev, in_dev));
  return check_status(c);
}

int pd_qs_load_step(pd_ctx* c, double t_prev, double t_cur, const pd_qs_options* o, pd_stats* st) {
  CHECK_CTX(c);
  if (!o) return fail(c, PD_ERR_ARG, "pd_qs_load_step: null options");
  if (!(t_cur > t_prev) || o->preconditioner < 0 || o->preconditioner > 3 || o->max_cg_iterations <= 0 ||
      o->max_newton_iterations < 0 || !(o->cg_relative_tolerance > 0.0))
    return fail(c, PD_ERR_ARG, "pd_qs_load_step: bad options");
  if (!c->state_init) TRY(pd_set_state(c, nullptr, nullptr));
  return qs_load_step(c, t_prev, t_cur, o, st);
}

int pd_implicit_run(pd_ctx* c, double dt, double t0, int64_t nsteps, const pd_implicit_options* o, pd_stats* st) {
  CHECK_CTX(c);
  if (!o) return fail(c, PD_ERR_ARG, "pd_implicit_run: null options");
  if (!(dt > 0.0) || nsteps < 0 || !(o->beta > 0.0) || !(o->gamma >= 0.0) || !(o->absolute_tolerance >= 0.0) ||
      !(o->cg_relative_tolerance > 0.0) || o->max_newton_iterations < 0 || o->max_cg_iterations <= 0 ||
      (o->preconditioner != PD_PRECOND_NONE && o->preconditioner != PD_PRECOND_BLOCK_JACOBI))
    return fail(c, PD_ERR_ARG, "pd_implicit_run: bad options");
  if (!c->state_init) TRY(pd_set_state(c, nullptr, nullptr));
  return implicit_run(c, dt, t0, nsteps, o, st);
}

int pd_mpnn_init(pd_ctx* c, uint64_t seed, double patch) {
  CHECK_CTX(c);
  if (!(patch > 0.0) || !std::isfinite(patch)) return fail(c, PD_ERR_ARG, "pd_mpnn_init: patch side must be positive");
  TRY(ensure_ready(c));
  return mpnn_init(c, seed, patch);
}

int pd_mpnn_collect(pd_ctx* c, int32_t every) {
  CHECK_CTX(c);
  if (every < 0) return fail(c, PD_ERR_ARG, "pd_mpnn_collect: every must be >= 0");
  return mpnn_set_capture(c, every);
}

int pd_mpnn_num_pairs(pd_ctx* c, int64_t* count) {
  CHECK_CTX(c);
  if (!count) return fail(c, PD_ERR_ARG, "null count");
  *count = mpnn_num_pairs(c);
  return PD_OK;
}

int pd_mpnn_train(pd_ctx* c, int32_t epochs, double learning_rate, int32_t batch, double* loss) {
  CHECK_CTX(c);
  if (epochs < 0 || !(learning_rate > 0.0) || batch <= 0) return fail(c, PD_ERR_ARG, "pd_mpnn_train: bad arguments");
  TRY(ensure_device(c));
  return mpnn_train(c, epochs, learning_rate, batch, loss);
}

int pd_mpnn_num_params(int64_t* count) {
  if (!count) return PD_ERR_ARG;
  *count = mpnn_num_params();
  return PD_OK;
}

int pd_mpnn_get_weights(pd_ctx* c, float* w) {
  CHECK_CTX(c);
  if (!w) return fail(c, PD_ERR_ARG, "null weights");
  TRY(ensure_device(c));
  return mpnn_get_weights(c, w);
}

int pd_mpnn_set_weights(pd_ctx* c, const float* w) {
  CHECK_CTX(c);
  if (!w) return fail(c, PD_ERR_ARG, "null weights");
  TRY(ensure_device(c));
  return mpnn_set_weights(c, w);
}

int pd_mpnn_coarse(pd_ctx* c, double cell) {
  CHECK_CTX(c);
  if (!std::isfinite(cell)) return fail(c, PD_ERR_ARG, "pd_mpnn_coarse: cell must be finite");
  return mpnn_set_coarse(c, cell);
}

int pd_qs_coarse_modes(pd_ctx* c, int32_t modes) {
  CHECK_CTX(c);
  if (modes != 3 && modes != 6) return fail(c, PD_ERR_ARG, "pd_qs_coarse_modes: modes must be 3 or 6");
  if (modes != c->coarse_modes) {
    c->coarse_modes = modes;
    coarse_release(c);
  }
  return PD_OK;
}

int pd_qs_coarse_operator(pd_ctx* c, const double* u, double cell, int64_t* n_coarse, int32_t* aggregate, double* A,
                          double* A_inv) {
  CHECK_CTX(c);
  if (!u || !n_coarse || !std::isfinite(cell)) return fail(c, PD_ERR_ARG, "pd_qs_coarse_operator: bad arguments");
  TRY(ensure_ready(c));
  DBuf<double> ud;
  PD_CUDA_TRY(c, ud.alloc(3 * c->n));
  PD_CUDA_TRY(c, cudaMemcpyAsync(ud.p, u, 3 * c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int64_t nc = 0;
  TRY(qs_coarse_operator(c, ud.p, cell, &nc, nullptr, nullptr, nullptr));
  const bool want = aggregate || A || A_inv;
  if (want && *n_coarse < nc) {
    *n_coarse = nc;
    return fail(c, PD_ERR_ARG, "pd_qs_coarse_operator: n_coarse on entry is smaller than the coarse space");
  }
  *n_coarse = nc;
  if (!want) return check_status(c);
  DBuf<int32_t> ag;
  DBuf<double> ad, ai;
  PD_CUDA_TRY(c, ag.alloc(c->n));
  PD_CUDA_TRY(c, ad.alloc((size_t)nc * nc));
  PD_CUDA_TRY(c, ai.alloc((size_t)nc * nc));
  TRY(qs_coarse_operator(c, ud.p, cell, &nc, ag.p, ad.p, ai.p));
  if (aggregate) PD_CUDA_TRY(c, d2h(c, aggregate, ag.p, c->n * sizeof(int32_t)));
  if (A) PD_CUDA_TRY(c, d2h(c, A, ad.p, (size_t)nc * nc * sizeof(double)));
  if (A_inv) PD_CUDA_TRY(c, d2h(c, A_inv, ai.p, (size_t)nc * nc * sizeof(double)));
  return check_status(c);
}

int pd_mpnn_loss_grad(pd_ctx* c, const float* pair, double* loss, float* grad) {
  CHECK_CTX(c);
  if (!pair || !loss) return fail(c, PD_ERR_ARG, "null argument");
  TRY(ensure_device(c));
  return mpnn_loss_grad(c, pair, loss, grad);
}

int pd_mpnn_apply(pd_ctx* c, const double* r, double* z) {
  CHECK_CTX(c);
  if (!r || !z) return fail(c, PD_ERR_ARG, "pd_mpnn_apply: null argument");
  TRY(ensure_device(c));
  return mpnn_middle_apply(c, r, z);
}

int pd_jacobian_apply(pd_ctx* c, const double* u, const double* w, double* kw) {
  CHECK_CTX(c);
  if (!u || !w || !kw) return fail(c, PD_ERR_ARG, "pd_jacobian_apply: null argument");
  TRY(ensure_ready(c));
  const size_t b3 = 3 * (size_t)c->n * sizeof(double);
  DBuf<double> ud, wd, kd;
  PD_CUDA_TRY(c, ud.alloc(3 * c->n));
  PD_CUDA_TRY(c, wd.alloc(3 * c->n));
  PD_CUDA_TRY(c, kd.alloc(3 * c->n));
  PD_CUDA_TRY(c, cudaMemcpyAsync(ud.p, u, b3, cudaMemcpyHostToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(wd.p, w, b3, cudaMemcpyHostToDevice, c->stream));
  TRY(qs_tangent_apply(c, ud.p, wd.p, kd.p));
  PD_CUDA_TRY(c, cudaMemcpyAsync(kw, kd.p, b3, cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}

int pd_jacobian_block_diagonal(pd_ctx* c, const double* u, double* blocks) {
  CHECK_CTX(c);
  if (!u || !blocks) return fail(c, PD_ERR_ARG, "pd_jacobian_block_diagonal: null argument");
  TRY(ensure_ready(c));
  DBuf<double> ud, bd;
  PD_CUDA_TRY(c, ud.alloc(3 * c->n));
  PD_CUDA_TRY(c, bd.alloc(9 * c->n));
  PD_CUDA_TRY(c, cudaMemcpyAsync(ud.p, u, 3 * c->n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  TRY(qs_tangent_blocks(c, ud.p, bd.p));
  PD_CUDA_TRY(c, cudaMemcpyAsync(blocks, bd.p, 9 * c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
}

int pd_contact_short_range(pd_ctx* c, double r_search, int32_t freq, double r_contact, double k_spring,
                           double friction) {
  CHECK_CTX(c);
  if (c->n == 0 || !c->row.p) return fail(c, PD_ERR_STATE, "contact: points and bonds must be set first");
  TRY(ensure_device(c));
  return contact_configure(c, r_search, freq, r_contact, k_spring, friction);
}

int pd_contact_force(pd_ctx* c, const double* y, const double* v, double* fc_out) {
  CHECK_CTX(c);
  if (!y || !v || !fc_out) return fail(c, PD_ERR_ARG, "pd_contact_force: null argument");
  if (!c->contact) return fail(c, PD_ERR_STATE, "pd_contact_force: contact not configured");
  TRY(ensure_ready(c));
  const size_t bytes = 3 * (size_t)c->n * sizeof(double);
  DBuf<double> yd, vd, fd;
  PD_CUDA_TRY(c, yd.alloc(3 * c->n));
  PD_CUDA_TRY(c, vd.alloc(3 * c->n));
  PD_CUDA_TRY(c, fd.alloc(3 * c->n));
  PD_CUDA_TRY(c, cudaMemcpyAsync(yd.p, y, bytes, cudaMemcpyHostToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(vd.p, v, bytes, cudaMemcpyHostToDevice, c->stream));
  TRY(contact_force_from(c, yd.p, vd.p, fd.p));
  PD_CUDA_TRY(c, cudaMemcpyAsync(fc_out, fd.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  TRY(check_status(c));
  return PD_OK;
}

int pd_set_kernel_timing(pd_ctx* c, int enable) {
  CHECK_CTX(c);
  TRY(ensure_device(c));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (c->ktime) PD_CUDA_TRY(c, collect_kernel_times(c));
  c->ktime = enable != 0;
  c->kms[0] = c->kms[1] = 0.0;
  c->klaunches = 0;
  return PD_OK;
}

int pd_get_kernel_timing(pd_ctx* c, double* ms_out, int64_t* launches_out) {
  CHECK_CTX(c);
  TRY(ensure_device(c));
  PD_CUDA_TRY(c, collect_kernel_times(c));
  if (ms_out) {
    ms_out[0] = c->kms[0];
    ms_out[1] = c->kms[1];
  }
  if (launches_out) *launches_out = c->klaunches;
  return PD_OK;
}

int pd_get_field(pd_ctx* c, int32_t field, double* out) {
  CHECK_CTX(c);
  if (!out) return fail(c, PD_ERR_ARG, "pd_get_field: null output");
  TRY(ensure_ready(c));
  const int64_t n = c->n;
  const size_t b3 = 3 * (size_t)n * sizeof(double);
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  switch (field) {
    case PD_FIELD_DISPLACEMENT:
    case PD_FIELD_COORDINATES: {
      PD_CUDA_TRY(c, d2h(c, out, c->u.p, b3));
      if (field == PD_FIELD_COORDINATES)
        for (int64_t k = 0; k < 3 * n; ++k) out[k] = c->hx[k] + out[k];
      return PD_OK;
    }
    case PD_FIELD_VELOCITY: PD_CUDA_TRY(c, d2h(c, out, c->v.p, b3)); return PD_OK;
    case PD_FIELD_ACCELERATION: PD_CUDA_TRY(c, d2h(c, out, c->a.p, b3)); return PD_OK;
    case PD_FIELD_FORCE_DENSITY: PD_CUDA_TRY(c, d2h(c, out, c->f.p, b3)); return PD_OK;
    case PD_FIELD_CONTACT_FORCE: PD_CUDA_TRY(c, d2h(c, out, c->fc.p, b3)); return PD_OK;
    case PD_FIELD_DILATATION:
      PD_CUDA_TRY(c, d2h(c, out, c->theta.p, n * sizeof(double)));
      return PD_OK;
    case PD_FIELD_DAMAGE:
      PD_CUDA_TRY(c, d2h(c, out, c->node_damage.p, n * sizeof(double)));
      return PD_OK;
    case PD_FIELD_WEIGHTED_VOLUME: return pd_weighted_volume(c, out);
    case PD_FIELD_BOND_DAMAGE: {
      std::vector<uint8_t> h((size_t)std::max<int64_t>(c->nb, 1));
      const uint8_t* src = c->trial_valid ? c->dmg_trial.p : c->dmg.p;
      PD_CUDA_TRY(c, d2h(c, h.data(), src, (size_t)c->nb));
      for (int64_t b = 0, u = 0; b < c->nb; ++b)  // the row's own half, the families' bonds only
        if (!c->phantoms || c->h_orig[b]) out[u++] = (double)(h[b] & 1);
      return PD_OK;
    }
    case PD_FIELD_FORCE: {
      PD_CUDA_TRY(c, d2h(c, out, c->f.p, b3));
      for (int64_t k = 0; k < 3 * n; ++k) out[k] *= c->hvol[k / 3];
      return PD_OK;
    }
    case PD_FIELD_VOLUME:
      for (int64_t i = 0; i < n; ++i) out[i] = c->hvol[i];
      return PD_OK;
    case PD_FIELD_MODEL_COORDINATES:
      for (int64_t k = 0; k < 3 * n; ++k) out[k] = c->hx[k];
      return PD_OK;
    case PD_FIELD_NUM_NEIGHBORS: {
      std::vector<int64_t> row(n + 1);
      PD_CUDA_TRY(c, d2h(c, row.data(), c->row.p, (n + 1) * sizeof(int64_t)));
      for (int64_t i = 0; i < n; ++i) out[i] = (double)(row[i + 1] - row[i] - (c->phantoms ? c->h_nph[i] : 0));
      return PD_OK;
    }
    default: return fail(c, PD_ERR_ARG, "pd_get_field: unknown field");
  }
}

int pd_block_data(pd_ctx* c, int32_t field, int32_t block, int32_t calculation, double* out) {
  CHECK_CTX(c);
  if (!out) return fail(c, PD_ERR_ARG, "pd_block_data: null output");
  TRY(ensure_ready(c));
  TRY(compute_block_data(c, field, block, calculation, out));
  return check_status(c);
}

int pd_kinetic_energy(pd_ctx* c, double* global, double* per_point) {
  CHECK_CTX(c);
  if (!global) return fail(c, PD_ERR_ARG, "pd_kinetic_energy: null output");
  TRY(ensure_ready(c));
  TRY(compute_energy_momentum(c, 0, global, per_point));
  return check_status(c);
}

int pd_linear_momentum(pd_ctx* c, double* global, double* per_point) {
  CHECK_CTX(c);
  if (!global) return fail(c, PD_ERR_ARG, "pd_linear_momentum: null output");
  TRY(ensure_ready(c));
  TRY(compute_energy_momentum(c, 1, global, per_point));
  return check_status(c);
}

}  // extern "C"
