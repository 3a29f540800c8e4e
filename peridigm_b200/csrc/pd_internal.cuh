// Internal declarations of the B200 Peridigm hot path: the device-side data
// layout of a context and the kernels' launch helpers.
//
// HBM layout (n points, nb directed bonds, all in the caller's point order):
//   xv[n]        double4 (x, y, z, V) FP64 model coordinates and volume
//   row[n+1]     int64 bond row pointers          col[nb] int32 neighbor ids
//   dmg[nb]      uint8 bond damage (0/1), monotone, updated in place
//   pt[n]        double4 (m, K, mu, rho) per-point material, sc[n] critical stretch, hp[n] horizon
//   u[3n], v[3n], a[3n], f[3n], fc[3n] FP64 integration state (interleaved xyz)
// Split-FP32 path:
//   bx3          X = x_j - x_i per bond in FP32 (formed in FP64, rounded once,
//                constant), streamed; 32-bond groups of x[32], y[32], z[32]
//   ur[2][n]     Rec8 (u_hi[3], lo_xy, lo_z|q, V, A, B) gathered per neighbor
//                with one 256-bit load; u = u_hi + 16-bit residuals times a
//                shared power of two q; double buffered across steps
//   own[n]       float4 (3/m, (3K-5mu)/m, 15mu/m, s_c)  owner terms
// FP64 paths:
//   st[2][n]     double4 (y_x, y_y, y_z, V) current coordinates and volume, double buffered
//   ab64[n]      double4 (theta, 3K/m - alpha/3, alpha, 0); on the FP64 sliced
//                path (A, B, theta, 0) with A = theta*(3K/m - alpha/3), B = alpha
//   bx64         X per bond in FP64 on the sliced stream (FP64 sliced path)
// A = theta*(3K-5mu)/m and B = 15mu/m are the owner terms of the LPS force
// state t = (1-d)[A*omega*|xi| + (1-d)*B*omega*e] (elastic.cxx:99,119-120).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pd_b200.h"

namespace pdb {

// Point chunks of pd_compute_force's host transfers: the coordinates go up in
// chunks while the dilatation of the chunks already there computes, and the
// force density comes down chunk by chunk while the later chunks compute. The
// transfers that cannot overlap (the first chunks up, the last one down)
// shrink with the chunk: 32 chunks against 16 took the 32,000,000-point step
// from 32.4 to 31.8 ms; 64 were slower again (32.2 against 31.9 ms).
constexpr int kHostChunks = 32;

// One 32-byte record per point, fetched with a single 256-bit load.
struct __align__(32) Rec8 {
  float v[8];
};

// ---------------------------------------------------------------------------
// Kernel parameter blocks
// ---------------------------------------------------------------------------
struct BondView {
  const int64_t* row;
  const int32_t* col;
  uint8_t* dmg;
  int64_t n;
};

struct StepParams {
  // integration
  double dt;
  double t0;
  int64_t step;     // step index n being completed by this evaluation (0 = initial)
  int mode;         // EvalMode
  int influence;
  int damage_on;
  int has_contact;
  int has_bc;
  // outputs
  double* f_out;    // force density [3n] (may be null)
  double* f_host = nullptr;  // host copy of f_out, overlapped with the force pass where it can be
  // host coordinates [3n] to evaluate at, uploaded through f_out (which then
  // receives the force density), overlapped with the dilatation where it can be
  const double* y_host = nullptr;
};

// EVAL_ONLY: evaluation (force out) with no integration; EVAL_ADVANCE: finish
// evaluation `step` and advance the state to step+1; EVAL_LAST: finish the
// last step (v, a final, no advance).
enum EvalMode { EVAL_ONLY = 0, EVAL_ADVANCE = 2, EVAL_LAST = 3 };

// ---------------------------------------------------------------------------
// Device buffer
// ---------------------------------------------------------------------------
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t count = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  cudaError_t alloc(size_t n) {
    release();
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)&p, n * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    count = n;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    count = 0;
  }
  size_t bytes() const { return count * sizeof(T); }
  // At least n elements, reallocating (with a quarter's headroom) only when
  // smaller: repeated work reuses its buffers instead of allocating each time.
  cudaError_t reserve(size_t n) {
    if (p && count >= n) return cudaSuccess;
    return alloc(n + n / 4 + 16);
  }
};

struct ContactState;
struct QsState;
struct CoarseState;

}  // namespace pdb

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct pd_ctx {
  int device = 0;
  int precision = PD_SPLIT_FP32;
  int influence = PD_INFLUENCE_ONE;
  int tpo = 16;       // lanes per point (FP64 path and setup kernels)
  int tpo_split = 4;  // lanes per point of the split-FP32 bond passes
  cudaStream_t stream = nullptr;
  // chunked force download of pd_compute_force (created on first use)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t chunk_ev[pdb::kHostChunks + 1] = {};
  cudaEvent_t up_ev[pdb::kHostChunks] = {};  // the chunked coordinate upload
  // per upload chunk: the largest neighbor index of its rows (the last upload
  // chunk its dilatation reads), for the bond set of (chunk_hi_row, chunk_hi_nb)
  std::vector<int64_t> chunk_hi;
  const int64_t* chunk_hi_row = nullptr;
  int64_t chunk_hi_nb = -1;
  std::string err;

  // points
  int64_t n = 0;
  std::vector<double> hx, hvol;
  std::vector<int32_t> hblock;
  pdb::DBuf<int32_t> blk_dev;  // block id per point on the device (compute classes), built on demand
  int32_t n_blocks = 1;
  std::vector<double> block_h, block_K, block_mu, block_rho, block_sc;
  bool have_material = false;
  std::vector<int> block_model;  // PD_MATERIAL_* per block (-1: not set)
  int material_model = PD_MATERIAL_LPS;
  int coarse_modes = 3;  // coarse dofs per aggregate of the two-level preconditioner: 3 or 6 (rotations)
  int bb_plane = 0;              // bond-based: plane strain/stress constant
  double bb_height = 0.0;
  std::vector<double> field_K, field_mu, field_sc;  // per-point overrides (empty = none)
  pdb::DBuf<double4> xv;
  pdb::DBuf<double> hp;  // horizon per point

  // bonds
  int64_t nb = 0;
  int max_row = 0;
  bool symmetric = true;
  // Families with j in H(i) but i not in H(j) (blocks of different horizons,
  // or a caller's list): the device CSR holds every bond in both rows, the
  // added reverse (j, i) as a phantom whose own half does not exist (damage
  // bits 0 and kPhantomOwn), the original (i, j) then without a partner half
  // (bits 1 and kPhantomPartner). nb counts the device CSR, nb_user the
  // caller's families; h_orig marks the device bonds that are the caller's,
  // h_nph counts each row's phantoms.
  bool phantoms = false;
  int64_t nb_user = 0;
  std::vector<uint8_t> h_orig;
  std::vector<int32_t> h_nph;
  std::vector<uint8_t> h_dmg0;  // the device CSR's damage bytes with no bond broken
  pdb::DBuf<int64_t> row;
  pdb::DBuf<int32_t> col;
  pdb::DBuf<uint8_t> dmg;        // committed (N) bond damage
  pdb::DBuf<uint8_t> dmg_trial;  // NP1 scratch for non-committing evaluations
  bool trial_valid = false;

  // material
  bool wv_done = false;
  pdb::DBuf<double4> pt;     // (m, K, mu, rho)
  pdb::DBuf<double> sc;      // critical stretch (<0: off)
  pdb::DBuf<float> bx3;      // split path: per bond X in FP32, 32-slot groups of x/y/z planes, CSR or sliced order
  pdb::DBuf<double> bx64;    // FP64 sliced path: per bond X in FP64, the sliced order and planes of bx3
  // Sliced (SELL) bond stream of the 4-lanes-per-point split passes: slot
  // offsets per 8-owner slice, neighbor ids and a damage mirror in slice
  // order (bx3 holds the bond vectors in that order). dmg_gen counts writes to the
  // CSR damage outside the passes; the mirror is refreshed when it lags.
  bool sell = false;
  pdb::DBuf<int64_t> sell_off;
  pdb::DBuf<int32_t> sell_col;
  pdb::DBuf<uint8_t> sell_dmg;
  const uint8_t* sell_src = nullptr;
  int64_t dmg_gen = 0, sell_gen = -1;
  pdb::DBuf<float4> own;     // split path: (3/m, (3K-5mu)/m, 15mu/m, s_c)
  pdb::DBuf<float> scf;      // split path: s_c per point, gathered for the partner half's test
  bool any_damage = false;
  // Half-bond damage (bit 1 of the damage bytes differs from bit 0 somewhere,
  // or can come to): the critical stretch differs across some bond, or the
  // caller set damage whose two halves differ.
  bool sc_pair = false;
  bool dmg_asym = false;
  float sc_min = 0.0f;  // smallest critical stretch >= 0 of the points (FP32; +inf when none)
  double sc_gate64 = 0.0;  // FP64 sliced path: the smallest s_c >= 0 times (1 - 1e-12) (+inf when none)

  // state
  pdb::DBuf<double4> st[2];   // FP64 path gathered coordinates
  pdb::DBuf<pdb::Rec8> ur[2]; // split path gathered displacement records
  int cur = 0;
  pdb::DBuf<double4> ab64;
  pdb::DBuf<double> u, v, a, f, fc, theta, node_damage;
  bool state_init = false;
  // stepping form of the Verlet loop (pd_verlet_begin / _step / _finish)
  bool vrun = false;
  double vdt = 0.0, vt0 = 0.0;
  int64_t vstep = 0;
  cudaEvent_t vbeg = nullptr;

  // boundary conditions
  std::vector<uint8_t> h_bc_mask;
  std::vector<double> h_bc_a, h_bc_b;
  bool bc_dirty = true;
  bool has_bc = false;
  pdb::DBuf<uint8_t> bc_mask;
  pdb::DBuf<double> bc_a, bc_b;
  // prescribed functions of x, y, z, t (bc_expr.cuh): per dof the start of its
  // program in h_bc_code (-1: a*t + b); bit 3 + c of the mask marks such dofs
  std::vector<int64_t> h_bc_prog;
  std::vector<int32_t> h_bc_code;
  std::vector<double> h_bc_konst;
  int64_t n_bc_expr = 0;              // function dofs on the device
  pdb::DBuf<int32_t> bc_dofs, bc_start, bc_code;
  pdb::DBuf<double> bc_konst;
  pdb::DBuf<double2> bc_cp;           // per dof (u(t_c), u(t_p)) of the evaluation in flight

  // misc
  pdb::DBuf<int> status;      // device status word (non-finite etc.)
  pdb::DBuf<double> scratch;  // reduction partials
  bool ktime = false;                 // bracket bond-pass launches with events
  std::vector<cudaEvent_t> kev;        // 3 per evaluation while ktime
  size_t kev_used = 0;
  double kms[2] = {0.0, 0.0};
  int64_t klaunches = 0;
  pdb::ContactState* contact = nullptr;
  pdb::QsState* qs = nullptr;
  pdb::CoarseState* coarse = nullptr;  // aggregate coarse level of the QS preconditioners (k_coarse.cu)
  void* mpnn = nullptr;        // learned preconditioner state (k_mpnn.cu)
  int64_t qs_fallbacks = 0;    // learned-preconditioner solves that fell back to block Jacobi
};

// A device copy src -> dst of the bond damage: the sliced damage mirror, if it
// matched src, matches dst afterwards (the contents are equal); any other
// write to a damage array only advances the generation, and the mirror is
// refreshed before the next sliced pass.
inline void note_damage_copy(pd_ctx* c, const uint8_t* dst, const uint8_t* src) {
  const bool follows = c->sell_src == src && c->sell_gen == c->dmg_gen;
  c->dmg_gen++;
  if (follows) {
    c->sell_src = dst;
    c->sell_gen = c->dmg_gen;
  }
}

// ---------------------------------------------------------------------------
// Launch helpers (implemented in the .cu files)
// ---------------------------------------------------------------------------
namespace pdb {

cudaError_t launch_weighted_volume(const pd_ctx* c);
cudaError_t launch_pack_owner(pd_ctx* c);
cudaError_t launch_eval(pd_ctx* c, const StepParams& sp, uint8_t* dmg, bool* host_done = nullptr);
// Values of the prescribed functions for evaluation `step` (bc_cp).
cudaError_t launch_bc_expr(pd_ctx* c, int64_t step, double t0, double dt);
// The same at the given current and previous times (a quasi-static load step).
cudaError_t launch_bc_expr_at(pd_ctx* c, double t_cur, double t_prev);
// Gathered state of points i0 .. i1-1 (i1 < 0: all) from current coordinates y_dev [3n].
cudaError_t launch_state_from_y(pd_ctx* c, const double* y_dev, int64_t i0 = 0, int64_t i1 = -1);
cudaError_t launch_sync_state(pd_ctx* c);
cudaError_t launch_critical_dt(pd_ctx* c, double* dt_out);
// The critical-dt kernels with the block partials in caller memory: partial
// must hold critical_dt_partials(c) doubles; nothing is allocated.
int64_t critical_dt_partials(const pd_ctx* c);
cudaError_t launch_critical_dt_into(pd_ctx* c, double* partial, double* dt_out_dev);
cudaError_t collect_kernel_times(pd_ctx* c);
cudaError_t launch_fp64_eval_at(pd_ctx* c, const double4* y4, double4* ab, double* theta, double* nd, double* f_out);
int ensure_ready_internal(pd_ctx* c);

// quasi-static (k_qs.cu) and the learned preconditioner (k_mpnn.cu)
int qs_load_step(pd_ctx* c, double t_prev, double t_cur, const pd_qs_options* o, pd_stats* st);
int implicit_run(pd_ctx* c, double dt, double t0, int64_t nsteps, const pd_implicit_options* o, pd_stats* st);
int qs_tangent_apply(pd_ctx* c, const double* u_dev, const double* w_dev, double* kw_dev);
int qs_tangent_blocks(pd_ctx* c, const double* u_dev, double* blocks_dev);
int qs_prepare_current(pd_ctx* c);
int qs_apply_K(pd_ctx* c, const double* w_dev, double* kw_dev);
constexpr int kQsMulti = 6;  // vectors per multi-vector tangent product
int qs_apply_K_multi(pd_ctx* c, const double* p_dev, double* q_dev, double* dth_dev);
bool mpnn_ready(const pd_ctx* c);
int mpnn_apply_add(pd_ctx* c, const double* r, double* z);
// PD_ERR_TIMEOUT (status bit cleared) when a grid barrier wait of the apply ran out.
int mpnn_check_status(pd_ctx* c);
int mpnn_prepare(pd_ctx* c, const double* dinv);
int qs_block_jacobi_current(pd_ctx* c, const double** dinv_out);
void mpnn_release(pd_ctx* c);
int mpnn_init(pd_ctx* c, uint64_t seed, double patch);
int mpnn_train(pd_ctx* c, int epochs, double lr, int batch, double* loss_out);
int mpnn_loss_grad(pd_ctx* c, const float* pair_host, double* loss, float* grad_host);
int mpnn_middle_apply(pd_ctx* c, const double* r_host, double* z_host);
int mpnn_set_capture(pd_ctx* c, int every);
int mpnn_capture_every(const pd_ctx* c);
int mpnn_snapshot(pd_ctx* c, const double* r, const double* x);
int mpnn_commit_snapshots(pd_ctx* c, const double* x_final, const double* dinv);
void mpnn_drop_snapshots(pd_ctx* c);
int64_t mpnn_num_pairs(const pd_ctx* c);
int mpnn_get_weights(pd_ctx* c, float* w);
int mpnn_set_weights(pd_ctx* c, const float* w);
int mpnn_num_params();
const uint8_t* qs_fixed_mask(const pd_ctx* c);
int qs_build_coarse_current(pd_ctx* c, double cell);
double mpnn_coarse_cell(const pd_ctx* c);
int mpnn_set_coarse(pd_ctx* c, double cell);

// aggregate coarse level (k_coarse.cu)
int coarse_build(pd_ctx* c, const double4* y, const double4* ab, const uint8_t* fixed, double cell,
                 double* assembled);
int coarse_apply_add(pd_ctx* c, const double* r, double* z, const uint8_t* fixed);
int coarse_apply_add_f(pd_ctx* c, const float* r, double* z, const uint8_t* fixed, double scale);
int coarse_aggregates(pd_ctx* c, int32_t* agg_dev);
int coarse_copy_inverse(pd_ctx* c, double* dst_dev);
int64_t coarse_size(const pd_ctx* c);
int compute_block_data(pd_ctx* c, int field, int block, int calc, double* out3);
int compute_energy_momentum(pd_ctx* c, int what, double* global, double* per_point_host);
void coarse_release(pd_ctx* c);
void coarse_invalidate(pd_ctx* c);  // the model changed: rebuild the operator before its next use
bool coarse_valid(const pd_ctx* c);
int qs_coarse_operator(pd_ctx* c, const double* u_dev, double cell, int64_t* n_coarse, int32_t* agg_dev,
                       double* A_dev, double* Ainv_dev);

// bonds
int build_bonds_device(pd_ctx* c, const pd_plane_filter* filters, int nf);
int finalize_bonds(pd_ctx* c, bool sort_rows);

// contact (k_contact.cu) and quasi-static state hooks
void contact_release(pd_ctx* c);
int contact_prepare(pd_ctx* c, int64_t step);  // search when due at this step
int contact_eval(pd_ctx* c);                   // contact force density into c->fc
int64_t contact_pairs(const pd_ctx* c);
int contact_configure(pd_ctx* c, double r_search, int freq, double r_contact, double k_spring, double friction);
int contact_force_from(pd_ctx* c, const double* y_dev, const double* v_dev, double* fc_dev);
cudaError_t launch_u_from_record(pd_ctx* c, int parity, double* u_out);  // split path: hi + lo
// Ghost-state exchange: (u, y) of the listed points in the state the next
// evaluation reads, 6 doubles per point; unpack overwrites it.
cudaError_t launch_pack_state(pd_ctx* c, int64_t n_idx, const int32_t* idx, double* out);
cudaError_t launch_unpack_state(pd_ctx* c, int64_t n_idx, const int32_t* idx, const double* in);
// Number of broken bonds (own half, bit 0 of the damage byte) of the committed damage.
int count_broken(pd_ctx* c, int64_t* out);
// Damage bytes of both halves (bit 1 = the partner's bit 0) from src into dst; sets dmg_asym.
int mirror_damage(pd_ctx* c, const uint8_t* src, uint8_t* dst);
// Sets sc_pair: whether some bond joins points of different critical stretch.
int check_sc_pairs(pd_ctx* c);
void qs_release(pd_ctx* c);

// status bits
// Damage-byte markers of phantom halves (bits 0 and 1 are also set for them).
constexpr int kPhantomOwn = 8, kPhantomPartner = 16;

enum StatusBits { ST_NONFINITE_FORCE = 1, ST_NONFINITE_CONTACT = 2, ST_TIMEOUT = 4, ST_BAD_INDEX = 8, ST_NONFINITE_BC = 16 };

}  // namespace pdb

namespace pdb {
// Host <-> device transfers and fills in the context's stream order. The
// context stream is non-blocking, so the legacy-stream cudaMemcpy/cudaMemset
// would not be ordered with its kernels (a pageable cudaMemcpy may even return
// before its DMA lands). The copies return once complete.
inline cudaError_t h2d(const pd_ctx* c, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(c->stream);
}
inline cudaError_t d2h(const pd_ctx* c, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(c->stream);
}
inline cudaError_t dzero(const pd_ctx* c, void* dst, size_t bytes) { return cudaMemsetAsync(dst, 0, bytes, c->stream); }
}  // namespace pdb

#define TRY_RC(expr)              \
  do {                            \
    int rc_ = (expr);             \
    if (rc_ != PD_OK) return rc_; \
  } while (0)

#define PD_CUDA_TRY(ctx, expr)                                                   \
  do {                                                                           \
    cudaError_t e_ = (expr);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      (ctx)->err = std::string(#expr) + ": " + cudaGetErrorString(e_);           \
      return e_ == cudaErrorMemoryAllocation ? PD_ERR_NOMEM : PD_ERR_CUDA;       \
    }                                                                            \
  } while (0)
