// Compute classes as device reductions (sm_100a):
//   Block_Data            src/compute/Peridigm_Compute_Block_Data.cpp:121-210
//                         (Minimum / Maximum / Sum of a scalar or vector field
//                         over the owned points of one block)
//   Kinetic_Energy        src/compute/Peridigm_Compute_Kinetic_Energy.cpp:79-150
//                         (0.5 V rho |v|^2 per point and its global sum)
//   Linear_Momentum       src/compute/Peridigm_Compute_Linear_Momentum.cpp:110-150
//                         (rho V v per point and its global sum)
// Reductions run in a fixed order (a fixed grid of 296 blocks, grid-stride
// partials, fixed-shape trees), so results are bit-reproducible run to run;
// they differ from the reference's serial sums by rounding only. Maximum
// starts from DBL_MIN as the reference does (:137-140), so a maximum of a
// field with no positive entry is DBL_MIN.
#include <cfloat>
#include <vector>

#include "pd_internal.cuh"

namespace pdb {

constexpr int kCBlock = 256;
constexpr int kCGrid = 296;  // 2 x 148 SMs, fixed for determinism

enum CalcType { CALC_MIN = 0, CALC_MAX = 1, CALC_SUM = 2 };

struct FieldView {
  const double* p;  // per-point data (stride `width`), or null for derived fields
  int width;        // 1 or 3
  int kind;         // 0 plain, 1 force = force density x volume, 2 coordinates = x + u, 3 volume, 4 neighbors
};

__device__ __forceinline__ double field_value(const FieldView& f, int64_t i, int c, const double4* xv,
                                              const int64_t* row) {
  switch (f.kind) {
    case 1: return f.p[3 * i + c] * xv[i].w;
    case 2: return (c == 0 ? xv[i].x : (c == 1 ? xv[i].y : xv[i].z)) + f.p[3 * i + c];
    case 3: return xv[i].w;
    case 4: return (double)(row[i + 1] - row[i]);
    default: return f.p[(int64_t)f.width * i + c];
  }
}

__device__ __forceinline__ double combine(int calc, double a, double b) {
  return calc == CALC_MIN ? fmin(a, b) : (calc == CALC_MAX ? fmax(a, b) : a + b);
}

// partial[3 * blockIdx + c] over the points of `block` (-1: all points).
__global__ void __launch_bounds__(kCBlock) k_block_data(int64_t n, FieldView f, const int32_t* __restrict__ blk,
                                                        int block, int calc, const double4* __restrict__ xv,
                                                        const int64_t* __restrict__ row, double* __restrict__ partial) {
  __shared__ double s[3][kCBlock];
  const double init = calc == CALC_MIN ? DBL_MAX : (calc == CALC_MAX ? DBL_MIN : 0.0);
  double a[3] = {init, init, init};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (block >= 0 && (blk ? blk[i] : 0) != block) continue;
    for (int c = 0; c < f.width; ++c) a[c] = combine(calc, a[c], field_value(f, i, c, xv, row));
  }
  for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = a[c];
  __syncthreads();
  for (int o = kCBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = combine(calc, s[c][threadIdx.x], s[c][threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) partial[3 * blockIdx.x + c] = s[c][0];
}

// Kinetic energy (what = 0: 0.5 V rho |v|^2, one value) or linear momentum
// (what = 1: rho V v, three values) per point (optional) and block partials.
__global__ void __launch_bounds__(kCBlock) k_energy_momentum(int64_t n, int what, const double* __restrict__ v,
                                                             const double4* __restrict__ xv,
                                                             const double4* __restrict__ pt,
                                                             double* __restrict__ per_point,
                                                             double* __restrict__ partial) {
  __shared__ double s[3][kCBlock];
  double a[3] = {0.0, 0.0, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double v1 = v[3 * i], v2 = v[3 * i + 1], v3 = v[3 * i + 2];
    const double vol = xv[i].w, density = pt[i].w;
    if (what == 0) {
      const double ke = 0.5 * vol * density * (v1 * v1 + v2 * v2 + v3 * v3);
      if (per_point) per_point[i] = ke;
      a[0] += ke;
    } else {
      const double mass = density * vol;
      const double p1 = mass * v1, p2 = mass * v2, p3 = mass * v3;
      if (per_point) per_point[3 * i] = p1, per_point[3 * i + 1] = p2, per_point[3 * i + 2] = p3;
      a[0] += p1;
      a[1] += p2;
      a[2] += p3;
    }
  }
  for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = a[c];
  __syncthreads();
  for (int o = kCBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) s[c][threadIdx.x] += s[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) partial[3 * blockIdx.x + c] = s[c][0];
}

__global__ void k_reduce_partials(int nblk, int calc, const double* __restrict__ partial, double* __restrict__ out) {
  __shared__ double s[3][kCBlock];
  const double init = calc == CALC_MIN ? DBL_MAX : (calc == CALC_MAX ? DBL_MIN : 0.0);
  double a[3] = {init, init, init};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    for (int c = 0; c < 3; ++c) a[c] = combine(calc, a[c], partial[3 * b + c]);
  for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = a[c];
  __syncthreads();
  for (int o = kCBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) s[c][threadIdx.x] = combine(calc, s[c][threadIdx.x], s[c][threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) out[c] = s[c][0];
}

// ---------------------------------------------------------------------------
// Host side (called from api.cu with the context ready)
// ---------------------------------------------------------------------------
static int ensure_block_ids(pd_ctx* c) {
  if (c->blk_dev.p || c->hblock.empty()) return PD_OK;
  PD_CUDA_TRY(c, c->blk_dev.alloc(c->n));
  PD_CUDA_TRY(c, h2d(c, c->blk_dev.p, c->hblock.data(), c->n * sizeof(int32_t)));
  return PD_OK;
}

int compute_block_data(pd_ctx* c, int field, int block, int calc, double* out3) {
  FieldView f{nullptr, 3, 0};
  switch (field) {
    case PD_FIELD_DISPLACEMENT: f.p = c->u.p; break;
    case PD_FIELD_VELOCITY: f.p = c->v.p; break;
    case PD_FIELD_ACCELERATION: f.p = c->a.p; break;
    case PD_FIELD_FORCE_DENSITY: f.p = c->f.p; break;
    case PD_FIELD_CONTACT_FORCE: f.p = c->fc.p; break;
    case PD_FIELD_FORCE: f.p = c->f.p, f.kind = 1; break;
    case PD_FIELD_COORDINATES: f.p = c->u.p, f.kind = 2; break;
    case PD_FIELD_DILATATION: f.p = c->theta.p, f.width = 1; break;
    case PD_FIELD_DAMAGE: f.p = c->node_damage.p, f.width = 1; break;
    case PD_FIELD_VOLUME: f.width = 1, f.kind = 3; break;
    case PD_FIELD_NUM_NEIGHBORS: f.width = 1, f.kind = 4; break;
    default:
      c->err = "pd_block_data: the field is not a per-point scalar or vector field";
      return PD_ERR_ARG;
  }
  if (calc < CALC_MIN || calc > CALC_SUM) {
    c->err = "pd_block_data: invalid calculation type, must be minimum, maximum or sum";
    return PD_ERR_ARG;
  }
  if (block < 0 || block >= c->n_blocks) {
    c->err = "pd_block_data: no such block";
    return PD_ERR_ARG;
  }
  TRY_RC(ensure_block_ids(c));
  DBuf<double> nn;
  if (f.kind == 4 && c->phantoms) {  // own-family sizes (rows also hold phantom halves)
    std::vector<int64_t> row(c->n + 1);
    PD_CUDA_TRY(c, d2h(c, row.data(), c->row.p, (c->n + 1) * sizeof(int64_t)));
    std::vector<double> h(std::max<int64_t>(c->n, 1));
    for (int64_t i = 0; i < c->n; ++i) h[i] = (double)(row[i + 1] - row[i] - c->h_nph[i]);
    PD_CUDA_TRY(c, nn.alloc(h.size()));
    PD_CUDA_TRY(c, h2d(c, nn.p, h.data(), h.size() * sizeof(double)));
    f.p = nn.p, f.kind = 0;
  }
  DBuf<double> part, out;
  PD_CUDA_TRY(c, part.alloc(3 * kCGrid));
  PD_CUDA_TRY(c, out.alloc(3));
  k_block_data<<<kCGrid, kCBlock, 0, c->stream>>>(c->n, f, c->blk_dev.p, c->hblock.empty() ? 0 : block, calc,
                                                 c->xv.p, c->row.p, part.p);
  k_reduce_partials<<<1, kCBlock, 0, c->stream>>>(kCGrid, calc, part.p, out.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  double h[3];
  PD_CUDA_TRY(c, d2h(c, h, out.p, sizeof(h)));
  for (int k = 0; k < 3; ++k) out3[k] = k < f.width ? h[k] : 0.0;
  return PD_OK;
}

int compute_energy_momentum(pd_ctx* c, int what, double* global, double* per_point_host) {
  DBuf<double> part, out, pp;
  PD_CUDA_TRY(c, part.alloc(3 * kCGrid));
  PD_CUDA_TRY(c, out.alloc(3));
  const int width = what == 0 ? 1 : 3;
  if (per_point_host) PD_CUDA_TRY(c, pp.alloc((size_t)width * c->n));
  k_energy_momentum<<<kCGrid, kCBlock, 0, c->stream>>>(c->n, what, c->v.p, c->xv.p, c->pt.p,
                                                      per_point_host ? pp.p : nullptr, part.p);
  k_reduce_partials<<<1, kCBlock, 0, c->stream>>>(kCGrid, CALC_SUM, part.p, out.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  double h[3];
  PD_CUDA_TRY(c, d2h(c, h, out.p, sizeof(h)));
  for (int k = 0; k < width; ++k) global[k] = h[k];
  if (per_point_host) PD_CUDA_TRY(c, d2h(c, per_point_host, pp.p, (size_t)width * c->n * sizeof(double)));
  return PD_OK;
}

}  // namespace pdb
