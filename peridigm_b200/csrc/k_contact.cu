// Short-range force contact (sm_100a): device contact search and the gather
// form of ShortRangeForceContactModel::computeForce.
//
// Search (ContactManager::contactSearch, src/core/Peridigm_ContactManager.cpp:696-748):
// every point within the search radius of the current coordinates (Zoltan
// predicate dx*dx+dy*dy+dz*dz <= r^2, self excluded), minus every pair of the
// bond family, broken bonds included (:741). Rebuilt at setup and whenever
// step % search_frequency == 0 (Peridigm.cpp:1473) from the coordinates at the
// start of that step.
//
// Force (Peridigm_ShortRangeForceContactModel.cpp:98-261): for a pair with
// d^2 < r_c^2 (strict, :139), temp = 9k/(pi h^4) * (r_c - d)/h with h the
// owner's block horizon (:142-143). Both points list each other, and each
// owner's loop adds to itself and to its neighbor, so the total on i is
//   f_i = -(temp_i + temp_j) V_j [ (y_j - y_i)/d + mu * w_i/|w_i| ]
// where w_i is i's velocity perpendicular to the pair minus the pair's mean
// perpendicular velocity (:150-234; the mu term only when mu != 0 and
// |w_i| != 0). Computed per owner, FP64, no atomics.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "cells.cuh"
#include "pd_internal.cuh"

namespace pdb {

struct ContactState {
  double r_search = 0.0;
  int freq = 0;
  double r_contact = 0.0;
  double k_spring = 0.0;
  double friction = 0.0;
  DBuf<double> kappa;    // 9k/(pi h^5) per point (temp = kappa*(r_c - d))
  DBuf<double4> pos;     // search positions (x, y, z, -)
  DBuf<double> y;        // current coordinates [3n] for the force pass
  DBuf<int64_t> crow;    // contact CSR
  DBuf<int32_t> ccol;
  int64_t npairs = 0;
  bool have_list = false;
  // search temporaries kept between searches (grown only): a search between
  // steps then allocates and frees no device memory, whose driver calls can
  // wait behind other processes' queries of the device
  DBuf<double> part;
  DBuf<int32_t> idx_s;
  DBuf<int64_t> cell_start, counts;
  DBuf<unsigned char> stmp;
  BinScratch bins;
};

__device__ __forceinline__ double sq3(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ bool in_row(const int64_t* __restrict__ row, const int32_t* __restrict__ col, int64_t i,
                                       int32_t j) {
  int64_t lo = row[i], hi = row[i + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (col[mid] < j) lo = mid + 1;
    else hi = mid;
  }
  return lo < row[i + 1] && col[lo] == j;
}

// Coordinates for the search: y = x + u (FP64 path: the stored y).
__global__ void k_contact_positions(int64_t n, const double4* __restrict__ xv, const double* __restrict__ u,
                                    const double4* __restrict__ st, double4* __restrict__ pos,
                                    double* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p;
  if (st) {
    p = st[i];
  } else {
    const double4 x = xv[i];
    p = make_double4(__dadd_rn(x.x, u[3 * i]), __dadd_rn(x.y, u[3 * i + 1]), __dadd_rn(x.z, u[3 * i + 2]), 0.0);
  }
  pos[i] = make_double4(p.x, p.y, p.z, 0.0);
  if (y) {
    y[3 * i] = p.x;
    y[3 * i + 1] = p.y;
    y[3 * i + 2] = p.z;
  }
}

// One warp per point; FILL = false counts, FILL = true writes the row.
template <bool FILL>
__global__ void __launch_bounds__(256) k_contact_search(int64_t n, const double4* __restrict__ pos, Grid g,
                                                       const int64_t* __restrict__ cell_start,
                                                       const int32_t* __restrict__ sorted_idx, double r_search,
                                                       const int64_t* __restrict__ brow,
                                                       const int32_t* __restrict__ bcol, int64_t* __restrict__ counts,
                                                       const int64_t* __restrict__ crow, int32_t* __restrict__ ccol) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const double4 pi = pos[i];
  const double R2 = __dmul_rn(r_search, r_search);
  const int c0 = cell_coord(g, pi.x, 0), c1 = cell_coord(g, pi.y, 1), c2 = cell_coord(g, pi.z, 2);
  int64_t cnt = 0;
  int64_t base = FILL ? crow[i] : 0;
  for (int zc = c2 - 1; zc <= c2 + 1; ++zc) {
    if (zc < 0 || zc >= g.dims[2]) continue;
    for (int yc = c1 - 1; yc <= c1 + 1; ++yc) {
      if (yc < 0 || yc >= g.dims[1]) continue;
      for (int xc = c0 - 1; xc <= c0 + 1; ++xc) {
        if (xc < 0 || xc >= g.dims[0]) continue;
        const int64_t q = ((int64_t)zc * g.dims[1] + yc) * g.dims[0] + xc;
        const int64_t s0 = cell_start[q], s1 = cell_start[q + 1];
        for (int64_t s = s0; s < s1; s += 32) {
          bool hit = false;
          int32_t j = -1;
          if (s + lane < s1) {
            j = sorted_idx[s + lane];
            if (j != i) {
              const double4 pj = pos[j];
              hit = sq3(__dsub_rn(pj.x, pi.x), __dsub_rn(pj.y, pi.y), __dsub_rn(pj.z, pi.z)) <= R2 &&
                    !in_row(brow, bcol, i, j);
            }
          }
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (FILL) {
            if (hit) ccol[base + __popc(m & ((1u << lane) - 1u))] = j;
            base += __popc(m);
          } else {
            cnt += __popc(m);
          }
        }
      }
    }
  }
  if (!FILL && lane == 0) counts[i] = cnt;
}

// Contact force density on each point (gather over its contact list).
__global__ void __launch_bounds__(256) k_contact_force(int64_t n, const int64_t* __restrict__ crow,
                                                      const int32_t* __restrict__ ccol,
                                                      const double* __restrict__ y, const double* __restrict__ v,
                                                      const double4* __restrict__ xv,
                                                      const double* __restrict__ kappa, double r_contact,
                                                      double friction, double* __restrict__ fc,
                                                      int* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double yi0 = y[3 * i], yi1 = y[3 * i + 1], yi2 = y[3 * i + 2];
  const double vi0 = v[3 * i], vi1 = v[3 * i + 1], vi2 = v[3 * i + 2];
  const double rc2 = __dmul_rn(r_contact, r_contact);
  const double ki = kappa[i];
  double f0 = 0.0, f1 = 0.0, f2 = 0.0;
  for (int64_t b = crow[i]; b < crow[i + 1]; ++b) {
    const int32_t j = ccol[b];
    const double d0 = __dsub_rn(y[3 * j], yi0), d1 = __dsub_rn(y[3 * j + 1], yi1), d2 = __dsub_rn(y[3 * j + 2], yi2);
    const double dd = sq3(__dsub_rn(yi0, y[3 * j]), __dsub_rn(yi1, y[3 * j + 1]), __dsub_rn(yi2, y[3 * j + 2]));
    if (!(dd < rc2)) continue;
    const double d = __dsqrt_rn(dd);
    const double gap = __dsub_rn(r_contact, d);
    const double temp = __dadd_rn(__dmul_rn(ki, gap), __dmul_rn(kappa[j], gap));
    const double Vj = xv[j].w;
    const double s = __dmul_rn(temp, Vj);
    f0 = __dsub_rn(f0, __ddiv_rn(__dmul_rn(s, d0), d));
    f1 = __dsub_rn(f1, __ddiv_rn(__dmul_rn(s, d1), d));
    f2 = __dsub_rn(f2, __ddiv_rn(__dmul_rn(s, d2), d));
    if (friction != 0.0) {
      const double n0 = d0 / d, n1 = d1 / d, n2 = d2 / d;
      const double vj0 = v[3 * j], vj1 = v[3 * j + 1], vj2 = v[3 * j + 2];
      const double ci = vi0 * n0 + vi1 * n1 + vi2 * n2;
      const double cj = vj0 * n0 + vj1 * n1 + vj2 * n2;
      const double pi0 = vi0 - ci * n0, pi1 = vi1 - ci * n1, pi2 = vi2 - ci * n2;
      const double pj0 = vj0 - cj * n0, pj1 = vj1 - cj * n1, pj2 = vj2 - cj * n2;
      const double w0 = pi0 - 0.5 * (pi0 + pj0), w1 = pi1 - 0.5 * (pi1 + pj1), w2 = pi2 - 0.5 * (pi2 + pj2);
      const double wn = sqrt(w0 * w0 + w1 * w1 + w2 * w2);
      if (wn != 0.0) {
        const double fr = friction * s / wn;
        f0 -= fr * w0;
        f1 -= fr * w1;
        f2 -= fr * w2;
      }
    }
  }
  if (!isfinite(f0) || !isfinite(f1) || !isfinite(f2)) atomicOr(status, ST_NONFINITE_CONTACT);
  fc[3 * i] = f0;
  fc[3 * i + 1] = f1;
  fc[3 * i + 2] = f2;
}

__global__ void k_bbox(int64_t n, const double4* __restrict__ pos, double* __restrict__ partial) {
  __shared__ double s[6][256];
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = pos[i];
    lo[0] = fmin(lo[0], p.x), lo[1] = fmin(lo[1], p.y), lo[2] = fmin(lo[2], p.z);
    hi[0] = fmax(hi[0], p.x), hi[1] = fmax(hi[1], p.y), hi[2] = fmax(hi[2], p.z);
  }
  for (int k = 0; k < 3; ++k) {
    s[k][threadIdx.x] = lo[k];
    s[k + 3][threadIdx.x] = hi[k];
  }
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = fmin(s[k][threadIdx.x], s[k][threadIdx.x + o]);
        s[k + 3][threadIdx.x] = fmax(s[k + 3][threadIdx.x], s[k + 3][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) partial[6 * blockIdx.x + k] = s[k][0];
}

__global__ void k_pos_from_y(int64_t n, const double* y, double4* pos) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  pos[i] = make_double4(y[3 * i], y[3 * i + 1], y[3 * i + 2], 0.0);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int contact_search(pd_ctx* c, const double4* pos) {
  ContactState* cs = c->contact;
  const int64_t n = c->n;
  // bounding box of the search positions
  const int nblk = 148;
  DBuf<double>& part = cs->part;
  PD_CUDA_TRY(c, part.reserve(6 * nblk));
  k_bbox<<<nblk, 256, 0, c->stream>>>(n, pos, part.p);
  std::vector<double> hp(6 * nblk);
  PD_CUDA_TRY(c, cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int b = 0; b < nblk; ++b)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], hp[6 * b + k]);
      hi[k] = std::max(hi[k], hp[6 * b + 3 + k]);
    }
  if (!(std::isfinite(lo[0]) && std::isfinite(hi[0]) && std::isfinite(lo[1]) && std::isfinite(hi[1]) &&
        std::isfinite(lo[2]) && std::isfinite(hi[2]))) {
    c->err = "non-finite coordinates in the contact search";
    return PD_ERR_NONFINITE;
  }
  const Grid g = make_grid(n, lo, hi, cs->r_search);
  DBuf<int32_t>& idx_s = cs->idx_s;
  DBuf<int64_t>& cell_start = cs->cell_start;
  DBuf<int64_t>& counts = cs->counts;
  int rc = bin_points(c, pos, n, g, idx_s, cell_start, &cs->bins);
  if (rc != PD_OK) return rc;
  PD_CUDA_TRY(c, counts.reserve(n + 1));
  const unsigned gw = (unsigned)((n * 32 + 255) / 256);
  k_contact_search<false><<<gw, 256, 0, c->stream>>>(n, pos, g, cell_start.p, idx_s.p, cs->r_search, c->row.p,
                                                     c->col.p, counts.p, nullptr, nullptr);
  PD_CUDA_TRY(c, cudaGetLastError());
  if (cs->crow.count < (size_t)(n + 1)) PD_CUDA_TRY(c, cs->crow.alloc(n + 1));
  PD_CUDA_TRY(c, cudaMemsetAsync(counts.p + n, 0, sizeof(int64_t), c->stream));
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts.p, cs->crow.p, (int)(n + 1), c->stream);
  DBuf<unsigned char>& stmp = cs->stmp;
  PD_CUDA_TRY(c, stmp.reserve(scan_bytes));
  scan_bytes = stmp.count;
  PD_CUDA_TRY(c, cub::DeviceScan::ExclusiveSum(stmp.p, scan_bytes, counts.p, cs->crow.p, (int)(n + 1), c->stream));
  int64_t np = 0;
  PD_CUDA_TRY(c, cudaMemcpyAsync(&np, cs->crow.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (cs->ccol.count < (size_t)std::max<int64_t>(np, 1)) PD_CUDA_TRY(c, cs->ccol.alloc((size_t)std::max<int64_t>(np, 1) * 5 / 4 + 16));
  k_contact_search<true><<<gw, 256, 0, c->stream>>>(n, pos, g, cell_start.p, idx_s.p, cs->r_search, c->row.p,
                                                    c->col.p, nullptr, cs->crow.p, cs->ccol.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  cs->npairs = np;
  cs->have_list = true;
  return PD_OK;
}

static int ensure_contact_buffers(pd_ctx* c) {
  ContactState* cs = c->contact;
  const int64_t n = c->n;
  if (cs->pos.count < (size_t)n) {
    PD_CUDA_TRY(c, cs->pos.alloc(n));
    PD_CUDA_TRY(c, cs->y.alloc(3 * n));
    PD_CUDA_TRY(c, cs->kappa.alloc(n));
  }
  std::vector<double> kap(n);
  const double pi = 3.14159265358979323846;
  for (int64_t i = 0; i < n; ++i) {
    const double h = c->block_h[c->hblock.empty() ? 0 : c->hblock[i]];
    kap[i] = (9.0 * cs->k_spring / (pi * h * h * h * h)) / h;
  }
  PD_CUDA_TRY(c, h2d(c, cs->kappa.p, kap.data(), n * sizeof(double)));
  return PD_OK;
}

void contact_release(pd_ctx* c) {
  delete c->contact;
  c->contact = nullptr;
}

int64_t contact_pairs(const pd_ctx* c) { return c->contact ? c->contact->npairs : 0; }

// Positions at the start of evaluation `step` come from the previous state
// buffer (the current one already holds this step's displacement).
int contact_prepare(pd_ctx* c, int64_t step) {
  ContactState* cs = c->contact;
  if (!cs) return PD_OK;
  const bool search = step == 0 || !cs->have_list || (cs->freq > 0 && step % cs->freq == 0);
  if (!search) return PD_OK;
  const int64_t n = c->n;
  const unsigned g1 = (unsigned)((n + 255) / 256);
  if (c->precision != PD_SPLIT_FP32) {
    const double4* src = step == 0 ? c->st[c->cur].p : c->st[c->cur ^ 1].p;
    k_contact_positions<<<g1, 256, 0, c->stream>>>(n, c->xv.p, nullptr, src, cs->pos.p, nullptr);
  } else if (step == 0) {
    k_contact_positions<<<g1, 256, 0, c->stream>>>(n, c->xv.p, c->u.p, nullptr, cs->pos.p, nullptr);
  } else {
    // u of the previous step from the previous hi/lo record
    PD_CUDA_TRY(c, launch_u_from_record(c, c->cur ^ 1, cs->y.p));
    k_contact_positions<<<g1, 256, 0, c->stream>>>(n, c->xv.p, cs->y.p, nullptr, cs->pos.p, nullptr);
  }
  PD_CUDA_TRY(c, cudaGetLastError());
  return contact_search(c, cs->pos.p);
}

// Contact force density of the current configuration into c->fc.
int contact_eval(pd_ctx* c) {
  ContactState* cs = c->contact;
  if (!cs) return PD_OK;
  const int64_t n = c->n;
  const unsigned g1 = (unsigned)((n + 255) / 256);
  const double4* st = c->precision != PD_SPLIT_FP32 ? c->st[c->cur].p : nullptr;
  k_contact_positions<<<g1, 256, 0, c->stream>>>(n, c->xv.p, c->u.p, st, cs->pos.p, cs->y.p);
  k_contact_force<<<g1, 256, 0, c->stream>>>(n, cs->crow.p, cs->ccol.p, cs->y.p, c->v.p, c->xv.p, cs->kappa.p,
                                             cs->r_contact, cs->friction, c->fc.p, c->status.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

int contact_configure(pd_ctx* c, double r_search, int freq, double r_contact, double k_spring, double friction) {
  if (r_contact <= 0.0) {
    contact_release(c);
    return PD_OK;
  }
  if (!(r_search >= r_contact) || freq < 0 || !(k_spring > 0.0) || friction < 0.0) {
    c->err = "contact: need search radius >= contact radius > 0, spring constant > 0, friction >= 0";
    return PD_ERR_ARG;
  }
  if (!c->contact) c->contact = new ContactState();
  ContactState* cs = c->contact;
  cs->r_search = r_search;
  cs->freq = freq;
  cs->r_contact = r_contact;
  cs->k_spring = k_spring;
  cs->friction = friction;
  cs->have_list = false;
  return ensure_contact_buffers(c);
}

// Drop-in ShortRangeForceContactModel::computeForce on caller coordinates and
// velocities (device pointers): search with y, then the force.
int contact_force_from(pd_ctx* c, const double* y_dev, const double* v_dev, double* fc_dev) {
  ContactState* cs = c->contact;
  const int64_t n = c->n;
  const unsigned g1 = (unsigned)((n + 255) / 256);
  PD_CUDA_TRY(c, cudaMemcpyAsync(cs->y.p, y_dev, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  k_pos_from_y<<<g1, 256, 0, c->stream>>>(n, cs->y.p, cs->pos.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  int rc = contact_search(c, cs->pos.p);
  if (rc != PD_OK) return rc;
  k_contact_force<<<g1, 256, 0, c->stream>>>(n, cs->crow.p, cs->ccol.p, cs->y.p, v_dev, c->xv.p, cs->kappa.p,
                                             cs->r_contact, cs->friction, fc_dev, c->status.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}



}  // namespace pdb
