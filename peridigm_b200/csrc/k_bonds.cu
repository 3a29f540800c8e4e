// Bond-family construction on the device (compiled with --fmad=false).
//
// Replaces NeighborhoodList::buildNeighborhoodList (src/io/pdneigh/NeighborhoodList.cxx:621-761):
//  1. points are binned into a uniform grid of cells whose side covers the
//     largest horizon (CUB radix sort by cell id, stable, so each cell lists
//     its points in ascending id);
//  2. per point, the 27 surrounding cells are scanned with the predicate of
//     ZoltanSearchTree::FindPointsWithinRadius (Peridigm_ZoltanSearchTree.cpp:238-245):
//     dx = x_j - x_i, keep when dx*dx+dy*dy+dz*dz <= h*h in FP64 without
//     contraction; self is excluded (BondFilterDefault, BondFilter.cxx:108-121)
//     and each plane filter is evaluated from the owner side
//     (FinitePlaneFilter::filterBonds, BondFilter.cxx:123-150);
//  3. count -> exclusive scan (int64 row pointers) -> fill -> per-row sort,
//     giving rows ascending by neighbor id like NeighborhoodList.cxx:705.
// The grid only generates candidates; membership is decided by the
// predicate alone, so the family equals the reference's.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>

#include "cells.cuh"
#include "pd_internal.cuh"

namespace pdb {

struct PlaneDev {
  double n[3], r0[3], ub[3], ua[3];
  double a, b;
};
constexpr int kMaxPlanes = 16;
struct Planes {
  PlaneDev p[kMaxPlanes];
  int count;
};

__global__ void k_cell_ids(int64_t n, const double4* __restrict__ xv, Grid g, int32_t* __restrict__ cid,
                           int32_t* __restrict__ idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = xv[i];
  const int a = cell_coord(g, p.x, 0), b = cell_coord(g, p.y, 1), c = cell_coord(g, p.z, 2);
  cid[i] = (c * g.dims[1] + b) * g.dims[0] + a;
  idx[i] = (int32_t)i;
}

// cell_start[c] = first position of cell c in the sorted order; cell_start[ncell] = n.
__global__ void k_cell_bounds(int64_t n, int64_t ncell, const int32_t* __restrict__ sorted_cid,
                              int64_t* __restrict__ cell_start) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s > n) return;
  const int64_t cur = s < n ? sorted_cid[s] : ncell;
  const int64_t prev = s > 0 ? sorted_cid[s - 1] : -1;
  for (int64_t c = prev + 1; c <= cur; ++c) cell_start[c] = s;
}

// FinitePlane::bondIntersectInfinitePlane + bondIntersect (BondFilter.cxx:63-106),
// tolerance 1e-15 of FinitePlaneFilter (BondFilter.h:122).
__device__ bool plane_cuts(const PlaneDev& P, const double* p0, const double* p1) {
  const double num = (P.r0[0] - p0[0]) * P.n[0] + (P.r0[1] - p0[1]) * P.n[1] + (P.r0[2] - p0[2]) * P.n[2];
  const double den = (p1[0] - p0[0]) * P.n[0] + (p1[1] - p0[1]) * P.n[1] + (p1[2] - p0[2]) * P.n[2];
  double t;
  if (fabs(den) < 1.0e-14)
    t = DBL_MAX;
  else
    t = num / den;
  if (!(t >= 0.0 && t <= 1.0)) return false;
  const double x0 = p0[0] + t * (p1[0] - p0[0]);
  const double x1 = p0[1] + t * (p1[1] - p0[1]);
  const double x2 = p0[2] + t * (p1[2] - p0[2]);
  const double zero = 1.0e-15, one = 1.0 + zero;
  const double d0 = x0 - P.r0[0], d1 = x1 - P.r0[1], d2 = x2 - P.r0[2];
  const double aa = d0 * P.ua[0] + d1 * P.ua[1] + d2 * P.ua[2];
  const double bb = d0 * P.ub[0] + d1 * P.ub[1] + d2 * P.ub[2];
  return -zero < aa && aa / P.a < one && -zero < bb && bb / P.b < one;
}

__device__ __forceinline__ bool is_bond(int64_t i, int64_t j, const double* pi, const double4& xj, double R2,
                                        const Planes& pl) {
  if (j == i) return false;
  const double dx = (xj.x - pi[0]);
  const double dy = (xj.y - pi[1]);
  const double dz = (xj.z - pi[2]);
  if (!(dx * dx + dy * dy + dz * dz <= R2)) return false;
  const double pj[3] = {xj.x, xj.y, xj.z};
  for (int f = 0; f < pl.count; ++f)
    if (plane_cuts(pl.p[f], pi, pj)) return false;
  return true;
}

// One warp per point; FILL = false counts, FILL = true writes the row.
template <bool FILL>
__global__ void __launch_bounds__(256) k_neighbors(int64_t n, const double4* __restrict__ xv,
                                                  const double* __restrict__ hp, Grid g,
                                                  const int64_t* __restrict__ cell_start,
                                                  const int32_t* __restrict__ sorted_idx, Planes pl,
                                                  int64_t* __restrict__ counts, const int64_t* __restrict__ row,
                                                  int32_t* __restrict__ col) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;  // whole warp exits together
  const double4 xi4 = xv[i];
  const double pi[3] = {xi4.x, xi4.y, xi4.z};
  const double h = hp[i];
  const double R2 = h * h;
  const int c0 = cell_coord(g, pi[0], 0), c1 = cell_coord(g, pi[1], 1), c2 = cell_coord(g, pi[2], 2);
  int64_t cnt = 0;
  int64_t base = FILL ? row[i] : 0;
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
            hit = is_bond(i, j, pi, xv[j], R2, pl);
          }
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (FILL) {
            if (hit) col[base + __popc(m & ((1u << lane) - 1u))] = j;
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

// Sort each row ascending. One warp per row, bitonic sort in shared memory on
// the next power of two >= row length (<= P), padded with INT_MAX.
template <int P>
__global__ void __launch_bounds__(128) k_sort_rows(int64_t n, const int64_t* __restrict__ row,
                                                   int32_t* __restrict__ col) {
  __shared__ int32_t buf[4][P];
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t i = (int64_t)blockIdx.x * 4 + w;
  if (i >= n) return;
  const int64_t b0 = row[i];
  const int len = (int)(row[i + 1] - b0);
  if (len <= 1 || len > P) return;
  int p2 = 1;
  while (p2 < len) p2 <<= 1;
  int32_t* s = buf[w];
  for (int k = lane; k < p2; k += 32) s[k] = k < len ? col[b0 + k] : INT_MAX;
  __syncwarp();
  for (int size = 2; size <= p2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = lane; k < p2; k += 32) {
        const int partner = k ^ stride;
        if (partner > k) {
          const bool up = (k & size) == 0;
          const int32_t a = s[k], b = s[partner];
          if ((a > b) == up) {
            s[k] = b;
            s[partner] = a;
          }
        }
      }
      __syncwarp();
    }
  }
  for (int k = lane; k < len; k += 32) col[b0 + k] = s[k];
}

// Block-wide variant for long rows (up to 16384 entries, dynamic shared memory).
__global__ void __launch_bounds__(512) k_sort_long_rows(const int64_t* __restrict__ rows_list, int nrows,
                                                        const int64_t* __restrict__ row, int32_t* __restrict__ col) {
  extern __shared__ int32_t s[];
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int64_t i = rows_list[r];
    const int64_t b0 = row[i];
    const int len = (int)(row[i + 1] - b0);
    int p2 = 1;
    while (p2 < len) p2 <<= 1;
    for (int k = threadIdx.x; k < p2; k += blockDim.x) s[k] = k < len ? col[b0 + k] : INT_MAX;
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int k = threadIdx.x; k < p2; k += blockDim.x) {
          const int partner = k ^ stride;
          if (partner > k) {
            const bool up = (k & size) == 0;
            const int32_t a = s[k], b = s[partner];
            if ((a > b) == up) {
              s[k] = b;
              s[partner] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    for (int k = threadIdx.x; k < len; k += blockDim.x) col[b0 + k] = s[k];
    __syncthreads();
  }
}

// Flags bonds i->j whose reverse j->i is absent (binary search, rows sorted),
// and records the longest row.
__global__ void k_check_rows(int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col,
                             int* __restrict__ flags) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t b0 = row[i], b1 = row[i + 1];
  if (lane == 0) atomicMax(&flags[1], (int)(b1 - b0));
  for (int64_t b = b0 + lane; b < b1; b += 32) {
    const int32_t j = col[b];
    if (j < 0 || j >= n) {
      atomicOr(&flags[0], 2);
      continue;
    }
    if (b > b0 && col[b - 1] >= j) atomicOr(&flags[0], 4);  // not strictly ascending
    int64_t lo = row[j], hi = row[j + 1];
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (col[mid] < (int32_t)i) lo = mid + 1;
      else hi = mid;
    }
    if (!(lo < row[j + 1] && col[lo] == (int32_t)i)) atomicOr(&flags[0], 1);
  }
}

static int sort_and_check_rows(pd_ctx* c, bool sort_rows) {
  if (c->n == 0) return PD_OK;
  // short rows: warp bitonic in static shared memory
  if (sort_rows) {
    k_sort_rows<1024><<<(unsigned)((c->n + 3) / 4), 128, 0, c->stream>>>(c->n, c->row.p, c->col.p);
    PD_CUDA_TRY(c, cudaGetLastError());
  }
  DBuf<int> flags;
  PD_CUDA_TRY(c, flags.alloc(2));
  PD_CUDA_TRY(c, cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), c->stream));
  k_check_rows<<<(unsigned)((c->n * 32 + 255) / 256), 256, 0, c->stream>>>(c->n, c->row.p, c->col.p, flags.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  int hf[2];
  PD_CUDA_TRY(c, cudaMemcpyAsync(hf, flags.p, sizeof(hf), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->max_row = hf[1];
  if (hf[0] & 2) {
    c->err = "neighbor list holds an index outside [0, n)";
    return PD_ERR_ARG;
  }
  if (sort_rows && c->max_row > 1024) {
    if (c->max_row > 16384) {
      c->err = "a bond family longer than 16384 neighbors is not supported";
      return PD_ERR_UNSUPPORTED;
    }
    // long rows: block-wide sort over the list of long rows
    std::vector<int64_t> hrow(c->n + 1);
    PD_CUDA_TRY(c, d2h(c, hrow.data(), c->row.p, (c->n + 1) * sizeof(int64_t)));
    std::vector<int64_t> longs;
    for (int64_t i = 0; i < c->n; ++i)
      if (hrow[i + 1] - hrow[i] > 1024) longs.push_back(i);
    DBuf<int64_t> dl;
    PD_CUDA_TRY(c, dl.alloc(longs.size()));
    PD_CUDA_TRY(c, h2d(c, dl.p, longs.data(), longs.size() * sizeof(int64_t)));
    PD_CUDA_TRY(c, cudaFuncSetAttribute(k_sort_long_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 16384 * 4));
    k_sort_long_rows<<<(unsigned)std::min<size_t>(longs.size(), 1024), 512, 16384 * 4, c->stream>>>(
        dl.p, (int)longs.size(), c->row.p, c->col.p);
    PD_CUDA_TRY(c, cudaGetLastError());
    PD_CUDA_TRY(c, cudaMemsetAsync(flags.p, 0, 2 * sizeof(int), c->stream));
    k_check_rows<<<(unsigned)((c->n * 32 + 255) / 256), 256, 0, c->stream>>>(c->n, c->row.p, c->col.p, flags.p);
    PD_CUDA_TRY(c, cudaMemcpyAsync(hf, flags.p, sizeof(hf), cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  c->symmetric = (hf[0] & 1) == 0;
  if (hf[0] & 4) {
    c->err = "each family of the neighbor list must be strictly ascending (as NeighborhoodList builds it)";
    return PD_ERR_ARG;
  }
  return PD_OK;
}

// Families with j in H(i) but i not in H(j): the reference builds each
// point's family with its own block's horizon (NeighborhoodList.cxx:382-389,
// Peridigm_HorizonManager.cpp:71-77) and scatters both halves of each of its
// own bonds, so the force on i holds t_ij for j in H(i) and t_ji for j with i
// in H(j). The gather passes read both halves from row i, so the missing
// reverse (j, i) joins row j as a phantom: its own half marked absent (bit 0
// and kPhantomOwn), and (i, j) marked without a partner half (bit 1 and
// kPhantomPartner). Rows stay strictly ascending (merge of two ascending
// lists); the caller's families are recorded in h_orig for the outputs.
static int symmetrize_bonds(pd_ctx* c) {
  const int64_t n = c->n, nb = c->nb;
  std::vector<int64_t> row(n + 1);
  std::vector<int32_t> col((size_t)std::max<int64_t>(nb, 1));
  PD_CUDA_TRY(c, d2h(c, row.data(), c->row.p, (n + 1) * sizeof(int64_t)));
  if (nb) PD_CUDA_TRY(c, d2h(c, col.data(), c->col.p, nb * sizeof(int32_t)));
  auto has = [&](int64_t i, int32_t j) {  // j in row i (ascending)
    const int32_t* b = col.data() + row[i];
    const int32_t* e = col.data() + row[i + 1];
    const int32_t* p = std::lower_bound(b, e, j);
    return p != e && *p == j;
  };
  std::vector<uint8_t> norev((size_t)std::max<int64_t>(nb, 1), 0);
  std::vector<int64_t> extra(n + 1, 0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t b = row[i]; b < row[i + 1]; ++b)
      if (!has(col[b], (int32_t)i)) {
        norev[b] = 1;
        extra[col[b] + 1]++;
      }
  for (int64_t i = 0; i < n; ++i) extra[i + 1] += extra[i];  // phantom offsets per row
  std::vector<int32_t> ph((size_t)std::max<int64_t>(extra[n], 1));
  {
    std::vector<int64_t> cur(extra.begin(), extra.end() - 1);
    for (int64_t i = 0; i < n; ++i)  // ascending i: each row's phantoms come out ascending
      for (int64_t b = row[i]; b < row[i + 1]; ++b)
        if (norev[b]) ph[cur[col[b]]++] = (int32_t)i;
  }
  const int64_t nbs = nb + extra[n];
  std::vector<int64_t> nrow(n + 1, 0);
  std::vector<int32_t> ncol((size_t)std::max<int64_t>(nbs, 1));
  c->h_orig.assign((size_t)nbs, 0);
  c->h_dmg0.assign((size_t)nbs, 0);
  c->h_nph.assign(n, 0);
  int64_t k = 0;
  for (int64_t i = 0; i < n; ++i) {
    nrow[i] = k;
    int64_t a = row[i], p = extra[i];
    const int64_t ae = row[i + 1], pe = extra[i + 1];
    c->h_nph[i] = (int32_t)(pe - p);
    while (a < ae || p < pe) {
      if (p >= pe || (a < ae && col[a] < ph[p])) {
        ncol[k] = col[a];
        c->h_orig[k] = 1;
        c->h_dmg0[k] = norev[a] ? (uint8_t)(2 | kPhantomPartner) : 0;
        ++a;
      } else {
        ncol[k] = ph[p];
        c->h_dmg0[k] = (uint8_t)(1 | kPhantomOwn);
        ++p;
      }
      ++k;
    }
  }
  nrow[n] = k;
  c->row.release();
  c->col.release();
  PD_CUDA_TRY(c, c->row.alloc(n + 1));
  PD_CUDA_TRY(c, c->col.alloc((size_t)std::max<int64_t>(nbs, 1)));
  PD_CUDA_TRY(c, h2d(c, c->row.p, nrow.data(), (n + 1) * sizeof(int64_t)));
  if (nbs) PD_CUDA_TRY(c, h2d(c, c->col.p, ncol.data(), nbs * sizeof(int32_t)));
  int mx = 0;
  for (int64_t i = 0; i < n; ++i) mx = std::max<int>(mx, (int)(nrow[i + 1] - nrow[i]));
  c->max_row = mx;
  c->nb_user = nb;
  c->nb = nbs;
  c->phantoms = true;
  c->symmetric = true;
  return PD_OK;
}

int finalize_bonds(pd_ctx* c, bool sort_rows) {
  int rc = sort_and_check_rows(c, sort_rows);
  if (rc != PD_OK) return rc;
  c->phantoms = false;
  c->nb_user = c->nb;
  c->h_orig.clear();
  c->h_nph.clear();
  c->h_dmg0.clear();
  if (!c->symmetric) {
    rc = symmetrize_bonds(c);
    if (rc != PD_OK) return rc;
  }
  PD_CUDA_TRY(c, c->dmg.alloc((size_t)c->nb));
  PD_CUDA_TRY(c, c->dmg_trial.alloc((size_t)c->nb));
  PD_CUDA_TRY(c, cudaMemsetAsync(c->dmg.p, 0, c->dmg.bytes(), c->stream));
  if (c->phantoms && c->nb) PD_CUDA_TRY(c, h2d(c, c->dmg.p, c->h_dmg0.data(), (size_t)c->nb));
  c->dmg_gen++;
  c->dmg_asym = c->phantoms;  // the two halves differ along every phantom bond
  c->chunk_hi_nb = -1;  // the upload chunks' neighbor bounds follow the bond set
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->trial_valid = false;
  c->wv_done = false;
  return PD_OK;
}

Grid make_grid(int64_t n, const double lo[3], const double hi[3], double reach) {
  Grid g;
  double cell = reach * 1.0001;
  if (!(cell > 0.0)) cell = 1.0;
  for (;;) {
    double tot = 1.0;
    for (int k = 0; k < 3; ++k) {
      g.dims[k] = (int)std::floor((hi[k] - lo[k]) / cell) + 1;
      tot *= g.dims[k];
    }
    if (tot <= 4.0 * (double)n + 64.0 && tot < 2.0e9) break;
    cell *= 1.5;
  }
  for (int k = 0; k < 3; ++k) g.lo[k] = lo[k];
  g.cell = cell;
  return g;
}

int bin_points(pd_ctx* c, const double4* pos, int64_t n, const Grid& g, DBuf<int32_t>& idx_s,
               DBuf<int64_t>& cell_start, BinScratch* scratch) {
  const int64_t ncell = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
  BinScratch local;
  BinScratch& S = scratch ? *scratch : local;
  if (scratch) {
    PD_CUDA_TRY(c, S.cid.reserve(n));
    PD_CUDA_TRY(c, S.idx.reserve(n));
    PD_CUDA_TRY(c, S.cid_s.reserve(n));
    PD_CUDA_TRY(c, idx_s.reserve(n));
    PD_CUDA_TRY(c, cell_start.reserve(ncell + 1));
  } else {
    PD_CUDA_TRY(c, S.cid.alloc(n));
    PD_CUDA_TRY(c, S.idx.alloc(n));
    PD_CUDA_TRY(c, S.cid_s.alloc(n));
    PD_CUDA_TRY(c, idx_s.alloc(n));
    PD_CUDA_TRY(c, cell_start.alloc(ncell + 1));
  }
  const unsigned g1 = (unsigned)((n + 255) / 256);
  k_cell_ids<<<g1, 256, 0, c->stream>>>(n, pos, g, S.cid.p, S.idx.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  int end_bit = 1;
  while (end_bit < 31 && (int64_t(1) << end_bit) <= ncell) ++end_bit;
  size_t tmp_bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, S.cid.p, S.cid_s.p, S.idx.p, idx_s.p, (int)n, 0, end_bit,
                                  c->stream);
  if (scratch) PD_CUDA_TRY(c, S.tmp.reserve(tmp_bytes));
  else PD_CUDA_TRY(c, S.tmp.alloc(tmp_bytes));
  tmp_bytes = S.tmp.count;
  PD_CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(S.tmp.p, tmp_bytes, S.cid.p, S.cid_s.p, S.idx.p, idx_s.p, (int)n, 0,
                                                 end_bit, c->stream));
  k_cell_bounds<<<(unsigned)((n + 1 + 255) / 256), 256, 0, c->stream>>>(n, ncell, S.cid_s.p, cell_start.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

int build_bonds_device(pd_ctx* c, const pd_plane_filter* filters, int nf) {
  const int64_t n = c->n;
  if (nf < 0 || nf > kMaxPlanes) {
    c->err = "at most 16 plane filters are supported";
    return PD_ERR_ARG;
  }
  Planes pl;
  pl.count = nf;
  for (int f = 0; f < nf; ++f) {
    PlaneDev& P = pl.p[f];
    for (int k = 0; k < 3; ++k) {
      P.n[k] = filters[f].normal[k];
      P.r0[k] = filters[f].lower_left[k];
      P.ub[k] = filters[f].bottom_unit[k];
    }
    // ua = cross(ub, n) in UTILITIES::Cross's component order (Vector3D.h:119-128)
    P.ua[0] = -P.ub[2] * P.n[1] + P.ub[1] * P.n[2];
    P.ua[1] = P.ub[2] * P.n[0] - P.ub[0] * P.n[2];
    P.ua[2] = -P.ub[1] * P.n[0] + P.ub[0] * P.n[1];
    P.a = filters[f].side_length;
    P.b = filters[f].bottom_length;
  }
  // grid over the bounding box, cell side >= the largest horizon
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], c->hx[3 * i + k]);
      hi[k] = std::max(hi[k], c->hx[3 * i + k]);
    }
  double hmax = 0.0;
  for (double h : c->block_h) hmax = std::max(hmax, h);
  if (!(hmax > 0.0)) {
    c->err = "horizon must be positive";
    return PD_ERR_ARG;
  }
  const Grid g = make_grid(n, lo, hi, hmax);
  DBuf<int32_t> idx_s;
  DBuf<int64_t> cell_start, counts;
  {
    int rc = bin_points(c, c->xv.p, n, g, idx_s, cell_start);
    if (rc != PD_OK) return rc;
  }
  PD_CUDA_TRY(c, counts.alloc(n + 1));
  const unsigned gw = (unsigned)((n * 32 + 255) / 256);
  k_neighbors<false><<<gw, 256, 0, c->stream>>>(n, c->xv.p, c->hp.p, g, cell_start.p, idx_s.p, pl, counts.p, nullptr,
                                                nullptr);
  PD_CUDA_TRY(c, cudaGetLastError());
  PD_CUDA_TRY(c, c->row.alloc(n + 1));
  PD_CUDA_TRY(c, cudaMemsetAsync(counts.p + n, 0, sizeof(int64_t), c->stream));
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts.p, c->row.p, (int)(n + 1), c->stream);
  DBuf<unsigned char> stmp;
  PD_CUDA_TRY(c, stmp.alloc(scan_bytes));
  PD_CUDA_TRY(c, cub::DeviceScan::ExclusiveSum(stmp.p, scan_bytes, counts.p, c->row.p, (int)(n + 1), c->stream));
  int64_t nb = 0;
  PD_CUDA_TRY(c, cudaMemcpyAsync(&nb, c->row.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->nb = nb;
  PD_CUDA_TRY(c, c->col.alloc((size_t)nb));
  k_neighbors<true><<<gw, 256, 0, c->stream>>>(n, c->xv.p, c->hp.p, g, cell_start.p, idx_s.p, pl, nullptr, c->row.p,
                                               c->col.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return finalize_bonds(c, true);
}

}  // namespace pdb
