// Aggregate coarse space of the quasi-static CG preconditioners (sm_100a).
// No counterpart in the reference (Peridigm's CG is unpreconditioned or block
// Jacobi, src/core/Peridigm.cpp:2740, 1603-1646); it is the coarse level of the
// two-level and learned preconditioners:
//
//   z = P_bj r + P0 Ac^-1 P0^T r  (+ the network's correction, k_mpnn.cu)
//
// P0: piecewise-constant translations on aggregates = the non-empty cells of a
// grid of side >= 2 * max horizon (3 coarse dofs per aggregate, prescribed dofs
// excluded). Ac = P0^T K P0 is the exact Galerkin product with the tangent K of
// k_qs.cu, assembled from the bonds without forming K:
//
//   K w|_i = -V_i [ sum_j V_j B_ij (w_j - w_i) + q_i dth_i H_i + sum_j h_ij q_j dth_j ]
//   B_ij = om (a_i + a_j) Yh Yh^T + (T_ij / |Y|) (I - Yh Yh^T)
//   h_ij = V_j om zeta Yh,  H_i = sum_j h_ij,  dth_i = sum_j g_ij . (w_j - w_i),
//   g_ij = 3 om zeta V_j Yh / m_i
//
// (om = omega(zeta, horizon of the bond's owner), a = alpha, q = 3K/m - alpha/3,
// T_ij the force-state sum of k_qs_bond_geom). The pair term couples each point to its
// bonds; the dilatation term is a sum of rank-one terms, one per point p,
// (force response to dth_p) x (dth_p as a function of w). A family of radius
// delta spans at most 2 cells per axis of a grid of side >= 2 delta, so every
// point's contributions fall in 8 "slots" (the 2x2x2 cells from the cell of
// x_p - delta); k_coarse_point sums them per slot, k_coarse_rows adds them into
// the dense Ac one aggregate row per warp in a fixed order (deterministic, no
// atomics). Ac is inverted in place by blocked Gauss-Jordan (SPD, no pivoting)
// and applied as a dense matrix-vector product. Bond damage is taken as
// symmetric (d_ij = d_ji), as the critical-stretch law produces it.
//
// Rigid coarse space (6 modes per aggregate, pd_qs_coarse_modes): the three
// translations and the three rotations about the aggregate's center (scaled
// by 1/side), prescribed dofs masked, orthonormalised per aggregate through
// the Cholesky factor of their 6x6 Gram matrix (modes whose pivot falls
// below 1e-8 of the largest diagonal entry are dropped: identity rows). Ac is
// assembled by colored probing: aggregates colored by their cell coordinates
// mod 3 per axis (27 colors) have disjoint 3x3x3 cell neighborhoods, and K
// couples points at most 2 delta <= one cell apart, so one tangent product
// per (color, mode) gives the columns of every aggregate of that color; each
// aggregate row reads its one neighbor of that color. The 6 modes of a color
// go through one multi-vector tangent pass (27 per build), deterministic, no
// atomics.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cells.cuh"
#include "pd_internal.cuh"

namespace pdb {

constexpr int kSlots = 8;
constexpr int kSlotVals = 15;  // pair 3x3 (9), force response a (3), dtheta functional b (3)
constexpr int kGjB = 64;       // Gauss-Jordan block
constexpr int kMaxCoarse = 6144;

struct CoarseState {
  int modes = 3;           // coarse dofs per aggregate: 3 translations, or 6 with the rotations
  bool built = false;      // aggregates
  bool have_op = false;    // Ac^-1 ready
  double cell = 0.0;
  Grid g;
  int64_t n = 0, nagg = 0;
  int nc = 0;
  DBuf<int32_t> sorted, agg_of, cell_agg, agg_cell, clo;
  DBuf<int64_t> cstart;
  DBuf<double> slots;      // [n][8][15]
  DBuf<double> A;          // nc x nc, the inverse after coarse_build
  DBuf<float> Af;          // its FP32 copy, the one each CG iteration reads
  DBuf<double> P, R, C;    // Gauss-Jordan work: pivot inverse, row panel, column panel (transposed)
  DBuf<double> D;          // the next pivot block, updated ahead of the trailing update
  cudaStream_t aux = nullptr;  // the next pivot's inverse, beside the trailing update
  cudaEvent_t e_diag = nullptr, e_piv = nullptr;
  DBuf<double> rc, zc;
  DBuf<int> status;
  DBuf<double> center, T;   // rigid modes: aggregate centers [4 nagg], orthonormalising transforms [36 nagg]
  DBuf<double> probe, kprobe, pdth;  // rigid modes: 6 probes, their tangent images [18n], scratch [6n]
  ~CoarseState() {
    if (e_diag) cudaEventDestroy(e_diag);
    if (e_piv) cudaEventDestroy(e_piv);
    if (aux) cudaStreamDestroy(aux);
  }
};

__device__ __forceinline__ double co_omega(int kind, double zeta, double h) {
  if (kind == PD_INFLUENCE_ONE) return 1.0;
  if (kind == PD_INFLUENCE_PARABOLIC_DECAY) {
    if (zeta > h) return 0.0;
    const double s = zeta / h;
    return s < 0.5 ? 1.0 : -4.0 * s * s + 4.0 * s;
  }
  return exp(-(zeta * zeta) / (h * h * 0.16));
}

__device__ __forceinline__ int slot_of(const Grid& g, const int lo[3], const double4& x, int* bad) {
  const int dx = cell_coord(g, x.x, 0) - lo[0], dy = cell_coord(g, x.y, 1) - lo[1], dz = cell_coord(g, x.z, 2) - lo[2];
  if ((unsigned)dx > 1u || (unsigned)dy > 1u || (unsigned)dz > 1u) {
    *bad = 1;
    return -1;
  }
  return dx + 2 * dy + 4 * dz;
}

// Per point p: slot sums of the pair rows of p, and of p's dilatation
// rank-one term (a: rows, b: columns), prescribed dofs masked.
__global__ void __launch_bounds__(128) k_coarse_point(int64_t n, const int64_t* __restrict__ row,
                                                      const int32_t* __restrict__ col,
                                                      const uint8_t* __restrict__ dmg,
                                                      const double4* __restrict__ xv, const double4* __restrict__ y,
                                                      const double4* __restrict__ ab, const double4* __restrict__ pt,
                                                      const double* __restrict__ hp, int influence,
                                                      const uint8_t* __restrict__ fixed, Grid g,
                                                      int32_t* __restrict__ clo_out, double* __restrict__ out,
                                                      int* __restrict__ status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[kSlots][kSlotVals];
#pragma unroll
  for (int s = 0; s < kSlots; ++s)
#pragma unroll
    for (int k = 0; k < kSlotVals; ++k) acc[s][k] = 0.0;
  const double4 xi = xv[i], yi = y[i], ai = ab[i];
  const double hi = hp[i], mi = pt[i].x, Vi = xi.w, qi = ai.y;
  const uint8_t fi = fixed[i];
  // slots: cells lo .. lo+1 per axis from the cell of x_i - reach
  const double reach = hi * (1.0 + 1.0e-9);
  int lo[3] = {cell_coord(g, xi.x - reach, 0), cell_coord(g, xi.y - reach, 1), cell_coord(g, xi.z - reach, 2)};
  int bad = 0;
  const int si = slot_of(g, lo, xi, &bad);
  for (int64_t b = row[i]; b < row[i + 1] && !bad; ++b) {
    if (dmg[b]) continue;
    const int32_t j = col[b];
    const double4 xj = xv[j], yj = y[j], aj = ab[j];
    const double hj = hp[j], Vj = xj.w;
    const uint8_t fj = fixed[j];
    const int sj = slot_of(g, lo, xj, &bad);
    if (bad) break;
    const double X0 = xj.x - xi.x, X1 = xj.y - xi.y, X2 = xj.z - xi.z;
    const double Y0 = yj.x - yi.x, Y1 = yj.y - yi.y, Y2 = yj.z - yi.z;
    const double zeta = sqrt(X0 * X0 + X1 * X1 + X2 * X2);
    const double dY = sqrt(Y0 * Y0 + Y1 * Y1 + Y2 * Y2);
    const double e = dY - zeta;
    const double yh[3] = {Y0 / dY, Y1 / dY, Y2 / dY};
    const double omi = co_omega(influence, zeta, hi), omj = co_omega(influence, zeta, hj);
    const double T = omi * (zeta * (ai.x * ai.y + aj.x * aj.y) + (ai.z + aj.z) * e);
    const double tg = T / dY, ax = omi * (ai.z + aj.z) - tg;
    const double vv = Vi * Vj;
    const double gs = 3.0 * omi * zeta * Vj / mi;            // g_ij = gs * yh
    const double ri = -Vi * qi * Vj * omi * zeta;            // row i of the dth_i response
    const double rj = Vj * Vi * omj * zeta * qi;             // row j of the dth_i response
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const bool ci = !((fi >> c) & 1), cj = !((fj >> c) & 1);
      if (ci) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double w = vv * (ax * yh[c] * yh[d] + (c == d ? tg : 0.0));
          if (!((fj >> d) & 1)) acc[sj][3 * c + d] -= w;
          if (!((fi >> d) & 1)) acc[si][3 * c + d] += w;
        }
        acc[si][9 + c] += ri * yh[c];
      }
      if (cj) acc[sj][9 + c] += rj * yh[c];
      if (cj) acc[sj][12 + c] += gs * yh[c];
      if (ci) acc[si][12 + c] -= gs * yh[c];
    }
  }
  if (bad) atomicOr(status, ST_BAD_INDEX);
  clo_out[4 * i] = lo[0];
  clo_out[4 * i + 1] = lo[1];
  clo_out[4 * i + 2] = lo[2];
  clo_out[4 * i + 3] = si;
  double* o = out + (size_t)i * kSlots * kSlotVals;
#pragma unroll
  for (int s = 0; s < kSlots; ++s)
#pragma unroll
    for (int k = 0; k < kSlotVals; ++k) o[s * kSlotVals + k] = acc[s][k];
}

// One warp per aggregate row I: Ac[I, J] for the 5x5x5 cells J around I,
// accumulated in shared memory over the points of the 3x3x3 cells around I in
// cell order (each lane owns fixed (slot, entry) items: deterministic).
constexpr int kRowWarps = 4;
__global__ void __launch_bounds__(32 * kRowWarps) k_coarse_rows(int64_t nagg, int nc, Grid g,
                                                                 const int32_t* __restrict__ agg_cell,
                                                                 const int32_t* __restrict__ cell_agg,
                                                                 const int64_t* __restrict__ cstart,
                                                                 const int32_t* __restrict__ sorted,
                                                                 const int32_t* __restrict__ clo,
                                                                 const double* __restrict__ slots,
                                                                 double* __restrict__ A) {
  __shared__ double acc[kRowWarps][125 * 9];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t I = (int64_t)blockIdx.x * kRowWarps + w;
  if (I >= nagg) return;
  double* s = acc[w];
  for (int k = lane; k < 125 * 9; k += 32) s[k] = 0.0;
  __syncwarp();
  const int cell = agg_cell[I];
  const int cx = cell % g.dims[0], cy = (cell / g.dims[0]) % g.dims[1], cz = cell / (g.dims[0] * g.dims[1]);
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int qx = cx + dx, qy = cy + dy, qz = cz + dz;
        if (qx < 0 || qy < 0 || qz < 0 || qx >= g.dims[0] || qy >= g.dims[1] || qz >= g.dims[2]) continue;
        const int q = (qz * g.dims[1] + qy) * g.dims[0] + qx;
        const bool own_cell = (dx == 0 && dy == 0 && dz == 0);
        for (int64_t t = cstart[q]; t < cstart[q + 1]; ++t) {
          const int32_t p = sorted[t];
          const int lx = clo[4 * p], ly = clo[4 * p + 1], lz = clo[4 * p + 2];
          const int ox = cx - lx, oy = cy - ly, oz = cz - lz;
          if ((unsigned)ox > 1u || (unsigned)oy > 1u || (unsigned)oz > 1u) continue;
          const double* sp = slots + (size_t)p * kSlots * kSlotVals;
          const int srow = ox + 2 * oy + 4 * oz;
          const double a0 = sp[srow * kSlotVals + 9], a1 = sp[srow * kSlotVals + 10], a2 = sp[srow * kSlotVals + 11];
          for (int it = lane; it < kSlots * 9; it += 32) {
            const int sl = it / 9, cd = it - 9 * sl, c = cd / 3, d = cd - 3 * c;
            const int jx = lx + (sl & 1) - cx + 2, jy = ly + ((sl >> 1) & 1) - cy + 2, jz = lz + (sl >> 2) - cz + 2;
            const double av = c == 0 ? a0 : (c == 1 ? a1 : a2);
            double v = av * sp[sl * kSlotVals + 12 + d];
            if (own_cell) v += sp[sl * kSlotVals + cd];
            s[((jz * 5 + jy) * 5 + jx) * 9 + cd] += v;
          }
          __syncwarp();
        }
      }
  // write the row block
  for (int jl = lane; jl < 125; jl += 32) {
    const int jx = cx + jl % 5 - 2, jy = cy + (jl / 5) % 5 - 2, jz = cz + jl / 25 - 2;
    if (jx < 0 || jy < 0 || jz < 0 || jx >= g.dims[0] || jy >= g.dims[1] || jz >= g.dims[2]) continue;
    const int J = cell_agg[(jz * g.dims[1] + jy) * g.dims[0] + jx];
    if (J < 0) continue;
    for (int cd = 0; cd < 9; ++cd)
      A[(size_t)(3 * I + cd / 3) * nc + 3 * J + cd % 3] = s[jl * 9 + cd];
  }
}

// Coarse dofs with no free fine dof: identity rows.
__global__ void k_coarse_unit_diag(int nc, double* __restrict__ A) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nc && A[(size_t)k * nc + k] == 0.0) A[(size_t)k * nc + k] = 1.0;
}

// aggregate id per cell (-1: empty) and cell of each aggregate, in cell order
__global__ void k_coarse_cells(int64_t ncell, const int64_t* __restrict__ cstart, int32_t* __restrict__ cell_agg,
                               int32_t* __restrict__ agg_cell, int64_t* __restrict__ nagg_out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int32_t k = 0;
  for (int64_t q = 0; q < ncell; ++q) {
    if (cstart[q + 1] > cstart[q]) {
      cell_agg[q] = k;
      agg_cell[k] = (int32_t)q;
      ++k;
    } else {
      cell_agg[q] = -1;
    }
  }
  *nagg_out = k;
}

__global__ void k_coarse_agg_of(int64_t n, const double4* __restrict__ xv, Grid g, const int32_t* __restrict__ cell_agg,
                                int32_t* __restrict__ agg_of) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = xv[i];
  agg_of[i] = cell_agg[(cell_coord(g, p.z, 2) * g.dims[1] + cell_coord(g, p.y, 1)) * g.dims[0] + cell_coord(g, p.x, 0)];
}

// ---------------------------------------------------------------------------
// Dense SPD inverse: blocked in-place Gauss-Jordan (no pivoting), 64-wide steps
//   P = A_kk^-1; R = P A_k* (new block row); C = A_*k (old block column);
//   A_ij -= C_i R_j (i, j outside block k); A_kj = R_j; A_ik = -C_i P; A_kk = P
// With P written into R's block-k columns, every row outside block k takes
// A_ij = [j outside block k] A_ij - C_i R_j, and the rows of block k take R.
// The matrix stays sign-symmetric under these sweeps: A_ba = -A_ab when
// exactly one of a, b lies in a block already swept, A_ba = A_ab otherwise.
// So only the 128 x 128 tiles on and above the diagonal are updated (the
// diagonal tiles whole); the panel reads the true block row and column from
// where they are kept, and the entries below the diagonal are mirrored from
// those above once every block is swept (the inverse is symmetric).
// ---------------------------------------------------------------------------
constexpr int kUT = 128, kUK = 16;  // update tile side, k chunk of the staged panels
// P = inverse of a bk x bk diagonal block (src, leading dimension ld; one
// block of 256 threads; each elimination step reads the old row and column
// k, then writes: two barriers a step).
__global__ void __launch_bounds__(256) k_gj_pivot(const double* __restrict__ src, int ld, int bk,
                                                  double* __restrict__ P) {
  __shared__ double S[kGjB][kGjB + 1];
  constexpr int kPer = kGjB * kGjB / 256;
  static_assert(kPer * 256 == kGjB * kGjB, "launched with 256 threads");
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int r = t / kGjB, c = t % kGjB;
    S[r][c] = (r < bk && c < bk) ? src[(size_t)r * ld + c] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < bk; ++k) {
    const double p = 1.0 / S[k][k];
    double nv[kPer];
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int t = threadIdx.x + 256 * q, r = t / kGjB, c = t % kGjB;
      double v = S[r][c];
      if (r < bk && c < bk) {
        if (r == k) {
          v = (c == k) ? p : S[k][c] * p;
        } else if (c == k) {
          v = -S[r][k] * p;
        } else {
          const double nkc = S[k][c] * p;  // the new row k
          v = S[r][c] - S[r][k] * nkc;
        }
      }
      nv[q] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int t = threadIdx.x + 256 * q;
      S[t / kGjB][t % kGjB] = nv[q];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < bk * bk; t += blockDim.x) P[t] = S[t / bk][t % bk];
}

// Row panel of block k: W = the true block row A_k* (A[k0+t][j] where column
// j's tile is at or right of block k's, else -A[j][k0+t], transposed through
// shared memory), R = P W with P itself in the block-k columns, and
// Ct = s W (s_j = -1 for j < k0, the swept columns): the true old block
// column A_*k, transposed. One block per 64 columns (which share a tile).
constexpr size_t kPanelSmem = 2 * sizeof(double[kGjB][kGjB + 1]);  // 65 KiB: dynamic
__global__ void __launch_bounds__(256) k_gj_panel(int nc, int k0, int bk, const double* __restrict__ A,
                                                  const double* __restrict__ P, double* __restrict__ R,
                                                  double* __restrict__ Ct) {
  extern __shared__ __align__(16) double psm[];
  double(*sW)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(psm);
  double(*sP)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(psm + kGjB * (kGjB + 1));
  static_assert(kUT % kGjB == 0, "a block's 64 columns lie in one update tile");
  const int j0 = blockIdx.x * kGjB;
  const bool row_kept = j0 / kUT >= k0 / kUT;
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int r = t / kGjB, c = t % kGjB;
    if (row_kept)
      sW[r][c] = (r < bk && j0 + c < nc) ? A[(size_t)(k0 + r) * nc + j0 + c] : 0.0;
    else
      sW[c][r] = (j0 + r < nc && c < bk) ? -A[(size_t)(j0 + r) * nc + k0 + c] : 0.0;
    sP[r][c] = (r < bk && c < bk) ? P[r * bk + c] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int r = t / kGjB, c = t % kGjB, j = j0 + c;
    if (r >= bk || j >= nc) continue;
    const double w = sW[r][c];
    Ct[(size_t)r * nc + j] = j < k0 ? -w : w;
    double v;
    if (j >= k0 && j < k0 + bk) {
      v = sP[r][j - k0];
    } else {
      v = 0.0;
      for (int k = 0; k < bk; ++k) v = fma(sP[r][k], sW[k][c], v);
    }
    R[(size_t)r * nc + j] = v;
  }
}

// The diagonal block of the next step (rows and columns k1..k1+bk1) as the
// trailing update of block k will leave it, A_ij - sum_t Ct[t][i] R[t][j]
// (sum over t in order), into D (bk1 x bk1): read before that update runs,
// so the next pivot can run beside it. The update still writes the block in
// place, but the next step replaces it with P before anything reads it.
__global__ void __launch_bounds__(256) k_gj_next_diag(int nc, int k1, int bk1, int bk, const double* __restrict__ A,
                                                      const double* __restrict__ R, const double* __restrict__ Ct,
                                                      double* __restrict__ D) {
  extern __shared__ __align__(16) double psm[];
  double(*sC)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(psm);                      // sC[t][r]
  double(*sR)[kGjB + 1] = reinterpret_cast<double(*)[kGjB + 1]>(psm + kGjB * (kGjB + 1));  // sR[t][c]
  for (int e = threadIdx.x; e < kGjB * kGjB; e += blockDim.x) {
    const int t = e / kGjB, x = e % kGjB;
    const bool in = t < bk && x < bk1;
    sC[t][x] = in ? Ct[(size_t)t * nc + k1 + x] : 0.0;
    sR[t][x] = in ? R[(size_t)t * nc + k1 + x] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // rows ty + 16a, columns tx + 16b
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int t = 0; t < bk; ++t) {
    double cv[4], rv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) cv[a] = sC[t][ty + 16 * a];
#pragma unroll
    for (int b = 0; b < 4; ++b) rv[b] = sR[t][tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(cv[a], rv[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int r = ty + 16 * a, cc = tx + 16 * b;
      if (r < bk1 && cc < bk1) D[r * bk1 + cc] = A[(size_t)(k1 + r) * nc + k1 + cc] - acc[a][b];
    }
}

// Entries below the diagonal from those above, once every block is swept:
// 64 x 64 blocks (rows bi, columns bj <= bi) transposed through shared memory.
__global__ void __launch_bounds__(256) k_gj_mirror(int nc, double* __restrict__ A) {
  __shared__ double sT[kGjB][kGjB + 1];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi) return;
  const int r0 = bi * kGjB, c0 = bj * kGjB;
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {  // sT[r][c] = A[c0 + r][r0 + c]
    const int r = t / kGjB, c = t % kGjB;
    sT[r][c] = (c0 + r < nc && r0 + c < nc) ? A[(size_t)(c0 + r) * nc + r0 + c] : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kGjB * kGjB; t += blockDim.x) {
    const int r = t / kGjB, c = t % kGjB, a = r0 + r, b = c0 + c;
    if (a < nc && b < nc && a > b) A[(size_t)a * nc + b] = sT[c][r];
  }
}

// Trailing update on the 128x128 tiles on and above the diagonal (block x =
// the upper-triangle tile pair, row-major) on the FP64 tensor cores:
// mma.sync m8n8k4 (D = A B + C in FP64), each warp a 32 x 32 region (4 x 4
// outputs of 8 x 8), one block of 16 warps per SM (16 warps cover the MMA
// latency that 8 warps with twice the outputs each left exposed). The two bk x nc panels come
// in k chunks of 16, double-buffered by cp.async (rows padded to kUP doubles
// so that a fragment load is two wavefronts); the block's A tile (read back
// for the final A - C R) follows the first chunk by cp.async and is first
// waited for with the second, so the first chunk's products overlap its load.
constexpr int kUP = kUT + 8;  // padded panel row (doubles)
constexpr size_t kUpdSmem = (size_t)(kUT * kUT + 4 * kUK * kUP) * sizeof(double);  // 196 KiB

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// d += a b for one 8 x 8 x 4 FP64 product: a = A[lane / 4][lane % 4],
// b = B[lane % 4][lane / 4], d = D[lane / 4][2 (lane % 4) + {0, 1}].
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

constexpr int kUpdT = 512;
__global__ void __launch_bounds__(kUpdT, 1) k_gj_update(int nc, int k0, int bk, double* __restrict__ A,
                                                        const double* __restrict__ R, const double* __restrict__ Ct) {
  extern __shared__ __align__(16) double smem[];
  double* sA = smem;                   // [kUT][kUT]
  double* sC = smem + kUT * kUT;       // [2][kUK][kUP]: Ct rows (k), tile rows i
  double* sR = sC + 2 * kUK * kUP;     // [2][kUK][kUP]: R rows (k), tile columns j
  int bj = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);  // tile pair L = bj (bj + 1) / 2 + bi, bi <= bj
  while ((bj + 1) * (bj + 2) / 2 <= (int)blockIdx.x) ++bj;
  while (bj * (bj + 1) / 2 > (int)blockIdx.x) --bj;
  const int bi = (int)blockIdx.x - bj * (bj + 1) / 2;
  const int i0 = bi * kUT, j0 = bj * kUT;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int wr = 32 * (w >> 2), wc = 32 * (w & 3);  // the warp's region: rows wr.., columns wc..
  auto stage = [&](int buf, int kc) {  // one group per chunk; zeros past the edges
#pragma unroll
    for (int q = 0; q < kUK * kUT / kUpdT; ++q) {
      const int t = threadIdx.x + kUpdT * q, k = t / kUT, x = t % kUT;
      double* dc = sC + (buf * kUK + k) * kUP + x;
      double* dr = sR + (buf * kUK + k) * kUP + x;
      const bool kin = kc + k < bk;
      if (kin && i0 + x < nc) cp_async8(dc, Ct + (size_t)(kc + k) * nc + i0 + x);
      else *dc = 0.0;
      if (kin && j0 + x < nc) cp_async8(dr, R + (size_t)(kc + k) * nc + j0 + x);
      else *dr = 0.0;
    }
    cp_async_commit();
  };
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  stage(0, 0);  // group 0
  for (int t = threadIdx.x; t < kUT * kUT; t += blockDim.x) {  // group 1: the A tile
    const int r = t / kUT, x = t % kUT;
    if (i0 + r < nc && j0 + x < nc) cp_async8(sA + t, A + (size_t)(i0 + r) * nc + j0 + x);
  }
  cp_async_commit();
  int buf = 0;
  for (int kc = 0; kc < bk; kc += kUK, buf ^= 1) {
    if (kc + kUK < bk) {
      stage(buf ^ 1, kc + kUK);
      if (kc == 0) cp_async_wait<2>();  // chunk 0; the A tile and chunk 1 may still land
      else cp_async_wait<1>();          // everything but the chunk just issued
    } else if (kc == 0) {
      cp_async_wait<1>();  // a single chunk: the A tile may still land
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* cb = sC + buf * kUK * kUP;
    const double* rb = sR + buf * kUK * kUP;
#pragma unroll
    for (int ks = 0; ks < kUK; ks += 4) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = cb[(ks + t4) * kUP + wr + 8 * a + g];  // A[i][k] = Ct[k][i]
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = rb[(ks + t4) * kUP + wc + 8 * b + g];  // B[k][j] = R[k][j]
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dmma(acc[a][b], av[a], bv[b]);
    }
    __syncthreads();  // the next iteration's stage overwrites this buffer
  }
  cp_async_wait<0>();  // the A tile
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int r = wr + 8 * a + g, i = i0 + r;
    if (i >= nc) continue;
    const bool rowk = i >= k0 && i < k0 + bk;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int x = wc + 8 * b + 2 * t4 + e, j = j0 + x;
        if (j >= nc) continue;
        double v;
        if (rowk) v = R[(size_t)(i - k0) * nc + j];
        else if (j >= k0 && j < k0 + bk) v = -acc[a][b][e];
        else v = sA[r * kUT + x] - acc[a][b][e];
        A[(size_t)i * nc + j] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Application: rc = P0^T r (block per aggregate), zc = Ac^-1 rc (warp per row,
// the FP32 copy of the inverse), z += P0 zc on free dofs
// ---------------------------------------------------------------------------
// Block sum of kRestrictT threads' partial sums, in a fixed order (thread 0
// gets the total): a tree over shared memory.
constexpr int kRestrictT = 128;
template <int K>
__device__ __forceinline__ void block_sum(double (&acc)[K], double (*sh)[kRestrictT]) {
  for (int k = 0; k < K; ++k) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = kRestrictT / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int k = 0; k < K; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + o];
    __syncthreads();
  }
  for (int k = 0; k < K; ++k) acc[k] = sh[k][0];
}

// rc_I = sum of r over the free dofs of aggregate I's points (a block of
// kRestrictT threads per aggregate: the points in flight at once, then one
// fixed-order block sum).
template <typename T>
__global__ void __launch_bounds__(kRestrictT) k_coarse_restrict(int64_t nagg, const int32_t* __restrict__ agg_cell,
                                                                const int64_t* __restrict__ cstart,
                                                                const int32_t* __restrict__ sorted,
                                                                const T* __restrict__ r, double* __restrict__ rc) {
  __shared__ double sh[3][kRestrictT];
  const int64_t I = blockIdx.x;
  const int q = agg_cell[I];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t t = cstart[q] + threadIdx.x; t < cstart[q + 1]; t += kRestrictT) {
    const int64_t p = sorted[t];
    acc[0] += (double)r[3 * p];
    acc[1] += (double)r[3 * p + 1];
    acc[2] += (double)r[3 * p + 2];
  }
  block_sum<3>(acc, sh);
  if (threadIdx.x == 0) rc[3 * I] = acc[0], rc[3 * I + 1] = acc[1], rc[3 * I + 2] = acc[2];
}

// y = A x with the FP32 copy of the inverse, FP64 products and sums (warp per
// row, four entries per lane per load: the row's order of terms is fixed).
__global__ void k_coarse_gemv_f(int nc, const float* __restrict__ A, const double* __restrict__ x,
                                double* __restrict__ y) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= nc) return;
  const float* a = A + (size_t)i * nc;
  double s = 0.0;
  const int n4 = (nc & 3) == 0 ? nc / 4 : 0;  // rows start 16-byte aligned when nc % 4 == 0
  const float4* a4 = reinterpret_cast<const float4*>(a);
  for (int k = lane; k < n4; k += 32) {
    const float4 v = a4[k];
    s = fma((double)v.x, x[4 * k], s);
    s = fma((double)v.y, x[4 * k + 1], s);
    s = fma((double)v.z, x[4 * k + 2], s);
    s = fma((double)v.w, x[4 * k + 3], s);
  }
  for (int k = 4 * n4 + lane; k < nc; k += 32) s = fma((double)a[k], x[k], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[i] = s;
}

__global__ void k_to_f32(int64_t m, const double* __restrict__ a, float* __restrict__ b) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) b[k] = (float)a[k];
}

__global__ void k_coarse_prolong(int64_t n, const int32_t* __restrict__ agg_of, const double* __restrict__ zc,
                                 double scale, const uint8_t* __restrict__ fixed, double* __restrict__ z) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t I = agg_of[i];
  const uint8_t f = fixed[i];
  for (int c = 0; c < 3; ++c)
    if (!((f >> c) & 1)) z[3 * i + c] += scale * zc[3 * I + c];
}

// ---------------------------------------------------------------------------
// Rigid coarse space (6 modes per aggregate)
// ---------------------------------------------------------------------------
// Component c of raw mode k at offset d from the center (scaled by 1/side).
__device__ __forceinline__ double rigid_raw(const double d[3], double inv_side, int c, int k) {
  switch (k) {
    case 0: case 1: case 2: return c == k ? 1.0 : 0.0;
    case 3: return c == 0 ? -d[1] * inv_side : (c == 1 ? d[0] * inv_side : 0.0);  // about z
    case 4: return c == 1 ? -d[2] * inv_side : (c == 2 ? d[1] * inv_side : 0.0);  // about x
    default: return c == 2 ? -d[0] * inv_side : (c == 0 ? d[2] * inv_side : 0.0);  // about y
  }
}

// The orthonormal mode values of point i (3 x 6, masked): out[c][k].
__device__ __forceinline__ void rigid_modes(const double4& x, const double* center, const double* T, double inv_side,
                                            uint8_t fixed, double out[3][6]) {
  const double d[3] = {x.x - center[0], x.y - center[1], x.z - center[2]};
  for (int c = 0; c < 3; ++c) {
    const bool fr = !((fixed >> c) & 1);
    for (int k = 0; k < 6; ++k) {
      double v = 0.0;
      if (fr)
        for (int l = 0; l < 6; ++l) v += rigid_raw(d, inv_side, c, l) * T[6 * l + k];
      out[c][k] = v;
    }
  }
}

__device__ __forceinline__ void agg_cell_xyz(const Grid& g, int q, int* cx, int* cy, int* cz) {
  *cx = q % g.dims[0];
  *cy = (q / g.dims[0]) % g.dims[1];
  *cz = q / (g.dims[0] * g.dims[1]);
}

// Warp per aggregate: center (mean of its points), Gram matrix of the masked
// raw modes, Cholesky with dropping, T = L^-T on the kept modes.
__global__ void k_rigid_setup(int64_t nagg, const int32_t* __restrict__ agg_cell, const int64_t* __restrict__ cstart,
                              const int32_t* __restrict__ sorted, const double4* __restrict__ xv,
                              const uint8_t* __restrict__ fixed, double inv_side, double* __restrict__ center,
                              double* __restrict__ Tm) {
  const int64_t I = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (I >= nagg) return;
  const int q = agg_cell[I];
  const int64_t t0 = cstart[q], t1 = cstart[q + 1];
  double c0 = 0.0, c1 = 0.0, c2 = 0.0;
  for (int64_t t = t0 + lane; t < t1; t += 32) {
    const double4 x = xv[sorted[t]];
    c0 += x.x, c1 += x.y, c2 += x.z;
  }
  for (int o = 16; o > 0; o >>= 1) {
    c0 += __shfl_xor_sync(0xffffffffu, c0, o);
    c1 += __shfl_xor_sync(0xffffffffu, c1, o);
    c2 += __shfl_xor_sync(0xffffffffu, c2, o);
  }
  const double cnt = (double)(t1 - t0);
  const double cen[3] = {c0 / cnt, c1 / cnt, c2 / cnt};
  double G[21];  // lower triangle, row-major
  for (int k = 0; k < 21; ++k) G[k] = 0.0;
  for (int64_t t = t0 + lane; t < t1; t += 32) {
    const int64_t p = sorted[t];
    const double4 x = xv[p];
    const double d[3] = {x.x - cen[0], x.y - cen[1], x.z - cen[2]};
    const uint8_t f = fixed[p];
    for (int c = 0; c < 3; ++c) {
      if ((f >> c) & 1) continue;
      double v[6];
      for (int k = 0; k < 6; ++k) v[k] = rigid_raw(d, inv_side, c, k);
      for (int a = 0, e = 0; a < 6; ++a)
        for (int b = 0; b <= a; ++b, ++e) G[e] += v[a] * v[b];
    }
  }
  for (int k = 0; k < 21; ++k)
    for (int o = 16; o > 0; o >>= 1) G[k] += __shfl_xor_sync(0xffffffffu, G[k], o);
  if (lane != 0) return;
  center[4 * I] = cen[0], center[4 * I + 1] = cen[1], center[4 * I + 2] = cen[2], center[4 * I + 3] = cnt;
  double L[6][6] = {}, gmax = 0.0;
  bool keep[6];
  auto gv = [&](int a, int b) { return a >= b ? G[a * (a + 1) / 2 + b] : G[b * (b + 1) / 2 + a]; };
  for (int k = 0; k < 6; ++k) gmax = fmax(gmax, gv(k, k));
  for (int k = 0; k < 6; ++k) {
    double sd = gv(k, k);
    for (int j = 0; j < k; ++j) sd -= L[k][j] * L[k][j];
    keep[k] = gmax > 0.0 && sd > 1.0e-8 * gmax;
    if (!keep[k]) continue;
    L[k][k] = sqrt(sd);
    for (int i = k + 1; i < 6; ++i) {
      double v = gv(i, k);
      for (int j = 0; j < k; ++j) v -= L[i][j] * L[k][j];
      L[i][k] = v / L[k][k];
    }
  }
  // M = L^-1 on the kept modes (forward substitution), T = M^T
  double M[6][6] = {};
  for (int k = 0; k < 6; ++k) {
    if (!keep[k]) continue;
    for (int i = k; i < 6; ++i) {
      if (!keep[i]) continue;
      double v = i == k ? 1.0 : 0.0;
      for (int j = k; j < i; ++j) v -= L[i][j] * M[j][k];
      M[i][k] = v / L[i][i];
    }
  }
  double* T = Tm + 36 * I;
  for (int l = 0; l < 6; ++l)
    for (int k = 0; k < 6; ++k) T[6 * l + k] = M[k][l];
}

// Probes of color cc, all 6 modes at once (point-major: w[(i*6 + m)*3 + c]).
__global__ void k_rigid_probe6(int64_t n, const int32_t* __restrict__ agg_of, const int32_t* __restrict__ agg_cell,
                               Grid g, int cc, const double* __restrict__ center, const double* __restrict__ Tm,
                               const double4* __restrict__ xv, const uint8_t* __restrict__ fixed, double inv_side,
                               double* __restrict__ w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int I = agg_of[i];
  int cx, cy, cz;
  agg_cell_xyz(g, agg_cell[I], &cx, &cy, &cz);
  double v[3][6];
  const bool on = (cx % 3) + 3 * (cy % 3) + 9 * (cz % 3) == cc;
  if (on) rigid_modes(xv[i], center + 4 * I, Tm + 36 * I, inv_side, fixed[i], v);
  for (int m = 0; m < 6; ++m)
    for (int c = 0; c < 3; ++c) w[(i * 6 + m) * 3 + c] = on ? v[c][m] : 0.0;
}

// Warp per aggregate row I: Ac[6I + k][6J + m] for all 6 probe modes m of color cc.
__global__ void k_rigid_block6(int64_t nagg, int nc, Grid g, int cc, const int32_t* __restrict__ agg_cell,
                               const int32_t* __restrict__ cell_agg, const int64_t* __restrict__ cstart,
                               const int32_t* __restrict__ sorted, const double* __restrict__ center,
                               const double* __restrict__ Tm, const double4* __restrict__ xv,
                               const uint8_t* __restrict__ fixed, double inv_side, const double* __restrict__ kw,
                               double* __restrict__ A) {
  const int64_t I = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (I >= nagg) return;
  const int q = agg_cell[I];
  int c3[3];
  agg_cell_xyz(g, q, &c3[0], &c3[1], &c3[2]);
  const int want[3] = {cc % 3, (cc / 3) % 3, cc / 9};
  int jc[3];
  for (int a = 0; a < 3; ++a) {
    int d = -1;
    while (((c3[a] + d) % 3 + 3) % 3 != want[a]) ++d;
    jc[a] = c3[a] + d;
    if (jc[a] < 0 || jc[a] >= g.dims[a]) return;
  }
  const int J = cell_agg[(jc[2] * g.dims[1] + jc[1]) * g.dims[0] + jc[0]];
  if (J < 0) return;
  double acc[6][6];
  for (int k = 0; k < 6; ++k)
    for (int m = 0; m < 6; ++m) acc[k][m] = 0.0;
  for (int64_t t = cstart[q] + lane; t < cstart[q + 1]; t += 32) {
    const int64_t p = sorted[t];
    double v[3][6];
    rigid_modes(xv[p], center + 4 * I, Tm + 36 * I, inv_side, fixed[p], v);
    const double* y = kw + p * 18;
    for (int m = 0; m < 6; ++m)
      for (int k = 0; k < 6; ++k) acc[k][m] += v[0][k] * y[3 * m] + v[1][k] * y[3 * m + 1] + v[2][k] * y[3 * m + 2];
  }
  for (int k = 0; k < 6; ++k)
    for (int m = 0; m < 6; ++m)
      for (int o = 16; o > 0; o >>= 1) acc[k][m] += __shfl_xor_sync(0xffffffffu, acc[k][m], o);
  if (lane == 0)
    for (int k = 0; k < 6; ++k)
      for (int m = 0; m < 6; ++m) A[(size_t)(6 * I + k) * nc + 6 * J + m] = acc[k][m];
}

// rc_I = P0_I^T r: the orthonormalised rigid modes of aggregate I at its
// points against r (a block of kRestrictT threads per aggregate, fixed-order
// block sum).
template <typename T>
__global__ void __launch_bounds__(kRestrictT) k_rigid_restrict(int64_t nagg, const int32_t* __restrict__ agg_cell,
                                                               const int64_t* __restrict__ cstart,
                                                               const int32_t* __restrict__ sorted,
                                                               const double* __restrict__ center,
                                                               const double* __restrict__ Tm,
                                                               const double4* __restrict__ xv,
                                                               const uint8_t* __restrict__ fixed, double inv_side,
                                                               const T* __restrict__ r, double* __restrict__ rc) {
  __shared__ double sh[6][kRestrictT];
  const int64_t I = blockIdx.x;
  const int q = agg_cell[I];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t t = cstart[q] + threadIdx.x; t < cstart[q + 1]; t += kRestrictT) {
    const int64_t p = sorted[t];
    double v[3][6];
    rigid_modes(xv[p], center + 4 * I, Tm + 36 * I, inv_side, fixed[p], v);
    const double r0 = (double)r[3 * p], r1 = (double)r[3 * p + 1], r2 = (double)r[3 * p + 2];
    for (int k = 0; k < 6; ++k) acc[k] += v[0][k] * r0 + v[1][k] * r1 + v[2][k] * r2;
  }
  block_sum<6>(acc, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) rc[6 * I + k] = acc[k];
}

__global__ void k_rigid_prolong(int64_t n, const int32_t* __restrict__ agg_of, const double* __restrict__ center,
                                const double* __restrict__ Tm, const double4* __restrict__ xv,
                                const uint8_t* __restrict__ fixed, double inv_side, const double* __restrict__ zc,
                                double scale, double* __restrict__ z) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t I = agg_of[i];
  double v[3][6];
  rigid_modes(xv[i], center + 4 * I, Tm + 36 * I, inv_side, fixed[i], v);
  for (int c = 0; c < 3; ++c) {
    double s = 0.0;
    for (int k = 0; k < 6; ++k) s += v[c][k] * zc[6 * I + k];
    if (!((fixed[i] >> c) & 1)) z[3 * i + c] += scale * s;
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static CoarseState* co_state(pd_ctx* c) {
  if (!c->coarse) c->coarse = new CoarseState();
  return c->coarse;
}

void coarse_release(pd_ctx* c) {
  delete c->coarse;
  c->coarse = nullptr;
}

void coarse_invalidate(pd_ctx* c) {
  if (c->coarse) c->coarse->have_op = false;
}

bool coarse_valid(const pd_ctx* c) { return c->coarse && c->coarse->have_op; }

int64_t coarse_size(const pd_ctx* c) { return c->coarse && c->coarse->have_op ? c->coarse->nc : 0; }

// Aggregates: the non-empty cells of a grid of side max(cell, 2 * max
// horizon) over the model coordinates, the side grown by 1.25x until the
// coarse space has at most kMaxCoarse dofs.
static int co_aggregates(pd_ctx* c, CoarseState* s, double cell) {
  const int64_t n = c->n;
  double hmax = 0.0;
  for (double h : c->block_h) hmax = std::max(hmax, h);
  double side = std::max(cell, 2.0 * hmax * (1.0 + 1.0e-6));
  const int modes = c->coarse_modes == 6 ? 6 : 3;
  if (s->built && s->n == n && s->cell == side && s->modes == modes) return PD_OK;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], c->hx[3 * i + k]), hi[k] = std::max(hi[k], c->hx[3 * i + k]);
  DBuf<int64_t> nagg_d;
  PD_CUDA_TRY(c, nagg_d.alloc(1));
  const double want = side;
  for (;;) {
    Grid g;
    for (int k = 0; k < 3; ++k) {
      g.lo[k] = lo[k];
      g.dims[k] = (int)std::floor((hi[k] - lo[k]) / side) + 1;
    }
    g.cell = side;
    const int64_t ncell = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
    if (3 * std::min<int64_t>(ncell, n) > 64 * (int64_t)kMaxCoarse) {  // far too fine: grow before binning
      side *= 1.25;
      continue;
    }
    TRY_RC(bin_points(c, c->xv.p, n, g, s->sorted, s->cstart));
    PD_CUDA_TRY(c, s->cell_agg.alloc(ncell));
    PD_CUDA_TRY(c, s->agg_cell.alloc(std::min<int64_t>(ncell, n)));
    k_coarse_cells<<<1, 32, 0, c->stream>>>(ncell, s->cstart.p, s->cell_agg.p, s->agg_cell.p, nagg_d.p);
    PD_CUDA_TRY(c, cudaGetLastError());
    int64_t nagg = 0;
    PD_CUDA_TRY(c, d2h(c, &nagg, nagg_d.p, sizeof(int64_t)));
    if (modes * nagg > kMaxCoarse) {
      side *= 1.25;
      continue;
    }
    s->g = g;
    s->nagg = nagg;
    s->nc = (int)(modes * nagg);
    break;
  }
  PD_CUDA_TRY(c, s->agg_of.alloc(n));
  k_coarse_agg_of<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, c->xv.p, s->g, s->cell_agg.p, s->agg_of.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  const int nc = s->nc;
  PD_CUDA_TRY(c, s->clo.alloc(4 * (size_t)n));
  PD_CUDA_TRY(c, s->slots.alloc((size_t)n * kSlots * kSlotVals));
  PD_CUDA_TRY(c, s->A.alloc((size_t)nc * nc));
  PD_CUDA_TRY(c, s->P.alloc(kGjB * kGjB));
  PD_CUDA_TRY(c, s->R.alloc((size_t)kGjB * nc));
  PD_CUDA_TRY(c, s->C.alloc((size_t)kGjB * nc));
  PD_CUDA_TRY(c, s->rc.alloc(nc));
  PD_CUDA_TRY(c, s->zc.alloc(nc));
  PD_CUDA_TRY(c, s->status.alloc(1));
  if (modes == 6) {
    PD_CUDA_TRY(c, s->center.alloc(4 * (size_t)s->nagg));
    PD_CUDA_TRY(c, s->T.alloc(36 * (size_t)s->nagg));
    PD_CUDA_TRY(c, s->probe.alloc(18 * (size_t)n));
    PD_CUDA_TRY(c, s->kprobe.alloc(18 * (size_t)n));
    PD_CUDA_TRY(c, s->pdth.alloc(6 * (size_t)n));
  }
  s->modes = modes;
  s->n = n;
  s->cell = want;
  s->built = true;
  s->have_op = false;
  return PD_OK;
}

// Assembles Ac = P0^T K P0 at the tangent state (y, ab = (theta, q, alpha, .),
// fixed) and inverts it in place. A copy of the assembled matrix goes to
// `assembled` (device, nc*nc) when not null.
int coarse_build(pd_ctx* c, const double4* y, const double4* ab, const uint8_t* fixed, double cell,
                 double* assembled) {
  CoarseState* s = co_state(c);
  TRY_RC(co_aggregates(c, s, cell));
  const int64_t n = c->n;
  const int nc = s->nc;
  if (s->modes == 6) {  // rigid modes: orthonormal bases, then colored probing with the tangent
    const double inv_side = 1.0 / s->g.cell;
    const unsigned gw = (unsigned)((s->nagg * 32 + 255) / 256), gp = (unsigned)((n + 255) / 256);
    k_rigid_setup<<<gw, 256, 0, c->stream>>>(s->nagg, s->agg_cell.p, s->cstart.p, s->sorted.p, c->xv.p, fixed,
                                             inv_side, s->center.p, s->T.p);
    PD_CUDA_TRY(c, dzero(c, s->A.p, s->A.bytes()));
    for (int cc = 0; cc < 27; ++cc) {  // one multi-vector tangent product per color (its 6 modes)
      k_rigid_probe6<<<gp, 256, 0, c->stream>>>(n, s->agg_of.p, s->agg_cell.p, s->g, cc, s->center.p, s->T.p, c->xv.p,
                                                fixed, inv_side, s->probe.p);
      PD_CUDA_TRY(c, cudaGetLastError());
      TRY_RC(qs_apply_K_multi(c, s->probe.p, s->kprobe.p, s->pdth.p));
      k_rigid_block6<<<gw, 256, 0, c->stream>>>(s->nagg, nc, s->g, cc, s->agg_cell.p, s->cell_agg.p, s->cstart.p,
                                                s->sorted.p, s->center.p, s->T.p, c->xv.p, fixed, inv_side,
                                                s->kprobe.p, s->A.p);
    }
    k_coarse_unit_diag<<<(nc + 255) / 256, 256, 0, c->stream>>>(nc, s->A.p);
    PD_CUDA_TRY(c, cudaGetLastError());
    (void)y;
    (void)ab;
  } else {
  PD_CUDA_TRY(c, dzero(c, s->status.p, sizeof(int)));
  k_coarse_point<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, y, ab,
                                                                     c->pt.p, c->hp.p, c->influence, fixed, s->g,
                                                                     s->clo.p, s->slots.p, s->status.p);
  PD_CUDA_TRY(c, dzero(c, s->A.p, s->A.bytes()));
  k_coarse_rows<<<(unsigned)((s->nagg + kRowWarps - 1) / kRowWarps), 32 * kRowWarps, 0, c->stream>>>(
      s->nagg, nc, s->g, s->agg_cell.p, s->cell_agg.p, s->cstart.p, s->sorted.p, s->clo.p, s->slots.p, s->A.p);
  k_coarse_unit_diag<<<(nc + 255) / 256, 256, 0, c->stream>>>(nc, s->A.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  int st = 0;
  PD_CUDA_TRY(c, d2h(c, &st, s->status.p, sizeof(int)));
  if (st) {
    c->err = "coarse space: a bond reaches past its point's 2x2x2 aggregate cells";
    return PD_ERR_STATE;
  }
  }
  if (assembled)
    PD_CUDA_TRY(c, cudaMemcpyAsync(assembled, s->A.p, s->A.bytes(), cudaMemcpyDeviceToDevice, c->stream));
  const int ntile = (nc + kGjB - 1) / kGjB, nut = (nc + kUT - 1) / kUT;
  PD_CUDA_TRY(c, cudaFuncSetAttribute(k_gj_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmem));
  PD_CUDA_TRY(c, cudaFuncSetAttribute(k_gj_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem));
  PD_CUDA_TRY(c, cudaFuncSetAttribute(k_gj_next_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem));
  if (!s->aux) {
    int lo = 0, hi = 0;  // the highest priority: the pivot takes the first SM the update frees
    PD_CUDA_TRY(c, cudaDeviceGetStreamPriorityRange(&lo, &hi));
    PD_CUDA_TRY(c, cudaStreamCreateWithPriority(&s->aux, cudaStreamNonBlocking, hi));
    PD_CUDA_TRY(c, cudaEventCreateWithFlags(&s->e_diag, cudaEventDisableTiming));
    PD_CUDA_TRY(c, cudaEventCreateWithFlags(&s->e_piv, cudaEventDisableTiming));
  }
  if (s->D.count < (size_t)kGjB * kGjB) PD_CUDA_TRY(c, s->D.alloc((size_t)kGjB * kGjB));
  // Lookahead: after the panel of block k, the next diagonal block as the
  // trailing update will leave it goes to D, and its inverse runs on the
  // second stream beside that update; the next panel waits for it.
  k_gj_pivot<<<1, 256, 0, c->stream>>>(s->A.p, nc, std::min(kGjB, nc), s->P.p);
  for (int k0 = 0; k0 < nc; k0 += kGjB) {
    const int bk = std::min(kGjB, nc - k0), k1 = k0 + bk;
    if (k0 > 0) PD_CUDA_TRY(c, cudaStreamWaitEvent(c->stream, s->e_piv, 0));
    k_gj_panel<<<ntile, 256, kPanelSmem, c->stream>>>(nc, k0, bk, s->A.p, s->P.p, s->R.p, s->C.p);
    if (k1 < nc) {
      const int bk1 = std::min(kGjB, nc - k1);
      k_gj_next_diag<<<1, 256, kPanelSmem, c->stream>>>(nc, k1, bk1, bk, s->A.p, s->R.p, s->C.p, s->D.p);
      PD_CUDA_TRY(c, cudaEventRecord(s->e_diag, c->stream));
      PD_CUDA_TRY(c, cudaStreamWaitEvent(s->aux, s->e_diag, 0));
      k_gj_pivot<<<1, 256, 0, s->aux>>>(s->D.p, bk1, bk1, s->P.p);
      PD_CUDA_TRY(c, cudaEventRecord(s->e_piv, s->aux));
    }
    k_gj_update<<<(unsigned)(nut * (nut + 1) / 2), kUpdT, kUpdSmem, c->stream>>>(nc, k0, bk, s->A.p, s->R.p,
                                                                                 s->C.p);
  }
  k_gj_mirror<<<dim3(ntile, ntile), 256, 0, c->stream>>>(nc, s->A.p);
  // the FP32 copy each CG iteration's coarse product reads (half the bytes;
  // the products and sums stay FP64)
  if (s->Af.count < (size_t)nc * nc) PD_CUDA_TRY(c, s->Af.alloc((size_t)nc * nc));
  k_to_f32<<<(unsigned)(((int64_t)nc * nc + 255) / 256), 256, 0, c->stream>>>((int64_t)nc * nc, s->A.p, s->Af.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  s->have_op = true;
  return PD_OK;
}

// z += scale P0 Ac^-1 P0^T r on the free dofs (r double or float).
template <typename T>
static int co_apply(pd_ctx* c, const T* r, double* z, const uint8_t* fixed, double scale) {
  CoarseState* s = c->coarse;
  if (!s || !s->have_op) {
    c->err = "coarse operator not built";
    return PD_ERR_STATE;
  }
  const int64_t n = c->n;
  const unsigned ga = (unsigned)s->nagg, gv = (unsigned)(((int64_t)s->nc * 32 + 255) / 256);
  if (s->modes == 6) {
    const double inv_side = 1.0 / s->g.cell;
    k_rigid_restrict<T><<<ga, kRestrictT, 0, c->stream>>>(s->nagg, s->agg_cell.p, s->cstart.p, s->sorted.p,
                                                          s->center.p, s->T.p, c->xv.p, fixed, inv_side, r, s->rc.p);
    k_coarse_gemv_f<<<gv, 256, 0, c->stream>>>(s->nc, s->Af.p, s->rc.p, s->zc.p);
    k_rigid_prolong<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, s->agg_of.p, s->center.p, s->T.p, c->xv.p,
                                                                        fixed, inv_side, s->zc.p, scale, z);
    PD_CUDA_TRY(c, cudaGetLastError());
    return PD_OK;
  }
  k_coarse_restrict<T><<<ga, kRestrictT, 0, c->stream>>>(s->nagg, s->agg_cell.p, s->cstart.p, s->sorted.p, r,
                                                         s->rc.p);
  k_coarse_gemv_f<<<gv, 256, 0, c->stream>>>(s->nc, s->Af.p, s->rc.p, s->zc.p);
  k_coarse_prolong<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, s->agg_of.p, s->zc.p, scale, fixed, z);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

int coarse_apply_add(pd_ctx* c, const double* r, double* z, const uint8_t* fixed) {
  return co_apply(c, r, z, fixed, 1.0);
}
int coarse_apply_add_f(pd_ctx* c, const float* r, double* z, const uint8_t* fixed, double scale) {
  return co_apply(c, r, z, fixed, scale);
}

// Aggregate of every point (device, n) of the current coarse space.
int coarse_aggregates(pd_ctx* c, int32_t* agg_dev) {
  CoarseState* s = c->coarse;
  if (!s || !s->built) {
    c->err = "coarse space not built";
    return PD_ERR_STATE;
  }
  PD_CUDA_TRY(c, cudaMemcpyAsync(agg_dev, s->agg_of.p, c->n * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
  return PD_OK;
}

int coarse_copy_inverse(pd_ctx* c, double* dst) {
  CoarseState* s = c->coarse;
  if (!s || !s->have_op) {
    c->err = "coarse operator not built";
    return PD_ERR_STATE;
  }
  PD_CUDA_TRY(c, cudaMemcpyAsync(dst, s->A.p, (size_t)s->nc * s->nc * sizeof(double), cudaMemcpyDeviceToDevice,
                                 c->stream));
  return PD_OK;
}

}  // namespace pdb
