// Quasi-static Newton / CG (sm_100a), FP64.
//
// Replaces Peridigm::executeQuasiStatic (src/core/Peridigm.cpp:2470-3043) with
// its residual (computeQuasiStaticResidual, :4176-4317), tangent
// (ElasticMaterial::computeAutomaticDifferentiationJacobian,
// src/materials/Peridigm_ElasticMaterial.cpp:258-383, Scale(-1) at
// Peridigm.cpp:2800) and Belos CG (:2551-2573, :3321-3362):
//  * residual r = V (f_int + f_ext), rows of prescribed dofs zeroed;
//  * tangent K = -d r / d u applied matrix-free: the exact linearization of
//    the LPS force in two bond passes (d theta, then d f) over per-bond
//    geometry built once per state (unit deformed bond, V_j om zeta,
//    V_j T/|Y|, V_j om (alpha_i + alpha_j)), rows and columns of prescribed
//    dofs replaced by identity (applyKinematicBC_InsertZerosAndSetDiagonal);
//  * preconditioned CG with deterministic FP64 dot products; block-Jacobi
//    preconditioner = inverses of the analytic 3x3 diagonal blocks of K
//    (the reference's "Block 3x3" preconditioner, Peridigm.cpp:1603-1646);
//    the two-level and learned preconditioners add k_coarse.cu's coarse
//    correction and k_mpnn.cu's learned middle level to it;
//  * Newton with a backtracking step on the reference's convergence metric
//    ||r||_2 + 20 ||r||_inf (Peridigm.cpp:4316).
// For a bond (i,j) with Y = y_j - y_i, e = |Y| - |X|, de = Yhat.(w_j - w_i):
//   d theta_i = sum 3 omega zeta de V_j / m_i
//   t_ij = omega (zeta theta_i q_i + alpha_i e),  q = 3K/m - alpha/3, alpha = 15mu/m
//   dt_ij = omega (zeta dtheta_i q_i + alpha_i de)
//   d f_i = sum V_j [ (dt_ij + dt_ji) Yhat + (t_ij + t_ji) (dw - Yhat de)/|Y| ]
#include <algorithm>
#include <cmath>
#include <vector>

#include "pd_internal.cuh"

namespace pdb {

constexpr int kQsBlock = 256;
constexpr int kQsTpo = 8;
#ifndef PD_QS_BATCH
#define PD_QS_BATCH 4
#endif
constexpr int kQsBatch = PD_QS_BATCH;  // bonds per lane in flight in the tangent passes
constexpr int kRedBlocks = 296;  // 2 x 148 SMs: fixed, so reductions are deterministic

struct QsState {
  DBuf<double4> yq;    // coordinates x + u + du
  DBuf<double4> abq;   // (theta, q, alpha, q/m)
  DBuf<double4> w;     // CG direction (p, dtheta)
  DBuf<double> th, nd, f, r, du, x, z, q, pred, dinv, partial, scal;
  DBuf<uint8_t> fixed;  // bit c: dof c prescribed
  int64_t n = 0;
  bool coarse_on = false;  // the preconditioner adds the aggregate coarse correction (k_coarse.cu)
  // Per-bond tangent geometry at the current (y, theta, q, alpha), rebuilt
  // after every change of the state (geo_dirty): g = (yh, V_j om zeta),
  // gc = (V_j T / |Y|, V_j om (alpha_i + alpha_j)); zero for broken bonds.
  DBuf<double4> geo;
  DBuf<double2> gco;
  bool geo_dirty = true;
  // Coarse-operator reuse: the operator is rebuilt when the model changed, or
  // when a solve needs more than 1.3x (+5) the CG iterations of the first solve
  // after the last rebuild (the tangent drifted from the one it was built at).
  double coarse_cell = -1.0;
  int64_t coarse_ref_iters = -1;
  bool coarse_rebuild = true;
  // The operator the CG products and block-Jacobi blocks use: jm rho I + jk K
  // (quasi-static: K; implicit dynamics: rho I + beta dt^2 K).
  double jk = 1.0, jm = 0.0;
  DBuf<double> v2;  // implicit dynamics: velocity predictor
  DBuf<double> cg_b, cg_x0;  // learned-preconditioner CG: right-hand side and restart point (kept, not reallocated)
};

__device__ __forceinline__ double qs_omega(int kind, double zeta, double h) {
  if (kind == PD_INFLUENCE_ONE) return 1.0;
  if (kind == PD_INFLUENCE_PARABOLIC_DECAY) {
    if (zeta > h) return 0.0;
    const double s = zeta / h;
    return s < 0.5 ? 1.0 : -4.0 * s * s + 4.0 * s;
  }
  return exp(-(zeta * zeta) / (h * h * 0.16));
}

template <typename T>
__device__ __forceinline__ T qs_group_sum(T v) {
#pragma unroll
  for (int o = kQsTpo / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// y = (x + u) + du (Peridigm.cpp:2684-2687 operation order)
__global__ void k_qs_positions(int64_t n, const double4* __restrict__ xv, const double* __restrict__ u,
                               const double* __restrict__ du, double4* __restrict__ y) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 x = xv[i];
  y[i] = make_double4((x.x + u[3 * i]) + du[3 * i], (x.y + u[3 * i + 1]) + du[3 * i + 1],
                      (x.z + u[3 * i + 2]) + du[3 * i + 2], 0.0);
}

// abq.w = q/m for the block-diagonal term
__global__ void k_qs_qm(int64_t n, const double4* __restrict__ pt, double4* __restrict__ ab) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ab[i].w = ab[i].y / pt[i].x;
}

// r = V f with prescribed rows zeroed; block partials of sum r^2 and max |r|.
__global__ void k_qs_residual(int64_t n, const double* __restrict__ f, const double4* __restrict__ xv,
                              const uint8_t* __restrict__ fixed, double* __restrict__ r,
                              double* __restrict__ partial) {
  __shared__ double s2[kQsBlock], sm[kQsBlock];
  double a2 = 0.0, am = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < 3 * n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k / 3;
    const int c = (int)(k - 3 * i);
    double v = f[k] * xv[i].w;
    if ((fixed[i] >> c) & 1) v = 0.0;
    r[k] = v;
    a2 += v * v;
    am = fmax(am, fabs(v));
  }
  s2[threadIdx.x] = a2;
  sm[threadIdx.x] = am;
  __syncthreads();
  for (int o = kQsBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s2[threadIdx.x] += s2[threadIdx.x + o];
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s2[0];
    partial[2 * blockIdx.x + 1] = sm[0];
  }
}

// Sums (even slots) and maxima (odd slots) of kRedBlocks partial pairs, or
// plain sums of `width` interleaved partials; fixed order.
__global__ void k_qs_reduce(const double* __restrict__ partial, int nblk, int width, int mode,
                            double* __restrict__ out) {
  __shared__ double s[kQsBlock];
  for (int c = 0; c < width; ++c) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
      const double v = partial[width * b + c];
      a = (mode == 1 && c == 1) ? fmax(a, v) : a + v;
    }
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = kQsBlock / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) s[threadIdx.x] = (mode == 1 && c == 1) ? fmax(s[threadIdx.x], s[threadIdx.x + o])
                                                                   : s[threadIdx.x] + s[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = s[0];
    __syncthreads();
  }
}

// Per-bond tangent geometry (one lane group per owner, bonds strided over lanes).
__global__ void __launch_bounds__(kQsBlock) k_qs_bond_geom(int64_t n, const int64_t* __restrict__ row,
                                                           const int32_t* __restrict__ col,
                                                           const uint8_t* __restrict__ dmg,
                                                           const double4* __restrict__ xv,
                                                           const double4* __restrict__ y,
                                                           const double4* __restrict__ ab,
                                                           const double* __restrict__ hp, int influence,
                                                           double4* __restrict__ g, double2* __restrict__ gc) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kQsTpo;
  const int lane = threadIdx.x & (kQsTpo - 1);
  if (i >= n) return;
  const double4 xi = xv[i], yi = y[i], ai = ab[i];
  const double h = hp[i];
  for (int64_t b = row[i] + lane; b < row[i + 1]; b += kQsTpo) {
    if (dmg[b]) {
      g[b] = make_double4(0.0, 0.0, 0.0, 0.0);
      gc[b] = make_double2(0.0, 0.0);
      continue;
    }
    const int32_t j = col[b];
    const double4 xj = xv[j], yj = y[j], aj = ab[j];
    const double X0 = xj.x - xi.x, X1 = xj.y - xi.y, X2 = xj.z - xi.z;
    const double Y0 = yj.x - yi.x, Y1 = yj.y - yi.y, Y2 = yj.z - yi.z;
    const double zeta = sqrt(X0 * X0 + X1 * X1 + X2 * X2);
    const double dY = sqrt(Y0 * Y0 + Y1 * Y1 + Y2 * Y2);
    const double e = dY - zeta;
    const double om = qs_omega(influence, zeta, h);
    const double T = om * (zeta * (ai.x * ai.y + aj.x * aj.y) + (ai.z + aj.z) * e);
    const double V = xj.w;
    g[b] = make_double4(Y0 / dY, Y1 / dY, Y2 / dY, V * om * zeta);
    gc[b] = make_double2(V * T / dY, V * om * (ai.z + aj.z));
  }
}

// Tangent pass 1 on the geometry: w[i].w = q_i dtheta_i = 3 (q_i/m_i) sum_j V_j om zeta yh.(w_j - w_i)
__global__ void __launch_bounds__(kQsBlock) k_qs_dtheta_g(int64_t n, const int64_t* __restrict__ row,
                                                          const int32_t* __restrict__ col,
                                                          const double4* __restrict__ g,
                                                          const double4* __restrict__ ab,
                                                          const double4* __restrict__ pt, double4* __restrict__ w) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kQsTpo;
  const int lane = threadIdx.x & (kQsTpo - 1);
  const bool valid = i < n;
  double acc = 0.0;
  if (valid) {
    const double4 wi = w[i];
    const int64_t b1 = row[i + 1];
    int64_t b = row[i] + lane;
    // batches of kQsBatch bonds per lane: stream loads, then gathers, then the
    // sums in bond order (the same order as one bond at a time)
    for (; b + (kQsBatch - 1) * kQsTpo < b1; b += kQsBatch * kQsTpo) {
      double4 gb[kQsBatch], wj[kQsBatch];
      int32_t j[kQsBatch];
#pragma unroll
      for (int k = 0; k < kQsBatch; ++k) gb[k] = g[b + k * kQsTpo], j[k] = col[b + k * kQsTpo];
#pragma unroll
      for (int k = 0; k < kQsBatch; ++k) wj[k] = w[j[k]];
#pragma unroll
      for (int k = 0; k < kQsBatch; ++k)
        acc += gb[k].w * (gb[k].x * (wj[k].x - wi.x) + gb[k].y * (wj[k].y - wi.y) + gb[k].z * (wj[k].z - wi.z));
    }
    for (; b < b1; b += kQsTpo) {
      const double4 gb = g[b];
      const double4 wj = w[col[b]];
      acc += gb.w * (gb.x * (wj.x - wi.x) + gb.y * (wj.y - wi.y) + gb.z * (wj.z - wi.z));
    }
  }
  acc = qs_group_sum(acc);
  if (valid && lane == 0) w[i].w = 3.0 * (ab[i].y / pt[i].x) * acc;
}

// Tangent pass 2 on the geometry: q = K p = -V d f (prescribed rows: q = p), or
// (jm rho I + jk K) p for implicit dynamics; block partials of p.q
//   V_j [dT yh + (T/|Y|)(dw - yh de)] = c2 (q dth_i + q dth_j) yh + V_j om (a_i + a_j) de yh + V_j T/|Y| (dw - yh de)
__global__ void __launch_bounds__(kQsBlock) k_qs_df_g(int64_t n, const int64_t* __restrict__ row,
                                                      const int32_t* __restrict__ col,
                                                      const double4* __restrict__ g,
                                                      const double2* __restrict__ gc,
                                                      const double4* __restrict__ xv,
                                                      const double4* __restrict__ w,
                                                      const uint8_t* __restrict__ fixed, double* __restrict__ q,
                                                      double* __restrict__ partial, const double4* __restrict__ pt,
                                                      double jk, double jm) {
  __shared__ double spq[kQsBlock];
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kQsTpo;
  const int lane = threadIdx.x & (kQsTpo - 1);
  const bool valid = i < n;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
  double4 wi = make_double4(0, 0, 0, 0);
  if (valid) {
    wi = w[i];
    const int64_t b1 = row[i + 1];
    int64_t b = row[i] + lane;
    auto bond = [&](const double4& gb, const double2& cb, const double4& wj) {
      const double w0 = wj.x - wi.x, w1 = wj.y - wi.y, w2 = wj.z - wi.z;
      const double de = gb.x * w0 + gb.y * w1 + gb.z * w2;
      const double sy = gb.w * (wi.w + wj.w) + (cb.y - cb.x) * de;
      d0 += sy * gb.x + cb.x * w0;
      d1 += sy * gb.y + cb.x * w1;
      d2 += sy * gb.z + cb.x * w2;
    };
    for (; b + (kQsBatch - 1) * kQsTpo < b1; b += kQsBatch * kQsTpo) {  // batched as in k_qs_dtheta_g
      double4 gb[kQsBatch], wj[kQsBatch];
      double2 cb[kQsBatch];
      int32_t j[kQsBatch];
#pragma unroll
      for (int k = 0; k < kQsBatch; ++k) gb[k] = g[b + k * kQsTpo], cb[k] = gc[b + k * kQsTpo], j[k] = col[b + k * kQsTpo];
#pragma unroll
      for (int k = 0; k < kQsBatch; ++k) wj[k] = w[j[k]];
#pragma unroll
      for (int k = 0; k < kQsBatch; ++k) bond(gb[k], cb[k], wj[k]);
    }
    for (; b < b1; b += kQsTpo) bond(g[b], gc[b], w[col[b]]);
  }
  d0 = qs_group_sum(d0);
  d1 = qs_group_sum(d1);
  d2 = qs_group_sum(d2);
  double pq = 0.0;
  if (valid && lane < 3) {
    const double d = lane == 0 ? d0 : (lane == 1 ? d1 : d2);
    const double p = lane == 0 ? wi.x : (lane == 1 ? wi.y : wi.z);
    double kd = -xv[i].w * d;
    if (jm != 0.0) kd = jm * pt[i].w * p + jk * kd;  // implicit dynamics: (rho I + beta dt^2 K) p
    const double out = ((fixed[i] >> lane) & 1) ? p : kd;
    q[3 * i + lane] = out;
    pq = p * out;
  }
  spq[threadIdx.x] = pq;
  __syncthreads();
  for (int o = kQsBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) spq[threadIdx.x] += spq[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = spq[0];
}

// Inverse 3x3 diagonal blocks of K (prescribed rows/columns set to identity).
__global__ void __launch_bounds__(kQsBlock) k_qs_block_diag(int64_t n, const int64_t* __restrict__ row,
                                                            const int32_t* __restrict__ col,
                                                            const uint8_t* __restrict__ dmg,
                                                            const double4* __restrict__ xv,
                                                            const double4* __restrict__ y,
                                                            const double4* __restrict__ ab,
                                                            const double4* __restrict__ pt,
                                                            const double* __restrict__ hp, int influence,
                                                            const uint8_t* __restrict__ fixed,
                                                            double* __restrict__ dinv, int invert, double jk = 1.0,
                                                            double jm = 0.0) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kQsTpo;
  const int lane = threadIdx.x & (kQsTpo - 1);
  const bool valid = i < n;
  double D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double hv[3] = {0, 0, 0};
  double4 xi = make_double4(0, 0, 0, 1), ai = make_double4(0, 0, 0, 0);
  double mi = 1.0;
  if (valid) {
    xi = xv[i];
    const double4 yi = y[i];
    ai = ab[i];
    mi = pt[i].x;
    const double h = hp[i];
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += kQsTpo) {
      if (dmg[b]) continue;
      const int32_t j = col[b];
      const double4 xj = xv[j], yj = y[j], aj = ab[j];
      const double X0 = xj.x - xi.x, X1 = xj.y - xi.y, X2 = xj.z - xi.z;
      const double Y0 = yj.x - yi.x, Y1 = yj.y - yi.y, Y2 = yj.z - yi.z;
      const double zeta = sqrt(X0 * X0 + X1 * X1 + X2 * X2);
      const double dY = sqrt(Y0 * Y0 + Y1 * Y1 + Y2 * Y2);
      const double e = dY - zeta;
      const double om = qs_omega(influence, zeta, h);
      const double T = om * (zeta * (ai.x * ai.y + aj.x * aj.y) + (ai.z + aj.z) * e);
      const double V = xj.w;
      const double yh[3] = {Y0 / dY, Y1 / dY, Y2 / dY};
      const double a = -V * om * ((ai.z + aj.z) + 3.0 * om * zeta * zeta * aj.w * xi.w);
      const double g = -V * T / dY;
      for (int r = 0; r < 3; ++r) {
        hv[r] += V * om * zeta * yh[r];
        for (int c = 0; c < 3; ++c) D[3 * r + c] += (a - g) * yh[r] * yh[c] + (r == c ? g : 0.0);
      }
    }
  }
  for (int k = 0; k < 9; ++k) D[k] = qs_group_sum(D[k]);
  for (int k = 0; k < 3; ++k) hv[k] = qs_group_sum(hv[k]);
  if (valid && lane == 0) {
    const double s = 3.0 * ai.y / mi;
    double A[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) A[3 * r + c] = -xi.w * (D[3 * r + c] - s * hv[r] * hv[c]);  // K_ii = -V_i D_i
    if (jm != 0.0)  // implicit dynamics: blocks of rho I + beta dt^2 K
      for (int k = 0; k < 9; ++k) A[k] = jk * A[k] + ((k % 4 == 0) ? jm * pt[i].w : 0.0);
    const uint8_t fx = fixed[i];
    for (int c = 0; c < 3; ++c)
      if ((fx >> c) & 1)
        for (int k = 0; k < 3; ++k) {
          A[3 * c + k] = (k == c) ? 1.0 : 0.0;
          A[3 * k + c] = (k == c) ? 1.0 : 0.0;
        }
    if (!invert) {
      for (int k = 0; k < 9; ++k) dinv[9 * i + k] = A[k];
      return;
    }
    const double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
    const double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
    const double id = 1.0 / det;
    double* o = dinv + 9 * i;
    o[0] = c00 * id;
    o[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    o[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    o[3] = c01 * id;
    o[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    o[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    o[6] = c02 * id;
    o[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    o[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  }
}

// z = P r (block Jacobi or identity); optional partial sums of r.z and r.r.
__global__ void k_qs_precond(int64_t n, const double* __restrict__ dinv, const double* __restrict__ r,
                             double* __restrict__ z, int use_bj) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
  if (!use_bj) {
    z[3 * i] = r0, z[3 * i + 1] = r1, z[3 * i + 2] = r2;
    return;
  }
  const double* d = dinv + 9 * i;
  z[3 * i] = d[0] * r0 + d[1] * r1 + d[2] * r2;
  z[3 * i + 1] = d[3] * r0 + d[4] * r1 + d[5] * r2;
  z[3 * i + 2] = d[6] * r0 + d[7] * r1 + d[8] * r2;
}

// Partial dot products: out[3b] = a.b, out[3b+1] = a.c, out[3b+2] = a.a (c may equal b)
__global__ void k_qs_dots(int64_t m, const double* __restrict__ a, const double* __restrict__ b,
                          const double* __restrict__ c, double* __restrict__ partial) {
  __shared__ double s[3][kQsBlock];
  double ab = 0.0, ac = 0.0, aa = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
    const double va = a[k];
    ab += va * b[k];
    ac += va * c[k];
    aa += va * va;
  }
  s[0][threadIdx.x] = ab;
  s[1][threadIdx.x] = ac;
  s[2][threadIdx.x] = aa;
  __syncthreads();
  for (int o = kQsBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) partial[3 * blockIdx.x + k] = s[k][0];
}

// x += alpha p ; r -= alpha q   (alpha = scal[0]/scal[1])
__global__ void k_qs_axpy2(int64_t m, const double* __restrict__ scal, const double4* __restrict__ w,
                           const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double alpha = scal[0] / scal[1];
  const double4 p = w[k / 3];
  const int c = (int)(k % 3);
  const double pk = c == 0 ? p.x : (c == 1 ? p.y : p.z);
  x[k] += alpha * pk;
  r[k] -= alpha * q[k];
}

// p = z + beta p  with beta = scal[2]/scal[0] (flexible: (z.r - z.r_old)/rz_old folded by the host)
__global__ void k_qs_update_p(int64_t n, const double* __restrict__ scal, const double* __restrict__ z,
                              double4* __restrict__ w, int first) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = w[i];
  if (first) {  // p = z; the previous direction is not read (it may be unset)
    p.x = z[3 * i];
    p.y = z[3 * i + 1];
    p.z = z[3 * i + 2];
  } else {
    const double beta = scal[3];
    p.x = z[3 * i] + beta * p.x;
    p.y = z[3 * i + 1] + beta * p.y;
    p.z = z[3 * i + 2] + beta * p.z;
  }
  w[i] = p;
}

__global__ void k_qs_set_scalars(double* scal, const double* red, int what) {
  // scal: [0] r.z, [1] p.q, [3] beta, [4] r.r; red: [0] z.r, [2] r.r of the new
  // residual, [4] z.q (flexible only).
  // what 0: scal[1] = p.q ; what 1: beta = rz_new/rz_old (Fletcher-Reeves on the
  // preconditioned residual); what 2: flexible beta = max(0, z_new.(r_new -
  // r_old)/rz_old) with z_new.r_old = z_new.r_new + alpha z_new.q (Polak-Ribiere).
  if (threadIdx.x != 0) return;
  if (what == 0) {
    scal[1] = red[0];
  } else if (what == 1) {
    const double rz_new = red[0];
    scal[3] = rz_new / scal[0];
    scal[0] = rz_new;
    scal[4] = red[2];
  } else {
    const double rz_old = scal[0];
    const double alpha = __ddiv_rn(rz_old, scal[1]);
    const double zr_new = red[0];
    const double zr_old = __dadd_rn(zr_new, __dmul_rn(alpha, red[4]));
    const double beta = __ddiv_rn(__dsub_rn(zr_new, zr_old), rz_old);
    scal[3] = beta > 0.0 ? beta : 0.0;  // also 0 for a NaN beta
    scal[0] = zr_new;
    scal[2] = 0.0;
    scal[4] = red[2];
  }
}

__global__ void k_qs_axpy(int64_t m, double a, const double* __restrict__ x, double* __restrict__ y) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) y[k] += a * x[k];
}

__global__ void k_qs_apply_bc(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ a,
                              const double* __restrict__ b, const double2* __restrict__ fcp, double tc, double tp,
                              const double* __restrict__ u, double* __restrict__ du) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c)
    if ((mask[i] >> c) & 1) {
      const int64_t k = 3 * i + c;
      // DirichletIncrementBC coeff 1 (Peridigm_BoundaryCondition.cpp:235); a
      // zero increment takes the previous value from the displacement
      // (:137-142); function dofs (mask bit 3 + c) from their values at the
      // two times (fcp)
      double cur, prev;
      if (fcp && ((mask[i] >> (c + 3)) & 1)) {
        cur = fcp[k].x, prev = fcp[k].y;
      } else {
        cur = a[k] * tc + b[k], prev = a[k] * tp + b[k];
      }
      const double d = cur - prev;
      du[k] = d == 0.0 ? cur - u[k] : d;
    }
}

__global__ void k_qs_finish(int64_t m, double inv_dt, const double* __restrict__ du, double* __restrict__ u,
                            double* __restrict__ v) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  u[k] += du[k];
  v[k] = du[k] * inv_dt;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static unsigned g1(int64_t m) { return (unsigned)((m + kQsBlock - 1) / kQsBlock); }
static unsigned gt(int64_t n) { return (unsigned)((n * kQsTpo + kQsBlock - 1) / kQsBlock); }

static int qs_alloc(pd_ctx* c) {
  if (!c->qs) c->qs = new QsState();
  QsState* s = c->qs;
  if (s->n == c->n) return PD_OK;
  const int64_t n = c->n;
  PD_CUDA_TRY(c, s->yq.alloc(n));
  PD_CUDA_TRY(c, s->abq.alloc(n));
  PD_CUDA_TRY(c, s->w.alloc(n));
  PD_CUDA_TRY(c, s->th.alloc(n));
  PD_CUDA_TRY(c, s->nd.alloc(n));
  for (auto* b : {&s->f, &s->r, &s->du, &s->x, &s->z, &s->q, &s->pred}) PD_CUDA_TRY(c, b->alloc(3 * n));
  PD_CUDA_TRY(c, s->dinv.alloc(9 * n));
  PD_CUDA_TRY(c, s->partial.alloc(3 * (size_t)std::max<int64_t>(kRedBlocks, gt(n)) + 8));
  PD_CUDA_TRY(c, s->scal.alloc(16));
  PD_CUDA_TRY(c, s->fixed.alloc(n));
  PD_CUDA_TRY(c, dzero(c, s->pred.p, s->pred.bytes()));
  s->n = n;
  return PD_OK;
}

const uint8_t* qs_fixed_mask(const pd_ctx* c) { return c->qs ? c->qs->fixed.p : nullptr; }

void qs_release(pd_ctx* c) {
  delete c->qs;
  c->qs = nullptr;
}

// Residual at y = x + u + du; returns ||r||_2 and ||r||_inf.
static int qs_residual(pd_ctx* c, double* l2, double* linf) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  k_qs_positions<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->xv.p, c->u.p, s->du.p, s->yq.p);
  PD_CUDA_TRY(c, launch_fp64_eval_at(c, s->yq.p, s->abq.p, s->th.p, s->nd.p, s->f.p));
  s->geo_dirty = true;
  k_qs_residual<<<kRedBlocks, kQsBlock, 0, c->stream>>>(n, s->f.p, c->xv.p, s->fixed.p, s->r.p, s->partial.p);
  k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 2, 1, s->scal.p + 8);
  PD_CUDA_TRY(c, cudaGetLastError());
  double h[2];
  PD_CUDA_TRY(c, cudaMemcpyAsync(h, s->scal.p + 8, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *l2 = std::sqrt(h[0]);
  *linf = h[1];
  if (!std::isfinite(*l2)) {
    c->err = "NaN returned by force evaluation";
    return PD_ERR_NONFINITE;
  }
  return PD_OK;
}

// z = M r: block Jacobi, plus the coarse correction (two-level), plus the
// network's correction (learned).
static int qs_apply_precond(pd_ctx* c, int precond, const double* r, double* z) {
  QsState* s = c->qs;
  k_qs_precond<<<g1(c->n), kQsBlock, 0, c->stream>>>(c->n, s->dinv.p, r, z, precond != PD_PRECOND_NONE);
  PD_CUDA_TRY(c, cudaGetLastError());
  if (precond == PD_PRECOND_MPNN) TRY_RC(mpnn_apply_add(c, r, z));
  if (s->coarse_on && (precond == PD_PRECOND_MPNN || precond == PD_PRECOND_TWO_LEVEL))
    TRY_RC(coarse_apply_add(c, r, z, s->fixed.p));
  return PD_OK;
}

// Tangent-vector product q = K w.xyz (w.w receives q dtheta) on the per-bond
// geometry, rebuilt first when the state changed.
static int qs_geometry(pd_ctx* c) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  if (s->geo_dirty || s->geo.count < (size_t)c->nb) {
    if (s->geo.count < (size_t)c->nb) {
      PD_CUDA_TRY(c, s->geo.alloc((size_t)c->nb));
      PD_CUDA_TRY(c, s->gco.alloc((size_t)c->nb));
    }
    k_qs_bond_geom<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, s->yq.p, s->abq.p,
                                                      c->hp.p, c->influence, s->geo.p, s->gco.p);
    s->geo_dirty = false;
  }
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

static int qs_tangent(pd_ctx* c) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  TRY_RC(qs_geometry(c));
  k_qs_dtheta_g<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, s->geo.p, s->abq.p, c->pt.p, s->w.p);
  k_qs_df_g<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, s->geo.p, s->gco.p, c->xv.p, s->w.p,
                                               s->fixed.p, s->q.p, s->partial.p, c->pt.p, s->jk, s->jm);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// Preconditioned CG on K x = r (Belos BlockCG in the reference). Flexible
// (Polak-Ribiere) beta when the preconditioner is not a fixed linear operator.
__global__ void k_qs_true_residual(int64_t m, const double* __restrict__ b, const double* __restrict__ q,
                                   double* __restrict__ r) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) r[k] = b[k] - q[k];
}

__global__ void k_qs_x_to_w(int64_t n, const double* __restrict__ x, double4* __restrict__ w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  w[i] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], 0.0);
}

static void k_qs_pack_x(int64_t n, QsState* s, pd_ctx* c) {
  k_qs_x_to_w<<<g1(n), kQsBlock, 0, c->stream>>>(n, s->x.p, s->w.p);
}

static int qs_cg_run(pd_ctx* c, int precond, double rel_tol, int max_it, int* iters, double* rel_out,
                     bool* stalled);

// CG with the learned preconditioner first and 3x3 block Jacobi (the
// reference's "Block 3x3") as the fallback: when the flexible iteration
// stalls, or when the true FP64 residual |b - K x| (recomputed, not the
// recursive one) misses the tolerance, the solve restarts from the current x
// with block Jacobi. The true residual decides.
static int qs_cg(pd_ctx* c, int precond, double rel_tol, int max_it, int* iters, double* rel_out) {
  QsState* s = c->qs;
  const int64_t m = 3 * c->n;
  if (precond != PD_PRECOND_MPNN) {
    bool stalled = false;
    return qs_cg_run(c, precond, rel_tol, max_it, iters, rel_out, &stalled);
  }
  if (s->cg_b.count < (size_t)m) PD_CUDA_TRY(c, s->cg_b.alloc(m));
  if (s->cg_x0.count < (size_t)m) PD_CUDA_TRY(c, s->cg_x0.alloc(m));
  DBuf<double>& b = s->cg_b;
  DBuf<double>& x0 = s->cg_x0;
  PD_CUDA_TRY(c, cudaMemcpyAsync(b.p, s->r.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  bool stalled = false;
  int its = 0;
  double rel = 0.0;
  int rc = qs_cg_run(c, PD_PRECOND_MPNN, rel_tol, max_it, &its, &rel, &stalled);
  if (rc != PD_OK && rc != PD_ERR_NOT_CONVERGED && rc != PD_ERR_NONFINITE) return rc;
  TRY_RC(mpnn_check_status(c));
  // true residual r = b - K x
  const int64_t n = c->n;
  k_qs_pack_x(n, s, c);
  TRY_RC(qs_tangent(c));
  k_qs_true_residual<<<g1(m), kQsBlock, 0, c->stream>>>(m, b.p, s->q.p, s->r.p);
  k_qs_dots<<<kRedBlocks, kQsBlock, 0, c->stream>>>(m, s->r.p, s->r.p, b.p, s->partial.p);
  k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 3, 0, s->scal.p + 8);
  double h[3];
  PD_CUDA_TRY(c, cudaMemcpyAsync(h, s->scal.p + 8, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  k_qs_dots<<<kRedBlocks, kQsBlock, 0, c->stream>>>(m, b.p, b.p, b.p, s->partial.p);
  k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 3, 0, s->scal.p + 12);
  double hb[3];
  PD_CUDA_TRY(c, cudaMemcpyAsync(hb, s->scal.p + 12, sizeof(hb), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const double true_rel = hb[0] > 0 ? std::sqrt(h[0] / hb[0]) : 0.0;

  if (std::isfinite(true_rel) && true_rel <= rel_tol && !stalled) {
    *iters = its;
    *rel_out = true_rel;
    return PD_OK;
  }
  // fall back: block Jacobi on the remaining system K dx = b - K x (x kept when finite)
  c->qs_fallbacks += 1;
  if (!std::isfinite(true_rel)) {
    PD_CUDA_TRY(c, cudaMemsetAsync(s->x.p, 0, m * sizeof(double), c->stream));
    PD_CUDA_TRY(c, cudaMemcpyAsync(s->r.p, b.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  PD_CUDA_TRY(c, cudaMemcpyAsync(x0.p, s->x.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  // the remaining system is solved to the tolerance relative to |b|
  const double tol2 = (std::isfinite(true_rel) && true_rel > 0) ? std::min(1.0, rel_tol / true_rel) : rel_tol;
  int its2 = 0;
  double rel2 = 0.0;
  rc = qs_cg_run(c, PD_PRECOND_BLOCK_JACOBI, tol2, max_it, &its2, &rel2, &stalled);
  k_qs_axpy<<<g1(m), kQsBlock, 0, c->stream>>>(m, 1.0, x0.p, s->x.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  *iters = its + its2;
  *rel_out = rel2 * (std::isfinite(true_rel) && true_rel > 0 ? true_rel : 1.0);
  return rc;
}

static int qs_cg_run(pd_ctx* c, int precond, double rel_tol, int max_it, int* iters, double* rel_out,
                     bool* stalled) {
  QsState* s = c->qs;
  const int64_t n = c->n, m = 3 * n;
  const bool flexible = precond == PD_PRECOND_MPNN;
  const int every =
      (precond == PD_PRECOND_BLOCK_JACOBI || precond == PD_PRECOND_TWO_LEVEL) ? mpnn_capture_every(c) : 0;
  double best = 1.0;
  int best_it = 0;
  *stalled = false;
  PD_CUDA_TRY(c, cudaMemsetAsync(s->x.p, 0, s->x.bytes(), c->stream));
  TRY_RC(qs_apply_precond(c, precond, s->r.p, s->z.p));
  // scal: [0] rz, [1] pq, [3] beta, [4] rr
  k_qs_dots<<<kRedBlocks, kQsBlock, 0, c->stream>>>(m, s->r.p, s->z.p, s->z.p, s->partial.p);
  k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 3, 0, s->scal.p + 8);
  double h[3];
  PD_CUDA_TRY(c, cudaMemcpyAsync(h, s->scal.p + 8, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const double r0 = std::sqrt(h[2]);
  const double rz = h[0];
  *iters = 0;
  *rel_out = 0.0;
  if (r0 == 0.0) return PD_OK;
  PD_CUDA_TRY(c, cudaMemcpyAsync(s->scal.p, &rz, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_qs_update_p<<<g1(n), kQsBlock, 0, c->stream>>>(n, s->scal.p, s->z.p, s->w.p, 1);
  double rel = 1.0;
  int it = 0;
  if (every > 0) TRY_RC(mpnn_snapshot(c, s->r.p, s->x.p));
  while (it < max_it) {
    TRY_RC(qs_tangent(c));
    k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, (int)gt(n), 1, 0, s->scal.p + 8);
    k_qs_set_scalars<<<1, 32, 0, c->stream>>>(s->scal.p, s->scal.p + 8, 0);
    k_qs_axpy2<<<g1(m), kQsBlock, 0, c->stream>>>(m, s->scal.p, s->w.p, s->q.p, s->x.p, s->r.p);
    TRY_RC(qs_apply_precond(c, precond, s->r.p, s->z.p));
    k_qs_dots<<<kRedBlocks, kQsBlock, 0, c->stream>>>(m, s->r.p, s->z.p, s->z.p, s->partial.p);
    k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 3, 0, s->scal.p + 8);
    if (flexible) {  // z_new.q for beta = z_new.(r_new - r_old)/rz_old, r_old = r_new + alpha q
      k_qs_dots<<<kRedBlocks, kQsBlock, 0, c->stream>>>(m, s->z.p, s->q.p, s->q.p, s->partial.p);
      k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 3, 0, s->scal.p + 12);
    }
    k_qs_set_scalars<<<1, 32, 0, c->stream>>>(s->scal.p, s->scal.p + 8, flexible ? 2 : 1);
    double rr;  // the only host read of the iteration: |r|^2 for the stopping test
    PD_CUDA_TRY(c, cudaMemcpyAsync(&rr, s->scal.p + 4, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    rel = std::sqrt(rr) / r0;
    ++it;
    if (!std::isfinite(rel)) {
      if (every > 0) mpnn_drop_snapshots(c);
      c->err = "CG diverged (non-finite residual)";
      return PD_ERR_NONFINITE;
    }
    if (rel <= rel_tol) break;
    if (every > 0 && it % every == 0) TRY_RC(mpnn_snapshot(c, s->r.p, s->x.p));
    if (flexible) {  // stall: no 10x decrease of the residual over 60 iterations
      if (rel < 0.1 * best) best = rel, best_it = it;
      if (it - best_it > 60) {
        *stalled = true;
        break;
      }
    }
    k_qs_update_p<<<g1(n), kQsBlock, 0, c->stream>>>(n, s->scal.p, s->z.p, s->w.p, 0);
  }
  PD_CUDA_TRY(c, cudaGetLastError());
  if (every > 0) {
    if (rel <= rel_tol) TRY_RC(mpnn_commit_snapshots(c, s->x.p, s->dinv.p));
    else mpnn_drop_snapshots(c);
  }
  *iters = it;
  *rel_out = rel;
  return rel <= rel_tol ? PD_OK : PD_ERR_NOT_CONVERGED;
}

__global__ void k_qs_pack_w(int64_t n, const double* __restrict__ w, const uint8_t* __restrict__ fixed,
                            double4* __restrict__ w4) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t f = fixed[i];
  w4[i] = make_double4((f & 1) ? 0.0 : w[3 * i], (f & 2) ? 0.0 : w[3 * i + 1], (f & 4) ? 0.0 : w[3 * i + 2], 0.0);
}

__global__ void k_qs_fixed_rows(int64_t n, const double* __restrict__ w, const uint8_t* __restrict__ fixed,
                                double* __restrict__ q) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c)
    if ((fixed[i] >> c) & 1) q[3 * i + c] = w[3 * i + c];
}

static int qs_prepare_at(pd_ctx* c, const double* u_dev) {
  TRY_RC(ensure_ready_internal(c));
  if (c->material_model != PD_MATERIAL_LPS) {
    c->err = "the quasi-static solve supports the LPS material model only";
    return PD_ERR_UNSUPPORTED;
  }
  if (c->phantoms) {
    c->err = "the implicit and quasi-static solves need symmetric bond families (one horizon across the blocks)";
    return PD_ERR_UNSUPPORTED;
  }
  TRY_RC(qs_alloc(c));
  QsState* s = c->qs;
  const int64_t n = c->n;
  std::vector<uint8_t> fx(n, 0);
  for (int64_t i = 0; i < n; ++i) fx[i] = c->h_bc_mask.empty() ? 0 : (uint8_t)(c->h_bc_mask[i] & 7);  // the coordinates held
  PD_CUDA_TRY(c, cudaMemcpyAsync(s->fixed.p, fx.data(), n, cudaMemcpyHostToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemsetAsync(s->du.p, 0, 3 * n * sizeof(double), c->stream));
  k_qs_positions<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->xv.p, u_dev, s->du.p, s->yq.p);
  PD_CUDA_TRY(c, launch_fp64_eval_at(c, s->yq.p, s->abq.p, s->th.p, s->nd.p, s->f.p));
  s->geo_dirty = true;
  k_qs_qm<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->pt.p, s->abq.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// Matrix-free tangent K w at displacement u (prescribed rows/columns identity).
int qs_tangent_apply(pd_ctx* c, const double* u_dev, const double* w_dev, double* kw_dev) {
  TRY_RC(qs_prepare_at(c, u_dev));
  QsState* s = c->qs;
  const int64_t n = c->n;
  k_qs_pack_w<<<g1(n), kQsBlock, 0, c->stream>>>(n, w_dev, s->fixed.p, s->w.p);
  TRY_RC(qs_tangent(c));
  k_qs_fixed_rows<<<g1(n), kQsBlock, 0, c->stream>>>(n, w_dev, s->fixed.p, s->q.p);
  PD_CUDA_TRY(c, cudaMemcpyAsync(kw_dev, s->q.p, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return PD_OK;
}

// 3x3 diagonal blocks of K at displacement u (row-major, 9 per point).
int qs_tangent_blocks(pd_ctx* c, const double* u_dev, double* blocks_dev) {
  TRY_RC(qs_prepare_at(c, u_dev));
  QsState* s = c->qs;
  const int64_t n = c->n;
  k_qs_block_diag<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, s->yq.p, s->abq.p,
                                                     c->pt.p, c->hp.p, c->influence, s->fixed.p, blocks_dev, 0);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// Tangent at the context's current displacement, for repeated products.
int qs_prepare_current(pd_ctx* c) { return qs_prepare_at(c, c->u.p); }

// Block-Jacobi inverse blocks at the tangent prepared by qs_prepare_current.
int qs_block_jacobi_current(pd_ctx* c, const double** dinv_out) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  k_qs_block_diag<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, s->yq.p, s->abq.p,
                                                     c->pt.p, c->hp.p, c->influence, s->fixed.p, s->dinv.p, 1);
  PD_CUDA_TRY(c, cudaGetLastError());
  *dinv_out = s->dinv.p;
  return PD_OK;
}

// Coarse operator at the tangent prepared by qs_prepare_current.
int qs_build_coarse_current(pd_ctx* c, double cell) {
  QsState* s = c->qs;
  TRY_RC(coarse_build(c, s->yq.p, s->abq.p, s->fixed.p, cell, nullptr));
  s->coarse_on = true;
  s->coarse_rebuild = true;  // the next load step builds its own
  return PD_OK;
}

// Coarse space at displacement u: size, aggregates, assembled matrix and inverse (device buffers, may be null).
int qs_coarse_operator(pd_ctx* c, const double* u_dev, double cell, int64_t* n_coarse, int32_t* agg_dev,
                       double* A_dev, double* Ainv_dev) {
  TRY_RC(qs_prepare_at(c, u_dev));
  QsState* s = c->qs;
  TRY_RC(coarse_build(c, s->yq.p, s->abq.p, s->fixed.p, cell, A_dev));
  s->coarse_rebuild = true;
  *n_coarse = coarse_size(c);
  if (agg_dev) TRY_RC(coarse_aggregates(c, agg_dev));
  if (Ainv_dev) TRY_RC(coarse_copy_inverse(c, Ainv_dev));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return PD_OK;
}

// kw = K w with the tangent prepared by qs_prepare_current.
int qs_apply_K(pd_ctx* c, const double* w_dev, double* kw_dev) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  k_qs_pack_w<<<g1(n), kQsBlock, 0, c->stream>>>(n, w_dev, s->fixed.p, s->w.p);
  TRY_RC(qs_tangent(c));
  k_qs_fixed_rows<<<g1(n), kQsBlock, 0, c->stream>>>(n, w_dev, s->fixed.p, s->q.p);
  PD_CUDA_TRY(c, cudaMemcpyAsync(kw_dev, s->q.p, 3 * n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return PD_OK;
}

// Tangent products of kQsMulti vectors at once (the probes of the rigid coarse
// space): the bond geometry is streamed once for all of them. p and q hold the
// vectors point-major, p[(i * kQsMulti + v) * 3 + c]; prescribed components of
// p are dropped; prescribed rows of q = p. dth [kQsMulti n] scratch.
__global__ void __launch_bounds__(kQsBlock) k_qs_dtheta_multi(int64_t n, const int64_t* __restrict__ row,
                                                              const int32_t* __restrict__ col,
                                                              const double4* __restrict__ g,
                                                              const double4* __restrict__ ab,
                                                              const double4* __restrict__ pt,
                                                              const uint8_t* __restrict__ fixed,
                                                              const double* __restrict__ p, double* __restrict__ dth) {
  constexpr int NV = kQsMulti;
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kQsTpo;
  const int lane = threadIdx.x & (kQsTpo - 1);
  const bool valid = i < n;
  double acc[NV];
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
  if (valid) {
    double pi[NV][3];
    const uint8_t fi = fixed[i];
    for (int v = 0; v < NV; ++v)
      for (int c = 0; c < 3; ++c) pi[v][c] = ((fi >> c) & 1) ? 0.0 : p[(i * NV + v) * 3 + c];
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += kQsTpo) {
      const double4 gb = g[b];
      const int32_t j = col[b];
      const uint8_t fj = fixed[j];
      const double* pj = p + (int64_t)j * NV * 3;
      for (int v = 0; v < NV; ++v) {
        const double w0 = ((fj & 1) ? 0.0 : pj[3 * v]) - pi[v][0];
        const double w1 = ((fj & 2) ? 0.0 : pj[3 * v + 1]) - pi[v][1];
        const double w2 = ((fj & 4) ? 0.0 : pj[3 * v + 2]) - pi[v][2];
        acc[v] += gb.w * (gb.x * w0 + gb.y * w1 + gb.z * w2);
      }
    }
  }
  for (int v = 0; v < NV; ++v) acc[v] = qs_group_sum(acc[v]);
  if (valid && lane == 0) {
    const double s = 3.0 * (ab[i].y / pt[i].x);
    for (int v = 0; v < NV; ++v) dth[i * NV + v] = s * acc[v];
  }
}

__global__ void __launch_bounds__(kQsBlock) k_qs_df_multi(int64_t n, const int64_t* __restrict__ row,
                                                          const int32_t* __restrict__ col,
                                                          const double4* __restrict__ g,
                                                          const double2* __restrict__ gc,
                                                          const double4* __restrict__ xv,
                                                          const uint8_t* __restrict__ fixed,
                                                          const double* __restrict__ p,
                                                          const double* __restrict__ dth, double* __restrict__ q) {
  constexpr int NV = kQsMulti;
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kQsTpo;
  const int lane = threadIdx.x & (kQsTpo - 1);
  const bool valid = i < n;
  double d[NV][3];
  for (int v = 0; v < NV; ++v) d[v][0] = d[v][1] = d[v][2] = 0.0;
  uint8_t fi = 0;
  if (valid) {
    double pi[NV][3], ti[NV];
    fi = fixed[i];
    for (int v = 0; v < NV; ++v) {
      ti[v] = dth[i * NV + v];
      for (int c = 0; c < 3; ++c) pi[v][c] = ((fi >> c) & 1) ? 0.0 : p[(i * NV + v) * 3 + c];
    }
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += kQsTpo) {
      const double4 gb = g[b];
      const double2 cb = gc[b];
      const int32_t j = col[b];
      const uint8_t fj = fixed[j];
      const double* pj = p + (int64_t)j * NV * 3;
      const double* tj = dth + (int64_t)j * NV;
      for (int v = 0; v < NV; ++v) {
        const double w0 = ((fj & 1) ? 0.0 : pj[3 * v]) - pi[v][0];
        const double w1 = ((fj & 2) ? 0.0 : pj[3 * v + 1]) - pi[v][1];
        const double w2 = ((fj & 4) ? 0.0 : pj[3 * v + 2]) - pi[v][2];
        const double de = gb.x * w0 + gb.y * w1 + gb.z * w2;
        const double sy = gb.w * (ti[v] + tj[v]) + (cb.y - cb.x) * de;
        d[v][0] += sy * gb.x + cb.x * w0;
        d[v][1] += sy * gb.y + cb.x * w1;
        d[v][2] += sy * gb.z + cb.x * w2;
      }
    }
  }
  for (int v = 0; v < NV; ++v)
    for (int c = 0; c < 3; ++c) d[v][c] = qs_group_sum(d[v][c]);
  if (valid && lane < 3) {
    const int c = lane;
    const double V = xv[i].w;
    for (int v = 0; v < NV; ++v) {
      const int64_t k = (i * NV + v) * 3 + c;
      const double dv = c == 0 ? d[v][0] : (c == 1 ? d[v][1] : d[v][2]);
      q[k] = ((fi >> c) & 1) ? p[k] : -V * dv;
    }
  }
}

// q = K p for kQsMulti vectors (point-major, see k_qs_dtheta_multi) with the
// tangent prepared by qs_prepare_current; dth [kQsMulti n] scratch.
int qs_apply_K_multi(pd_ctx* c, const double* p_dev, double* q_dev, double* dth_dev) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  TRY_RC(qs_geometry(c));
  k_qs_dtheta_multi<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, s->geo.p, s->abq.p, c->pt.p,
                                                       s->fixed.p, p_dev, dth_dev);
  k_qs_df_multi<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, s->geo.p, s->gco.p, c->xv.p, s->fixed.p,
                                                   p_dev, dth_dev, q_dev);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

int qs_load_step(pd_ctx* c, double t_prev, double t_cur, const pd_qs_options* o, pd_stats* st) {
  TRY_RC(ensure_ready_internal(c));
  if (c->material_model != PD_MATERIAL_LPS) {
    c->err = "the quasi-static solve supports the LPS material model only";
    return PD_ERR_UNSUPPORTED;
  }
  if (c->phantoms) {
    c->err = "the implicit and quasi-static solves need symmetric bond families (one horizon across the blocks)";
    return PD_ERR_UNSUPPORTED;
  }
  TRY_RC(qs_alloc(c));
  QsState* s = c->qs;
  const int64_t n = c->n, m = 3 * n;
  const int precond = o->preconditioner;
  if (precond == PD_PRECOND_MPNN && !mpnn_ready(c)) {
    c->err = "the learned preconditioner is not trained (pd_mpnn_train) or loaded";
    return PD_ERR_STATE;
  }
  // prescribed dofs and their increments (DirichletIncrementBC on deltaU)
  std::vector<uint8_t> fx(n, 0);
  for (int64_t i = 0; i < n; ++i) fx[i] = c->h_bc_mask.empty() ? 0 : (uint8_t)(c->h_bc_mask[i] & 7);  // the coordinates held
  PD_CUDA_TRY(c, cudaMemcpyAsync(s->fixed.p, fx.data(), n, cudaMemcpyHostToDevice, c->stream));
  const double dt = t_cur - t_prev;
  const bool predict = o->use_predictor && st && st->steps > 0;
  // prescribed functions of x, y, z, t: their values at the two times
  const double2* fcp = nullptr;
  if (c->n_bc_expr && c->has_bc) {
    PD_CUDA_TRY(c, launch_bc_expr_at(c, t_cur, t_prev));
    fcp = c->bc_cp.p;
  }
  double l2, linf;
  // Negative tolerance: relative to the metric of this load step's start
  // without the predictor (prescribed increments only), the scale of the load
  // increment; the predicted start can sit close to the FP64 floor.
  double ref_metric = 0.0;
  if (o->newton_tolerance < 0.0 || !predict) {
    PD_CUDA_TRY(c, cudaMemsetAsync(s->du.p, 0, m * sizeof(double), c->stream));
    if (c->has_bc)
      k_qs_apply_bc<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->bc_mask.p, c->bc_a.p, c->bc_b.p, fcp, t_cur, t_prev,
                                                        c->u.p, s->du.p);
    TRY_RC(qs_residual(c, &l2, &linf));
    ref_metric = l2 + 20.0 * linf;
  }
  if (predict) {
    PD_CUDA_TRY(c, cudaMemcpyAsync(s->du.p, s->pred.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (c->has_bc)
      k_qs_apply_bc<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->bc_mask.p, c->bc_a.p, c->bc_b.p, fcp, t_cur, t_prev,
                                                        c->u.p, s->du.p);
    TRY_RC(qs_residual(c, &l2, &linf));
  }
  double metric = l2 + 20.0 * linf;
  const double newton_tol = o->newton_tolerance < 0.0 ? -o->newton_tolerance * ref_metric : o->newton_tolerance;
  int newton = 0, cg_total = 0;
  int64_t coarse_builds = 0;
  double last_rel = 0.0;
  const int64_t fallbacks0 = c->qs_fallbacks;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  const bool two_level =
      precond == PD_PRECOND_TWO_LEVEL || (precond == PD_PRECOND_MPNN && mpnn_coarse_cell(c) >= 0.0);
  const double cell = precond == PD_PRECOND_MPNN ? mpnn_coarse_cell(c) : o->coarse_cell;
  s->coarse_on = false;
  while (metric > newton_tol && newton < o->max_newton_iterations) {
    if (precond != PD_PRECOND_NONE) {
      k_qs_qm<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->pt.p, s->abq.p);
      k_qs_block_diag<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, s->yq.p, s->abq.p,
                                                         c->pt.p, c->hp.p, c->influence, s->fixed.p, s->dinv.p, 1);
      PD_CUDA_TRY(c, cudaGetLastError());
      if (precond == PD_PRECOND_MPNN) TRY_RC(mpnn_prepare(c, s->dinv.p));
    }
    if (two_level) {
      if (s->coarse_rebuild || !coarse_valid(c) || s->coarse_cell != std::max(0.0, cell)) {
        TRY_RC(coarse_build(c, s->yq.p, s->abq.p, s->fixed.p, std::max(0.0, cell), nullptr));
        s->coarse_cell = std::max(0.0, cell);
        s->coarse_ref_iters = -1;
        s->coarse_rebuild = false;
        ++coarse_builds;
      }
      s->coarse_on = true;
    }
    int its = 0;
    double rel = 0.0;
    int rc = qs_cg(c, precond, o->cg_relative_tolerance, o->max_cg_iterations, &its, &rel);
    cg_total += its;
    last_rel = rel;
    if (two_level) {
      // rebuild when a solve needs clearly more iterations than the first one
      // after the last build: 1.3x + 5 for the translations (a build costs a
      // few CG iterations), 2x + 10 with the rotations (a build costs ~150)
      const bool rigid = c->coarse_modes == 6;
      if (s->coarse_ref_iters < 0) s->coarse_ref_iters = its;
      else if (its > (rigid ? 2 * s->coarse_ref_iters + 10 : (13 * s->coarse_ref_iters) / 10 + 5))
        s->coarse_rebuild = true;
    }
    if (rc != PD_OK && rc != PD_ERR_NOT_CONVERGED) return rc;
    // du += alpha * x, backtracking on the convergence metric
    double alpha = 1.0, prev = metric;
    k_qs_axpy<<<g1(m), kQsBlock, 0, c->stream>>>(m, alpha, s->x.p, s->du.p);
    TRY_RC(qs_residual(c, &l2, &linf));
    metric = l2 + 20.0 * linf;
    for (int k = 0; k < 8 && !(metric < prev); ++k) {
      k_qs_axpy<<<g1(m), kQsBlock, 0, c->stream>>>(m, -0.5 * alpha, s->x.p, s->du.p);
      alpha *= 0.5;
      TRY_RC(qs_residual(c, &l2, &linf));
      metric = l2 + 20.0 * linf;
    }
    ++newton;
  }
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // commit: u += du, v = du/dt (Peridigm.cpp:2858-2862); predictor for the next step
  k_qs_finish<<<g1(m), kQsBlock, 0, c->stream>>>(m, dt != 0.0 ? 1.0 / dt : 0.0, s->du.p, c->u.p, c->v.p);
  PD_CUDA_TRY(c, cudaMemcpyAsync(s->pred.p, s->du.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->f.p, s->f.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->theta.p, s->th.p, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  c->cur = 0;
  PD_CUDA_TRY(c, launch_sync_state(c));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (st) {
    st->steps += 1;
    st->newton_iterations += newton;
    st->cg_iterations += cg_total;
    st->final_residual = last_rel;
    st->preconditioner_fallbacks += c->qs_fallbacks - fallbacks0;
    st->coarse_builds += coarse_builds;
    st->device_ms += ms;
    st->bonds = c->nb_user;
  }
  if (metric > newton_tol) {
    c->err = "quasi-static Newton iteration did not reach its tolerance";
    return PD_ERR_NOT_CONVERGED;
  }
  return PD_OK;
}

// ---------------------------------------------------------------------------
// Implicit dynamics (Peridigm::executeImplicit, src/core/Peridigm.cpp:3620-4016):
// Newmark-beta steps, each solved by Newton on R = beta dt^2 (rho a - f) with
// the prescribed rows zeroed, the operator rho I + beta dt^2 K
// (computeImplicitJacobian :4319-4338, K = -d(V f)/du as in the quasi-static
// tangent) applied matrix-free, CG on it (Belos BlockCG in the reference).
// Vector updates follow the reference's Epetra Update/Scale order, without
// fused multiply-adds.
// ---------------------------------------------------------------------------
// u2 = un + dt vn + cu an, v2 = vn + cv an (:3726-3730); u = u2, a = (u - u2)
// * (1/(beta dt^2)) = 0, v = v2 + dt gamma a = v2 (:3752-3759).
__global__ void k_imp_predict(int64_t m, double dt, double cu, double cv, double* __restrict__ u,
                              double* __restrict__ v, double* __restrict__ a, double* __restrict__ u2,
                              double* __restrict__ v2) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double un = u[k], vn = v[k], an = a[k];
  const double p = __dadd_rn(__dadd_rn(un, __dmul_rn(dt, vn)), __dmul_rn(cu, an));
  const double q = __dadd_rn(vn, __dmul_rn(cv, an));
  u2[k] = p;
  v2[k] = q;
  u[k] = p;
  a[k] = 0.0;
  v[k] = q;
}

// u += du; a = (u - u2) * (1/(beta dt^2)); v = v2 + dt gamma a (:3893-3902).
__global__ void k_imp_correct(int64_t m, double ibdt2, double dtg, const double* __restrict__ du,
                              double* __restrict__ u, const double* __restrict__ u2, double* __restrict__ a,
                              const double* __restrict__ v2, double* __restrict__ v) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const double uu = __dadd_rn(u[k], du[k]);
  const double aa = __dmul_rn(__dsub_rn(uu, u2[k]), ibdt2);
  u[k] = uu;
  a[k] = aa;
  v[k] = __dadd_rn(v2[k], __dmul_rn(dtg, aa));
}

// R = beta dt^2 (rho a - f) (:3803-3806) with the prescribed rows zeroed
// (:3810); rhs = -R for J du = -R; block partials (sum R^2, max |R|).
__global__ void k_imp_residual(int64_t n, double bdt2, const double* __restrict__ f, const double* __restrict__ a,
                               const double4* __restrict__ pt, const uint8_t* __restrict__ fixed,
                               double* __restrict__ rhs, double* __restrict__ partial) {
  __shared__ double s2[kQsBlock], sm[kQsBlock];
  double a2 = 0.0, am = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < 3 * n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k / 3;
    const int c = (int)(k - 3 * i);
    double r = __dmul_rn(bdt2, __dsub_rn(__dmul_rn(pt[i].w, a[k]), f[k]));
    if ((fixed[i] >> c) & 1) r = 0.0;
    rhs[k] = -r;
    a2 += r * r;
    am = fmax(am, fabs(r));
  }
  s2[threadIdx.x] = a2;
  sm[threadIdx.x] = am;
  __syncthreads();
  for (int o = kQsBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s2[threadIdx.x] += s2[threadIdx.x + o];
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s2[0];
    partial[2 * blockIdx.x + 1] = sm[0];
  }
}

// Prescribed dofs at the run's start: u = a t0 + b, v = a (the rate).
__global__ void k_imp_bc_start(int64_t n, const uint8_t* __restrict__ mask, const double* __restrict__ ba,
                               const double* __restrict__ bb, double t0, double* __restrict__ u,
                               double* __restrict__ v, double* __restrict__ a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c)
    if ((mask[i] >> c) & 1) {
      const int64_t k = 3 * i + c;
      u[k] = ba[k] * t0 + bb[k];
      v[k] = ba[k];
      a[k] = 0.0;
    }
}

// Force density at x + u (frozen bond damage) and the residual norm ||R||_2.
static int imp_residual(pd_ctx* c, double bdt2, double* norm) {
  QsState* s = c->qs;
  const int64_t n = c->n;
  k_qs_positions<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->xv.p, c->u.p, s->du.p, s->yq.p);
  PD_CUDA_TRY(c, launch_fp64_eval_at(c, s->yq.p, s->abq.p, s->th.p, s->nd.p, s->f.p));
  s->geo_dirty = true;
  k_imp_residual<<<kRedBlocks, kQsBlock, 0, c->stream>>>(n, bdt2, s->f.p, c->a.p, c->pt.p, s->fixed.p, s->r.p,
                                                         s->partial.p);
  k_qs_reduce<<<1, kQsBlock, 0, c->stream>>>(s->partial.p, kRedBlocks, 2, 1, s->scal.p + 8);
  PD_CUDA_TRY(c, cudaGetLastError());
  double h[2];
  PD_CUDA_TRY(c, cudaMemcpyAsync(h, s->scal.p + 8, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *norm = std::sqrt(h[0]);
  if (!std::isfinite(*norm)) {
    c->err = "NaN returned by force evaluation";
    return PD_ERR_NONFINITE;
  }
  return PD_OK;
}

int implicit_run(pd_ctx* c, double dt, double t0, int64_t nsteps, const pd_implicit_options* o, pd_stats* st) {
  TRY_RC(ensure_ready_internal(c));
  if (c->material_model != PD_MATERIAL_LPS) {
    c->err = "the implicit solve supports the LPS material model only";
    return PD_ERR_UNSUPPORTED;
  }
  if (c->n_bc_expr) {
    c->err = "prescribed displacement functions of x, y, z, t run on the explicit and quasi-static paths; give "
             "the implicit solve a*t + b";
    return PD_ERR_UNSUPPORTED;
  }
  if (c->phantoms) {
    c->err = "the implicit and quasi-static solves need symmetric bond families (one horizon across the blocks)";
    return PD_ERR_UNSUPPORTED;
  }
  TRY_RC(qs_alloc(c));
  QsState* s = c->qs;
  const int64_t n = c->n, m = 3 * n;
  PD_CUDA_TRY(c, s->v2.alloc(m));
  std::vector<uint8_t> fx(n, 0);
  for (int64_t i = 0; i < n; ++i) fx[i] = c->h_bc_mask.empty() ? 0 : (uint8_t)(c->h_bc_mask[i] & 7);  // the coordinates held
  PD_CUDA_TRY(c, cudaMemcpyAsync(s->fixed.p, fx.data(), n, cudaMemcpyHostToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemsetAsync(s->du.p, 0, m * sizeof(double), c->stream));
  if (c->has_bc)
    k_imp_bc_start<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->bc_mask.p, c->bc_a.p, c->bc_b.p, t0, c->u.p, c->v.p,
                                                      c->a.p);
  const double beta = o->beta, gamma = o->gamma;
  const double dt2 = dt * dt, bdt2 = beta * dt2, ibdt2 = 1.0 / bdt2, dtg = dt * gamma;
  const double cu = 0.5 * dt2 * (1.0 - 2.0 * beta), cv = dt * (1.0 - gamma);
  s->jk = bdt2;
  s->jm = 1.0;
  s->coarse_on = false;
  const int precond = o->preconditioner;
  int64_t newton_total = 0, cg_total = 0;
  double last_rel = 0.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  int rc = PD_OK;
  for (int64_t step = 0; step < nsteps && rc == PD_OK; ++step) {
    k_imp_predict<<<g1(m), kQsBlock, 0, c->stream>>>(m, dt, cu, cv, c->u.p, c->v.p, c->a.p, s->pred.p, s->v2.p);
    double norm = 0.0;
    rc = imp_residual(c, bdt2, &norm);
    int it = 0;
    while (rc == PD_OK && norm > o->absolute_tolerance && it <= o->max_newton_iterations) {
      if (precond == PD_PRECOND_BLOCK_JACOBI) {
        k_qs_qm<<<g1(n), kQsBlock, 0, c->stream>>>(n, c->pt.p, s->abq.p);
        k_qs_block_diag<<<gt(n), kQsBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, s->yq.p,
                                                           s->abq.p, c->pt.p, c->hp.p, c->influence, s->fixed.p,
                                                           s->dinv.p, 1, s->jk, s->jm);
      }
      int its = 0;
      double rel = 0.0;
      bool stalled = false;
      const int r2 = qs_cg_run(c, precond, o->cg_relative_tolerance, o->max_cg_iterations, &its, &rel, &stalled);
      if (r2 != PD_OK && r2 != PD_ERR_NOT_CONVERGED) {  // a CG that stops short is used as it is (:3870-3872)
        rc = r2;
        break;
      }
      cg_total += its;
      last_rel = rel;
      k_imp_correct<<<g1(m), kQsBlock, 0, c->stream>>>(m, ibdt2, dtg, s->x.p, c->u.p, s->pred.p, c->a.p, s->v2.p,
                                                       c->v.p);
      rc = imp_residual(c, bdt2, &norm);
      ++it;
    }
    newton_total += it;
  }
  s->jk = 1.0;
  s->jm = 0.0;
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != PD_OK) return rc;
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->f.p, s->f.p, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(c->theta.p, s->th.p, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  c->cur = 0;
  PD_CUDA_TRY(c, launch_sync_state(c));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (st) {
    st->steps += nsteps;
    st->newton_iterations += newton_total;
    st->cg_iterations += cg_total;
    st->final_residual = last_rel;
    st->device_ms += ms;
    st->bonds = c->nb_user;
  }
  return PD_OK;
}

}  // namespace pdb
