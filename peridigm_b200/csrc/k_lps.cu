// LPS elastic + critical-stretch damage + velocity-Verlet kernels (sm_100a).
//
// Two bond passes per evaluation, both gathers, no atomics:
//   pass 1 (k_dilatation_*): per bond, critical-stretch test and the
//     dilatation term; per point theta, node damage and the owner force-state
//     terms the second pass gathers.
//   pass 2 (k_force_*): per bond f_i += (t_ij + t_ji) * Y/|Y| * V_j, the gather
//     form of the reference's scatter (elastic.cxx:125-130: the owner adds
//     t_ij*Y*V_j, the neighbor's own loop subtracts t_ji*(-Y)*V_j), followed
//     by the Verlet epilogue of Peridigm::executeExplicit (Peridigm.cpp:1480-1577).
// A group of TPO consecutive lanes owns one point's bond family; lanes stride
// through the row (coalesced col/damage loads), partial sums are combined by
// a fixed xor-shuffle tree, so results are deterministic.
//
// Split-FP32 path data:
//   bx[b] = (X, omega*V_j)             per bond, streamed: X = fp32(x_j - x_i)
//                                      formed in FP64, rounded once
//   ur[j] = (u_hi[3], u_lo[3], A, B)   per point, one 256-bit gather per bond;
//                                      u_hi = fp32(u), u_lo = fp32(u - u_hi)
// du = (u_hi_j - u_hi_i) + (u_lo_j - u_lo_i) is the displacement difference to
// within one FP32 ulp, with no FP64 instruction in the bond loop. The FP64
// displacement u[3n] stays the integration state.
#include <math.h>

#include <cub/cub.cuh>

#include "pd_internal.cuh"

namespace pdb {

constexpr int kBlock = 256;

// ---------------------------------------------------------------------------
// Influence functions (src/core/Peridigm_InfluenceFunction.hpp:69-87)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double omega_d(int kind, double zeta, double h) {
  if (kind == PD_INFLUENCE_ONE) return 1.0;
  if (kind == PD_INFLUENCE_PARABOLIC_DECAY) {
    if (zeta > h) return 0.0;
    double s = __ddiv_rn(zeta, h);
    return s < 0.5 ? 1.0 : __dadd_rn(__dmul_rn(__dmul_rn(-4.0, s), s), __dmul_rn(4.0, s));
  }
  double h2 = __dmul_rn(__dmul_rn(__dmul_rn(h, h), 0.4), 0.4);
  return exp(-__ddiv_rn(__dmul_rn(zeta, zeta), h2));
}

// Squared distance exactly as the reference computes it (dx*dx+dy*dy)+dz*dz,
// with no fused multiply-add, so FP64 distances round like the reference's.
__device__ __forceinline__ double sq3_rn(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

template <int TPO, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = TPO / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// 256-bit record loads. nc: read-only path, for data no thread writes during
// the kernel. The coherent form is used where another lane of the same kernel
// writes other bytes of the same records.
__device__ __forceinline__ Rec8 ld_rec_nc(const Rec8* p) {
  Rec8 r;
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]), "=f"(r.v[6]),
        "=f"(r.v[7])
      : "l"(p));
  return r;
}
__device__ __forceinline__ Rec8 ld_rec(const Rec8* p) {
  Rec8 r;
  asm("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]), "=f"(r.v[4]), "=f"(r.v[5]), "=f"(r.v[6]),
        "=f"(r.v[7])
      : "l"(p));
  return r;
}

__device__ __forceinline__ void split_hi_lo(double v, float* hi, float* lo) {
  const float h = __double2float_rn(v);
  *hi = h;
  *lo = __double2float_rn(v - (double)h);
}

// Bond geometry of the split path from the bond's stored X (FP32, q.xyz) and
// the two endpoints' displacement records. Identical operations in both passes;
// with both endpoints swapped X, du and Y are exactly negated (X_ji = -X_ij is
// rounded from an exactly negated FP64 difference), so e and |X| are identical
// and bond damage stays symmetric.
struct SplitBond {
  float Yx, Yy, Yz, zeta, ry, e, xu, xx;  // xu = X.du, xx = |X|^2 (the linear LPS terms)
};
__device__ __forceinline__ SplitBond split_bond(const float4& q, const Rec8& ui, const Rec8& uj) {
  SplitBond s;
  const float Ux = (uj.v[0] - ui.v[0]) + (uj.v[3] - ui.v[3]);
  const float Uy = (uj.v[1] - ui.v[1]) + (uj.v[4] - ui.v[4]);
  const float Uz = (uj.v[2] - ui.v[2]) + (uj.v[5] - ui.v[5]);
  const float xx = fmaf(q.z, q.z, fmaf(q.y, q.y, q.x * q.x));
  s.Yx = q.x + Ux;
  s.Yy = q.y + Uy;
  s.Yz = q.z + Uz;
  const float yy = fmaf(s.Yz, s.Yz, fmaf(s.Yy, s.Yy, s.Yx * s.Yx));
  s.ry = rsqrtf(yy);
  s.zeta = xx * rsqrtf(xx);
  const float dY = yy * s.ry;
  const float xu = fmaf(q.z, Uz, fmaf(q.y, Uy, q.x * Ux));
  const float uu = fmaf(Uz, Uz, fmaf(Uy, Uy, Ux * Ux));
  s.e = __fdividef(fmaf(2.0f, xu, uu), dY + s.zeta);  // |Y| - |X| without cancellation
  s.xu = xu;
  s.xx = xx;
  return s;
}

// Streaming loads of bond-ordered data (read once per pass; kept out of L1 so
// the neighbor records stay resident there).
//
// The split passes walk a row kUnroll bonds per lane at a time: first the
// bond-ordered loads of the batch (damage, neighbor id, X), all independent,
// then the batch's neighbor-record gathers, then the arithmetic. Loads do not
// wait on the damage byte, so each lane keeps 2*kUnroll loads in flight
// instead of a damage -> id -> record chain per bond.
// Batch depth and the launch bound were swept on the 320,000-point notched
// plate (1, 2 or 4 bonds per batch; 4 or 6 resident blocks per SM): with the
// sliced stream loaded straight into registers, 4 bonds per batch and 4
// blocks per SM (64 registers per thread, no shared memory) are the fastest.
// (Staging the stream through shared memory by cp.async paid off only while
// the stream was row-major; once each warp load is 32 consecutive records,
// direct loads are faster: the force pass 139 -> 126 us on that plate.)
// The neighbor ids of the next batch are loaded one batch ahead, so a batch's
// gathers never wait on its own id loads (dilatation 130 -> 114 us). Neither a
// bulk L2 prefetch of the next 1 to 4 batches of the sliced streams (one lane
// per warp, cp.async.bulk.prefetch) nor carrying the damage flag in the top
// bit of the sliced ids instead of a damage byte made the passes faster.
#ifndef PD_BOND_UNROLL
#define PD_BOND_UNROLL 4
#endif
#ifndef PD_BOND_MINB
#define PD_BOND_MINB 8
#endif
constexpr int kUnroll = PD_BOND_UNROLL;
// Threads per block of the split bond passes: 8 blocks of 128 fill an SM's
// 1024 threads at 64 registers, and the last partial wave of a ~5000-block
// grid costs half of what it does with 256-thread blocks.
constexpr int kSplitBlock = 128;

// Bond-stream cursor of a lane. CSR: the owner's row, the lane's bonds TPO
// apart. Sliced (4 lanes per point, SELL): the bonds of the 8 owners of a
// warp interleaved so that one warp load is 32 consecutive records
// (record of owner o, row offset r at soff[s]*32 + (r/4)*32 + 4o + r%4), each
// row padded with dummy bonds (damage byte 2) to the slice's longest row.
template <int TPO, bool SELL>
__device__ __forceinline__ void bond_cursor(int64_t i, int lane, int64_t b0, int64_t b1,
                                            const int64_t* __restrict__ soff, int64_t* base, int* left) {
  if (SELL) {
    const int64_t s = i >> 3, so = soff[s];
    *base = so * 32 + (i & 7) * 4 + lane;
    *left = (int)(soff[s + 1] - so);
  } else {
    const int rem = (int)(b1 - b0) - lane;
    *base = b0 + lane;
    *left = rem > 0 ? (rem + TPO - 1) / TPO : 0;
  }
}

// ---------------------------------------------------------------------------
// K1: weighted volume m_i = sum_j omega*|xi|^2*V_j (material_utilities.cxx:161-188)
// ---------------------------------------------------------------------------
template <int TPO>
__global__ void __launch_bounds__(kBlock) k_weighted_volume(int64_t n, const int64_t* __restrict__ row,
                                                            const int32_t* __restrict__ col,
                                                            const double4* __restrict__ xv,
                                                            const double* __restrict__ hp, int influence,
                                                            double4* __restrict__ pt) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double acc = 0.0;
  if (valid) {
    const double4 xi = xv[i];
    const double h = hp[i];
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += TPO) {
      const double4 xj = xv[col[b]];
      const double z2 = sq3_rn(__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z));
      const double om = omega_d(influence, __dsqrt_rn(z2), h);
      acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(om, z2), xj.w));
    }
  }
  acc = group_sum<TPO>(acc);
  if (valid && lane == 0) pt[i].x = acc;
}

// Split-path owner terms own = (3/m, (3K-5mu)/m, 15mu/m, s_c).
__global__ void k_pack_owner(int64_t n, const double4* __restrict__ pt, const double* __restrict__ sc,
                             float4* __restrict__ own) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pt[i];  // (m, K, mu, rho)
  own[i] = make_float4((float)(3.0 / p.x), (float)((3.0 * p.y - 5.0 * p.z) / p.x), (float)(15.0 * p.z / p.x),
                       (float)sc[i]);
}

// Split-path bond stream bx = (X = x_j - x_i, omega(|X|, h_i) * V_j): the
// difference and the influence weight in FP64, each rounded once to FP32. In
// CSR order (SELL false), or in the sliced order of bond_cursor (SELL true,
// with the neighbor ids and damage bytes copied alongside).
__device__ __forceinline__ int64_t sell_index(const int64_t* __restrict__ soff, int64_t i, int64_t r) {
  return soff[i >> 3] * 32 + (r >> 2) * 32 + (i & 7) * 4 + (r & 3);
}

template <int TPO, bool SELL>
__global__ void __launch_bounds__(kBlock) k_pack_bonds(int64_t n, const int64_t* __restrict__ row,
                                                       const int32_t* __restrict__ col,
                                                       const double4* __restrict__ xv,
                                                       const double* __restrict__ hp, int influence,
                                                       float4* __restrict__ bx, const int64_t* __restrict__ soff,
                                                       const uint8_t* __restrict__ dmg, int32_t* __restrict__ scol,
                                                       uint8_t* __restrict__ sdmg) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  if (i >= n) return;
  const double4 xi = xv[i];
  const double h = hp[i];
  const int64_t b0 = row[i];
  for (int64_t b = b0 + lane; b < row[i + 1]; b += TPO) {
    const int32_t j = col[b];
    const double4 xj = xv[j];
    const double dx = __dsub_rn(xj.x, xi.x), dy = __dsub_rn(xj.y, xi.y), dz = __dsub_rn(xj.z, xi.z);
    const double om = omega_d(influence, __dsqrt_rn(sq3_rn(dx, dy, dz)), h);
    const float4 rec = make_float4((float)dx, (float)dy, (float)dz, (float)__dmul_rn(om, xj.w));
    if (SELL) {
      const int64_t k = sell_index(soff, i, b - b0);
      bx[k] = rec;
      scol[k] = j;
      sdmg[k] = dmg[b];
    } else {
      bx[b] = rec;
    }
  }
  if (SELL) {  // padding to the slice's longest row: dummy bonds, damage byte 2
    const int64_t len = row[i + 1] - b0, ms = soff[(i >> 3) + 1] - soff[i >> 3];
    for (int64_t r = len + lane; r < 4 * ms; r += TPO) {
      const int64_t k = sell_index(soff, i, r);
      bx[k] = make_float4(1.f, 0.f, 0.f, 0.f);
      scol[k] = (int32_t)i;
      sdmg[k] = 2;
    }
  }
}

// Slots per slice (groups of 4 bonds of its longest row).
__global__ void k_sell_count(int64_t n, const int64_t* __restrict__ row, int64_t* __restrict__ cnt) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ns = (n + 7) / 8;
  if (s > ns) return;
  int64_t m = 0;
  if (s < ns)
    for (int o = 0; o < 8; ++o) {
      const int64_t i = 8 * s + o;
      if (i < n) m = max(m, (row[i + 1] - row[i] + 3) / 4);
    }
  cnt[s] = m;
}

// The sliced damage mirror from the CSR damage (after writes outside the passes).
__global__ void __launch_bounds__(kBlock) k_sell_dmg(int64_t n, const int64_t* __restrict__ row,
                                                     const int64_t* __restrict__ soff,
                                                     const uint8_t* __restrict__ dmg, uint8_t* __restrict__ sdmg) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / 4;
  const int lane = threadIdx.x & 3;
  if (i >= n) return;
  const int64_t b0 = row[i];
  for (int64_t b = b0 + lane; b < row[i + 1]; b += 4) sdmg[sell_index(soff, i, b - b0)] = dmg[b];
}

// ---------------------------------------------------------------------------
// K2: damage + dilatation, split-FP32.
//   break when e > s_c*|X|, i.e. (|Y|-|X|)/|X| > s_c (CriticalStretchDamageModel.cpp:155-158)
//   theta_i = 3/m_i * sum omega*(1-d)*|X|*e*V_j  (material_utilities.cxx:284)
// Writes the owner terms A_i = theta_i*(3K-5mu)/m, B_i = 15mu/m into ur[i].
// ---------------------------------------------------------------------------
template <int TPO, bool SELL, bool LIN = false>
__global__ void __launch_bounds__(kSplitBlock, PD_BOND_MINB) k_dilatation_split(
    int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
    const float4* __restrict__ bx, Rec8* __restrict__ ur, const float4* __restrict__ own, int damage_on,
    double* __restrict__ theta_out, double* __restrict__ node_damage, const int64_t* __restrict__ soff,
    uint8_t* __restrict__ dmg_csr) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  float th = 0.0f;
  int broken = 0;
  int len = 0;
  if (valid) {
    const int64_t b0 = row[i];
    len = (int)(row[i + 1] - b0);
    const Rec8 ui = ld_rec(ur + i);
    const float s_c = damage_on ? own[i].w : -1.0f;
    // Branch-free masking (selects) of past-the-end and broken bonds; the
    // batch's bond-ordered loads first (independent), then its gathers.
    constexpr int kS = SELL ? 32 : TPO;
    int64_t base;
    int left;
    bond_cursor<TPO, SELL>(i, lane, b0, b0 + len, soff, &base, &left);
    const float4* nbx = bx + base;
    const int32_t* ncol = col + base;
    uint8_t* pdm = dmg + base;
    uint8_t* cdm = SELL ? dmg_csr + b0 + lane : nullptr;  // the lane's bonds in the canonical CSR damage
    int32_t jn[kUnroll];  // neighbor ids of the next batch, loaded one batch ahead
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) jn[k] = k < left ? __ldcs(ncol + kS * k) : (int32_t)i;
#pragma unroll 1
    for (; left > 0; left -= kUnroll, pdm += kUnroll * kS, nbx += kUnroll * kS, ncol += kUnroll * kS,
                     cdm += SELL ? kUnroll * TPO : 0) {
      int dd[kUnroll];
      float4 qq[kUnroll];
      int32_t jj[kUnroll];
      Rec8 uu[kUnroll];
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        jj[k] = jn[k];
        jn[k] = k + kUnroll < left ? __ldcs(ncol + kS * (k + kUnroll)) : (int32_t)i;
      }
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const bool in = k < left;
        dd[k] = in ? (int)pdm[kS * k] : 2;  // 2: past the row end
        qq[k] = in ? __ldcs(nbx + kS * k) : make_float4(1.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) uu[k] = ld_rec(ur + jj[k]);
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const float4 q = qq[k];
        const SplitBond sb = split_bond(q, ui, uu[k]);
        const bool intact = dd[k] == 0;
        const bool brk = intact && s_c >= 0.0f && sb.e > s_c * sb.zeta;
        if (brk) {
          pdm[kS * k] = 1;
          if (SELL) cdm[TPO * k] = 1;  // the CSR copy stays canonical
        }
        broken += (dd[k] == 1 || brk) ? 1 : 0;
        // LPS: omega V_j |X| e; linear LPS: omega V_j X.du
        th = fmaf((intact && !brk) ? (LIN ? q.w : q.w * sb.zeta) : 0.0f, LIN ? sb.xu : sb.e, th);
      }
    }
  }
  th = group_sum<TPO>(th);
  broken = group_sum<TPO>(broken);
  if (valid && lane == 0) {
    const float4 ow = own[i];
    const float theta = th * ow.x;
    *reinterpret_cast<float2*>(&ur[i].v[6]) = make_float2(theta * ow.y, ow.z);
    theta_out[i] = (double)theta;
    node_damage[i] = len > 0 ? (double)broken / (double)len : 0.0;
  }
}

// ---------------------------------------------------------------------------
// K2: damage + dilatation, FP64, the reference's operation order:
//   rel = (|Y|-|X|)/|X| > s_c                     (CriticalStretchDamageModel.cpp:147-158)
//   theta += 3*omega*(1-d)*|X|*e*V_j/m_i           (material_utilities.cxx:284)
// Writes ab64[i] = (theta, 3K/m - alpha/3, alpha) (elastic.cxx:99,119).
// ---------------------------------------------------------------------------
template <int TPO>
__global__ void __launch_bounds__(kBlock) k_dilatation_fp64(
    int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
    const double4* __restrict__ xv, const double4* __restrict__ st, const double4* __restrict__ pt,
    const double* __restrict__ sc, const double* __restrict__ hp, int influence, int damage_on,
    double4* __restrict__ ab64, double* __restrict__ theta_out, double* __restrict__ node_damage) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double th = 0.0;
  int broken = 0;
  int64_t b0 = 0, b1 = 0;
  double m = 1.0;
  if (valid) {
    b0 = row[i];
    b1 = row[i + 1];
    const double4 xi = xv[i];
    const double4 yi = st[i];
    m = pt[i].x;
    const double s_c = damage_on ? sc[i] : -1.0;
    const double h = hp[i];
    for (int64_t b = b0 + lane; b < b1; b += TPO) {
      if (dmg[b]) {
        broken++;
        continue;
      }
      const int32_t j = col[b];
      const double4 xj = xv[j];
      const double4 yj = st[j];
      const double zeta = __dsqrt_rn(sq3_rn(__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z)));
      const double dY = __dsqrt_rn(sq3_rn(__dsub_rn(yj.x, yi.x), __dsub_rn(yj.y, yi.y), __dsub_rn(yj.z, yi.z)));
      if (s_c >= 0.0 && __ddiv_rn(__dsub_rn(dY, zeta), zeta) > s_c) {
        dmg[b] = 1;
        broken++;
        continue;
      }
      const double e = __dsub_rn(dY, zeta);
      const double om = omega_d(influence, zeta, h);
      // 3.0*omega*(1.0-d)*d*e*cellVolume/m with d = 0
      double t = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(3.0, om), zeta), e), xj.w);
      th = __dadd_rn(th, __ddiv_rn(t, m));
    }
  }
  th = group_sum<TPO>(th);
  broken = group_sum<TPO>(broken);
  if (valid && lane == 0) {
    const double4 p = pt[i];
    const double alpha = __ddiv_rn(__dmul_rn(15.0, p.z), p.x);
    const double q = __dsub_rn(__ddiv_rn(__dmul_rn(3.0, p.y), p.x), __ddiv_rn(alpha, 3.0));
    ab64[i] = make_double4(th, q, alpha, 0.0);
    theta_out[i] = th;
    node_damage[i] = (b1 > b0) ? (double)broken / (double)(b1 - b0) : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Verlet epilogue shared by both precisions. Lane c (< 3) of the group handles
// component c of point i; f is the internal force density of that component.
// Order of Peridigm::executeExplicit: f += f_contact (Peridigm.cpp:1567),
// a = (f + f_ext)/rho (:1569-1573), v += dt/2*a (:1577); then the next step's
// v += dt/2*a (:1480), kinematic BC (:1486, DirichletIncrementBC
// Peridigm_BoundaryCondition.cpp:232-237), y = x+u+dt*v (:1497), u += dt*v (:1501).
// FP64 operations use explicit round-to-nearest intrinsics (no contraction)
// so the state rounds like the reference's scalar build.
// ---------------------------------------------------------------------------
struct EpiArgs {
  double dt, t0;
  int64_t step;  // evaluation index: 0 = initial evaluation at t0, s = step s
  int mode;
  int has_contact, has_bc, split;
  const double* fc;
  double* f_out;
  double* u;  // FP64 displacement [3n]
  double* v;
  double* a;
  const uint8_t* bc_mask;
  const double* bc_a;
  const double* bc_b;
  double4* st_next;  // FP64 path: next coordinates
  Rec8* ur_next;     // split path: next displacement record
  int* status;
};

__device__ __forceinline__ double comp3(const double4& q, int c) { return c == 0 ? q.x : (c == 1 ? q.y : q.z); }
__device__ __forceinline__ double* comp_ptr(double4* q, int c) {
  return c == 0 ? &q->x : (c == 1 ? &q->y : &q->z);
}

__device__ __forceinline__ void verlet_epilogue(const EpiArgs& E, int64_t i, int c, double f, double xc,
                                                double rho) {
  const int64_t k = 3 * i + c;
  double ftot = f;
  if (E.has_contact) ftot = __dadd_rn(ftot, E.fc[k]);
  if (!isfinite(ftot)) atomicOr(E.status, ST_NONFINITE_FORCE);
  if (E.f_out) E.f_out[k] = ftot;
  if (E.mode == EVAL_ONLY) return;
  const double dt = E.dt, dt2 = E.dt / 2.0;
  const double acc = __ddiv_rn(__dadd_rn(ftot, 0.0), rho);
  double v = E.v[k];
  if (E.step > 0) v = __dadd_rn(v, __dmul_rn(dt2, acc));  // end of step (none after the initial evaluation)
  if (E.mode == EVAL_LAST) {
    E.v[k] = v;
    E.a[k] = acc;
    return;
  }
  // first half of step s+1
  double vh = __dadd_rn(v, __dmul_rn(dt2, acc));
  if (E.has_bc && ((E.bc_mask[i] >> c) & 1)) {
    const double tc = __dadd_rn(E.t0, __dmul_rn((double)(E.step + 1), dt));
    const double tp = E.step == 0 ? E.t0 : __dadd_rn(E.t0, __dmul_rn((double)E.step, dt));
    if (tc != tp) {
      const double cur = __dadd_rn(__dmul_rn(E.bc_a[k], tc), E.bc_b[k]);
      const double prev = __dadd_rn(__dmul_rn(E.bc_a[k], tp), E.bc_b[k]);
      const double d = __dsub_rn(cur, prev);
      vh = __dadd_rn(__dmul_rn(0.0, d), __dmul_rn(__dmul_rn(1.0, d), __ddiv_rn(1.0, __dsub_rn(tc, tp))));
    }
  }
  E.v[k] = vh;
  E.a[k] = acc;
  const double step_dx = __dmul_rn(dt, vh);
  const double u = E.u[k];
  const double un = __dadd_rn(u, step_dx);  // u += dt*v
  E.u[k] = un;
  if (E.split) {
    float hi, lo;
    split_hi_lo(un, &hi, &lo);
    E.ur_next[i].v[c] = hi;
    E.ur_next[i].v[c + 3] = lo;
  } else {
    *comp_ptr(&E.st_next[i], c) = __dadd_rn(__dadd_rn(xc, u), step_dx);  // y = x+u+dt*v
  }
}

// ---------------------------------------------------------------------------
// K3: force gather, split-FP32:
//   t_ij + t_ji = omega*(|X|*(A_i + A_j) + e*(B_i + B_j))   (bond intact)
//   f_i += (t_ij + t_ji) * V_j * Y/|Y|
// Broken bonds carry t = 0 (elastic.cxx:120 with d = 1) and are skipped.
// ---------------------------------------------------------------------------
template <int TPO, bool SELL, bool LIN = false, bool CHUNK = false>
__global__ void __launch_bounds__(kSplitBlock, PD_BOND_MINB) k_force_split(int64_t n, const int64_t* __restrict__ row,
                                                                      const int32_t* __restrict__ col,
                                                                      const uint8_t* __restrict__ dmg,
                                                                      const float4* __restrict__ bx,
                                                                      const Rec8* __restrict__ ur,
                                                                      const double4* __restrict__ pt, EpiArgs E,
                                                                      const int64_t* __restrict__ soff,
                                                                      int64_t i0 = 0) {
  // CHUNK: owners i0 .. n-1 (a chunk of the points starts at a multiple of 64
  // owners); otherwise i0 is not used and the pass covers 0 .. n-1
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = (CHUNK ? i0 : 0) + g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (valid) {
    const Rec8 ui = ld_rec_nc(ur + i);
    const int64_t b1 = row[i + 1];
    constexpr int kS = SELL ? 32 : TPO;
    const int64_t b0 = row[i];
    int64_t base;
    int left;
    bond_cursor<TPO, SELL>(i, lane, b0, b1, soff, &base, &left);
    const float4* nbx = bx + base;
    const int32_t* ncol = col + base;
    const uint8_t* pdm = dmg + base;
    int32_t jn[kUnroll];  // neighbor ids of the next batch, loaded one batch ahead
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) jn[k] = k < left ? __ldcs(ncol + kS * k) : (int32_t)i;
#pragma unroll 1
    for (; left > 0; left -= kUnroll, pdm += kUnroll * kS, nbx += kUnroll * kS, ncol += kUnroll * kS) {
      bool live[kUnroll];
      float4 qq[kUnroll];
      int32_t jj[kUnroll];
      Rec8 uu[kUnroll];
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        jj[k] = jn[k];
        jn[k] = k + kUnroll < left ? __ldcs(ncol + kS * (k + kUnroll)) : (int32_t)i;
      }
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const bool in = k < left;
        live[k] = in ? pdm[kS * k] == 0 : false;
        qq[k] = in ? __ldcs(nbx + kS * k) : make_float4(1.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) uu[k] = ld_rec_nc(ur + jj[k]);
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const float4 q = qq[k];
        const SplitBond sb = split_bond(q, ui, uu[k]);
        if constexpr (LIN) {
          // omega V_j ((A_i + A_j) X + (B_i + B_j) (X.du / |X|^2) X), along the reference bond X
          const float c = fmaf(ui.v[7] + uu[k].v[7], __fdividef(sb.xu, sb.xx), ui.v[6] + uu[k].v[6]);
          const float w = live[k] ? c * q.w : 0.0f;
          fx = fmaf(w, q.x, fx);
          fy = fmaf(w, q.y, fy);
          fz = fmaf(w, q.z, fz);
        } else {
          const float T = fmaf(sb.zeta, ui.v[6] + uu[k].v[6], sb.e * (ui.v[7] + uu[k].v[7]));
          const float w = live[k] ? T * q.w * sb.ry : 0.0f;
          fx = fmaf(w, sb.Yx, fx);
          fy = fmaf(w, sb.Yy, fy);
          fz = fmaf(w, sb.Yz, fz);
        }
      }
    }
  }
  fx = group_sum<TPO>(fx);
  fy = group_sum<TPO>(fy);
  fz = group_sum<TPO>(fz);
  if (valid && lane < 3) {
    const double f = lane == 0 ? (double)fx : (lane == 1 ? (double)fy : (double)fz);
    verlet_epilogue(E, i, lane, f, 0.0, pt[i].w);
  }
}

// ---------------------------------------------------------------------------
// K3: force gather, FP64, each term in the reference's operation order:
//   c1 = omega*theta*(3K/m - alpha/3); t = c1*|X| + omega*alpha*e   (elastic.cxx:119-120)
//   own term  +  (t_ij*Y)/|Y| * V_j      (elastic.cxx:121-127)
//   neighbor  -  (t_ji*(-Y))/|Y| * V_j   (elastic.cxx:128-130 from j's loop)
// ---------------------------------------------------------------------------
template <int TPO>
__global__ void __launch_bounds__(kBlock) k_force_fp64(int64_t n, const int64_t* __restrict__ row,
                                                       const int32_t* __restrict__ col,
                                                       const uint8_t* __restrict__ dmg,
                                                       const double4* __restrict__ xv,
                                                       const double4* __restrict__ st,
                                                       const double4* __restrict__ ab64,
                                                       const double4* __restrict__ pt,
                                                       const double* __restrict__ hp, int influence,
                                                       EpiArgs E) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  double4 xi = make_double4(0, 0, 0, 0);
  if (valid) {
    xi = xv[i];
    const double4 yi = st[i];
    const double4 ai = ab64[i];  // (theta, q, alpha)
    const double hi = hp[i];
    const int64_t b1 = row[i + 1];
    for (int64_t b = row[i] + lane; b < b1; b += TPO) {
      if (dmg[b]) continue;
      const int32_t j = col[b];
      const double4 xj = xv[j];
      const double4 yj = st[j];
      const double4 aj = ab64[j];
      const double zeta = __dsqrt_rn(sq3_rn(__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z)));
      const double Yx = __dsub_rn(yj.x, yi.x), Yy = __dsub_rn(yj.y, yi.y), Yz = __dsub_rn(yj.z, yi.z);
      const double dY = __dsqrt_rn(sq3_rn(Yx, Yy, Yz));
      const double e = __dsub_rn(dY, zeta);
      const double om_i = omega_d(influence, zeta, hi);
      const double om_j = influence == PD_INFLUENCE_ONE ? 1.0 : omega_d(influence, zeta, hp[j]);
      const double ti = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(om_i, ai.x), ai.y), zeta),
                                  __dmul_rn(__dmul_rn(om_i, ai.z), e));
      const double tj = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(om_j, aj.x), aj.y), zeta),
                                  __dmul_rn(__dmul_rn(om_j, aj.z), e));
      const double V = xj.w;
      fx = __dadd_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yx), dY), V));
      fy = __dadd_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yy), dY), V));
      fz = __dadd_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yz), dY), V));
      fx = __dsub_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yx), dY), V));
      fy = __dsub_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yy), dY), V));
      fz = __dsub_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yz), dY), V));
    }
  }
  fx = group_sum<TPO>(fx);
  fy = group_sum<TPO>(fy);
  fz = group_sum<TPO>(fz);
  if (valid && lane < 3) {
    const double f = lane == 0 ? fx : (lane == 1 ? fy : fz);
    verlet_epilogue(E, i, lane, f, comp3(xi, lane), pt[i].w);
  }
}

// ---------------------------------------------------------------------------
// Linear LPS ("Linear LPS Partial Volume" without partial volumes or improved
// quadrature): the loops PeridigmNS::LinearLPSPVMaterial::precompute and
// ::computeForce run (src/materials/Peridigm_LinearLPSPVMaterial.cpp:231-394),
// FP64, each term in the class's operation order:
//   theta_i = (sum omega (1-d) zeta.(u_j - u_i) V_j) * (3/m_i)          (:283-290)
//   t1 = (9K - 15mu) omega theta_i / (3 m_i), t2 = 15mu omega / (m_i |zeta|^2)
//   f_ij = (1-d) (t1 zeta + t2 (zeta zeta^T)(u_j - u_i))                (:351-362)
//   f_i += f_ij V_j, and from j's loop f_i -= f_ji V_j (:363-385), which in
//   the gather form is + (t1_j zeta + t2_j (zeta zeta^T)(u_j - u_i)) V_j
//   (zeta and u_j - u_i are exactly negated in j's frame).
// The critical-stretch damage test runs first, on the actual stretch.
// ab64[i] = (theta, 9K - 15mu, 15mu, m).
// ---------------------------------------------------------------------------
template <int TPO>
__global__ void __launch_bounds__(kBlock) k_dilatation_lin_fp64(
    int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
    const double4* __restrict__ xv, const double4* __restrict__ st, const double4* __restrict__ pt,
    const double* __restrict__ sc, const double* __restrict__ hp, int influence, int damage_on,
    double4* __restrict__ ab64, double* __restrict__ theta_out, double* __restrict__ node_damage) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double th = 0.0;
  int broken = 0;
  int64_t b0 = 0, b1 = 0;
  if (valid) {
    b0 = row[i];
    b1 = row[i + 1];
    const double4 xi = xv[i];
    const double4 yi = st[i];
    const double s_c = damage_on ? sc[i] : -1.0;
    const double h = hp[i];
    const double ui0 = __dsub_rn(yi.x, xi.x), ui1 = __dsub_rn(yi.y, xi.y), ui2 = __dsub_rn(yi.z, xi.z);
    for (int64_t b = b0 + lane; b < b1; b += TPO) {
      if (dmg[b]) {
        broken++;
        continue;
      }
      const int32_t j = col[b];
      const double4 xj = xv[j];
      const double4 yj = st[j];
      const double z0 = __dsub_rn(xj.x, xi.x), z1 = __dsub_rn(xj.y, xi.y), z2 = __dsub_rn(xj.z, xi.z);
      const double zeta = __dsqrt_rn(sq3_rn(z0, z1, z2));
      if (s_c >= 0.0) {
        const double dY = __dsqrt_rn(sq3_rn(__dsub_rn(yj.x, yi.x), __dsub_rn(yj.y, yi.y), __dsub_rn(yj.z, yi.z)));
        if (__ddiv_rn(__dsub_rn(dY, zeta), zeta) > s_c) {
          dmg[b] = 1;
          broken++;
          continue;
        }
      }
      const double d0 = __dsub_rn(__dsub_rn(yj.x, xj.x), ui0), d1 = __dsub_rn(__dsub_rn(yj.y, xj.y), ui1),
                   d2 = __dsub_rn(__dsub_rn(yj.z, xj.z), ui2);
      const double dot = __dadd_rn(__dadd_rn(__dmul_rn(z0, d0), __dmul_rn(z1, d1)), __dmul_rn(z2, d2));
      const double om = omega_d(influence, zeta, h);
      th = __dadd_rn(th, __dmul_rn(__dmul_rn(om, dot), xj.w));  // omega*(1-d)*dot*V with d = 0
    }
  }
  th = group_sum<TPO>(th);
  broken = group_sum<TPO>(broken);
  if (valid && lane == 0) {
    const double4 p = pt[i];
    if (b1 > b0) th = __dmul_rn(th, __ddiv_rn(3.0, p.x));
    ab64[i] = make_double4(th, __dsub_rn(__dmul_rn(9.0, p.y), __dmul_rn(15.0, p.z)), __dmul_rn(15.0, p.z), p.x);
    theta_out[i] = th;
    node_damage[i] = (b1 > b0) ? (double)broken / (double)(b1 - b0) : 0.0;
  }
}

template <int TPO>
__global__ void __launch_bounds__(kBlock) k_force_lin_fp64(int64_t n, const int64_t* __restrict__ row,
                                                           const int32_t* __restrict__ col,
                                                           const uint8_t* __restrict__ dmg,
                                                           const double4* __restrict__ xv,
                                                           const double4* __restrict__ st,
                                                           const double4* __restrict__ ab64,
                                                           const double4* __restrict__ pt,
                                                           const double* __restrict__ hp, int influence,
                                                           EpiArgs E) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double f[3] = {0.0, 0.0, 0.0};
  double4 xi = make_double4(0, 0, 0, 0);
  if (valid) {
    xi = xv[i];
    const double4 yi = st[i];
    const double4 ai = ab64[i];  // (theta, 9K - 15mu, 15mu, m)
    const double hi = hp[i];
    const double ui0 = __dsub_rn(yi.x, xi.x), ui1 = __dsub_rn(yi.y, xi.y), ui2 = __dsub_rn(yi.z, xi.z);
    const int64_t b1 = row[i + 1];
    for (int64_t b = row[i] + lane; b < b1; b += TPO) {
      if (dmg[b]) continue;
      const int32_t j = col[b];
      const double4 xj = xv[j];
      const double4 yj = st[j];
      const double4 aj = ab64[j];
      const double z[3] = {__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z)};
      const double du[3] = {__dsub_rn(__dsub_rn(yj.x, xj.x), ui0), __dsub_rn(__dsub_rn(yj.y, xj.y), ui1),
                            __dsub_rn(__dsub_rn(yj.z, xj.z), ui2)};
      const double z2 = sq3_rn(z[0], z[1], z[2]);
      const double zeta = __dsqrt_rn(z2);
      const double om_i = omega_d(influence, zeta, hi);
      const double om_j = influence == PD_INFLUENCE_ONE ? 1.0 : omega_d(influence, zeta, hp[j]);
      const double t1i = __ddiv_rn(__dmul_rn(__dmul_rn(ai.y, om_i), ai.x), __dmul_rn(3.0, ai.w));
      const double t2i = __ddiv_rn(__dmul_rn(ai.z, om_i), __dmul_rn(ai.w, z2));
      const double t1j = __ddiv_rn(__dmul_rn(__dmul_rn(aj.y, om_j), aj.x), __dmul_rn(3.0, aj.w));
      const double t2j = __ddiv_rn(__dmul_rn(aj.z, om_j), __dmul_rn(aj.w, z2));
      const double V = xj.w;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double mv = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(z[r], z[0]), du[0]), __dmul_rn(__dmul_rn(z[r], z[1]), du[1])),
                                    __dmul_rn(__dmul_rn(z[r], z[2]), du[2]));
        f[r] = __dadd_rn(f[r], __dmul_rn(__dadd_rn(__dmul_rn(t1i, z[r]), __dmul_rn(t2i, mv)), V));
        f[r] = __dadd_rn(f[r], __dmul_rn(__dadd_rn(__dmul_rn(t1j, z[r]), __dmul_rn(t2j, mv)), V));
      }
    }
  }
  const double fx = group_sum<TPO>(f[0]), fy = group_sum<TPO>(f[1]), fz = group_sum<TPO>(f[2]);
  if (valid && lane < 3) {
    const double fc = lane == 0 ? fx : (lane == 1 ? fy : fz);
    verlet_epilogue(E, i, lane, fc, comp3(xi, lane), pt[i].w);
  }
}

// ---------------------------------------------------------------------------
// Elastic bond-based material (MATERIAL_EVALUATION::computeInternalForceElasticBondBased,
// src/materials/elastic_bond_based.cxx:55-124): one bond pass per evaluation,
// the bond's critical-stretch damage first (CriticalStretchDamageModel order),
// then the pair force of the intact bond
//   t_ij = 0.5 (1 - d) s c_i,  s = (|Y| - |X|)/|X|,
//   c = 18K/(pi delta^4) (3D, :77) or 12K/(pi H delta^3) (plane strain/stress, :75),
//   f_i += (t_ij + t_ji) V_j Y/|Y|   (gather form of the scatter at :118-123),
// then the Verlet epilogue. No dilatation, no influence function.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double bb_constant(double K, double h, int plane, double height) {
  const double pi = 3.14159265358979323846;
  return plane ? __ddiv_rn(__dmul_rn(12.0, K), __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(pi, height), h), h), h))
               : __ddiv_rn(__dmul_rn(18.0, K), __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(pi, h), h), h), h));
}

// Split path: 0.5 c_i of every point in record slot 6 of both state buffers
// (the Verlet epilogue writes only slots 0-5).
__global__ void k_bb_terms(int64_t n, const double4* __restrict__ pt, const double* __restrict__ hp, int plane,
                           double height, Rec8* __restrict__ ur0, Rec8* __restrict__ ur1) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float c = (float)(0.5 * bb_constant(pt[i].y, hp[i], plane, height));
  ur0[i].v[6] = c;
  ur0[i].v[7] = 0.0f;
  ur1[i].v[6] = c;
  ur1[i].v[7] = 0.0f;
}

// FP64 path, each term in the reference's operation order.
template <int TPO>
__global__ void __launch_bounds__(kBlock) k_bb_fp64(int64_t n, const int64_t* __restrict__ row,
                                                    const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
                                                    const double4* __restrict__ xv, const double4* __restrict__ st,
                                                    const double4* __restrict__ pt, const double* __restrict__ sc,
                                                    const double* __restrict__ hp, int damage_on, int plane,
                                                    double height, double* __restrict__ node_damage, EpiArgs E) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  int broken = 0;
  int64_t nbond = 0;
  if (valid) {
    const double4 xi = xv[i], yi = st[i];
    const double ci = bb_constant(pt[i].y, hp[i], plane, height);
    const double s_c = damage_on ? sc[i] : -1.0;
    nbond = row[i + 1] - row[i];
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += TPO) {
      if (dmg[b]) {
        broken++;
        continue;
      }
      const int32_t j = col[b];
      const double4 xj = xv[j], yj = st[j];
      const double zeta = __dsqrt_rn(sq3_rn(__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z)));
      const double Yx = __dsub_rn(yj.x, yi.x), Yy = __dsub_rn(yj.y, yi.y), Yz = __dsub_rn(yj.z, yi.z);
      const double dY = __dsqrt_rn(sq3_rn(Yx, Yy, Yz));
      const double stretch = __ddiv_rn(__dsub_rn(dY, zeta), zeta);
      if (s_c >= 0.0 && stretch > s_c) {
        dmg[b] = 1;
        broken++;
        continue;
      }
      const double cj = bb_constant(pt[j].y, hp[j], plane, height);
      const double ti = __dmul_rn(__dmul_rn(0.5, stretch), ci);  // 0.5*(1-d)*stretch*constant, d = 0
      const double tj = __dmul_rn(__dmul_rn(0.5, stretch), cj);
      const double V = xj.w;
      fx = __dadd_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yx), dY), V));
      fy = __dadd_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yy), dY), V));
      fz = __dadd_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yz), dY), V));
      fx = __dsub_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yx), dY), V));
      fy = __dsub_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yy), dY), V));
      fz = __dsub_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yz), dY), V));
    }
  }
  fx = group_sum<TPO>(fx);
  fy = group_sum<TPO>(fy);
  fz = group_sum<TPO>(fz);
  broken = group_sum<TPO>(broken);
  if (valid && lane == 0) node_damage[i] = nbond > 0 ? (double)broken / (double)nbond : 0.0;
  if (valid && lane < 3) {
    const double4 xi = xv[i];
    const double f = lane == 0 ? fx : (lane == 1 ? fy : fz);
    verlet_epilogue(E, i, lane, f, comp3(xi, lane), pt[i].w);
  }
}

// Split-FP32 path: one pass (bond stream and neighbor ids loaded directly as
// in the LPS passes), damage and pair force per bond, FP64 epilogue.
template <int TPO, bool SELL>
__global__ void __launch_bounds__(kSplitBlock, PD_BOND_MINB) k_bb_split(int64_t n, const int64_t* __restrict__ row,
                                                                   const int32_t* __restrict__ col,
                                                                   uint8_t* __restrict__ dmg,
                                                                   const float4* __restrict__ bx,
                                                                   const Rec8* __restrict__ ur,
                                                                   const float4* __restrict__ own, int damage_on,
                                                                   const double4* __restrict__ pt,
                                                                   double* __restrict__ node_damage, EpiArgs E,
                                                                   const int64_t* __restrict__ soff,
                                                                   uint8_t* __restrict__ dmg_csr) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  int broken = 0;
  int len = 0;
  if (valid) {
    const int64_t b0 = row[i];
    len = (int)(row[i + 1] - b0);
    const Rec8 ui = ld_rec_nc(ur + i);
    const float s_c = damage_on ? own[i].w : -1.0f;
    constexpr int kS = SELL ? 32 : TPO;
    int64_t base;
    int left;
    bond_cursor<TPO, SELL>(i, lane, b0, b0 + len, soff, &base, &left);
    const float4* nbx = bx + base;
    const int32_t* ncol = col + base;
    uint8_t* pdm = dmg + base;
    uint8_t* cdm = SELL ? dmg_csr + b0 + lane : nullptr;  // the lane's bonds in the canonical CSR damage
    int32_t jn[kUnroll];  // neighbor ids of the next batch, loaded one batch ahead
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) jn[k] = k < left ? __ldcs(ncol + kS * k) : (int32_t)i;
#pragma unroll 1
    for (; left > 0; left -= kUnroll, pdm += kUnroll * kS, nbx += kUnroll * kS, ncol += kUnroll * kS,
                     cdm += SELL ? kUnroll * TPO : 0) {
      int dd[kUnroll];
      float4 qq[kUnroll];
      int32_t jj[kUnroll];
      Rec8 uu[kUnroll];
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        jj[k] = jn[k];
        jn[k] = k + kUnroll < left ? __ldcs(ncol + kS * (k + kUnroll)) : (int32_t)i;
      }
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const bool in = k < left;
        dd[k] = in ? (int)pdm[kS * k] : 2;  // 2: past the row end
        qq[k] = in ? __ldcs(nbx + kS * k) : make_float4(1.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) uu[k] = ld_rec_nc(ur + jj[k]);
#pragma unroll
      for (int k = 0; k < kUnroll; ++k) {
        const float4 q = qq[k];
        const SplitBond sb = split_bond(q, ui, uu[k]);
        const bool intact = dd[k] == 0;
        const bool brk = intact && s_c >= 0.0f && sb.e > s_c * sb.zeta;
        if (brk) {
          pdm[kS * k] = 1;
          if (SELL) cdm[TPO * k] = 1;
        }
        broken += (dd[k] == 1 || brk) ? 1 : 0;
        const float t = (ui.v[6] + uu[k].v[6]) * __fdividef(sb.e, sb.zeta);  // t_ij + t_ji
        const float w = (intact && !brk) ? t * q.w * sb.ry : 0.0f;
        fx = fmaf(w, sb.Yx, fx);
        fy = fmaf(w, sb.Yy, fy);
        fz = fmaf(w, sb.Yz, fz);
      }
    }
  }
  fx = group_sum<TPO>(fx);
  fy = group_sum<TPO>(fy);
  fz = group_sum<TPO>(fz);
  broken = group_sum<TPO>(broken);
  if (valid && lane == 0) node_damage[i] = len > 0 ? (double)broken / (double)len : 0.0;
  if (valid && lane < 3) {
    const double f = lane == 0 ? (double)fx : (lane == 1 ? (double)fy : (double)fz);
    verlet_epilogue(E, i, lane, f, 0.0, pt[i].w);
  }
}

// ---------------------------------------------------------------------------
// State conversions and the stable time step
// ---------------------------------------------------------------------------
// State from current coordinates y [3n]: u = y - x (FP64), then the gathered
// copy (split: hi/lo record, FP64: y itself).
__global__ void k_state_from_y(int64_t n, const double* __restrict__ y, const double4* __restrict__ xv,
                               double* __restrict__ u, double4* __restrict__ st, Rec8* __restrict__ ur) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 x = xv[i];
  const double y0 = y[3 * i], y1 = y[3 * i + 1], y2 = y[3 * i + 2];
  const double u0 = y0 - x.x, u1 = y1 - x.y, u2 = y2 - x.z;
  u[3 * i] = u0;
  u[3 * i + 1] = u1;
  u[3 * i + 2] = u2;
  if (ur) {
    split_hi_lo(u0, &ur[i].v[0], &ur[i].v[3]);
    split_hi_lo(u1, &ur[i].v[1], &ur[i].v[4]);
    split_hi_lo(u2, &ur[i].v[2], &ur[i].v[5]);
  } else {
    st[i] = make_double4(y0, y1, y2, 0.0);
  }
}

// Gathered state from the displacement u [3n] (after pd_set_state): split ->
// hi/lo record, FP64 -> y = x + u.
__global__ void k_state_from_u(int64_t n, const double* __restrict__ u, const double4* __restrict__ xv,
                               double4* __restrict__ st, Rec8* __restrict__ ur) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 x = xv[i];
  if (ur) {
    split_hi_lo(u[3 * i], &ur[i].v[0], &ur[i].v[3]);
    split_hi_lo(u[3 * i + 1], &ur[i].v[1], &ur[i].v[4]);
    split_hi_lo(u[3 * i + 2], &ur[i].v[2], &ur[i].v[5]);
  } else {
    st[i] = make_double4(__dadd_rn(x.x, u[3 * i]), __dadd_rn(x.y, u[3 * i + 1]), __dadd_rn(x.z, u[3 * i + 2]), 0.0);
  }
}

// ComputeCriticalTimeStep (Peridigm_CriticalTimeStep.cpp:52-130): per point
// dt_i = sqrt(2 rho / sum_j V_j*k/|xi|), k = 18K/(pi h^4); block minima go to
// partial[] and k_min_reduce takes the minimum (order-independent, exact).
template <int TPO>
__global__ void __launch_bounds__(kBlock) k_critical_dt(int64_t n, const int64_t* __restrict__ row,
                                                        const int32_t* __restrict__ col,
                                                        const double4* __restrict__ xv,
                                                        const double4* __restrict__ pt,
                                                        const double* __restrict__ hp, double* __restrict__ partial) {
  __shared__ double smin[kBlock / TPO];
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double den = 0.0;
  int64_t nn = 0;
  if (valid) {
    const double4 xi = xv[i];
    const double4 p = pt[i];
    const double h = hp[i];
    const double spring =
        __ddiv_rn(__dmul_rn(18.0, p.y), __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(3.14159265358979323846, h), h), h), h));
    nn = row[i + 1] - row[i];
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += TPO) {
      const double4 xj = xv[col[b]];
      const double d = __dsqrt_rn(sq3_rn(__dsub_rn(xi.x, xj.x), __dsub_rn(xi.y, xj.y), __dsub_rn(xi.z, xj.z)));
      den = __dadd_rn(den, __ddiv_rn(__dmul_rn(xj.w, spring), d));
    }
  }
  den = group_sum<TPO>(den);
  double cts = 1.0e50;
  if (valid && nn > 0) cts = __dsqrt_rn(__ddiv_rn(__dmul_rn(2.0, pt[i].w), den));
  if (lane == 0) smin[threadIdx.x / TPO] = cts;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mn = 1.0e50;
    for (int k = 0; k < kBlock / TPO; ++k) mn = fmin(mn, smin[k]);
    partial[blockIdx.x] = mn;
  }
}

__global__ void k_min_reduce(int64_t m, const double* __restrict__ partial, double* __restrict__ out) {
  __shared__ double s[kBlock];
  double mn = 1.0e50;
  for (int64_t k = threadIdx.x; k < m; k += blockDim.x) mn = fmin(mn, partial[k]);
  s[threadIdx.x] = mn;
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] = fmin(s[threadIdx.x], s[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
static inline unsigned grid_for(int64_t n, int tpo) { return (unsigned)((n * tpo + kBlock - 1) / kBlock); }
static inline unsigned grid1(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }
static inline unsigned grid_split(int64_t n, int tpo) {
  return (unsigned)((n * tpo + kSplitBlock - 1) / kSplitBlock);
}

#define PD_DISPATCH_TPO_CSR(tpo, KERNEL, GRID, BLOCK, ...)                          \
  switch (tpo) {                                                                     \
    case 4: KERNEL<4, false><<<GRID, BLOCK, 0, c->stream>>>(__VA_ARGS__); break;     \
    case 8: KERNEL<8, false><<<GRID, BLOCK, 0, c->stream>>>(__VA_ARGS__); break;     \
    case 16: KERNEL<16, false><<<GRID, BLOCK, 0, c->stream>>>(__VA_ARGS__); break;   \
    default: KERNEL<32, false><<<GRID, BLOCK, 0, c->stream>>>(__VA_ARGS__); break;   \
  }

#define PD_DISPATCH_TPO(tpo, KERNEL, GRID, ...)                                      \
  switch (tpo) {                                                                     \
    case 4: KERNEL<4><<<GRID, kBlock, 0, c->stream>>>(__VA_ARGS__); break;           \
    case 8: KERNEL<8><<<GRID, kBlock, 0, c->stream>>>(__VA_ARGS__); break;           \
    case 16: KERNEL<16><<<GRID, kBlock, 0, c->stream>>>(__VA_ARGS__); break;         \
    default: KERNEL<32><<<GRID, kBlock, 0, c->stream>>>(__VA_ARGS__); break;         \
  }

cudaError_t launch_weighted_volume(const pd_ctx* c) {
  if (c->n == 0) return cudaSuccess;
  PD_DISPATCH_TPO(c->tpo, k_weighted_volume, grid_for(c->n, c->tpo), c->n, c->row.p, c->col.p, c->xv.p, c->hp.p,
                  c->influence, c->pt.p);
  return cudaGetLastError();
}

cudaError_t launch_pack_owner(pd_ctx* c) {
  if (c->n == 0 || c->precision != PD_SPLIT_FP32) return cudaSuccess;
  const bool bb = c->material_model == PD_MATERIAL_BOND_BASED;
  const int64_t n = c->n;
  k_pack_owner<<<grid1(n), kBlock, 0, c->stream>>>(n, c->pt.p, c->sc.p, c->own.p);
  // the bond-based material has no influence function: bx.w = V_j
  const int infl = bb ? PD_INFLUENCE_ONE : c->influence;
  c->sell = c->tpo_split == 4;
  if (c->sell) {  // sliced bond stream of the 4-lanes-per-point passes
    const int64_t ns = (n + 7) / 8;
    pdb::DBuf<int64_t> cnt;
    cudaError_t e;
    if ((e = cnt.alloc(ns + 1)) != cudaSuccess) return e;
    if ((e = c->sell_off.alloc(ns + 1)) != cudaSuccess) return e;
    k_sell_count<<<(unsigned)((ns + 1 + kBlock - 1) / kBlock), kBlock, 0, c->stream>>>(n, c->row.p, cnt.p);
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt.p, c->sell_off.p, (int)(ns + 1), c->stream);
    pdb::DBuf<unsigned char> tmp;
    if ((e = tmp.alloc(tmp_bytes)) != cudaSuccess) return e;
    if ((e = cub::DeviceScan::ExclusiveSum(tmp.p, tmp_bytes, cnt.p, c->sell_off.p, (int)(ns + 1), c->stream)) !=
        cudaSuccess)
      return e;
    int64_t slots = 0;
    if ((e = cudaMemcpyAsync(&slots, c->sell_off.p + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream)) !=
        cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return e;
    const size_t recs = (size_t)std::max<int64_t>(32 * slots, 1);
    if ((e = c->bx.alloc(recs)) != cudaSuccess) return e;
    if ((e = c->sell_col.alloc(recs)) != cudaSuccess) return e;
    if ((e = c->sell_dmg.alloc(recs)) != cudaSuccess) return e;
    k_pack_bonds<4, true><<<grid_for(n, 4), kBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->xv.p, c->hp.p, infl,
                                                                    c->bx.p, c->sell_off.p, c->dmg.p, c->sell_col.p,
                                                                    c->sell_dmg.p);
    c->sell_src = c->dmg.p;
    c->sell_gen = c->dmg_gen;
  } else {
    PD_DISPATCH_TPO_CSR(c->tpo, k_pack_bonds, grid_for(n, c->tpo), kBlock, n, c->row.p, c->col.p, c->xv.p, c->hp.p, infl,
                        c->bx.p, nullptr, nullptr, nullptr, nullptr);
  }
  if (bb)
    k_bb_terms<<<grid1(n), kBlock, 0, c->stream>>>(n, c->pt.p, c->hp.p, c->bb_plane, c->bb_height, c->ur[0].p,
                                                   c->ur[1].p);
  return cudaGetLastError();
}

cudaError_t launch_state_from_y(pd_ctx* c, const double* y_dev) {
  if (c->n == 0) return cudaSuccess;
  const bool split = c->precision == PD_SPLIT_FP32;
  k_state_from_y<<<grid1(c->n), kBlock, 0, c->stream>>>(c->n, y_dev, c->xv.p, c->u.p, split ? nullptr : c->st[c->cur].p,
                                                        split ? c->ur[c->cur].p : nullptr);
  return cudaGetLastError();
}

cudaError_t launch_sync_state(pd_ctx* c) {
  if (c->n == 0) return cudaSuccess;
  const bool split = c->precision == PD_SPLIT_FP32;
  k_state_from_u<<<grid1(c->n), kBlock, 0, c->stream>>>(c->n, c->u.p, c->xv.p, split ? nullptr : c->st[c->cur].p,
                                                        split ? c->ur[c->cur].p : nullptr);
  return cudaGetLastError();
}

#define TRY_CUDA(expr)                 \
  do {                                 \
    const cudaError_t e_ = (expr);     \
    if (e_ != cudaSuccess) return e_;  \
  } while (0)

// The stream and events of the chunked force download (created on first use).
static cudaError_t ensure_copy_stream(pd_ctx* c) {
  if (c->copy_stream) return cudaSuccess;
  TRY_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  for (int k = 0; k <= kHostChunks; ++k) TRY_CUDA(cudaEventCreateWithFlags(&c->chunk_ev[k], cudaEventDisableTiming));
  return cudaSuccess;
}

// One model evaluation (damage -> dilatation -> force [-> Verlet epilogue]) on
// the gathered state of parity c->cur, with bond damage dmg updated in place.
// With sp.f_host set, the split sliced force pass also copies the force
// density to that host buffer, overlapped with its own later chunks, and sets
// *host_done; other paths leave the copy to the caller.
cudaError_t launch_eval(pd_ctx* c, const StepParams& sp, uint8_t* dmg, bool* host_done) {
  bool unused = false;
  if (!host_done) host_done = &unused;
  *host_done = false;
  if (c->n == 0) return cudaSuccess;
  const bool split = c->precision == PD_SPLIT_FP32;
  const int tpo = split ? c->tpo_split : c->tpo;
  const unsigned grid = grid_for(c->n, tpo), sgrid = grid_split(c->n, tpo);
  cudaEvent_t* ev = nullptr;
  if (c->ktime) {
    if (c->kev_used + 3 > c->kev.size()) {
      for (int k = 0; k < 3 * 256; ++k) {
        cudaEvent_t e;
        cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) return err;
        c->kev.push_back(e);
      }
    }
    ev = &c->kev[c->kev_used];
    c->kev_used += 3;
    cudaEventRecord(ev[0], c->stream);
  }
  EpiArgs E;
  E.dt = sp.dt;
  E.t0 = sp.t0;
  E.step = sp.step;
  E.mode = sp.mode;
  E.has_contact = sp.has_contact;
  E.has_bc = sp.has_bc;
  E.split = split;
  E.fc = c->fc.p;
  E.f_out = sp.f_out;
  E.u = c->u.p;
  E.v = c->v.p;
  E.a = c->a.p;
  E.bc_mask = c->bc_mask.p;
  E.bc_a = c->bc_a.p;
  E.bc_b = c->bc_b.p;
  E.st_next = split ? nullptr : c->st[c->cur ^ 1].p;
  E.ur_next = split ? c->ur[c->cur ^ 1].p : nullptr;
  E.status = c->status.p;
  // Split passes at 4 lanes per point read the sliced bond stream; its damage
  // mirror follows the CSR damage array this evaluation uses.
  const bool sell = split && c->sell && tpo == 4;
  if (sell && (c->sell_src != dmg || c->sell_gen != c->dmg_gen)) {
    k_sell_dmg<<<grid_for(c->n, 4), kBlock, 0, c->stream>>>(c->n, c->row.p, c->sell_off.p, dmg, c->sell_dmg.p);
    c->sell_src = dmg;
    c->sell_gen = c->dmg_gen;
  }
  const int32_t* scol = sell ? c->sell_col.p : c->col.p;
  uint8_t* sdmg = sell ? c->sell_dmg.p : dmg;
  const int64_t* soff = sell ? c->sell_off.p : nullptr;
  if (c->material_model == PD_MATERIAL_BOND_BASED) {  // one pass: damage + pair force + epilogue
    if (ev) cudaEventRecord(ev[1], c->stream);
    if (sell) {
      k_bb_split<4, true><<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, scol, sdmg, c->bx.p, c->ur[c->cur].p,
                                                          c->own.p, sp.damage_on, c->pt.p, c->node_damage.p, E, soff,
                                                          dmg);
    } else if (split) {
      PD_DISPATCH_TPO_CSR(tpo, k_bb_split, sgrid, kSplitBlock, c->n, c->row.p, c->col.p, dmg, c->bx.p, c->ur[c->cur].p, c->own.p,
                          sp.damage_on, c->pt.p, c->node_damage.p, E, nullptr, nullptr);
    } else {
      PD_DISPATCH_TPO(tpo, k_bb_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p, c->pt.p, c->sc.p,
                      c->hp.p, sp.damage_on, c->bb_plane, c->bb_height, c->node_damage.p, E);
    }
    if (ev) cudaEventRecord(ev[2], c->stream);
    return cudaGetLastError();
  }
  if (sell) {
    (c->material_model == PD_MATERIAL_LINEAR_LPS ? k_dilatation_split<4, true, true> : k_dilatation_split<4, true>)
        <<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, scol, sdmg, c->bx.p,
                                                                c->ur[c->cur].p, c->own.p, sp.damage_on, c->theta.p,
                                                                c->node_damage.p, soff, dmg);
  } else if (split) {
    PD_DISPATCH_TPO_CSR(tpo, k_dilatation_split, sgrid, kSplitBlock, c->n, c->row.p, c->col.p, dmg, c->bx.p, c->ur[c->cur].p,
                        c->own.p, sp.damage_on, c->theta.p, c->node_damage.p, nullptr, nullptr);
  } else if (c->material_model == PD_MATERIAL_LINEAR_LPS) {
    PD_DISPATCH_TPO(tpo, k_dilatation_lin_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p,
                    c->pt.p, c->sc.p, c->hp.p, c->influence, sp.damage_on, c->ab64.p, c->theta.p, c->node_damage.p);
  } else {
    PD_DISPATCH_TPO(tpo, k_dilatation_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p, c->pt.p,
                    c->sc.p, c->hp.p, c->influence, sp.damage_on, c->ab64.p, c->theta.p, c->node_damage.p);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (ev) cudaEventRecord(ev[1], c->stream);
  if (sell) {
    const bool lin = c->material_model == PD_MATERIAL_LINEAR_LPS;
    if (sp.f_host && sp.f_out) {
      auto* kf = lin ? k_force_split<4, true, true, true> : k_force_split<4, true, false, true>;
      // Force in chunks of points; each chunk's force density goes to the host
      // on the copy stream while the next chunk computes.
      TRY_CUDA(ensure_copy_stream(c));
      const int64_t n = c->n, per = ((n + kHostChunks - 1) / kHostChunks + 63) / 64 * 64;
      // (all chunks are launched before the first copy: a copy to pageable
      // memory holds the host until it is done)
      for (int64_t i0 = 0, k = 0; i0 < n; i0 += per, ++k) {
        const int64_t i1 = std::min(n, i0 + per);
        kf<<<grid_split(i1 - i0, 4), kSplitBlock, 0, c->stream>>>(i1, c->row.p, scol, sdmg, c->bx.p, c->ur[c->cur].p, c->pt.p,
                                                           E, soff, i0);
        TRY_CUDA(cudaEventRecord(c->chunk_ev[k], c->stream));
      }
      for (int64_t i0 = 0, k = 0; i0 < n; i0 += per, ++k) {
        const int64_t i1 = std::min(n, i0 + per);
        TRY_CUDA(cudaStreamWaitEvent(c->copy_stream, c->chunk_ev[k], 0));
        TRY_CUDA(cudaMemcpyAsync(sp.f_host + 3 * i0, sp.f_out + 3 * i0, 3 * (i1 - i0) * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->copy_stream));
      }
      TRY_CUDA(cudaEventRecord(c->chunk_ev[kHostChunks], c->copy_stream));
      TRY_CUDA(cudaStreamWaitEvent(c->stream, c->chunk_ev[kHostChunks], 0));
      *host_done = true;
    } else {
      auto* kf = lin ? k_force_split<4, true, true> : k_force_split<4, true>;
      kf<<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, scol, sdmg, c->bx.p, c->ur[c->cur].p, c->pt.p, E, soff, 0);
    }
  } else if (split) {
    PD_DISPATCH_TPO_CSR(tpo, k_force_split, sgrid, kSplitBlock, c->n, c->row.p, c->col.p, dmg, c->bx.p, c->ur[c->cur].p, c->pt.p, E,
                        nullptr);
  } else if (c->material_model == PD_MATERIAL_LINEAR_LPS) {
    PD_DISPATCH_TPO(tpo, k_force_lin_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p, c->ab64.p,
                    c->pt.p, c->hp.p, c->influence, E);
  } else {
    PD_DISPATCH_TPO(tpo, k_force_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p, c->ab64.p,
                    c->pt.p, c->hp.p, c->influence, E);
  }
  if (ev) cudaEventRecord(ev[2], c->stream);
  return cudaGetLastError();
}

// Folds the recorded bond-pass events into c->kms (synchronizes on the last one).
cudaError_t collect_kernel_times(pd_ctx* c) {
  if (c->kev_used == 0) return cudaSuccess;
  cudaError_t e = cudaEventSynchronize(c->kev[c->kev_used - 1]);
  if (e != cudaSuccess) return e;
  for (size_t k = 0; k + 3 <= c->kev_used; k += 3) {
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, c->kev[k], c->kev[k + 1]);
    cudaEventElapsedTime(&b, c->kev[k + 1], c->kev[k + 2]);
    c->kms[0] += a;
    c->kms[1] += b;
    c->klaunches += 1;
  }
  c->kev_used = 0;
  return cudaSuccess;
}

// FP64 model evaluation at caller coordinates y4 (x, y, z, -): dilatation
// pass into ab (theta, 3K/m - alpha/3, alpha) and force density into f_out.
// No damage update; the committed bond damage is used as is.
cudaError_t launch_fp64_eval_at(pd_ctx* c, const double4* y4, double4* ab, double* theta, double* nd,
                                double* f_out) {
  if (c->n == 0) return cudaSuccess;
  const unsigned grid = grid_for(c->n, c->tpo);
  PD_DISPATCH_TPO(c->tpo, k_dilatation_fp64, grid, c->n, c->row.p, c->col.p, c->dmg.p, c->xv.p, y4, c->pt.p,
                  c->sc.p, c->hp.p, c->influence, 0, ab, theta, nd);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  EpiArgs E{};
  E.mode = EVAL_ONLY;
  E.f_out = f_out;
  E.status = c->status.p;
  PD_DISPATCH_TPO(c->tpo, k_force_fp64, grid, c->n, c->row.p, c->col.p, c->dmg.p, c->xv.p, y4, ab, c->pt.p, c->hp.p,
                  c->influence, E);
  return cudaGetLastError();
}

cudaError_t launch_critical_dt(pd_ctx* c, double* dt_out_dev) {
  const unsigned grid = grid_for(c->n, c->tpo);
  if (c->scratch.count < (size_t)grid + 1) {
    cudaError_t e = c->scratch.alloc((size_t)grid + 1);
    if (e != cudaSuccess) return e;
  }
  PD_DISPATCH_TPO(c->tpo, k_critical_dt, grid, c->n, c->row.p, c->col.p, c->xv.p, c->pt.p, c->hp.p, c->scratch.p);
  k_min_reduce<<<1, kBlock, 0, c->stream>>>((int64_t)grid, c->scratch.p, dt_out_dev);
  return cudaGetLastError();
}

int64_t critical_dt_partials(const pd_ctx* c) { return (int64_t)grid_for(c->n, c->tpo); }

cudaError_t launch_critical_dt_into(pd_ctx* c, double* partial, double* dt_out_dev) {
  const unsigned grid = grid_for(c->n, c->tpo);
  PD_DISPATCH_TPO(c->tpo, k_critical_dt, grid, c->n, c->row.p, c->col.p, c->xv.p, c->pt.p, c->hp.p, partial);
  k_min_reduce<<<1, kBlock, 0, c->stream>>>((int64_t)grid, partial, dt_out_dev);
  return cudaGetLastError();
}

}  // namespace pdb

namespace pdb {

__global__ void k_u_from_record(int64_t n, const Rec8* __restrict__ ur, double* __restrict__ u) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Rec8 r = ur[i];
  for (int c = 0; c < 3; ++c) u[3 * i + c] = (double)r.v[c] + (double)r.v[c + 3];
}

// Displacement held by the split-path record of the given parity.
cudaError_t launch_u_from_record(pd_ctx* c, int parity, double* u_out) {
  if (c->n == 0) return cudaSuccess;
  k_u_from_record<<<grid1(c->n), kBlock, 0, c->stream>>>(c->n, c->ur[parity].p, u_out);
  return cudaGetLastError();
}

// out[6k..6k+5] = (u, y) of point idx[k]; y is the FP64 path's gathered
// coordinate record (x + u on the split path, which gathers u itself).
__global__ void k_pack_state(int64_t n, int64_t n_idx, const int32_t* __restrict__ idx, const double* __restrict__ u,
                             const double4* __restrict__ xv, const double4* __restrict__ st, double* __restrict__ out,
                             int* __restrict__ status) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_idx) return;
  const int64_t i = idx[k];
  if (i < 0 || i >= n) {  // index outside the context: reported, not accessed
    atomicOr(status, ST_BAD_INDEX);
    return;
  }
  const double u0 = u[3 * i], u1 = u[3 * i + 1], u2 = u[3 * i + 2];
  double4 y;
  if (st) {
    y = st[i];
  } else {
    const double4 x = xv[i];
    y = make_double4(x.x + u0, x.y + u1, x.z + u2, 0.0);
  }
  double* o = out + 6 * k;
  o[0] = u0, o[1] = u1, o[2] = u2, o[3] = y.x, o[4] = y.y, o[5] = y.z;
}

// The receiving side: u and the record the next evaluation gathers (hi/lo
// split of u on the split path, y on the FP64 path), both as the owner holds them.
__global__ void k_unpack_state(int64_t n, int64_t n_idx, const int32_t* __restrict__ idx,
                               const double* __restrict__ in, double* __restrict__ u, double4* __restrict__ st,
                               Rec8* __restrict__ ur, int* __restrict__ status) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_idx) return;
  const int64_t i = idx[k];
  if (i < 0 || i >= n) {
    atomicOr(status, ST_BAD_INDEX);
    return;
  }
  const double* v = in + 6 * k;
  for (int c = 0; c < 3; ++c) u[3 * i + c] = v[c];
  if (ur) {
    for (int c = 0; c < 3; ++c) split_hi_lo(v[c], &ur[i].v[c], &ur[i].v[c + 3]);
  } else {
    st[i] = make_double4(v[3], v[4], v[5], 0.0);
  }
}

cudaError_t launch_pack_state(pd_ctx* c, int64_t n_idx, const int32_t* idx, double* out) {
  if (n_idx == 0) return cudaSuccess;
  const bool split = c->precision == PD_SPLIT_FP32;
  k_pack_state<<<grid1(n_idx), kBlock, 0, c->stream>>>(c->n, n_idx, idx, c->u.p, c->xv.p,
                                                        split ? nullptr : c->st[c->cur].p, out, c->status.p);
  return cudaGetLastError();
}

cudaError_t launch_unpack_state(pd_ctx* c, int64_t n_idx, const int32_t* idx, const double* in) {
  if (n_idx == 0) return cudaSuccess;
  const bool split = c->precision == PD_SPLIT_FP32;
  k_unpack_state<<<grid1(n_idx), kBlock, 0, c->stream>>>(c->n, n_idx, idx, in, c->u.p,
                                                          split ? nullptr : c->st[c->cur].p,
                                                          split ? c->ur[c->cur].p : nullptr, c->status.p);
  return cudaGetLastError();
}

__global__ void k_count_nonzero(int64_t m, const uint8_t* __restrict__ d, unsigned long long* __restrict__ out) {
  unsigned long long cnt = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
    cnt += d[k] != 0;
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

int count_broken(pd_ctx* c, int64_t* out) {
  *out = 0;
  if (c->nb == 0) return PD_OK;
  if (c->scratch.count < 1) PD_CUDA_TRY(c, c->scratch.alloc(1));
  unsigned long long* dcount = reinterpret_cast<unsigned long long*>(c->scratch.p);
  PD_CUDA_TRY(c, cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), c->stream));
  k_count_nonzero<<<4 * 148, kBlock, 0, c->stream>>>(c->nb, c->dmg.p, dcount);
  PD_CUDA_TRY(c, cudaGetLastError());
  unsigned long long h = 0;
  PD_CUDA_TRY(c, d2h(c, &h, dcount, sizeof(h)));
  *out = (int64_t)h;
  return PD_OK;
}

}  // namespace pdb
