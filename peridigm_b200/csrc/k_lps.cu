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
//   bx3 = X per bond, streamed (12 B): X = fp32(x_j - x_i) formed in FP64,
//         rounded once; 32-slot groups of three planes (x[32], y[32], z[32])
//         so that one warp load of a component is 128 consecutive bytes
//   ur[j] = (u_hi[3], lo_xy, lo_z|q, V, A, B) per point, one 256-bit gather
//         per bond: u_hi = fp32(u); the residual u - u_hi of each component as
//         a 16-bit multiple of a power of two q shared by the three (q in the
//         top half of slot 4, 2^-14 of the largest component's FP32 ulp, so
//         u_hi + lo carries u to ~2^-39 of |u|); V = the point's volume
// du = (u_hi_j - u_hi_i) + (lo_j - lo_i) is the displacement difference to
// within one FP32 ulp plus 2^-38 |u|, with no FP64 instruction in the bond
// loop. The influence weight omega(|X|) is evaluated in the loop (1 for the
// "One" function). The FP64 displacement u[3n] stays the integration state.
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

// ---------------------------------------------------------------------------
// Split-path displacement record (slots 0-4 of Rec8). The residual of each
// component, u_c - fp32(u_c), is stored as k_c * q with k_c a 16-bit integer
// (biased by 2^15) and q = 2^(eb - 165), eb the largest biased FP32 exponent
// of the three u_hi: |u_c - u_hi_c| <= ulp(u_hi_c)/2 <= 2^14 q, so k_c fits,
// and the rounding of k_c leaves an error of at most q/2 ~ 2^-39 |u|.
// ---------------------------------------------------------------------------
constexpr uint32_t kQShift = 38;  // q = 2^-14 * 2^-24 of the largest component's binade

// The record's 16-bit residual k (biased) as a float: 2^23 + k exactly.
__device__ __forceinline__ float lo_magic(uint32_t k16) { return __uint_as_float(0x4B000000u | k16); }

struct ULo {
  float x, y, z;
};
// Residuals of a record: (2^23 + k) q - (2^23 + 2^15) q = (k - 2^15) q, exact.
__device__ __forceinline__ ULo decode_lo(const Rec8& r) {
  const uint32_t w3 = __float_as_uint(r.v[3]), w4 = __float_as_uint(r.v[4]);
  const float q = __uint_as_float(w4 & 0xffff0000u);
  const float c = -8421376.0f * q;  // -(2^23 + 2^15) q
  ULo l;
  l.x = fmaf(lo_magic(w3 & 0xffffu), q, c);
  l.y = fmaf(__uint_as_float(__byte_perm(w3, 0x4B00u, 0x5432u)), q, c);  // high half of w3 under 0x4B00
  l.z = fmaf(lo_magic(w4 & 0xffffu), q, c);
  return l;
}

// 16-bit residual (biased) of component value uc with FP32 part h, quantum
// 2^(eb - 165); 0x8000 (zero residual) when the point's displacement is below
// 2^-88 and q would not be a normal float.
__device__ __forceinline__ uint32_t lo_code(double uc, float h, uint32_t eb) {
  if (eb <= kQShift) return 0x8000u;
  const double inv = __longlong_as_double((long long)(1023 + 127 + kQShift - eb) << 52);  // 1/q, exact
  int k = __double2int_rn((uc - (double)h) * inv);  // uc - h is exact in FP64
  k = min(max(k, -32768), 32767);
  return (uint32_t)(k + 32768);
}
__device__ __forceinline__ uint32_t q_bits(uint32_t eb) { return eb > kQShift ? (eb - kQShift) << 23 : 0u; }
__device__ __forceinline__ uint32_t f32_exp(float h) { return (__float_as_uint(h) >> 23) & 0xffu; }

// Record slots 0-4 from one thread's FP64 displacement (slots 5-7 untouched).
__device__ __forceinline__ void store_u_record(Rec8* rec, double u0, double u1, double u2) {
  const float h0 = __double2float_rn(u0), h1 = __double2float_rn(u1), h2 = __double2float_rn(u2);
  const uint32_t eb = max(f32_exp(h0), max(f32_exp(h1), f32_exp(h2)));
  const uint32_t k0 = lo_code(u0, h0, eb), k1 = lo_code(u1, h1, eb), k2 = lo_code(u2, h2, eb);
  *reinterpret_cast<float4*>(rec->v) = make_float4(h0, h1, h2, __uint_as_float(k0 | (k1 << 16)));
  rec->v[4] = __uint_as_float(k2 | q_bits(eb));
}

template <int TPO>
__device__ __forceinline__ uint32_t group_max_u32(uint32_t v) {
#pragma unroll
  for (int o = TPO / 2; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// The same from a lane group: lane c < 3 holds component c (other lanes pass
// 0). Every lane of the warp calls it; only groups with `store` write.
template <int TPO>
__device__ __forceinline__ void store_u_record_group(Rec8* rec, int lane, double uc, bool store) {
  const float h = __double2float_rn(uc);
  const uint32_t eb = group_max_u32<TPO>(lane < 3 ? f32_exp(h) : 0u);
  const uint32_t k = lo_code(uc, h, eb);
  const float h1 = __shfl_down_sync(0xffffffffu, h, 1, TPO);
  const float h2 = __shfl_down_sync(0xffffffffu, h, 2, TPO);
  const uint32_t k1 = __shfl_down_sync(0xffffffffu, k, 1, TPO);  // lane 0: k_y; lane 1: k_z
  if (store && lane == 0) *reinterpret_cast<float4*>(rec->v) = make_float4(h, h1, h2, __uint_as_float(k | (k1 << 16)));
  if (store && lane == 1) rec->v[4] = __uint_as_float(k1 | q_bits(eb));
}

// FP64 displacement held by a record.
__device__ __forceinline__ void load_u_record(const Rec8& r, double* u) {
  const ULo l = decode_lo(r);
  u[0] = (double)r.v[0] + (double)l.x;
  u[1] = (double)r.v[1] + (double)l.y;
  u[2] = (double)r.v[2] + (double)l.z;
}

// Influence function in FP32 for the split passes (same branches as omega_d).
__device__ __forceinline__ float omega_f(int kind, float zeta, float h) {
  if (kind == PD_INFLUENCE_ONE) return 1.0f;
  if (kind == PD_INFLUENCE_PARABOLIC_DECAY) {
    if (zeta > h) return 0.0f;
    const float s = zeta / h;
    return s < 0.5f ? 1.0f : fmaf(-4.0f * s, s, 4.0f * s);
  }
  return expf(-(zeta * zeta) / (h * h * 0.16f));
}

// The owner's own displacement (hi and decoded residual) and its volume-free
// record terms, read once per row.
struct OwnU {
  float hx, hy, hz, lx, ly, lz;
};
__device__ __forceinline__ OwnU own_u(const Rec8& r) {
  const ULo l = decode_lo(r);
  OwnU o;
  o.hx = r.v[0], o.hy = r.v[1], o.hz = r.v[2];
  o.lx = l.x, o.ly = l.y, o.lz = l.z;
  return o;
}

// Bond geometry of the split path from the bond's stored X (FP32) and the two
// endpoints' displacements. Identical operations in both passes; with both
// endpoints swapped X, du and Y are exactly negated (X_ji = -X_ij is rounded
// from an exactly negated FP64 difference), so e and |X| are identical and
// bond damage stays symmetric.
struct SplitBond {
  float Yx, Yy, Yz, zeta, ry, e, xu, xx;  // xu = X.du, xx = |X|^2 (the linear LPS terms)
};
// |Y|^2 = |X|^2 + (2X.du + du.du) and e = (2X.du + du.du)/(|Y| + |X|); Y = X +
// du and 1/|Y| only with Y (the dilatation pass needs neither).
template <bool Y = true>
__device__ __forceinline__ SplitBond split_bond(float X0, float X1, float X2, const OwnU& ui, const Rec8& uj) {
  SplitBond s;
  const ULo lj = decode_lo(uj);
  const float Ux = (uj.v[0] - ui.hx) + (lj.x - ui.lx);
  const float Uy = (uj.v[1] - ui.hy) + (lj.y - ui.ly);
  const float Uz = (uj.v[2] - ui.hz) + (lj.z - ui.lz);
  const float xx = fmaf(X2, X2, fmaf(X1, X1, X0 * X0));
  const float xu = fmaf(X2, Uz, fmaf(X1, Uy, X0 * Ux));
  const float uu = fmaf(Uz, Uz, fmaf(Uy, Uy, Ux * Ux));
  const float num = fmaf(2.0f, xu, uu);
  const float yy = xx + num;
  const float ry = rsqrtf(yy);
  s.zeta = xx * rsqrtf(xx);
  s.e = __fdividef(num, yy * ry + s.zeta);  // |Y| - |X| without cancellation
  s.xu = xu;
  s.xx = xx;
  if (Y) {
    s.ry = ry;
    s.Yx = X0 + Ux;
    s.Yy = X1 + Uy;
    s.Yz = X2 + Uz;
  }
  return s;
}

// Position of the X of stream slot k in bx3 (component c at +32c).
__device__ __forceinline__ int64_t xs_index(int64_t k) { return 96 * (k >> 5) + (k & 31); }

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
// Resident blocks of 128 threads per SM (the launch bound): 7 (72 registers,
// 28 warps) against 8 (64 registers, 32 warps, where the half-bond
// dilatation spills): dilatation 14.94 -> 13.84 ms and force 16.25 -> 15.46 ms
// at the 32,000,000-point heterogeneous plate, 0.1173 -> 0.1162 ms and
// 0.1196 -> 0.1090 ms at the notched plate; 6 blocks (80 registers) were
// slower than 8 on both.
#ifndef PD_BOND_MINB
#define PD_BOND_MINB 7
#endif
constexpr int kUnroll = PD_BOND_UNROLL;
// Threads per block of the split bond passes: 128-thread blocks keep the last
// partial wave of a ~5000-block grid at half the cost of 256-thread blocks.
constexpr int kSplitBlock = 128;

// Bond damage byte of bond (i, j) in row i: bit 0 = d_ij, the damage of the
// row's own half (the reference's bondDamage of i's family), bit 1 = d_ji,
// the partner half's (j's family), kept in step by evaluating j's own
// critical-stretch test in i's row as well: the stretch of a bond is computed
// identically in both rows, so the two bytes stay mirrored without a reverse
// index. With one critical stretch on both sides of every bond the two bits
// are equal. kDummyBond marks padding slots and masked lanes (neither half
// present). The force gathers t_ij with (1 - d_ij) and t_ji with (1 - d_ji),
// as the reference's scatter does from the two families
// (elastic.cxx:119-130).
constexpr int kDummyBond = 4;

// Bond-stream cursor of a lane in CSR order: the owner's row, the lane's
// bonds TPO apart.
template <int TPO>
__device__ __forceinline__ void csr_cursor(int lane, int64_t b0, int64_t b1, int64_t* base, int* left) {
  const int rem = (int)(b1 - b0) - lane;
  *base = b0 + lane;
  *left = rem > 0 ? (rem + TPO - 1) / TPO : 0;
}

// ---------------------------------------------------------------------------
// Sliced (SELL) bond stream of the 4-lanes-per-point passes. Slice s = the 8
// owners of a warp; lane l32 = 4*o + (r mod 4) of the warp takes owner o's
// bonds r = l32 mod 4, +4, +8, ...; each row is padded with dummy bonds
// (damage byte 2) to the slice's longest, G = soff[s+1] - soff[s] groups of
// 32 slots (one bond per lane) from slot 32*soff[s].
// Blocked layout: the slice's first 4*floor(G/4) groups form blocks of 4
// groups (128 slots) in which a lane's 4 bonds are adjacent (slot 4*l32 + k,
// k = group mod 4), so that a lane reads a block's 4 ids as one int4, its 4
// damage bytes as one word and each X component of its 4 bonds as one
// float4, and a warp load is 512 consecutive bytes. The tail (< 4 groups)
// keeps one slot per lane per group (slot l32 of the group). X sits in units
// of 3 planes: a block's X at 3*(its first slot), planes 128 floats apart; a
// tail group's at 3*(its first slot), planes 32 floats apart.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t sell_index(const int64_t* __restrict__ soff, int64_t i, int64_t r) {
  const int64_t s = i >> 3, so = soff[s], full = (soff[s + 1] - so) & ~int64_t(3), g = r >> 2;
  const int l32 = (int)((i & 7) * 4 + (r & 3));
  return g < full ? 32 * (so + (g & ~int64_t(3))) + 4 * l32 + (g & 3) : 32 * (so + g) + l32;
}
// Index of plane 0 of the X of that slot in bx3, and the plane stride.
__device__ __forceinline__ int64_t sell_x_index(const int64_t* __restrict__ soff, int64_t i, int64_t r, int* stride) {
  const int64_t s = i >> 3, so = soff[s], full = (soff[s + 1] - so) & ~int64_t(3), g = r >> 2;
  const int l32 = (int)((i & 7) * 4 + (r & 3));
  if (g < full) {
    *stride = 128;
    return 96 * (so + (g & ~int64_t(3))) + 4 * l32 + (g & 3);
  }
  *stride = 32;
  return 96 * (so + g) + l32;
}

// Slots 0-5 of a record (displacement and volume: what the dilatation pass
// reads of a neighbor), coherent; slots 6-7 are left 0.
__device__ __forceinline__ Rec8 ld_rec_u(const Rec8* p) {
  Rec8 r;
  asm("ld.global.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3]) : "l"(p));
  asm("ld.global.v2.f32 {%0,%1}, [%2];" : "=f"(r.v[4]), "=f"(r.v[5]) : "l"(p->v + 4));
  r.v[6] = r.v[7] = 0.0f;
  return r;
}
// Neighbor record loads of the walks: NC (0) coherent 256-bit load, (1) the
// read-only path (no record written by the kernel), (2) slots 0-5 only.
template <int NC>
__device__ __forceinline__ Rec8 ld_rec_t(const Rec8* p) {
  return NC == 2 ? ld_rec_u(p) : (NC == 1 ? ld_rec_nc(p) : ld_rec(p));
}

// Walks lane `lane` of owner i through its bonds of the sliced stream: the
// full blocks with one int4 of ids (loaded one block ahead), one damage word
// and three float4 of X per block, then the tail groups. For each bond, in
// the lane's row order, body(X0, X1, X2, damage byte, neighbor record,
// neighbor id, the bond's damage byte in the stream, row offset r - lane).
// NC: how neighbor records are loaded (ld_rec_t).
template <int NC, typename Body>
__device__ __forceinline__ void sell_walk(int64_t i, int lane, const int64_t* __restrict__ soff,
                                          const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
                                          const float* __restrict__ bx3, const Rec8* __restrict__ ur, Body&& body) {
  const int64_t s = i >> 3, so = soff[s];
  const int G = (int)(soff[s + 1] - so), F = G >> 2;
  const int l32 = (int)(i & 7) * 4 + lane;
  const int4* pc = reinterpret_cast<const int4*>(col + 32 * so + 4 * l32);
  uint32_t* pd = reinterpret_cast<uint32_t*>(dmg + 32 * so + 4 * l32);
  const float4* px = reinterpret_cast<const float4*>(bx3 + 96 * so + 4 * l32);
  int4 jn = F > 0 ? __ldcs(pc) : make_int4(0, 0, 0, 0);
#pragma unroll 1
  for (int b = 0; b < F; ++b, pc += 32, pd += 32, px += 96) {
    const int4 jj = jn;
    if (b + 1 < F) jn = __ldcs(pc + 32);
    const uint32_t dw = __ldcs(pd);
    const float4 xa = __ldcs(px), xb = __ldcs(px + 32), xc = __ldcs(px + 64);
    const Rec8 u0 = ld_rec_t<NC>(ur + jj.x), u1 = ld_rec_t<NC>(ur + jj.y), u2 = ld_rec_t<NC>(ur + jj.z),
               u3 = ld_rec_t<NC>(ur + jj.w);
    uint8_t* pb = reinterpret_cast<uint8_t*>(pd);
    const int r0 = 16 * b;
    body(xa.x, xb.x, xc.x, (int)(dw & 0xffu), u0, jj.x, pb, r0);
    body(xa.y, xb.y, xc.y, (int)((dw >> 8) & 0xffu), u1, jj.y, pb + 1, r0 + 4);
    body(xa.z, xb.z, xc.z, (int)((dw >> 16) & 0xffu), u2, jj.z, pb + 2, r0 + 8);
    body(xa.w, xb.w, xc.w, (int)(dw >> 24), u3, jj.w, pb + 3, r0 + 12);
  }
  const int T = G - 4 * F;
  if (T > 0) {  // tail groups: masked, one slot per lane per group
    const int64_t t0 = 32 * (so + 4 * F) + l32;
    const float* pt = bx3 + 96 * (so + 4 * F) + l32;
    int32_t jj[3];
    int dd[3];
    float X0[3], X1[3], X2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const bool in = k < T;
      jj[k] = in ? __ldcs(col + t0 + 32 * k) : (int32_t)i;
      dd[k] = in ? (int)dmg[t0 + 32 * k] : kDummyBond;
      X0[k] = in ? __ldcs(pt + 96 * k) : 1.0f;
      X1[k] = in ? __ldcs(pt + 96 * k + 32) : 0.0f;
      X2[k] = in ? __ldcs(pt + 96 * k + 64) : 0.0f;
    }
    Rec8 uu[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) uu[k] = ld_rec_t<NC>(ur + jj[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) body(X0[k], X1[k], X2[k], dd[k], uu[k], jj[k], dmg + t0 + 32 * k, 16 * F + 4 * k);
  }
}

// The same walk over a CSR row (TPO lanes per point, the lane's bonds TPO
// apart), kUnroll bonds per batch with the next batch's ids loaded ahead.
template <int TPO, int NC, typename Body>
__device__ __forceinline__ void csr_walk(int64_t i, int lane, int64_t b0, int64_t b1, const int32_t* __restrict__ col,
                                         uint8_t* __restrict__ dmg, const float* __restrict__ bx3,
                                         const Rec8* __restrict__ ur, Body&& body) {
  int64_t slot;
  int left;
  csr_cursor<TPO>(lane, b0, b1, &slot, &left);
  int32_t jn[kUnroll];
#pragma unroll
  for (int k = 0; k < kUnroll; ++k) jn[k] = k < left ? __ldcs(col + slot + TPO * k) : (int32_t)i;
#pragma unroll 1
  for (; left > 0; left -= kUnroll, slot += kUnroll * TPO) {
    int dd[kUnroll];
    float X0[kUnroll], X1[kUnroll], X2[kUnroll];
    int32_t jj[kUnroll];
    Rec8 uu[kUnroll];
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      jj[k] = jn[k];
      jn[k] = k + kUnroll < left ? __ldcs(col + slot + TPO * (k + kUnroll)) : (int32_t)i;
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) {
      const bool in = k < left;
      const float* p = bx3 + xs_index(slot + TPO * k);
      dd[k] = in ? (int)dmg[slot + TPO * k] : kDummyBond;  // past the row end
      X0[k] = in ? __ldcs(p) : 1.0f;
      X1[k] = in ? __ldcs(p + 32) : 0.0f;
      X2[k] = in ? __ldcs(p + 64) : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < kUnroll; ++k) uu[k] = ld_rec_t<NC>(ur + jj[k]);
#pragma unroll
    for (int k = 0; k < kUnroll; ++k)
      body(X0[k], X1[k], X2[k], dd[k], uu[k], jj[k], dmg + slot + TPO * k, (int)(slot + TPO * k - b0 - lane));
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
                                                            double4* __restrict__ pt,
                                                            const uint8_t* __restrict__ phantom) {
  // phantom: the damage bytes when the device rows hold phantom halves (not
  // in the point's own family), else null
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  double acc = 0.0;
  if (valid) {
    const double4 xi = xv[i];
    const double h = hp[i];
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += TPO) {
      if (phantom && (phantom[b] & kPhantomOwn)) continue;
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
  // a point with no bonds (m = 0) keeps theta = 0 and no force terms, as the
  // reference's loops over its empty family leave them
  const double im = p.x > 0.0 ? 1.0 / p.x : 0.0;
  own[i] = make_float4((float)(3.0 * im), (float)((3.0 * p.y - 5.0 * p.z) * im), (float)(15.0 * p.z * im),
                       (float)sc[i]);
}

// Split-path bond stream bx3: X = x_j - x_i in FP64, rounded once to FP32, at
// the slot's position in the grouped planes (xs_index). In CSR order (SELL
// false), or in the sliced order of bond_cursor (SELL true, with the neighbor
// ids and damage bytes copied alongside).
__device__ __forceinline__ void put_x(float* __restrict__ p, int stride, float X0, float X1, float X2) {
  p[0] = X0;
  p[stride] = X1;
  p[2 * stride] = X2;
}

template <int TPO, bool SELL>
__global__ void __launch_bounds__(kBlock) k_pack_bonds(int64_t n, const int64_t* __restrict__ row,
                                                       const int32_t* __restrict__ col,
                                                       const double4* __restrict__ xv, float* __restrict__ bx3,
                                                       const int64_t* __restrict__ soff,
                                                       const uint8_t* __restrict__ dmg, int32_t* __restrict__ scol,
                                                       uint8_t* __restrict__ sdmg) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  if (i >= n) return;
  const double4 xi = xv[i];
  const int64_t b0 = row[i];
  for (int64_t b = b0 + lane; b < row[i + 1]; b += TPO) {
    const int32_t j = col[b];
    const double4 xj = xv[j];
    const float X0 = (float)__dsub_rn(xj.x, xi.x), X1 = (float)__dsub_rn(xj.y, xi.y),
                X2 = (float)__dsub_rn(xj.z, xi.z);
    if (SELL) {
      const int64_t k = sell_index(soff, i, b - b0);
      int stride;
      if (bx3) put_x(bx3 + sell_x_index(soff, i, b - b0, &stride), stride, X0, X1, X2);
      scol[k] = j;
      sdmg[k] = dmg[b];
    } else {
      put_x(bx3 + xs_index(b), 32, X0, X1, X2);
    }
  }
  if (SELL) {  // padding to the slice's longest row: dummy bonds (kDummyBond)
    const int64_t len = row[i + 1] - b0, ms = soff[(i >> 3) + 1] - soff[i >> 3];
    for (int64_t r = len + lane; r < 4 * ms; r += TPO) {
      const int64_t k = sell_index(soff, i, r);
      int stride;
      if (bx3) put_x(bx3 + sell_x_index(soff, i, r, &stride), stride, 1.f, 0.f, 0.f);
      scol[k] = (int32_t)i;
      sdmg[k] = kDummyBond;
    }
  }
}

// Split-path point volumes in record slot 5 of both state buffers (the state
// writers touch slots 0-4, the dilatation pass slots 6-7).
__global__ void k_pack_volume(int64_t n, const double4* __restrict__ xv, Rec8* __restrict__ ur0,
                              Rec8* __restrict__ ur1) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float V = (float)xv[i].w;
  ur0[i].v[5] = V;
  ur1[i].v[5] = V;
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
// WEIGHT: an influence function other than "One", omega(|X|, h_i) evaluated per bond.
// (the weighted variants get 96 registers: the omega evaluation would spill at 64)
// PAIR: the two halves of a bond can differ (critical stretch varying along
// bonds, or half-broken bonds set by the caller): the partner's test runs
// with its own s_c,j, read only for bonds stretched past s_min, the smallest
// critical stretch of the body (no bond below it can break on either side).
#ifndef PD_DIL_MINB
#define PD_DIL_MINB 7
#endif
template <int TPO, bool SELL, bool LIN = false, bool WEIGHT = false, bool PAIR = false>
__global__ void __launch_bounds__(kSplitBlock, WEIGHT ? 5 : PD_DIL_MINB) k_dilatation_split(
    int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
    const float* __restrict__ bx3, Rec8* __restrict__ ur, const float4* __restrict__ own, int damage_on,
    double* __restrict__ theta_out, double* __restrict__ node_damage, const int64_t* __restrict__ soff,
    uint8_t* __restrict__ dmg_csr, const double* __restrict__ hp, int influence, const float* __restrict__ scf,
    float s_min, int64_t i0 = 0) {
  // owners i0 .. n-1 (a chunk starts at a multiple of 64 owners)
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = i0 + g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  float th = 0.0f;
  int broken = 0;
  int len = 0;
  if (valid) {
    const int64_t b0 = row[i];
    len = (int)(row[i + 1] - b0);
    const OwnU ui = own_u(ld_rec(ur + i));
    const float s_c = damage_on ? own[i].w : -1.0f;
    const float hi = WEIGHT ? (float)hp[i] : 1.0f;
    uint8_t* cdm = SELL ? dmg_csr + b0 + lane : nullptr;  // the lane's bonds in the canonical CSR damage
    // Branch-free masking (selects) of dummy and broken bonds.
    auto body = [&](float X0, float X1, float X2, int d, const Rec8& uj, int32_t, uint8_t* pdm, int r) {
      const SplitBond sb = split_bond<false>(X0, X1, X2, ui, uj);
      const bool own_ok = (d & 5) == 0;  // own half intact (and a real bond)
      // the partner's half: its own test, or the same test on both halves
      bool brk, brkp;
      if (PAIR) {
        // Every critical stretch of the body is at least s_min (products
        // round monotonically): a bond not past s_min breaks on neither side,
        // so both tests run only past it (rare).
        brk = brkp = false;
        if (damage_on && sb.e > s_min * sb.zeta) {
          brk = own_ok && s_c >= 0.0f && sb.e > s_c * sb.zeta;
          if ((d & 6) == 0) {
            // the neighbor id again from the bond's stream slot (keeping the
            // batch's ids live for this branch would cost registers)
            const float scj = __ldg(scf + __ldg(col + (pdm - dmg)));
            brkp = scj >= 0.0f && sb.e > scj * sb.zeta;
          }
        }
      } else {
        brk = brkp = own_ok && s_c >= 0.0f && sb.e > s_c * sb.zeta;
      }
      if (brk || brkp) {
        const uint8_t nd = (uint8_t)(d | (brk ? 1 : 0) | (brkp ? 2 : 0));
        *pdm = nd;
        if (SELL) cdm[r] = nd;  // the CSR copy stays canonical
      }
      broken += ((d & 1) || brk) ? 1 : 0;
      float wv = uj.v[5];  // V_j
      if constexpr (WEIGHT) wv *= omega_f(influence, sb.zeta, hi);
      // LPS: omega V_j |X| e; linear LPS: omega V_j X.du
      th = fmaf((own_ok && !brk) ? (LIN ? wv : wv * sb.zeta) : 0.0f, LIN ? sb.xu : sb.e, th);
    };
    // neighbor records: the whole record in one 256-bit load although the
    // pass reads slots 0-5 only (displacement, volume): two loads (16 + 8
    // bytes) double the L1 lookups, and at 7 blocks per SM the registers for
    // slots 6-7 are there (full-bond dilatation 0.1162 -> 0.1130 ms at the
    // notched plate, 15.09 -> 14.68 ms at the 32,000,000-point plate with one
    // material)
    constexpr int kRec = 0;
    if constexpr (SELL)
      sell_walk<kRec>(i, lane, soff, col, dmg, bx3, ur, body);
    else
      csr_walk<TPO, kRec>(i, lane, b0, b0 + len, col, dmg, bx3, ur, body);
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
    double4* __restrict__ ab64, double* __restrict__ theta_out, double* __restrict__ node_damage, int pair) {
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
      const int d = dmg[b];  // bit 0: this half broken, bit 1: the partner's half
      if ((d & 3) == 3) {
        broken++;
        continue;
      }
      const int32_t j = col[b];
      const double4 xj = xv[j];
      const double4 yj = st[j];
      const double zeta = __dsqrt_rn(sq3_rn(__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z)));
      const double dY = __dsqrt_rn(sq3_rn(__dsub_rn(yj.x, yi.x), __dsub_rn(yj.y, yi.y), __dsub_rn(yj.z, yi.z)));
      // this half's test with s_c,i; the partner's with s_c,j (the same test
      // on both halves when the critical stretch is one along every bond)
      const double scj = pair && damage_on ? sc[j] : s_c;
      bool brk = false, brkp = false;
      if ((s_c >= 0.0 && !(d & 1)) || (scj >= 0.0 && !(d & 2))) {
        const double rel = __ddiv_rn(__dsub_rn(dY, zeta), zeta);
        brk = !(d & 1) && s_c >= 0.0 && rel > s_c;
        brkp = !(d & 2) && scj >= 0.0 && rel > scj;
      }
      if (brk || brkp) dmg[b] = (uint8_t)(d | (brk ? 1 : 0) | (brkp ? 2 : 0));
      if ((d & 1) || brk) {
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
  const double2* bc_cp;  // (u(t_c), u(t_p)) of function dofs (mask bit 3 + c), or null
  double4* st_next;  // FP64 path: next coordinates
  Rec8* ur_next;     // split path: next displacement record
  int* status;
};

__device__ __forceinline__ double comp3(const double4& q, int c) { return c == 0 ? q.x : (c == 1 ? q.y : q.z); }
__device__ __forceinline__ double* comp_ptr(double4* q, int c) {
  return c == 0 ? &q->x : (c == 1 ? &q->y : &q->z);
}

// Returns the new displacement component (the FP64 u written back); the split
// passes pack it into the next record afterwards (store_u_record_group, which
// needs the group's three components at once).
__device__ __forceinline__ double verlet_epilogue(const EpiArgs& E, int64_t i, int c, double f, double xc,
                                                  double rho) {
  const int64_t k = 3 * i + c;
  double ftot = f;
  if (E.has_contact) ftot = __dadd_rn(ftot, E.fc[k]);
  if (!isfinite(ftot)) atomicOr(E.status, ST_NONFINITE_FORCE);
  if (E.f_out) E.f_out[k] = ftot;
  if (E.mode == EVAL_ONLY) return 0.0;
  const double dt = E.dt, dt2 = E.dt / 2.0;
  const double acc = __ddiv_rn(__dadd_rn(ftot, 0.0), rho);
  double v = E.v[k];
  if (E.step > 0) v = __dadd_rn(v, __dmul_rn(dt2, acc));  // end of step (none after the initial evaluation)
  if (E.mode == EVAL_LAST) {
    E.v[k] = v;
    E.a[k] = acc;
    return 0.0;
  }
  // first half of step s+1
  double vh = __dadd_rn(v, __dmul_rn(dt2, acc));
  if (E.has_bc && ((E.bc_mask[i] >> c) & 1)) {
    const double tc = __dadd_rn(E.t0, __dmul_rn((double)(E.step + 1), dt));
    const double tp = E.step == 0 ? E.t0 : __dadd_rn(E.t0, __dmul_rn((double)E.step, dt));
    if (tc != tp) {
      double cur, prev;
      if (E.bc_cp && ((E.bc_mask[i] >> (c + 3)) & 1)) {
        const double2 q = E.bc_cp[k];
        cur = q.x, prev = q.y;
      } else {
        cur = __dadd_rn(__dmul_rn(E.bc_a[k], tc), E.bc_b[k]);
        prev = __dadd_rn(__dmul_rn(E.bc_a[k], tp), E.bc_b[k]);
      }
      // a zero increment takes the previous value from the displacement
      // field (Peridigm_BoundaryCondition.cpp:137-142)
      double d = __dsub_rn(cur, prev);
      if (d == 0.0) d = __dsub_rn(cur, E.u[k]);
      vh = __dadd_rn(__dmul_rn(0.0, d), __dmul_rn(__dmul_rn(1.0, d), __ddiv_rn(1.0, __dsub_rn(tc, tp))));
      if (!isfinite(vh)) atomicOr(E.status, ST_NONFINITE_BC);
    }
  }
  E.v[k] = vh;
  E.a[k] = acc;
  const double step_dx = __dmul_rn(dt, vh);
  const double u = E.u[k];
  const double un = __dadd_rn(u, step_dx);  // u += dt*v
  E.u[k] = un;
  if (!E.split) *comp_ptr(&E.st_next[i], c) = __dadd_rn(__dadd_rn(xc, u), step_dx);  // y = x+u+dt*v
  return un;
}

// Split passes: the group's epilogue (lanes 0-2, one component each) and the
// next displacement record. Every lane of the warp calls it.
template <int TPO>
__device__ __forceinline__ void split_epilogue(const EpiArgs& E, int64_t i, int lane, bool valid, float fx, float fy,
                                               float fz, const double4* __restrict__ pt) {
  double un = 0.0;
  if (valid && lane < 3) {
    const double f = lane == 0 ? (double)fx : (lane == 1 ? (double)fy : (double)fz);
    un = verlet_epilogue(E, i, lane, f, 0.0, pt[i].w);
  }
  if (E.mode == EVAL_ADVANCE) store_u_record_group<TPO>(E.ur_next + i, lane, un, valid);
}

// ---------------------------------------------------------------------------
// K3: force gather, split-FP32:
//   t_ij + t_ji = omega*(|X|*(A_i + A_j) + e*(B_i + B_j))   (bond intact)
//   f_i += (t_ij + t_ji) * V_j * Y/|Y|
// Broken bonds carry t = 0 (elastic.cxx:120 with d = 1) and are skipped.
// ---------------------------------------------------------------------------
#ifndef PD_FORCE_NC
#define PD_FORCE_NC 1
#endif
template <int TPO, bool SELL, bool LIN = false, bool CHUNK = false, bool WEIGHT = false, bool PAIR = false>
__global__ void __launch_bounds__(kSplitBlock, WEIGHT ? 5 : PD_BOND_MINB) k_force_split(int64_t n, const int64_t* __restrict__ row,
                                                                      const int32_t* __restrict__ col,
                                                                      const uint8_t* __restrict__ dmg,
                                                                      const float* __restrict__ bx3,
                                                                      const Rec8* __restrict__ ur,
                                                                      const double4* __restrict__ pt, EpiArgs E,
                                                                      const int64_t* __restrict__ soff,
                                                                      const double* __restrict__ hp, int influence,
                                                                      int64_t i0 = 0) {
  // CHUNK: owners i0 .. n-1 (a chunk of the points starts at a multiple of 64
  // owners); otherwise i0 is not used and the pass covers 0 .. n-1
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = (CHUNK ? i0 : 0) + g / TPO;
  const int lane = threadIdx.x & (TPO - 1);
  const bool valid = i < n;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (valid) {
    const Rec8 ri = ld_rec_t<PD_FORCE_NC>(ur + i);
    const OwnU ui = own_u(ri);
    const float Ai = ri.v[6], Bi = ri.v[7];
    const float hi = WEIGHT ? (float)hp[i] : 1.0f;
    auto body = [&](float X0, float X1, float X2, int d, const Rec8& uj, int32_t, uint8_t*, int) {
      const SplitBond sb = split_bond<true>(X0, X1, X2, ui, uj);
      float wv = uj.v[5];  // V_j
      if constexpr (WEIGHT) wv *= omega_f(influence, sb.zeta, hi);
      // owner terms of the intact halves: t_ij with (1 - d_ij), t_ji with (1 - d_ji)
      float a, b;
      if constexpr (PAIR) {
        a = Ai + uj.v[6];
        b = Bi + uj.v[7];
        if (d != 0) {  // a broken half or a padding slot (both intact is the common case)
          const bool own_live = (d & 5) == 0, part_live = (d & 6) == 0;
          a = (own_live ? Ai : 0.0f) + (part_live ? uj.v[6] : 0.0f);
          b = (own_live ? Bi : 0.0f) + (part_live ? uj.v[7] : 0.0f);
        }
      } else {
        a = Ai + uj.v[6];
        b = Bi + uj.v[7];
        wv = d == 0 ? wv : 0.0f;
      }
      if constexpr (LIN) {
        // omega V_j ((A_i + A_j) X + (B_i + B_j) (X.du / |X|^2) X), along the reference bond X
        const float w = fmaf(b, __fdividef(sb.xu, sb.xx), a) * wv;
        fx = fmaf(w, X0, fx);
        fy = fmaf(w, X1, fy);
        fz = fmaf(w, X2, fz);
      } else {
        const float w = fmaf(sb.zeta, a, sb.e * b) * wv * sb.ry;
        fx = fmaf(w, sb.Yx, fx);
        fy = fmaf(w, sb.Yy, fy);
        fz = fmaf(w, sb.Yz, fz);
      }
    };
    uint8_t* dm = const_cast<uint8_t*>(dmg);  // not written by this pass
    if constexpr (SELL)
      sell_walk<PD_FORCE_NC>(i, lane, soff, col, dm, bx3, ur, body);
    else
      csr_walk<TPO, PD_FORCE_NC>(i, lane, row[i], row[i + 1], col, dm, bx3, ur, body);
  }
  fx = group_sum<TPO>(fx);
  fy = group_sum<TPO>(fy);
  fz = group_sum<TPO>(fz);
  split_epilogue<TPO>(E, i, lane, valid, fx, fy, fz, pt);
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
      const int d = dmg[b];  // bit 0: t_ij's half broken, bit 1: t_ji's
      if ((d & 3) == 3) continue;
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
      if (!(d & 1)) {
        fx = __dadd_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yx), dY), V));
        fy = __dadd_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yy), dY), V));
        fz = __dadd_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yz), dY), V));
      }
      if (!(d & 2)) {
        fx = __dsub_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yx), dY), V));
        fy = __dsub_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yy), dY), V));
        fz = __dsub_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yz), dY), V));
      }
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
// FP64 passes on the sliced bond stream (PD_FP64_SLICED): the FP64 LPS and
// critical-stretch formulas of k_dilatation_fp64 / k_force_fp64 on the split
// passes' layout, so that the two precisions compare on equal engineering.
// Per lane and block of 4 bonds: one int4 of neighbor ids (loaded a block
// ahead), one damage word and one 256-bit load per component of X (FP64
// planes of 128 values), then one gathered st record (y, V) per bond and, in
// the force pass, the neighbor's (A, B) from ab64. Owner constants are folded
// (theta = 3/m * sum V|X|e; t_ij + t_ji = (A_i + A_j)|X| + (B_i + B_j) e with
// A = theta (3K/m - alpha/3), B = alpha, elastic.cxx:99,119-120) and the force
// divides once per bond by |Y|, so the last bits differ from PD_FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ldcs_f64x4(const double* p, double* o) {
  asm("ld.global.cs.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3]) : "l"(p));
}
// 32-byte record of a point (read-only during the pass).
__device__ __forceinline__ double4 ld_f64x4_nc(const double4* p) {
  double4 r;
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(r.x), "=d"(r.y), "=d"(r.z), "=d"(r.w) : "l"(p));
  return r;
}
__device__ __forceinline__ double2 ld_f64x2_nc(const double4* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}

// Walks lane `lane` of owner i through its bonds of the sliced stream (the
// order of sell_walk): body(X0, X1, X2, damage byte, neighbor (y, V),
// neighbor (A, B) (zeros unless AB), the bond's damage byte in the stream,
// row offset r - lane).
template <bool AB, typename Body>
__device__ __forceinline__ void sell_walk64(int64_t i, int lane, const int64_t* __restrict__ soff,
                                            const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
                                            const double* __restrict__ bx, const double4* __restrict__ st,
                                            const double4* __restrict__ ab, Body&& body) {
  const int64_t s = i >> 3, so = soff[s];
  const int G = (int)(soff[s + 1] - so), F = G >> 2;
  const int l32 = (int)(i & 7) * 4 + lane;
  const int4* pc = reinterpret_cast<const int4*>(col + 32 * so + 4 * l32);
  uint32_t* pd = reinterpret_cast<uint32_t*>(dmg + 32 * so + 4 * l32);
  const double* px = bx + 96 * so + 4 * l32;
  int4 jn = F > 0 ? __ldcs(pc) : make_int4(0, 0, 0, 0);
#pragma unroll 1
  for (int b = 0; b < F; ++b, pc += 32, pd += 32, px += 384) {
    const int jv[4] = {jn.x, jn.y, jn.z, jn.w};
    if (b + 1 < F) jn = __ldcs(pc + 32);
    const uint32_t dw = __ldcs(pd);
    double X0[4], X1[4], X2[4];
    ldcs_f64x4(px, X0);
    ldcs_f64x4(px + 128, X1);
    ldcs_f64x4(px + 256, X2);
    double4 yj[4];
    double2 aj[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      yj[k] = ld_f64x4_nc(st + jv[k]);
      aj[k] = AB ? ld_f64x2_nc(ab + jv[k]) : make_double2(0.0, 0.0);
    }
    uint8_t* pb = reinterpret_cast<uint8_t*>(pd);
#pragma unroll
    for (int k = 0; k < 4; ++k) body(X0[k], X1[k], X2[k], (int)((dw >> (8 * k)) & 0xffu), yj[k], aj[k], pb + k, 16 * b + 4 * k);
  }
  const int T = G - 4 * F;
  if (T > 0) {  // tail groups: masked, one slot per lane per group
    const int64_t t0 = 32 * (so + 4 * F) + l32;
    const double* pt = bx + 96 * (so + 4 * F) + l32;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const bool in = k < T;
      const int32_t j = in ? __ldcs(col + t0 + 32 * k) : (int32_t)i;
      const int d = in ? (int)dmg[t0 + 32 * k] : kDummyBond;
      const double X0 = in ? __ldcs(pt + 96 * k) : 1.0;
      const double X1 = in ? __ldcs(pt + 96 * k + 32) : 0.0;
      const double X2 = in ? __ldcs(pt + 96 * k + 64) : 0.0;
      const double4 yj = ld_f64x4_nc(st + j);
      const double2 aj = AB ? ld_f64x2_nc(ab + j) : make_double2(0.0, 0.0);
      body(X0, X1, X2, d, yj, aj, dmg + t0 + 32 * k, 16 * F + 4 * k);
    }
  }
}

// Damage + dilatation. The break test is the reference's
// rel = (|Y| - |X|)/|X| > s_c (CriticalStretchDamageModel.cpp:155-158), run
// only for bonds with e > s_gate |X|, s_gate = s_min (1 - 1e-12) below every
// critical stretch of the body by more than the roundings of e/|X| and
// s_gate |X|, so that no bond the reference breaks skips it.
#ifndef PD_F64S_DIL_MINB
#define PD_F64S_DIL_MINB 4
#endif
#ifndef PD_F64S_FORCE_MINB
#define PD_F64S_FORCE_MINB 4
#endif
template <bool PAIR>
__global__ void __launch_bounds__(kSplitBlock, PD_F64S_DIL_MINB) k_dilatation_f64s(
    int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col, uint8_t* __restrict__ dmg,
    const double* __restrict__ bx, const double4* __restrict__ st, const double4* __restrict__ pt,
    const double* __restrict__ sc, int damage_on, double s_gate, double4* __restrict__ ab64,
    double* __restrict__ theta_out, double* __restrict__ node_damage, const int64_t* __restrict__ soff,
    uint8_t* __restrict__ dmg_csr) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / 4;
  const int lane = threadIdx.x & 3;
  const bool valid = i < n;
  double th = 0.0;
  int broken = 0;
  int len = 0;
  if (valid) {
    const int64_t b0 = row[i];
    len = (int)(row[i + 1] - b0);
    const double4 yi = ld_f64x4_nc(st + i);
    const double s_c = damage_on ? sc[i] : -1.0;
    uint8_t* cdm = dmg_csr + b0 + lane;  // the lane's bonds in the canonical CSR damage
    auto body = [&](double X0, double X1, double X2, int d, const double4& yj, const double2&, uint8_t* pdm,
                    int r) {
      // |X|, |Y| and e in the reference's operation order: the break test
      // sees the reference's stretch bit for bit
      const double Yx = __dsub_rn(yj.x, yi.x), Yy = __dsub_rn(yj.y, yi.y), Yz = __dsub_rn(yj.z, yi.z);
      const double zeta = __dsqrt_rn(sq3_rn(X0, X1, X2));
      const double e = __dsub_rn(__dsqrt_rn(sq3_rn(Yx, Yy, Yz)), zeta);
      const bool own_ok = (d & 5) == 0;  // own half intact (and a real bond)
      bool brk = false, brkp = false;
      if (damage_on && e > s_gate * zeta) {
        const double rel = __ddiv_rn(e, zeta);
        brk = own_ok && s_c >= 0.0 && rel > s_c;
        if (PAIR) {
          if ((d & 6) == 0) {
            const double scj = __ldg(sc + __ldg(col + (pdm - dmg)));
            brkp = scj >= 0.0 && rel > scj;
          }
        } else {
          brkp = brk;
        }
      }
      if (brk || brkp) {
        const uint8_t nd = (uint8_t)(d | (brk ? 1 : 0) | (brkp ? 2 : 0));
        *pdm = nd;
        cdm[r] = nd;  // the CSR copy stays canonical
      }
      broken += ((d & 1) || brk) ? 1 : 0;
      th = fma((own_ok && !brk) ? yj.w * zeta : 0.0, e, th);  // V_j |X| e
    };
    sell_walk64<false>(i, lane, soff, col, dmg, bx, st, nullptr, body);
  }
  th = group_sum<4>(th);
  broken = group_sum<4>(broken);
  if (valid && lane == 0) {
    const double4 p = pt[i];  // (m, K, mu, rho)
    // (a point with no own bonds, m = 0: theta = 0 and no force terms, as the
    // reference's loops over an empty family leave them)
    const bool fam = p.x > 0.0;
    const double theta = fam ? 3.0 * th / p.x : 0.0;
    const double alpha = fam ? 15.0 * p.z / p.x : 0.0;
    const double q = fam ? 3.0 * p.y / p.x - alpha / 3.0 : 0.0;
    ab64[i] = make_double4(theta * q, alpha, theta, 0.0);
    theta_out[i] = theta;
    node_damage[i] = len > 0 ? (double)broken / (double)len : 0.0;
  }
}

// Force gather + Verlet epilogue:
//   f_i += V_j (t_ij + t_ji) Y/|Y|,  t_ij = (1 - d_ij)(A_i |X| + B_i e),  t_ji likewise with j's terms
template <bool PAIR>
__global__ void __launch_bounds__(kSplitBlock, PD_F64S_FORCE_MINB) k_force_f64s(int64_t n, const int32_t* __restrict__ col,
                                                               const uint8_t* __restrict__ dmg,
                                                               const double* __restrict__ bx,
                                                               const double4* __restrict__ st,
                                                               const double4* __restrict__ ab64,
                                                               const double4* __restrict__ xv,
                                                               const double4* __restrict__ pt, EpiArgs E,
                                                               const int64_t* __restrict__ soff) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / 4;
  const int lane = threadIdx.x & 3;
  const bool valid = i < n;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (valid) {
    const double4 yi = ld_f64x4_nc(st + i);
    const double2 ai = ld_f64x2_nc(ab64 + i);
    auto body = [&](double X0, double X1, double X2, int d, const double4& yj, const double2& aj, uint8_t*, int) {
      const double Yx = __dsub_rn(yj.x, yi.x), Yy = __dsub_rn(yj.y, yi.y), Yz = __dsub_rn(yj.z, yi.z);
      const double zeta = __dsqrt_rn(sq3_rn(X0, X1, X2));
      const double dY = __dsqrt_rn(sq3_rn(Yx, Yy, Yz));
      const double e = __dsub_rn(dY, zeta);
      double a = ai.x + aj.x, b = ai.y + aj.y;
      if (d != 0) {  // a broken half or a padding slot (both intact is the common case)
        const bool own_live = (d & 5) == 0, part_live = PAIR ? (d & 6) == 0 : own_live;
        a = (own_live ? ai.x : 0.0) + (part_live ? aj.x : 0.0);
        b = (own_live ? ai.y : 0.0) + (part_live ? aj.y : 0.0);
      }
      // a padding slot gathers its own owner (Y = 0): no term, and no 0/0
      const double w = (d & kDummyBond) ? 0.0 : fma(zeta, a, e * b) * yj.w / dY;
      fx = fma(w, Yx, fx);
      fy = fma(w, Yy, fy);
      fz = fma(w, Yz, fz);
    };
    uint8_t* dm = const_cast<uint8_t*>(dmg);  // not written by this pass
    sell_walk64<true>(i, lane, soff, col, dm, bx, st, ab64, body);
  }
  fx = group_sum<4>(fx);
  fy = group_sum<4>(fy);
  fz = group_sum<4>(fz);
  if (valid && lane < 3) {
    const double f = lane == 0 ? fx : (lane == 1 ? fy : fz);
    verlet_epilogue(E, i, lane, f, comp3(xv[i], lane), pt[i].w);
  }
}

// FP64 X of the sliced stream (the slots and planes of k_pack_bonds<4, true>;
// padding slots X = (1, 0, 0)).
__global__ void __launch_bounds__(kBlock) k_pack_x64(int64_t n, const int64_t* __restrict__ row,
                                                     const int32_t* __restrict__ col,
                                                     const double4* __restrict__ xv, double* __restrict__ bx,
                                                     const int64_t* __restrict__ soff) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t i = g / 4;
  const int lane = threadIdx.x & 3;
  if (i >= n) return;
  const double4 xi = xv[i];
  const int64_t b0 = row[i], len = row[i + 1] - b0, ms = soff[(i >> 3) + 1] - soff[i >> 3];
  for (int64_t r = lane; r < 4 * ms; r += 4) {
    double X0 = 1.0, X1 = 0.0, X2 = 0.0;
    if (r < len) {
      const double4 xj = xv[col[b0 + r]];
      X0 = __dsub_rn(xj.x, xi.x);
      X1 = __dsub_rn(xj.y, xi.y);
      X2 = __dsub_rn(xj.z, xi.z);
    }
    int stride;
    double* p = bx + sell_x_index(soff, i, r, &stride);
    p[0] = X0;
    p[stride] = X1;
    p[2 * stride] = X2;
  }
}

// Volume in slot w of both FP64 coordinate records (the state writers keep it).
__global__ void k_st_volume(int64_t n, const double4* __restrict__ xv, double4* __restrict__ st0,
                            double4* __restrict__ st1) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double V = xv[i].w;
  st0[i].w = V;
  st1[i].w = V;
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
    double4* __restrict__ ab64, double* __restrict__ theta_out, double* __restrict__ node_damage, int pair) {
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
      const int d = dmg[b];  // bit 0: this half broken, bit 1: the partner's half
      if ((d & 3) == 3) {
        broken++;
        continue;
      }
      const int32_t j = col[b];
      const double4 xj = xv[j];
      const double4 yj = st[j];
      const double z0 = __dsub_rn(xj.x, xi.x), z1 = __dsub_rn(xj.y, xi.y), z2 = __dsub_rn(xj.z, xi.z);
      const double zeta = __dsqrt_rn(sq3_rn(z0, z1, z2));
      const double scj = pair && damage_on ? sc[j] : s_c;
      bool brk = false, brkp = false;
      if ((s_c >= 0.0 && !(d & 1)) || (scj >= 0.0 && !(d & 2))) {
        const double dY = __dsqrt_rn(sq3_rn(__dsub_rn(yj.x, yi.x), __dsub_rn(yj.y, yi.y), __dsub_rn(yj.z, yi.z)));
        const double rel = __ddiv_rn(__dsub_rn(dY, zeta), zeta);
        brk = !(d & 1) && s_c >= 0.0 && rel > s_c;
        brkp = !(d & 2) && scj >= 0.0 && rel > scj;
      }
      if (brk || brkp) dmg[b] = (uint8_t)(d | (brk ? 1 : 0) | (brkp ? 2 : 0));
      if ((d & 1) || brk) {
        broken++;
        continue;
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
      const int d = dmg[b];  // bit 0: t_ij's half broken, bit 1: t_ji's
      if ((d & 3) == 3) continue;
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
        if (!(d & 1)) f[r] = __dadd_rn(f[r], __dmul_rn(__dadd_rn(__dmul_rn(t1i, z[r]), __dmul_rn(t2i, mv)), V));
        if (!(d & 2)) f[r] = __dadd_rn(f[r], __dmul_rn(__dadd_rn(__dmul_rn(t1j, z[r]), __dmul_rn(t2j, mv)), V));
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
                                                    double height, double* __restrict__ node_damage, EpiArgs E, int pair) {
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
      const int d = dmg[b];  // bit 0: this half broken, bit 1: the partner's half
      if ((d & 3) == 3) {
        broken++;
        continue;
      }
      const int32_t j = col[b];
      const double4 xj = xv[j], yj = st[j];
      const double zeta = __dsqrt_rn(sq3_rn(__dsub_rn(xj.x, xi.x), __dsub_rn(xj.y, xi.y), __dsub_rn(xj.z, xi.z)));
      const double Yx = __dsub_rn(yj.x, yi.x), Yy = __dsub_rn(yj.y, yi.y), Yz = __dsub_rn(yj.z, yi.z);
      const double dY = __dsqrt_rn(sq3_rn(Yx, Yy, Yz));
      const double stretch = __ddiv_rn(__dsub_rn(dY, zeta), zeta);
      const double scj = pair && damage_on ? sc[j] : s_c;
      const bool brk = !(d & 1) && s_c >= 0.0 && stretch > s_c;
      const bool brkp = !(d & 2) && scj >= 0.0 && stretch > scj;
      if (brk || brkp) dmg[b] = (uint8_t)(d | (brk ? 1 : 0) | (brkp ? 2 : 0));
      const bool own_live = !(d & 1) && !brk, part_live = !(d & 2) && !brkp;
      if (!own_live) broken++;
      if (!own_live && !part_live) continue;
      const double cj = bb_constant(pt[j].y, hp[j], plane, height);
      const double ti = __dmul_rn(__dmul_rn(0.5, stretch), ci);  // 0.5*(1-d)*stretch*constant, d = 0
      const double tj = __dmul_rn(__dmul_rn(0.5, stretch), cj);
      const double V = xj.w;
      if (own_live) {
        fx = __dadd_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yx), dY), V));
        fy = __dadd_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yy), dY), V));
        fz = __dadd_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(ti, Yz), dY), V));
      }
      if (part_live) {
        fx = __dsub_rn(fx, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yx), dY), V));
        fy = __dsub_rn(fy, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yy), dY), V));
        fz = __dsub_rn(fz, __dmul_rn(__ddiv_rn(__dmul_rn(tj, -Yz), dY), V));
      }
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
template <int TPO, bool SELL, bool PAIR = false>
__global__ void __launch_bounds__(kSplitBlock, PD_BOND_MINB) k_bb_split(int64_t n, const int64_t* __restrict__ row,
                                                                   const int32_t* __restrict__ col,
                                                                   uint8_t* __restrict__ dmg,
                                                                   const float* __restrict__ bx3,
                                                                   const Rec8* __restrict__ ur,
                                                                   const float4* __restrict__ own, int damage_on,
                                                                   const double4* __restrict__ pt,
                                                                   double* __restrict__ node_damage, EpiArgs E,
                                                                   const int64_t* __restrict__ soff,
                                                                   uint8_t* __restrict__ dmg_csr,
                                                                   const float* __restrict__ scf, float s_min) {
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
    const Rec8 ri = ld_rec_nc(ur + i);
    const OwnU ui = own_u(ri);
    const float ci = ri.v[6];
    const float s_c = damage_on ? own[i].w : -1.0f;
    uint8_t* cdm = SELL ? dmg_csr + b0 + lane : nullptr;  // the lane's bonds in the canonical CSR damage
    auto body = [&](float X0, float X1, float X2, int d, const Rec8& uj, int32_t, uint8_t* pdm, int r) {
      const SplitBond sb = split_bond<true>(X0, X1, X2, ui, uj);
      const bool own_ok = (d & 5) == 0;
      const bool part_ok = PAIR ? (d & 6) == 0 : own_ok;
      bool brk, brkp;
      if (PAIR) {  // both tests only past the body's smallest s_c (as the dilatation pass)
        brk = brkp = false;
        if (damage_on && sb.e > s_min * sb.zeta) {
          brk = own_ok && s_c >= 0.0f && sb.e > s_c * sb.zeta;
          if (part_ok) {
            const float scj = __ldg(scf + __ldg(col + (pdm - dmg)));
            brkp = scj >= 0.0f && sb.e > scj * sb.zeta;
          }
        }
      } else {
        brk = brkp = own_ok && s_c >= 0.0f && sb.e > s_c * sb.zeta;
      }
      if (brk || brkp) {
        const uint8_t nd = (uint8_t)(d | (brk ? 1 : 0) | (brkp ? 2 : 0));
        *pdm = nd;
        if (SELL) cdm[r] = nd;
      }
      broken += ((d & 1) || brk) ? 1 : 0;
      // t_ij + t_ji over the intact halves
      const float c = ((own_ok && !brk) ? ci : 0.0f) + ((part_ok && !brkp) ? uj.v[6] : 0.0f);
      const float w = c * __fdividef(sb.e, sb.zeta) * uj.v[5] * sb.ry;
      fx = fmaf(w, sb.Yx, fx);
      fy = fmaf(w, sb.Yy, fy);
      fz = fmaf(w, sb.Yz, fz);
    };
    if constexpr (SELL)
      sell_walk<1>(i, lane, soff, col, dmg, bx3, ur, body);
    else
      csr_walk<TPO, 1>(i, lane, b0, b0 + len, col, dmg, bx3, ur, body);
  }
  fx = group_sum<TPO>(fx);
  fy = group_sum<TPO>(fy);
  fz = group_sum<TPO>(fz);
  broken = group_sum<TPO>(broken);
  if (valid && lane == 0) node_damage[i] = len > 0 ? (double)broken / (double)len : 0.0;
  split_epilogue<TPO>(E, i, lane, valid, fx, fy, fz, pt);
}

// ---------------------------------------------------------------------------
// State conversions and the stable time step
// ---------------------------------------------------------------------------
// State from current coordinates y [3n]: u = y - x (FP64), then the gathered
// copy (split: displacement record, FP64: y itself).
// (points i0 .. n-1)
__global__ void k_state_from_y(int64_t n, const double* __restrict__ y, const double4* __restrict__ xv,
                               double* __restrict__ u, double4* __restrict__ st, Rec8* __restrict__ ur,
                               int64_t i0 = 0) {
  const int64_t i = i0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 x = xv[i];
  const double y0 = y[3 * i], y1 = y[3 * i + 1], y2 = y[3 * i + 2];
  const double u0 = y0 - x.x, u1 = y1 - x.y, u2 = y2 - x.z;
  u[3 * i] = u0;
  u[3 * i + 1] = u1;
  u[3 * i + 2] = u2;
  if (ur) {
    store_u_record(ur + i, u0, u1, u2);
  } else {
    st[i] = make_double4(y0, y1, y2, x.w);
  }
}

// Gathered state from the displacement u [3n] (after pd_set_state): split ->
// displacement record, FP64 -> y = x + u.
__global__ void k_state_from_u(int64_t n, const double* __restrict__ u, const double4* __restrict__ xv,
                               double4* __restrict__ st, Rec8* __restrict__ ur) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 x = xv[i];
  if (ur) {
    store_u_record(ur + i, u[3 * i], u[3 * i + 1], u[3 * i + 2]);
  } else {
    st[i] = make_double4(__dadd_rn(x.x, u[3 * i]), __dadd_rn(x.y, u[3 * i + 1]), __dadd_rn(x.z, u[3 * i + 2]), x.w);
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
                                                        const double* __restrict__ hp, double* __restrict__ partial,
                                                        const uint8_t* __restrict__ phantom) {
  // phantom: as k_weighted_volume (the sum runs over the point's own family)
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
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += TPO) {
      if (phantom && (phantom[b] & kPhantomOwn)) continue;
      ++nn;
      const double4 xj = xv[col[b]];
      const double d = __dsqrt_rn(sq3_rn(__dsub_rn(xi.x, xj.x), __dsub_rn(xi.y, xj.y), __dsub_rn(xi.z, xj.z)));
      den = __dadd_rn(den, __ddiv_rn(__dmul_rn(xj.w, spring), d));
    }
  }
  den = group_sum<TPO>(den);
  nn = group_sum<TPO>(nn);
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
                  c->influence, c->pt.p, c->phantoms ? c->dmg.p : nullptr);
  return cudaGetLastError();
}

cudaError_t launch_pack_owner(pd_ctx* c) {
  if (c->n == 0 || c->precision == PD_FP64) return cudaSuccess;
  const bool f64s = c->precision == PD_FP64_SLICED;
  const bool bb = c->material_model == PD_MATERIAL_BOND_BASED;
  const int64_t n = c->n;
  if (f64s) {
    k_st_volume<<<grid1(n), kBlock, 0, c->stream>>>(n, c->xv.p, c->st[0].p, c->st[1].p);
  } else {
    k_pack_owner<<<grid1(n), kBlock, 0, c->stream>>>(n, c->pt.p, c->sc.p, c->own.p);
    k_pack_volume<<<grid1(n), kBlock, 0, c->stream>>>(n, c->xv.p, c->ur[0].p, c->ur[1].p);
  }
  c->sell = f64s || c->tpo_split == 4;
  cudaError_t e;
  if (c->sell) {  // sliced bond stream of the 4-lanes-per-point passes
    const int64_t ns = (n + 7) / 8;
    pdb::DBuf<int64_t> cnt;
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
    // slots counts 32-record groups: 32 ids and damage bytes, 96 values of X each
    const size_t groups = (size_t)std::max<int64_t>(slots, 1);
    c->bx3.release();  // the old stream first: at memory scale both would not fit
    c->bx64.release();
    if (f64s) {
      if ((e = c->bx64.alloc(96 * groups)) != cudaSuccess) return e;
    } else {
      if ((e = c->bx3.alloc(96 * groups)) != cudaSuccess) return e;
    }
    if ((e = c->sell_col.alloc(32 * groups)) != cudaSuccess) return e;
    if ((e = c->sell_dmg.alloc(32 * groups)) != cudaSuccess) return e;
    // ids, damage and (split) FP32 X; on the FP64 sliced path no FP32 X, and
    // k_pack_x64 writes the FP64 planes
    if (f64s) {
      k_pack_bonds<4, true><<<grid_for(n, 4), kBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->xv.p, nullptr,
                                                                      c->sell_off.p, c->dmg.p, c->sell_col.p,
                                                                      c->sell_dmg.p);
      k_pack_x64<<<grid_for(n, 4), kBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->xv.p, c->bx64.p,
                                                           c->sell_off.p);
    } else {
      k_pack_bonds<4, true><<<grid_for(n, 4), kBlock, 0, c->stream>>>(n, c->row.p, c->col.p, c->xv.p, c->bx3.p,
                                                                      c->sell_off.p, c->dmg.p, c->sell_col.p,
                                                                      c->sell_dmg.p);
    }
    c->sell_src = c->dmg.p;
    c->sell_gen = c->dmg_gen;
  } else {
    c->bx3.release();
    if ((e = c->bx3.alloc(96 * (size_t)((c->nb + 31) / 32))) != cudaSuccess) return e;
    PD_DISPATCH_TPO_CSR(c->tpo, k_pack_bonds, grid_for(n, c->tpo), kBlock, n, c->row.p, c->col.p, c->xv.p, c->bx3.p,
                        nullptr, nullptr, nullptr, nullptr);
  }
  if (bb)
    k_bb_terms<<<grid1(n), kBlock, 0, c->stream>>>(n, c->pt.p, c->hp.p, c->bb_plane, c->bb_height, c->ur[0].p,
                                                   c->ur[1].p);
  return cudaGetLastError();
}

cudaError_t launch_state_from_y(pd_ctx* c, const double* y_dev, int64_t i0, int64_t i1) {
  if (i1 < 0) i1 = c->n;
  if (i1 <= i0) return cudaSuccess;
  const bool split = c->precision == PD_SPLIT_FP32;
  k_state_from_y<<<grid1(i1 - i0), kBlock, 0, c->stream>>>(i1, y_dev, c->xv.p, c->u.p,
                                                           split ? nullptr : c->st[c->cur].p,
                                                           split ? c->ur[c->cur].p : nullptr, i0);
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

// Split-pass kernels by lanes per point (sliced stream at 4), material,
// influence weighting and half-bond damage (all instances of a pass share one
// signature).
template <bool LIN, bool W, bool P>
static decltype(&k_dilatation_split<4, true>) dil_split_kernel(int tpo, bool sell) {
  if (sell || LIN) return &k_dilatation_split<4, true, LIN, W, P>;  // linear LPS runs on the sliced stream only
  switch (tpo) {
    case 4: return &k_dilatation_split<4, false, false, W, P>;
    case 8: return &k_dilatation_split<8, false, false, W, P>;
    case 16: return &k_dilatation_split<16, false, false, W, P>;
    default: return &k_dilatation_split<32, false, false, W, P>;
  }
}
template <bool LIN, bool CHUNK, bool W, bool P>
static decltype(&k_force_split<4, true>) force_split_kernel(int tpo, bool sell) {
  if (sell || LIN || CHUNK) return &k_force_split<4, true, LIN, CHUNK, W, P>;
  switch (tpo) {
    case 4: return &k_force_split<4, false, false, false, W, P>;
    case 8: return &k_force_split<8, false, false, false, W, P>;
    case 16: return &k_force_split<16, false, false, false, W, P>;
    default: return &k_force_split<32, false, false, false, W, P>;
  }
}
template <bool LIN, bool W>
static decltype(&k_dilatation_split<4, true>) dil_split_for(bool pair, int tpo, bool sell) {
  return pair ? dil_split_kernel<LIN, W, true>(tpo, sell) : dil_split_kernel<LIN, W, false>(tpo, sell);
}
template <bool CHUNK, bool W>
static decltype(&k_force_split<4, true>) force_split_w(const pd_ctx* c, bool pair, int tpo, bool sell) {
  const bool lin = c->material_model == PD_MATERIAL_LINEAR_LPS;
  return lin ? (pair ? force_split_kernel<true, CHUNK, W, true>(tpo, sell) : force_split_kernel<true, CHUNK, W, false>(tpo, sell))
             : (pair ? force_split_kernel<false, CHUNK, W, true>(tpo, sell) : force_split_kernel<false, CHUNK, W, false>(tpo, sell));
}
template <bool CHUNK>
static decltype(&k_force_split<4, true>) force_split_for(const pd_ctx* c, bool pair, int tpo, bool sell) {
  return c->influence != PD_INFLUENCE_ONE ? force_split_w<CHUNK, true>(c, pair, tpo, sell)
                                          : force_split_w<CHUNK, false>(c, pair, tpo, sell);
}
template <bool P>
static decltype(&k_bb_split<4, true>) bb_split_kernel(int tpo, bool sell) {
  if (sell) return &k_bb_split<4, true, P>;
  switch (tpo) {
    case 4: return &k_bb_split<4, false, P>;
    case 8: return &k_bb_split<8, false, P>;
    case 16: return &k_bb_split<16, false, P>;
    default: return &k_bb_split<32, false, P>;
  }
}

// The stream and events of the chunked force download (created on first use).
static cudaError_t ensure_copy_stream(pd_ctx* c) {
  if (c->copy_stream) return cudaSuccess;
  TRY_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  for (int k = 0; k <= kHostChunks; ++k) TRY_CUDA(cudaEventCreateWithFlags(&c->chunk_ev[k], cudaEventDisableTiming));
  for (int k = 0; k < kHostChunks; ++k) TRY_CUDA(cudaEventCreateWithFlags(&c->up_ev[k], cudaEventDisableTiming));
  return cudaSuccess;
}

// Points per host-transfer chunk (a multiple of 64: whole slices of the
// sliced stream).
static int64_t host_chunk(int64_t n) { return ((n + kHostChunks - 1) / kHostChunks + 63) / 64 * 64; }

// hi[k] = the largest neighbor index of the rows of chunk k (at least the
// chunk's last point): a thread per point, then per chunk that the block's
// 256 points reach (chunks are multiples of 64 points: at most four) a block
// maximum and one atomicMax. hi must start at 0.
__global__ void __launch_bounds__(256) k_chunk_hi(int64_t n, int64_t per, const int64_t* __restrict__ row,
                                                  const int32_t* __restrict__ col, unsigned long long* __restrict__ hi) {
  __shared__ unsigned long long sm[256];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t first = (int64_t)blockIdx.x * blockDim.x;
  unsigned long long m = 0;
  if (i < n) {
    m = (unsigned long long)i;
    for (int64_t b = row[i]; b < row[i + 1]; ++b) m = max(m, (unsigned long long)col[b]);
  }
  const int64_t last = min(n, first + (int64_t)blockDim.x) - 1;
  for (int64_t k = first / per; k <= last / per; ++k) {  // block-uniform
    sm[threadIdx.x] = (i < n && i / per == k) ? m : 0ull;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) sm[threadIdx.x] = max(sm[threadIdx.x], sm[threadIdx.x + o]);
      __syncthreads();
    }
    if (threadIdx.x == 0) atomicMax(hi + k, sm[0]);
    __syncthreads();
  }
}

// c->chunk_hi for the current bond set (computed once per bond set).
static cudaError_t ensure_chunk_hi(pd_ctx* c) {
  if (c->chunk_hi_row == c->row.p && c->chunk_hi_nb == c->nb && (int)c->chunk_hi.size() == kHostChunks)
    return cudaSuccess;
  const int64_t n = c->n, per = host_chunk(n);
  DBuf<unsigned long long> hi;
  TRY_CUDA(hi.alloc(kHostChunks));
  TRY_CUDA(dzero(c, hi.p, kHostChunks * sizeof(unsigned long long)));
  if (n > 0)
    k_chunk_hi<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, per, c->row.p, c->col.p, hi.p);
  TRY_CUDA(cudaGetLastError());
  std::vector<unsigned long long> h(kHostChunks, 0);
  TRY_CUDA(d2h(c, h.data(), hi.p, kHostChunks * sizeof(unsigned long long)));
  c->chunk_hi.assign(h.begin(), h.end());
  c->chunk_hi_row = c->row.p;
  c->chunk_hi_nb = c->nb;
  return cudaSuccess;
}

__global__ void k_node_damage_own(int64_t n, const int64_t* __restrict__ row, const uint8_t* __restrict__ dmg,
                                  double* __restrict__ node_damage);
// With phantom halves in the rows the passes count them as broken; the node
// damage is then recounted over the own families.
static cudaError_t own_node_damage(pd_ctx* c, const uint8_t* dmg) {
  if (!c->phantoms || c->n == 0) return cudaSuccess;
  k_node_damage_own<<<(unsigned)((c->n * 8 + kBlock - 1) / kBlock), kBlock, 0, c->stream>>>(c->n, c->row.p, dmg,
                                                                                             c->node_damage.p);
  return cudaGetLastError();
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
  E.bc_cp = c->n_bc_expr ? c->bc_cp.p : nullptr;
  // values of the prescribed functions at this evaluation's two times
  if (c->n_bc_expr && sp.has_bc && sp.mode == EVAL_ADVANCE) TRY_CUDA(launch_bc_expr(c, sp.step, sp.t0, sp.dt));
  E.st_next = split ? nullptr : c->st[c->cur ^ 1].p;
  E.ur_next = split ? c->ur[c->cur ^ 1].p : nullptr;
  E.status = c->status.p;
  // Split passes at 4 lanes per point read the sliced bond stream; its damage
  // mirror follows the CSR damage array this evaluation uses.
  const bool f64s = c->precision == PD_FP64_SLICED;
  const bool sell = split && c->sell && tpo == 4;
  if ((sell || f64s) && (c->sell_src != dmg || c->sell_gen != c->dmg_gen)) {
    k_sell_dmg<<<grid_for(c->n, 4), kBlock, 0, c->stream>>>(c->n, c->row.p, c->sell_off.p, dmg, c->sell_dmg.p);
    c->sell_src = dmg;
    c->sell_gen = c->dmg_gen;
  }
  const int32_t* scol = sell ? c->sell_col.p : c->col.p;
  uint8_t* sdmg = sell ? c->sell_dmg.p : dmg;
  const int64_t* soff = sell ? c->sell_off.p : nullptr;
  // host coordinates: chunked beside the dilatation on the sliced split path
  // (LPS and linear LPS), else one upload before the passes
  const bool chunk_in = sp.y_host && sp.f_out && sell && c->material_model != PD_MATERIAL_BOND_BASED;
  if (sp.y_host && !chunk_in) {
    TRY_CUDA(cudaMemcpyAsync(sp.f_out, sp.y_host, 3 * (size_t)c->n * sizeof(double), cudaMemcpyHostToDevice,
                             c->stream));
    TRY_CUDA(launch_state_from_y(c, sp.f_out));
  }
  // half-bond damage: the two halves of a bond can differ (critical stretch
  // varying along bonds, or caller-set damage with differing halves)
  const bool pair = c->sc_pair || c->dmg_asym;
  const int ipair = pair ? 1 : 0;
  if (f64s) {  // LPS only (other materials are refused when the context is made ready)
    auto* kd = pair ? &k_dilatation_f64s<true> : &k_dilatation_f64s<false>;
    kd<<<grid_split(c->n, 4), kSplitBlock, 0, c->stream>>>(c->n, c->row.p, c->sell_col.p, c->sell_dmg.p, c->bx64.p,
                                                           c->st[c->cur].p, c->pt.p, c->sc.p, sp.damage_on,
                                                           c->sc_gate64, c->ab64.p, c->theta.p, c->node_damage.p,
                                                           c->sell_off.p, dmg);
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(own_node_damage(c, dmg));
    if (ev) cudaEventRecord(ev[1], c->stream);
    auto* kf = pair ? &k_force_f64s<true> : &k_force_f64s<false>;
    kf<<<grid_split(c->n, 4), kSplitBlock, 0, c->stream>>>(c->n, c->sell_col.p, c->sell_dmg.p, c->bx64.p,
                                                           c->st[c->cur].p, c->ab64.p, c->xv.p, c->pt.p, E,
                                                           c->sell_off.p);
    if (ev) cudaEventRecord(ev[2], c->stream);
    return cudaGetLastError();
  }
  if (c->material_model == PD_MATERIAL_BOND_BASED) {  // one pass: damage + pair force + epilogue
    if (ev) cudaEventRecord(ev[1], c->stream);
    if (split) {
      auto* kb = pair ? bb_split_kernel<true>(tpo, sell) : bb_split_kernel<false>(tpo, sell);
      kb<<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, scol, sdmg, c->bx3.p, c->ur[c->cur].p, c->own.p,
                                               sp.damage_on, c->pt.p, c->node_damage.p, E, soff, sell ? dmg : nullptr,
                                               c->scf.p, c->sc_min);
    } else {
      PD_DISPATCH_TPO(tpo, k_bb_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p, c->pt.p, c->sc.p,
                      c->hp.p, sp.damage_on, c->bb_plane, c->bb_height, c->node_damage.p, E, ipair);
    }
    TRY_CUDA(cudaGetLastError());
    TRY_CUDA(own_node_damage(c, dmg));
    if (ev) cudaEventRecord(ev[2], c->stream);
    return cudaGetLastError();
  }
  if (split) {
    const bool lin = c->material_model == PD_MATERIAL_LINEAR_LPS, w = c->influence != PD_INFLUENCE_ONE;
    auto* kd = lin ? (w ? dil_split_for<true, true>(pair, tpo, sell) : dil_split_for<true, false>(pair, tpo, sell))
                   : (w ? dil_split_for<false, true>(pair, tpo, sell) : dil_split_for<false, false>(pair, tpo, sell));
    if (chunk_in) {
      // The coordinates go up in chunks on the copy stream; the displacement
      // records of a chunk are formed once it has landed, and the dilatation
      // of chunk k runs once every chunk up to the one holding its rows'
      // largest neighbor index has its records.
      TRY_CUDA(ensure_copy_stream(c));
      TRY_CUDA(ensure_chunk_hi(c));
      // (every earlier use of the staging buffer ended with its call: the
      // entry points synchronise both streams before they return)
      const int64_t n = c->n, per = host_chunk(n);
      int nk = 0;
      for (int64_t i0 = 0; i0 < n; i0 += per, ++nk) {
        const int64_t i1 = std::min(n, i0 + per);
        TRY_CUDA(cudaMemcpyAsync(sp.f_out + 3 * i0, sp.y_host + 3 * i0, 3 * (i1 - i0) * sizeof(double),
                                 cudaMemcpyHostToDevice, c->copy_stream));
        TRY_CUDA(cudaEventRecord(c->up_ev[nk], c->copy_stream));
      }
      int formed = 0;  // chunks whose records are formed
      auto form_through = [&](int k) -> cudaError_t {
        for (; formed <= k && formed < nk; ++formed) {
          const int64_t j0 = formed * per, j1 = std::min(n, j0 + per);
          TRY_CUDA(cudaStreamWaitEvent(c->stream, c->up_ev[formed], 0));
          TRY_CUDA(launch_state_from_y(c, sp.f_out, j0, j1));
        }
        return cudaSuccess;
      };
      for (int k = 0; k < nk; ++k) {
        const int64_t i0 = k * per, i1 = std::min(n, i0 + per);
        TRY_CUDA(form_through(std::max<int>(k, (int)(c->chunk_hi[k] / per))));
        kd<<<grid_split(i1 - i0, tpo), kSplitBlock, 0, c->stream>>>(
            i1, c->row.p, scol, sdmg, c->bx3.p, c->ur[c->cur].p, c->own.p, sp.damage_on, c->theta.p,
            c->node_damage.p, soff, dmg, c->hp.p, c->influence, c->scf.p, c->sc_min, i0);
      }
      TRY_CUDA(form_through(nk - 1));
    } else {
      kd<<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, scol, sdmg, c->bx3.p, c->ur[c->cur].p, c->own.p,
                                               sp.damage_on, c->theta.p, c->node_damage.p, soff, sell ? dmg : nullptr,
                                               c->hp.p, c->influence, c->scf.p, c->sc_min, 0);
    }
  } else if (c->material_model == PD_MATERIAL_LINEAR_LPS) {
    PD_DISPATCH_TPO(tpo, k_dilatation_lin_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p,
                    c->pt.p, c->sc.p, c->hp.p, c->influence, sp.damage_on, c->ab64.p, c->theta.p, c->node_damage.p,
                    ipair);
  } else {
    PD_DISPATCH_TPO(tpo, k_dilatation_fp64, grid, c->n, c->row.p, c->col.p, dmg, c->xv.p, c->st[c->cur].p, c->pt.p,
                    c->sc.p, c->hp.p, c->influence, sp.damage_on, c->ab64.p, c->theta.p, c->node_damage.p, ipair);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  TRY_CUDA(own_node_damage(c, dmg));
  if (ev) cudaEventRecord(ev[1], c->stream);
  if (sell) {
    if (sp.f_host && sp.f_out) {
      auto* kf = force_split_for<true>(c, pair, tpo, sell);
      // Force in chunks of points; each chunk's force density goes to the host
      // on the copy stream while the next chunk computes.
      TRY_CUDA(ensure_copy_stream(c));
      const int64_t n = c->n, per = host_chunk(n);
      // (all chunks are launched before the first copy: a copy to pageable
      // memory holds the host until it is done)
      for (int64_t i0 = 0, k = 0; i0 < n; i0 += per, ++k) {
        const int64_t i1 = std::min(n, i0 + per);
        kf<<<grid_split(i1 - i0, 4), kSplitBlock, 0, c->stream>>>(i1, c->row.p, scol, sdmg, c->bx3.p, c->ur[c->cur].p,
                                                                  c->pt.p, E, soff, c->hp.p, c->influence, i0);
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
      auto* kf = force_split_for<false>(c, pair, tpo, sell);
      kf<<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, scol, sdmg, c->bx3.p, c->ur[c->cur].p, c->pt.p, E, soff,
                                               c->hp.p, c->influence, 0);
    }
  } else if (split) {
    auto* kf = force_split_for<false>(c, pair, tpo, false);
    kf<<<sgrid, kSplitBlock, 0, c->stream>>>(c->n, c->row.p, c->col.p, dmg, c->bx3.p, c->ur[c->cur].p, c->pt.p, E,
                                             nullptr, c->hp.p, c->influence, 0);
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

// Node damage over the points' own families (phantom halves are neither
// bonds nor breaks of the row): CriticalStretchDamageModel.cpp:170-183.
__global__ void k_node_damage_own(int64_t n, const int64_t* __restrict__ row, const uint8_t* __restrict__ dmg,
                                  double* __restrict__ node_damage) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const int lane = threadIdx.x & 7;
  int own = 0, broken = 0;
  if (i < n)  // (every lane reaches the shuffles)
    for (int64_t b = row[i] + lane; b < row[i + 1]; b += 8) {
      const int d = dmg[b];
      own += (d & kPhantomOwn) ? 0 : 1;
      broken += (d & (1 | kPhantomOwn)) == 1 ? 1 : 0;
    }
  for (int o = 4; o > 0; o >>= 1) {
    own += __shfl_xor_sync(0xffffffffu, own, o, 8);
    broken += __shfl_xor_sync(0xffffffffu, broken, o, 8);
  }
  if (i < n && lane == 0) node_damage[i] = own > 0 ? (double)broken / (double)own : 0.0;
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
                  c->sc.p, c->hp.p, c->influence, 0, ab, theta, nd, 0);
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
  PD_DISPATCH_TPO(c->tpo, k_critical_dt, grid, c->n, c->row.p, c->col.p, c->xv.p, c->pt.p, c->hp.p, c->scratch.p,
                  c->phantoms ? c->dmg.p : nullptr);
  k_min_reduce<<<1, kBlock, 0, c->stream>>>((int64_t)grid, c->scratch.p, dt_out_dev);
  return cudaGetLastError();
}

int64_t critical_dt_partials(const pd_ctx* c) { return (int64_t)grid_for(c->n, c->tpo); }

cudaError_t launch_critical_dt_into(pd_ctx* c, double* partial, double* dt_out_dev) {
  const unsigned grid = grid_for(c->n, c->tpo);
  PD_DISPATCH_TPO(c->tpo, k_critical_dt, grid, c->n, c->row.p, c->col.p, c->xv.p, c->pt.p, c->hp.p, partial,
                  c->phantoms ? c->dmg.p : nullptr);
  k_min_reduce<<<1, kBlock, 0, c->stream>>>((int64_t)grid, partial, dt_out_dev);
  return cudaGetLastError();
}

}  // namespace pdb

namespace pdb {

__global__ void k_u_from_record(int64_t n, const Rec8* __restrict__ ur, double* __restrict__ u) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double uu[3];
  load_u_record(ur[i], uu);
  for (int c = 0; c < 3; ++c) u[3 * i + c] = uu[c];
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

// The receiving side: u and the record the next evaluation gathers (the
// displacement record on the split path, y on the FP64 path), both as the
// owner holds them.
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
    store_u_record(ur + i, v[0], v[1], v[2]);
  } else {
    st[i] = make_double4(v[3], v[4], v[5], st[i].w);
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

// Broken bonds of the families: bond damage bytes with the row's own half (bit 0) set, phantom halves not counted.
__global__ void k_count_nonzero(int64_t m, const uint8_t* __restrict__ d, unsigned long long* __restrict__ out) {
  unsigned long long cnt = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
    cnt += (d[k] & (1 | kPhantomOwn)) == 1 ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

// Position of bond (j, i) in row j (rows strictly ascending; families symmetric).
__device__ __forceinline__ int64_t partner_bond(const int64_t* __restrict__ row, const int32_t* __restrict__ col,
                                                int64_t i, int32_t j) {
  int64_t lo = row[j], hi = row[j + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (col[mid] < (int32_t)i) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Half-bond damage bytes from per-bond damage of the rows' own halves (src,
// bit 0): bit 1 of bond (i, j) = bit 0 of bond (j, i). flag[0] is set when a
// bond's two halves differ.
__global__ void k_mirror_damage(int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col,
                                const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int* __restrict__ flag) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const int lane = threadIdx.x & 7;
  if (i >= n) return;
  bool asym = false;
  for (int64_t b = row[i] + lane; b < row[i + 1]; b += 8) {
    const int32_t j = col[b];
    const int64_t bp = partner_bond(row, col, i, j);
    const bool found = bp < row[j + 1] && col[bp] == (int32_t)i;
    const int own = src[b] & 1, part = found ? (src[bp] & 1) : own;
    // phantom halves keep their markers: the own one from this byte, the
    // partner one from the partner's own marker
    const int mk = (src[b] & kPhantomOwn) | (found && (src[bp] & kPhantomOwn) ? kPhantomPartner : 0);
    dst[b] = (uint8_t)(own | (part << 1) | mk);
    asym |= own != part;
  }
  if (asym) atomicOr(flag, 1);
}

// flag[0] set when some bond joins points of different critical stretch.
__global__ void k_pair_check(int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col,
                             const double* __restrict__ sc, int* __restrict__ flag) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const int lane = threadIdx.x & 7;
  if (i >= n) return;
  const double si = sc[i];
  bool diff = false;
  for (int64_t b = row[i] + lane; b < row[i + 1]; b += 8) diff |= sc[col[b]] != si;
  if (diff) atomicOr(flag, 1);
}

static int run_flag_kernel(pd_ctx* c, int which, const uint8_t* src, uint8_t* dst, bool* out) {
  DBuf<int> flag;
  PD_CUDA_TRY(c, flag.alloc(1));
  PD_CUDA_TRY(c, cudaMemsetAsync(flag.p, 0, sizeof(int), c->stream));
  const unsigned g = (unsigned)((c->n * 8 + kBlock - 1) / kBlock);
  if (c->n > 0) {
    if (which == 0) k_mirror_damage<<<g, kBlock, 0, c->stream>>>(c->n, c->row.p, c->col.p, src, dst, flag.p);
    else k_pair_check<<<g, kBlock, 0, c->stream>>>(c->n, c->row.p, c->col.p, c->sc.p, flag.p);
    PD_CUDA_TRY(c, cudaGetLastError());
  }
  int h = 0;
  PD_CUDA_TRY(c, d2h(c, &h, flag.p, sizeof(int)));
  *out = h != 0;
  return PD_OK;
}

// Damage bytes of both halves from own-half damage in src (device), into dst.
int mirror_damage(pd_ctx* c, const uint8_t* src, uint8_t* dst) { return run_flag_kernel(c, 0, src, dst, &c->dmg_asym); }

// Whether the critical stretch differs across some bond (the sc array is uploaded).
int check_sc_pairs(pd_ctx* c) { return run_flag_kernel(c, 1, nullptr, nullptr, &c->sc_pair); }

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
