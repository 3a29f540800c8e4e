// Learned middle level of the quasi-static CG preconditioner (sm_100a).
// No counterpart in the reference. The preconditioner is
//
//   z = P_bj r  +  P0 Ac^-1 P0^T r  +  Q S G^T G S Q^T r
//       block      exact coarse        learned middle level
//       Jacobi     (k_coarse.cu)       (this file)
//
// Q: piecewise-constant prolongation from "patches" (the non-empty cells of a
// grid of side `patch`, about two lattice spacings) to the free dofs of their
// points; S: one positive scale per patch, s_I = sqrt(sum_{i in I} tr'(D_i^-1)/3)
// / |I| from the block-Jacobi inverse blocks D_i^-1 (tr': free dofs only; the
// patch's Galerkin diagonal is about |I| / that sum); G: a linear message-passing network on
// the patch graph (patches joined to the non-empty cells of their 3x3x3
// neighborhood, whose points are bonded):
//
//   h0 = W0 v                                   v = S Q^T r, 3 -> 64 channels
//   h_l = h_{l-1} + Ws_l h_{l-1} + Wn_l mean_{J in N(I)} h_{l-1,J},  l = 1..3
//
// with hidden 64, BF16 weights and FP32 activations and accumulation. G^T G is
// symmetric positive semi-definite and S diagonal positive, so M stays
// symmetric positive definite and CG keeps its optimality (the solver takes
// the flexible Polak-Ribiere beta, equal to the standard one for a fixed SPD
// M, against the FP32 rounding of the network's product). The middle
// level covers the band between block Jacobi (the nearest neighbors) and the
// coarse cells (two horizons): an exact patch-level solve halves the two-level
// CG iterations on a 24^3 cube; G^T G is trained to approximate it locally.
//
// Training: pairs (r_k, e_k = x* - x_k) captured from two-level CG solves
// (K e_k = r_k); loss = the energy-norm error left by one optimally scaled
// preconditioned step, L = min_alpha |e - alpha z|_K^2 / |e|_K^2
// = 1 - (r.z)^2 / ((z.K z)(e.r)), with K the matrix-free tangent rescaled to
// each pair's modulus. It is invariant to the scale of z (additive multilevel
// preconditioners overshoot by design, which a residual-norm loss punishes)
// and needs one tangent product per pair. With w = G^T G v the weight
// gradient of g^T w is the gradient of <G g_c, G v> (g_c = S Q^T dL/dz): two
// forward passes of G and two backward passes, each with the other's output
// as its upstream gradient.
// Adam on FP32 master weights, cast to BF16 after every step. All reductions
// run in a fixed order (bit-reproducible).
#include <cuda_bf16.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "cells.cuh"
#include "pd_internal.cuh"

namespace pdb {

constexpr int H = 64;
constexpr int NL = 3;
constexpr int OFF_W0 = 0;       // W0 [H][3]
constexpr int OFF_L = 3 * H;    // per layer: Ws [H][H], Wn [H][H]
constexpr int LSZ = 2 * H * H;
constexpr int NPARAM = OFF_L + NL * LSZ;
// The BF16 copy holds the parameters in their own layout [0, NPARAM) and, from
// OFF_KM, every layer's [Ws | Wn] again k-major ([l][part*H + k][o]), the
// layout the forward layer multiplies in, so that its staging is a copy.
constexpr int OFF_KM = NPARAM;
constexpr int WB_SIZE = NPARAM + NL * LSZ;
static_assert((OFF_L * 2) % 16 == 0 && (OFF_KM * 2) % 16 == 0 && (LSZ * 2) % 16 == 0,
              "16-byte weight loads need 16-byte aligned layer offsets");
constexpr int kRed = 148;
constexpr int kTile = 16;       // patches per block tile of the layer kernels (half a warp each)

struct MpnnState {
  bool ready = false;    // weights initialised (trained or loaded)
  bool trained = false;
  bool patches = false;  // patch graph built
  double patch = 0.0;    // patch cell side
  double coarse_cell = 0.0;  // >= 0: the coarse level sits under the network (aggregate cell side)
  int64_t n = 0, np = 0;
  Grid g;
  DBuf<int32_t> sorted, pid, cell_patch, patch_cell, pcol;
  DBuf<int64_t> cstart, prow;
  DBuf<float> scale;     // s_I
  DBuf<float> w, g_, am, av, gpart;
  DBuf<__nv_bfloat16> wb;
  int64_t adam_t = 0;
  // activations: two sets (v and the gradient input), FP32; the fused apply's
  // transposed layers write (s_buf, t_buf), (d, t_alt), (s_alt, t_alt2)
  DBuf<float> v[2], h[2][NL + 1], m[2][NL], d, s_buf, t_buf, s_alt, t_alt, t_alt2, out3;
  // training set: per pair a, r, e (float, 3n each)
  DBuf<float> pairs;
  int64_t npairs = 0, cap = 0;
  std::vector<double> pair_k;  // bulk modulus at capture (the tangent scales with it)
  // capture from CG
  int every = 0;
  std::vector<DBuf<double>*> snap_r, snap_x;
  int nsnap = 0;
  // Inference apply: one cooperative launch of apply_grid blocks; bar holds
  // its grid barrier (arrivals, generation).
  DBuf<unsigned int> bar;
  int apply_grid = 0;
  ~MpnnState() {
    for (auto* p : snap_r) delete p;
    for (auto* p : snap_x) delete p;
  }
};

// ---------------------------------------------------------------------------
// Patch graph
// ---------------------------------------------------------------------------
__global__ void k_pt_cells(int64_t ncell, const int64_t* __restrict__ cstart, int32_t* __restrict__ cell_patch,
                           int32_t* __restrict__ patch_cell, int64_t* __restrict__ np_out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int32_t k = 0;
  for (int64_t q = 0; q < ncell; ++q) {
    if (cstart[q + 1] > cstart[q]) {
      cell_patch[q] = k;
      patch_cell[k] = (int32_t)q;
      ++k;
    } else {
      cell_patch[q] = -1;
    }
  }
  *np_out = k;
}

__global__ void k_pt_pid(int64_t n, const double4* __restrict__ xv, Grid g, const int32_t* __restrict__ cell_patch,
                         int32_t* __restrict__ pid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = xv[i];
  pid[i] = cell_patch[(cell_coord(g, p.z, 2) * g.dims[1] + cell_coord(g, p.y, 1)) * g.dims[0] + cell_coord(g, p.x, 0)];
}

// neighbors of patch I: the non-empty cells of its 3x3x3 neighborhood (itself excluded), in cell order
template <bool FILL>
__global__ void k_pt_adj(int64_t np, Grid g, const int32_t* __restrict__ patch_cell,
                         const int32_t* __restrict__ cell_patch, int64_t* __restrict__ cnt,
                         const int64_t* __restrict__ prow, int32_t* __restrict__ pcol) {
  const int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= np) return;
  const int q = patch_cell[I];
  const int cx = q % g.dims[0], cy = (q / g.dims[0]) % g.dims[1], cz = q / (g.dims[0] * g.dims[1]);
  int64_t k = FILL ? prow[I] : 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (!dx && !dy && !dz) continue;
        const int x = cx + dx, y = cy + dy, z = cz + dz;
        if (x < 0 || y < 0 || z < 0 || x >= g.dims[0] || y >= g.dims[1] || z >= g.dims[2]) continue;
        const int32_t J = cell_patch[(z * g.dims[1] + y) * g.dims[0] + x];
        if (J < 0) continue;
        if (FILL) pcol[k] = J;
        ++k;
      }
  if (!FILL) cnt[I] = k;
}

// s_I = sqrt(sum_{i in I} sum_{c free} (D_i^-1)_cc / 3) / |I|  (warp per patch;
// the identity rows of prescribed dofs are left out)
__global__ void k_pt_scale(int64_t np, const int32_t* __restrict__ patch_cell, const int64_t* __restrict__ cstart,
                           const int32_t* __restrict__ sorted, const double* __restrict__ dinv,
                           const uint8_t* __restrict__ fixed, float* __restrict__ scale) {
  const int64_t I = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (I >= np) return;
  const int q = patch_cell[I];
  double s = 0.0;
  for (int64_t t = cstart[q] + lane; t < cstart[q + 1]; t += 32) {
    const int64_t p = sorted[t];
    const double* d = dinv + 9 * p;
    const uint8_t f = fixed ? fixed[p] : 0;
    s += ((f & 1 ? 0.0 : d[0]) + (f & 2 ? 0.0 : d[4]) + (f & 4 ? 0.0 : d[8])) / 3.0;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const double cnt = (double)(cstart[q + 1] - cstart[q]);
  if (lane == 0) scale[I] = (float)(s > 0.0 ? sqrt(s) / cnt : 0.0);
}

// v_I = mul * s_I * sum_{i in I, free} r_i  (warp per patch; fixed order)
template <typename T>
__global__ void k_pt_restrict(int64_t np, const int32_t* __restrict__ patch_cell, const int64_t* __restrict__ cstart,
                              const int32_t* __restrict__ sorted, const T* __restrict__ r,
                              const uint8_t* __restrict__ fixed, const float* __restrict__ scale, double mul,
                              float* __restrict__ v) {
  const int64_t I = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (I >= np) return;
  const int q = patch_cell[I];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t t = cstart[q] + lane; t < cstart[q + 1]; t += 32) {
    const int64_t p = sorted[t];
    const uint8_t f = fixed ? fixed[p] : 0;
    if (!(f & 1)) s0 += (double)r[3 * p];
    if (!(f & 2)) s1 += (double)r[3 * p + 1];
    if (!(f & 4)) s2 += (double)r[3 * p + 2];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    const double sc = mul * (double)scale[I];
    v[3 * I] = (float)(sc * s0), v[3 * I + 1] = (float)(sc * s1), v[3 * I + 2] = (float)(sc * s2);
  }
}

// z_i += mul * s_I * out_I on the free dofs of point i (I = patch of i)
__global__ void k_pt_prolong(int64_t n, const int32_t* __restrict__ pid, const float* __restrict__ out,
                             const float* __restrict__ scale, double mul, const uint8_t* __restrict__ fixed,
                             double* __restrict__ z) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t I = pid[i];
  const uint8_t f = fixed ? fixed[i] : 0;
  const double sc = mul * (double)scale[I];
  for (int c = 0; c < 3; ++c)
    if (!((f >> c) & 1)) z[3 * i + c] += sc * (double)out[3 * I + c];
}

// ---------------------------------------------------------------------------
// Network G and its transpose
// ---------------------------------------------------------------------------
// h0[I][o] = sum_c W0[o][c] v[I][c]
__global__ void k_pt_encode(int64_t np, const float* __restrict__ v, const __nv_bfloat16* __restrict__ wb,
                            float* __restrict__ h0) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np * H) return;
  const int64_t I = k / H;
  const int o = (int)(k - I * H);
  float s = 0.f;
  for (int c = 0; c < 3; ++c) s = fmaf(__bfloat162float(wb[OFF_W0 + 3 * o + c]), v[3 * I + c], s);
  h0[k] = s;
}

// out[I][c] = sum_o W0[o][c] x[I][o]  (warp per patch)
__global__ void k_pt_encode_t(int64_t np, const float* __restrict__ x, const __nv_bfloat16* __restrict__ wb,
                              float* __restrict__ out) {
  const int64_t I = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (I >= np) return;
  const float x0 = x[(int64_t)H * I + 2 * lane], x1 = x[(int64_t)H * I + 2 * lane + 1];
  float s[3];
  for (int c = 0; c < 3; ++c) {
    s[c] = __bfloat162float(wb[OFF_W0 + 3 * (2 * lane) + c]) * x0 + __bfloat162float(wb[OFF_W0 + 3 * (2 * lane + 1) + c]) * x1;
    for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_xor_sync(0xffffffffu, s[c], o);
  }
  if (lane == 0) out[3 * I] = s[0], out[3 * I + 1] = s[1], out[3 * I + 2] = s[2];
}

// Sum over the patch's neighbor rows J (CSR b0..b1) of x_J's features
// 4hl..4hl+3 (half a warp per patch, 16 lanes x float4 = 64 features): eight
// rows in flight, added in groups of four in row order.
__device__ __forceinline__ float4 nbr_sum4(const float4* __restrict__ x4, const int32_t* __restrict__ pcol, int64_t b0,
                                           int64_t b1, int hl, float4 a) {
  auto add4 = [&](const float4& u0, const float4& u1, const float4& u2, const float4& u3) {
    a.x += (u0.x + u1.x) + (u2.x + u3.x);
    a.y += (u0.y + u1.y) + (u2.y + u3.y);
    a.z += (u0.z + u1.z) + (u2.z + u3.z);
    a.w += (u0.w + u1.w) + (u2.w + u3.w);
  };
  int64_t b = b0;
  for (; b + 8 <= b1; b += 8) {
    int32_t j[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) j[k] = pcol[b + k];
    float4 u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) u[k] = x4[(int64_t)(H / 4) * j[k] + hl];
    add4(u[0], u[1], u[2], u[3]);
    add4(u[4], u[5], u[6], u[7]);
  }
  if (b + 4 <= b1) {
    const int32_t j0 = pcol[b], j1 = pcol[b + 1], j2 = pcol[b + 2], j3 = pcol[b + 3];
    add4(x4[(int64_t)(H / 4) * j0 + hl], x4[(int64_t)(H / 4) * j1 + hl], x4[(int64_t)(H / 4) * j2 + hl],
         x4[(int64_t)(H / 4) * j3 + hl]);
    b += 4;
  }
  for (; b < b1; ++b) {
    const float4 u = x4[(int64_t)(H / 4) * pcol[b] + hl];
    a.x += u.x;
    a.y += u.y;
    a.z += u.z;
    a.w += u.w;
  }
  return a;
}

// Shared memory of one layer tile: the k-major weights [Ws | Wn] (rows padded
// to 144 B, 16-byte aligned) and the tile's [h | mean] rows.
struct LayerSmem {
  __nv_bfloat16 sW[2 * H][H + 8];
  float sX[kTile][2 * H + 4];
};
// ... of one transposed-layer tile: sW[o][k'] (k' < H: Ws[o][k'], else
// Wn[o][k'-H]) and the tile's input rows.
struct LayerTSmem {
  __nv_bfloat16 sW[H][2 * H];
  float sX[kTile][H + 4];
};

// Copy a layer's k-major [Ws | Wn] into shared memory (16-byte loads, 4 per
// thread, all in flight before the first store; 256 threads).
__device__ __forceinline__ void layer_stage_w(LayerSmem& S, const __nv_bfloat16* __restrict__ wk) {
  constexpr int kW16 = 2 * H * H / 8;  // 16-byte words of [Ws | Wn]
  static_assert(kW16 == 4 * 256, "launched with 256 threads");
  const uint4* w4 = reinterpret_cast<const uint4*>(wk);
  uint4 wr[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) wr[q] = __ldg(w4 + threadIdx.x + 256 * q);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int t8 = threadIdx.x + 256 * q;
    *reinterpret_cast<uint4*>(&S.sW[t8 / (H / 8)][(t8 % (H / 8)) * 8]) = wr[q];
  }
}

// One tile of 16 patches from i0 of a layer: hout = hin + Ws hin + Wn mean_J
// hin_J (mout, when given, receives the mean). Phase 1 gathers [h | mean]
// rows (half a warp per patch, 4 features per lane, eight neighbor rows in
// flight); phase 2 multiplies (4 outputs per thread, 8-byte weight reads,
// FP32 accumulation). Block-uniform; leaves shared memory free for reuse.
__device__ __forceinline__ void layer_tile(LayerSmem& S, int64_t i0, int64_t np, const int64_t* __restrict__ prow,
                                           const int32_t* __restrict__ pcol, const float* hin, float* hout,
                                           float* mout) {
  const int hl = threadIdx.x & 15, r = threadIdx.x >> 4;  // phase 1: patch r of the tile
  const int nl = threadIdx.x >> 4, ob = (threadIdx.x & 15) * 4;  // phase 2: patch nl, outputs ob..ob+3
  const float4* h4 = reinterpret_cast<const float4*>(hin);
  {
    const int64_t I = i0 + r;
    float4 hv = make_float4(0.f, 0.f, 0.f, 0.f), mv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (I < np) {
      hv = h4[(int64_t)(H / 4) * I + hl];
      const int64_t b0 = prow[I], b1 = prow[I + 1];
      mv = nbr_sum4(h4, pcol, b0, b1, hl, mv);
      const float inv = b1 > b0 ? 1.0f / (float)(b1 - b0) : 0.0f;
      mv.x *= inv;
      mv.y *= inv;
      mv.z *= inv;
      mv.w *= inv;
      if (mout) reinterpret_cast<float4*>(mout)[(int64_t)(H / 4) * I + hl] = mv;
    }
    *reinterpret_cast<float4*>(&S.sX[r][4 * hl]) = hv;
    *reinterpret_cast<float4*>(&S.sX[r][H + 4 * hl]) = mv;
  }
  __syncthreads();
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 8
  for (int k = 0; k < 2 * H; ++k) {
    const float x = S.sX[nl][k];
    const uint2 wv = *reinterpret_cast<const uint2*>(&S.sW[k][ob]);
    const __nv_bfloat162* w2 = reinterpret_cast<const __nv_bfloat162*>(&wv);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const float2 f = __bfloat1622float2(w2[j]);
      acc[2 * j] = fmaf(x, f.x, acc[2 * j]);
      acc[2 * j + 1] = fmaf(x, f.y, acc[2 * j + 1]);
    }
  }
  const int64_t I = i0 + nl;
  if (I < np)
    *reinterpret_cast<float4*>(hout + (int64_t)H * I + ob) = make_float4(
        S.sX[nl][ob] + acc[0], S.sX[nl][ob + 1] + acc[1], S.sX[nl][ob + 2] + acc[2], S.sX[nl][ob + 3] + acc[3]);
  __syncthreads();
}

// One layer over all patches in block tiles of 16 (256 threads).
__global__ void __launch_bounds__(256) k_pt_layer(int64_t np, const int64_t* __restrict__ prow,
                                                  const int32_t* __restrict__ pcol,
                                                  const __nv_bfloat16* __restrict__ wk, const float* __restrict__ hin,
                                                  float* __restrict__ hout, float* __restrict__ mout) {
  __shared__ __align__(16) LayerSmem S;
  layer_stage_w(S, wk);
  for (int64_t i0 = (int64_t)blockIdx.x * kTile; i0 < np; i0 += (int64_t)gridDim.x * kTile)
    layer_tile(S, i0, np, prow, pcol, hin, hout, mout);
}

// Copy a layer's [Ws | Wn] (their own layout) into shared memory as sW[o][k'].
__device__ __forceinline__ void layer_t_stage_w(LayerTSmem& S, const __nv_bfloat16* __restrict__ wl) {
  constexpr int kW16 = 2 * H * H / 8;  // 16-byte words of [Ws | Wn] in their own layout
  static_assert(kW16 == 4 * 256, "launched with 256 threads");
  const uint4* w4 = reinterpret_cast<const uint4*>(wl);
  uint4 wr[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) wr[q] = __ldg(w4 + threadIdx.x + 256 * q);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int t8 = threadIdx.x + 256 * q;  // part, row o, 8-column segment
    const int part = t8 / (H * H / 8), o = (t8 % (H * H / 8)) / (H / 8), seg = t8 % (H / 8);
    *reinterpret_cast<uint4*>(&S.sW[o][part * H + seg * 8]) = wr[q];
  }
}

// Transposed-layer input rows of the tile at i0: d_I (zero past np).
__device__ __forceinline__ void layer_t_load(LayerTSmem& S, int64_t i0, int64_t np, const float* d) {
  const float4* d4 = reinterpret_cast<const float4*>(d);
#pragma unroll
  for (int q = 0; q < kTile * H / 4 / 256; ++q) {
    const int t = threadIdx.x + 256 * q, r = t / (H / 4), o4 = t % (H / 4);
    const int64_t I = i0 + r;
    *reinterpret_cast<float4*>(&S.sX[r][4 * o4]) =
        I < np ? d4[(int64_t)(H / 4) * I + o4] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// Transposed layer on the tile's rows in shared memory: s = d + Ws^T d,
// t = Wn^T d / deg (the gather of t over the symmetric patch graph completes
// it). Block-uniform; leaves shared memory free for reuse.
__device__ __forceinline__ void layer_t_mul(LayerTSmem& S, int64_t i0, int64_t np, const int64_t* __restrict__ prow,
                                            float* s_out, float* t_out) {
  __syncthreads();
  const int nl = threadIdx.x >> 4, ob = (threadIdx.x & 15) * 8;  // patch nl, outputs ob..ob+7 of [s | t]
  float acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = 0.f;
#pragma unroll 4
  for (int o = 0; o < H; ++o) {
    const float x = S.sX[nl][o];
    const uint4 wv = *reinterpret_cast<const uint4*>(&S.sW[o][ob]);
    const __nv_bfloat162* w2 = reinterpret_cast<const __nv_bfloat162*>(&wv);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float2 f = __bfloat1622float2(w2[j]);
      acc[2 * j] = fmaf(x, f.x, acc[2 * j]);
      acc[2 * j + 1] = fmaf(x, f.y, acc[2 * j + 1]);
    }
  }
  const int64_t I = i0 + nl;
  if (I < np) {  // the 8 outputs lie in one part: s (ob < H) or t
    float4* o4;
    float v[8];
    if (ob < H) {
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = S.sX[nl][ob + j] + acc[j];
      o4 = reinterpret_cast<float4*>(s_out + (int64_t)H * I + ob);
    } else {
      const int64_t deg = prow[I + 1] - prow[I];
      const float inv = deg > 0 ? 1.0f / (float)deg : 0.0f;
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = acc[j] * inv;
      o4 = reinterpret_cast<float4*>(t_out + (int64_t)H * I + (ob - H));
    }
    o4[0] = make_float4(v[0], v[1], v[2], v[3]);
    o4[1] = make_float4(v[4], v[5], v[6], v[7]);
  }
  __syncthreads();
}

// Transposed layer, per patch, over all patches in block tiles of 16.
__global__ void __launch_bounds__(256) k_pt_layer_t(int64_t np, const int64_t* __restrict__ prow,
                                                    const __nv_bfloat16* __restrict__ wl, const float* __restrict__ d,
                                                    float* __restrict__ s_out, float* __restrict__ t_out) {
  __shared__ __align__(16) LayerTSmem S;
  layer_t_stage_w(S, wl);
  for (int64_t i0 = (int64_t)blockIdx.x * kTile; i0 < np; i0 += (int64_t)gridDim.x * kTile) {
    layer_t_load(S, i0, np, d);
    layer_t_mul(S, i0, np, prow, s_out, t_out);
  }
}

// x_J = s_J + sum_{I in N(J)} t_I  (half a warp per patch, 4 features per lane).
// No __launch_bounds__ here: with (256) ptxas held it to 32 registers and
// spilled; without it it takes 34, no spills.
__global__ void k_pt_gather_t(int64_t np, const int64_t* __restrict__ prow, const int32_t* __restrict__ pcol,
                              const float* __restrict__ s, const float* __restrict__ t, float* __restrict__ x) {
  const int64_t J = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
  const int hl = threadIdx.x & 15;
  if (J >= np) return;  // no shuffles below: each half warp may leave on its own
  float4 a = reinterpret_cast<const float4*>(s)[(int64_t)(H / 4) * J + hl];
  a = nbr_sum4(reinterpret_cast<const float4*>(t), pcol, prow[J], prow[J + 1], hl, a);
  reinterpret_cast<float4*>(x)[(int64_t)(H / 4) * J + hl] = a;
}

// ---------------------------------------------------------------------------
// Inference apply, one cooperative launch
// ---------------------------------------------------------------------------
// The apply's phases are chains of dependent loads (neighbor ids, then their
// rows; point ids, then their masks and residuals), so a block keeps its
// tile's ids in shared memory for the whole launch and every phase starts
// from them: no more tiles than blocks leaves each block one tile.
constexpr int kMaxDeg = 26;     // a patch's neighbors: the other non-empty cells of its 3x3x3 block
constexpr int kTilePts = 1024;  // point ids of a tile kept in shared memory (past that, read per use)

struct ApplyArgs {
  int64_t np;
  const int64_t* prow;
  const int32_t* pcol;
  const int32_t* patch_cell;
  const int64_t* cstart;
  const int32_t* sorted;
  const double* r;
  const uint8_t* fixed;
  const float* scale;
  const __nv_bfloat16* wb;
  float* h[NL + 1];  // encoder output and the layers' outputs
  float* s[NL];      // transposed layers' s and t, one pair per layer (each
  float* t[NL];      // written once per launch)
  double* z;
  unsigned int* bar;  // grid barrier: arrivals, generation
  int* status;
};

// A tile's patches: neighbor ids and counts, point ids and fixed masks.
struct __align__(16) TileMeta {
  int32_t nbr[kTile][kMaxDeg];
  int32_t deg[kTile];
  int32_t cnt[kTile];
  int32_t pbeg[kTile + 1];  // tile-local offsets into pts
  int32_t pts[kTilePts];
  uint8_t pfix[kTilePts];
};
// The tile's rows ([h | mean] of a layer, 2H, or the input of a transposed
// layer, H) and the phase's weights as B fragments: word [ks][n][t] holds
// B[16ks + 2t .. +1][n] and word [ks][n][4 + t] B[16ks + 2t + 8 .. +9][n]
// (K = 128, N = 64 for a layer; K = 64, N = 128 for a transposed one).
struct ApplySmem {
  float sX[kTile][2 * H + 4];
  uint32_t sB[2 * H * H / 2];
};
// Tiles whose ids a block keeps (a block of a grid smaller than the tile
// count takes two or more tiles; past kMetaSlots they are reloaded per use).
constexpr int kMetaSlots = 2;
constexpr size_t kApplySmem = kMetaSlots * sizeof(TileMeta) + sizeof(ApplySmem);

// Polls of the barrier's generation before a block gives up (0.2 to 1.5 s
// depending on how long the sleeps between polls last).
constexpr unsigned kBarSpin = 1u << 22;

// Grid-wide barrier of a cooperative launch (every block resident). Arrival
// is a release-acquire add on the count; the last block to arrive resets it
// and advances the generation with a release; the others poll the generation
// with acquire loads, at most kBarSpin times, after which the block sets
// ST_TIMEOUT and returns false (the kernel then ends; blocks still waiting
// for it run out the same way).
__device__ bool grid_barrier(unsigned int* bar, int* status) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int g, old;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(bar + 1) : "memory");
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(bar) : "memory");
    int good = 1;
    if (old == gridDim.x - 1) {
      asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(bar), "r"(0u) : "memory");
      asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar + 1) : "memory");
    } else {
      for (unsigned it = 0;; ++it) {
        unsigned int cur;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(bar + 1) : "memory");
        if (cur != g) break;
        if (it >= kBarSpin) {
          atomicOr(status, ST_TIMEOUT);
          good = 0;
          break;
        }
        __nanosleep(20);
      }
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// The tile's ids at i0 into shared memory (half a warp per patch).
__device__ void load_tile_meta(TileMeta& M, const ApplyArgs& a, int64_t i0) {
  const int r = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const int64_t I = i0 + r;
  int deg = 0, cnt = 0;
  int64_t b0 = 0, c0 = 0;
  if (I < a.np) {
    b0 = a.prow[I];
    deg = (int)(a.prow[I + 1] - b0);
    const int q = a.patch_cell[I];
    c0 = a.cstart[q];
    cnt = (int)(a.cstart[q + 1] - c0);
  }
  if (deg > kMaxDeg) {  // not from the patch graph's construction: keep shared memory in bounds
    if (hl == 0) atomicOr(a.status, ST_BAD_INDEX);
    deg = kMaxDeg;
  }
  for (int k = hl; k < deg; k += 16) M.nbr[r][k] = a.pcol[b0 + k];
  if (hl == 0) M.deg[r] = deg, M.cnt[r] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int o = 0;
    for (int k = 0; k < kTile; ++k) M.pbeg[k] = o, o += M.cnt[k];
    M.pbeg[kTile] = o;
  }
  __syncthreads();
  if (M.pbeg[kTile] <= kTilePts)
    for (int k = hl; k < cnt; k += 16) {
      const int32_t p = a.sorted[c0 + k];
      M.pts[M.pbeg[r] + k] = p;
      M.pfix[M.pbeg[r] + k] = a.fixed ? a.fixed[p] : 0;
    }
  __syncthreads();
}

// Sum of the rows x_J, J in idx[0..deg) (shared memory), features
// 4hl..4hl+3, eight rows in flight: groups of four in order, then the last
// deg mod 4 rows one by one (the order of nbr_sum4). Plain loads: every
// buffer the apply gathers from is written once per launch, before the
// barrier that precedes its reads.
__device__ __forceinline__ float4 nbr_sum_idx(const float4* x4, const int32_t* idx, int deg, int hl, float4 a) {
  auto add4 = [&](const float4& u0, const float4& u1, const float4& u2, const float4& u3) {
    a.x += (u0.x + u1.x) + (u2.x + u3.x);
    a.y += (u0.y + u1.y) + (u2.y + u3.y);
    a.z += (u0.z + u1.z) + (u2.z + u3.z);
    a.w += (u0.w + u1.w) + (u2.w + u3.w);
  };
  for (int b = 0; b < deg; b += 8) {
    const int m = min(8, deg - b);
    float4 u[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k < m) u[k] = x4[(int64_t)(H / 4) * idx[b + k] + hl];
    if (m >= 4) add4(u[0], u[1], u[2], u[3]);
    if (m == 8) {
      add4(u[4], u[5], u[6], u[7]);
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k >= (m & 4) && k < m) {  // the last batch's rows past its group
          a.x += u[k].x;
          a.y += u[k].y;
          a.z += u[k].z;
          a.w += u[k].w;
        }
    }
  }
  return a;
}

// D += A B on the tensor cores: m16n8k16, BF16 operands, FP32 accumulation.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// An FP32 pair as three BF16 pairs, x = hi + mid + lo: each residual is
// exact in FP32, so the three parts carry x's 24 bits and the BF16 products
// with the (BF16) weights are exact.
__device__ __forceinline__ void split3(float2 x, uint32_t& hi, uint32_t& mid, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x.x, x.y);
  const float2 hf = __bfloat1622float2(h);
  const float r0 = x.x - hf.x, r1 = x.y - hf.y;
  const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
  const float2 mf = __bfloat1622float2(m);
  hi = bf2_bits(h);
  mid = bf2_bits(m);
  lo = bf2_bits(__floats2bfloat162_rn(r0 - mf.x, r1 - mf.y));
}

// acc += X[16 x 16 at column k0] B for the warp's B fragment (b0, b1): the
// row-major A fragment of the tile's rows g, g+8 (sX, FP32) in three BF16
// parts, smallest first.
__device__ __forceinline__ void mma_rows(float (&acc)[4], const float (*sX)[2 * H + 4], int k0, uint32_t b0,
                                         uint32_t b1) {
  const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
  uint32_t hi[4], mid[4], lo[4];
  split3(*reinterpret_cast<const float2*>(&sX[g][k0 + 2 * t]), hi[0], mid[0], lo[0]);
  split3(*reinterpret_cast<const float2*>(&sX[g + 8][k0 + 2 * t]), hi[1], mid[1], lo[1]);
  split3(*reinterpret_cast<const float2*>(&sX[g][k0 + 2 * t + 8]), hi[2], mid[2], lo[2]);
  split3(*reinterpret_cast<const float2*>(&sX[g + 8][k0 + 2 * t + 8]), hi[3], mid[3], lo[3]);
  mma_bf16(acc, lo, b0, b1);
  mma_bf16(acc, mid, b0, b1);
  mma_bf16(acc, hi, b0, b1);
}

// A layer's B fragments into shared memory: B[k][n] = Ws[n][k] (k < H),
// Wn[n][k - H], from the weights' own layout (pairs of consecutive k are one
// 32-bit word: word (n, k/2) of part k / H).
__device__ __forceinline__ void stage_layer_b(uint32_t* sB, const __nv_bfloat16* __restrict__ wl) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(wl);
  for (int e = threadIdx.x; e < H * H; e += blockDim.x) {  // e = (ks, n, j): j < 8
    const int j = e & 7, n = (e >> 3) % H, ks = (e >> 3) / H;
    const int k = 16 * ks + 2 * (j & 3) + 8 * (j >> 2);
    sB[e] = __ldg(w + ((k / H) * H * H + n * H + k % H) / 2);
  }
}

// ... a transposed layer's: B[o][n'] = Ws[o][n'] (n' < H), Wn[o][n' - H],
// from the k-major copy ([part*H + k][o]: pairs of consecutive o are one word).
__device__ __forceinline__ void stage_layer_t_b(uint32_t* sB, const __nv_bfloat16* __restrict__ wk) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(wk);
  for (int e = threadIdx.x; e < H * H; e += blockDim.x) {  // e = (ks, n', j)
    const int j = e & 7, n = (e >> 3) % (2 * H), ks = (e >> 3) / (2 * H);
    const int o = 16 * ks + 2 * (j & 3) + 8 * (j >> 2);
    sB[e] = __ldg(w + (n * H + o) / 2);
  }
}

// Layer tile: h_out = h + Ws h + Wn mean_J h_J on the tile at i0 (the gather
// of layer_tile; the product on the tensor cores, FP32-exact operands in
// three BF16 parts and FP32 accumulation: warp w, outputs 8w..8w+7).
__device__ __forceinline__ void apply_layer_tile(ApplySmem& S, const TileMeta& M, int64_t i0, int64_t np,
                                                 const float* hin, float* hout) {
  const int hl = threadIdx.x & 15, r = threadIdx.x >> 4;
  const float4* h4 = reinterpret_cast<const float4*>(hin);
  {
    const int64_t I = i0 + r;
    float4 hv = make_float4(0.f, 0.f, 0.f, 0.f), mv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (I < np) {
      hv = h4[(int64_t)(H / 4) * I + hl];
      const int deg = M.deg[r];
      mv = nbr_sum_idx(h4, M.nbr[r], deg, hl, mv);
      const float inv = deg > 0 ? 1.0f / (float)deg : 0.0f;
      mv.x *= inv;
      mv.y *= inv;
      mv.z *= inv;
      mv.w *= inv;
    }
    *reinterpret_cast<float4*>(&S.sX[r][4 * hl]) = hv;
    *reinterpret_cast<float4*>(&S.sX[r][H + 4 * hl]) = mv;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
  for (int ks = 0; ks < 2 * H / 16; ++ks) {
    const uint32_t* bw = S.sB + ((ks * H) + 8 * w + g) * 8;
    mma_rows(acc, S.sX, 16 * ks, bw[t], bw[4 + t]);
  }
  const int n = 8 * w + 2 * t;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int row = g + 8 * h;
    const int64_t I = i0 + row;
    if (I < np)
      *reinterpret_cast<float2*>(hout + (int64_t)H * I + n) =
          make_float2(S.sX[row][n] + acc[2 * h], S.sX[row][n + 1] + acc[2 * h + 1]);
  }
  __syncthreads();
}

// Transposed-layer tile: rows of d (own rows) or the gathered s_J + sum t_I,
// then s = x + Ws^T x, t = Wn^T x / deg (warp w: outputs 16w..16w+15 of [s | t]).
__device__ __forceinline__ void apply_layer_t_tile(ApplySmem& S, const TileMeta& M, int64_t i0, int64_t np,
                                                   const float* d, const float* sin, const float* tin, float* s_out,
                                                   float* t_out) {
  const int hl = threadIdx.x & 15, r = threadIdx.x >> 4;
  {
    const int64_t J = i0 + r;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    if (J < np) {
      if (d) {
        x = reinterpret_cast<const float4*>(d)[(int64_t)(H / 4) * J + hl];
      } else {
        x = reinterpret_cast<const float4*>(sin)[(int64_t)(H / 4) * J + hl];
        x = nbr_sum_idx(reinterpret_cast<const float4*>(tin), M.nbr[r], M.deg[r], hl, x);
      }
    }
    *reinterpret_cast<float4*>(&S.sX[r][4 * hl]) = x;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
    for (int ks = 0; ks < H / 16; ++ks) {
      const uint32_t* bw = S.sB + ((ks * 2 * H) + 16 * w + 8 * j + g) * 8;
      mma_rows(acc, S.sX, 16 * ks, bw[t], bw[4 + t]);
    }
    const int n = 16 * w + 8 * j + 2 * t;  // the pair lies in one part: s (n < H) or t
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = g + 8 * h;
      const int64_t I = i0 + row;
      if (I >= np) continue;
      if (n < H) {
        *reinterpret_cast<float2*>(s_out + (int64_t)H * I + n) =
            make_float2(S.sX[row][n] + acc[2 * h], S.sX[row][n + 1] + acc[2 * h + 1]);
      } else {
        const int deg = M.deg[row];
        const float inv = deg > 0 ? 1.0f / (float)deg : 0.0f;
        *reinterpret_cast<float2*>(t_out + (int64_t)H * I + (n - H)) =
            make_float2(acc[2 * h] * inv, acc[2 * h + 1] * inv);
      }
    }
  }
  __syncthreads();
}

// z += Q S G^T G S Q^T r on the free dofs in phases separated by grid
// barriers: the head (restrict, W0), three layers, three transposed layers
// with the gathers between them, the tail (last gather, W0^T,
// prolongation). Per patch it computes what the one-pass kernels of the
// training path do (k_pt_restrict + k_pt_encode, k_pt_layer, k_pt_layer_t,
// k_pt_gather_t, k_pt_encode_t + k_pt_prolong): the same gathers in the same
// order, the point sums in FP64 over half a warp, the layer products on the
// tensor cores (mma.sync, FP32 accumulation, which rounds in its own order).
// Every phase walks the same tiles, so the last layer and the first
// transposed layer need no barrier between them.
__global__ void __launch_bounds__(256, 4) k_pt_apply(ApplyArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  TileMeta* slots = reinterpret_cast<TileMeta*>(smem);
  ApplySmem& S = *reinterpret_cast<ApplySmem*>(smem + kMetaSlots * sizeof(TileMeta));
  static_assert(sizeof(TileMeta) % 16 == 0, "16-byte aligned layer tiles");
  const int64_t np = a.np;
  const int hl = threadIdx.x & 15, r = threadIdx.x >> 4;
  const int64_t tile0 = (int64_t)blockIdx.x * kTile, tstride = (int64_t)gridDim.x * kTile;
  int64_t held[kMetaSlots];  // the tiles whose ids the slots hold
  for (int k = 0; k < kMetaSlots; ++k) held[k] = -1;
  const TileMeta* cur_meta = slots;
  auto meta = [&](int64_t i0) {  // the block's k-th tile goes to slot min(k, kMetaSlots - 1)
    const int64_t kt = (i0 - tile0) / tstride;
    const int k = kt < kMetaSlots - 1 ? (int)kt : kMetaSlots - 1;
    if (held[k] != i0) load_tile_meta(slots[k], a, i0), held[k] = i0;
    cur_meta = slots + k;
  };
  auto point = [&](int64_t I, int k) -> int32_t {  // point k of patch r of the tile at I - r
    return cur_meta->pbeg[kTile] <= kTilePts ? cur_meta->pts[cur_meta->pbeg[r] + k] : a.sorted[a.cstart[a.patch_cell[I]] + k];
  };
  auto pfixed = [&](int k, int32_t p) -> uint8_t {
    return cur_meta->pbeg[kTile] <= kTilePts ? cur_meta->pfix[cur_meta->pbeg[r] + k] : (a.fixed ? a.fixed[p] : (uint8_t)0);
  };

  // head: v_I = s_I sum_{i in I, free} r_i, h0_I = W0 v_I
  for (int64_t i0 = tile0; i0 < np; i0 += tstride) {
    meta(i0);
    const int64_t I = i0 + r;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    if (I < np) {
      const int cnt = cur_meta->cnt[r];
      for (int k = hl; k < cnt; k += 16) {
        const int32_t p = point(I, k);
        const uint8_t f = pfixed(k, p);
        if (!(f & 1)) s0 += a.r[3 * (int64_t)p];
        if (!(f & 2)) s1 += a.r[3 * (int64_t)p + 1];
        if (!(f & 4)) s2 += a.r[3 * (int64_t)p + 2];
      }
    }
    for (int o = 8; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o, 16);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o, 16);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o, 16);
    }
    // the half warp's first lane's sums (the butterfly leaves each lane its own rounding)
    s0 = __shfl_sync(0xffffffffu, s0, 0, 16);
    s1 = __shfl_sync(0xffffffffu, s1, 0, 16);
    s2 = __shfl_sync(0xffffffffu, s2, 0, 16);
    if (I < np) {
      const double sc = 1.0 * (double)a.scale[I];
      const float v[3] = {(float)(sc * s0), (float)(sc * s1), (float)(sc * s2)};
      float h[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int o = 4 * hl + j;
        float acc = 0.f;
        for (int c = 0; c < 3; ++c) acc = fmaf(__bfloat162float(a.wb[OFF_W0 + 3 * o + c]), v[c], acc);
        h[j] = acc;
      }
      reinterpret_cast<float4*>(a.h[0])[(int64_t)(H / 4) * I + hl] = make_float4(h[0], h[1], h[2], h[3]);
    }
  }
  if (!grid_barrier(a.bar, a.status)) return;

  // layers: h_{l+1} = h_l + Ws h_l + Wn mean_J h_l,J
  for (int l = 0; l < NL; ++l) {
    stage_layer_b(S.sB, a.wb + OFF_L + l * LSZ);  // read after the tile's first barrier
    for (int64_t i0 = tile0; i0 < np; i0 += tstride) {
      meta(i0);
      apply_layer_tile(S, *cur_meta, i0, np, a.h[l], a.h[l + 1]);
    }
    if (l + 1 < NL && !grid_barrier(a.bar, a.status)) return;
  }

  // transposed layers, last first: the first on the block's own rows of h_NL,
  // the others on the gathered output of the one before; layer l writes pair
  // NL-1-l
  for (int l = NL - 1; l >= 0; --l) {
    __syncthreads();  // the last tile's products have read the layer's fragments
    stage_layer_t_b(S.sB, a.wb + OFF_KM + l * LSZ);
    const int out = NL - 1 - l, in = out - 1;
    for (int64_t i0 = tile0; i0 < np; i0 += tstride) {
      meta(i0);
      apply_layer_t_tile(S, *cur_meta, i0, np, l == NL - 1 ? a.h[NL] : nullptr, in >= 0 ? a.s[in] : nullptr,
                         in >= 0 ? a.t[in] : nullptr, a.s[out], a.t[out]);
    }
    if (!grid_barrier(a.bar, a.status)) return;
  }

  // tail: x_J = s_J + sum_{I in N(J)} t_I, out_J = W0^T x_J, z_i += s_J out_J
  // on the free dofs of J's points (half a warp per patch; the shuffles see
  // both halves: the tile loop is block-uniform)
  const float* sl = a.s[NL - 1];
  const float* tl = a.t[NL - 1];
  for (int64_t i0 = tile0; i0 < np; i0 += tstride) {
    meta(i0);
    const int64_t J = i0 + r;
    const bool live = J < np;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    if (live) {
      x = reinterpret_cast<const float4*>(sl)[(int64_t)(H / 4) * J + hl];
      x = nbr_sum_idx(reinterpret_cast<const float4*>(tl), cur_meta->nbr[r], cur_meta->deg[r], hl, x);
    }
    auto w0t = [&](int c) {  // sum over the 64 features of W0[o][c] x_o
      const int o = 4 * hl;
      float v = __bfloat162float(a.wb[OFF_W0 + 3 * o + c]) * x.x;
      v = fmaf(__bfloat162float(a.wb[OFF_W0 + 3 * (o + 1) + c]), x.y, v);
      v = fmaf(__bfloat162float(a.wb[OFF_W0 + 3 * (o + 2) + c]), x.z, v);
      v = fmaf(__bfloat162float(a.wb[OFF_W0 + 3 * (o + 3) + c]), x.w, v);
      for (int k = 8; k > 0; k >>= 1) v += __shfl_xor_sync(0xffffffffu, v, k, 16);
      return (double)__shfl_sync(0xffffffffu, v, 0, 16);  // the half warp's first lane
    };
    const double out0 = w0t(0), out1 = w0t(1), out2 = w0t(2);
    if (live) {
      const double sc = 1.0 * (double)a.scale[J];
      const int cnt = cur_meta->cnt[r];
#pragma unroll 4
      for (int k = hl; k < cnt; k += 16) {
        const int32_t p = point(J, k);
        const uint8_t f = pfixed(k, p);
        if (!(f & 1)) a.z[3 * (int64_t)p] += sc * out0;
        if (!(f & 2)) a.z[3 * (int64_t)p + 1] += sc * out1;
        if (!(f & 4)) a.z[3 * (int64_t)p + 2] += sc * out2;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Training kernels
// ---------------------------------------------------------------------------
// Weight-gradient partials: part[b][o*K+k] = sum_{i in block b's range} A[i][o] B[i][k]
__global__ void __launch_bounds__(256) k_pt_wgrad(int64_t n, int K, const float* __restrict__ A,
                                                  const float* __restrict__ B, float* __restrict__ part) {
  __shared__ float sa[H], sbv[H];
  const int entries = H * K;
  float acc[16];
  for (int q = 0; q < 16; ++q) acc[q] = 0.f;
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(n, i0 + per);
  for (int64_t i = i0; i < i1; ++i) {
    if (threadIdx.x < H) sa[threadIdx.x] = A[(int64_t)H * i + threadIdx.x];
    if (threadIdx.x < K) sbv[threadIdx.x] = B[(int64_t)K * i + threadIdx.x];
    __syncthreads();
    int q = 0;
    for (int e = threadIdx.x; e < entries; e += blockDim.x, ++q) acc[q] = fmaf(sa[e / K], sbv[e % K], acc[q]);
    __syncthreads();
  }
  int q = 0;
  for (int e = threadIdx.x; e < entries; e += blockDim.x, ++q) part[(int64_t)blockIdx.x * entries + e] = acc[q];
}

// g[dst + e] += sum_b part[b][e]  (fixed order)
__global__ void k_pt_wgrad_reduce(int nblk, int entries, const float* __restrict__ part, float* __restrict__ g,
                                  int dst) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < entries; e += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * entries + e];
    g[dst + e] += s;
  }
}

// BF16 weight k into both places it lives (its own layout; for a layer weight
// also the k-major copy at OFF_KM).
__device__ __forceinline__ void put_wb(int k, float x, __nv_bfloat16* __restrict__ wb) {
  const __nv_bfloat16 b = __float2bfloat16(x);
  wb[k] = b;
  if (k >= OFF_L) {
    const int r = k - OFF_L, l = r / LSZ, q = r % LSZ;
    const int part = q / (H * H), o = (q % (H * H)) / H, kk = q % H;
    wb[OFF_KM + l * LSZ + (part * H + kk) * H + o] = b;
  }
}

__global__ void k_mp_adam(int np, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, float lr, float b1, float b2, float c1, float c2, float scale,
                          __nv_bfloat16* __restrict__ wb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const float gk = g[k] * scale;
  m[k] = b1 * m[k] + (1.f - b1) * gk;
  v[k] = b2 * v[k] + (1.f - b2) * gk * gk;
  w[k] -= lr * (m[k] / c1) / (sqrtf(v[k] / c2) + 1e-8f);
  put_wb(k, w[k], wb);
}

__global__ void k_mp_cast(int np, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < np) put_wb(k, w[k], wb);
}

// z = a (FP64 from float), prescribed dofs zero
__global__ void k_mp_base(int64_t m, const float* __restrict__ a, const uint8_t* __restrict__ fixed,
                          double* __restrict__ z) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const bool fx = fixed && ((fixed[k / 3] >> (k % 3)) & 1);
  z[k] = fx ? 0.0 : (double)a[k];
}

// partials of r.z, z.Kz, e.r over the free dofs (3 per block, fixed order)
__global__ void k_mp_dots3(int64_t m, const float* __restrict__ r, const double* __restrict__ z,
                           const double* __restrict__ kz, const float* __restrict__ e,
                           const uint8_t* __restrict__ fixed, double* __restrict__ partial) {
  __shared__ double s0[256], s1[256], s2[256];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
    if (fixed && ((fixed[k / 3] >> (k % 3)) & 1)) continue;
    const double rk = (double)r[k], zk = z[k];
    a0 += rk * zk;
    a1 += zk * kz[k];
    a2 += (double)e[k] * rk;
  }
  s0[threadIdx.x] = a0;
  s1[threadIdx.x] = a1;
  s2[threadIdx.x] = a2;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      s0[threadIdx.x] += s0[threadIdx.x + o], s1[threadIdx.x] += s1[threadIdx.x + o],
          s2[threadIdx.x] += s2[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    partial[3 * blockIdx.x] = s0[0], partial[3 * blockIdx.x + 1] = s1[0], partial[3 * blockIdx.x + 2] = s2[0];
}

// gz = ca * r + cb * kz (prescribed dofs zero)
__global__ void k_mp_gz(int64_t m, double ca, const float* __restrict__ r, double cb, const double* __restrict__ kz,
                        const uint8_t* __restrict__ fixed, double* __restrict__ gz) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const bool fx = fixed && ((fixed[k / 3] >> (k % 3)) & 1);
  gz[k] = fx ? 0.0 : ca * (double)r[k] + cb * kz[k];
}

// random probe e: uniform in [-1, 1) on the free dofs from a counter hash
__global__ void k_mp_rand_e(int64_t m, uint64_t seed, const uint8_t* __restrict__ fixed, double* __restrict__ e,
                            double* __restrict__ zero) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  uint64_t x = seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(k + 1));
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 31;
  const bool fx = fixed && ((fixed[k / 3] >> (k % 3)) & 1);
  e[k] = fx ? 0.0 : (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  zero[k] = 0.0;
}

// pair capture: a = P_bj r, r, e = x* - x_k, as float
__global__ void k_mp_make_pair(int64_t n, const double* __restrict__ dinv, const double* __restrict__ r,
                               const double* __restrict__ xs, const double* __restrict__ xk, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* d = dinv + 9 * i;
  const double r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
  float* A = out;
  float* R = out + 3 * n;
  float* E = out + 6 * n;
  A[3 * i] = (float)(d[0] * r0 + d[1] * r1 + d[2] * r2);
  A[3 * i + 1] = (float)(d[3] * r0 + d[4] * r1 + d[5] * r2);
  A[3 * i + 2] = (float)(d[6] * r0 + d[7] * r1 + d[8] * r2);
  for (int c = 0; c < 3; ++c) {
    R[3 * i + c] = (float)r[3 * i + c];
    E[3 * i + c] = (float)(xs[3 * i + c] - xk[3 * i + c]);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static unsigned gw(int64_t n) { return (unsigned)((n * 32 + 255) / 256); }
static unsigned g1(int64_t n) { return (unsigned)((n + 255) / 256); }
static unsigned gh(int64_t n) { return (unsigned)((n * 16 + 255) / 256); }  // half a warp per patch
static unsigned gtile(int64_t np) { return (unsigned)std::min<int64_t>((np + kTile - 1) / kTile, 148 * 8); }

static MpnnState* mp_state(pd_ctx* c) { return reinterpret_cast<MpnnState*>(c->mpnn); }

// Bulk modulus of block 0 (or the median of a per-point field): the tangent of
// a body with a fixed K/mu ratio scales with it.
static double current_modulus(const pd_ctx* c) {
  if (!c->field_K.empty()) {
    std::vector<double> v(c->field_K);
    std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
    return v[v.size() / 2];
  }
  return c->block_K.empty() ? 1.0 : c->block_K[0];
}

// Patches: the non-empty cells of a grid of side `side` over the model coordinates.
static int mp_patches(pd_ctx* c, MpnnState* s, double side) {
  const int64_t n = c->n;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], c->hx[3 * i + k]), hi[k] = std::max(hi[k], c->hx[3 * i + k]);
  Grid g;
  double tot = 1.0;
  for (int k = 0; k < 3; ++k) {
    g.lo[k] = lo[k];
    g.dims[k] = (int)std::floor((hi[k] - lo[k]) / side) + 1;
    tot *= g.dims[k];
  }
  if (tot > 2.0e9) {
    c->err = "pd_mpnn_init: the patch side is too small for the body";
    return PD_ERR_ARG;
  }
  g.cell = side;
  const int64_t ncell = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
  TRY_RC(bin_points(c, c->xv.p, n, g, s->sorted, s->cstart));
  DBuf<int64_t> npd, cnt;
  PD_CUDA_TRY(c, npd.alloc(1));
  PD_CUDA_TRY(c, s->cell_patch.alloc(ncell));
  PD_CUDA_TRY(c, s->patch_cell.alloc(std::min<int64_t>(ncell, n)));
  k_pt_cells<<<1, 32, 0, c->stream>>>(ncell, s->cstart.p, s->cell_patch.p, s->patch_cell.p, npd.p);
  int64_t np = 0;
  PD_CUDA_TRY(c, d2h(c, &np, npd.p, sizeof(int64_t)));
  PD_CUDA_TRY(c, s->pid.alloc(n));
  k_pt_pid<<<g1(n), 256, 0, c->stream>>>(n, c->xv.p, g, s->cell_patch.p, s->pid.p);
  PD_CUDA_TRY(c, cnt.alloc(np + 1));
  PD_CUDA_TRY(c, s->prow.alloc(np + 1));
  k_pt_adj<false><<<g1(np), 256, 0, c->stream>>>(np, g, s->patch_cell.p, s->cell_patch.p, cnt.p, nullptr, nullptr);
  PD_CUDA_TRY(c, cudaMemsetAsync(cnt.p + np, 0, sizeof(int64_t), c->stream));
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, cnt.p, s->prow.p, (int)(np + 1), c->stream);
  DBuf<unsigned char> stmp;
  PD_CUDA_TRY(c, stmp.alloc(scan_bytes));
  PD_CUDA_TRY(c, cub::DeviceScan::ExclusiveSum(stmp.p, scan_bytes, cnt.p, s->prow.p, (int)(np + 1), c->stream));
  int64_t ne = 0;
  PD_CUDA_TRY(c, d2h(c, &ne, s->prow.p + np, sizeof(int64_t)));
  PD_CUDA_TRY(c, s->pcol.alloc(std::max<int64_t>(ne, 1)));
  k_pt_adj<true><<<g1(np), 256, 0, c->stream>>>(np, g, s->patch_cell.p, s->cell_patch.p, nullptr, s->prow.p,
                                                s->pcol.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  PD_CUDA_TRY(c, s->scale.alloc(np));
  PD_CUDA_TRY(c, dzero(c, s->scale.p, np * sizeof(float)));
  for (int k = 0; k < 2; ++k) {
    PD_CUDA_TRY(c, s->v[k].alloc(3 * np));
    for (int l = 0; l <= NL; ++l) PD_CUDA_TRY(c, s->h[k][l].alloc((size_t)H * np));
    for (int l = 0; l < NL; ++l) PD_CUDA_TRY(c, s->m[k][l].alloc((size_t)H * np));
  }
  PD_CUDA_TRY(c, s->d.alloc((size_t)H * np));
  PD_CUDA_TRY(c, s->s_buf.alloc((size_t)H * np));
  PD_CUDA_TRY(c, s->t_buf.alloc((size_t)H * np));
  PD_CUDA_TRY(c, s->s_alt.alloc((size_t)H * np));
  PD_CUDA_TRY(c, s->t_alt.alloc((size_t)H * np));
  PD_CUDA_TRY(c, s->t_alt2.alloc((size_t)H * np));
  PD_CUDA_TRY(c, s->out3.alloc(3 * np));
  s->g = g;
  s->np = np;
  s->n = n;
  s->patch = side;
  s->patches = true;
  s->apply_grid = 0;  // the fused apply's grid follows the patch count
  return PD_OK;
}

int mpnn_init(pd_ctx* c, uint64_t seed, double patch) {
  if (!c->mpnn) c->mpnn = new MpnnState();
  MpnnState* s = mp_state(c);
  TRY_RC(mp_patches(c, s, patch));
  // weights: W0 = 0.5 [I3; 0] and near-zero layers plus small uniform noise
  // from the seed, so G^T G starts near 0.25 I (a Jacobi-scaled middle level)
  std::vector<float> w(NPARAM, 0.f);
  std::mt19937_64 rng(seed);
  auto uni = [&](float lim) { return (float)((rng() >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0) * lim; };
  for (int k = 0; k < 3 * H; ++k) w[OFF_W0 + k] = uni(0.01f) + ((k % 4 == 0 && k < 12) ? 0.5f : 0.0f);
  for (int l = 0; l < NL; ++l)
    for (int k = 0; k < LSZ; ++k) w[OFF_L + l * LSZ + k] = uni(0.01f);
  PD_CUDA_TRY(c, s->w.alloc(NPARAM));
  PD_CUDA_TRY(c, s->wb.alloc(WB_SIZE));
  PD_CUDA_TRY(c, s->g_.alloc(NPARAM));
  PD_CUDA_TRY(c, s->am.alloc(NPARAM));
  PD_CUDA_TRY(c, s->av.alloc(NPARAM));
  PD_CUDA_TRY(c, s->gpart.alloc((size_t)kRed * H * H + 16));
  PD_CUDA_TRY(c, h2d(c, s->w.p, w.data(), NPARAM * sizeof(float)));
  PD_CUDA_TRY(c, dzero(c, s->am.p, NPARAM * sizeof(float)));
  PD_CUDA_TRY(c, dzero(c, s->av.p, NPARAM * sizeof(float)));
  k_mp_cast<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(NPARAM, s->w.p, s->wb.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  s->adam_t = 0;
  s->ready = true;
  s->trained = false;
  return PD_OK;
}

bool mpnn_ready(const pd_ctx* c) { return c->mpnn && reinterpret_cast<const MpnnState*>(c->mpnn)->ready; }

void mpnn_release(pd_ctx* c) {
  delete mp_state(c);
  c->mpnn = nullptr;
}

// Patch scales from the block-Jacobi inverse blocks of the current tangent.
int mpnn_prepare(pd_ctx* c, const double* dinv) {
  MpnnState* s = mp_state(c);
  if (!s || !s->patches || s->n != c->n) {
    c->err = "learned preconditioner not initialised for these points";
    return PD_ERR_STATE;
  }
  k_pt_scale<<<gw(s->np), 256, 0, c->stream>>>(s->np, s->patch_cell.p, s->cstart.p, s->sorted.p, dinv,
                                               qs_fixed_mask(c), s->scale.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// h[k][0..NL] = G v[k] (means saved when `save`)
static int mp_forward(pd_ctx* c, MpnnState* s, int k, bool save) {
  const int64_t np = s->np;
  k_pt_encode<<<g1(np * H), 256, 0, c->stream>>>(np, s->v[k].p, s->wb.p, s->h[k][0].p);
  for (int l = 0; l < NL; ++l)
    k_pt_layer<<<gtile(np), 256, 0, c->stream>>>(np, s->prow.p, s->pcol.p, s->wb.p + OFF_KM + l * LSZ, s->h[k][l].p,
                                                 s->h[k][l + 1].p, save ? s->m[k][l].p : nullptr);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// out3 = G^T y (y: 64 channels per patch, not modified)
static int mp_transpose(pd_ctx* c, MpnnState* s, const float* y) {
  const int64_t np = s->np;
  const float* cur = y;
  for (int l = NL - 1; l >= 0; --l) {
    k_pt_layer_t<<<gtile(np), 256, 0, c->stream>>>(np, s->prow.p, s->wb.p + OFF_L + l * LSZ, cur, s->s_buf.p,
                                                   s->t_buf.p);
    k_pt_gather_t<<<gh(np), 256, 0, c->stream>>>(np, s->prow.p, s->pcol.p, s->s_buf.p, s->t_buf.p, s->d.p);
    cur = s->d.p;
  }
  k_pt_encode_t<<<gw(np), 256, 0, c->stream>>>(np, cur, s->wb.p, s->out3.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

static void mp_wgrad(pd_ctx* c, MpnnState* s, int K, const float* A, const float* B, int dst) {
  k_pt_wgrad<<<kRed, 256, 0, c->stream>>>(s->np, K, A, B, s->gpart.p);
  k_pt_wgrad_reduce<<<(H * K + 255) / 256, 256, 0, c->stream>>>(kRed, H * K, s->gpart.p, s->g_.p, dst);
}

// Weight gradients of <U, G v[k]> (activations of set k saved), added into g_.
static int mp_backward(pd_ctx* c, MpnnState* s, int k, const float* U) {
  const int64_t np = s->np;
  const float* cur = U;
  for (int l = NL - 1; l >= 0; --l) {
    mp_wgrad(c, s, H, cur, s->h[k][l].p, OFF_L + l * LSZ);
    mp_wgrad(c, s, H, cur, s->m[k][l].p, OFF_L + l * LSZ + H * H);
    k_pt_layer_t<<<gtile(np), 256, 0, c->stream>>>(np, s->prow.p, s->wb.p + OFF_L + l * LSZ, cur, s->s_buf.p,
                                                   s->t_buf.p);
    k_pt_gather_t<<<gh(np), 256, 0, c->stream>>>(np, s->prow.p, s->pcol.p, s->s_buf.p, s->t_buf.p, s->d.p);
    cur = s->d.p;
  }
  mp_wgrad(c, s, 3, cur, s->v[k].p, OFF_W0);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// z += Q S G^T G S Q^T r on the free dofs (inference): one cooperative
// launch of k_pt_apply (every block resident, so its grid barriers are met).
int mpnn_apply_add(pd_ctx* c, const double* r, double* z) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready || !s->patches || s->n != c->n) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  if (!s->bar.p) {
    PD_CUDA_TRY(c, s->bar.alloc(2));
    PD_CUDA_TRY(c, dzero(c, s->bar.p, 2 * sizeof(unsigned int)));
  }
  if (s->apply_grid == 0) {
    int per_sm = 0, sms = 0;
    PD_CUDA_TRY(c, cudaFuncSetAttribute(k_pt_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kApplySmem));
    PD_CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pt_apply, 256, kApplySmem));
    PD_CUDA_TRY(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    if (per_sm < 1) {
      c->err = "learned preconditioner: the fused apply kernel cannot be resident";
      return PD_ERR_CUDA;
    }
    const int64_t tiles = std::max<int64_t>(1, (s->np + kTile - 1) / kTile);
    s->apply_grid = (int)std::min<int64_t>(tiles, (int64_t)per_sm * sms);
  }
  ApplyArgs a{};
  a.np = s->np;
  a.prow = s->prow.p;
  a.pcol = s->pcol.p;
  a.patch_cell = s->patch_cell.p;
  a.cstart = s->cstart.p;
  a.sorted = s->sorted.p;
  a.r = r;
  a.fixed = qs_fixed_mask(c);
  a.scale = s->scale.p;
  a.wb = s->wb.p;
  for (int l = 0; l <= NL; ++l) a.h[l] = s->h[0][l].p;
  a.s[0] = s->s_buf.p;
  a.t[0] = s->t_buf.p;
  a.s[1] = s->d.p;
  a.t[1] = s->t_alt.p;
  a.s[2] = s->s_alt.p;
  a.t[2] = s->t_alt2.p;
  static_assert(NL == 3, "one (s, t) pair per transposed layer");
  a.z = z;
  a.bar = s->bar.p;
  a.status = c->status.p;
  void* args[] = {&a};
  PD_CUDA_TRY(c, cudaLaunchCooperativeKernel((const void*)k_pt_apply, dim3((unsigned)s->apply_grid), dim3(256), args,
                                             kApplySmem, c->stream));
  return PD_OK;
}

// After a stream synchronisation: PD_ERR_TIMEOUT when a barrier wait of the
// fused apply ran out (the status bit is cleared and the barrier reset).
int mpnn_check_status(pd_ctx* c) {
  int st = 0;
  PD_CUDA_TRY(c, d2h(c, &st, c->status.p, sizeof(int)));
  if (!(st & ST_TIMEOUT)) return PD_OK;
  const int rest = st & ~(int)ST_TIMEOUT;
  PD_CUDA_TRY(c, h2d(c, c->status.p, &rest, sizeof(int)));
  MpnnState* s = mp_state(c);
  if (s && s->bar.p) PD_CUDA_TRY(c, dzero(c, s->bar.p, 2 * sizeof(unsigned int)));
  c->err = "learned preconditioner: a grid barrier wait of the fused apply ran out";
  return PD_ERR_TIMEOUT;
}

// One pair (a = P_bj r, r, e as float [3n] each, captured at modulus kscale x
// the current one): z = a + [coarse] + Q S G^T G S Q^T r (coarse and middle
// terms at the pair's modulus, 1/kscale); L = 1 - (r.z)^2 / ((z.Kp z)(e.r)),
// Kp = kscale K with K the tangent prepared by qs_prepare_current; the weight
// gradient is added into g_.
static int mp_pair_grad(pd_ctx* c, MpnnState* s, const float* pair, double kscale, double* loss) {
  const int64_t n = c->n, m = 3 * n, np = s->np;
  const float* A = pair;
  const float* R = pair + 3 * n;
  const float* E = pair + 6 * n;
  const uint8_t* fixed = qs_fixed_mask(c);
  DBuf<double> part, z, kz;
  PD_CUDA_TRY(c, part.alloc(3 * kRed));
  PD_CUDA_TRY(c, z.alloc(m));
  PD_CUDA_TRY(c, kz.alloc(m));
  k_mp_base<<<g1(m), 256, 0, c->stream>>>(m, A, fixed, z.p);
  if (s->coarse_cell >= 0.0) TRY_RC(coarse_apply_add_f(c, R, z.p, fixed, 1.0 / kscale));
  k_pt_restrict<float><<<gw(np), 256, 0, c->stream>>>(np, s->patch_cell.p, s->cstart.p, s->sorted.p, R, fixed,
                                                      s->scale.p, 1.0, s->v[0].p);
  TRY_RC(mp_forward(c, s, 0, true));
  TRY_RC(mp_transpose(c, s, s->h[0][NL].p));
  k_pt_prolong<<<g1(n), 256, 0, c->stream>>>(n, s->pid.p, s->out3.p, s->scale.p, 1.0 / kscale, fixed, z.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  TRY_RC(qs_apply_K(c, z.p, kz.p));
  k_mp_dots3<<<kRed, 256, 0, c->stream>>>(m, R, z.p, kz.p, E, fixed, part.p);
  std::vector<double> hp(3 * kRed);
  PD_CUDA_TRY(c, d2h(c, hp.data(), part.p, hp.size() * sizeof(double)));
  double a = 0.0, b = 0.0, e = 0.0;
  for (int k = 0; k < kRed; ++k) a += hp[3 * k], b += hp[3 * k + 1], e += hp[3 * k + 2];
  b *= kscale;
  if (!(b > 0.0) || !(e > 0.0)) {
    *loss = 1.0;  // z (or the pair) carries no energy: nothing to learn from it
    return PD_OK;
  }
  // dL/dz = -2a/(b e) r + 2a^2/(b^2 e) kscale K z (into z); dL/dw = (1/kscale) S Q^T dL/dz
  k_mp_gz<<<g1(m), 256, 0, c->stream>>>(m, -2.0 * a / (b * e), R, 2.0 * a * a * kscale / (b * b * e), kz.p, fixed,
                                        z.p);
  k_pt_restrict<double><<<gw(np), 256, 0, c->stream>>>(np, s->patch_cell.p, s->cstart.p, s->sorted.p, z.p, fixed,
                                                       s->scale.p, 1.0 / kscale, s->v[1].p);
  TRY_RC(mp_forward(c, s, 1, true));
  TRY_RC(mp_backward(c, s, 0, s->h[1][NL].p));
  TRY_RC(mp_backward(c, s, 1, s->h[0][NL].p));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *loss = 1.0 - a * a / (b * e);
  return PD_OK;
}

// Tangent, block Jacobi, patch scales and (when on) the coarse operator at
// the context's current displacement.
static int mp_prepare_training(pd_ctx* c, MpnnState* s) {
  TRY_RC(qs_prepare_current(c));
  const double* dinv = nullptr;
  TRY_RC(qs_block_jacobi_current(c, &dinv));
  TRY_RC(mpnn_prepare(c, dinv));
  if (s->coarse_cell >= 0.0) TRY_RC(qs_build_coarse_current(c, s->coarse_cell));
  return PD_OK;
}

int mpnn_loss_grad(pd_ctx* c, const float* pair_host, double* loss, float* grad_host) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  TRY_RC(mp_prepare_training(c, s));
  DBuf<float> pair;
  PD_CUDA_TRY(c, pair.alloc(9 * c->n));
  PD_CUDA_TRY(c, h2d(c, pair.p, pair_host, 9 * c->n * sizeof(float)));
  PD_CUDA_TRY(c, cudaMemsetAsync(s->g_.p, 0, NPARAM * sizeof(float), c->stream));
  TRY_RC(mp_pair_grad(c, s, pair.p, 1.0, loss));
  if (grad_host) PD_CUDA_TRY(c, d2h(c, grad_host, s->g_.p, NPARAM * sizeof(float)));
  return PD_OK;
}

// z = Q S G^T G S Q^T r (the middle level alone, host arrays [3n]) with the
// scales of the current displacement's block-Jacobi blocks, through the same
// fused apply the CG iterations use.
int mpnn_middle_apply(pd_ctx* c, const double* r_host, double* z_host) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready || !s->patches || s->n != c->n) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  TRY_RC(qs_prepare_current(c));
  const double* dinv = nullptr;
  TRY_RC(qs_block_jacobi_current(c, &dinv));
  TRY_RC(mpnn_prepare(c, dinv));
  const size_t b3 = 3 * (size_t)c->n * sizeof(double);
  DBuf<double> r, z;
  PD_CUDA_TRY(c, r.alloc(3 * c->n));
  PD_CUDA_TRY(c, z.alloc(3 * c->n));
  PD_CUDA_TRY(c, h2d(c, r.p, r_host, b3));
  PD_CUDA_TRY(c, dzero(c, z.p, b3));
  TRY_RC(mpnn_apply_add(c, r.p, z.p));
  PD_CUDA_TRY(c, d2h(c, z_host, z.p, b3));
  return mpnn_check_status(c);
}

int mpnn_train(pd_ctx* c, int epochs, double lr, int batch, double* loss_out) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  if (s->npairs == 0) {
    c->err = "no training pairs collected";
    return PD_ERR_STATE;
  }
  TRY_RC(mp_prepare_training(c, s));
  const int64_t n = c->n;
  const double k_now = current_modulus(c);
  std::mt19937_64 rng(12345 + s->adam_t);
  // Random probes (e uniform on the free dofs, r = K e) join every batch, one
  // per four captured pairs: CG iterates' errors are smooth, and without the
  // rough modes the network could amplify them unseen.
  const double* dinv = nullptr;
  TRY_RC(qs_block_jacobi_current(c, &dinv));
  DBuf<double> pe, pz, pr;
  DBuf<float> ppair;
  PD_CUDA_TRY(c, pe.alloc(3 * n));
  PD_CUDA_TRY(c, pz.alloc(3 * n));
  PD_CUDA_TRY(c, pr.alloc(3 * n));
  PD_CUDA_TRY(c, ppair.alloc(9 * n));
  const int nprobe = std::max(1, batch / 4);
  uint64_t probe_seed = 0x5DEECE66Dull + 7919ull * (uint64_t)s->adam_t;
  std::vector<int64_t> order(s->npairs);
  double last = 0.0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int64_t k = 0; k < s->npairs; ++k) order[k] = k;
    std::shuffle(order.begin(), order.end(), rng);
    double acc = 0.0;
    int64_t cnt = 0;
    for (int64_t b0 = 0; b0 < s->npairs; b0 += batch) {
      PD_CUDA_TRY(c, cudaMemsetAsync(s->g_.p, 0, NPARAM * sizeof(float), c->stream));
      const int64_t b1 = std::min<int64_t>(s->npairs, b0 + batch);
      for (int64_t q = b0; q < b1; ++q) {
        double l = 0.0;
        TRY_RC(mp_pair_grad(c, s, s->pairs.p + (size_t)order[q] * 9 * n, s->pair_k[order[q]] / k_now, &l));
        acc += l;
        ++cnt;
      }
      for (int q = 0; q < nprobe; ++q) {
        k_mp_rand_e<<<g1(3 * n), 256, 0, c->stream>>>(3 * n, probe_seed++, qs_fixed_mask(c), pe.p, pz.p);
        TRY_RC(qs_apply_K(c, pe.p, pr.p));
        k_mp_make_pair<<<g1(n), 256, 0, c->stream>>>(n, dinv, pr.p, pe.p, pz.p, ppair.p);
        double l = 0.0;
        TRY_RC(mp_pair_grad(c, s, ppair.p, 1.0, &l));
      }
      s->adam_t += 1;
      const float b1c = 0.9f, b2c = 0.999f;
      const float c1 = 1.f - std::pow(b1c, (float)s->adam_t), c2 = 1.f - std::pow(b2c, (float)s->adam_t);
      k_mp_adam<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(NPARAM, s->w.p, s->g_.p, s->am.p, s->av.p, (float)lr, b1c,
                                                             b2c, c1, c2, 1.0f / (float)(b1 - b0 + nprobe), s->wb.p);
      PD_CUDA_TRY(c, cudaGetLastError());
    }
    last = cnt ? acc / cnt : 0.0;
  }
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  s->trained = true;
  if (loss_out) *loss_out = last;
  return PD_OK;
}

// ---- pair capture from the block-Jacobi / two-level CG ----------------------
int mpnn_set_capture(pd_ctx* c, int every) {
  if (!c->mpnn) c->mpnn = new MpnnState();
  mp_state(c)->every = every;
  return PD_OK;
}

bool mpnn_capturing(const pd_ctx* c) { return c->mpnn && reinterpret_cast<const MpnnState*>(c->mpnn)->every > 0; }

int mpnn_capture_every(const pd_ctx* c) { return c->mpnn ? reinterpret_cast<const MpnnState*>(c->mpnn)->every : 0; }

int mpnn_snapshot(pd_ctx* c, const double* r, const double* x) {
  MpnnState* s = mp_state(c);
  const int64_t m = 3 * c->n;
  if (s->nsnap >= 64) return PD_OK;
  if ((int)s->snap_r.size() <= s->nsnap) {
    s->snap_r.push_back(new DBuf<double>());
    s->snap_x.push_back(new DBuf<double>());
  }
  DBuf<double>* R = s->snap_r[s->nsnap];
  DBuf<double>* X = s->snap_x[s->nsnap];
  if (R->count < (size_t)m) {
    PD_CUDA_TRY(c, R->alloc(m));
    PD_CUDA_TRY(c, X->alloc(m));
  }
  PD_CUDA_TRY(c, cudaMemcpyAsync(R->p, r, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(X->p, x, m * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  s->nsnap++;
  return PD_OK;
}

int mpnn_commit_snapshots(pd_ctx* c, const double* x_final, const double* dinv) {
  MpnnState* s = mp_state(c);
  const int64_t n = c->n;
  const size_t per = 9 * (size_t)n;
  if (s->npairs + s->nsnap > s->cap) {
    const int64_t cap = std::max<int64_t>(2 * s->cap, s->npairs + s->nsnap + 64);
    DBuf<float> np;
    PD_CUDA_TRY(c, np.alloc(per * cap));
    if (s->npairs)
      PD_CUDA_TRY(c, cudaMemcpyAsync(np.p, s->pairs.p, per * s->npairs * sizeof(float), cudaMemcpyDeviceToDevice,
                                     c->stream));
    PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    std::swap(np.p, s->pairs.p);
    std::swap(np.count, s->pairs.count);
    s->cap = cap;
  }
  for (int k = 0; k < s->nsnap; ++k) {
    k_mp_make_pair<<<g1(n), 256, 0, c->stream>>>(n, dinv, s->snap_r[k]->p, x_final, s->snap_x[k]->p,
                                                 s->pairs.p + per * (s->npairs + k));
  }
  PD_CUDA_TRY(c, cudaGetLastError());
  for (int k = 0; k < s->nsnap; ++k) s->pair_k.push_back(current_modulus(c));
  s->npairs += s->nsnap;
  s->nsnap = 0;
  return PD_OK;
}

void mpnn_drop_snapshots(pd_ctx* c) {
  if (c->mpnn) mp_state(c)->nsnap = 0;
}

int64_t mpnn_num_pairs(const pd_ctx* c) { return c->mpnn ? reinterpret_cast<const MpnnState*>(c->mpnn)->npairs : 0; }

int mpnn_get_weights(pd_ctx* c, float* w) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  PD_CUDA_TRY(c, d2h(c, w, s->w.p, NPARAM * sizeof(float)));
  return PD_OK;
}

int mpnn_set_weights(pd_ctx* c, const float* w) {
  MpnnState* s = mp_state(c);
  if (!s || !s->w.p) {
    c->err = "call pd_mpnn_init before loading weights";
    return PD_ERR_STATE;
  }
  PD_CUDA_TRY(c, h2d(c, s->w.p, w, NPARAM * sizeof(float)));
  k_mp_cast<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(NPARAM, s->w.p, s->wb.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  s->ready = true;
  s->trained = true;
  return PD_OK;
}

int mpnn_num_params() { return NPARAM; }

double mpnn_coarse_cell(const pd_ctx* c) {
  return c->mpnn ? reinterpret_cast<const MpnnState*>(c->mpnn)->coarse_cell : -1.0;
}

int mpnn_set_coarse(pd_ctx* c, double cell) {
  if (!c->mpnn) c->mpnn = new MpnnState();
  mp_state(c)->coarse_cell = cell < 0.0 ? -1.0 : cell;
  return PD_OK;
}

}  // namespace pdb
