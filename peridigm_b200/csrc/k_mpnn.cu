// Learned message-passing preconditioner for the quasi-static CG (sm_100a).
// No counterpart in the reference; it plugs into the block-Jacobi CG of
// k_qs.cu as z = P_bj r + s_a * N(a/s_a, r/s_r), a = P_bj r, s_a = rms(a),
// s_r = rms(r) (so z scales with r), on the subgraph of bonds shorter than a
// radius (the nearest shells of the bond family).
//
// Network (hidden 64, BF16 weights and BF16 node activations, FP32 accumulate):
//   h0 = relu(W0 f + b0)                         f = (a/s_a, r/s_r), 6 inputs
//   h_l = h_{l-1} + relu(Ws_l h_{l-1} + Wn_l m_l + b_l),  m_l = mean_{j in N(i)} h_{l-1,j},  l = 1..3
//   out = Wd h3 + bd                              3 outputs
// Training: residuals r_k captured from block-Jacobi CG solves, loss
// |K z - r|^2 / |r|^2 per residual (z approximates a local inverse of the
// tangent, the part a 3-hop network can represent), Adam on FP32 master
// weights; forward and backward are the kernels below, one warp per node,
// gathers only (the transpose of the mean aggregation is a gather over the
// symmetric subgraph), deterministic block reductions for weight gradients.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "pd_internal.cuh"

namespace pdb {

constexpr int H = 64;
constexpr int F = 6;
constexpr int NL = 3;
constexpr int OFF_W0 = 0, OFF_B0 = H * F;
constexpr int OFF_L = OFF_B0 + H;               // per layer: Ws (H*H), Wn (H*H), b (H)
constexpr int LSZ = 2 * H * H + H;
constexpr int OFF_WD = OFF_L + NL * LSZ, OFF_BD = OFF_WD + 3 * H;
constexpr int NPARAM = OFF_BD + 3;
constexpr int kRed = 148;

struct MpnnState {
  bool ready = false;    // weights initialised (trained or loaded)
  bool trained = false;
  double radius = 0.0;
  DBuf<int64_t> mrow;
  DBuf<int32_t> mcol;
  int64_t n = 0;
  DBuf<float> w, g, am, av, gpart;
  DBuf<__nv_bfloat16> wb;
  int64_t adam_t = 0;
  // activations
  DBuf<float> feat, pre[NL + 1], m[NL], dh, dhs, dm, gout, scal;
  DBuf<__nv_bfloat16> h[NL + 1];
  DBuf<double> a;  // P_bj r of the current application
  DBuf<double> bjpart, dscal;  // inference reduction partials and scales
  // training set: per pair a, r, e (float, 3n each)
  DBuf<float> pairs;
  int64_t npairs = 0, cap = 0;
  std::vector<double> pair_k;  // bulk modulus at capture (the tangent scales with it)
  // capture from CG
  int every = 0;
  std::vector<DBuf<double>*> snap_r, snap_x;
  int nsnap = 0;
  ~MpnnState() {
    for (auto* p : snap_r) delete p;
    for (auto* p : snap_x) delete p;
  }
};

// ---------------------------------------------------------------------------
// Subgraph of bonds shorter than the radius (symmetric when the bond family is)
// ---------------------------------------------------------------------------
template <bool FILL>
__global__ void k_mp_subgraph(int64_t n, const int64_t* __restrict__ row, const int32_t* __restrict__ col,
                              const uint8_t* __restrict__ dmg, const double4* __restrict__ xv, double r2,
                              int64_t* __restrict__ cnt, const int64_t* __restrict__ mrow, int32_t* __restrict__ mcol) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 xi = xv[i];
  int64_t k = FILL ? mrow[i] : 0;
  for (int64_t b = row[i]; b < row[i + 1]; ++b) {
    if (dmg[b]) continue;
    const int32_t j = col[b];
    const double4 xj = xv[j];
    const double d0 = xj.x - xi.x, d1 = xj.y - xi.y, d2 = xj.z - xi.z;
    if (d0 * d0 + d1 * d1 + d2 * d2 <= r2) {
      if (FILL) mcol[k] = j;
      ++k;
    }
  }
  if (!FILL) cnt[i] = k;
}

__global__ void k_mp_scan_small(int64_t n, const int64_t* __restrict__ cnt, int64_t* __restrict__ out) {
  // single-thread exclusive scan (setup only, n up to a few million)
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int64_t s = 0;
  for (int64_t i = 0; i < n; ++i) {
    out[i] = s;
    s += cnt[i];
  }
  out[n] = s;
}

// ---------------------------------------------------------------------------
// Inference / training forward
// ---------------------------------------------------------------------------
__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// a = P_bj r (FP64) and block partials of sum a^2, sum r^2
__global__ void k_mp_bj(int64_t n, const double* __restrict__ dinv, const double* __restrict__ r,
                        double* __restrict__ a, float* __restrict__ feat, double* __restrict__ partial) {
  __shared__ double s0[256], s1[256];
  double aa = 0.0, rr = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
    const double* d = dinv + 9 * i;
    const double a0 = d[0] * r0 + d[1] * r1 + d[2] * r2;
    const double a1 = d[3] * r0 + d[4] * r1 + d[5] * r2;
    const double a2 = d[6] * r0 + d[7] * r1 + d[8] * r2;
    a[3 * i] = a0, a[3 * i + 1] = a1, a[3 * i + 2] = a2;
    aa += a0 * a0 + a1 * a1 + a2 * a2;
    rr += r0 * r0 + r1 * r1 + r2 * r2;
  }
  s0[threadIdx.x] = aa;
  s1[threadIdx.x] = rr;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s0[threadIdx.x] += s0[threadIdx.x + o], s1[threadIdx.x] += s1[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[2 * blockIdx.x] = s0[0], partial[2 * blockIdx.x + 1] = s1[0];
}

// scal[0] = s_a, scal[1] = s_r (rms, floored)
__global__ void k_mp_scales(int nblk, const double* __restrict__ partial, int64_t n, float* __restrict__ scal,
                            double* __restrict__ dscal) {
  if (threadIdx.x != 0) return;
  double sa = 0.0, sr = 0.0;
  for (int b = 0; b < nblk; ++b) sa += partial[2 * b], sr += partial[2 * b + 1];
  sa = sqrt(sa / (3.0 * (double)n));
  sr = sqrt(sr / (3.0 * (double)n));
  dscal[0] = sa;
  dscal[1] = sr;
  scal[0] = (float)(sa > 0 ? 1.0 / sa : 0.0);
  scal[1] = (float)(sr > 0 ? 1.0 / sr : 0.0);
}

// features from FP64 a, r (inference) or FP32 stored pair arrays (training)
template <typename T>
__global__ void k_mp_features(int64_t n, const T* __restrict__ a, const T* __restrict__ r,
                              const float* __restrict__ scal, float* __restrict__ feat) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float ia = scal[0], ir = scal[1];
  for (int c = 0; c < 3; ++c) {
    feat[F * i + c] = (float)a[3 * i + c] * ia;
    feat[F * i + 3 + c] = (float)r[3 * i + c] * ir;
  }
}

// h0 = relu(W0 f + b0); lane l owns outputs 2l, 2l+1
__global__ void __launch_bounds__(256) k_mp_encode(int64_t n, const float* __restrict__ feat,
                                                   const __nv_bfloat16* __restrict__ wb, float* __restrict__ pre0,
                                                   __nv_bfloat16* __restrict__ h0) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  float f[F];
  for (int k = 0; k < F; ++k) f[k] = feat[F * i + k];
  for (int q = 0; q < 2; ++q) {
    const int o = 2 * lane + q;
    float s = bf(wb[OFF_B0 + o]);
    for (int k = 0; k < F; ++k) s = fmaf(bf(wb[OFF_W0 + o * F + k]), f[k], s);
    if (pre0) pre0[(int64_t)H * i + o] = s;
    h0[(int64_t)H * i + o] = __float2bfloat16(fmaxf(s, 0.0f));
  }
}

// one message-passing layer; weights staged in shared memory transposed
// (wT[k][o]) so lane l reads the bf16 pair (2l, 2l+1) conflict-free.
__global__ void __launch_bounds__(256) k_mp_layer(int64_t n, const int64_t* __restrict__ mrow,
                                                  const int32_t* __restrict__ mcol,
                                                  const __nv_bfloat16* __restrict__ wl,
                                                  const __nv_bfloat16* __restrict__ hin, __nv_bfloat16* __restrict__ hout,
                                                  float* __restrict__ pre_out, float* __restrict__ m_out) {
  __shared__ __nv_bfloat162 sWs[H][H / 2], sWn[H][H / 2];
  __shared__ float sb[H];
  for (int t = threadIdx.x; t < H * H / 2; t += blockDim.x) {
    const int k = t / (H / 2), op = t % (H / 2);
    sWs[k][op] = __halves2bfloat162(wl[(2 * op) * H + k], wl[(2 * op + 1) * H + k]);
    sWn[k][op] = __halves2bfloat162(wl[H * H + (2 * op) * H + k], wl[H * H + (2 * op + 1) * H + k]);
  }
  for (int t = threadIdx.x; t < H; t += blockDim.x) sb[t] = bf(wl[2 * H * H + t]);
  __syncthreads();
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const __nv_bfloat162* hin2 = reinterpret_cast<const __nv_bfloat162*>(hin);
  const float2 hs = __bfloat1622float2(hin2[(int64_t)(H / 2) * i + lane]);
  float2 mm = make_float2(0.f, 0.f);
  const int64_t b0 = mrow[i], b1 = mrow[i + 1];
  for (int64_t b = b0; b < b1; ++b) {
    const float2 hj = __bfloat1622float2(hin2[(int64_t)(H / 2) * mcol[b] + lane]);
    mm.x += hj.x;
    mm.y += hj.y;
  }
  const float inv = b1 > b0 ? 1.0f / (float)(b1 - b0) : 0.0f;
  mm.x *= inv;
  mm.y *= inv;
  float o0 = sb[2 * lane], o1 = sb[2 * lane + 1];
#pragma unroll 8
  for (int k = 0; k < H; ++k) {
    const float hk = __shfl_sync(0xffffffffu, (k & 1) ? hs.y : hs.x, k >> 1);
    const float mk = __shfl_sync(0xffffffffu, (k & 1) ? mm.y : mm.x, k >> 1);
    const float2 ws = __bfloat1622float2(sWs[k][lane]);
    const float2 wn = __bfloat1622float2(sWn[k][lane]);
    o0 = fmaf(ws.x, hk, fmaf(wn.x, mk, o0));
    o1 = fmaf(ws.y, hk, fmaf(wn.y, mk, o1));
  }
  if (pre_out) {
    pre_out[(int64_t)H * i + 2 * lane] = o0;
    pre_out[(int64_t)H * i + 2 * lane + 1] = o1;
    m_out[(int64_t)H * i + 2 * lane] = mm.x;
    m_out[(int64_t)H * i + 2 * lane + 1] = mm.y;
  }
  reinterpret_cast<__nv_bfloat162*>(hout)[(int64_t)(H / 2) * i + lane] =
      __floats2bfloat162_rn(hs.x + fmaxf(o0, 0.0f), hs.y + fmaxf(o1, 0.0f));
}

// out = Wd h3 + bd ; z = a + s_a * out (inference, FP64 z)
__global__ void __launch_bounds__(256) k_mp_decode(int64_t n, const __nv_bfloat16* __restrict__ h3,
                                                   const __nv_bfloat16* __restrict__ wb,
                                                   const double* __restrict__ a, const double* __restrict__ dscal,
                                                   const uint8_t* __restrict__ fixed, double* __restrict__ z) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const float2 hv = __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(h3)[(int64_t)(H / 2) * i + lane]);
  float o[3];
  for (int c = 0; c < 3; ++c) {
    float s = bf(wb[OFF_WD + c * H + 2 * lane]) * hv.x + bf(wb[OFF_WD + c * H + 2 * lane + 1]) * hv.y;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    o[c] = s + bf(wb[OFF_BD + c]);
  }
  if (lane < 3) {
    const uint8_t fx = fixed ? fixed[i] : 0;
    const double v = ((fx >> lane) & 1) ? 0.0 : a[3 * i + lane] + dscal[0] * (double)o[lane];
    z[3 * i + lane] = v;
  }
}

// ---------------------------------------------------------------------------
// Training: loss and backward
// ---------------------------------------------------------------------------
// dh3 = Wd^T g
__global__ void __launch_bounds__(256) k_mp_decode_back(int64_t n, const __nv_bfloat16* __restrict__ wb,
                                                        const float* __restrict__ gout, float* __restrict__ dh) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  for (int q = 0; q < 2; ++q) {
    const int k = 2 * lane + q;
    float s = 0.0f;
    for (int c = 0; c < 3; ++c) s = fmaf(bf(wb[OFF_WD + c * H + k]), gout[3 * i + c], s);
    dh[(int64_t)H * i + k] = s;
  }
}

// per node of layer l: dpre = dh * [pre > 0]; dhs = dh + Ws^T dpre ; dm = (Wn^T dpre)/deg
__global__ void __launch_bounds__(256) k_mp_layer_back(int64_t n, const int64_t* __restrict__ mrow,
                                                       const __nv_bfloat16* __restrict__ wl,
                                                       const float* __restrict__ pre, float* __restrict__ dh,
                                                       float* __restrict__ dhs, float* __restrict__ dm) {
  __shared__ __nv_bfloat162 sWs[H][H / 2], sWn[H][H / 2];  // [o][k pair]
  for (int t = threadIdx.x; t < H * H / 2; t += blockDim.x) {
    const int o = t / (H / 2), kp = t % (H / 2);
    sWs[o][kp] = __halves2bfloat162(wl[o * H + 2 * kp], wl[o * H + 2 * kp + 1]);
    sWn[o][kp] = __halves2bfloat162(wl[H * H + o * H + 2 * kp], wl[H * H + o * H + 2 * kp + 1]);
  }
  __syncthreads();
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int64_t base = (int64_t)H * i;
  float d0 = dh[base + 2 * lane], d1 = dh[base + 2 * lane + 1];
  const float p0 = pre[base + 2 * lane] > 0.f ? d0 : 0.f;
  const float p1 = pre[base + 2 * lane + 1] > 0.f ? d1 : 0.f;
  // dpre written back into dh for the weight-gradient pass
  dh[base + 2 * lane] = p0;
  dh[base + 2 * lane + 1] = p1;
  float s0 = d0, s1 = d1, m0 = 0.f, m1 = 0.f;
#pragma unroll 8
  for (int o = 0; o < H; ++o) {
    const float po = __shfl_sync(0xffffffffu, (o & 1) ? p1 : p0, o >> 1);
    const float2 ws = __bfloat1622float2(sWs[o][lane]);
    const float2 wn = __bfloat1622float2(sWn[o][lane]);
    s0 = fmaf(ws.x, po, s0);
    s1 = fmaf(ws.y, po, s1);
    m0 = fmaf(wn.x, po, m0);
    m1 = fmaf(wn.y, po, m1);
  }
  const int64_t deg = mrow[i + 1] - mrow[i];
  const float inv = deg > 0 ? 1.0f / (float)deg : 0.0f;
  dhs[base + 2 * lane] = s0;
  dhs[base + 2 * lane + 1] = s1;
  dm[base + 2 * lane] = m0 * inv;
  dm[base + 2 * lane + 1] = m1 * inv;
}

// dh_prev[j] = dhs[j] + sum_{i in N(j)} dm[i]   (transpose of the mean over a symmetric graph)
__global__ void __launch_bounds__(256) k_mp_gather_back(int64_t n, const int64_t* __restrict__ mrow,
                                                        const int32_t* __restrict__ mcol,
                                                        const float* __restrict__ dhs, const float* __restrict__ dm,
                                                        float* __restrict__ dh_prev) {
  const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  const float2* dm2 = reinterpret_cast<const float2*>(dm);
  float2 s = reinterpret_cast<const float2*>(dhs)[(int64_t)(H / 2) * j + lane];
  for (int64_t b = mrow[j]; b < mrow[j + 1]; ++b) {
    const float2 v = dm2[(int64_t)(H / 2) * mcol[b] + lane];
    s.x += v.x;
    s.y += v.y;
  }
  reinterpret_cast<float2*>(dh_prev)[(int64_t)(H / 2) * j + lane] = s;
}

// encoder: dpre0 = dh0 * [pre0 > 0] (in place)
__global__ void k_mp_relu_back(int64_t m, const float* __restrict__ pre, float* __restrict__ dh) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m && !(pre[k] > 0.f)) dh[k] = 0.f;
}

// Weight gradient partials: G[o][k] += sum_i A[i][o] B[i][k]; A = dpre [n][H],
// B [n][K] (bf16 activations, fp32 means or features); bias row: sum_i A[i][o].
template <typename TB>
__global__ void __launch_bounds__(256) k_mp_wgrad(int64_t n, int K, const float* __restrict__ A,
                                                  const TB* __restrict__ B, float* __restrict__ part) {
  __shared__ float sa[H], sbv[H];
  const int entries = H * K + H;
  float acc[17];
  for (int q = 0; q < 17; ++q) acc[q] = 0.f;
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(n, i0 + per);
  for (int64_t i = i0; i < i1; ++i) {
    if (threadIdx.x < H) sa[threadIdx.x] = A[(int64_t)H * i + threadIdx.x];
    if (threadIdx.x < K) sbv[threadIdx.x] = (float)B[(int64_t)K * i + threadIdx.x];
    __syncthreads();
    int q = 0;
    for (int e = threadIdx.x; e < entries; e += blockDim.x, ++q) {
      if (e < H * K) acc[q] = fmaf(sa[e / K], sbv[e % K], acc[q]);
      else acc[q] += sa[e - H * K];
    }
    __syncthreads();
  }
  int q = 0;
  for (int e = threadIdx.x; e < entries; e += blockDim.x, ++q) part[(int64_t)blockIdx.x * entries + e] = acc[q];
}

template <>
__global__ void __launch_bounds__(256) k_mp_wgrad<__nv_bfloat16>(int64_t n, int K, const float* __restrict__ A,
                                                                 const __nv_bfloat16* __restrict__ B,
                                                                 float* __restrict__ part) {
  __shared__ float sa[H], sbv[H];
  const int entries = H * K + H;
  float acc[17];
  for (int q = 0; q < 17; ++q) acc[q] = 0.f;
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(n, i0 + per);
  for (int64_t i = i0; i < i1; ++i) {
    if (threadIdx.x < H) sa[threadIdx.x] = A[(int64_t)H * i + threadIdx.x];
    if (threadIdx.x < K) sbv[threadIdx.x] = __bfloat162float(B[(int64_t)K * i + threadIdx.x]);
    __syncthreads();
    int q = 0;
    for (int e = threadIdx.x; e < entries; e += blockDim.x, ++q) {
      if (e < H * K) acc[q] = fmaf(sa[e / K], sbv[e % K], acc[q]);
      else acc[q] += sa[e - H * K];
    }
    __syncthreads();
  }
  int q = 0;
  for (int e = threadIdx.x; e < entries; e += blockDim.x, ++q) part[(int64_t)blockIdx.x * entries + e] = acc[q];
}

// g[dst_w + o*K + k] += sum_b part[b][o*K+k]; g[dst_b + o] += sum_b part[b][H*K+o]
__global__ void k_mp_wgrad_reduce(int nblk, int K, const float* __restrict__ part, float* __restrict__ g, int dst_w,
                                  int dst_b) {
  const int entries = H * K + H;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < entries; e += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * entries + e];
    if (e < H * K) g[dst_w + e] += s;
    else if (dst_b >= 0) g[dst_b + (e - H * K)] += s;  // dst_b < 0: no bias for this matrix
  }
}

// decoder weight gradient: dWd[c][k] += sum_i g[i][c] h3[i][k]; dbd[c] += sum_i g[i][c]
__global__ void k_mp_dec_wgrad(int64_t n, const float* __restrict__ gout, const __nv_bfloat16* __restrict__ h3,
                               float* __restrict__ g) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. 3*H+3
  if (e >= 3 * H + 3) return;
  double s = 0.0;
  if (e < 3 * H) {
    const int c = e / H, k = e % H;
    for (int64_t i = 0; i < n; ++i) s += (double)gout[3 * i + c] * (double)__bfloat162float(h3[(int64_t)H * i + k]);
    g[OFF_WD + e] += (float)s;
  } else {
    const int c = e - 3 * H;
    for (int64_t i = 0; i < n; ++i) s += gout[3 * i + c];
    g[OFF_BD + c] += (float)s;
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
  wb[k] = __float2bfloat16(w[k]);
}

__global__ void k_mp_cast(int np, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < np) wb[k] = __float2bfloat16(w[k]);
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

static int mp_alloc(pd_ctx* c, MpnnState* s, bool train) {
  const int64_t n = c->n;
  if (s->n != n) {
    for (int l = 0; l <= NL; ++l) PD_CUDA_TRY(c, s->h[l].alloc((size_t)H * n));
    PD_CUDA_TRY(c, s->feat.alloc((size_t)F * n));
    PD_CUDA_TRY(c, s->a.alloc(3 * n));
    PD_CUDA_TRY(c, s->scal.alloc(8));
    PD_CUDA_TRY(c, s->bjpart.alloc(2 * kRed));
    PD_CUDA_TRY(c, s->dscal.alloc(2));
    s->n = n;
    for (int l = 0; l <= NL; ++l) s->pre[l].release();
  }
  if (train && s->pre[0].count < (size_t)H * n) {
    for (int l = 0; l <= NL; ++l) PD_CUDA_TRY(c, s->pre[l].alloc((size_t)H * n));
    for (int l = 0; l < NL; ++l) PD_CUDA_TRY(c, s->m[l].alloc((size_t)H * n));
    PD_CUDA_TRY(c, s->dh.alloc((size_t)H * n));
    PD_CUDA_TRY(c, s->dhs.alloc((size_t)H * n));
    PD_CUDA_TRY(c, s->dm.alloc((size_t)H * n));
    PD_CUDA_TRY(c, s->gout.alloc(3 * n));
    PD_CUDA_TRY(c, s->gpart.alloc((size_t)kRed * (H * H + H) + 16));
  }
  return PD_OK;
}

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

int mpnn_init(pd_ctx* c, uint64_t seed, double radius) {
  if (!c->mpnn) c->mpnn = new MpnnState();
  MpnnState* s = mp_state(c);
  const int64_t n = c->n;
  s->radius = radius;
  // subgraph
  DBuf<int64_t> cnt;
  PD_CUDA_TRY(c, cnt.alloc(n + 1));
  PD_CUDA_TRY(c, s->mrow.alloc(n + 1));
  const double r2 = radius * radius;
  k_mp_subgraph<false><<<g1(n), 256, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, r2, cnt.p, nullptr,
                                                     nullptr);
  k_mp_scan_small<<<1, 32, 0, c->stream>>>(n, cnt.p, s->mrow.p);
  int64_t nm = 0;
  PD_CUDA_TRY(c, cudaMemcpyAsync(&nm, s->mrow.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  PD_CUDA_TRY(c, s->mcol.alloc(std::max<int64_t>(nm, 1)));
  k_mp_subgraph<true><<<g1(n), 256, 0, c->stream>>>(n, c->row.p, c->col.p, c->dmg.p, c->xv.p, r2, nullptr, s->mrow.p,
                                                    s->mcol.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  // weights: He-style uniform init from the seed; zero decoder so z starts at P_bj r
  std::vector<float> w(NPARAM, 0.f);
  std::mt19937_64 rng(seed);
  auto uni = [&](float lim) { return (float)((rng() >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0) * lim; };
  for (int k = 0; k < H * F; ++k) w[OFF_W0 + k] = uni(std::sqrt(6.0f / F));
  for (int l = 0; l < NL; ++l)
    for (int k = 0; k < 2 * H * H; ++k) w[OFF_L + l * LSZ + k] = uni(0.5f * std::sqrt(6.0f / (2 * H)));
  PD_CUDA_TRY(c, s->w.alloc(NPARAM));
  PD_CUDA_TRY(c, s->wb.alloc(NPARAM));
  PD_CUDA_TRY(c, s->g.alloc(NPARAM));
  PD_CUDA_TRY(c, s->am.alloc(NPARAM));
  PD_CUDA_TRY(c, s->av.alloc(NPARAM));
  PD_CUDA_TRY(c, h2d(c, s->w.p, w.data(), NPARAM * sizeof(float)));
  PD_CUDA_TRY(c, dzero(c, s->am.p, NPARAM * sizeof(float)));
  PD_CUDA_TRY(c, dzero(c, s->av.p, NPARAM * sizeof(float)));
  k_mp_cast<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(NPARAM, s->w.p, s->wb.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  s->adam_t = 0;
  s->ready = true;
  s->trained = false;
  return mp_alloc(c, s, false);
}

bool mpnn_ready(const pd_ctx* c) { return c->mpnn && reinterpret_cast<const MpnnState*>(c->mpnn)->ready; }

void mpnn_release(pd_ctx* c) {
  delete mp_state(c);
  c->mpnn = nullptr;
}

// Layers 1..3 from h[0]; training saves pre-activations and means.
static int mp_forward_layers(pd_ctx* c, MpnnState* s, bool save) {
  const int64_t n = c->n;
  for (int l = 0; l < NL; ++l) {
    k_mp_layer<<<gw(n), 256, 0, c->stream>>>(n, s->mrow.p, s->mcol.p, s->wb.p + OFF_L + l * LSZ, s->h[l].p,
                                             s->h[l + 1].p, save ? s->pre[l + 1].p : nullptr,
                                             save ? s->m[l].p : nullptr);
  }
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

int mpnn_apply(pd_ctx* c, const double* r, double* z, const double* dinv) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  TRY_RC(mp_alloc(c, s, false));
  const int64_t n = c->n;
  k_mp_bj<<<kRed, 256, 0, c->stream>>>(n, dinv, r, s->a.p, s->feat.p, s->bjpart.p);
  k_mp_scales<<<1, 32, 0, c->stream>>>(kRed, s->bjpart.p, n, s->scal.p, s->dscal.p);
  k_mp_features<double><<<g1(n), 256, 0, c->stream>>>(n, s->a.p, r, s->scal.p, s->feat.p);
  k_mp_encode<<<gw(n), 256, 0, c->stream>>>(n, s->feat.p, s->wb.p, nullptr, s->h[0].p);
  TRY_RC(mp_forward_layers(c, s, false));
  k_mp_decode<<<gw(n), 256, 0, c->stream>>>(n, s->h[NL].p, s->wb.p, s->a.p, s->dscal.p, qs_fixed_mask(c), z);
  PD_CUDA_TRY(c, cudaGetLastError());
  return PD_OK;
}

// z = a + s_a (Wd h3 + bd) in FP64 from a float `a`; prescribed dofs zero.
__global__ void __launch_bounds__(256) k_mp_zout(int64_t n, const __nv_bfloat16* __restrict__ h3,
                                                 const __nv_bfloat16* __restrict__ wb, const float* __restrict__ a,
                                                 double sa, const uint8_t* __restrict__ fixed,
                                                 double* __restrict__ z) {
  const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const float2 hv = __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(h3)[(int64_t)(H / 2) * i + lane]);
  float o[3];
  for (int c = 0; c < 3; ++c) {
    float s = bf(wb[OFF_WD + c * H + 2 * lane]) * hv.x + bf(wb[OFF_WD + c * H + 2 * lane + 1]) * hv.y;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    o[c] = s + bf(wb[OFF_BD + c]);
  }
  if (lane < 3) {
    const uint8_t fx = fixed ? fixed[i] : 0;
    z[3 * i + lane] = ((fx >> lane) & 1) ? 0.0 : (double)a[3 * i + lane] + sa * (double)o[lane];
  }
}

// res = scale*q - r (prescribed dofs zero); partials of |res|^2 and |r|^2
__global__ void k_mp_residual(int64_t m, double scale, const double* __restrict__ q, const float* __restrict__ r,
                              const uint8_t* __restrict__ fixed, double* __restrict__ res,
                              double* __restrict__ partial) {
  __shared__ double s0[256], s1[256];
  double a0 = 0.0, a1 = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
    const bool fx = fixed && ((fixed[k / 3] >> (k % 3)) & 1);
    const double rk = fx ? 0.0 : (double)r[k];
    const double v = fx ? 0.0 : scale * q[k] - rk;
    res[k] = v;
    a0 += v * v;
    a1 += rk * rk;
  }
  s0[threadIdx.x] = a0;
  s1[threadIdx.x] = a1;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s0[threadIdx.x] += s0[threadIdx.x + o], s1[threadIdx.x] += s1[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[2 * blockIdx.x] = s0[0], partial[2 * blockIdx.x + 1] = s1[0];
}

// gout = coef * kres (prescribed dofs zero)
__global__ void k_mp_gout(int64_t m, double coef, const double* __restrict__ kres, const uint8_t* __restrict__ fixed,
                          float* __restrict__ gout) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const bool fx = fixed && ((fixed[k / 3] >> (k % 3)) & 1);
  gout[k] = fx ? 0.f : (float)(coef * kres[k]);
}

// One pair (a = P_bj r, r as float [3n] each): forward with saved activations,
// residual-space loss L = |kscale K z - r|^2 / |r|^2 with K the tangent prepared
// by qs_prepare_current (kscale rescales it to the modulus of the pair), and
// backward accumulating into s->g. dL/dz = 2 kscale K (kscale K z - r)/|r|^2.
static int mp_pair_grad(pd_ctx* c, MpnnState* s, const float* pair, double kscale, double* loss) {
  const int64_t n = c->n, m = 3 * n;
  const float* A = pair;
  const float* R = pair + 3 * n;
  const uint8_t* fixed = qs_fixed_mask(c);
  DBuf<double> part, z, kz, res, kres;
  PD_CUDA_TRY(c, part.alloc(2 * kRed));
  PD_CUDA_TRY(c, z.alloc(m));
  PD_CUDA_TRY(c, kz.alloc(m));
  PD_CUDA_TRY(c, res.alloc(m));
  PD_CUDA_TRY(c, kres.alloc(m));
  std::vector<float> ha(m), hr(m);
  PD_CUDA_TRY(c, cudaMemcpyAsync(ha.data(), A, m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaMemcpyAsync(hr.data(), R, m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  double a2 = 0.0, r2 = 0.0;
  for (int64_t k = 0; k < m; ++k) a2 += (double)ha[k] * ha[k], r2 += (double)hr[k] * hr[k];
  const double sa = std::sqrt(a2 / (double)m), sr = std::sqrt(r2 / (double)m);
  const float hs[2] = {(float)(sa > 0 ? 1.0 / sa : 0.0), (float)(sr > 0 ? 1.0 / sr : 0.0)};
  PD_CUDA_TRY(c, cudaMemcpyAsync(s->scal.p, hs, sizeof(hs), cudaMemcpyHostToDevice, c->stream));
  k_mp_features<float><<<g1(n), 256, 0, c->stream>>>(n, A, R, s->scal.p, s->feat.p);
  k_mp_encode<<<gw(n), 256, 0, c->stream>>>(n, s->feat.p, s->wb.p, s->pre[0].p, s->h[0].p);
  TRY_RC(mp_forward_layers(c, s, true));
  k_mp_zout<<<gw(n), 256, 0, c->stream>>>(n, s->h[NL].p, s->wb.p, A, sa, fixed, z.p);
  PD_CUDA_TRY(c, cudaGetLastError());
  TRY_RC(qs_apply_K(c, z.p, kz.p));
  k_mp_residual<<<kRed, 256, 0, c->stream>>>(m, kscale, kz.p, R, fixed, res.p, part.p);
  TRY_RC(qs_apply_K(c, res.p, kres.p));
  std::vector<double> hp(2 * kRed);
  PD_CUDA_TRY(c, cudaMemcpyAsync(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  double rs2 = 0.0, rr2 = 0.0;
  for (int b = 0; b < kRed; ++b) rs2 += hp[2 * b], rr2 += hp[2 * b + 1];
  const double inv_r2 = rr2 > 0 ? 1.0 / rr2 : 0.0;
  // dL/dout = s_a dL/dz
  k_mp_gout<<<g1(m), 256, 0, c->stream>>>(m, 2.0 * kscale * inv_r2 * sa, kres.p, fixed, s->gout.p);
  // backward
  k_mp_dec_wgrad<<<1, 3 * H + 3, 0, c->stream>>>(n, s->gout.p, s->h[NL].p, s->g.p);
  k_mp_decode_back<<<gw(n), 256, 0, c->stream>>>(n, s->wb.p, s->gout.p, s->dh.p);
  for (int l = NL - 1; l >= 0; --l) {
    const __nv_bfloat16* wl = s->wb.p + OFF_L + l * LSZ;
    k_mp_layer_back<<<gw(n), 256, 0, c->stream>>>(n, s->mrow.p, wl, s->pre[l + 1].p, s->dh.p, s->dhs.p, s->dm.p);
    k_mp_wgrad<__nv_bfloat16><<<kRed, 256, 0, c->stream>>>(n, H, s->dh.p, s->h[l].p, s->gpart.p);
    k_mp_wgrad_reduce<<<17, 256, 0, c->stream>>>(kRed, H, s->gpart.p, s->g.p, OFF_L + l * LSZ, OFF_L + l * LSZ + 2 * H * H);
    k_mp_wgrad<float><<<kRed, 256, 0, c->stream>>>(n, H, s->dh.p, s->m[l].p, s->gpart.p);
    // Wn has no bias of its own: only the matrix part of this reduction is kept
    k_mp_wgrad_reduce<<<17, 256, 0, c->stream>>>(kRed, H, s->gpart.p, s->g.p, OFF_L + l * LSZ + H * H, -1);
    k_mp_gather_back<<<gw(n), 256, 0, c->stream>>>(n, s->mrow.p, s->mcol.p, s->dhs.p, s->dm.p, s->dh.p);
  }
  k_mp_relu_back<<<g1((int64_t)H * n), 256, 0, c->stream>>>((int64_t)H * n, s->pre[0].p, s->dh.p);
  k_mp_wgrad<float><<<kRed, 256, 0, c->stream>>>(n, F, s->dh.p, s->feat.p, s->gpart.p);
  k_mp_wgrad_reduce<<<2, 256, 0, c->stream>>>(kRed, F, s->gpart.p, s->g.p, OFF_W0, OFF_B0);
  PD_CUDA_TRY(c, cudaGetLastError());
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *loss = rs2 * inv_r2;
  return PD_OK;
}

int mpnn_loss_grad(pd_ctx* c, const float* pair_host, double* loss, float* grad_host) {
  MpnnState* s = mp_state(c);
  if (!s || !s->ready) {
    c->err = "learned preconditioner not initialised";
    return PD_ERR_STATE;
  }
  TRY_RC(mp_alloc(c, s, true));
  TRY_RC(qs_prepare_current(c));
  DBuf<float> pair;
  PD_CUDA_TRY(c, pair.alloc(6 * c->n));
  PD_CUDA_TRY(c, h2d(c, pair.p, pair_host, 6 * c->n * sizeof(float)));
  PD_CUDA_TRY(c, cudaMemsetAsync(s->g.p, 0, NPARAM * sizeof(float), c->stream));
  TRY_RC(mp_pair_grad(c, s, pair.p, 1.0, loss));
  if (grad_host) PD_CUDA_TRY(c, d2h(c, grad_host, s->g.p, NPARAM * sizeof(float)));
  return PD_OK;
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
  TRY_RC(mp_alloc(c, s, true));
  TRY_RC(qs_prepare_current(c));
  const int64_t n = c->n;
  const double k_now = current_modulus(c);
  std::mt19937_64 rng(12345 + s->adam_t);
  std::vector<int64_t> order(s->npairs);
  double last = 0.0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int64_t k = 0; k < s->npairs; ++k) order[k] = k;
    std::shuffle(order.begin(), order.end(), rng);
    double acc = 0.0;
    int64_t cnt = 0;
    for (int64_t b0 = 0; b0 < s->npairs; b0 += batch) {
      PD_CUDA_TRY(c, cudaMemsetAsync(s->g.p, 0, NPARAM * sizeof(float), c->stream));
      const int64_t b1 = std::min<int64_t>(s->npairs, b0 + batch);
      for (int64_t q = b0; q < b1; ++q) {
        double l = 0.0;
        TRY_RC(mp_pair_grad(c, s, s->pairs.p + (size_t)order[q] * 9 * n, s->pair_k[order[q]] / k_now, &l));
        acc += l;
        ++cnt;
      }
      s->adam_t += 1;
      const float b1c = 0.9f, b2c = 0.999f;
      const float c1 = 1.f - std::pow(b1c, (float)s->adam_t), c2 = 1.f - std::pow(b2c, (float)s->adam_t);
      k_mp_adam<<<(NPARAM + 255) / 256, 256, 0, c->stream>>>(NPARAM, s->w.p, s->g.p, s->am.p, s->av.p, (float)lr, b1c,
                                                             b2c, c1, c2, 1.0f / (float)(b1 - b0), s->wb.p);
      PD_CUDA_TRY(c, cudaGetLastError());
    }
    last = cnt ? acc / cnt : 0.0;
  }
  PD_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  s->trained = true;
  if (loss_out) *loss_out = last;
  return PD_OK;
}

// ---- pair capture from the block-Jacobi CG ---------------------------------
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
  if (!s || !s->mrow.p) {
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

}  // namespace pdb
