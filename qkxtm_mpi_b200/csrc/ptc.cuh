// ptc.cuh -- device kernels of the learned preconditioner: a linear,
// gauge-covariant parallel-transport convolution (PTC) network.
//
// Layer l maps C_in to C_out channels (each a colour 3-vector per site):
//   out[x][c] = sum_{p=0..8} sum_c' W[p][c][c'] (T_p in[.][c'])(x)
// with the paths p = 0 identity, p = 1 + 2 mu: U_mu(x) in(x + mu), p = 2 + 2 mu:
// U_mu(x - mu)^dag in(x - mu).  The links are the operator's (12-real FP32,
// SU(3), boundary sign applied from the t coordinate), so the network
// commutes with gauge transformations as M^-1 does.  No reference counterpart.
//
// Why the channels are colour vectors.  A gauge transformation acts on the
// colour index of every site.  A layer whose weights mixed colour components
// (a 12 -> 16 complex map of a site's spin-colour numbers) would not commute
// with it; the weights must act on a channel index and leave colour to the
// transports.  A spin-colour spinor is therefore 4 channels of colour vectors,
// and a hidden width of 16 channels is 16 colour vectors (48 complex numbers a
// site): the gauge-covariant form of a 12 -> 16 -> 16 -> 12 complex network has
// 4 spin channels in and out and 16 hidden, 4 -> 16 -> ... -> 16 -> 4 here.
//
// Activation fields.  Channel c, colour b of a site is complex number
// k = c*3 + b; the four channels of group q = c/4 are 12 complex numbers in
// three 16-byte words (word k'/4, slot k'%4 for k' = k - 12q).
//   BF16 (hidden activations and their gradients): per parity [C/4][3][Vh]
//         uint4, each complex one __nv_bfloat162 (re, im) -- 48 B a site and
//         group, half of FP32;
//   FP32 (network input and output, C = 4): the solver's FP32 spinor, per
//         parity [6][Vh] float4 with complex k in word k/2 (channel = spin).
// A PtcField holds the two parity bases separately, so the solver's
// single-parity fields are network inputs and outputs without copies.
//
// Weights are BF16 (one __nv_bfloat162 per complex weight) in [9][C_out][C_in]
// per layer; arithmetic is FP32 (packed FFMA2), weight-gradient sums FP64.
#pragma once
#include <cuda_bf16.h>

#include "qkx_common.cuh"

namespace qkx {

constexpr int PTC_NT = 128;  // threads of the weight-gradient kernel
constexpr int PTC_TS = 32;   // sites per tile of the weight-gradient kernel
constexpr int PTC_SB = 64;   // sites per block of the layer kernel (x 3 colour threads)

struct PtcField {
  void* p[2];  // per parity: BF16 [C/4][3][Vh] uint4, or FP32 [6][Vh] float4 (C = 4)
};

// neighbour, link and sign of path p at site (par, cb) with coordinates x and
// lexicographic index s.  Returns the link already daggered for backward paths
// and multiplied by the boundary sign.
struct PtcHop {
  int npar, n;
};

__device__ __forceinline__ PtcHop ptc_hop(const GaugeF32x12& u, const Geom& g, int par, int cb, const int x[4], int s,
                                          int p, Link<float>& U) {
  if (p == 0) return {par, cb};
  const int mu = (p - 1) >> 1;
  const bool fwd = ((p - 1) & 1) == 0;
  const int L0 = g.L[0], L01 = L0 * g.L[1];
  const int stride = mu == 0 ? 1 : (mu == 1 ? L0 : (mu == 2 ? L01 : L01 * g.L[2]));
  const int Lm = g.L[mu];
  float sg = 1.0f;
  int n;
  if (fwd) {
    n = (x[mu] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    U = u.load(par, mu, cb);
    if (mu == 3 && g.bc_sign < 0 && x[3] == Lm - 1) sg = -1.0f;
  } else {
    n = (x[mu] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    const Link<float> v = u.load(1 - par, mu, n);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) U.m[i][j] = conj(v.m[j][i]);
    if (mu == 3 && g.bc_sign < 0 && x[3] == 0) sg = -1.0f;
  }
  if (sg < 0)
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) U.m[i][j] = {-U.m[i][j].re, -U.m[i][j].im};
  return {1 - par, n};
}

__device__ __forceinline__ void ptc_mv(const Link<float>& U, const float2 v[3], float2 s[3]) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    float re = 0.f, im = 0.f;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      re = fmaf(U.m[i][j].re, v[j].x, fmaf(-U.m[i][j].im, v[j].y, re));
      im = fmaf(U.m[i][j].re, v[j].y, fmaf(U.m[i][j].im, v[j].x, im));
    }
    s[i] = make_float2(re, im);
  }
}

// BF16 pair <-> FP32 pair (the widening is exact: a BF16 is the upper half of an FP32)
__device__ __forceinline__ float2 ptc_bf2f(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}
__device__ __forceinline__ uint32_t ptc_f2bf(float2 v) {
  __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
  return *reinterpret_cast<uint32_t*>(&h);
}

// the four channels of group q at site (par, n), all colours: v[channel][colour]
template <bool F32>
__device__ __forceinline__ void ptc_load4(const PtcField& f, int Vh, int par, int n, int q, float2 v[4][3]) {
  if constexpr (F32) {
    const float4* b = static_cast<const float4*>(f.p[par]) + n;  // C = 4: q = 0
#pragma unroll
    for (int w = 0; w < 6; w++) {
      const float4 x = __ldg(b + (size_t)w * Vh);
      v[(2 * w) / 3][(2 * w) % 3] = make_float2(x.x, x.y);
      v[(2 * w + 1) / 3][(2 * w + 1) % 3] = make_float2(x.z, x.w);
    }
  } else {
    const uint4* b = static_cast<const uint4*>(f.p[par]) + (size_t)(3 * q) * Vh + n;
    const uint4 w0 = __ldg(b), w1 = __ldg(b + Vh), w2 = __ldg(b + 2 * (size_t)Vh);
    const uint32_t ws[12] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
#pragma unroll
    for (int k = 0; k < 12; k++) v[k / 3][k % 3] = ptc_bf2f(ws[k]);
  }
}

// one complex number: channel ch, colour a of site (par, cb)
template <bool F32>
__device__ __forceinline__ void ptc_store1(const PtcField& f, int Vh, int par, int cb, int ch, int a, float2 v) {
  if constexpr (F32) {
    const int k = ch * 3 + a;  // C = 4
    float2* b = reinterpret_cast<float2*>(static_cast<float4*>(f.p[par]) + (size_t)(k >> 1) * Vh + cb) + (k & 1);
    *b = v;
  } else {
    const int q = ch >> 2, k = (ch & 3) * 3 + a;
    uint32_t* b = reinterpret_cast<uint32_t*>(static_cast<uint4*>(f.p[par]) + (size_t)(3 * q + (k >> 2)) * Vh + cb) +
                  (k & 3);
    *b = ptc_f2bf(v);
  }
}

// acc += w * s (complex), as two packed FMAs: (w.re, w.re) (s.re, s.im) + (-w.im, w.im) (s.im, s.re)
__device__ __forceinline__ float2 cfma2(float2 wa, float2 wb, float2 s, float2 acc) {
  return __ffma2_rn(wb, make_float2(s.y, s.x), __ffma2_rn(wa, s, acc));
}

// One PTC layer on the FP32 pipe.  Each site is split over three colour threads
// (block PTC_SB x 3): thread (site, a) transports every input channel with row a
// of the path's link and accumulates the CO outputs of colour a only, so a
// thread holds CO complex accumulators instead of 3 CO.  Blocks alternate
// parities when npar = 2; npar = 1 computes parity par0 only.  The weights are
// staged in dynamic shared memory as the pairs (w.re, w.re), (-w.im, w.im).
template <int CI, int CO, bool IN32, bool OUT32>
__global__ void __launch_bounds__(PTC_SB * 3, 3)
    k_ptc_layer(PtcField in, PtcField out, const __nv_bfloat162* __restrict__ w, GaugeF32x12 u, Geom g, int par0,
                int npar) {
  static_assert(CI % 4 == 0 && CO % 4 == 0 && (!IN32 || CI == 4) && (!OUT32 || CO == 4), "widths");
  extern __shared__ float4 ptc_sw[];  // [9][CO][CI]
  const int tid = threadIdx.y * PTC_SB + threadIdx.x;
  for (int i = tid; i < 9 * CO * CI; i += PTC_SB * 3) {
    const float2 f = __bfloat1622float2(w[i]);
    ptc_sw[i] = make_float4(f.x, f.x, -f.y, f.y);
  }
  __syncthreads();
  const int par = npar == 2 ? (blockIdx.x & 1) : par0;
  const int sb = npar == 2 ? (blockIdx.x >> 1) : blockIdx.x;
  const int cb = sb * PTC_SB + threadIdx.x, a = threadIdx.y;
  if (cb >= g.Vh) return;
  int x[4];
  cb_coords(g, cb, par, x);
  const int s = x[0] + g.L[0] * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]));
  float2 acc[CO];
#pragma unroll
  for (int c = 0; c < CO; c++) acc[c] = make_float2(0.f, 0.f);
#pragma unroll 1
  for (int p = 0; p < 9; p++) {
    Link<float> U;
    const PtcHop h = ptc_hop(u, g, par, cb, x, s, p, U);
    // row a of the link
    Cx<float> ur[3];
#pragma unroll
    for (int b = 0; b < 3; b++) ur[b] = a == 0 ? U.m[0][b] : (a == 1 ? U.m[1][b] : U.m[2][b]);
    // with few outputs the registers allow every input group's loads in flight at once
    constexpr bool PF = !IN32 && CO <= 8;
    uint4 raw[PF ? CI / 4 : 1][3];
    if constexpr (PF) {
#pragma unroll
      for (int q = 0; q < CI / 4; q++)
#pragma unroll
        for (int k = 0; k < 3; k++)
          raw[q][k] = __ldg(static_cast<const uint4*>(in.p[h.npar]) + (size_t)(3 * q + k) * g.Vh + h.n);
    }
#pragma unroll(PF ? CI / 4 : 1)
    for (int q = 0; q < CI / 4; q++) {
      float2 v[4][3], t[4];
      if constexpr (PF) {
        const uint32_t ws[12] = {raw[q][0].x, raw[q][0].y, raw[q][0].z, raw[q][0].w, raw[q][1].x, raw[q][1].y,
                                 raw[q][1].z, raw[q][1].w, raw[q][2].x, raw[q][2].y, raw[q][2].z, raw[q][2].w};
#pragma unroll
        for (int k = 0; k < 12; k++) v[k / 3][k % 3] = ptc_bf2f(ws[k]);
      } else {
        ptc_load4<IN32>(in, g.Vh, h.npar, h.n, q, v);
      }
#pragma unroll
      for (int cl = 0; cl < 4; cl++) {
        if (p == 0) {
          t[cl] = a == 0 ? v[cl][0] : (a == 1 ? v[cl][1] : v[cl][2]);
        } else {
          float re = 0.f, im = 0.f;
#pragma unroll
          for (int b = 0; b < 3; b++) {
            re = fmaf(ur[b].re, v[cl][b].x, fmaf(-ur[b].im, v[cl][b].y, re));
            im = fmaf(ur[b].re, v[cl][b].y, fmaf(ur[b].im, v[cl][b].x, im));
          }
          t[cl] = make_float2(re, im);
        }
      }
      const float4* wr = ptc_sw + (p * CO) * CI + 4 * q;
#pragma unroll
      for (int c = 0; c < CO; c++)
#pragma unroll
        for (int cl = 0; cl < 4; cl++) {
          const float4 wv = wr[c * CI + cl];
          acc[c] = cfma2(make_float2(wv.x, wv.y), make_float2(wv.z, wv.w), t[cl], acc[c]);
        }
    }
  }
#pragma unroll
  for (int c = 0; c < CO; c++) ptc_store1<OUT32>(out, g.Vh, par, cb, c, a, acc[c]);
}

// Weight gradient of one layer: dW[p][c][c'] = sum_{x, colour} gy[x][c] conj((T_p a)[x][c'])
// (dL/dW^* for dL/dy^* = gy).  Each block walks tiles of PTC_TS sites of one
// parity; per path it stages the transported input and the output gradient of
// the tile in shared memory and each thread sums whole entries.  Tile sums are
// FP32 (PTC_TS * 3 terms), accumulated across tiles in FP64; the block's
// totals go to part[block][9][CO][CI] for a fixed-order reduction.
template <int CI, int CO, bool A32, bool G32>
__global__ void __launch_bounds__(PTC_NT) k_ptc_wgrad(PtcField a, PtcField gy, GaugeF32x12 u, Geom g,
                                                      double2* __restrict__ part) {
  constexpr int NE = CO * CI;
  constexpr int EPT = (NE + PTC_NT - 1) / PTC_NT;  // entries per thread
  __shared__ float2 sS[PTC_TS][CI][3];
  __shared__ float2 sG[PTC_TS][CO][3];
  double2 accd[9][EPT];
#pragma unroll
  for (int p = 0; p < 9; p++)
#pragma unroll
    for (int j = 0; j < EPT; j++) accd[p][j] = make_double2(0.0, 0.0);
  const int tpp = (g.Vh + PTC_TS - 1) / PTC_TS;  // tiles per parity
  for (int t = blockIdx.x; t < 2 * tpp; t += gridDim.x) {
    const int par = t / tpp;
    const int cb0 = (t % tpp) * PTC_TS;
    __syncthreads();
    // output gradient of the tile
    for (int i = threadIdx.x; i < PTC_TS * (CO / 4); i += PTC_NT) {
      const int site = i % PTC_TS, q = i / PTC_TS;
      const int cb = cb0 + site;
      float2 v[4][3];
      if (cb < g.Vh) {
        ptc_load4<G32>(gy, g.Vh, par, cb, q, v);
      } else {
#pragma unroll
        for (int cl = 0; cl < 4; cl++)
#pragma unroll
          for (int k = 0; k < 3; k++) v[cl][k] = make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int cl = 0; cl < 4; cl++)
#pragma unroll
        for (int k = 0; k < 3; k++) sG[site][4 * q + cl][k] = v[cl][k];
    }
#pragma unroll 1
    for (int p = 0; p < 9; p++) {
      for (int i = threadIdx.x; i < PTC_TS * (CI / 4); i += PTC_NT) {
        const int site = i % PTC_TS, q = i / PTC_TS;
        const int cb = cb0 + site;
        float2 s[4][3];
        if (cb < g.Vh) {
          int x[4];
          cb_coords(g, cb, par, x);
          const int sl = x[0] + g.L[0] * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]));
          Link<float> U;
          const PtcHop h = ptc_hop(u, g, par, cb, x, sl, p, U);
          float2 v[4][3];
          ptc_load4<A32>(a, g.Vh, h.npar, h.n, q, v);
#pragma unroll
          for (int cl = 0; cl < 4; cl++) {
            if (p == 0) {
#pragma unroll
              for (int k = 0; k < 3; k++) s[cl][k] = v[cl][k];
            } else {
              ptc_mv(U, v[cl], s[cl]);
            }
          }
        } else {
#pragma unroll
          for (int cl = 0; cl < 4; cl++)
#pragma unroll
            for (int k = 0; k < 3; k++) s[cl][k] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int cl = 0; cl < 4; cl++)
#pragma unroll
          for (int k = 0; k < 3; k++) sS[site][4 * q + cl][k] = s[cl][k];
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < EPT; j++) {
        const int e = threadIdx.x + j * PTC_NT;
        if (e < NE) {
          const int c = e / CI, cp = e % CI;
          float re = 0.f, im = 0.f;
#pragma unroll 4
          for (int site = 0; site < PTC_TS; site++)
#pragma unroll
            for (int k = 0; k < 3; k++) {
              const float2 gg = sG[site][c][k], ss = sS[site][cp][k];
              re = fmaf(gg.x, ss.x, fmaf(gg.y, ss.y, re));
              im = fmaf(gg.y, ss.x, fmaf(-gg.x, ss.y, im));
            }
          accd[p][j].x += re;
          accd[p][j].y += im;
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int p = 0; p < 9; p++)
#pragma unroll
    for (int j = 0; j < EPT; j++) {
      const int e = threadIdx.x + j * PTC_NT;
      if (e < NE) part[((size_t)blockIdx.x * 9 + p) * NE + e] = accd[p][j];
    }
}

// grad[i] = sum over blocks of part[b][i], fixed order
static __global__ void k_ptc_wgrad_reduce(const double2* __restrict__ part, int nblocks, int n,
                                          double2* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 s = make_double2(0.0, 0.0);
  for (int b = 0; b < nblocks; b++) {
    const double2 v = part[(size_t)b * n + i];
    s.x += v.x;
    s.y += v.y;
  }
  grad[i] = s;
}

// backward weights of a layer: Wt[q(p)][c'][c] = conj(W[p][c][c']), q(p) the reversed path
static __global__ void k_ptc_wtrans(const __nv_bfloat162* __restrict__ w, __nv_bfloat162* __restrict__ wt, int ci,
                                    int co) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 9 * ci * co) return;
  const int p = i / (co * ci), c = (i / ci) % co, cp = i % ci;
  const int q = p == 0 ? 0 : (((p - 1) & 1) == 0 ? p + 1 : p - 1);
  const __nv_bfloat162 v = w[i];
  wt[((size_t)q * ci + cp) * co + c] = __halves2bfloat162(v.x, __hneg(v.y));
}

// Adam on the complex weights as pairs of reals; the real gradient of the loss
// is 2 (Re, Im) of dL/dW^*.  Writes the BF16 copy the layer kernels read.
static __global__ void k_ptc_adam(float2* __restrict__ w, float2* __restrict__ m, float2* __restrict__ v,
                                  const double2* __restrict__ grad, __nv_bfloat162* __restrict__ wb, int n, float lr,
                                  float b1, float b2, float bc1, float bc2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gx = 2.0f * (float)grad[i].x, gy = 2.0f * (float)grad[i].y;
  float2 mm = m[i], vv = v[i], ww = w[i];
  mm.x = b1 * mm.x + (1.f - b1) * gx;
  mm.y = b1 * mm.y + (1.f - b1) * gy;
  vv.x = b2 * vv.x + (1.f - b2) * gx * gx;
  vv.y = b2 * vv.y + (1.f - b2) * gy * gy;
  ww.x -= lr * (mm.x / bc1) / (sqrtf(vv.x / bc2) + eps);
  ww.y -= lr * (mm.y / bc1) / (sqrtf(vv.y / bc2) + eps);
  m[i] = mm;
  v[i] = vv;
  w[i] = ww;
  wb[i] = __floats2bfloat162_rn(ww.x, ww.y);
}

}  // namespace qkx
