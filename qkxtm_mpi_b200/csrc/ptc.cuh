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
// Activation layout: even-odd, [parity][3C/2][Vh] float4, complex number
// k = c*3 + colour in word k/2, so channels c, c+1 fill three float4 words.
// For C = 4 this is exactly the FP32 spinor layout (SpinorF32), which lets the
// solver's fields be the network's input and output.
//
// Weights are BF16 (one __nv_bfloat162 per complex weight) in [9][C_out][C_in]
// per layer; arithmetic is FP32 (packed FFMA2), reductions FP64.
#pragma once
#include <cuda_bf16.h>

#include "qkx_common.cuh"

namespace qkx {

constexpr int PTC_NT = 128;  // threads (sites) per block of the layer kernels
constexpr int PTC_TS = 32;   // sites per tile of the weight-gradient kernel

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

// channels c, c+1 (c even) of an activation at site (par, n): 3 float4 words
__device__ __forceinline__ void ptc_load_pair(const float4* f, int C, int Vh, int par, int n, int c, float2 v0[3],
                                              float2 v1[3]) {
  const float4* b = f + ((size_t)par * (3 * C / 2) + (3 * c) / 2) * Vh + n;
  const float4 q0 = __ldg(b), q1 = __ldg(b + Vh), q2 = __ldg(b + 2 * (size_t)Vh);
  v0[0] = make_float2(q0.x, q0.y);
  v0[1] = make_float2(q0.z, q0.w);
  v0[2] = make_float2(q1.x, q1.y);
  v1[0] = make_float2(q1.z, q1.w);
  v1[1] = make_float2(q2.x, q2.y);
  v1[2] = make_float2(q2.z, q2.w);
}

// acc += w * s (complex), as two packed FMAs: (w.re, w.re) (s.re, s.im) + (-w.im, w.im) (s.im, s.re)
__device__ __forceinline__ float2 cfma2(float2 wa, float2 wb, float2 s, float2 acc) {
  return __ffma2_rn(wb, make_float2(s.y, s.x), __ffma2_rn(wa, s, acc));
}

// One PTC layer, one thread per site.  Blocks alternate parities.  The weights
// are staged in shared memory as the pairs (w.re, w.re), (-w.im, w.im).
template <int CI, int CO>
__global__ void __launch_bounds__(PTC_NT) k_ptc_layer(const float4* __restrict__ in, float4* __restrict__ out,
                                                      const __nv_bfloat162* __restrict__ w, GaugeF32x12 u, Geom g) {
  __shared__ float4 sw[9 * CO * CI];
  for (int i = threadIdx.x; i < 9 * CO * CI; i += PTC_NT) {
    const float2 f = __bfloat1622float2(w[i]);
    sw[i] = make_float4(f.x, f.x, -f.y, f.y);
  }
  __syncthreads();
  const int par = blockIdx.x & 1;
  const int cb = (blockIdx.x >> 1) * PTC_NT + threadIdx.x;
  if (cb >= g.Vh) return;
  int x[4];
  cb_coords(g, cb, par, x);
  const int s = x[0] + g.L[0] * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]));
  float2 acc[CO][3];
#pragma unroll
  for (int c = 0; c < CO; c++)
#pragma unroll
    for (int a = 0; a < 3; a++) acc[c][a] = make_float2(0.f, 0.f);
#pragma unroll 1
  for (int p = 0; p < 9; p++) {
    Link<float> U;
    const PtcHop h = ptc_hop(u, g, par, cb, x, s, p, U);
#pragma unroll 1
    for (int cp = 0; cp < CI; cp += 2) {
      float2 v0[3], v1[3], s0[3], s1[3];
      ptc_load_pair(in, CI, g.Vh, h.npar, h.n, cp, v0, v1);
      if (p == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
          s0[a] = v0[a];
          s1[a] = v1[a];
        }
      } else {
        ptc_mv(U, v0, s0);
        ptc_mv(U, v1, s1);
      }
      const float4* wr = sw + (p * CO) * CI + cp;
#pragma unroll
      for (int c = 0; c < CO; c++) {
        const float4 w0 = wr[c * CI], w1 = wr[c * CI + 1];
#pragma unroll
        for (int a = 0; a < 3; a++) {
          acc[c][a] = cfma2(make_float2(w0.x, w0.y), make_float2(w0.z, w0.w), s0[a], acc[c][a]);
          acc[c][a] = cfma2(make_float2(w1.x, w1.y), make_float2(w1.z, w1.w), s1[a], acc[c][a]);
        }
      }
    }
  }
  float4* o = out + (size_t)par * (3 * CO / 2) * g.Vh + cb;
#pragma unroll
  for (int q = 0; q < 3 * CO / 2; q++) {
    const int k0 = 2 * q, k1 = 2 * q + 1;
    o[(size_t)q * g.Vh] = make_float4(acc[k0 / 3][k0 % 3].x, acc[k0 / 3][k0 % 3].y, acc[k1 / 3][k1 % 3].x,
                                      acc[k1 / 3][k1 % 3].y);
  }
}

// Weight gradient of one layer: dW[p][c][c'] = sum_{x, colour} gy[x][c] conj((T_p a)[x][c'])
// (dL/dW^* for dL/dy^* = gy).  Each block walks tiles of PTC_TS sites of one
// parity; per path it stages the transported input and the output gradient of
// the tile in shared memory and each thread sums whole entries.  Tile sums are
// FP32 (PTC_TS * 3 terms), accumulated across tiles in FP64; the block's
// totals go to part[block][9][CO][CI] for a fixed-order reduction.
template <int CI, int CO>
__global__ void __launch_bounds__(PTC_NT) k_ptc_wgrad(const float4* __restrict__ a, const float4* __restrict__ gy,
                                                      GaugeF32x12 u, Geom g, double2* __restrict__ part) {
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
    for (int i = threadIdx.x; i < PTC_TS * (CO / 2); i += PTC_NT) {
      const int site = i % PTC_TS, cp = 2 * (i / PTC_TS);
      const int cb = cb0 + site;
      float2 v0[3], v1[3];
      if (cb < g.Vh) {
        ptc_load_pair(gy, CO, g.Vh, par, cb, cp, v0, v1);
      } else {
#pragma unroll
        for (int k = 0; k < 3; k++) v0[k] = v1[k] = make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        sG[site][cp][k] = v0[k];
        sG[site][cp + 1][k] = v1[k];
      }
    }
#pragma unroll 1
    for (int p = 0; p < 9; p++) {
      for (int i = threadIdx.x; i < PTC_TS * (CI / 2); i += PTC_NT) {
        const int site = i % PTC_TS, cp = 2 * (i / PTC_TS);
        const int cb = cb0 + site;
        float2 s0[3], s1[3];
        if (cb < g.Vh) {
          int x[4];
          cb_coords(g, cb, par, x);
          const int sl = x[0] + g.L[0] * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]));
          Link<float> U;
          const PtcHop h = ptc_hop(u, g, par, cb, x, sl, p, U);
          float2 v0[3], v1[3];
          ptc_load_pair(a, CI, g.Vh, h.npar, h.n, cp, v0, v1);
          if (p == 0) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
              s0[k] = v0[k];
              s1[k] = v1[k];
            }
          } else {
            ptc_mv(U, v0, s0);
            ptc_mv(U, v1, s1);
          }
        } else {
#pragma unroll
          for (int k = 0; k < 3; k++) s0[k] = s1[k] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int k = 0; k < 3; k++) {
          sS[site][cp][k] = s0[k];
          sS[site][cp + 1][k] = s1[k];
        }
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
