// hop_pair.cuh -- the FP16 multi-RHS hop on the packed FP32 pipe.
//
// Same operator, tiles and epilogues as hop_mrhs_kernel (reference
// Vector::applyDslash, lib/lattice_util.cpp:1158-1213, with the twist site
// factors of applyTwistAddDslash :1420 / applyTwistInv :1588 fused), for FP16
// spinors and 12-real FP16 links with an even number of right-hand sides per
// thread.  The right-hand sides of a thread are taken in pairs (j, j+1) and
// every complex component is held as two float2 values,
//     re = (re_j, re_{j+1}),  im = (im_j, im_{j+1}),
// so each projection add, link multiply-add and accumulation is one
// f32x2 instruction (fma.rn.f32x2 / add.rn.f32x2 / mul.rn.f32x2) for both
// right-hand sides of the pair.  Multiplying by +-1, +-i is a choice of lane
// pair and sign, never an instruction, and the link entries are broadcast to
// both lanes.  The hop of an FP16 batch is bound by instruction issue (about
// 1.2k instructions per site and right-hand side in scalar FP32); the packed
// form removes about a third of them.
//
// The per-site FP16 scale and the boundary sign are applied after the (linear)
// projection and link multiplication, as in hop_mrhs_kernel; the factor 2 of
// the diagonal projector (gamma_4 in the UKQCD basis) is folded into that
// scale.  Right-hand sides that are outside the batch or masked inactive read
// their partner's input (valid memory) and store nothing.
#pragma once
#include <cuda_fp16.h>

#include "hop_mrhs.cuh"

namespace qkx {

// one complex component for a pair of right-hand sides
struct CP {
  float2 re, im;
};

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, rounded once
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// a + phase<PH>(z), phase codes as in phase(): 0 -> 1, 1 -> i, 2 -> -1, 3 -> -i
template <int PH>
__device__ __forceinline__ CP addph(const CP& a, const CP& z) {
  if constexpr ((PH & 3) == 0) return {add2(a.re, z.re), add2(a.im, z.im)};
  else if constexpr ((PH & 3) == 1) return {sub2(a.re, z.im), add2(a.im, z.re)};
  else if constexpr ((PH & 3) == 2) return {sub2(a.re, z.re), sub2(a.im, z.im)};
  else return {add2(a.re, z.im), sub2(a.im, z.re)};
}

// acc += f * phase<PH>(z), fn = -f
template <int PH>
__device__ __forceinline__ void accph(CP& acc, const CP& z, float2 f, float2 fn) {
  if constexpr ((PH & 3) == 0) {
    acc.re = fma2(f, z.re, acc.re);
    acc.im = fma2(f, z.im, acc.im);
  } else if constexpr ((PH & 3) == 1) {
    acc.re = fma2(fn, z.im, acc.re);
    acc.im = fma2(f, z.re, acc.im);
  } else if constexpr ((PH & 3) == 2) {
    acc.re = fma2(fn, z.re, acc.re);
    acc.im = fma2(fn, z.im, acc.im);
  } else {
    acc.re = fma2(f, z.im, acc.re);
    acc.im = fma2(fn, z.re, acc.im);
  }
}

// the 12 stored components of right-hand sides j and k at one site, without the
// site scale; component q*4 + w is spin (q*4+w)/3, colour (q*4+w)%3
__device__ __forceinline__ void load_pair_raw(const uint4* bj, const uint4* bk, int Vh, CP (&v)[4][3]) {
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const uint4 wj = __ldg(bj + (size_t)q * Vh), wk = __ldg(bk + (size_t)q * Vh);
    const uint32_t sj[4] = {wj.x, wj.y, wj.z, wj.w}, sk[4] = {wk.x, wk.y, wk.z, wk.w};
#pragma unroll
    for (int w = 0; w < 4; w++) {
      const __half2 hj = *reinterpret_cast<const __half2*>(&sj[w]);
      const __half2 hk = *reinterpret_cast<const __half2*>(&sk[w]);
      const int k = 4 * q + w;
      v[k / 3][k % 3].re = make_float2(__low2float(hj), __low2float(hk));
      v[k / 3][k % 3].im = make_float2(__high2float(hj), __high2float(hk));
    }
  }
}

// rows h0, h1 of (1 + SIGN gamma_mu) s; for the diagonal gamma_4 the rows are
// taken as they are and the factor 2 goes into the caller's scale
template <int B, int MU, int SIGN>
__device__ __forceinline__ void proj_pair(const CP (&s)[4][3], CP (&h)[2][3]) {
  using PJ = Proj<B, MU, SIGN>;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if constexpr (PJ::diag) {
      h[0][a] = s[PJ::drow][a];
      h[1][a] = s[PJ::drow + 1][a];
    } else {
      h[0][a] = addph<PJ::p0>(s[0][a], s[PJ::c0][a]);
      h[1][a] = addph<PJ::p1>(s[1][a], s[PJ::c1][a]);
    }
  }
}

// acc += f * (the 4-spinor rebuilt from the rows h0, h1)
template <int B, int MU, int SIGN>
__device__ __forceinline__ void recon_pair(CP (&acc)[4][3], const CP (&h)[2][3], float2 f, float2 fn) {
  using PJ = Proj<B, MU, SIGN>;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if constexpr (PJ::diag) {
      accph<0>(acc[PJ::drow][a], h[0][a], f, fn);
      accph<0>(acc[PJ::drow + 1][a], h[1][a], f, fn);
    } else {
      accph<0>(acc[0][a], h[0][a], f, fn);
      accph<0>(acc[1][a], h[1][a], f, fn);
      accph<PJ::q0>(acc[PJ::c0][a], h[0][a], f, fn);
      accph<PJ::q1>(acc[PJ::c1][a], h[1][a], f, fn);
    }
  }
}

// o = U h (DG false) or U^+ h (DG true) on both spin rows of a pair
template <bool DG>
__device__ __forceinline__ void mul_link_pair(const Link<float>& u, const CP (&h)[2][3], CP (&o)[2][3]) {
#pragma unroll
  for (int s = 0; s < 2; s++) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      float2 re, im;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        // entry (a, b) of U, or of U^+ = conj(U^T)
        const float ur = DG ? u.m[b][a].re : u.m[a][b].re;
        const float ui = DG ? -u.m[b][a].im : u.m[a][b].im;
        if (b == 0) {
          re = mul2(bc2(ur), h[s][b].re);
          im = mul2(bc2(ur), h[s][b].im);
        } else {
          re = fma2(bc2(ur), h[s][b].re, re);
          im = fma2(bc2(ur), h[s][b].im, im);
        }
        re = fma2(bc2(-ui), h[s][b].im, re);
        im = fma2(bc2(ui), h[s][b].re, im);
      }
      o[s][a] = {re, im};
    }
  }
}

// gamma5 acting on the spin index: (gamma5 v)[s] = g5sign(s) * v[g5row(s)]
template <int B>
__host__ __device__ constexpr int g5row(int s) { return B == 0 ? (s + 2) % 4 : s; }
template <int B>
__host__ __device__ constexpr float g5sign(int s) { return (B == 0 || s < 2) ? 1.f : -1.f; }

template <int NP, int B, bool DAG, int MU>
__device__ __forceinline__ void hop_dir_pair(const uint4* const (&pin)[2 * NP], const float* const (&nin)[2 * NP],
                                             const GaugeF16x12& gauge, const Geom& g, int par, int cb,
                                             const int x[4], int s, int stride, const bool (&pact)[NP],
                                             CP (&acc)[NP][4][3]) {
  constexpr int SF = DAG ? +1 : -1;  // forward projector 1 + SF*g
  const int Vh = g.Vh;
  const int Lm = g.L[MU];
#pragma unroll
  for (int dir = 0; dir < 2; dir++) {
    int n;
    bool flip;
    Link<float> u;
    if (dir == 0) {
      n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
      flip = (MU == 3) && g.bc_sign < 0 && x[3] == Lm - 1;
      u = gauge.load(par, MU, cb);
    } else {
      n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
      flip = (MU == 3) && g.bc_sign < 0 && x[3] == 0;
      u = gauge.load(1 - par, MU, n);
    }
    constexpr bool diag_f = Proj<B, MU, SF>::diag, diag_b = Proj<B, MU, -SF>::diag;
    const float sg = (flip ? -1.f : 1.f) * ((dir == 0 ? diag_f : diag_b) ? 2.f : 1.f);
#pragma unroll
    for (int p = 0; p < NP; p++) {
      if (!pact[p]) continue;
      CP v[4][3], h[2][3], uh[2][3];
      load_pair_raw(pin[2 * p] + n, pin[2 * p + 1] + n, Vh, v);
      const float2 f = make_float2(sg * __ldg(nin[2 * p] + n), sg * __ldg(nin[2 * p + 1] + n));
      const float2 fn = make_float2(-f.x, -f.y);
      if (dir == 0) {
        proj_pair<B, MU, SF>(v, h);
        mul_link_pair<false>(u, h, uh);
        recon_pair<B, MU, SF>(acc[p], uh, f, fn);
      } else {
        proj_pair<B, MU, -SF>(v, h);
        mul_link_pair<true>(u, h, uh);
        recon_pair<B, MU, -SF>(acc[p], uh, f, fn);
      }
    }
  }
}

// store lanes j (if sj) and k (if sk) of a pair at one site in the FP16 format of
// SpinorF16::store (scale = max |real or imaginary part|, zero below FLT_MIN)
__device__ __forceinline__ void store_pair(uint4* oj, float* nj, uint4* ok, float* nk, int Vh, const CP (&o)[4][3],
                                           bool sj, bool sk) {
  float mj = 0.f, mk = 0.f;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const CP& z = o[k / 3][k % 3];
    mj = fmaxf(mj, fmaxf(fabsf(z.re.x), fabsf(z.im.x)));
    mk = fmaxf(mk, fmaxf(fabsf(z.re.y), fabsf(z.im.y)));
  }
  if (!(mj >= 1.17549435e-38f)) mj = 0.f;
  if (!(mk >= 1.17549435e-38f)) mk = 0.f;
  const float2 inv = make_float2(mj > 0.f ? 1.f / mj : 0.f, mk > 0.f ? 1.f / mk : 0.f);
  uint32_t wj[12], wk[12];
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const CP& z = o[k / 3][k % 3];
    const float2 re = mul2(z.re, inv), im = mul2(z.im, inv);
    __half2 a = __floats2half2_rn(re.x, im.x), b = __floats2half2_rn(re.y, im.y);
    wj[k] = *reinterpret_cast<uint32_t*>(&a);
    wk[k] = *reinterpret_cast<uint32_t*>(&b);
  }
  if (sj) {
#pragma unroll
    for (int q = 0; q < 3; q++) oj[(size_t)q * Vh] = make_uint4(wj[4 * q], wj[4 * q + 1], wj[4 * q + 2], wj[4 * q + 3]);
    *nj = mj;
  }
  if (sk) {
#pragma unroll
    for (int q = 0; q < 3; q++) ok[(size_t)q * Vh] = make_uint4(wk[4 * q], wk[4 * q + 1], wk[4 * q + 2], wk[4 * q + 3]);
    *nk = mk;
  }
}

// the scaled components of an FP16 pair (epilogue operand)
__device__ __forceinline__ void load_pair(const uint4* bj, const float* nj, const uint4* bk, const float* nk, int Vh,
                                          CP (&v)[4][3]) {
  load_pair_raw(bj, bk, Vh, v);
  const float2 n = make_float2(__ldg(nj), __ldg(nk));
#pragma unroll
  for (int k = 0; k < 12; k++) {
    CP& z = v[k / 3][k % 3];
    z.re = mul2(z.re, n);
    z.im = mul2(z.im, n);
  }
}

template <int NT, int NP, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT) hop_pair_kernel(HopArgs<SpinorF16, GaugeF16x12> A) {
  constexpr int NR = 2 * NP;
  const int ngrp = (A.nrhs + NR - 1) / NR;
  const int grp = blockIdx.x % ngrp;
  const int blk = blockIdx.x / ngrp;
  const int r0 = grp * NR;
  bool act[NR];
  bool any = false;
#pragma unroll
  for (int j = 0; j < NR; j++) {
    act[j] = (r0 + j < A.nrhs) && (!A.active || A.active[r0 + j]);
    any = any || act[j];
  }
  if (!any) {
    if (A.norm_part && threadIdx.x < NR && r0 + (int)threadIdx.x < A.nrhs)
      A.norm_part[(size_t)(r0 + threadIdx.x) * A.nblk + blk] = 0.0;
    return;
  }
  const int par = A.out_parity;
  const int cb = blk * NT + threadIdx.x;
  double nrm[NR];
#pragma unroll
  for (int j = 0; j < NR; j++) nrm[j] = 0.0;
  if (cb < A.g.Vh) {
    const int Vh = A.g.Vh;
    int x[4];
    cb_coords(A.g, cb, par, x);
    const int L0 = A.g.L[0], L01 = L0 * A.g.L[1], L012 = L01 * A.g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    // each lane's right-hand side; an inactive lane takes its partner's
    bool pact[NP];
    int rr[NR];
#pragma unroll
    for (int p = 0; p < NP; p++) {
      const int j = 2 * p;
      pact[p] = act[j] || act[j + 1];
      rr[j] = act[j] ? r0 + j : r0 + j + 1;
      rr[j + 1] = act[j + 1] ? r0 + j + 1 : r0 + j;
    }
    const uint4* pin[NR];
    const float* nin[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) {
      const SpinorF16 t = A.in.shift(rr[j]);
      pin[j] = par ? t.p0 : t.p1;  // neighbours have the other parity
      nin[j] = par ? t.n0 : t.n1;
    }
    CP acc[NP][4][3];
#pragma unroll
    for (int p = 0; p < NP; p++)
#pragma unroll
      for (int k = 0; k < 12; k++) acc[p][k / 3][k % 3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    hop_dir_pair<NP, B, DAG, 0>(pin, nin, A.gauge, A.g, par, cb, x, s, 1, pact, acc);
    hop_dir_pair<NP, B, DAG, 1>(pin, nin, A.gauge, A.g, par, cb, x, s, L0, pact, acc);
    hop_dir_pair<NP, B, DAG, 2>(pin, nin, A.gauge, A.g, par, cb, x, s, L01, pact, acc);
    hop_dir_pair<NP, B, DAG, 3>(pin, nin, A.gauge, A.g, par, cb, x, s, L012, pact, acc);

    const float2 a2 = bc2(float(A.a));
#pragma unroll
    for (int p = 0; p < NP; p++) {
      if (!pact[p]) continue;
      const int j = 2 * p, rj = rr[j], rk = rr[j + 1];
      const float2 c2 = make_float2(float(A.c * (A.cvec ? A.cvec[rj] : 1.0)), float(A.c * (A.cvec ? A.cvec[rk] : 1.0)));
      const float2 s2 = make_float2(float(A.s * (A.svec ? A.svec[rj] : 1.0)), float(A.s * (A.svec ? A.svec[rk] : 1.0)));
      CP o[4][3];
      if constexpr (EPI == EPI_PLAIN) {
#pragma unroll
        for (int k = 0; k < 12; k++) o[k / 3][k % 3] = acc[p][k / 3][k % 3];
      } else if constexpr (EPI == EPI_XPAY || EPI == EPI_XPAY_G5) {
        // o = a acc + v + i c gamma5 v   (then gamma5 for XPAY_G5)
        const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
        CP v[4][3];
        load_pair((par ? xj.p1 : xj.p0) + cb, (par ? xj.n1 : xj.n0) + cb, (par ? xk.p1 : xk.p0) + cb,
                  (par ? xk.n1 : xk.n0) + cb, Vh, v);
        CP t[4][3];
#pragma unroll
        for (int k = 0; k < 12; k++) {
          const int sp = k / 3, a = k % 3;
          const CP& z = v[g5row<B>(sp)][a];
          const float gs = g5sign<B>(sp);
          const float2 cp = make_float2(gs * c2.x, gs * c2.y), cn = make_float2(-cp.x, -cp.y);
          CP w;
          w.re = fma2(a2, acc[p][sp][a].re, v[sp][a].re);
          w.im = fma2(a2, acc[p][sp][a].im, v[sp][a].im);
          w.re = fma2(cn, z.im, w.re);
          w.im = fma2(cp, z.re, w.im);
          t[sp][a] = w;
        }
#pragma unroll
        for (int k = 0; k < 12; k++) {
          const int sp = k / 3, a = k % 3;
          if constexpr (EPI == EPI_XPAY_G5) {
            const CP& z = t[g5row<B>(sp)][a];
            if (g5sign<B>(sp) > 0.f) o[sp][a] = z;
            else o[sp][a] = {mul2(bc2(-1.f), z.re), mul2(bc2(-1.f), z.im)};
          } else {
            o[sp][a] = t[sp][a];
          }
        }
      } else {
        // EPI_TWIST_INV: o = s (v - i c gamma5 v), v = acc
        // EPI_XPAY_TWINV: the same with v = a acc + x
        CP v[4][3];
        if constexpr (EPI == EPI_XPAY_TWINV) {
          const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
          load_pair((par ? xj.p1 : xj.p0) + cb, (par ? xj.n1 : xj.n0) + cb, (par ? xk.p1 : xk.p0) + cb,
                    (par ? xk.n1 : xk.n0) + cb, Vh, v);
#pragma unroll
          for (int k = 0; k < 12; k++) {
            CP& z = v[k / 3][k % 3];
            z.re = fma2(a2, acc[p][k / 3][k % 3].re, z.re);
            z.im = fma2(a2, acc[p][k / 3][k % 3].im, z.im);
          }
        } else {
#pragma unroll
          for (int k = 0; k < 12; k++) v[k / 3][k % 3] = acc[p][k / 3][k % 3];
        }
        const float2 cs = mul2(c2, s2);
#pragma unroll
        for (int k = 0; k < 12; k++) {
          const int sp = k / 3, a = k % 3;
          const CP& z = v[g5row<B>(sp)][a];
          const float gs = g5sign<B>(sp);
          const float2 cp = make_float2(gs * cs.x, gs * cs.y), cn = make_float2(-cp.x, -cp.y);
          o[sp][a].re = fma2(cp, z.im, mul2(s2, v[sp][a].re));
          o[sp][a].im = fma2(cn, z.re, mul2(s2, v[sp][a].im));
        }
      }
      const SpinorF16 oj = A.out.shift(rj), ok = A.out.shift(rk);
      store_pair((par ? oj.p1 : oj.p0) + cb, (par ? oj.n1 : oj.n0) + cb, (par ? ok.p1 : ok.p0) + cb,
                 (par ? ok.n1 : ok.n0) + cb, Vh, o, act[j], act[j + 1]);
      if (A.norm_part) {
        float2 n2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 0; k < 12; k++) {
          n2 = fma2(o[k / 3][k % 3].re, o[k / 3][k % 3].re, n2);
          n2 = fma2(o[k / 3][k % 3].im, o[k / 3][k % 3].im, n2);
        }
        nrm[j] = act[j] ? double(n2.x) : 0.0;
        nrm[j + 1] = act[j + 1] ? double(n2.y) : 0.0;
      }
    }
  }
  if (A.norm_part) block_partials<NR, NT>(nrm, A.norm_part, A.nblk, r0, A.nrhs, blk);
}

}  // namespace qkx
