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

#include <type_traits>

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

// EPI_XPAY_G5_CGR: the pair's output o = A p is not stored; the CG residual of each
// stored lane takes it, r -= alpha o (FP32 batch racc32), and |r|^2 is summed in FP64
__device__ __forceinline__ void pair_cg_update(const HopArgs<SpinorF16, GaugeF16x12>& A, int par, int cb, int rj,
                                               int rk, bool sj, bool sk, const CP (&o)[4][3], double& nrj,
                                               double& nrk) {
#pragma unroll
  for (int lane = 0; lane < 2; lane++) {
    const bool on = lane ? sk : sj;
    if (!on) continue;
    const int r = lane ? rk : rj;
    const float al = float(A.alpha[r]);
    const SpinorF32 rr = A.racc32.shift(r);
    Spinor<float> v = rr.load(par, cb);
    double n = 0.0;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      Cx<float>& q = v.c[k / 3][k % 3];
      const CP& z = o[k / 3][k % 3];
      q.re = fmaf(-al, lane ? z.re.y : z.re.x, q.re);
      q.im = fmaf(-al, lane ? z.im.y : z.im.x, q.im);
      n += double(q.re) * double(q.re) + double(q.im) * double(q.im);
    }
    rr.store(par, cb, v);
    if (lane) nrk = n;
    else nrj = n;
  }
}

template <int NT, int NP, int B, bool DAG, int EPI, int MINB = 1>
__global__ void __launch_bounds__(NT, MINB) hop_pair_kernel(HopArgs<SpinorF16, GaugeF16x12> A) {
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
      } else if constexpr (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_CGR) {
        // o = a acc + v + i c gamma5 v   (then gamma5 for XPAY_G5 / XPAY_G5_CGR)
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
          if constexpr (EPI != EPI_XPAY) {
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
      if constexpr (EPI == EPI_XPAY_G5_CGR) {
        pair_cg_update(A, par, cb, rj, rk, act[j], act[j + 1], o, nrm[j], nrm[j + 1]);
        continue;
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

namespace qkx {

// ---------------------------------------------------------------- software-pipelined variant
// One pair of right-hand sides per thread.  The eight neighbour terms are
// processed as a pipeline of depth two: the loads of term D+1 (both spinors,
// their scales and the link, as raw FP16 words) are issued before term D is
// converted and computed, so every thread keeps one term's loads in flight
// behind its arithmetic.  MINB is the launch-bounds occupancy hint (0: none).

struct NbRaw {
  uint4 a[3], b[3];  // stored words of lanes j and k
  float na, nb;      // their site scales
  uint4 la;          // link, complex 0..3
  uint2 lb;          // link, complex 4..5
};

struct PairPtrs {
  const uint4* pj;
  const uint4* pk;
  const float* nj;
  const float* nk;
};

// term D: direction MU = D / 2, forward (D even) or backward (D odd)
template <int D>
__device__ __forceinline__ void nb_fetch(NbRaw& r, const PairPtrs& P, const GaugeF16x12& G, const Geom& g, int par,
                                         int cb, const int x[4], int s, int stride) {
  constexpr int MU = D >> 1;
  const int Lm = g.L[MU];
  int n, o;
  if constexpr ((D & 1) == 0) {
    n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    o = (par * 4 + MU) * g.Vh + cb;
  } else {
    n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    o = ((1 - par) * 4 + MU) * g.Vh + n;
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    r.a[q] = __ldg(P.pj + n + (size_t)q * g.Vh);
    r.b[q] = __ldg(P.pk + n + (size_t)q * g.Vh);
  }
  r.na = __ldg(P.nj + n);
  r.nb = __ldg(P.nk + n);
  r.la = __ldg(G.a + o);
  r.lb = __ldg(G.b + o);
}

template <int B, bool DAG, int D>
__device__ __forceinline__ void nb_compute(const NbRaw& r, const Geom& g, const int x[4], CP (&acc)[4][3]) {
  constexpr int MU = D >> 1;
  constexpr bool BWD = (D & 1) != 0;
  constexpr int SF = DAG ? +1 : -1;
  constexpr int SG = BWD ? -SF : SF;  // projector 1 + SG*g
  const bool flip = (MU == 3) && g.bc_sign < 0 && x[3] == (BWD ? 0 : g.L[3] - 1);
  const float sg = (flip ? -1.f : 1.f) * (Proj<B, MU, SG>::diag ? 2.f : 1.f);
  Link<float> u;
  {
    const uint32_t ws[6] = {r.la.x, r.la.y, r.la.z, r.la.w, r.lb.x, r.lb.y};
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&ws[k]));
      u.m[k / 3][k % 3] = {f.x, f.y};
    }
    rebuild_row2(u);
  }
  CP v[4][3], h[2][3], uh[2][3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const uint32_t sj[4] = {r.a[q].x, r.a[q].y, r.a[q].z, r.a[q].w};
    const uint32_t sk[4] = {r.b[q].x, r.b[q].y, r.b[q].z, r.b[q].w};
#pragma unroll
    for (int w = 0; w < 4; w++) {
      const __half2 hj = *reinterpret_cast<const __half2*>(&sj[w]);
      const __half2 hk = *reinterpret_cast<const __half2*>(&sk[w]);
      const int k = 4 * q + w;
      v[k / 3][k % 3].re = make_float2(__low2float(hj), __low2float(hk));
      v[k / 3][k % 3].im = make_float2(__high2float(hj), __high2float(hk));
    }
  }
  const float2 f = make_float2(sg * r.na, sg * r.nb);
  const float2 fn = make_float2(-f.x, -f.y);
  proj_pair<B, MU, SG>(v, h);
  mul_link_pair<BWD>(u, h, uh);
  recon_pair<B, MU, SG>(acc, uh, f, fn);
}

// the epilogue of hop_pair_kernel for one pair, from its accumulated hopping term
// (XPRE: the epilogue operand x of the pair is already in xpre, scaled)
template <int B, int EPI, bool XPRE = false>
__device__ __forceinline__ void pair_epilogue(const HopArgs<SpinorF16, GaugeF16x12>& A, int par, int cb, int rj,
                                              int rk, bool sj, bool sk, const CP (&acc)[4][3], double& nrj,
                                              double& nrk, const CP (*xpre)[3] = nullptr) {
  const int Vh = A.g.Vh;
  const float2 a2 = bc2(float(A.a));
  const float2 c2 = make_float2(float(A.c * (A.cvec ? A.cvec[rj] : 1.0)), float(A.c * (A.cvec ? A.cvec[rk] : 1.0)));
  const float2 s2 = make_float2(float(A.s * (A.svec ? A.svec[rj] : 1.0)), float(A.s * (A.svec ? A.svec[rk] : 1.0)));
  CP o[4][3];
  if constexpr (EPI == EPI_PLAIN) {
#pragma unroll
    for (int k = 0; k < 12; k++) o[k / 3][k % 3] = acc[k / 3][k % 3];
  } else if constexpr (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_CGR) {
    CP v[4][3];
    if constexpr (XPRE) {
#pragma unroll
      for (int k = 0; k < 12; k++) v[k / 3][k % 3] = xpre[k / 3][k % 3];
    } else {
      const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
      load_pair((par ? xj.p1 : xj.p0) + cb, (par ? xj.n1 : xj.n0) + cb, (par ? xk.p1 : xk.p0) + cb,
                (par ? xk.n1 : xk.n0) + cb, Vh, v);
    }
    CP t[4][3];
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const int sp = k / 3, a = k % 3;
      const CP& z = v[g5row<B>(sp)][a];
      const float gs = g5sign<B>(sp);
      const float2 cp = make_float2(gs * c2.x, gs * c2.y), cn = make_float2(-cp.x, -cp.y);
      CP w;
      w.re = fma2(a2, acc[sp][a].re, v[sp][a].re);
      w.im = fma2(a2, acc[sp][a].im, v[sp][a].im);
      w.re = fma2(cn, z.im, w.re);
      w.im = fma2(cp, z.re, w.im);
      t[sp][a] = w;
    }
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const int sp = k / 3, a = k % 3;
      if constexpr (EPI != EPI_XPAY) {
        const CP& z = t[g5row<B>(sp)][a];
        if (g5sign<B>(sp) > 0.f) o[sp][a] = z;
        else o[sp][a] = {mul2(bc2(-1.f), z.re), mul2(bc2(-1.f), z.im)};
      } else {
        o[sp][a] = t[sp][a];
      }
    }
  } else {
    CP v[4][3];
    if constexpr (EPI == EPI_XPAY_TWINV) {
      if constexpr (XPRE) {
#pragma unroll
        for (int k = 0; k < 12; k++) v[k / 3][k % 3] = xpre[k / 3][k % 3];
      } else {
        const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
        load_pair((par ? xj.p1 : xj.p0) + cb, (par ? xj.n1 : xj.n0) + cb, (par ? xk.p1 : xk.p0) + cb,
                  (par ? xk.n1 : xk.n0) + cb, Vh, v);
      }
#pragma unroll
      for (int k = 0; k < 12; k++) {
        CP& z = v[k / 3][k % 3];
        z.re = fma2(a2, acc[k / 3][k % 3].re, z.re);
        z.im = fma2(a2, acc[k / 3][k % 3].im, z.im);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 12; k++) v[k / 3][k % 3] = acc[k / 3][k % 3];
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
  if constexpr (EPI == EPI_XPAY_G5_CGR) {
    pair_cg_update(A, par, cb, rj, rk, sj, sk, o, nrj, nrk);
    return;
  }
  const SpinorF16 oj = A.out.shift(rj), ok = A.out.shift(rk);
  store_pair((par ? oj.p1 : oj.p0) + cb, (par ? oj.n1 : oj.n0) + cb, (par ? ok.p1 : ok.p0) + cb,
             (par ? ok.n1 : ok.n0) + cb, Vh, o, sj, sk);
  if (A.norm_part) {
    float2 n2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      n2 = fma2(o[k / 3][k % 3].re, o[k / 3][k % 3].re, n2);
      n2 = fma2(o[k / 3][k % 3].im, o[k / 3][k % 3].im, n2);
    }
    nrj = sj ? double(n2.x) : 0.0;
    nrk = sk ? double(n2.y) : 0.0;
  }
}

template <int NT, int MINB, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT, MINB > 0 ? MINB : 1) hop_pair_pf_kernel(HopArgs<SpinorF16, GaugeF16x12> A) {
  const int ngrp = (A.nrhs + 1) / 2;
  const int grp = blockIdx.x % ngrp;
  const int blk = blockIdx.x / ngrp;
  const int r0 = grp * 2;
  const bool actj = (r0 < A.nrhs) && (!A.active || A.active[r0]);
  const bool actk = (r0 + 1 < A.nrhs) && (!A.active || A.active[r0 + 1]);
  if (!actj && !actk) {
    if (A.norm_part && threadIdx.x < 2 && r0 + (int)threadIdx.x < A.nrhs)
      A.norm_part[(size_t)(r0 + threadIdx.x) * A.nblk + blk] = 0.0;
    return;
  }
  const int par = A.out_parity;
  const int cb = blk * NT + threadIdx.x;
  double nrm[2] = {0.0, 0.0};
  if (cb < A.g.Vh) {
    int x[4];
    cb_coords(A.g, cb, par, x);
    const int L0 = A.g.L[0], L01 = L0 * A.g.L[1], L012 = L01 * A.g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    const int rj = actj ? r0 : r0 + 1, rk = actk ? r0 + 1 : r0;
    PairPtrs P;
    {
      const SpinorF16 tj = A.in.shift(rj), tk = A.in.shift(rk);
      P.pj = par ? tj.p0 : tj.p1;  // neighbours have the other parity
      P.pk = par ? tk.p0 : tk.p1;
      P.nj = par ? tj.n0 : tj.n1;
      P.nk = par ? tk.n0 : tk.n1;
    }
    CP acc[4][3];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k / 3][k % 3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    NbRaw r0b, r1b;
    nb_fetch<0>(r0b, P, A.gauge, A.g, par, cb, x, s, 1);
    nb_fetch<1>(r1b, P, A.gauge, A.g, par, cb, x, s, 1);
    nb_compute<B, DAG, 0>(r0b, A.g, x, acc);
    nb_fetch<2>(r0b, P, A.gauge, A.g, par, cb, x, s, L0);
    nb_compute<B, DAG, 1>(r1b, A.g, x, acc);
    nb_fetch<3>(r1b, P, A.gauge, A.g, par, cb, x, s, L0);
    nb_compute<B, DAG, 2>(r0b, A.g, x, acc);
    nb_fetch<4>(r0b, P, A.gauge, A.g, par, cb, x, s, L01);
    nb_compute<B, DAG, 3>(r1b, A.g, x, acc);
    nb_fetch<5>(r1b, P, A.gauge, A.g, par, cb, x, s, L01);
    nb_compute<B, DAG, 4>(r0b, A.g, x, acc);
    nb_fetch<6>(r0b, P, A.gauge, A.g, par, cb, x, s, L012);
    nb_compute<B, DAG, 5>(r1b, A.g, x, acc);
    nb_fetch<7>(r1b, P, A.gauge, A.g, par, cb, x, s, L012);
    nb_compute<B, DAG, 6>(r0b, A.g, x, acc);
    nb_compute<B, DAG, 7>(r1b, A.g, x, acc);
    pair_epilogue<B, EPI>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1]);
  }
  if (A.norm_part) block_partials<2, NT>(nrm, A.norm_part, A.nblk, r0, A.nrhs, blk);
}


// ---------------------------------------------------------------- shared-memory pipelined variant
// As hop_pair_pf_kernel, but each thread stages its next S-1 terms in shared
// memory with cp.async (16/8/4-byte copies, L1-allocating) instead of holding
// them in registers: term i goes to slot i % S of the thread's own column of
// the block's stage buffers, and item 8 is the epilogue operand x.  Only the
// issuing thread reads a slot, after its own cp.async.wait_group, so no
// block-level barrier is needed; the asm statements carry a memory clobber so
// the compiler keeps each slot's shared-memory reads before the copy that
// refills it.

__device__ __forceinline__ void cpa16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa8(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa4(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// one slot for every thread of the block: [word][thread], so a warp's copies and
// reads of one word are 32 consecutive 16-byte (8-, 4-byte) elements
template <int NT>
struct PairSlot {
  uint4 sp[6][NT];  // lanes j (words 0..2) and k (words 3..5)
  float nm[2][NT];
  uint4 la[NT];
  uint2 lb[NT];
};

template <int D, int NT>
__device__ __forceinline__ void nb_issue(PairSlot<NT>& st, int tid, const PairPtrs& P, const GaugeF16x12& G,
                                         const Geom& g, int par, int cb, const int x[4], int s, int stride) {
  constexpr int MU = D >> 1;
  const int Lm = g.L[MU];
  int n, o;
  if constexpr ((D & 1) == 0) {
    n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    o = (par * 4 + MU) * g.Vh + cb;
  } else {
    n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    o = ((1 - par) * 4 + MU) * g.Vh + n;
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    cpa16(&st.sp[q][tid], P.pj + n + (size_t)q * g.Vh);
    cpa16(&st.sp[3 + q][tid], P.pk + n + (size_t)q * g.Vh);
  }
  cpa4(&st.nm[0][tid], P.nj + n);
  cpa4(&st.nm[1][tid], P.nk + n);
  cpa16(&st.la[tid], G.a + o);
  cpa8(&st.lb[tid], G.b + o);
}

template <int NT>
__device__ __forceinline__ void slot_read(const PairSlot<NT>& st, int tid, NbRaw& r) {
#pragma unroll
  for (int q = 0; q < 3; q++) {
    r.a[q] = st.sp[q][tid];
    r.b[q] = st.sp[3 + q][tid];
  }
  r.na = st.nm[0][tid];
  r.nb = st.nm[1][tid];
  r.la = st.la[tid];
  r.lb = st.lb[tid];
}

template <int NT, int S, int MINB, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT, MINB > 0 ? MINB : 1) hop_pair_as_kernel(HopArgs<SpinorF16, GaugeF16x12> A) {
  static_assert(S == 2 || S == 3, "pipeline depth");
  __shared__ PairSlot<NT> st[S];
  const int ngrp = (A.nrhs + 1) / 2;
  const int grp = blockIdx.x % ngrp;
  const int blk = blockIdx.x / ngrp;
  const int r0 = grp * 2;
  const int tid = threadIdx.x;
  const bool actj = (r0 < A.nrhs) && (!A.active || A.active[r0]);
  const bool actk = (r0 + 1 < A.nrhs) && (!A.active || A.active[r0 + 1]);
  if (!actj && !actk) {
    if (A.norm_part && tid < 2 && r0 + tid < A.nrhs) A.norm_part[(size_t)(r0 + tid) * A.nblk + blk] = 0.0;
    return;
  }
  constexpr bool XOP = (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_CGR || EPI == EPI_XPAY_TWINV);
  const int par = A.out_parity;
  const int cb = blk * NT + tid;
  double nrm[2] = {0.0, 0.0};
  if (cb < A.g.Vh) {
    const Geom& g = A.g;
    int x[4];
    cb_coords(g, cb, par, x);
    const int L0 = g.L[0], L01 = L0 * g.L[1], L012 = L01 * g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    const int rj = actj ? r0 : r0 + 1, rk = actk ? r0 + 1 : r0;
    PairPtrs P;
    {
      const SpinorF16 tj = A.in.shift(rj), tk = A.in.shift(rk);
      P.pj = par ? tj.p0 : tj.p1;  // neighbours have the other parity
      P.pk = par ? tk.p0 : tk.p1;
      P.nj = par ? tj.n0 : tj.n1;
      P.nk = par ? tk.n0 : tk.n1;
    }
    const int strd[4] = {1, L0, L01, L012};
    // item i < 8: neighbour term i into slot i % S; item 8: the epilogue operand
    auto issue = [&](auto ic) {
      constexpr int I = decltype(ic)::value;
      if constexpr (I < 8) {
        nb_issue<I, NT>(st[I % S], tid, P, A.gauge, g, par, cb, x, s, strd[I >> 1]);
      } else if constexpr (XOP) {
        const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
        PairSlot<NT>& t = st[8 % S];
        const uint4* bj = (par ? xj.p1 : xj.p0) + cb;
        const uint4* bk = (par ? xk.p1 : xk.p0) + cb;
#pragma unroll
        for (int q = 0; q < 3; q++) {
          cpa16(&t.sp[q][tid], bj + (size_t)q * g.Vh);
          cpa16(&t.sp[3 + q][tid], bk + (size_t)q * g.Vh);
        }
        cpa4(&t.nm[0][tid], (par ? xj.n1 : xj.n0) + cb);
        cpa4(&t.nm[1][tid], (par ? xk.n1 : xk.n0) + cb);
      }
      cpa_commit();
    };
    issue(std::integral_constant<int, 0>{});
    issue(std::integral_constant<int, 1>{});
    if constexpr (S == 3) issue(std::integral_constant<int, 2>{});
    CP acc[4][3];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k / 3][k % 3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    auto step = [&](auto dc) {
      constexpr int D = decltype(dc)::value;
      cpa_wait<S - 1>();
      NbRaw r;
      slot_read(st[D % S], tid, r);
      nb_compute<B, DAG, D>(r, g, x, acc);
      if constexpr (D + S <= 8) issue(std::integral_constant<int, D + S>{});
      else cpa_commit();
    };
    step(std::integral_constant<int, 0>{});
    step(std::integral_constant<int, 1>{});
    step(std::integral_constant<int, 2>{});
    step(std::integral_constant<int, 3>{});
    step(std::integral_constant<int, 4>{});
    step(std::integral_constant<int, 5>{});
    step(std::integral_constant<int, 6>{});
    step(std::integral_constant<int, 7>{});
    cpa_wait<0>();
    if constexpr (XOP) {
      const PairSlot<NT>& t = st[8 % S];
      CP xv[4][3];
      const float2 n = make_float2(t.nm[0][tid], t.nm[1][tid]);
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const uint4 wj = t.sp[q][tid], wk = t.sp[3 + q][tid];
        const uint32_t sj[4] = {wj.x, wj.y, wj.z, wj.w}, sk[4] = {wk.x, wk.y, wk.z, wk.w};
#pragma unroll
        for (int w = 0; w < 4; w++) {
          const __half2 hj = *reinterpret_cast<const __half2*>(&sj[w]);
          const __half2 hk = *reinterpret_cast<const __half2*>(&sk[w]);
          const int k = 4 * q + w;
          xv[k / 3][k % 3].re = mul2(make_float2(__low2float(hj), __low2float(hk)), n);
          xv[k / 3][k % 3].im = mul2(make_float2(__high2float(hj), __high2float(hk)), n);
        }
      }
      pair_epilogue<B, EPI, true>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1], xv);
    } else {
      pair_epilogue<B, EPI>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1]);
    }
  }
  if (A.norm_part) block_partials<2, NT>(nrm, A.norm_part, A.nblk, r0, A.nrhs, blk);
}


// ---------------------------------------------------------------- half2 projection variants
// The spin projection h = s_a +- (i) s_b of each right-hand side is formed in
// FP16 on the stored half2 words (one add or fma with a +-1 multiplier and the
// real/imaginary halves swapped for +-i: one rounding of a sum of two
// site-normalised values, the size of the storage rounding), and only the six
// projected complex numbers are widened, so a term converts 12 halves a
// right-hand side instead of 24.  The link format LK: 0 the 12-real FP16 links
// (row 2 rebuilt, boundary sign from the t coordinate); 1 the operator's own 18
// reals in FP32 (boundary sign included): no conversion, no third-row rebuild;
// 2 the 18 reals in FP16 (boundary sign included): nine conversions, no rebuild.

// a + phase<PH>(z) on one (re, im) half2
template <int PH>
__device__ __forceinline__ __half2 addph_h(__half2 a, __half2 z) {
  if constexpr ((PH & 3) == 0) return __hadd2(a, z);
  else if constexpr ((PH & 3) == 2) return __hsub2(a, z);
  else if constexpr ((PH & 3) == 1) return __hfma2(__lowhigh2highlow(z), __floats2half2_rn(-1.f, 1.f), a);
  else return __hfma2(__lowhigh2highlow(z), __floats2half2_rn(1.f, -1.f), a);
}

template <int B, int MU, int SIGN>
__device__ __forceinline__ void proj_h(const uint32_t (&w)[12], __half2 (&h)[2][3]) {
  using PJ = Proj<B, MU, SIGN>;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const __half2 s0 = *reinterpret_cast<const __half2*>(&w[a]);
    const __half2 s1 = *reinterpret_cast<const __half2*>(&w[3 + a]);
    if constexpr (PJ::diag) {
      h[0][a] = *reinterpret_cast<const __half2*>(&w[PJ::drow * 3 + a]);
      h[1][a] = *reinterpret_cast<const __half2*>(&w[(PJ::drow + 1) * 3 + a]);
    } else {
      h[0][a] = addph_h<PJ::p0>(s0, *reinterpret_cast<const __half2*>(&w[PJ::c0 * 3 + a]));
      h[1][a] = addph_h<PJ::p1>(s1, *reinterpret_cast<const __half2*>(&w[PJ::c1 * 3 + a]));
    }
  }
}

template <int NT, int LK>
struct HSlot {
  uint4 sp[6][NT];
  float nm[2][NT];
  uint4 la[LK == 1 ? 4 : (LK == 2 ? 2 : 1)][NT];
  uint2 lb[LK == 2 ? 1 : NT];      // FP16 complex 4..5 (LK 0), or the FP32 complex 8 (LK 1)
  uint32_t lc[LK == 2 ? NT : 1];   // the FP16 complex 8 (LK 2)
};

// the links of a variant, as raw words:
//   LK 0: FP16 12-real as GaugeF16x12, [parity*4+mu][Vh] uint4 of complex 0..3 (a)
//         and uint2 of complex 4..5 (b);
//   LK 1: FP32 18-real with the boundary sign, [parity*4+mu][4][Vh] float4 of
//         complex 0..7 (a) and [parity*4+mu][Vh] float2 of complex 8 (b);
//   LK 2: FP16 18-real with the boundary sign, [parity*4+mu][Vh] uint4 of complex
//         0..3 (a), uint4 of complex 4..7 (a2) and uint32 of complex 8 (c).
template <int LK>
struct HLinks {
  const uint4* a;
  const uint2* b;
  const uint4* a2 = nullptr;
  const uint32_t* c = nullptr;
};

template <int D, int NT, int LK>
__device__ __forceinline__ void nb_issue_h(HSlot<NT, LK>& st, int tid, const PairPtrs& P, const HLinks<LK>& G,
                                           const Geom& g, int par, int cb, const int x[4], int s, int stride) {
  constexpr int MU = D >> 1;
  const int Lm = g.L[MU];
  int n, pm, li;  // neighbour; the link's (parity*4 + mu) and site
  if constexpr ((D & 1) == 0) {
    n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    pm = par * 4 + MU;
    li = cb;
  } else {
    n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    pm = (1 - par) * 4 + MU;
    li = n;
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    cpa16(&st.sp[q][tid], P.pj + n + (size_t)q * g.Vh);
    cpa16(&st.sp[3 + q][tid], P.pk + n + (size_t)q * g.Vh);
  }
  cpa4(&st.nm[0][tid], P.nj + n);
  cpa4(&st.nm[1][tid], P.nk + n);
  if constexpr (LK == 1) {
#pragma unroll
    for (int q = 0; q < 4; q++) cpa16(&st.la[q][tid], G.a + (size_t)(pm * 4 + q) * g.Vh + li);
    cpa8(&st.lb[tid], G.b + (size_t)pm * g.Vh + li);
  } else if constexpr (LK == 2) {
    cpa16(&st.la[0][tid], G.a + (size_t)pm * g.Vh + li);
    cpa16(&st.la[1][tid], G.a2 + (size_t)pm * g.Vh + li);
    cpa4(&st.lc[tid], G.c + (size_t)pm * g.Vh + li);
  } else {
    cpa16(&st.la[0][tid], G.a + (size_t)pm * g.Vh + li);
    cpa8(&st.lb[tid], G.b + (size_t)pm * g.Vh + li);
  }
}

template <int B, bool DAG, int D, int NT, int LK>
__device__ __forceinline__ void nb_compute_h(const HSlot<NT, LK>& st, int tid, const Geom& g, const int x[4],
                                             CP (&acc)[4][3]) {
  constexpr int MU = D >> 1;
  constexpr bool BWD = (D & 1) != 0;
  constexpr int SF = DAG ? +1 : -1;
  constexpr int SG = BWD ? -SF : SF;  // projector 1 + SG*g
  bool flip = false;
  if constexpr (LK == 0) flip = (MU == 3) && g.bc_sign < 0 && x[3] == (BWD ? 0 : g.L[3] - 1);
  const float sg = (flip ? -1.f : 1.f) * (Proj<B, MU, SG>::diag ? 2.f : 1.f);
  Link<float> u;
  if constexpr (LK == 1) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint4 w = st.la[q][tid];
      u.m[(2 * q) / 3][(2 * q) % 3] = {__uint_as_float(w.x), __uint_as_float(w.y)};
      u.m[(2 * q + 1) / 3][(2 * q + 1) % 3] = {__uint_as_float(w.z), __uint_as_float(w.w)};
    }
    const uint2 w = st.lb[tid];
    u.m[2][2] = {__uint_as_float(w.x), __uint_as_float(w.y)};
  } else if constexpr (LK == 2) {
    const uint4 w0 = st.la[0][tid], w1 = st.la[1][tid];
    const uint32_t ws[9] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w, st.lc[tid]};
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&ws[k]));
      u.m[k / 3][k % 3] = {f.x, f.y};
    }
  } else {
    const uint4 w0 = st.la[0][tid];
    const uint2 w1 = st.lb[tid];
    const uint32_t ws[6] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y};
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&ws[k]));
      u.m[k / 3][k % 3] = {f.x, f.y};
    }
    rebuild_row2(u);
  }
  __half2 hj[2][3], hk[2][3];
  {
    uint32_t wj[12], wk[12];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const uint4 a = st.sp[q][tid], b = st.sp[3 + q][tid];
      wj[4 * q] = a.x; wj[4 * q + 1] = a.y; wj[4 * q + 2] = a.z; wj[4 * q + 3] = a.w;
      wk[4 * q] = b.x; wk[4 * q + 1] = b.y; wk[4 * q + 2] = b.z; wk[4 * q + 3] = b.w;
    }
    proj_h<B, MU, SG>(wj, hj);
    proj_h<B, MU, SG>(wk, hk);
  }
  CP h[2][3], uh[2][3];
#pragma unroll
  for (int sp = 0; sp < 2; sp++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      h[sp][a].re = make_float2(__low2float(hj[sp][a]), __low2float(hk[sp][a]));
      h[sp][a].im = make_float2(__high2float(hj[sp][a]), __high2float(hk[sp][a]));
    }
  const float2 f = make_float2(sg * st.nm[0][tid], sg * st.nm[1][tid]);
  const float2 fn = make_float2(-f.x, -f.y);
  mul_link_pair<BWD>(u, h, uh);
  recon_pair<B, MU, SG>(acc, uh, f, fn);
}

template <int NT, int S, int MINB, int LK, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT, MINB > 0 ? MINB : 1)
    hop_pair_hp_kernel(HopArgs<SpinorF16, GaugeF16x12> A, HLinks<LK> G) {
  static_assert(S == 2 || S == 3, "pipeline depth");
  __shared__ HSlot<NT, LK> st[S];
  const int ngrp = (A.nrhs + 1) / 2;
  const int grp = blockIdx.x % ngrp;
  const int blk = blockIdx.x / ngrp;
  const int r0 = grp * 2;
  const int tid = threadIdx.x;
  const bool actj = (r0 < A.nrhs) && (!A.active || A.active[r0]);
  const bool actk = (r0 + 1 < A.nrhs) && (!A.active || A.active[r0 + 1]);
  if (!actj && !actk) {
    if (A.norm_part && tid < 2 && r0 + tid < A.nrhs) A.norm_part[(size_t)(r0 + tid) * A.nblk + blk] = 0.0;
    return;
  }
  constexpr bool XOP = (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_CGR || EPI == EPI_XPAY_TWINV);
  const int par = A.out_parity;
  const int cb = blk * NT + tid;
  double nrm[2] = {0.0, 0.0};
  if (cb < A.g.Vh) {
    const Geom& g = A.g;
    int x[4];
    cb_coords(g, cb, par, x);
    const int L0 = g.L[0], L01 = L0 * g.L[1], L012 = L01 * g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    const int rj = actj ? r0 : r0 + 1, rk = actk ? r0 + 1 : r0;
    PairPtrs P;
    {
      const SpinorF16 tj = A.in.shift(rj), tk = A.in.shift(rk);
      P.pj = par ? tj.p0 : tj.p1;  // neighbours have the other parity
      P.pk = par ? tk.p0 : tk.p1;
      P.nj = par ? tj.n0 : tj.n1;
      P.nk = par ? tk.n0 : tk.n1;
    }
    const int strd[4] = {1, L0, L01, L012};
    auto issue = [&](auto ic) {
      constexpr int I = decltype(ic)::value;
      if constexpr (I < 8) {
        nb_issue_h<I, NT, LK>(st[I % S], tid, P, G, g, par, cb, x, s, strd[I >> 1]);
      } else if constexpr (XOP) {
        const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
        HSlot<NT, LK>& t = st[8 % S];
        const uint4* bj = (par ? xj.p1 : xj.p0) + cb;
        const uint4* bk = (par ? xk.p1 : xk.p0) + cb;
#pragma unroll
        for (int q = 0; q < 3; q++) {
          cpa16(&t.sp[q][tid], bj + (size_t)q * g.Vh);
          cpa16(&t.sp[3 + q][tid], bk + (size_t)q * g.Vh);
        }
        cpa4(&t.nm[0][tid], (par ? xj.n1 : xj.n0) + cb);
        cpa4(&t.nm[1][tid], (par ? xk.n1 : xk.n0) + cb);
      }
      cpa_commit();
    };
    issue(std::integral_constant<int, 0>{});
    issue(std::integral_constant<int, 1>{});
    if constexpr (S == 3) issue(std::integral_constant<int, 2>{});
    CP acc[4][3];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k / 3][k % 3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    auto step = [&](auto dc) {
      constexpr int D = decltype(dc)::value;
      cpa_wait<S - 1>();
      nb_compute_h<B, DAG, D, NT, LK>(st[D % S], tid, g, x, acc);
      if constexpr (D + S <= 8) issue(std::integral_constant<int, D + S>{});
      else cpa_commit();
    };
    step(std::integral_constant<int, 0>{});
    step(std::integral_constant<int, 1>{});
    step(std::integral_constant<int, 2>{});
    step(std::integral_constant<int, 3>{});
    step(std::integral_constant<int, 4>{});
    step(std::integral_constant<int, 5>{});
    step(std::integral_constant<int, 6>{});
    step(std::integral_constant<int, 7>{});
    cpa_wait<0>();
    if constexpr (XOP) {
      const HSlot<NT, LK>& t = st[8 % S];
      CP xv[4][3];
      const float2 n = make_float2(t.nm[0][tid], t.nm[1][tid]);
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const uint4 wj = t.sp[q][tid], wk = t.sp[3 + q][tid];
        const uint32_t sj[4] = {wj.x, wj.y, wj.z, wj.w}, sk[4] = {wk.x, wk.y, wk.z, wk.w};
#pragma unroll
        for (int w = 0; w < 4; w++) {
          const __half2 hj = *reinterpret_cast<const __half2*>(&sj[w]);
          const __half2 hk = *reinterpret_cast<const __half2*>(&sk[w]);
          const int k = 4 * q + w;
          xv[k / 3][k % 3].re = mul2(make_float2(__low2float(hj), __low2float(hk)), n);
          xv[k / 3][k % 3].im = mul2(make_float2(__high2float(hj), __high2float(hk)), n);
        }
      }
      pair_epilogue<B, EPI, true>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1], xv);
    } else {
      pair_epilogue<B, EPI>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1]);
    }
  }
  if (A.norm_part) block_partials<2, NT>(nrm, A.norm_part, A.nblk, r0, A.nrhs, blk);
}


// ---------------------------------------------------------------- FP16 link multiply variant
// As hop_pair_hp_kernel (FP16 projection, cp.async staging), with the link
// multiply also done in FP16: the projected rows of both right-hand sides are
// put in lane form (re_j, re_k), (im_j, im_k) as half2 with byte permutes, the
// link entries are broadcast to both lanes from the stored words, and U h or
// U^+ h is 4 HFMA2 per complex multiply-add for the pair.  Only U h is widened
// to FP32; the accumulation over the eight terms, the site scales and the
// epilogue stay FP32.  The links are the operator's 18 reals in FP16 with the
// boundary sign included ([parity*4+mu][Vh] uint4 of complex 0..3, uint4 of
// complex 4..7, uint32 of complex 8), so nothing is rebuilt.  The products
// round to FP16 (2^-11 relative, |U h| <= 6 for site-normalised rows), the
// same order as the storage rounding of the inputs.

struct CPH {
  __half2 re, im;
};

template <int NT>
struct MSlot {
  uint4 sp[6][NT];
  float nm[2][NT];
  uint4 la[2][NT];
  uint32_t lc[NT];
};

struct HLinks18 {
  const uint4* a;
  const uint4* b;
  const uint32_t* c;
};

template <int D, int NT>
__device__ __forceinline__ void nb_issue_m(MSlot<NT>& st, int tid, const PairPtrs& P, const HLinks18& G,
                                           const Geom& g, int par, int cb, const int x[4], int s, int stride) {
  constexpr int MU = D >> 1;
  const int Lm = g.L[MU];
  int n, o;
  if constexpr ((D & 1) == 0) {
    n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    o = (par * 4 + MU) * g.Vh + cb;
  } else {
    n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    o = ((1 - par) * 4 + MU) * g.Vh + n;
  }
#pragma unroll
  for (int q = 0; q < 3; q++) {
    cpa16(&st.sp[q][tid], P.pj + n + (size_t)q * g.Vh);
    cpa16(&st.sp[3 + q][tid], P.pk + n + (size_t)q * g.Vh);
  }
  cpa4(&st.nm[0][tid], P.nj + n);
  cpa4(&st.nm[1][tid], P.nk + n);
  cpa16(&st.la[0][tid], G.a + o);
  cpa16(&st.la[1][tid], G.b + o);
  cpa4(&st.lc[tid], G.c + o);
}

// o = U h (DG false) or U^+ h (DG true) for a pair in half2 lane form; w[k] is
// link entry k = row*3 + column as a (re, im) half2
template <bool DG>
__device__ __forceinline__ void mul_link_h(const uint32_t (&w)[9], const CPH (&h)[2][3], CPH (&o)[2][3]) {
  const __half2 sgn = __floats2half2_rn(-1.f, -1.f);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    __half2 ur[3], ui[3], un[3];
#pragma unroll
    for (int b = 0; b < 3; b++) {
      const __half2 e = *reinterpret_cast<const __half2*>(&w[DG ? b * 3 + a : a * 3 + b]);
      ur[b] = __low2half2(e);
      const __half2 im = __high2half2(e);
      // U: (ur, ui); U^+: (ur, -ui)
      ui[b] = DG ? __hmul2(im, sgn) : im;
      un[b] = DG ? im : __hmul2(im, sgn);
    }
#pragma unroll
    for (int sp = 0; sp < 2; sp++) {
      __half2 re = __hmul2(ur[0], h[sp][0].re), im = __hmul2(ur[0], h[sp][0].im);
      re = __hfma2(un[0], h[sp][0].im, re);
      im = __hfma2(ui[0], h[sp][0].re, im);
#pragma unroll
      for (int b = 1; b < 3; b++) {
        re = __hfma2(ur[b], h[sp][b].re, re);
        im = __hfma2(ur[b], h[sp][b].im, im);
        re = __hfma2(un[b], h[sp][b].im, re);
        im = __hfma2(ui[b], h[sp][b].re, im);
      }
      o[sp][a] = {re, im};
    }
  }
}

template <int B, bool DAG, int D, int NT>
__device__ __forceinline__ void nb_compute_m(const MSlot<NT>& st, int tid, const int x[4], CP (&acc)[4][3]) {
  constexpr int MU = D >> 1;
  constexpr bool BWD = (D & 1) != 0;
  constexpr int SF = DAG ? +1 : -1;
  constexpr int SG = BWD ? -SF : SF;  // projector 1 + SG*g
  constexpr float sg = Proj<B, MU, SG>::diag ? 2.f : 1.f;
  uint32_t lw[9];
  {
    const uint4 a = st.la[0][tid], b = st.la[1][tid];
    lw[0] = a.x; lw[1] = a.y; lw[2] = a.z; lw[3] = a.w;
    lw[4] = b.x; lw[5] = b.y; lw[6] = b.z; lw[7] = b.w;
    lw[8] = st.lc[tid];
  }
  __half2 hj[2][3], hk[2][3];
  {
    uint32_t wj[12], wk[12];
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const uint4 a = st.sp[q][tid], b = st.sp[3 + q][tid];
      wj[4 * q] = a.x; wj[4 * q + 1] = a.y; wj[4 * q + 2] = a.z; wj[4 * q + 3] = a.w;
      wk[4 * q] = b.x; wk[4 * q + 1] = b.y; wk[4 * q + 2] = b.z; wk[4 * q + 3] = b.w;
    }
    proj_h<B, MU, SG>(wj, hj);
    proj_h<B, MU, SG>(wk, hk);
  }
  CPH h[2][3], uh[2][3];
#pragma unroll
  for (int sp = 0; sp < 2; sp++)
#pragma unroll
    for (int a = 0; a < 3; a++) h[sp][a] = {__lows2half2(hj[sp][a], hk[sp][a]), __highs2half2(hj[sp][a], hk[sp][a])};
  mul_link_h<BWD>(lw, h, uh);
  CP u32[2][3];
#pragma unroll
  for (int sp = 0; sp < 2; sp++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      u32[sp][a].re = __half22float2(uh[sp][a].re);
      u32[sp][a].im = __half22float2(uh[sp][a].im);
    }
  const float2 f = make_float2(sg * st.nm[0][tid], sg * st.nm[1][tid]);
  const float2 fn = make_float2(-f.x, -f.y);
  recon_pair<B, MU, SG>(acc, u32, f, fn);
}

template <int NT, int MINB, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT, MINB > 0 ? MINB : 1)
    hop_pair_hm_kernel(HopArgs<SpinorF16, GaugeF16x12> A, HLinks18 G) {
  constexpr int S = 2;
  __shared__ MSlot<NT> st[S];
  const int ngrp = (A.nrhs + 1) / 2;
  const int grp = blockIdx.x % ngrp;
  const int blk = blockIdx.x / ngrp;
  const int r0 = grp * 2;
  const int tid = threadIdx.x;
  const bool actj = (r0 < A.nrhs) && (!A.active || A.active[r0]);
  const bool actk = (r0 + 1 < A.nrhs) && (!A.active || A.active[r0 + 1]);
  if (!actj && !actk) {
    if (A.norm_part && tid < 2 && r0 + tid < A.nrhs) A.norm_part[(size_t)(r0 + tid) * A.nblk + blk] = 0.0;
    return;
  }
  constexpr bool XOP = (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_CGR || EPI == EPI_XPAY_TWINV);
  const int par = A.out_parity;
  const int cb = blk * NT + tid;
  double nrm[2] = {0.0, 0.0};
  if (cb < A.g.Vh) {
    const Geom& g = A.g;
    int x[4];
    cb_coords(g, cb, par, x);
    const int L0 = g.L[0], L01 = L0 * g.L[1], L012 = L01 * g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    const int rj = actj ? r0 : r0 + 1, rk = actk ? r0 + 1 : r0;
    PairPtrs P;
    {
      const SpinorF16 tj = A.in.shift(rj), tk = A.in.shift(rk);
      P.pj = par ? tj.p0 : tj.p1;  // neighbours have the other parity
      P.pk = par ? tk.p0 : tk.p1;
      P.nj = par ? tj.n0 : tj.n1;
      P.nk = par ? tk.n0 : tk.n1;
    }
    const int strd[4] = {1, L0, L01, L012};
    auto issue = [&](auto ic) {
      constexpr int I = decltype(ic)::value;
      if constexpr (I < 8) {
        nb_issue_m<I, NT>(st[I % S], tid, P, G, g, par, cb, x, s, strd[I >> 1]);
      } else if constexpr (XOP) {
        const SpinorF16 xj = A.x.shift(rj), xk = A.x.shift(rk);
        MSlot<NT>& t = st[8 % S];
        const uint4* bj = (par ? xj.p1 : xj.p0) + cb;
        const uint4* bk = (par ? xk.p1 : xk.p0) + cb;
#pragma unroll
        for (int q = 0; q < 3; q++) {
          cpa16(&t.sp[q][tid], bj + (size_t)q * g.Vh);
          cpa16(&t.sp[3 + q][tid], bk + (size_t)q * g.Vh);
        }
        cpa4(&t.nm[0][tid], (par ? xj.n1 : xj.n0) + cb);
        cpa4(&t.nm[1][tid], (par ? xk.n1 : xk.n0) + cb);
      }
      cpa_commit();
    };
    issue(std::integral_constant<int, 0>{});
    issue(std::integral_constant<int, 1>{});
    CP acc[4][3];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k / 3][k % 3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
    auto step = [&](auto dc) {
      constexpr int D = decltype(dc)::value;
      cpa_wait<S - 1>();
      nb_compute_m<B, DAG, D, NT>(st[D % S], tid, x, acc);
      if constexpr (D + S <= 8) issue(std::integral_constant<int, D + S>{});
      else cpa_commit();
    };
    step(std::integral_constant<int, 0>{});
    step(std::integral_constant<int, 1>{});
    step(std::integral_constant<int, 2>{});
    step(std::integral_constant<int, 3>{});
    step(std::integral_constant<int, 4>{});
    step(std::integral_constant<int, 5>{});
    step(std::integral_constant<int, 6>{});
    step(std::integral_constant<int, 7>{});
    cpa_wait<0>();
    if constexpr (XOP) {
      const MSlot<NT>& t = st[8 % S];
      CP xv[4][3];
      const float2 n = make_float2(t.nm[0][tid], t.nm[1][tid]);
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const uint4 wj = t.sp[q][tid], wk = t.sp[3 + q][tid];
        const uint32_t sj[4] = {wj.x, wj.y, wj.z, wj.w}, sk[4] = {wk.x, wk.y, wk.z, wk.w};
#pragma unroll
        for (int w = 0; w < 4; w++) {
          const __half2 hj = *reinterpret_cast<const __half2*>(&sj[w]);
          const __half2 hk = *reinterpret_cast<const __half2*>(&sk[w]);
          const int k = 4 * q + w;
          xv[k / 3][k % 3].re = mul2(make_float2(__low2float(hj), __low2float(hk)), n);
          xv[k / 3][k % 3].im = mul2(make_float2(__high2float(hj), __high2float(hk)), n);
        }
      }
      pair_epilogue<B, EPI, true>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1], xv);
    } else {
      pair_epilogue<B, EPI>(A, par, cb, rj, rk, actj, actk, acc, nrm[0], nrm[1]);
    }
  }
  if (A.norm_part) block_partials<2, NT>(nrm, A.norm_part, A.nblk, r0, A.nrhs, blk);
}

}  // namespace qkx
