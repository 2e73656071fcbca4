// hop_mrhs.cuh -- the hopping term for a batch of right-hand sides with NR of
// them per thread: each thread computes one output site for NR right-hand
// sides, so every link is loaded, converted and rebuilt from its 12 reals once
// and applied to NR spinors.  The FP16 site scale (and the boundary sign) is
// applied after the projection and link multiplication (both linear), folded
// into the FMAs that accumulate the rebuilt spinor.  Neighbours are found from
// the lexicographic index with one add and a wrap test per direction, and each
// right-hand side's base pointers are formed once per thread.
//
// Same operator and epilogues as hop.cuh (reference Vector::applyDslash,
// lib/lattice_util.cpp:1158-1213, with the twist site factors of
// applyTwistAddDslash :1420 / applyTwistInv :1588 fused); one output parity.
//
// Grid: blockIdx.x = site_block * ngroups + group, group g covering the
// right-hand sides [g*NR, g*NR + NR) of the batch.  (NR, NT) are chosen per
// lattice and batch by the autotuner (tune_tile in mixed.cu).
#pragma once
#include <type_traits>

#include "hop.cuh"

namespace qkx {

template <int NR, int NT>
__device__ __forceinline__ void block_partials(const double (&v)[NR], double* part, size_t stride, int r0,
                                               int nrhs, int blk) {
  __shared__ double red[NR][NT / 32];
#pragma unroll
  for (int j = 0; j < NR; j++) {
    double w = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0) red[j][threadIdx.x >> 5] = w;
  }
  __syncthreads();
  if (threadIdx.x < NR && r0 + (int)threadIdx.x < nrhs) {
    double w = 0.0;
#pragma unroll
    for (int k = 0; k < NT / 32; k++) w += red[threadIdx.x][k];
    part[(size_t)(r0 + threadIdx.x) * stride + blk] = w;
  }
}

template <int NR, class SP, class GA, typename R, int B, bool DAG, int MU>
__device__ __forceinline__ void hop_dir_m(const SP (&in)[NR], const GA& gauge, const Geom& g, int par, int cb,
                                          const int x[4], int s, int stride, const bool (&act)[NR],
                                          Spinor<R> (&acc)[NR]) {
  constexpr int SF = DAG ? +1 : -1;  // forward projector 1 + SF*g
  const int Lm = g.L[MU];
  {
    const int n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    const bool flip = (MU == 3) && g.bc_sign < 0 && x[3] == Lm - 1;
    const Link<R> u = gauge.load(par, MU, cb);
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (!act[j]) continue;
      R nrm;
      const Spinor<R> v = in[j].load_raw(1 - par, n, nrm);
      HalfSpinor<R> h, uh;
      Proj<B, MU, SF>::project(v, h);
      mul_link(u, h, uh);
      Proj<B, MU, SF>::reconstruct_scaled(acc[j], uh, flip ? -nrm : nrm);
    }
  }
  {
    const int n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    const bool flip = (MU == 3) && g.bc_sign < 0 && x[3] == 0;
    const Link<R> u = gauge.load(1 - par, MU, n);
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (!act[j]) continue;
      R nrm;
      const Spinor<R> v = in[j].load_raw(1 - par, n, nrm);
      HalfSpinor<R> h, uh;
      Proj<B, MU, -SF>::project(v, h);
      mul_link_dag(u, h, uh);
      Proj<B, MU, -SF>::reconstruct_scaled(acc[j], uh, flip ? -nrm : nrm);
    }
  }
}

template <int NT, int NR, class SP, class GA, typename R, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT) hop_mrhs_kernel(HopArgs<SP, GA> A) {
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
    int x[4];
    cb_coords(A.g, cb, par, x);
    const int L0 = A.g.L[0], L01 = L0 * A.g.L[1], L012 = L01 * A.g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    SP in[NR];  // each right-hand side's input, shifted once per thread
#pragma unroll
    for (int j = 0; j < NR; j++) in[j] = A.in.shift(r0 + j);
    Spinor<R> acc[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) zero(acc[j]);
    hop_dir_m<NR, SP, GA, R, B, DAG, 0>(in, A.gauge, A.g, par, cb, x, s, 1, act, acc);
    hop_dir_m<NR, SP, GA, R, B, DAG, 1>(in, A.gauge, A.g, par, cb, x, s, L0, act, acc);
    hop_dir_m<NR, SP, GA, R, B, DAG, 2>(in, A.gauge, A.g, par, cb, x, s, L01, act, acc);
    hop_dir_m<NR, SP, GA, R, B, DAG, 3>(in, A.gauge, A.g, par, cb, x, s, L012, act, acc);

    const R a = R(A.a);
#pragma unroll
    for (int j = 0; j < NR; j++) {
      if (!act[j]) continue;
      const int r = r0 + j;
      const R c = R(A.c * (A.cvec ? A.cvec[r] : 1.0));
      const R sc = R(A.s * (A.svec ? A.svec[r] : 1.0));
      Spinor<R> o;
      if constexpr (EPI == EPI_PLAIN) {
        o = acc[j];
      } else if constexpr (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_CGR) {
        const Spinor<R> v = A.x.shift(r).load(par, cb);
        const Spinor<R> g5v = gamma5<B>(v);
#pragma unroll
        for (int k = 0; k < 12; k++)
          o.c[k / 3][k % 3] = a * acc[j].c[k / 3][k % 3] + (v.c[k / 3][k % 3] + c * phase<1>(g5v.c[k / 3][k % 3]));
        if constexpr (EPI != EPI_XPAY) o = gamma5<B>(o);
      } else if constexpr (EPI == EPI_TWIST_INV) {
        o = twist_inv<B>(acc[j], c, sc);
      } else {  // EPI_XPAY_TWINV
        Spinor<R> v = A.x.shift(r).load(par, cb);
#pragma unroll
        for (int k = 0; k < 12; k++) v.c[k / 3][k % 3] = a * acc[j].c[k / 3][k % 3] + v.c[k / 3][k % 3];
        o = twist_inv<B>(v, c, sc);
      }
      if constexpr (EPI == EPI_XPAY_G5_CGR) {
        // the CG residual takes A p directly: r -= alpha A p, |r|^2 in FP64
        const R al = R(A.alpha[r]);
        auto rr = [&]() {
          if constexpr (std::is_same<R, double>::value) return A.racc64.shift(r);
          else return A.racc32.shift(r);
        }();
        Spinor<R> v = rr.load(par, cb);
#pragma unroll
        for (int k = 0; k < 12; k++) {
          Cx<R>& q = v.c[k / 3][k % 3];
          q.re = q.re - al * o.c[k / 3][k % 3].re;
          q.im = q.im - al * o.c[k / 3][k % 3].im;
          nrm[j] += double(q.re) * double(q.re) + double(q.im) * double(q.im);
        }
        rr.store(par, cb, v);
      } else {
        A.out.shift(r).store(par, cb, o);
        if (A.norm_part) {
#pragma unroll
          for (int k = 0; k < 12; k++)
            nrm[j] += double(o.c[k / 3][k % 3].re) * double(o.c[k / 3][k % 3].re) +
                      double(o.c[k / 3][k % 3].im) * double(o.c[k / 3][k % 3].im);
        }
      }
    }
  }
  if (A.norm_part) block_partials<NR, NT>(nrm, A.norm_part, A.nblk, r0, A.nrhs, blk);
}

// blocks per RHS group for hop_mrhs_kernel (one parity)
template <int NT>
inline int mrhs_site_blocks(int Vh) {
  return (Vh + NT - 1) / NT;
}

}  // namespace qkx
