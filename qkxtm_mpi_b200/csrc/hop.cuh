// hop.cuh -- the Wilson hopping term D (and D^+) with fused site-local
// epilogues, one thread per output site, even-odd addressed, batched over
// right-hand sides.
//
//   D psi(x)  = sum_mu (1 - g_mu) U_mu(x) psi(x+mu) + (1 + g_mu) U_mu(x-mu)^+ psi(x-mu)
//   D+ psi(x) = the same with the two projectors exchanged
// (reference: Vector::applyDslash / applyDslashDag, lib/lattice_util.cpp:1158-1213
//  and 1643-1699, macros include/hopping_term.h and hopping_term_chiral.h).
//
// Output sites of parity p read only neighbours of parity 1-p, so the full
// operator is two parity halves and the even-odd operators are one half each.
// The antiperiodic time boundary is applied here from the site coordinate
// (sign bc_sign on t-hops crossing t = Lt-1 -> 0), so compressed links stay SU(3).
//
// Grid: blockIdx.x = site_block * nrhs + rhs, so the blocks that work on the
// same sites for different right-hand sides run back to back and share the
// links through L2.  When both parities are covered the site blocks alternate
// parity for the same reason (a link is used forward by its own site and
// backward by the neighbour of the other parity).
#pragma once
#include "qkx_common.cuh"

namespace qkx {

enum Epilogue {
  EPI_PLAIN = 0,       // out = D psi
  EPI_XPAY = 1,        // out = a D psi + x + i c g5 x           (tm, tm^+, Wilson, last step of tm_xx)
  EPI_XPAY_G5 = 2,     // out = g5 (a D psi + x + i c g5 x)      (normal operator through the g5 trick)
  EPI_TWIST_INV = 3,   // out = s (v - i c g5 v), v = D psi      (A^-1 D, first step of tm_xx)
  EPI_XPAY_TWINV = 4,  // out = s (v - i c g5 v), v = a D psi + x (odd-parity reconstruction)
  EPI_XPAY_G5_RES = 5, // res = w - g5 (a D psi + x + i c g5 x), stored in FP32 (hop_c3_kernel only)
  EPI_XPAY_RES = 6,    // res = w - (a D psi + x + i c g5 x), its norm only (hop_c3_kernel only)
  EPI_XPAY_G5_CGR = 7, // o = g5 (a D psi + x + i c g5 x) is not stored: the CG residual of the batch
                       // takes it, r -= alpha o, and |r|^2 goes to the norm partials (multi-RHS
                       // kernels of the mixed solver only; r is racc32, or racc64 for FP64 sloppy)
  EPI_XPAY_TWINV_RES = 8,  // as EPI_XPAY_TWINV, and |v - (out + i c g5 out)|^2 to the norm partials: with
                           // x = b_o, a = kappa the odd half of ||b - M x||^2 (hop_c3_kernel only)
};

// extra operands of EPI_XPAY_G5_RES / EPI_XPAY_RES: w, and the FP32 field the residual
// goes to (the output's parity; a null pointer stores nothing); |res|^2 is summed from
// the FP64 values before they are rounded
struct HopRes {
  SpinorF64 w;
  SpinorF32 res32;
};

template <class SP, class GA>
struct HopArgs {
  SP out;
  SP in;
  SP x;                // epilogue operand, parity of the output
  GA gauge;
  Geom g;
  int out_parity;      // 0 or 1; -1 = both parities
  double a, c, s;      // epilogue coefficients
  double* norm_part;   // if non-null: per-block partial sums of |out|^2, [rhs][site_block]
  int nrhs;            // right-hand sides in the batch (>= 1)
  int nblk;            // site blocks per right-hand side
  const double* cvec;  // optional per-RHS factor on c (twisted mass per RHS)
  const double* svec;  // optional per-RHS factor on s
  const int* active;   // optional per-RHS mask; inactive blocks do nothing
  // EPI_XPAY_G5_CGR only: per-RHS CG step length and the residual batch it updates
  const double* alpha = nullptr;
  SpinorF32 racc32{nullptr, nullptr, 0};
  SpinorF64 racc64{nullptr, nullptr, 0};
};

template <typename R>
__device__ __forceinline__ void zero(Spinor<R>& s) {
#pragma unroll
  for (int k = 0; k < 12; k++) s.c[k / 3][k % 3] = {R(0), R(0)};
}

template <class SP, class GA, typename R, int B, bool DAG, int MU>
__device__ __forceinline__ void hop_dir(const SP& in, const GA& gauge, const Geom& g, int par, int cb,
                                        const int x[4], Spinor<R>& acc) {
  constexpr int SF = DAG ? +1 : -1;  // forward projector 1 + SF*g
  HalfSpinor<R> h, uh;
  {
    int n = cb_neighbour(g, x, MU, +1);
    Spinor<R> s = in.load(1 - par, n);
    Proj<B, MU, SF>::project(s, h);
    Link<R> u = gauge.load(par, MU, cb);
    mul_link(u, h, uh);
    if (MU == 3 && g.bc_sign < 0 && x[3] == g.L[3] - 1) {
#pragma unroll
      for (int k = 0; k < 6; k++) uh.c[k / 3][k % 3] = R(-1) * uh.c[k / 3][k % 3];
    }
    Proj<B, MU, SF>::reconstruct(acc, uh);
  }
  {
    int n = cb_neighbour(g, x, MU, -1);
    Spinor<R> s = in.load(1 - par, n);
    Proj<B, MU, -SF>::project(s, h);
    Link<R> u = gauge.load(1 - par, MU, n);
    mul_link_dag(u, h, uh);
    if (MU == 3 && g.bc_sign < 0 && x[3] == 0) {
#pragma unroll
      for (int k = 0; k < 6; k++) uh.c[k / 3][k % 3] = R(-1) * uh.c[k / 3][k % 3];
    }
    Proj<B, MU, -SF>::reconstruct(acc, uh);
  }
}

// deterministic two-level sum: each block writes one partial; the caller
// reduces the partials in a fixed order.
template <int NT>
__device__ __forceinline__ void block_partial(double v, double* slot) {
  __shared__ double red[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) *slot = w;
  }
}

template <int B, typename R>
__device__ __forceinline__ Spinor<R> twist_inv(const Spinor<R>& v, R c, R s) {
  Spinor<R> g5v = gamma5<B>(v), o;
#pragma unroll
  for (int k = 0; k < 12; k++) o.c[k / 3][k % 3] = s * (v.c[k / 3][k % 3] - c * phase<1>(g5v.c[k / 3][k % 3]));
  return o;
}

template <int NT, class SP, class GA, typename R, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT) hop_kernel(HopArgs<SP, GA> A) {
  const int rhs = blockIdx.x % A.nrhs;
  const int blk = blockIdx.x / A.nrhs;
  double* slot = A.norm_part ? A.norm_part + (size_t)rhs * A.nblk + blk : nullptr;
  if (A.active && !A.active[rhs]) {
    if (slot && threadIdx.x == 0) *slot = 0.0;
    return;
  }
  int par, idx;
  if (A.out_parity < 0) {
    par = blk & 1;
    idx = (blk >> 1) * NT + threadIdx.x;
  } else {
    par = A.out_parity;
    idx = blk * NT + threadIdx.x;
  }
  double nrm = 0.0;
  if (idx < A.g.Vh) {
    const SP in = A.in.shift(rhs);
    const int cb = idx;
    int x[4];
    cb_coords(A.g, cb, par, x);
    Spinor<R> acc;
    zero(acc);
    hop_dir<SP, GA, R, B, DAG, 0>(in, A.gauge, A.g, par, cb, x, acc);
    hop_dir<SP, GA, R, B, DAG, 1>(in, A.gauge, A.g, par, cb, x, acc);
    hop_dir<SP, GA, R, B, DAG, 2>(in, A.gauge, A.g, par, cb, x, acc);
    hop_dir<SP, GA, R, B, DAG, 3>(in, A.gauge, A.g, par, cb, x, acc);

    const R c = R(A.c * (A.cvec ? A.cvec[rhs] : 1.0));
    const R s = R(A.s * (A.svec ? A.svec[rhs] : 1.0));
    const R a = R(A.a);
    Spinor<R> o;
    if constexpr (EPI == EPI_PLAIN) {
      o = acc;
    } else if constexpr (EPI == EPI_XPAY || EPI == EPI_XPAY_G5) {
      Spinor<R> v = A.x.shift(rhs).load(par, cb);
      Spinor<R> g5v = gamma5<B>(v);
#pragma unroll
      for (int k = 0; k < 12; k++)
        o.c[k / 3][k % 3] = a * acc.c[k / 3][k % 3] + (v.c[k / 3][k % 3] + c * phase<1>(g5v.c[k / 3][k % 3]));
      if constexpr (EPI == EPI_XPAY_G5) o = gamma5<B>(o);
    } else if constexpr (EPI == EPI_TWIST_INV) {
      o = twist_inv<B>(acc, c, s);
    } else {  // EPI_XPAY_TWINV
      Spinor<R> v = A.x.shift(rhs).load(par, cb);
#pragma unroll
      for (int k = 0; k < 12; k++) v.c[k / 3][k % 3] = a * acc.c[k / 3][k % 3] + v.c[k / 3][k % 3];
      o = twist_inv<B>(v, c, s);
    }
    A.out.shift(rhs).store(par, cb, o);
    if (slot) {
#pragma unroll
      for (int k = 0; k < 12; k++)
        nrm += double(o.c[k / 3][k % 3].re) * double(o.c[k / 3][k % 3].re) +
               double(o.c[k / 3][k % 3].im) * double(o.c[k / 3][k % 3].im);
    }
  }
  if (slot) block_partial<NT>(nrm, slot);
}

// launch geometry for hop_kernel: blocks per RHS and total grid
template <int NT>
inline int hop_blocks_per_rhs(int Vh, int out_parity) {
  int per_par = (Vh + NT - 1) / NT;
  return out_parity < 0 ? 2 * per_par : per_par;
}

}  // namespace qkx
