// hop.cuh -- the Wilson hopping term D (and D^+) with fused site-local
// epilogues, one thread per output site, even-odd addressed.
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
#pragma once
#include "qkx_common.cuh"

namespace qkx {

enum Epilogue {
  EPI_PLAIN = 0,      // out = D psi
  EPI_XPAY = 1,       // out = a D psi + x + i c g5 x           (tm, tm^+, Wilson, last step of tm_xx)
  EPI_XPAY_G5 = 2,    // out = g5 (a D psi + x + i c g5 x)      (normal operator through the g5 trick)
  EPI_TWIST_INV = 3,  // out = s (D psi - i c g5 D psi)          (A^-1 D, first step of tm_xx)
};

template <class SP, class GA>
struct HopArgs {
  SP out;
  SP in;
  SP x;                // epilogue operand, parity of the output
  GA gauge;
  Geom g;
  int out_parity;      // 0 or 1; -1 = both parities (grid covers 2*Vh sites)
  double a, c, s;      // epilogue coefficients
  double* norm_part;   // if non-null: per-block partial sums of |out|^2
};

template <typename R>
__device__ __forceinline__ void zero(Spinor<R>& s) {
#pragma unroll
  for (int k = 0; k < 12; k++) s.c[k / 3][k % 3] = {R(0), R(0)};
}

template <class SP, class GA, typename R, int B, bool DAG, int MU>
__device__ __forceinline__ void hop_dir(const HopArgs<SP, GA>& A, int par, int cb, const int x[4],
                                        Spinor<R>& acc) {
  constexpr int SF = DAG ? +1 : -1;  // forward projector 1 + SF*g
  HalfSpinor<R> h, uh;
  {
    int n = cb_neighbour(A.g, x, MU, +1);
    Spinor<R> s = A.in.load(1 - par, n);
    Proj<B, MU, SF>::project(s, h);
    Link<R> u = A.gauge.load(par, MU, cb);
    mul_link(u, h, uh);
    if (MU == 3 && A.g.bc_sign < 0 && x[3] == A.g.L[3] - 1) {
#pragma unroll
      for (int k = 0; k < 6; k++) uh.c[k / 3][k % 3] = R(-1) * uh.c[k / 3][k % 3];
    }
    Proj<B, MU, SF>::reconstruct(acc, uh);
  }
  {
    int n = cb_neighbour(A.g, x, MU, -1);
    Spinor<R> s = A.in.load(1 - par, n);
    Proj<B, MU, -SF>::project(s, h);
    Link<R> u = A.gauge.load(1 - par, MU, n);
    mul_link_dag(u, h, uh);
    if (MU == 3 && A.g.bc_sign < 0 && x[3] == 0) {
#pragma unroll
      for (int k = 0; k < 6; k++) uh.c[k / 3][k % 3] = R(-1) * uh.c[k / 3][k % 3];
    }
    Proj<B, MU, -SF>::reconstruct(acc, uh);
  }
}

// deterministic two-level sum: each block writes one partial; the caller
// reduces the partials in a fixed order.
template <int NT>
__device__ __forceinline__ void block_partial(double v, double* part) {
  __shared__ double red[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) part[blockIdx.x] = w;
  }
}

template <int NT, class SP, class GA, typename R, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NT) hop_kernel(HopArgs<SP, GA> A) {
  const int idx = blockIdx.x * NT + threadIdx.x;
  const int n = A.out_parity < 0 ? 2 * A.g.Vh : A.g.Vh;
  double nrm = 0.0;
  if (idx < n) {
    const int par = A.out_parity < 0 ? (idx >= A.g.Vh ? 1 : 0) : A.out_parity;
    const int cb = idx - (A.out_parity < 0 ? par * A.g.Vh : 0);
    int x[4];
    cb_coords(A.g, cb, par, x);
    Spinor<R> acc;
    zero(acc);
    hop_dir<SP, GA, R, B, DAG, 0>(A, par, cb, x, acc);
    hop_dir<SP, GA, R, B, DAG, 1>(A, par, cb, x, acc);
    hop_dir<SP, GA, R, B, DAG, 2>(A, par, cb, x, acc);
    hop_dir<SP, GA, R, B, DAG, 3>(A, par, cb, x, acc);

    Spinor<R> o;
    if constexpr (EPI == EPI_PLAIN) {
      o = acc;
    } else if constexpr (EPI == EPI_XPAY || EPI == EPI_XPAY_G5) {
      const R a = R(A.a), c = R(A.c);
      Spinor<R> v = A.x.load(par, cb);
      Spinor<R> g5v = gamma5<B>(v);
#pragma unroll
      for (int k = 0; k < 12; k++) {
        Cx<R> t = phase<1>(g5v.c[k / 3][k % 3]);  // i g5 v
        o.c[k / 3][k % 3] = a * acc.c[k / 3][k % 3] + (v.c[k / 3][k % 3] + c * t);
      }
      if constexpr (EPI == EPI_XPAY_G5) o = gamma5<B>(o);
    } else {  // EPI_TWIST_INV
      const R c = R(A.c), s = R(A.s);
      Spinor<R> g5d = gamma5<B>(acc);
#pragma unroll
      for (int k = 0; k < 12; k++) {
        Cx<R> t = phase<1>(g5d.c[k / 3][k % 3]);
        o.c[k / 3][k % 3] = s * (acc.c[k / 3][k % 3] - c * t);
      }
    }
    A.out.store(par, cb, o);
    if (A.norm_part) {
#pragma unroll
      for (int k = 0; k < 12; k++)
        nrm += double(o.c[k / 3][k % 3].re) * double(o.c[k / 3][k % 3].re) +
               double(o.c[k / 3][k % 3].im) * double(o.c[k / 3][k % 3].im);
    }
  }
  if (A.norm_part) block_partial<NT>(nrm, A.norm_part);
}

}  // namespace qkx
