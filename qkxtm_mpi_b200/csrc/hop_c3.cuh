// hop_c3.cuh -- FP64 hopping term with each output site split over three
// threads, one per colour row.
//
// The FP64 operator is bound by memory latency: one thread per site holds a
// 24-double accumulator, a neighbour spinor and a link at once (~150
// registers), which leaves 12 resident warps per SM to cover two dependent
// load round trips per direction.  Here thread (site, a) accumulates only
// colour a of the four output spins, multiplies by row a of U (forward) or
// column a of U (backward, for U^+), and projects the whole neighbour spinor
// itself; the three colour threads of a site read the same spinor words, so
// two of the three reads hit L1.  Same operator and epilogues as hop.cuh
// (reference Vector::applyDslash / applyDslashDag, lib/lattice_util.cpp:1158-1213,
// 1643-1699; 18-real links as given).
//
// Block: (NS sites) x (3 colours).  Grid: blockIdx.x = site_block * nrhs + rhs;
// with both parities the site blocks alternate parity (link reuse through L2).
#pragma once
#include "hop.cuh"

namespace qkx {

__device__ __forceinline__ Cx<double> ldc(const double2* p) {
  double2 d = __ldg(p);
  return {d.x, d.y};
}

template <int B, bool DAG, int MU, bool FW>
__device__ __forceinline__ void hop_side_c3(const double2* nb, const double2* ub, int Vh, bool flip, int a,
                                            Spin4<double>& acc) {
  constexpr int SF = DAG ? +1 : -1;
  using P = Proj<B, MU, FW ? SF : -SF>;
  Spinor<double> v;
  if constexpr (P::diag) {
#pragma unroll
    for (int sp = 0; sp < 2; sp++)
#pragma unroll
      for (int b = 0; b < 3; b++) v.c[P::drow + sp][b] = ldc(nb + (size_t)((P::drow + sp) * 3 + b) * Vh);
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) v.c[k / 3][k % 3] = ldc(nb + (size_t)k * Vh);
  }
  HalfSpinor<double> h;
  P::project(v, h);
  // row a of U_mu(x) (forward) or of U_mu(x-mu)^+ (backward)
  Cx<double> u[3];
#pragma unroll
  for (int b = 0; b < 3; b++) u[b] = FW ? ldc(ub + (size_t)(a * 3 + b) * Vh) : conj(ldc(ub + (size_t)(b * 3 + a) * Vh));
  Cx<double> t0 = cmul(u[0], h.c[0][0]) + cmul(u[1], h.c[0][1]) + cmul(u[2], h.c[0][2]);
  Cx<double> t1 = cmul(u[0], h.c[1][0]) + cmul(u[1], h.c[1][1]) + cmul(u[2], h.c[1][2]);
  if (flip) {
    t0 = -1.0 * t0;
    t1 = -1.0 * t1;
  }
  P::reconstruct1(acc, t0, t1);
}

template <class SP, int B, bool DAG, int MU>
__device__ __forceinline__ void hop_dir_c3(const SP& in, const GaugeF64x18& U, const Geom& g, int par, int cb,
                                           const int x[4], int s, int stride, int a, Spin4<double>& acc) {
  const int Lm = g.L[MU];
  const int Vh = g.Vh;
  const double2* inb = 1 - par ? in.p1 : in.p0;
  {
    const int n = (x[MU] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    const bool flip = (MU == 3) && g.bc_sign < 0 && x[3] == Lm - 1;
    hop_side_c3<B, DAG, MU, true>(inb + n, U.p + ((size_t)par * 4 + MU) * 9 * Vh + cb, Vh, flip, a, acc);
  }
  {
    const int n = (x[MU] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    const bool flip = (MU == 3) && g.bc_sign < 0 && x[3] == 0;
    hop_side_c3<B, DAG, MU, false>(inb + n, U.p + ((size_t)(1 - par) * 4 + MU) * 9 * Vh + n, Vh, flip, a, acc);
  }
}

template <int B>
__device__ __forceinline__ Spin4<double> twist_inv4(const Spin4<double>& v, double c, double s) {
  Spin4<double> g = gamma5_4<B>(v), o;
#pragma unroll
  for (int sp = 0; sp < 4; sp++) o.s[sp] = s * (v.s[sp] - c * phase<1>(g.s[sp]));
  return o;
}

// The fused epilogue of one colour thread (colour a of output site cb, parity par, right-hand
// side rhs) from its accumulated hopping term; stores the output (or, for the residual
// epilogues, the FP32 residual) and returns this thread's share of |output|^2 (|residual|^2).
template <class SP, int B, int EPI>
__device__ __forceinline__ double c3_epilogue(const HopArgs<SP, GaugeF64x18>& A, const HopRes& Rz, int rhs, int par,
                                              int cb, int a, const Spin4<double>& acc) {
  const double c = A.c * (A.cvec ? A.cvec[rhs] : 1.0);
  const double sc = A.s * (A.svec ? A.svec[rhs] : 1.0);
  const int Vh = A.g.Vh;
  double nrm = 0.0;
  Spin4<double> o;
  if constexpr (EPI == EPI_PLAIN) {
    o = acc;
  } else if constexpr (EPI == EPI_TWIST_INV) {
    o = twist_inv4<B>(acc, c, sc);
  } else {
    const SP xs = A.x.shift(rhs);
    const double2* xb = (par ? xs.p1 : xs.p0) + cb;
    Spin4<double> v;
#pragma unroll
    for (int sp = 0; sp < 4; sp++) v.s[sp] = ldc(xb + (size_t)(sp * 3 + a) * Vh);
    if constexpr (EPI == EPI_XPAY_TWINV || EPI == EPI_XPAY_TWINV_RES) {
#pragma unroll
      for (int sp = 0; sp < 4; sp++) v.s[sp] = A.a * acc.s[sp] + v.s[sp];
      o = twist_inv4<B>(v, c, sc);
      if constexpr (EPI == EPI_XPAY_TWINV_RES) {
        // the residual of the reconstructed sites, v - A o with A = 1 + i c g5
        const Spin4<double> g5o = gamma5_4<B>(o);
#pragma unroll
        for (int sp = 0; sp < 4; sp++) {
          const Cx<double> z = v.s[sp] - (o.s[sp] + c * phase<1>(g5o.s[sp]));
          nrm += z.re * z.re + z.im * z.im;
        }
      }
    } else {
      const Spin4<double> g5v = gamma5_4<B>(v);
#pragma unroll
      for (int sp = 0; sp < 4; sp++) o.s[sp] = A.a * acc.s[sp] + (v.s[sp] + c * phase<1>(g5v.s[sp]));
      if constexpr (EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_G5_RES) o = gamma5_4<B>(o);
    }
  }
  if constexpr (EPI == EPI_XPAY_G5_RES || EPI == EPI_XPAY_RES) {
    // res = w - o in FP64 and its norm; stored (when a target is given) as FP32, complex
    // k = sp*3 + a in half k%2 of float4 word k/2
    const SpinorF64 ws = Rz.w.shift(rhs);
    const double2* wb = (par ? ws.p1 : ws.p0) + cb;
    const SpinorF32 rs = Rz.res32.shift(rhs);
    float4* rq = par ? rs.p1 : rs.p0;
    float2* rb = rq ? reinterpret_cast<float2*>(rq + cb) : nullptr;
#pragma unroll
    for (int sp = 0; sp < 4; sp++) {
      const Cx<double> z = ldc(wb + (size_t)(sp * 3 + a) * Vh) - o.s[sp];
      nrm += z.re * z.re + z.im * z.im;
      const int k = sp * 3 + a;
      if (rb) rb[2 * (size_t)(k >> 1) * Vh + (k & 1)] = make_float2(float(z.re), float(z.im));
    }
  } else {
    const SP os = A.out.shift(rhs);
    double2* ob = (par ? os.p1 : os.p0) + cb;
#pragma unroll
    for (int sp = 0; sp < 4; sp++) {
      ob[(size_t)(sp * 3 + a) * Vh] = make_double2(o.s[sp].re, o.s[sp].im);
      if constexpr (EPI != EPI_XPAY_TWINV_RES) nrm += o.s[sp].re * o.s[sp].re + o.s[sp].im * o.s[sp].im;
    }
  }
  return nrm;
}

template <int NS, class SP, int B, bool DAG, int EPI>
__global__ void __launch_bounds__(NS * 3) hop_c3_kernel(HopArgs<SP, GaugeF64x18> A, HopRes Rz) {
  const int rhs = blockIdx.x % A.nrhs;
  const int blk = blockIdx.x / A.nrhs;
  double* slot = A.norm_part ? A.norm_part + (size_t)rhs * A.nblk + blk : nullptr;
  if (A.active && !A.active[rhs]) {
    if (slot && threadIdx.x == 0 && threadIdx.y == 0) *slot = 0.0;
    return;
  }
  int par, cb;
  if (A.out_parity < 0) {
    par = blk & 1;
    cb = (blk >> 1) * NS + threadIdx.x;
  } else {
    par = A.out_parity;
    cb = blk * NS + threadIdx.x;
  }
  const int a = threadIdx.y;
  double nrm = 0.0;
  if (cb < A.g.Vh) {
    const SP in = A.in.shift(rhs);
    int x[4];
    cb_coords(A.g, cb, par, x);
    const int L0 = A.g.L[0], L01 = L0 * A.g.L[1], L012 = L01 * A.g.L[2];
    const int s = x[0] + L0 * x[1] + L01 * x[2] + L012 * x[3];
    Spin4<double> acc;
#pragma unroll
    for (int sp = 0; sp < 4; sp++) acc.s[sp] = {0.0, 0.0};
    hop_dir_c3<SP, B, DAG, 0>(in, A.gauge, A.g, par, cb, x, s, 1, a, acc);
    hop_dir_c3<SP, B, DAG, 1>(in, A.gauge, A.g, par, cb, x, s, L0, a, acc);
    hop_dir_c3<SP, B, DAG, 2>(in, A.gauge, A.g, par, cb, x, s, L01, a, acc);
    hop_dir_c3<SP, B, DAG, 3>(in, A.gauge, A.g, par, cb, x, s, L012, a, acc);
    nrm = c3_epilogue<SP, B, EPI>(A, Rz, rhs, par, cb, a, acc);
  }
  if (slot) {
    __shared__ double red[(NS * 3 + 31) / 32];
    const int tid = threadIdx.y * NS + threadIdx.x;
    double w = nrm;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if ((tid & 31) == 0) red[tid >> 5] = w;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int k = 0; k < (NS * 3 + 31) / 32; k++) t += red[k];
      *slot = t;
    }
  }
}

template <int NS>
inline int c3_blocks_per_rhs(int Vh, int out_parity) {
  int per_par = (Vh + NS - 1) / NS;
  return out_parity < 0 ? 2 * per_par : per_par;
}

}  // namespace qkx
