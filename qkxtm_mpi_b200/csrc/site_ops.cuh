// site_ops.cuh -- site-local operators on FP64 even-odd fields:
// gamma5, the twist factor A = 1 + i c g5 and its inverse, and the basis
// rotation from the chiral basis to UKQCD.
// (reference lib/lattice_util.cpp:1563-1613 applyTwist/applyTwistInv,
//  :1726-1776 applyTwistDag/applyTwistDagInv, :1778-1820 applyGamma5(_chiral),
//  :1834-1864 rotateFromChiralToUKQCD)
#pragma once
#include "qkx_common.cuh"

namespace qkx {

enum SiteOp { SITE_GAMMA5 = 0, SITE_TWIST = 1, SITE_TWIST_INV = 2, SITE_ROTATE_CH2UK = 3 };

// out = op(in) on n sites (a flat run of sites of one or both parities,
// stored [12][Vh] per parity; `n` counts sites over the parities covered).
template <int B>
__global__ void k_site_op(SpinorF64 in, SpinorF64 out, int npar_first, int npar, int op, double c, double s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npar * in.Vh) return;
  int par = npar_first + i / in.Vh;
  int cb = i % in.Vh;
  Spinor<double> v = in.load(par, cb), o;
  if (op == SITE_GAMMA5) {
    o = gamma5<B>(v);
  } else if (op == SITE_TWIST || op == SITE_TWIST_INV) {
    Spinor<double> g = gamma5<B>(v);
    double cc = (op == SITE_TWIST) ? c : -c;
    double ss = (op == SITE_TWIST) ? 1.0 : s;
#pragma unroll
    for (int k = 0; k < 12; k++) o.c[k / 3][k % 3] = ss * (v.c[k / 3][k % 3] + cc * phase<1>(g.c[k / 3][k % 3]));
  } else {
    const double h = 0.70710678118654752440;
    // T = (1/sqrt2) [[-1,0,1,0],[0,-1,0,1],[1,0,1,0],[0,1,0,1]]
#pragma unroll
    for (int a = 0; a < 3; a++) {
      o.c[0][a] = h * (v.c[2][a] - v.c[0][a]);
      o.c[1][a] = h * (v.c[3][a] - v.c[1][a]);
      o.c[2][a] = h * (v.c[0][a] + v.c[2][a]);
      o.c[3][a] = h * (v.c[1][a] + v.c[3][a]);
    }
  }
  out.store(par, cb, o);
}

}  // namespace qkx
