// smear.cuh -- device kernels of the gauge-side stencils and of the propagator
// workflow around the solver:
//   plaquette             Gauge::calculatePlaquette  lib/lattice_util.cpp:923-946
//   SU(3) projection      qcd_projectSU33d           lib/blas.cpp:6-404
//   APE smearing step     Gauge::APE_smearing        lib/lattice_util.cpp:948-1078
//   Gaussian smearing     Vector::Gaussian_smearing  lib/lattice_util.cpp:1080-1145
//   propagator assembly   Propagator::absorbVector   lib/lattice_util.cpp:2073-2081
// All FP64 on the even-odd SoA layouts of qkx_common.cuh.
#pragma once
#include "blas.cuh"
#include "qkx_common.cuh"

namespace qkx {

using Lk = Link<double>;
using Cd = Cx<double>;

// ---------------------------------------------------------------- 3x3 algebra
__device__ __forceinline__ Lk lk_mul(const Lk& a, const Lk& b) {  // a b
  Lk r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) r.m[i][j] = cmul(a.m[i][0], b.m[0][j]) + cmul(a.m[i][1], b.m[1][j]) + cmul(a.m[i][2], b.m[2][j]);
  return r;
}
__device__ __forceinline__ Lk lk_mul_dag(const Lk& a, const Lk& b) {  // a b^dag
  Lk r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      r.m[i][j] = cmulc(b.m[j][0], a.m[i][0]) + cmulc(b.m[j][1], a.m[i][1]) + cmulc(b.m[j][2], a.m[i][2]);
  return r;
}
__device__ __forceinline__ Lk lk_dag_mul(const Lk& a, const Lk& b) {  // a^dag b
  Lk r;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) r.m[i][j] = cmulc(a.m[0][i], b.m[0][j]) + cmulc(a.m[1][i], b.m[1][j]) + cmulc(a.m[2][i], b.m[2][j]);
  return r;
}
__device__ __forceinline__ double abs2(Cd z) { return z.re * z.re + z.im * z.im; }

// ---------------------------------------------------------------- SU(3) projection
// Constants of the closed-form cubic, computed on the host with the same
// library calls as the reference (pow(x, 1./3.), sqrt(3.)).
struct ProjConst {
  double r18, r12, r23, s3;  // 18^(1/3), 12^(1/3), (2/3)^(1/3), sqrt(3)
};

// z^a as |z|^a (cos(a arg z), sin(a arg z))
__device__ __forceinline__ Cd cpow_polar(Cd z, double a) {
  const double r = pow(sqrt(abs2(z)), a);
  double s, c;
  sincos(atan2(z.im, z.re) * a, &s, &c);
  return {r * c, r * s};
}
// Re(x / y)
__device__ __forceinline__ double cdiv_re(Cd x, Cd y) { return (x.re * y.re + x.im * y.im) / abs2(y); }

// One matrix of qcd_projectSU33d (lib/blas.cpp:6-404): the unitary polar factor
// M (M^dag M)^(-1/2) built from the eigen-decomposition of H = M^dag M (closed
// cubic for the eigenvalues, 2x2 cofactors for two eigenvectors, the third
// their conjugated cross product), times exp(-i arg(det M)/3); then columns 0
// and 1 re-orthonormalised and column 2 = conj(col0 x col1).  An H whose
// off-diagonal moduli sum to <= 1e-8 takes the reference's shortcut of scaling
// row i of M by 1/sqrt(H_ii).  The orthogonalisation coefficients keep the
// reference's convention (sum_j a_j conj(b_j)) so both codes round alike.
__device__ __forceinline__ void su3_project(Lk& M, const ProjConst& k) {
  const Lk& m = M;
  const Cd det = (cmul(m.m[0][0], cmul(m.m[1][1], m.m[2][2])) + cmul(m.m[0][1], cmul(m.m[1][2], m.m[2][0])) +
                  cmul(m.m[0][2], cmul(m.m[1][0], m.m[2][1]))) -
                 (cmul(m.m[0][2], cmul(m.m[1][1], m.m[2][0])) + cmul(m.m[0][0], cmul(m.m[1][2], m.m[2][1])) +
                  cmul(m.m[0][1], cmul(m.m[1][0], m.m[2][2])));
  const double phase = atan2(det.im, det.re) / 3.0;

  Lk H = lk_dag_mul(m, m);
  H.m[0][1] = 0.5 * (H.m[0][1] + conj(H.m[1][0]));
  H.m[1][0] = conj(H.m[0][1]);
  H.m[0][2] = 0.5 * (H.m[0][2] + conj(H.m[2][0]));
  H.m[2][0] = conj(H.m[0][2]);
  H.m[1][2] = 0.5 * (H.m[1][2] + conj(H.m[2][1]));
  H.m[2][1] = conj(H.m[1][2]);
  double h0 = H.m[0][0].re, h1 = H.m[1][1].re, h2 = H.m[2][2].re;

  if (sqrt(abs2(H.m[0][1])) + sqrt(abs2(H.m[0][2])) + sqrt(abs2(H.m[1][2])) <= 1e-8) {
    const double f[3] = {1.0 / sqrt(h0), 1.0 / sqrt(h1), 1.0 / sqrt(h2)};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) M.m[i][j] = f[i] * M.m[i][j];
    return;
  }

  // eigenvalues of the traceless part, e^3 + a e + b = 0
  const double tr = (h0 + h1 + h2) / 3.0;
  h0 -= tr;
  h1 -= tr;
  h2 -= tr;
  const Cd h01 = H.m[0][1], h02 = H.m[0][2], h12 = H.m[1][2];
  const double a = -(h2 * h2 - h0 * h1 + abs2(h01) + abs2(h02) + abs2(h12));
  const Cd t1 = cmul(h01, cmul(h12, conj(h02))), t2 = cmul(h02, cmul(conj(h01), conj(h12)));
  const Cd b = {-h0 * h1 * h2 + h2 * abs2(h01) - t1.re + h1 * abs2(h02) + h0 * abs2(h12) - t2.re, -t1.im - t2.im};
  const Cd bb = cmul(b, b);
  const Cd w = cpow_polar({12.0 * a * a * a + 81.0 * bb.re, 81.0 * bb.im}, 0.5);
  const Cd D = cpow_polar({-9.0 * b.re + w.re, -9.0 * b.im + w.im}, 1.0 / 3.0);
  double e[3];
  e[0] = D.re / k.r18 - cdiv_re({a * k.r23, 0.0}, D);
  e[1] = a * cdiv_re({1.0, k.s3}, {D.re * k.r12, D.im * k.r12}) - cmul(Cd{1.0, -k.s3}, D).re / (k.r18 * 2.0);
  e[2] = -e[0] - e[1];
  e[0] += tr;
  e[1] += tr;
  e[2] += tr;
  h0 += tr;
  h1 += tr;

  // eigenvectors 0, 1 (conjugates of H's, as the reference forms them)
  Cd v[3][3];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const Cd p = cmul(H.m[1][0], H.m[2][1]);
    v[q][0] = {-(e[q] * H.m[2][0].re - H.m[2][0].re * h1 + p.re), -(e[q] * H.m[2][0].im - H.m[2][0].im * h1 + p.im)};
    const Cd r = cmul(H.m[2][0], H.m[0][1]);
    v[q][1] = {-(r.re + e[q] * H.m[2][1].re - h0 * H.m[2][1].re), -(r.im + e[q] * H.m[2][1].im - h0 * H.m[2][1].im)};
    v[q][2] = {-e[q] * e[q] + e[q] * h0 + abs2(H.m[0][1]) + e[q] * h1 - h0 * h1, 0.0};
  }
  double n0 = abs2(v[0][0]) + abs2(v[0][1]) + abs2(v[0][2]);
  Cd c = cmulc(v[1][0], v[0][0]) + cmulc(v[1][1], v[0][1]) + cmulc(v[1][2], v[0][2]);
  c = (1.0 / n0) * c;
#pragma unroll
  for (int j = 0; j < 3; j++) v[1][j] = v[1][j] - cmul(c, v[0][j]);
  n0 = 1.0 / sqrt(n0);
#pragma unroll
  for (int j = 0; j < 3; j++) v[0][j] = n0 * v[0][j];
  double n1 = 1.0 / sqrt(abs2(v[1][0]) + abs2(v[1][1]) + abs2(v[1][2]));
#pragma unroll
  for (int j = 0; j < 3; j++) v[1][j] = n1 * v[1][j];
  v[2][0] = conj(cmul(v[0][1], v[1][2]) - cmul(v[0][2], v[1][1]));
  v[2][1] = conj(cmul(v[0][2], v[1][0]) - cmul(v[0][0], v[1][2]));
  v[2][2] = conj(cmul(v[0][0], v[1][1]) - cmul(v[0][1], v[1][0]));

  // U = M sum_q e_q^(-1/2) conj(v_q) v_q^T exp(-i phase)
  double sp, cp;
  sincos(phase, &sp, &cp);
  Lk Mv;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int q = 0; q < 3; q++)
      Mv.m[i][q] = cmulc(v[q][0], m.m[i][0]) + cmulc(v[q][1], m.m[i][1]) + cmulc(v[q][2], m.m[i][2]);
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const double de = 1.0 / sqrt(e[q]);
    const Cd f = {de * cp, -de * sp};
#pragma unroll
    for (int j = 0; j < 3; j++) v[q][j] = cmul(f, v[q][j]);
  }
  Lk U;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) U.m[i][j] = cmul(Mv.m[i][0], v[0][j]) + cmul(Mv.m[i][1], v[1][j]) + cmul(Mv.m[i][2], v[2][j]);

  // columns 0, 1 orthonormalised, column 2 = conj(col0 x col1)
  n0 = abs2(U.m[0][0]) + abs2(U.m[1][0]) + abs2(U.m[2][0]);
  c = cmulc(U.m[0][1], U.m[0][0]) + cmulc(U.m[1][1], U.m[1][0]) + cmulc(U.m[2][1], U.m[2][0]);
  c = (1.0 / n0) * c;
#pragma unroll
  for (int i = 0; i < 3; i++) U.m[i][1] = U.m[i][1] - cmul(c, U.m[i][0]);
  n0 = 1.0 / sqrt(n0);
#pragma unroll
  for (int i = 0; i < 3; i++) U.m[i][0] = n0 * U.m[i][0];
  n1 = 1.0 / sqrt(abs2(U.m[0][1]) + abs2(U.m[1][1]) + abs2(U.m[2][1]));
#pragma unroll
  for (int i = 0; i < 3; i++) U.m[i][1] = n1 * U.m[i][1];
  U.m[0][2] = conj(cmul(U.m[1][0], U.m[2][1]) - cmul(U.m[2][0], U.m[1][1]));
  U.m[1][2] = conj(cmul(U.m[2][0], U.m[0][1]) - cmul(U.m[0][0], U.m[2][1]));
  U.m[2][2] = conj(cmul(U.m[0][0], U.m[1][1]) - cmul(U.m[1][0], U.m[0][1]));
  M = U;
}

__device__ __forceinline__ void store_link(double2* eo, int Vh, int parity, int mu, int cb, const Lk& u) {
  double2* b = eo + ((size_t)(parity * 4 + mu) * 9) * Vh + cb;
#pragma unroll
  for (int k = 0; k < 9; k++) b[(size_t)k * Vh] = make_double2(u.m[k / 3][k % 3].re, u.m[k / 3][k % 3].im);
}

// cb index of x shifted by d along mu (x's coordinates given)
__device__ __forceinline__ int cb_shift(const Geom& g, int x[4], int mu, int d) {
  const int o = x[mu];
  int v = o + d;
  x[mu] = v < 0 ? v + g.L[mu] : (v >= g.L[mu] ? v - g.L[mu] : v);
  const int r = cb_index(g, x);
  x[mu] = o;
  return r;
}

// ---------------------------------------------------------------- plaquette
// Per-block partial sums of Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
// over mu < nu, as tr[(U_mu(x) U_nu(x+mu)) (U_nu(x) U_mu(x+nu))^dag].
// Blocks [0, nblk) cover the even sites, [nblk, 2 nblk) the odd ones.
template <int NT>
__global__ void __launch_bounds__(NT) k_plaquette(GaugeF64x18 u, Geom g, double* __restrict__ part) {
  const int nblk = (g.Vh + NT - 1) / NT;
  const int par = blockIdx.x / nblk;
  const int cb = (blockIdx.x % nblk) * NT + threadIdx.x;
  double acc = 0.0;
  if (cb < g.Vh) {
    int x[4];
    cb_coords(g, cb, par, x);
#pragma unroll 1
    for (int mu = 0; mu < 3; mu++) {
      const Lk a = u.load(par, mu, cb);
      const int xm = cb_shift(g, x, mu, 1);
#pragma unroll 1
      for (int nu = mu + 1; nu < 4; nu++) {
        const Lk p = lk_mul(a, u.load(1 - par, nu, xm));
        const Lk q = lk_mul(u.load(par, nu, cb), u.load(1 - par, mu, cb_shift(g, x, nu, 1)));
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) acc += p.m[i][j].re * q.m[i][j].re + p.m[i][j].im * q.m[i][j].im;
      }
    }
  }
  const double s = block_sum<NT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ---------------------------------------------------------------- APE step
// out_mu(x) = P_SU3[ in_mu(x) + alpha * (sum of the 4 spatial staples) ] for
// mu = 0..2; forward staples U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag first, then the
// backward ones U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu), in nu order.
// blockIdx.x = (parity * 3 + mu) * nblk + block.  The t-links are not touched.
template <int NT>
__global__ void __launch_bounds__(NT) k_ape_step(GaugeF64x18 in, double2* __restrict__ out, Geom g, double alpha,
                                                 ProjConst pc) {
  const int nblk = (g.Vh + NT - 1) / NT;
  const int pm = blockIdx.x / nblk;
  const int par = pm / 3, mu = pm % 3;
  const int cb = (blockIdx.x % nblk) * NT + threadIdx.x;
  if (cb >= g.Vh) return;
  int x[4];
  cb_coords(g, cb, par, x);
  Lk S;
#pragma unroll
  for (int k = 0; k < 9; k++) S.m[k / 3][k % 3] = {0.0, 0.0};
  const int xm = cb_shift(g, x, mu, 1);
#pragma unroll 1
  for (int nu = 0; nu < 3; nu++) {
    if (nu == mu) continue;
    const Lk t = lk_mul(in.load(par, nu, cb), in.load(1 - par, mu, cb_shift(g, x, nu, 1)));
    const Lk f = lk_mul_dag(t, in.load(1 - par, nu, xm));
#pragma unroll
    for (int k = 0; k < 9; k++) S.m[k / 3][k % 3] = S.m[k / 3][k % 3] + f.m[k / 3][k % 3];
  }
#pragma unroll 1
  for (int nu = 0; nu < 3; nu++) {
    if (nu == mu) continue;
    const int o = x[nu];
    x[nu] = o == 0 ? g.L[nu] - 1 : o - 1;  // x - nu
    const int xb = cb_index(g, x);
    const int xbm = cb_shift(g, x, mu, 1);
    x[nu] = o;
    const Lk t = lk_mul(in.load(1 - par, mu, xb), in.load(par, nu, xbm));
    const Lk f = lk_dag_mul(in.load(1 - par, nu, xb), t);
#pragma unroll
    for (int k = 0; k < 9; k++) S.m[k / 3][k % 3] = S.m[k / 3][k % 3] + f.m[k / 3][k % 3];
  }
  const Lk u = in.load(par, mu, cb);
  Lk M;
#pragma unroll
  for (int k = 0; k < 9; k++) M.m[k / 3][k % 3] = fma_s(alpha, S.m[k / 3][k % 3], u.m[k / 3][k % 3]);
  su3_project(M, pc);
  store_link(out, g.Vh, par, mu, cb, M);
}

// qcd_projectSU33d on the spatial links of an even-odd field, in place
template <int NT>
__global__ void __launch_bounds__(NT) k_project_su3(double2* __restrict__ eo, Geom g, ProjConst pc) {
  const int nblk = (g.Vh + NT - 1) / NT;
  const int pm = blockIdx.x / nblk;
  const int par = pm / 3, mu = pm % 3;
  const int cb = (blockIdx.x % nblk) * NT + threadIdx.x;
  if (cb >= g.Vh) return;
  GaugeF64x18 u{eo, g.Vh};
  Lk M = u.load(par, mu, cb);
  su3_project(M, pc);
  store_link(eo, g.Vh, par, mu, cb, M);
}

// ---------------------------------------------------------------- Gaussian smearing
// A batch of even-odd FP64 fields [2][12][Vh], one pointer per right-hand side.
struct FieldPtrs {
  const double2* p[MAX_RHS];
};

__device__ __forceinline__ void load_sp(const double2* f, int Vh, int parity, int cb, Spinor<double>& s) {
  const double2* b = f + (size_t)parity * 12 * Vh + cb;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const double2 d = __ldg(b + (size_t)k * Vh);
    s.c[k / 3][k % 3] = {d.x, d.y};
  }
}

// acc += U v (dag = false) or U^dag v (dag = true), on all four spins
template <bool DAG>
__device__ __forceinline__ void link_spinor_acc(const Lk& u, const Spinor<double>& v, Spinor<double>& acc) {
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      Cd t = acc.c[s][a];
#pragma unroll
      for (int b = 0; b < 3; b++) t = t + (DAG ? cmulc(u.m[b][a], v.c[s][b]) : cmul(u.m[a][b], v.c[s][b]));
      acc.c[s][a] = t;
    }
}

// One smearing iteration on sites cb in [cb0, cb0 + ncb) of both parities:
//   out = norm * (in + alpha * sum_{mu<3} [U_mu(x) in(x+mu) + U_mu(x-mu)^dag in(x-mu)])
// Each thread takes one site for NR right-hand sides, so every link is loaded
// once per NR fields.  blockIdx.x = ((block * 2) + parity) * ngroups + group,
// the groups of one site block adjacent so their shared links stay in L2.
template <int NT, int NR>
__global__ void __launch_bounds__(NT) k_gauss_step(FieldPtrs in, FieldPtrs out, GaugeF64x18 u, Geom g, int nrhs,
                                                   int cb0, int ncb, double alpha, double norm) {
  const int ngrp = (nrhs + NR - 1) / NR;
  const int grp = blockIdx.x % ngrp;
  const int bp = blockIdx.x / ngrp;
  const int par = bp & 1;
  const int i = (bp >> 1) * NT + threadIdx.x;
  if (i >= ncb) return;
  const int cb = cb0 + i;
  const int r0 = grp * NR;
  int x[4];
  cb_coords(g, cb, par, x);
  const int L0 = g.L[0], L01 = L0 * g.L[1];
  const int s = x[0] + L0 * x[1] + L01 * x[2] + L01 * g.L[2] * x[3];
  const int Vh = g.Vh;
  Spinor<double> acc[NR];
#pragma unroll
  for (int j = 0; j < NR; j++)
#pragma unroll
    for (int k = 0; k < 12; k++) acc[j].c[k / 3][k % 3] = {0.0, 0.0};
#pragma unroll
  for (int mu = 0; mu < 3; mu++) {
    const int stride = mu == 0 ? 1 : (mu == 1 ? L0 : L01);
    const int Lm = g.L[mu];
    const int nf = (x[mu] == Lm - 1 ? s - (Lm - 1) * stride : s + stride) >> 1;
    const int nb = (x[mu] == 0 ? s + (Lm - 1) * stride : s - stride) >> 1;
    {
      const Lk uf = u.load(par, mu, cb);
#pragma unroll
      for (int j = 0; j < NR; j++) {
        if (r0 + j >= nrhs) break;
        Spinor<double> v;
        load_sp(in.p[r0 + j], Vh, 1 - par, nf, v);
        link_spinor_acc<false>(uf, v, acc[j]);
      }
    }
    {
      const Lk ub = u.load(1 - par, mu, nb);
#pragma unroll
      for (int j = 0; j < NR; j++) {
        if (r0 + j >= nrhs) break;
        Spinor<double> v;
        load_sp(in.p[r0 + j], Vh, 1 - par, nb, v);
        link_spinor_acc<true>(ub, v, acc[j]);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NR; j++) {
    if (r0 + j >= nrhs) break;
    Spinor<double> v;
    load_sp(in.p[r0 + j], Vh, par, cb, v);
    double2* o = const_cast<double2*>(out.p[r0 + j]) + (size_t)par * 12 * Vh + cb;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const Cd t = fma_s(alpha, acc[j].c[k / 3][k % 3], v.c[k / 3][k % 3]);
      o[(size_t)k * Vh] = make_double2(norm * t.re, norm * t.im);
    }
  }
}

// ---------------------------------------------------------------- propagator
// prop[x][mu][nu][c1][c2] = sol_{nu*3+c2}[x][mu][c1] over the whole lattice,
// prop in the host layout (LEXIC sites), one thread per complex element.
static __global__ void k_prop_assemble(FieldPtrs sol, double2* __restrict__ prop, Geom g) {
  const size_t n = (size_t)2 * g.Vh * 144;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = (int)(i / 144), e = (int)(i % 144);
  const int mu = e / 36, nu = (e / 9) & 3, c1 = (e / 3) % 3, c2 = e % 3;
  int x[4];
  x[0] = s % g.L[0];
  int r = s / g.L[0];
  x[1] = r % g.L[1];
  r /= g.L[1];
  x[2] = r % g.L[2];
  x[3] = r / g.L[2];
  const int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  prop[i] = __ldg(sol.p[nu * 3 + c2] + ((size_t)par * 12 + mu * 3 + c1) * g.Vh + (s >> 1));
}

// unit point sources: field r (< 12) gets 1 at spin-colour r of site (parity, cb)
static __global__ void k_point_sources(FieldPtrs f, int Vh, int parity, int cb) {
  const int r = threadIdx.x;
  if (r < 12) const_cast<double2*>(f.p[r])[((size_t)parity * 12 + r) * Vh + cb] = make_double2(1.0, 0.0);
}

}  // namespace qkx
