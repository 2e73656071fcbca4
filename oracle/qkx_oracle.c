/*
 * qkx_oracle.c -- CPU oracle for the twisted-mass Dslash / CG hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see qkx_oracle.h).  Plain C99, FP64, serial.
 * It restates the reference's arithmetic with full 4x4 spin matrices instead
 * of the reference's hand-unrolled half-spinor macros, so that it is an
 * independent statement of the same operator; agreement with the compiled
 * reference (oracle/_ref) is what pins it.
 */
#include "qkx_oracle.h"

#define _POSIX_C_SOURCE 200809L
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef double _Complex cplx;

/* ------------------------------------------------------------------ */
/* geometry: LEXIC ordering, include/qkxTM.h:130; periodic neighbours as
 * LatticeGeometry's pointPlus/pointMinus tables, lib/lattice_util.cpp:79-103 */

long orc_volume(const int L[4]) { return (long)L[0] * L[1] * L[2] * L[3]; }

static void site_coords(const int L[4], long s, int c[4]) {
  c[0] = (int)(s % L[0]); s /= L[0];
  c[1] = (int)(s % L[1]); s /= L[1];
  c[2] = (int)(s % L[2]); s /= L[2];
  c[3] = (int)s;
}

static long site_index(const int L[4], const int c[4]) {
  return (long)c[0] + (long)L[0] * (c[1] + (long)L[1] * (c[2] + (long)L[2] * c[3]));
}

static long neighbour(const int L[4], long s, int mu, int step) {
  int c[4];
  site_coords(L, s, c);
  c[mu] = (c[mu] + step + L[mu]) % L[mu];
  return site_index(L, c);
}

/* parity of a site, (x+y+z+t)&1 -- getOddBit, lib/lattice_util.cpp:1148-1155 */
static int site_parity(const int L[4], long s) {
  int c[4];
  site_coords(L, s, c);
  return (c[0] + c[1] + c[2] + c[3]) & 1;
}

/* ------------------------------------------------------------------ */
/* gamma matrices.  UKQCD basis: lib/lattice_util.cpp:281-290.  Chiral basis:
 * read off the projectors of include/hopping_term_chiral.h:1-300 and the
 * chiral gamma5 of lib/lattice_util.cpp:1800-1820. */

static cplx gam[2][5][4][4];
static int gam_ready = 0;

static void set4(cplx g[4][4], int r0, int c0, cplx v0, int r1, int c1, cplx v1,
                 int r2, int c2, cplx v2, int r3, int c3, cplx v3) {
  memset(g, 0, sizeof(cplx) * 16);
  g[r0][c0] = v0; g[r1][c1] = v1; g[r2][c2] = v2; g[r3][c3] = v3;
}

static void init_gammas(void) {
  if (gam_ready) return;
  const cplx j = _Complex_I;
  /* UKQCD */
  set4(gam[0][0], 0, 3, j, 1, 2, j, 2, 1, -j, 3, 0, -j);
  set4(gam[0][1], 0, 3, 1, 1, 2, -1, 2, 1, -1, 3, 0, 1);
  set4(gam[0][2], 0, 2, j, 1, 3, -j, 2, 0, -j, 3, 1, j);
  set4(gam[0][3], 0, 0, 1, 1, 1, 1, 2, 2, -1, 3, 3, -1);
  set4(gam[0][4], 0, 2, 1, 1, 3, 1, 2, 0, 1, 3, 1, 1);
  /* chiral */
  set4(gam[1][0], 0, 3, -j, 1, 2, -j, 2, 1, j, 3, 0, j);
  set4(gam[1][1], 0, 3, -1, 1, 2, 1, 2, 1, 1, 3, 0, -1);
  set4(gam[1][2], 0, 2, -j, 1, 3, j, 2, 0, j, 3, 1, -j);
  set4(gam[1][3], 0, 2, -1, 1, 3, -1, 2, 0, -1, 3, 1, -1);
  set4(gam[1][4], 0, 0, 1, 1, 1, 1, 2, 2, -1, 3, 3, -1);
  gam_ready = 1;
}

/* ------------------------------------------------------------------ */
/* hopping term, Vector::applyDslash / applyDslashDag
 * (lib/lattice_util.cpp:1158-1213, 1643-1699; include/hopping_term.h):
 *   D  psi(x) = sum_mu (1-g_mu) U_mu(x) psi(x+mu) + (1+g_mu) U_mu(x-mu)^+ psi(x-mu)
 *   D+ psi(x) = sum_mu (1+g_mu) U_mu(x) psi(x+mu) + (1-g_mu) U_mu(x-mu)^+ psi(x-mu) */

static void hop_site(const int L[4], const cplx* U, const cplx* psi, long s, int dagger,
                     int basis, cplx out[12]) {
  const double sg = dagger ? 1.0 : -1.0;
  memset(out, 0, sizeof(cplx) * 12);
  for (int mu = 0; mu < 4; mu++) {
    const cplx(*g)[4] = gam[basis][mu];
    for (int dir = 0; dir < 2; dir++) {
      long n = neighbour(L, s, mu, dir == 0 ? 1 : -1);
      const cplx* Um = U + ((dir == 0 ? s : n) * 4 + mu) * 9;
      const cplx* pn = psi + n * 12;
      cplx chi[4][3];
      for (int sp = 0; sp < 4; sp++)
        for (int a = 0; a < 3; a++) {
          cplx acc = 0;
          for (int b = 0; b < 3; b++)
            acc += (dir == 0 ? Um[a * 3 + b] : conj(Um[b * 3 + a])) * pn[sp * 3 + b];
          chi[sp][a] = acc;
        }
      const double pm = (dir == 0) ? sg : -sg; /* projector 1 + pm*g_mu */
      for (int sp = 0; sp < 4; sp++)
        for (int a = 0; a < 3; a++) {
          cplx gc = 0;
          for (int t = 0; t < 4; t++) gc += g[sp][t] * chi[t][a];
          out[sp * 3 + a] += chi[sp][a] + pm * gc;
        }
    }
  }
}

void orc_dslash(const int L[4], const double* U, const double* psi, double* out, int dagger,
                int basis) {
  init_gammas();
  long V = orc_volume(L);
  cplx* o = (cplx*)malloc(sizeof(cplx) * 12 * V);
  for (long s = 0; s < V; s++) hop_site(L, (const cplx*)U, (const cplx*)psi, s, dagger, basis, o + s * 12);
  memcpy(out, o, sizeof(cplx) * 12 * V);
  free(o);
}

/* Vector::applyDslash_xx (lib/lattice_util.cpp:1272-1344): EO keeps the even
 * output sites, OE the odd ones; the other parity is written as zero. */
void orc_dslash_xx(const int L[4], const double* U, const double* psi, double* out, int parity,
                   int basis) {
  init_gammas();
  long V = orc_volume(L);
  int keep = (parity == ORC_EO) ? 0 : 1;
  cplx* o = (cplx*)malloc(sizeof(cplx) * 12 * V);
  for (long s = 0; s < V; s++) {
    if (site_parity(L, s) == keep)
      hop_site(L, (const cplx*)U, (const cplx*)psi, s, 0, basis, o + s * 12);
    else
      memset(o + s * 12, 0, sizeof(cplx) * 12);
  }
  memcpy(out, o, sizeof(cplx) * 12 * V);
  free(o);
}

/* ------------------------------------------------------------------ */
/* site-local operators */

static void g5_site(const cplx* in, cplx* out, int basis) {
  for (int sp = 0; sp < 4; sp++)
    for (int a = 0; a < 3; a++) {
      cplx acc = 0;
      for (int t = 0; t < 4; t++) acc += gam[basis][4][sp][t] * in[t * 3 + a];
      out[sp * 3 + a] = acc;
    }
}

/* applyGamma5 / applyGamma5_chiral, lib/lattice_util.cpp:1778-1820 */
void orc_gamma5(const int L[4], const double* psi, double* out, int basis) {
  init_gammas();
  long V = orc_volume(L);
  cplx tmp[12];
  for (long s = 0; s < V; s++) {
    g5_site((const cplx*)psi + s * 12, tmp, basis);
    memcpy((cplx*)out + s * 12, tmp, sizeof tmp);
  }
}

/* applyTwist / applyTwistDag / applyTwistInv / applyTwistDagInv
 * (lib/lattice_util.cpp:1563-1613, 1726-1776):
 *   twist      psi + i c g5 psi,  c = 2 kappa mu twistSign  (dagger: c -> -c)
 *   inverse   (psi - i c g5 psi) / (1 + (2 kappa mu)^2) */
void orc_twist(const orc_params* p, const double* psi, double* out, int dagger, int inverse,
               int basis) {
  init_gammas();
  long V = orc_volume(p->L);
  double c = 2.0 * p->kappa * p->mu * p->twistSign * (dagger ? -1.0 : 1.0);
  double nrm = 1.0 + (2.0 * p->kappa * p->mu) * (2.0 * p->kappa * p->mu);
  cplx g5[12];
  for (long s = 0; s < V; s++) {
    const cplx* in = (const cplx*)psi + s * 12;
    cplx* o = (cplx*)out + s * 12;
    g5_site(in, g5, basis);
    for (int k = 0; k < 12; k++) {
      cplx v = inverse ? (in[k] - _Complex_I * c * g5[k]) : (in[k] + _Complex_I * c * g5[k]);
      o[k] = inverse ? v / nrm : v;
    }
  }
}

/* out = -kappa*d + psi + i c g5 psi  (applyTwistAddDslash, lib/lattice_util.cpp:1420-1442;
 * applyTwistDagAddDslashDag :1701-1724 has c -> -c) */
static void twist_add_hop(const orc_params* p, const double* d, const double* psi, double* out,
                          double c, int basis) {
  long V = orc_volume(p->L);
  cplx g5[12];
  for (long s = 0; s < V; s++) {
    const cplx* in = (const cplx*)psi + s * 12;
    const cplx* ds = (const cplx*)d + s * 12;
    cplx* o = (cplx*)out + s * 12;
    g5_site(in, g5, basis);
    for (int k = 0; k < 12; k++) o[k] = -p->kappa * ds[k] + in[k] + _Complex_I * c * g5[k];
  }
}

/* Vector::tm, lib/lattice_util.cpp:1925-1933 */
void orc_tm(const orc_params* p, const double* U, const double* psi, double* out, int basis) {
  long V = orc_volume(p->L);
  double* d = (double*)malloc(sizeof(double) * 24 * V);
  orc_dslash(p->L, U, psi, d, 0, basis);
  twist_add_hop(p, d, psi, out, 2.0 * p->kappa * p->mu * p->twistSign, basis);
  free(d);
}

/* Vector::tmDag, lib/lattice_util.cpp:1935-1938 */
void orc_tm_dag(const orc_params* p, const double* U, const double* psi, double* out, int basis) {
  long V = orc_volume(p->L);
  double* d = (double*)malloc(sizeof(double) * 24 * V);
  orc_dslash(p->L, U, psi, d, 1, basis);
  twist_add_hop(p, d, psi, out, -2.0 * p->kappa * p->mu * p->twistSign, basis);
  free(d);
}

/* Vector::tmDagtm, lib/lattice_util.cpp:1940-1947 */
void orc_tm_dagtm(const orc_params* p, const double* U, const double* psi, double* out, int basis) {
  long V = orc_volume(p->L);
  double* t = (double*)malloc(sizeof(double) * 24 * V);
  orc_tm(p, U, psi, t, basis);
  orc_tm_dag(p, U, t, out, basis);
  free(t);
}

/* Vector::Wilson, lib/lattice_util.cpp:1949-1952: psi - kappa*D psi */
void orc_wilson(const orc_params* p, const double* U, const double* psi, double* out) {
  long V = orc_volume(p->L);
  double* d = (double*)malloc(sizeof(double) * 24 * V);
  orc_dslash(p->L, U, psi, d, 0, ORC_UKQCD);
  for (long k = 0; k < 24 * V; k++) out[k] = psi[k] - p->kappa * d[k];
  free(d);
}

/* Vector::tm_xx, lib/lattice_util.cpp:2001-2022 (chiral :2037-2058):
 *   EE: out_e = A psi_e - kappa^2 D_eo A^-1 D_oe psi_e,  A = 1 + i c g5; odd sites zero.
 *   OO: the same with the parities exchanged. */
void orc_tm_xx(const orc_params* p, const double* U, const double* psi, double* out, int parity,
               int basis) {
  init_gammas();
  long V = orc_volume(p->L);
  int keep = (parity == ORC_EE) ? 0 : 1;
  double* t1 = (double*)malloc(sizeof(double) * 24 * V);
  double* t2 = (double*)malloc(sizeof(double) * 24 * V);
  orc_dslash_xx(p->L, U, psi, t1, keep == 0 ? ORC_OE : ORC_EO, basis);
  orc_twist(p, t1, t2, 0, 1, basis);
  orc_dslash_xx(p->L, U, t2, t1, keep == 0 ? ORC_EO : ORC_OE, basis);
  double c = 2.0 * p->kappa * p->mu * p->twistSign;
  cplx g5[12];
  for (long s = 0; s < V; s++) {
    cplx* o = (cplx*)out + s * 12;
    if (site_parity(p->L, s) != keep) {
      memset(o, 0, sizeof(cplx) * 12);
      continue;
    }
    const cplx* in = (const cplx*)psi + s * 12;
    const cplx* ds = (const cplx*)t1 + s * 12;
    g5_site(in, g5, basis);
    for (int k = 0; k < 12; k++)
      o[k] = -(p->kappa * p->kappa) * ds[k] + (in[k] + _Complex_I * c * g5[k]);
  }
  free(t1);
  free(t2);
}

/* Vector::tm_xxDagTm_xx, lib/lattice_util.cpp:2024-2035 (chiral :2060-2071):
 *   g5 M_xx(-twistSign) g5 M_xx(twistSign) psi */
void orc_tm_xx_dagtm_xx(const orc_params* p, const double* U, const double* psi, double* out,
                        int parity, int basis) {
  long V = orc_volume(p->L);
  double* t = (double*)malloc(sizeof(double) * 24 * V);
  double* u = (double*)malloc(sizeof(double) * 24 * V);
  orc_params flip = *p;
  flip.twistSign = -p->twistSign;
  orc_tm_xx(p, U, psi, t, parity, basis);
  orc_gamma5(p->L, t, u, basis);
  orc_tm_xx(&flip, U, u, t, parity, basis);
  orc_gamma5(p->L, t, out, basis);
  free(t);
  free(u);
}

/* Vector::rotateFromChiralToUKQCD, lib/lattice_util.cpp:1834-1864:
 * psi' = T psi with T = (1/sqrt2) [[-1,0,1,0],[0,-1,0,1],[1,0,1,0],[0,1,0,1]] */
void orc_rotate_chiral_to_ukqcd(const int L[4], double* psi) {
  long V = orc_volume(L);
  const double h = 1.0 / sqrt(2.0);
  const double T[4][4] = {{-h, 0, h, 0}, {0, -h, 0, h}, {h, 0, h, 0}, {0, h, 0, h}};
  for (long s = 0; s < V; s++) {
    cplx* v = (cplx*)psi + s * 12;
    cplx o[12];
    for (int sp = 0; sp < 4; sp++)
      for (int a = 0; a < 3; a++) {
        cplx acc = 0;
        for (int t = 0; t < 4; t++) acc += T[sp][t] * v[t * 3 + a];
        o[sp * 3 + a] = acc;
      }
    memcpy(v, o, sizeof o);
  }
}

/* Gauge::applyBoundaryCondition, lib/lattice_util.cpp:708-724: with boundaryT == -1
 * the t-links on the last time slice change sign. */
void orc_apply_bc(const int L[4], int boundaryT, double* U) {
  if (boundaryT != -1) return;
  long V3 = (long)L[0] * L[1] * L[2];
  long V = orc_volume(L);
  for (long s = V - V3; s < V; s++)
    for (int k = 0; k < 18; k++) U[(s * 4 + 3) * 18 + k] = -U[(s * 4 + 3) * 18 + k];
}

/* ------------------------------------------------------------------ */
/* BLAS, lib/blas_qkxTM.cpp:4-56 and Vector::norm2, lib/lattice_util.cpp:464-477 */

double orc_re_dot(long V, const double* x, const double* y) {
  double acc = 0;
  for (long k = 0; k < 12 * V; k++) acc += x[2 * k] * y[2 * k] + x[2 * k + 1] * y[2 * k + 1];
  return acc;
}

void orc_axpy(long V, double a, const double* y, double* x) {
  for (long k = 0; k < 24 * V; k++) x[k] = x[k] + a * y[k];
}

void orc_xpay(long V, double a, const double* y, double* x) {
  for (long k = 0; k < 24 * V; k++) x[k] = a * x[k] + y[k];
}

double orc_norm2(long V, const double* x) { return orc_re_dot(V, x, x); }

/* ------------------------------------------------------------------ */
/* CG::operator(), lib/solvers.cpp:16-81.  Zero initial guess for r, x
 * accumulated, stop when r2 <= tol^2 * |in|^2 or after maxIter iterations. */
int orc_cg(const orc_params* p, const double* U, const double* in, double* x, double* r2_trace,
           int max_trace) {
  long V = orc_volume(p->L);
  size_t bytes = sizeof(double) * 24 * V;
  double* r = (double*)malloc(bytes);
  double* pv = (double*)malloc(bytes);
  double* Ap = (double*)malloc(bytes);
  memcpy(r, in, bytes);
  memcpy(pv, r, bytes);
  double r2 = orc_re_dot(V, r, r);
  double stop = orc_re_dot(V, in, in) * p->tol * p->tol;
  int k = 0;
  while (r2 > stop && k < p->maxIter) {
    if (r2_trace && k < max_trace) r2_trace[k] = r2;
    orc_tm_dagtm(p, U, pv, Ap, ORC_UKQCD);
    double pAp = orc_re_dot(V, pv, Ap);
    double alpha = r2 / pAp;
    double r2_old = r2;
    orc_axpy(V, alpha, pv, x);
    orc_axpy(V, -alpha, Ap, r);
    r2 = orc_re_dot(V, r, r);
    double beta = r2 / r2_old;
    orc_xpay(V, beta, r, pv);
    k++;
  }
  if (r2_trace && k < max_trace) r2_trace[k] = r2;
  free(r);
  free(pv);
  free(Ap);
  return k;
}

/* ------------------------------------------------------------------ */
/* synthetic inputs.  Counter-based generator: every (seed, stream, counter)
 * hashes to one uniform in (0,1) with the splitmix64 finaliser; normals come
 * from Box-Muller pairs.  The device generator in the product library uses
 * the same construction so both sides build the same fields. */

static uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double uniform01(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t h = mix64(seed ^ mix64(stream ^ mix64(ctr)));
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static void normal_pair(uint64_t seed, uint64_t stream, uint64_t ctr, double* g0, double* g1) {
  double u1 = uniform01(seed, stream, 2 * ctr);
  double u2 = uniform01(seed, stream, 2 * ctr + 1);
  double r = sqrt(-2.0 * log(u1));
  double ang = 6.283185307179586476925286766559 * u2;
  *g0 = r * cos(ang);
  *g1 = r * sin(ang);
}

enum { STREAM_LINK = 1, STREAM_SPINOR = 2 };

static void mat_mul3(const cplx* a, const cplx* b, cplx* c) {
  cplx t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      cplx acc = 0;
      for (int k = 0; k < 3; k++) acc += a[i * 3 + k] * b[k * 3 + j];
      t[i * 3 + j] = acc;
    }
  memcpy(c, t, sizeof t);
}

/* exp(X) by scaling and squaring around a 16-term Taylor series */
static void mat_exp3(const cplx* X, cplx* E) {
  double fn = 0;
  for (int k = 0; k < 9; k++) fn += creal(X[k]) * creal(X[k]) + cimag(X[k]) * cimag(X[k]);
  fn = sqrt(fn);
  int sq = 0;
  while (fn > 0.25 && sq < 64) { fn *= 0.5; sq++; }
  double scale = ldexp(1.0, -sq);
  cplx Y[9], T[9];
  for (int k = 0; k < 9; k++) Y[k] = X[k] * scale;
  /* Horner: E = I + Y(I + Y/2(I + Y/3(...))) */
  for (int k = 0; k < 9; k++) E[k] = (k % 4 == 0) ? 1.0 : 0.0;
  for (int n = 16; n >= 1; n--) {
    mat_mul3(Y, E, T);
    for (int k = 0; k < 9; k++) E[k] = T[k] / n + ((k % 4 == 0) ? 1.0 : 0.0);
  }
  for (int i = 0; i < sq; i++) mat_mul3(E, E, E);
}

/* Gram-Schmidt on rows 0,1; row 2 = conj(row0 x row1): an exact SU(3) element */
static void reunitarize(cplx* u) {
  double n0 = 0;
  for (int b = 0; b < 3; b++) n0 += creal(u[b] * conj(u[b]));
  n0 = 1.0 / sqrt(n0);
  for (int b = 0; b < 3; b++) u[b] *= n0;
  cplx d = 0;
  for (int b = 0; b < 3; b++) d += conj(u[b]) * u[3 + b];
  for (int b = 0; b < 3; b++) u[3 + b] -= d * u[b];
  double n1 = 0;
  for (int b = 0; b < 3; b++) n1 += creal(u[3 + b] * conj(u[3 + b]));
  n1 = 1.0 / sqrt(n1);
  for (int b = 0; b < 3; b++) u[3 + b] *= n1;
  u[6] = conj(u[1] * u[5] - u[2] * u[4]);
  u[7] = conj(u[2] * u[3] - u[0] * u[5]);
  u[8] = conj(u[0] * u[4] - u[1] * u[3]);
}

/* U_mu(x) = exp(i eps H), H = (A + A^+)/2 minus its trace/3, A entries unit
 * complex Gaussians (E|A_ab|^2 = 1: real and imaginary parts N(0, 1/2)). */
static void gauge_random_range(const int L[4], double eps, unsigned long long seed, double* U, long s0,
                               long s1) {
  for (long s = s0; s < s1; s++)
    for (int mu = 0; mu < 4; mu++) {
      cplx A[9], X[9];
      for (int k = 0; k < 9; k++) {
        double g0, g1;
        normal_pair(seed, STREAM_LINK, (uint64_t)(s * 4 + mu) * 9 + k, &g0, &g1);
        A[k] = (g0 + _Complex_I * g1) * 0.70710678118654752440;
      }
      cplx tr = 0;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) X[i * 3 + j] = 0.5 * (A[i * 3 + j] + conj(A[j * 3 + i]));
      tr = (X[0] + X[4] + X[8]) / 3.0;
      X[0] -= tr; X[4] -= tr; X[8] -= tr;
      for (int k = 0; k < 9; k++) X[k] *= _Complex_I * eps;
      cplx* u = (cplx*)U + (s * 4 + mu) * 9;
      mat_exp3(X, u);
      reunitarize(u);
    }
}

/* the generators split the sites over host threads (the result does not
 * depend on the split: every entry is a pure function of its counter) */
typedef struct {
  const int* L;
  double eps;
  unsigned long long seed;
  double* out;
  long s0, s1;
  int kind;
} gen_job;

static void spinor_gaussian_range(const int L[4], unsigned long long seed, double* psi, long s0, long s1);

static void* gen_worker(void* arg) {
  gen_job* j = (gen_job*)arg;
  if (j->kind == 0)
    gauge_random_range(j->L, j->eps, j->seed, j->out, j->s0, j->s1);
  else
    spinor_gaussian_range(j->L, j->seed, j->out, j->s0, j->s1);
  return NULL;
}

static void gen_parallel(const int L[4], double eps, unsigned long long seed, double* out, int kind) {
  long V = orc_volume(L);
  long nt = sysconf(_SC_NPROCESSORS_ONLN);
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  if (V < 4096) nt = 1;
  pthread_t th[64];
  gen_job jobs[64];
  for (long t = 0; t < nt; t++) {
    jobs[t] = (gen_job){L, eps, seed, out, V * t / nt, V * (t + 1) / nt, kind};
    if (nt == 1) {
      gen_worker(&jobs[t]);
    } else {
      pthread_create(&th[t], NULL, gen_worker, &jobs[t]);
    }
  }
  if (nt > 1)
    for (long t = 0; t < nt; t++) pthread_join(th[t], NULL);
}

void orc_gauge_random(const int L[4], double eps, unsigned long long seed, double* U) {
  gen_parallel(L, eps, seed, U, 0);
}

void orc_gauge_unit(const int L[4], double* U) {
  long V = orc_volume(L);
  memset(U, 0, sizeof(double) * 72 * V);
  for (long s = 0; s < V; s++)
    for (int mu = 0; mu < 4; mu++)
      for (int a = 0; a < 3; a++) U[((s * 4 + mu) * 9 + a * 4) * 2] = 1.0;
}

void orc_spinor_gaussian(const int L[4], unsigned long long seed, double* psi) {
  gen_parallel(L, 0.0, seed, psi, 1);
}

static void spinor_gaussian_range(const int L[4], unsigned long long seed, double* psi, long s0, long s1) {
  (void)L;
  for (long s = s0; s < s1; s++)
    for (int k = 0; k < 12; k++) {
      double g0, g1;
      normal_pair(seed, STREAM_SPINOR, (uint64_t)s * 12 + k, &g0, &g1);
      psi[(s * 12 + k) * 2] = g0;
      psi[(s * 12 + k) * 2 + 1] = g1;
    }
}

void orc_spinor_point(const int L[4], const int x[4], int spin, int colour, double* psi) {
  long V = orc_volume(L);
  memset(psi, 0, sizeof(double) * 24 * V);
  long s = site_index(L, x);
  psi[(s * 12 + spin * 3 + colour) * 2] = 1.0;
}

/* average Re tr of the 1x1 plaquette over sites and the six planes, /3 */
double orc_plaquette(const int L[4], const double* Ud) {
  const cplx* U = (const cplx*)Ud;
  long V = orc_volume(L);
  double acc = 0;
  for (long s = 0; s < V; s++)
    for (int mu = 0; mu < 4; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        long smu = neighbour(L, s, mu, 1), snu = neighbour(L, s, nu, 1);
        cplx a[9], b[9], c[9], d[9], t[9];
        memcpy(a, U + (s * 4 + mu) * 9, sizeof a);
        memcpy(b, U + (smu * 4 + nu) * 9, sizeof b);
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) {
            c[i * 3 + j] = conj(U[(snu * 4 + mu) * 9 + j * 3 + i]);
            d[i * 3 + j] = conj(U[(s * 4 + nu) * 9 + j * 3 + i]);
          }
        mat_mul3(a, b, t);
        mat_mul3(t, c, t);
        mat_mul3(t, d, t);
        acc += creal(t[0] + t[4] + t[8]) / 3.0;
      }
  return acc / (6.0 * V);
}
