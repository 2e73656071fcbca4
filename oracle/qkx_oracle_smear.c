/*
 * qkx_oracle_smear.c -- CPU oracle for the gauge-side stencils and the
 * propagator workflow around the solver: plaquette, APE smearing with its
 * SU(3) projection, Gaussian smearing, propagator assembly.
 *
 * TEST INFRASTRUCTURE ONLY (see qkx_oracle.h).  Plain C99, FP64, serial.
 * Each function restates one reference routine (file:line given per function)
 * in the reference's host layouts; agreement with the reference's own sources,
 * compiled unmodified into oracle/_ref/, is what pins it.
 */
#include "qkx_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

static void coords(const int L[4], long s, int c[4]) {
  c[0] = (int)(s % L[0]); s /= L[0];
  c[1] = (int)(s % L[1]); s /= L[1];
  c[2] = (int)(s % L[2]); s /= L[2];
  c[3] = (int)s;
}

static long step(const int L[4], long s, int mu, int d) {
  int c[4];
  coords(L, s, c);
  c[mu] = (c[mu] + d + L[mu]) % L[mu];
  return (long)c[0] + (long)L[0] * (c[1] + (long)L[1] * (c[2] + (long)L[2] * c[3]));
}

/* 3x3 complex products on row-major [3][3] arrays: a.b, a.b^dag, a^dag.b */
static void mm(const cplx* a, const cplx* b, cplx* r) {
  cplx t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) t[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
  memcpy(r, t, sizeof t);
}
static void mm_dag(const cplx* a, const cplx* b, cplx* r) {
  cplx t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      t[i * 3 + j] = a[i * 3] * conj(b[j * 3]) + a[i * 3 + 1] * conj(b[j * 3 + 1]) + a[i * 3 + 2] * conj(b[j * 3 + 2]);
  memcpy(r, t, sizeof t);
}
static void dag_mm(const cplx* a, const cplx* b, cplx* r) {
  cplx t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) t[i * 3 + j] = conj(a[i]) * b[j] + conj(a[3 + i]) * b[3 + j] + conj(a[6 + i]) * b[6 + j];
  memcpy(r, t, sizeof t);
}

/* ------------------------------------------------------------------ */
/* Gauge::calculatePlaquette, lib/lattice_util.cpp:923-946: the mean over
 * sites and the six planes mu<nu of Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag
 * U_nu(x)^dag, divided by 3 (colours). */
double orc_plaquette_ref(const int L[4], const double* Ud) {
  const cplx* U = (const cplx*)Ud;
  const long V = orc_volume(L);
  double sum = 0;
  for (long s = 0; s < V; s++)
    for (int mu = 0; mu < 3; mu++)
      for (int nu = mu + 1; nu < 4; nu++) {
        cplx p[9];
        mm(U + (s * 4 + mu) * 9, U + (step(L, s, mu, 1) * 4 + nu) * 9, p);
        mm_dag(p, U + (step(L, s, nu, 1) * 4 + mu) * 9, p);
        mm_dag(p, U + (s * 4 + nu) * 9, p);
        sum += creal(p[0]) + creal(p[4]) + creal(p[8]);
      }
  return sum / ((double)V * 3.0 * 6.0);
}

/* ------------------------------------------------------------------ */
/* qcd_projectSU33d, lib/blas.cpp:6-404, for one matrix: the unitary factor
 * M (M^dag M)^(-1/2) from the eigen-decomposition of H = M^dag M (eigenvalues
 * from the closed-form cubic, eigenvectors from 2x2 cofactors), its
 * determinant phase removed by exp(-i arg(det M)/3), then columns 0 and 1
 * re-orthonormalised and column 2 = conj(col0 x col1).  The steps, the branch
 * for an already diagonal H and the coefficient conventions of the two
 * orthogonalisations follow the reference so the results agree to rounding. */
static double cabs2(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

/* z^a as |z|^a (cos(a arg z), sin(a arg z)), blas.h:320 */
static cplx cpow_ref(cplx z, double a) {
  double r = pow(sqrt(cabs2(z)), a), t = atan2(cimag(z), creal(z)) * a;
  return r * cos(t) + I * (r * sin(t));
}

/* Re(x / y) as (x.re y.re + x.im y.im) / |y|^2, blas.h:314 */
static double cdiv_re(cplx x, cplx y) { return (creal(x) * creal(y) + cimag(x) * cimag(y)) / cabs2(y); }

static void su3_project(cplx* M) {
  cplx det = M[0] * (M[4] * M[8]) + M[1] * (M[5] * M[6]) + M[2] * (M[3] * M[7]) -
             (M[2] * (M[4] * M[6]) + M[0] * (M[5] * M[7]) + M[1] * (M[3] * M[8]));
  const double phase = atan2(cimag(det), creal(det)) / 3.0;

  cplx H[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) H[i * 3 + j] = conj(M[i]) * M[j] + conj(M[3 + i]) * M[3 + j] + conj(M[6 + i]) * M[6 + j];
  /* Hermitian by construction: H_ij = (H_ij + conj H_ji)/2, H_ji = conj H_ij */
  const int off[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int q = 0; q < 3; q++) {
    int i = off[q][0], j = off[q][1];
    H[i * 3 + j] = 0.5 * (H[i * 3 + j] + conj(H[j * 3 + i]));
    H[j * 3 + i] = conj(H[i * 3 + j]);
  }
  double h[3] = {creal(H[0]), creal(H[4]), creal(H[8])};

  cplx U[9];
  if (sqrt(cabs2(H[1])) + sqrt(cabs2(H[2])) + sqrt(cabs2(H[5])) <= 1e-8) {
    /* diagonal H: row i of M scaled by 1/sqrt(H_ii) */
    for (int i = 0; i < 3; i++) {
      const double f = 1.0 / sqrt(h[i]);
      for (int j = 0; j < 3; j++) U[i * 3 + j] = M[i * 3 + j] * f;
    }
    memcpy(M, U, sizeof U);
    return;
  }

  /* eigenvalues of the traceless part: e^3 + a e + b = 0 */
  const double tr = (h[0] + h[1] + h[2]) / 3.0;
  for (int i = 0; i < 3; i++) h[i] -= tr;
  const cplx h01 = H[1], h02 = H[2], h12 = H[5];
  const double a = -(h[2] * h[2] - h[0] * h[1] + cabs2(h01) + cabs2(h02) + cabs2(h12));
  const cplx b = -h[0] * h[1] * h[2] + h[2] * cabs2(h01) - h01 * (h12 * conj(h02)) + h[1] * cabs2(h02) +
                 h[0] * cabs2(h12) - h02 * (conj(h01) * conj(h12));
  const cplx w = cpow_ref(12.0 * a * a * a + 81.0 * (b * b), 0.5);
  const cplx D = cpow_ref(-9.0 * b + w, 1.0 / 3.0);
  const double r18 = pow(18.0, 1.0 / 3.0), r12 = pow(12.0, 1.0 / 3.0), r23 = pow(2.0 / 3.0, 1.0 / 3.0);
  const cplx w0 = 1.0 + I * sqrt(3.0), w1 = 1.0 - I * sqrt(3.0);
  double e[3];
  e[0] = creal(D) / r18 - cdiv_re(a * r23, D);
  e[1] = a * cdiv_re(w0, D * r12) - creal(w1 * D) / (r18 * 2.0);
  e[2] = -e[0] - e[1];
  for (int k = 0; k < 3; k++) e[k] += tr;
  for (int i = 0; i < 3; i++) h[i] += tr;

  /* eigenvectors 0 and 1 (as the reference forms them: the complex
   * conjugates of H's eigenvectors), orthonormalised; 2 = conj(v0 x v1) */
  cplx v[3][3];
  for (int k = 0; k < 2; k++) {
    v[k][0] = -(e[k] * H[6] - H[6] * h[1] + H[3] * H[7]);
    v[k][1] = -(H[6] * H[1] + e[k] * H[7] - h[0] * H[7]);
    v[k][2] = -e[k] * e[k] + e[k] * h[0] + cabs2(H[1]) + e[k] * h[1] - h[0] * h[1];
  }
  double n0 = cabs2(v[0][0]) + cabs2(v[0][1]) + cabs2(v[0][2]);
  cplx c = (v[0][0] * conj(v[1][0]) + v[0][1] * conj(v[1][1]) + v[0][2] * conj(v[1][2])) / n0;
  for (int j = 0; j < 3; j++) v[1][j] -= c * v[0][j];
  n0 = 1.0 / sqrt(n0);
  for (int j = 0; j < 3; j++) v[0][j] *= n0;
  double n1 = 1.0 / sqrt(cabs2(v[1][0]) + cabs2(v[1][1]) + cabs2(v[1][2]));
  for (int j = 0; j < 3; j++) v[1][j] *= n1;
  v[2][0] = conj(v[0][1] * v[1][2] - v[0][2] * v[1][1]);
  v[2][1] = conj(v[0][2] * v[1][0] - v[0][0] * v[1][2]);
  v[2][2] = conj(v[0][0] * v[1][1] - v[0][1] * v[1][0]);

  /* U = M sum_k e_k^(-1/2) conj(v_k) v_k^T exp(-i phase) */
  cplx vr[3][3], Mv[9];
  for (int k = 0; k < 3; k++) {
    const cplx f = (1.0 / sqrt(e[k])) * (cos(phase) - I * sin(phase));
    for (int j = 0; j < 3; j++) vr[k][j] = f * v[k][j];
  }
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++)
      Mv[i * 3 + k] = M[i * 3] * conj(v[k][0]) + M[i * 3 + 1] * conj(v[k][1]) + M[i * 3 + 2] * conj(v[k][2]);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) U[i * 3 + j] = Mv[i * 3] * vr[0][j] + Mv[i * 3 + 1] * vr[1][j] + Mv[i * 3 + 2] * vr[2][j];

  /* columns 0, 1 orthonormalised, column 2 = conj(col0 x col1) */
  n0 = cabs2(U[0]) + cabs2(U[3]) + cabs2(U[6]);
  c = (U[0] * conj(U[1]) + U[3] * conj(U[4]) + U[6] * conj(U[7])) / n0;
  for (int i = 0; i < 3; i++) U[i * 3 + 1] -= c * U[i * 3];
  n0 = 1.0 / sqrt(n0);
  for (int i = 0; i < 3; i++) U[i * 3] *= n0;
  n1 = 1.0 / sqrt(cabs2(U[1]) + cabs2(U[4]) + cabs2(U[7]));
  for (int i = 0; i < 3; i++) U[i * 3 + 1] *= n1;
  U[2] = conj(U[3] * U[7] - U[6] * U[4]);
  U[5] = conj(U[6] * U[1] - U[0] * U[7]);
  U[8] = conj(U[0] * U[4] - U[3] * U[1]);
  memcpy(M, U, sizeof U);
}

void orc_su3_project_many(long n, double* m) {
  for (long i = 0; i < n; i++) su3_project((cplx*)m + 9 * i);
}

/* ------------------------------------------------------------------ */
/* Gauge::APE_smearing, lib/lattice_util.cpp:948-1078.  Spatial links only:
 *   U'_mu(x) = P_SU3[ U_mu(x) + alpha sum_{nu != mu, nu < 3} ( U_nu(x) U_mu(x+nu) U_nu(x+mu)^dag
 *                                     + U_nu(x-nu)^dag U_mu(x-nu) U_nu(x-nu+mu) ) ]
 * repeated nsmear times; the t-links are those of U_in.  nsmear == 0 leaves
 * U_out untouched, as the reference leaves *this. */
void orc_ape_smear(const int L[4], const double* Uin, double* Uout, int nsmear, double alpha) {
  if (nsmear == 0) return;
  const long V = orc_volume(L);
  cplx* a = (cplx*)malloc(sizeof(cplx) * 36 * V);
  cplx* b = (cplx*)malloc(sizeof(cplx) * 36 * V);
  memcpy(a, Uin, sizeof(cplx) * 36 * V);
  memcpy(b, Uin, sizeof(cplx) * 36 * V);
  cplx *in = a, *out = b;
  for (int it = 0; it < nsmear; it++) {
    for (long s = 0; s < V; s++)
      for (int mu = 0; mu < 3; mu++) {
        cplx S[9] = {0}, t[9];
        for (int nu = 0; nu < 3; nu++) { /* forward staples */
          if (nu == mu) continue;
          mm(in + (s * 4 + nu) * 9, in + (step(L, s, nu, 1) * 4 + mu) * 9, t);
          mm_dag(t, in + (step(L, s, mu, 1) * 4 + nu) * 9, t);
          for (int k = 0; k < 9; k++) S[k] += t[k];
        }
        for (int nu = 0; nu < 3; nu++) { /* backward staples, formed at x-nu */
          if (nu == mu) continue;
          const long xb = step(L, s, nu, -1);
          mm(in + (xb * 4 + mu) * 9, in + (step(L, xb, mu, 1) * 4 + nu) * 9, t);
          dag_mm(in + (xb * 4 + nu) * 9, t, t);
          for (int k = 0; k < 9; k++) S[k] += t[k];
        }
        cplx* o = out + (s * 4 + mu) * 9;
        for (int k = 0; k < 9; k++) o[k] = alpha * S[k] + in[(s * 4 + mu) * 9 + k];
        su3_project(o);
      }
    cplx* t = in;
    in = out;
    out = t;
  }
  memcpy(Uout, in, sizeof(cplx) * 36 * V);
  free(a);
  free(b);
}

/* ------------------------------------------------------------------ */
/* Vector::Gaussian_smearing, lib/lattice_util.cpp:1080-1145:
 *   psi' = (psi + alpha sum_{mu<3} [U_mu(x) psi(x+mu) + U_mu(x-mu)^dag psi(x-mu)]) / (1 + 6 alpha)
 * on every spin, repeated nsmear times.  The input is left unchanged (the
 * reference overwrites it with an intermediate iterate); nsmear == 0 leaves
 * out untouched, as the reference leaves *this. */
void orc_gaussian_smear(const int L[4], const double* Ud, const double* in_d, double* out_d, int nsmear,
                        double alpha) {
  if (nsmear == 0) return;
  const cplx* U = (const cplx*)Ud;
  const long V = orc_volume(L);
  const double norm = 1.0 / (1.0 + 6.0 * alpha);
  cplx* a = (cplx*)malloc(sizeof(cplx) * 12 * V);
  cplx* b = (cplx*)malloc(sizeof(cplx) * 12 * V);
  memcpy(a, in_d, sizeof(cplx) * 12 * V);
  cplx *in = a, *out = b;
  for (int it = 0; it < nsmear; it++) {
    for (long s = 0; s < V; s++) {
      cplx acc[12] = {0};
      for (int mu = 0; mu < 3; mu++) {
        const long f = step(L, s, mu, 1), g = step(L, s, mu, -1);
        const cplx* uf = U + (s * 4 + mu) * 9;
        const cplx* ub = U + (g * 4 + mu) * 9;
        for (int sp = 0; sp < 4; sp++)
          for (int i = 0; i < 3; i++) {
            cplx t = 0;
            for (int j = 0; j < 3; j++)
              t += uf[i * 3 + j] * in[f * 12 + sp * 3 + j] + conj(ub[j * 3 + i]) * in[g * 12 + sp * 3 + j];
            acc[sp * 3 + i] += t;
          }
      }
      for (int k = 0; k < 12; k++) out[s * 12 + k] = norm * (in[s * 12 + k] + alpha * acc[k]);
    }
    cplx* t = in;
    in = out;
    out = t;
  }
  memcpy(out_d, in, sizeof(cplx) * 12 * V);
  free(a);
  free(b);
}

/* ------------------------------------------------------------------ */
/* Propagator::absorbVector, lib/lattice_util.cpp:2073-2081:
 * prop[x][mu][nu][c1][c2] = phi[x][mu][c1] for the given (nu, c2). */
void orc_absorb_vector(long V, const double* phi_d, int nu, int c2, double* prop_d) {
  const cplx* phi = (const cplx*)phi_d;
  cplx* prop = (cplx*)prop_d;
  for (long s = 0; s < V; s++)
    for (int mu = 0; mu < 4; mu++)
      for (int c1 = 0; c1 < 3; c1++) prop[s * 144 + mu * 36 + nu * 9 + c1 * 3 + c2] = phi[s * 12 + mu * 3 + c1];
}
