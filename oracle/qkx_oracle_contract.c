/*
 * qkx_oracle_contract.c -- CPU oracle of the two-point contractions:
 * momentum lists, meson and nucleon contractions, and their Fourier transform.
 *
 * TEST INFRASTRUCTURE ONLY (see qkx_oracle.h).  Plain C99, FP64, serial.
 * Restates lib/contractions.cpp (Meson::contract :251, Meson::fourier :121,
 * Baryon::contract :494, Baryon::fourier :356, tabulateIndices :159, :387-492,
 * createMomenta :37) with the gamma and charge-conjugation tables of
 * LatticeGeometry's constructor (lib/lattice_util.cpp:255-305).  Agreement
 * with those sources, compiled unmodified into oracle/_ref/, pins it.
 *
 * A propagator is [V][4][4][3][3] complex (Propagator::M).  Correlators:
 *   meson   [Lt][Nmom]        complex per operator (Meson::F)
 *   baryon  [Lt][Nmom][4][4]  complex               (Baryon::F)
 */
#include "qkx_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

#define REF_PI 3.14159265359 /* the truncated pi of lib/contractions.cpp:5 */

static const int EPS[6][3] = {{0, 1, 2}, {2, 0, 1}, {1, 2, 0}, {2, 1, 0}, {0, 2, 1}, {1, 0, 2}};
static const int SGN_EPS[6] = {+1, +1, +1, -1, -1, -1};

/* gamma_1..4, gamma_5 (UKQCD), C = gamma_2 gamma_4, Cbar = g4 C^dag g4,
 * C gamma_i and its bar (g4 (C gamma_i)^dag g4) */
static cplx G[5][4][4], Cc[4][4], Cc_bar[4][4], CG[5][4][4], CG_bar[5][4][4];
static int tables_ready = 0;

static void tables(void) {
  if (tables_ready) return;
  memset(G, 0, sizeof G);
  const cplx j = _Complex_I;
  G[0][0][3] = j, G[0][1][2] = j, G[0][2][1] = -j, G[0][3][0] = -j;
  G[1][0][3] = 1, G[1][1][2] = -1, G[1][2][1] = -1, G[1][3][0] = 1;
  G[2][0][2] = j, G[2][1][3] = -j, G[2][2][0] = -j, G[2][3][1] = j;
  G[3][0][0] = 1, G[3][1][1] = 1, G[3][2][2] = -1, G[3][3][3] = -1;
  G[4][0][2] = 1, G[4][1][3] = 1, G[4][2][0] = 1, G[4][3][1] = 1;
  memset(Cc, 0, sizeof Cc);
  memset(Cc_bar, 0, sizeof Cc_bar);
  memset(CG, 0, sizeof CG);
  memset(CG_bar, 0, sizeof CG_bar);
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++)
      for (int k = 0; k < 4; k++) Cc[m][n] += G[1][m][k] * G[3][k][n];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++)
      for (int k = 0; k < 4; k++)
        for (int l = 0; l < 4; l++) Cc_bar[m][n] += G[3][m][l] * conj(Cc[k][l]) * G[3][k][n];
  for (int i = 0; i < 5; i++)
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++)
        for (int k = 0; k < 4; k++) CG[i][m][n] += Cc[m][k] * G[i][k][n];
  for (int i = 0; i < 5; i++)
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++)
        for (int k = 0; k < 4; k++)
          for (int l = 0; l < 4; l++) CG_bar[i][m][n] += G[3][m][l] * conj(CG[i][k][l]) * G[3][k][n];
  tables_ready = 1;
}

static double norm2c(cplx z) { return creal(z) * creal(z) + cimag(z) * cimag(z); }

/* createMomenta (lib/contractions.cpp:37-62): all (nx,ny,nz) with
 * nx^2+ny^2+nz^2 = q for q = 0..Q_sq, each component from +q down to -q */
int orc_momenta(int Q_sq, int* mom, int max) {
  int n = 0;
  for (int q = 0; q <= Q_sq; q++)
    for (int nx = q; nx >= -q; nx--)
      for (int ny = q; ny >= -q; ny--)
        for (int nz = q; nz >= -q; nz--)
          if (nx * nx + ny * ny + nz * nz == q) {
            if (n < max) {
              mom[3 * n] = nx;
              mom[3 * n + 1] = ny;
              mom[3 * n + 2] = nz;
            }
            n++;
          }
  return n;
}

/* the spin matrix of a meson operator (MESONS_OPERATOR order: ONE G5 G1 G2 G3 G4 G5G1..G5G4) */
static void meson_gamma(int op, cplx g[4][4]) {
  memset(g, 0, sizeof(cplx) * 16);
  if (op == 0) {
    for (int m = 0; m < 4; m++) g[m][m] = 1;
  } else if (op == 1) {
    memcpy(g, G[4], sizeof(cplx) * 16);
  } else if (op <= 5) {
    memcpy(g, G[op - 2], sizeof(cplx) * 16);
  } else {
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++)
        for (int k = 0; k < 4; k++) g[m][n] += G[4][m][k] * G[op - 6][k][n];
  }
}

/* Meson::contract then Meson::fourier(FORWARD): corr[t][imom] */
int orc_meson_2pt(const int L[4], const double* propd, int op, int Q_sq, const int x_src[4], double* corrd) {
  tables();
  const cplx* P = (const cplx*)propd;
  cplx* corr = (cplx*)corrd;
  const long V = orc_volume(L);
  cplx g[4][4];
  meson_gamma(op, g);
  cplx val[256];
  int ind[256][4], cnt = 0;
  for (int be = 0; be < 4; be++)
    for (int ga = 0; ga < 4; ga++)
      for (int de = 0; de < 4; de++)
        for (int al = 0; al < 4; al++) {
          const cplx t = g[be][ga] * g[de][al];
          if (norm2c(t) > 1e-3) {
            val[cnt] = t;
            ind[cnt][0] = be, ind[cnt][1] = ga, ind[cnt][2] = de, ind[cnt][3] = al;
            cnt++;
          }
        }
  cplx* M = (cplx*)calloc((size_t)V, sizeof(cplx));
  for (long v = 0; v < V; v++) {
    const cplx* pp = P + v * 144;  /* pp[mu][nu][c1][c2] = pp[mu*36 + nu*9 + c1*3 + c2] */
    cplx q[4][4][3][3];            /* g5 pp^dag g5 */
    for (int c1 = 0; c1 < 3; c1++)
      for (int c2 = 0; c2 < 3; c2++)
        for (int mu = 0; mu < 4; mu++)
          for (int nu = 0; nu < 4; nu++) {
            cplx s = 0;
            for (int k = 0; k < 4; k++)
              for (int l = 0; l < 4; l++) s += G[4][mu][k] * conj(pp[l * 36 + k * 9 + c2 * 3 + c1]) * G[4][l][nu];
            q[mu][nu][c1][c2] = s;
          }
    cplx m = 0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        for (int i = 0; i < cnt; i++)
          m += val[i] * pp[ind[i][3] * 36 + ind[i][0] * 9 + a * 3 + b] * q[ind[i][1]][ind[i][2]][b][a];
    M[v] = m;
  }
  int mom[3000];
  const int nmom = orc_momenta(Q_sq, mom, 1000);
  const long V3 = (long)L[0] * L[1] * L[2];
  for (int t = 0; t < L[3]; t++)
    for (int im = 0; im < nmom; im++) {
      cplx s = 0;
      for (int z = 0; z < L[2]; z++)
        for (int y = 0; y < L[1]; y++)
          for (int x = 0; x < L[0]; x++) {
            const long v = t * V3 + x + (long)L[0] * (y + (long)L[1] * z);
            const double th = (((double)mom[3 * im] * (x - x_src[0])) / L[0] +
                               ((double)mom[3 * im + 1] * (y - x_src[1])) / L[1] +
                               ((double)mom[3 * im + 2] * (z - x_src[2])) / L[2]) * 2 * REF_PI;
            s += M[v] * (cos(th) - _Complex_I * sin(th));
          }
      corr[t * nmom + im] = s;
    }
  free(M);
  return nmom;
}

/* Baryon::contract(prop1, prop2, op) then Baryon::fourier(FORWARD):
 * corr[t][imom][gamma][gammap]; op = 0 NTN, 1 NTR, 2 RTN, 3 RTR */
int orc_baryon_2pt(const int L[4], const double* p1d, const double* p2d, int op, int Q_sq, const int x_src[4],
                   double* corrd) {
  tables();
  const cplx* P1 = (const cplx*)p1d;
  const cplx* P2 = (const cplx*)p2d;
  cplx* corr = (cplx*)corrd;
  const long V = orc_volume(L);
  /* terms: value and (alpha, beta, betap, alphap, gamma, delta, gammap, deltap), -1 = free index */
  static cplx val[4096];
  static int ind[4096][8];
  int cnt = 0;
  for (int al = 0; al < 4; al++)
    for (int be = 0; be < 4; be++)
      for (int bp = 0; bp < 4; bp++)
        for (int ap = 0; ap < 4; ap++) {
          if (op == 0) {
            const cplx t = CG[4][al][be] * CG_bar[4][bp][ap];
            if (norm2c(t) > 1e-3) {
              val[cnt] = t;
              int r[8] = {al, be, bp, ap, -1, -1, -1, -1};
              memcpy(ind[cnt++], r, sizeof r);
            }
          } else if (op == 1) {
            for (int gp = 0; gp < 4; gp++)
              for (int dp = 0; dp < 4; dp++) {
                const cplx t = CG[4][al][be] * Cc_bar[bp][ap] * G[4][gp][dp];
                if (norm2c(t) > 1e-3) {
                  val[cnt] = t;
                  int r[8] = {al, be, bp, ap, -1, -1, gp, dp};
                  memcpy(ind[cnt++], r, sizeof r);
                }
              }
          } else if (op == 2) {
            for (int ga = 0; ga < 4; ga++)
              for (int de = 0; de < 4; de++) {
                const cplx t = Cc[al][be] * CG_bar[4][bp][ap] * G[4][ga][de];
                if (norm2c(t) > 1e-3) {
                  val[cnt] = t;
                  int r[8] = {al, be, bp, ap, ga, de, -1, -1};
                  memcpy(ind[cnt++], r, sizeof r);
                }
              }
          } else {
            for (int ga = 0; ga < 4; ga++)
              for (int de = 0; de < 4; de++)
                for (int gp = 0; gp < 4; gp++)
                  for (int dp = 0; dp < 4; dp++) {
                    const cplx t = Cc[al][be] * Cc_bar[bp][ap] * G[4][ga][de] * G[4][gp][dp];
                    if (norm2c(t) > 1e-3) {
                      val[cnt] = t;
                      int r[8] = {al, be, bp, ap, ga, de, gp, dp};
                      memcpy(ind[cnt++], r, sizeof r);
                    }
                  }
          }
        }
  cplx* M = (cplx*)calloc((size_t)V * 16, sizeof(cplx));
  /* M[g][gp] += s * f * P2[be][bp][b][b1] (P1[al][ap][a][a1] P1[X][Y][c][c1] - P1[al][Y][a][c1] P1[X][ap][c][a1])
   * with X, Y the sink/source spin of the third quark: (gamma, gammap) for NTN,
   * (gamma, deltap) for NTR, (delta, gammap) for RTN, (delta, deltap) for RTR;
   * s = +1 for NTN and RTN, -1 for NTR and RTR */
  const double sign = (op == 1 || op == 3) ? -1.0 : 1.0;
  for (long v = 0; v < V; v++) {
    const cplx* p1 = P1 + v * 144;
    const cplx* p2 = P2 + v * 144;
    cplx* m = M + v * 16;
    for (int g = 0; g < 4; g++)
      for (int gp = 0; gp < 4; gp++)
        for (int i = 0; i < cnt; i++) {
          const int* r = ind[i];
          if (r[4] >= 0 && r[4] != g) continue;  /* the term's sink spin (RTN, RTR) */
          if (r[6] >= 0 && r[6] != gp) continue; /* its source spin (NTR, RTR) */
          const int X = r[4] >= 0 ? r[5] : g, Y = r[6] >= 0 ? r[7] : gp;
          for (int e1 = 0; e1 < 6; e1++)
            for (int e2 = 0; e2 < 6; e2++) {
              const int a = EPS[e1][0], b = EPS[e1][1], c = EPS[e1][2];
              const int a1 = EPS[e2][0], b1 = EPS[e2][1], c1 = EPS[e2][2];
              const cplx f = (double)(SGN_EPS[e1] * SGN_EPS[e2]) * val[i];
              const cplx d = p1[r[0] * 36 + r[3] * 9 + a * 3 + a1] * p1[X * 36 + Y * 9 + c * 3 + c1] -
                             p1[r[0] * 36 + Y * 9 + a * 3 + c1] * p1[X * 36 + r[3] * 9 + c * 3 + a1];
              m[g * 4 + gp] += sign * (f * p2[r[1] * 36 + r[2] * 9 + b * 3 + b1] * d);
            }
        }
  }
  int mom[3000];
  const int nmom = orc_momenta(Q_sq, mom, 1000);
  const long V3 = (long)L[0] * L[1] * L[2];
  for (int t = 0; t < L[3]; t++)
    for (int im = 0; im < nmom; im++)
      for (int k = 0; k < 16; k++) {
        cplx s = 0;
        for (int z = 0; z < L[2]; z++)
          for (int y = 0; y < L[1]; y++)
            for (int x = 0; x < L[0]; x++) {
              const long v = t * V3 + x + (long)L[0] * (y + (long)L[1] * z);
              const double th = (((double)mom[3 * im] * (x - x_src[0])) / L[0] +
                                 ((double)mom[3 * im + 1] * (y - x_src[1])) / L[1] +
                                 ((double)mom[3 * im + 2] * (z - x_src[2])) / L[2]) * 2 * REF_PI;
              s += M[v * 16 + k] * (cos(th) - _Complex_I * sin(th));
            }
        corr[((long)t * nmom + im) * 16 + k] = s;
      }
  free(M);
  return nmom;
}

/* Baryon_Dec::contract(prop1, prop2, op) then Baryon_Dec::fourier(FORWARD)
 * (lib/contractions.cpp:744-870, :703-741, tabulateIndices_Delta :743-765):
 * corr[t][imom][i][gamma][gammap], i = 0..2 the spatial C gamma_i;
 * op 0 = DELTA_ISO1 (three prop1 quarks), 1 = DELTA_ISO1O2 (prop2 as the odd one).
 * Terms, colour sums and the eight (six) products of each term are accumulated in
 * the reference's order, so the result is the reference's to the last bit. */
int orc_delta_2pt(const int L[4], const double* p1d, const double* p2d, int op, int Q_sq, const int x_src[4],
                  double* corrd) {
  tables();
  const cplx* P1 = (const cplx*)p1d;
  const cplx* P2 = (const cplx*)p2d;
  cplx* corr = (cplx*)corrd;
  const long V = orc_volume(L);
  cplx val[3][16];
  int ind[3][4][16], cnt[3] = {0, 0, 0};
  for (int i = 0; i < 3; i++)
    for (int al = 0; al < 4; al++)
      for (int be = 0; be < 4; be++)
        for (int bp = 0; bp < 4; bp++)
          for (int ap = 0; ap < 4; ap++) {
            const cplx t = CG[i][al][be] * CG_bar[i][bp][ap];
            if (norm2c(t) > 1e-3) {
              val[i][cnt[i]] = t;
              ind[i][0][cnt[i]] = al, ind[i][1][cnt[i]] = be, ind[i][2][cnt[i]] = bp, ind[i][3][cnt[i]] = ap;
              cnt[i]++;
            }
          }
  cplx* M = (cplx*)calloc((size_t)V * 48, sizeof(cplx));
#define P(Q, s1, s2, c1, c2) (Q)[v * 144 + (s1) * 36 + (s2) * 9 + (c1) * 3 + (c2)]
  for (long v = 0; v < V; v++)
    for (int i = 0; i < 3; i++)
      for (int g = 0; g < 4; g++)
        for (int gp = 0; gp < 4; gp++) {
          cplx m = 0;
          for (int idx = 0; idx < cnt[i]; idx++) {
            const int al = ind[i][0][idx], be = ind[i][1][idx], bp = ind[i][2][idx], ap = ind[i][3][idx];
            for (int e1 = 0; e1 < 6; e1++) {
              const int a = EPS[e1][0], b = EPS[e1][1], c = EPS[e1][2];
              for (int e2 = 0; e2 < 6; e2++) {
                const int a1 = EPS[e2][0], b1 = EPS[e2][1], c1 = EPS[e2][2];
                const cplx factor = (double)(SGN_EPS[e1] * SGN_EPS[e2]) * val[i][idx];
                if (op == 0) {
                  const cplx t = -P(P1, al, gp, a, c1) * P(P1, be, bp, b, b1) * P(P1, g, ap, c, a1) +
                                 P(P1, al, bp, a, b1) * P(P1, be, gp, b, c1) * P(P1, g, ap, c, a1) +
                                 P(P1, al, gp, a, c1) * P(P1, be, ap, b, a1) * P(P1, g, bp, c, b1) -
                                 P(P1, al, ap, a, a1) * P(P1, be, gp, b, c1) * P(P1, g, bp, c, b1) -
                                 P(P1, al, bp, a, b1) * P(P1, be, ap, b, a1) * P(P1, g, gp, c, c1) +
                                 P(P1, al, ap, a, a1) * P(P1, be, bp, b, b1) * P(P1, g, gp, c, c1);
                  m = m + factor * t;
                } else {
                  const cplx t = -4.0 * P(P1, al, gp, a, c1) * P(P2, be, bp, b, b1) * P(P1, g, ap, c, a1) +
                                 2.0 * P(P1, al, bp, a, b1) * P(P2, be, gp, b, c1) * P(P1, g, ap, c, a1) +
                                 2.0 * P(P1, al, gp, a, c1) * P(P1, be, ap, b, a1) * P(P2, g, bp, c, b1) -
                                 2.0 * P(P1, al, ap, a, a1) * P(P1, be, gp, b, c1) * P(P2, g, bp, c, b1) -
                                 2.0 * P(P1, al, ap, a, a1) * P(P2, be, gp, b, c1) * P(P1, g, bp, c, b1) -
                                 P(P1, al, bp, a, b1) * P(P1, be, ap, b, a1) * P(P2, g, gp, c, c1) +
                                 P(P1, al, ap, a, a1) * P(P1, be, bp, b, b1) * P(P2, g, gp, c, c1) +
                                 4.0 * P(P1, al, ap, a, a1) * P(P2, be, bp, b, b1) * P(P1, g, gp, c, c1);
                  m = m + factor * (1. / 3.) * t;
                }
              }
            }
          }
          M[v * 48 + i * 16 + g * 4 + gp] = m;
        }
#undef P
  int mom[3000];
  const int nmom = orc_momenta(Q_sq, mom, 1000);
  const long V3 = (long)L[0] * L[1] * L[2];
  for (int i = 0; i < 3; i++)
    for (int t = 0; t < L[3]; t++)
      for (int im = 0; im < nmom; im++)
        for (int k = 0; k < 16; k++) {
          cplx s = 0;
          for (int z = 0; z < L[2]; z++)
            for (int y = 0; y < L[1]; y++)
              for (int x = 0; x < L[0]; x++) {
                const long v = t * V3 + x + (long)L[0] * (y + (long)L[1] * z);
                const double th = (((double)mom[3 * im] * (x - x_src[0])) / L[0] +
                                   ((double)mom[3 * im + 1] * (y - x_src[1])) / L[1] +
                                   ((double)mom[3 * im + 2] * (z - x_src[2])) / L[2]) * 2 * REF_PI;
                s = s + M[v * 48 + i * 16 + k] * (cos(th) - _Complex_I * sin(th));
              }
          corr[((long)t * nmom + im) * 48 + i * 16 + k] = s;
        }
  free(M);
  return nmom;
}

/* contractNucleon(prop1, prop2, output, Q_sq, x_src) (lib/lattice_util.cpp:3374-3528):
 * the nucleon two-point function with the explicit C gamma5 table of :3418-3428, per
 * time slice the spin block summed in the reference's order (each colour term as
 * two separate updates) and its Fourier transform; corr[t][imom][gamma][gamma1] are
 * the numbers that function prints. */
int orc_nucleon_2pt(const int L[4], const double* p1d, const double* p2d, int Q_sq, const int x_src[4],
                    double* corrd) {
  const cplx* P1 = (const cplx*)p1d;
  const cplx* P2 = (const cplx*)p2d;
  cplx* corr = (cplx*)corrd;
  cplx cg5[4][4], cg5b[4][4];
  memset(cg5, 0, sizeof cg5);
  memset(cg5b, 0, sizeof cg5b);
  cg5[0][1] = 1, cg5[1][0] = -1, cg5[2][3] = 1, cg5[3][2] = -1;
  cg5b[0][1] = -1, cg5b[1][0] = 1, cg5b[2][3] = -1, cg5b[3][2] = 1;
  cplx val[256];
  int ind[256][4], cnt = 0;
  for (int al = 0; al < 4; al++)
    for (int be = 0; be < 4; be++)
      for (int b1 = 0; b1 < 4; b1++)
        for (int a1 = 0; a1 < 4; a1++) {
          const cplx t = cg5[al][be] * cg5b[b1][a1];
          if (norm2c(t) > 1e-3) {
            val[cnt] = t;
            ind[cnt][0] = al, ind[cnt][1] = be, ind[cnt][2] = b1, ind[cnt][3] = a1;
            cnt++;
          }
        }
  int mom[3000];
  const int nmom = orc_momenta(Q_sq, mom, 1000);
  const long V3 = (long)L[0] * L[1] * L[2];
  cplx* block = (cplx*)calloc((size_t)V3 * 16, sizeof(cplx));
#define P(Q, s1, s2, c1, c2) (Q)[v * 144 + (s1) * 36 + (s2) * 9 + (c1) * 3 + (c2)]
  for (int t = 0; t < L[3]; t++) {
    memset(block, 0, sizeof(cplx) * V3 * 16);
    for (long v3 = 0; v3 < V3; v3++) {
      const long v = t * V3 + v3;
      for (int g = 0; g < 4; g++)
        for (int g1 = 0; g1 < 4; g1++) {
          cplx bl = 0;
          for (int idx = 0; idx < cnt; idx++) {
            const int al = ind[idx][0], be = ind[idx][1], bb1 = ind[idx][2], aa1 = ind[idx][3];
            for (int e1 = 0; e1 < 6; e1++) {
              const int a = EPS[e1][0], b = EPS[e1][1], c = EPS[e1][2];
              for (int e2 = 0; e2 < 6; e2++) {
                const int a1 = EPS[e2][0], b1 = EPS[e2][1], c1 = EPS[e2][2];
                const cplx factor = (double)(SGN_EPS[e1] * SGN_EPS[e2]) * val[idx];
                bl = bl + factor * P(P2, be, bb1, b, b1) * P(P1, al, aa1, a, a1) * P(P1, g, g1, c, c1);
                bl = bl - factor * P(P2, be, bb1, b, b1) * P(P1, al, g1, a, c1) * P(P1, g, aa1, c, a1);
              }
            }
          }
          block[v3 * 16 + g * 4 + g1] = bl;
        }
    }
    for (int im = 0; im < nmom; im++)
      for (int k = 0; k < 16; k++) {
        cplx s = 0;
        for (int z = 0; z < L[2]; z++)
          for (int y = 0; y < L[1]; y++)
            for (int x = 0; x < L[0]; x++) {
              const long v3 = x + (long)L[0] * (y + (long)L[1] * z);
              const double th = (((double)mom[3 * im] * (x - x_src[0])) / L[0] +
                                 ((double)mom[3 * im + 1] * (y - x_src[1])) / L[1] +
                                 ((double)mom[3 * im + 2] * (z - x_src[2])) / L[2]) * 2 * REF_PI;
              s = s + block[v3 * 16 + k] * (cos(th) - _Complex_I * sin(th));
            }
        corr[((long)t * nmom + im) * 16 + k] = s;
      }
  }
#undef P
  free(block);
  return nmom;
}
