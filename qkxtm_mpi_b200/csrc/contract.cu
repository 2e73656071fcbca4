// contract.cu -- meson, nucleon and decuplet two-point functions from propagators
// (lib/contractions.cpp: Meson::contract :251, Baryon::contract :494,
// Baryon_Dec::contract :768, their fourier(FORWARD) :121 / :356 / :703 and
// createMomenta :37; contractNucleon, lib/lattice_util.cpp:3374) on one B200.
//
// A propagator is [V][4][4][3][3] complex in the host layout (Propagator::M).
// Per site the contraction needs the whole site block (2304 bytes per
// propagator), so blocks stage 16 sites' blocks in shared memory with
// coalesced loads and then compute:
//   mesons   one thread per (site, operator)
//   nucleons one thread per (site, gamma, gamma'), each walking the tabulated
//            spin terms of its (gamma, gamma') and the 36 colour permutations.
//   decuplet one thread per (site, i, gamma, gamma'), i the spatial C gamma_i.
// The terms are tabulated on the host in the reference's order (same
// threshold |value|^2 > 1e-3) from the gamma and charge-conjugation matrices
// of lib/lattice_util.cpp:255-305.  The Fourier transform is one block per
// (time slice, momentum) with the reference's phase convention:
//   F[t][p] = sum_x C(x) exp(-2 pi i sum_mu p_mu (x_mu - x_src_mu) / L_mu),
// pi = 3.14159265359 as in lib/contractions.cpp:5, x - x_src not wrapped.
#include <string.h>

#include <algorithm>
#include <complex>
#include <vector>

#include "qkx_ctx.cuh"

using namespace qkx;

namespace qkx {
namespace {

constexpr int CT_SITES = 16;           // sites per block
constexpr int CT_STRIDE = 145;         // double2 per staged site: 144 + 1 of padding, so the 16 sites
                                       // of a warp fall on different shared-memory banks
constexpr double REF_PI = 3.14159265359;
using zc = std::complex<double>;

int bad(const char* what) {
  set_error("invalid argument: %s", what);
  return QKX_ERR_INVALID;
}

// ---------------------------------------------------------------- host tables
struct Gammas {
  zc G[5][4][4], C[4][4], Cbar[4][4], CG[5][4][4], CGbar[5][4][4];
  Gammas() {  // std::complex members start at zero
    const zc j(0, 1);
    G[0][0][3] = j, G[0][1][2] = j, G[0][2][1] = -j, G[0][3][0] = -j;
    G[1][0][3] = 1, G[1][1][2] = -1, G[1][2][1] = -1, G[1][3][0] = 1;
    G[2][0][2] = j, G[2][1][3] = -j, G[2][2][0] = -j, G[2][3][1] = j;
    G[3][0][0] = 1, G[3][1][1] = 1, G[3][2][2] = -1, G[3][3][3] = -1;
    G[4][0][2] = 1, G[4][1][3] = 1, G[4][2][0] = 1, G[4][3][1] = 1;
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++)
        for (int k = 0; k < 4; k++) C[m][n] += G[1][m][k] * G[3][k][n];
    for (int m = 0; m < 4; m++)
      for (int n = 0; n < 4; n++)
        for (int k = 0; k < 4; k++)
          for (int l = 0; l < 4; l++) Cbar[m][n] += G[3][m][l] * std::conj(C[k][l]) * G[3][k][n];
    for (int i = 0; i < 5; i++)
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++)
          for (int k = 0; k < 4; k++) CG[i][m][n] += C[m][k] * G[i][k][n];
    for (int i = 0; i < 5; i++)
      for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++)
          for (int k = 0; k < 4; k++)
            for (int l = 0; l < 4; l++) CGbar[i][m][n] += G[3][m][l] * std::conj(CG[i][k][l]) * G[3][k][n];
  }
};

bool keep(zc v) { return std::norm(v) > 1e-3; }

// ---- mesons: per operator, terms (value; beta, gamma, delta, alpha) in tabulateIndices order
constexpr int MESON_MAX_TERMS = 64;
struct MesonTerms {
  int n;
  double2 val[MESON_MAX_TERMS];
  char4 ind[MESON_MAX_TERMS];  // beta, gamma, delta, alpha
};

void meson_terms(const Gammas& g, int op, MesonTerms& t) {
  zc m[4][4] = {};
  if (op == 0) {
    for (int i = 0; i < 4; i++) m[i][i] = 1;
  } else if (op == 1) {
    memcpy((void*)m, g.G[4], sizeof m);
  } else if (op <= 5) {
    memcpy((void*)m, g.G[op - 2], sizeof m);
  } else {
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++)
        for (int k = 0; k < 4; k++) m[a][b] += g.G[4][a][k] * g.G[op - 6][k][b];
  }
  t.n = 0;
  for (int be = 0; be < 4; be++)
    for (int ga = 0; ga < 4; ga++)
      for (int de = 0; de < 4; de++)
        for (int al = 0; al < 4; al++) {
          const zc v = m[be][ga] * m[de][al];
          if (keep(v) && t.n < MESON_MAX_TERMS) {
            t.val[t.n] = make_double2(v.real(), v.imag());
            t.ind[t.n] = make_char4(be, ga, de, al);
            t.n++;
          }
        }
}

// ---- nucleons: per (gamma, gamma'), terms (value; alpha, beta, beta', alpha', X, Y)
// with X, Y the spins of the third quark's propagator element (see orc_baryon_2pt)
constexpr int BARYON_MAX_TERMS = 64;
struct BaryonTerms {
  int n[16];
  double2 val[16][BARYON_MAX_TERMS];
  char4 ab[16][BARYON_MAX_TERMS];  // alpha, beta, beta', alpha'
  char2 xy[16][BARYON_MAX_TERMS];  // X, Y
};

int baryon_terms(const Gammas& g, int op, BaryonTerms& t) {
  memset(t.n, 0, sizeof t.n);
  auto add = [&](int gg, int gp, zc v, int al, int be, int bp, int ap, int X, int Y) -> int {
    const int k = gg * 4 + gp;
    if (t.n[k] >= BARYON_MAX_TERMS) return QKX_ERR_INVALID;
    t.val[k][t.n[k]] = make_double2(v.real(), v.imag());
    t.ab[k][t.n[k]] = make_char4(al, be, bp, ap);
    t.xy[k][t.n[k]] = make_char2(X, Y);
    t.n[k]++;
    return QKX_OK;
  };
  for (int gg = 0; gg < 4; gg++)
    for (int gp = 0; gp < 4; gp++)
      for (int al = 0; al < 4; al++)
        for (int be = 0; be < 4; be++)
          for (int bp = 0; bp < 4; bp++)
            for (int ap = 0; ap < 4; ap++) {
              if (op == 0) {
                const zc v = g.CG[4][al][be] * g.CGbar[4][bp][ap];
                if (keep(v)) QKX_TRY(add(gg, gp, v, al, be, bp, ap, gg, gp));
              } else if (op == 1) {  // gamma' from the term, delta' the third quark's source spin
                for (int dp = 0; dp < 4; dp++) {
                  const zc v = g.CG[4][al][be] * g.Cbar[bp][ap] * g.G[4][gp][dp];
                  if (keep(v)) QKX_TRY(add(gg, gp, v, al, be, bp, ap, gg, dp));
                }
              } else if (op == 2) {  // gamma from the term, delta the third quark's sink spin
                for (int de = 0; de < 4; de++) {
                  const zc v = g.C[al][be] * g.CGbar[4][bp][ap] * g.G[4][gg][de];
                  if (keep(v)) QKX_TRY(add(gg, gp, v, al, be, bp, ap, de, gp));
                }
              } else {
                for (int de = 0; de < 4; de++)
                  for (int dp = 0; dp < 4; dp++) {
                    const zc v = g.C[al][be] * g.Cbar[bp][ap] * g.G[4][gg][de] * g.G[4][gp][dp];
                    if (keep(v)) QKX_TRY(add(gg, gp, v, al, be, bp, ap, de, dp));
                  }
              }
            }
  return QKX_OK;
}

// The reference accumulates each (gamma, gamma') over its terms in the
// order of the tabulated index list; the loops above visit (alpha, beta,
// beta', alpha') in that list's order and, within it, the free spins in the
// list's order, so each per-(gamma, gamma') list keeps the reference's order.

// ---------------------------------------------------------------- device
__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// stage NS site blocks (144 complex each) of a propagator into shared
// memory, site s at sp + s * CT_STRIDE
template <int NS = CT_SITES>
__device__ __forceinline__ void stage(double2* sp, const double2* __restrict__ prop, size_t s0, size_t V) {
  const size_t base = s0 * 144;
  const int total = NS * 144;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const size_t site = s0 + i / 144;
    sp[(i / 144) * CT_STRIDE + i % 144] = site < V ? __ldg(prop + base + i) : make_double2(0.0, 0.0);
  }
}

// C[op][site], block = CT_SITES sites x nop operators
__global__ void k_meson_sites(const double2* __restrict__ prop, size_t V, int nop, const MesonTerms* __restrict__ T,
                              double2* __restrict__ C) {
  __shared__ double2 sp[CT_SITES * CT_STRIDE];
  const size_t s0 = (size_t)blockIdx.x * CT_SITES;
  stage(sp, prop, s0, V);
  __syncthreads();
  const int ls = threadIdx.x % CT_SITES, o = threadIdx.x / CT_SITES;
  const size_t site = s0 + ls;
  if (o >= nop || site >= V) return;
  const double2* pp = sp + ls * CT_STRIDE;  // [mu][nu][c1][c2] at mu*36 + nu*9 + c1*3 + c2
  const MesonTerms& t = T[o];
  double2 m = make_double2(0.0, 0.0);
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      for (int i = 0; i < t.n; i++) {
        const char4 ix = t.ind[i];  // beta, gamma, delta, alpha
        // (g5 pp^+ g5)[gamma][delta][b][a] = conj(pp[g5(delta)][g5(gamma)][a][b]), g5 swapping spins 0<->2, 1<->3
        const double2 q = pp[((ix.z + 2) & 3) * 36 + ((ix.y + 2) & 3) * 9 + a * 3 + b];
        const double2 v = cm(cm(t.val[i], pp[ix.w * 36 + ix.x * 9 + a * 3 + b]), make_double2(q.x, -q.y));
        m.x += v.x;
        m.y += v.y;
      }
  C[(size_t)o * V + site] = m;
}

// the even then odd permutations of (0, 1, 2) and their signs, in the reference's order
// (lib/contractions.cpp:21-33)
__device__ constexpr int c_eps[6][3] = {{0, 1, 2}, {2, 0, 1}, {1, 2, 0}, {2, 1, 0}, {0, 2, 1}, {1, 0, 2}};
__device__ constexpr int c_sgn[6] = {+1, +1, +1, -1, -1, -1};

// C[gamma*4 + gamma'][site], block = CT_SITES sites x 16 spin pairs
__global__ void __launch_bounds__(CT_SITES * 16) k_baryon_sites(const double2* __restrict__ p1,
                                                                const double2* __restrict__ p2, size_t V, double sign,
                                                                const BaryonTerms* __restrict__ T,
                                                                double2* __restrict__ C) {
  extern __shared__ double2 sb[];
  double2* s1 = sb;
  double2* s2 = sb + CT_SITES * CT_STRIDE;
  const size_t s0 = (size_t)blockIdx.x * CT_SITES;
  stage(s1, p1, s0, V);
  stage(s2, p2, s0, V);
  __syncthreads();
  const int ls = threadIdx.x % CT_SITES, k = threadIdx.x / CT_SITES;
  const size_t site = s0 + ls;
  if (site >= V) return;
  const double2* q1 = s1 + ls * CT_STRIDE;
  const double2* q2 = s2 + ls * CT_STRIDE;
  double2 m = make_double2(0.0, 0.0);
  const int n = T->n[k];
  for (int i = 0; i < n; i++) {
    const double2 val = T->val[k][i];
    const char4 ab = T->ab[k][i];  // alpha, beta, beta', alpha'
    const char2 xy = T->xy[k][i];
    // the five colour matrices of the term, read once
    double2 A[9], B[9], Cm[9], D[9], E[9];
#pragma unroll
    for (int u = 0; u < 9; u++) {
      A[u] = q1[ab.x * 36 + ab.w * 9 + u];   // P1[alpha][alpha']
      B[u] = q1[xy.x * 36 + xy.y * 9 + u];   // P1[X][Y]
      Cm[u] = q1[ab.x * 36 + xy.y * 9 + u];  // P1[alpha][Y]
      D[u] = q1[xy.x * 36 + ab.w * 9 + u];   // P1[X][alpha']
      E[u] = q2[ab.y * 36 + ab.z * 9 + u];   // P2[beta][beta']
    }
#pragma unroll
    for (int e1 = 0; e1 < 6; e1++) {
      const int a = c_eps[e1][0], b = c_eps[e1][1], c = c_eps[e1][2];
#pragma unroll
      for (int e2 = 0; e2 < 6; e2++) {
        const int a1 = c_eps[e2][0], b1 = c_eps[e2][1], c1 = c_eps[e2][2];
        const double f = (double)(c_sgn[e1] * c_sgn[e2]);
        const double2 fv = make_double2(f * val.x, f * val.y);
        const double2 x1 = cm(A[a * 3 + a1], B[c * 3 + c1]);
        const double2 x2 = cm(Cm[a * 3 + c1], D[c * 3 + a1]);
        const double2 t = cm(cm(fv, E[b * 3 + b1]), make_double2(x1.x - x2.x, x1.y - x2.y));
        m.x += sign * t.x;
        m.y += sign * t.y;
      }
    }
  }
  C[(size_t)k * V + site] = m;
}

// ---- decuplet (Baryon_Dec): per spatial i, the terms (value; alpha, beta, beta', alpha')
// of (C gamma_i)[alpha][beta] (C gamma_i)bar[beta'][alpha'] in tabulateIndices_Delta's
// order (lib/contractions.cpp:743-765)
constexpr int DELTA_MAX_TERMS = 64;
struct DeltaTerms {
  int n[3];
  double2 val[3][DELTA_MAX_TERMS];
  char4 ab[3][DELTA_MAX_TERMS];  // alpha, beta, beta', alpha'
};

int delta_terms(const Gammas& g, DeltaTerms& t) {
  memset(t.n, 0, sizeof t.n);
  for (int i = 0; i < 3; i++)
    for (int al = 0; al < 4; al++)
      for (int be = 0; be < 4; be++)
        for (int bp = 0; bp < 4; bp++)
          for (int ap = 0; ap < 4; ap++) {
            const zc v = g.CG[i][al][be] * g.CGbar[i][bp][ap];
            if (!keep(v)) continue;
            if (t.n[i] >= DELTA_MAX_TERMS) return QKX_ERR_INVALID;
            t.val[i][t.n[i]] = make_double2(v.real(), v.imag());
            t.ab[i][t.n[i]] = make_char4(al, be, bp, ap);
            t.n[i]++;
          }
  return QKX_OK;
}

constexpr int DT_SITES = 8;  // sites per block of the decuplet kernel (48 threads a site)

// The six permutations (a, b, c) of lib/contractions.cpp:14-19 in their order, two bits a
// colour, six bits a permutation, as one constant (no table in memory); sign +1 for the first
// three, -1 for the others.
constexpr unsigned long long EPS_PACKED =
    (0ull | 1ull << 2 | 2ull << 4) | (2ull | 0ull << 2 | 1ull << 4) << 6 | (1ull | 2ull << 2 | 0ull << 4) << 12 |
    (2ull | 1ull << 2 | 0ull << 4) << 18 | (0ull | 2ull << 2 | 1ull << 4) << 24 | (1ull | 0ull << 2 | 2ull << 4) << 30;
__device__ __forceinline__ int eps_at(int e, int j) { return (int)((EPS_PACKED >> (6 * e + 2 * j)) & 3ull); }

// C[i*16 + gamma*4 + gamma'][site] of Baryon_Dec::contract (lib/contractions.cpp:768-866):
// one thread per (site, i, gamma, gamma'); op 0 DELTA_ISO1 (three quarks of p1),
// 1 DELTA_ISO1O2 (p2 for the odd quark, the reference's weights 1/3 x {4, 2, 1}).
// Each term reads its colour entries from the staged site blocks.
// Every index the kernel takes from its term table is checked before use: a value out of range
// records a code in *err and the term is skipped, so a bad table cannot address outside the
// staged blocks.
__global__ void __launch_bounds__(DT_SITES * 48) k_delta_sites(const double2* __restrict__ p1,
                                                               const double2* __restrict__ p2, size_t V, int op,
                                                               const DeltaTerms* __restrict__ T,
                                                               double2* __restrict__ C, int* __restrict__ err) {
  extern __shared__ double2 sb[];
  double2* s1 = sb;
  double2* s2 = sb + DT_SITES * CT_STRIDE;
  const size_t s0 = (size_t)blockIdx.x * DT_SITES;
  stage<DT_SITES>(s1, p1, s0, V);
  stage<DT_SITES>(s2, p2, s0, V);
  __syncthreads();
  const int ls = threadIdx.x % DT_SITES, k = threadIdx.x / DT_SITES;  // k = i*16 + gamma*4 + gamma'
  const size_t site = s0 + ls;
  if (site >= V) return;
  const int i = k >> 4, g = (k >> 2) & 3, gp = k & 3;
  const double2* q1 = s1 + ls * CT_STRIDE;
  const double2* q2 = s2 + ls * CT_STRIDE;
  // entry [s1][s2][c1][c2] of propagator q
  auto at = [](const double2* q, int sa, int sb_, int ca, int cb) { return q[sa * 36 + sb_ * 9 + ca * 3 + cb]; };
  double2 m = make_double2(0.0, 0.0);
  int n = T->n[i];
  if (n < 0 || n > DELTA_MAX_TERMS) {
    atomicCAS(err, 0, 1000 + n);
    n = 0;
  }
  for (int idx = 0; idx < n; idx++) {
    const double2 val = T->val[i][idx];
    const char4 ab = T->ab[i][idx];
    const int al = ab.x, be = ab.y, bp = ab.z, ap = ab.w;
    if ((unsigned)al > 3u || (unsigned)be > 3u || (unsigned)bp > 3u || (unsigned)ap > 3u) {
      atomicCAS(err, 0, 2000 + idx);
      continue;
    }
    for (int e1 = 0; e1 < 6; e1++) {
      const int a = eps_at(e1, 0), b = eps_at(e1, 1), c = eps_at(e1, 2);
      for (int e2 = 0; e2 < 6; e2++) {
        const int a1 = eps_at(e2, 0), b1 = eps_at(e2, 1), c1 = eps_at(e2, 2);
        const double f = (e1 < 3) == (e2 < 3) ? 1.0 : -1.0;
        double2 t;
        if (op == 0) {
          const double2 t1 = cm(cm(at(q1, al, gp, a, c1), at(q1, be, bp, b, b1)), at(q1, g, ap, c, a1));
          const double2 t2 = cm(cm(at(q1, al, bp, a, b1), at(q1, be, gp, b, c1)), at(q1, g, ap, c, a1));
          const double2 t3 = cm(cm(at(q1, al, gp, a, c1), at(q1, be, ap, b, a1)), at(q1, g, bp, c, b1));
          const double2 t4 = cm(cm(at(q1, al, ap, a, a1), at(q1, be, gp, b, c1)), at(q1, g, bp, c, b1));
          const double2 t5 = cm(cm(at(q1, al, bp, a, b1), at(q1, be, ap, b, a1)), at(q1, g, gp, c, c1));
          const double2 t6 = cm(cm(at(q1, al, ap, a, a1), at(q1, be, bp, b, b1)), at(q1, g, gp, c, c1));
          t = make_double2(-t1.x + t2.x + t3.x - t4.x - t5.x + t6.x, -t1.y + t2.y + t3.y - t4.y - t5.y + t6.y);
        } else {
          const double2 t1 = cm(cm(at(q1, al, gp, a, c1), at(q2, be, bp, b, b1)), at(q1, g, ap, c, a1));
          const double2 t2 = cm(cm(at(q1, al, bp, a, b1), at(q2, be, gp, b, c1)), at(q1, g, ap, c, a1));
          const double2 t3 = cm(cm(at(q1, al, gp, a, c1), at(q1, be, ap, b, a1)), at(q2, g, bp, c, b1));
          const double2 t4 = cm(cm(at(q1, al, ap, a, a1), at(q1, be, gp, b, c1)), at(q2, g, bp, c, b1));
          const double2 t5 = cm(cm(at(q1, al, ap, a, a1), at(q2, be, gp, b, c1)), at(q1, g, bp, c, b1));
          const double2 t6 = cm(cm(at(q1, al, bp, a, b1), at(q1, be, ap, b, a1)), at(q2, g, gp, c, c1));
          const double2 t7 = cm(cm(at(q1, al, ap, a, a1), at(q1, be, bp, b, b1)), at(q2, g, gp, c, c1));
          const double2 t8 = cm(cm(at(q1, al, ap, a, a1), at(q2, be, bp, b, b1)), at(q1, g, gp, c, c1));
          const double third = 1.0 / 3.0;
          t = make_double2(third * (-4 * t1.x + 2 * t2.x + 2 * t3.x - 2 * t4.x - 2 * t5.x - t6.x + t7.x + 4 * t8.x),
                           third * (-4 * t1.y + 2 * t2.y + 2 * t3.y - 2 * t4.y - 2 * t5.y - t6.y + t7.y + 4 * t8.y));
        }
        const double2 v = cm(make_double2(f * val.x, f * val.y), t);
        m.x += v.x;
        m.y += v.y;
      }
    }
  }
  C[(size_t)k * V + site] = m;
}

// F[t][p][k] = sum over the slice's sites of C[k][site] exp(-i theta), one block per (t, p)
__global__ void k_fourier(const double2* __restrict__ C, int K, size_t V, const int* __restrict__ mom, int nmom,
                          Geom g, int4 src, double2* __restrict__ F) {
  const int t = blockIdx.x / nmom, p = blockIdx.x % nmom;
  const int V3 = g.L[0] * g.L[1] * g.L[2];
  const int nx = mom[3 * p], ny = mom[3 * p + 1], nz = mom[3 * p + 2];
  double re[16], im[16];
#pragma unroll
  for (int k = 0; k < 16; k++) re[k] = im[k] = 0.0;
  for (int s = threadIdx.x; s < V3; s += blockDim.x) {
    const int x = s % g.L[0], y = (s / g.L[0]) % g.L[1], z = s / (g.L[0] * g.L[1]);
    const double th =
        (((double)nx * (x - src.x)) / g.L[0] + ((double)ny * (y - src.y)) / g.L[1] + ((double)nz * (z - src.z)) / g.L[2]) *
        2 * REF_PI;
    double sn, cs;
    sincos(th, &sn, &cs);
    const size_t v = (size_t)t * V3 + s;
#pragma unroll
    for (int k = 0; k < 16; k++) {
      if (k >= K) break;
      const double2 c = C[(size_t)k * V + v];
      re[k] += c.x * cs + c.y * sn;  // c * (cos - i sin)
      im[k] += c.y * cs - c.x * sn;
    }
  }
  for (int k = 0; k < K; k++) {
    const double r = block_sum<256>(re[k]);
    const double i = block_sum<256>(im[k]);
    if (threadIdx.x == 0) F[((size_t)t * nmom + p) * K + k] = make_double2(r, i);
  }
}

int host_momenta(int Q_sq, std::vector<int>& m) {
  m.clear();
  for (int q = 0; q <= Q_sq; q++)
    for (int nx = q; nx >= -q; nx--)
      for (int ny = q; ny >= -q; ny--)
        for (int nz = q; nz >= -q; nz--)
          if (nx * nx + ny * ny + nz * nz == q) m.insert(m.end(), {nx, ny, nz});
  return (int)(m.size() / 3);
}

// a device copy of a host propagator (or the pointer itself for device input)
struct PropIn {
  const double2* d = nullptr;
  void* owned = nullptr;
};

int prop_in(qkx_ctx* c, const double* p, bool host, PropIn& out) {
  if (!host) {
    out.d = (const double2*)p;
    return QKX_OK;
  }
  const size_t bytes = sizeof(double2) * 144 * c->V;
  if (cudaMallocAsync(&out.owned, bytes, c->st) != cudaSuccess) {
    cudaGetLastError();
    set_error("propagator copy: device allocation failed");
    return QKX_ERR_NOMEM;
  }
  QKX_CUDA(cudaMemcpyAsync(out.owned, p, bytes, cudaMemcpyHostToDevice, c->st));
  out.d = (const double2*)out.owned;
  return QKX_OK;
}

// run the Fourier transform of C [K][V] and return F [Lt][nmom][K] to the host
int fourier_to_host(qkx_ctx* c, const double2* C, int K, int Q_sq, const int x_src[4], double* out, int* nmom_out) {
  std::vector<int> m;
  const int nmom = host_momenta(Q_sq, m);
  if (nmom > 1000) return bad("Q_sq gives more than 1000 momenta (MOM_MAX)");
  int* dm = nullptr;
  double2* F = nullptr;
  const size_t nf = (size_t)c->p.L[3] * nmom * K;
  QKX_CUDA(cudaMallocAsync((void**)&dm, sizeof(int) * m.size(), c->st));
  QKX_CUDA(cudaMallocAsync((void**)&F, sizeof(double2) * nf, c->st));
  QKX_CUDA(cudaMemcpyAsync(dm, m.data(), sizeof(int) * m.size(), cudaMemcpyHostToDevice, c->st));
  k_fourier<<<c->p.L[3] * nmom, 256, 0, c->st>>>(C, K, c->V, dm, nmom, c->geom,
                                                 make_int4(x_src[0], x_src[1], x_src[2], x_src[3]), F);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaMemcpyAsync(out, F, sizeof(double2) * nf, cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaFreeAsync(dm, c->st));
  QKX_CUDA(cudaFreeAsync(F, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  if (nmom_out) *nmom_out = nmom;
  return QKX_OK;
}

int meson_2pt(qkx_ctx* c, const double* prop, bool host, int nop, const int* ops, int Q_sq, const int x_src[4],
              double* corr) {
  if (!c || !prop || !ops || !x_src || !corr) return bad("NULL argument");
  if (nop < 1 || nop > QKX_NUM_MESONS) return bad("nop must be in 1..10");
  for (int i = 0; i < nop; i++)
    if (ops[i] < 0 || ops[i] >= QKX_NUM_MESONS) return bad("meson operator id");
  if (Q_sq < 0) return bad("Q_sq < 0");
  QKX_CUDA(cudaSetDevice(c->device));
  static const Gammas g;
  std::vector<MesonTerms> T(nop);
  for (int i = 0; i < nop; i++) meson_terms(g, ops[i], T[i]);
  PropIn pin;
  QKX_TRY(prop_in(c, prop, host, pin));
  MesonTerms* dT = nullptr;
  double2* C = nullptr;
  QKX_CUDA(cudaMallocAsync((void**)&dT, sizeof(MesonTerms) * nop, c->st));
  QKX_CUDA(cudaMallocAsync((void**)&C, sizeof(double2) * nop * c->V, c->st));
  QKX_CUDA(cudaMemcpyAsync(dT, T.data(), sizeof(MesonTerms) * nop, cudaMemcpyHostToDevice, c->st));
  const unsigned nb = (unsigned)((c->V + CT_SITES - 1) / CT_SITES);
  k_meson_sites<<<nb, CT_SITES * QKX_NUM_MESONS, 0, c->st>>>(pin.d, c->V, nop, dT, C);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  // Fourier per operator: K = 1 each, laid out [op][Lt][Nmom]
  std::vector<int> m;
  const int nmom = host_momenta(Q_sq, m);
  int rc = QKX_OK;
  for (int i = 0; i < nop && rc == QKX_OK; i++)
    rc = fourier_to_host(c, C + (size_t)i * c->V, 1, Q_sq, x_src, corr + (size_t)i * 2 * c->p.L[3] * nmom, nullptr);
  cudaFreeAsync(dT, c->st);
  cudaFreeAsync(C, c->st);
  if (pin.owned) cudaFreeAsync(pin.owned, c->st);
  cudaStreamSynchronize(c->st);
  return rc;
}

int baryon_2pt(qkx_ctx* c, const double* p1, const double* p2, bool host, int op, int Q_sq, const int x_src[4],
               double* corr) {
  if (!c || !p1 || !p2 || !x_src || !corr) return bad("NULL argument");
  if (op < 0 || op > 3) return bad("baryon operator id");
  if (Q_sq < 0) return bad("Q_sq < 0");
  QKX_CUDA(cudaSetDevice(c->device));
  static const Gammas g;
  BaryonTerms T;
  if (baryon_terms(g, op, T) != QKX_OK) return bad("internal: too many spin terms");
  PropIn a, b;
  QKX_TRY(prop_in(c, p1, host, a));
  QKX_TRY(prop_in(c, p2, host, b));
  BaryonTerms* dT = nullptr;
  double2* C = nullptr;
  QKX_CUDA(cudaMallocAsync((void**)&dT, sizeof(BaryonTerms), c->st));
  QKX_CUDA(cudaMallocAsync((void**)&C, sizeof(double2) * 16 * c->V, c->st));
  QKX_CUDA(cudaMemcpyAsync(dT, &T, sizeof(BaryonTerms), cudaMemcpyHostToDevice, c->st));
  static bool attr = false;
  const int smem = (int)(sizeof(double2) * 2 * CT_SITES * CT_STRIDE);
  if (!attr) {
    QKX_CUDA(cudaFuncSetAttribute(k_baryon_sites, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  const unsigned nb = (unsigned)((c->V + CT_SITES - 1) / CT_SITES);
  const double sign = (op == 1 || op == 3) ? -1.0 : 1.0;
  k_baryon_sites<<<nb, CT_SITES * 16, smem, c->st>>>(a.d, b.d, c->V, sign, dT, C);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  // F is [Lt][Nmom][16] = Baryon::F [Lt][Nmom][4][4]
  const int rc = fourier_to_host(c, C, 16, Q_sq, x_src, corr, nullptr);
  cudaFreeAsync(dT, c->st);
  cudaFreeAsync(C, c->st);
  if (a.owned) cudaFreeAsync(a.owned, c->st);
  if (b.owned) cudaFreeAsync(b.owned, c->st);
  cudaStreamSynchronize(c->st);
  return rc;
}

int delta_2pt(qkx_ctx* c, const double* p1, const double* p2, bool host, int op, int Q_sq, const int x_src[4],
              double* corr) {
  if (!c || !p1 || !p2 || !x_src || !corr) return bad("NULL argument");
  if (op < 0 || op > 1) return bad("decuplet operator id (0 DELTA_ISO1, 1 DELTA_ISO1O2)");
  if (Q_sq < 0) return bad("Q_sq < 0");
  QKX_CUDA(cudaSetDevice(c->device));
  static const Gammas g;
  DeltaTerms T;
  if (delta_terms(g, T) != QKX_OK) return bad("internal: too many spin terms");
  std::vector<int> mv;
  const int nmom = host_momenta(Q_sq, mv);
  if (nmom > 1000) return bad("Q_sq gives more than 1000 momenta (MOM_MAX)");
  PropIn a, b;
  QKX_TRY(prop_in(c, p1, host, a));
  QKX_TRY(prop_in(c, p2, host, b));
  DeltaTerms* dT = nullptr;
  double2* C = nullptr;
  int* derr = nullptr;
  QKX_CUDA(cudaMallocAsync((void**)&dT, sizeof(DeltaTerms), c->st));
  QKX_CUDA(cudaMallocAsync((void**)&C, sizeof(double2) * 48 * c->V, c->st));
  QKX_CUDA(cudaMallocAsync((void**)&derr, sizeof(int), c->st));
  QKX_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), c->st));
  QKX_CUDA(cudaMemcpyAsync(dT, &T, sizeof(DeltaTerms), cudaMemcpyHostToDevice, c->st));
  static bool attr = false;
  const int smem = (int)(sizeof(double2) * 2 * DT_SITES * CT_STRIDE);
  if (!attr) {
    QKX_CUDA(cudaFuncSetAttribute(k_delta_sites, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  const unsigned nb = (unsigned)((c->V + DT_SITES - 1) / DT_SITES);
  k_delta_sites<<<nb, DT_SITES * 48, smem, c->st>>>(a.d, b.d, c->V, op, dT, C, derr);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  int herr = 0;
  QKX_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  cudaFreeAsync(derr, c->st);
  if (herr != 0) {
    set_error("decuplet kernel: bad spin-term table entry (code %d)", herr);
    cudaFreeAsync(dT, c->st);
    cudaFreeAsync(C, c->st);
    if (a.owned) cudaFreeAsync(a.owned, c->st);
    if (b.owned) cudaFreeAsync(b.owned, c->st);
    cudaStreamSynchronize(c->st);
    return QKX_ERR_CUDA;
  }
  // Baryon_Dec::F is [Lt][Nmom][3][4][4]: one transform of 16 components per i, interleaved
  const size_t per = (size_t)c->p.L[3] * nmom * 16;
  std::vector<double> tmp(2 * per);
  int rc = QKX_OK;
  for (int i = 0; i < 3 && rc == QKX_OK; i++) {
    rc = fourier_to_host(c, C + (size_t)i * 16 * c->V, 16, Q_sq, x_src, tmp.data(), nullptr);
    for (size_t tp = 0; rc == QKX_OK && tp < (size_t)c->p.L[3] * nmom; tp++)
      memcpy(corr + 2 * (tp * 48 + i * 16), tmp.data() + 2 * tp * 16, sizeof(double) * 32);
  }
  cudaFreeAsync(dT, c->st);
  cudaFreeAsync(C, c->st);
  if (a.owned) cudaFreeAsync(a.owned, c->st);
  if (b.owned) cudaFreeAsync(b.owned, c->st);
  cudaStreamSynchronize(c->st);
  return rc;
}

}  // namespace
}  // namespace qkx

extern "C" {

int qkx_momenta(int Q_sq, int* mom, int max) {
  if (Q_sq < 0) return bad("Q_sq < 0");
  std::vector<int> m;
  const int n = host_momenta(Q_sq, m);
  if (mom)
    for (int i = 0; i < std::min(n, max) * 3; i++) mom[i] = m[i];
  return n;
}

int qkx_meson_2pt(qkx_ctx* c, const double* prop_host, int nop, const int* ops, int Q_sq, const int x_src[4],
                  double* corr) {
  return meson_2pt(c, prop_host, true, nop, ops, Q_sq, x_src, corr);
}
int qkx_meson_2pt_dev(qkx_ctx* c, const double* prop_dev, int nop, const int* ops, int Q_sq, const int x_src[4],
                      double* corr) {
  return meson_2pt(c, prop_dev, false, nop, ops, Q_sq, x_src, corr);
}
int qkx_baryon_2pt(qkx_ctx* c, const double* prop1_host, const double* prop2_host, int op, int Q_sq,
                   const int x_src[4], double* corr) {
  return baryon_2pt(c, prop1_host, prop2_host, true, op, Q_sq, x_src, corr);
}
int qkx_baryon_2pt_dev(qkx_ctx* c, const double* prop1_dev, const double* prop2_dev, int op, int Q_sq,
                       const int x_src[4], double* corr) {
  return baryon_2pt(c, prop1_dev, prop2_dev, false, op, Q_sq, x_src, corr);
}
int qkx_delta_2pt(qkx_ctx* c, const double* prop1_host, const double* prop2_host, int op, int Q_sq,
                  const int x_src[4], double* corr) {
  return delta_2pt(c, prop1_host, prop2_host, true, op, Q_sq, x_src, corr);
}
int qkx_delta_2pt_dev(qkx_ctx* c, const double* prop1_dev, const double* prop2_dev, int op, int Q_sq,
                      const int x_src[4], double* corr) {
  return delta_2pt(c, prop1_dev, prop2_dev, false, op, Q_sq, x_src, corr);
}
// contractNucleon's spin terms (its explicit C gamma5 table, lib/lattice_util.cpp:3418-3428,
// times the table's bar) are Baryon::contract NTN's term for term: C gamma5 there is minus
// the C gamma_5 of the constructor's tables, and the signs cancel in the product
int qkx_nucleon_2pt(qkx_ctx* c, const double* prop1_host, const double* prop2_host, int Q_sq, const int x_src[4],
                    double* corr) {
  return baryon_2pt(c, prop1_host, prop2_host, true, 0, Q_sq, x_src, corr);
}
int qkx_nucleon_2pt_dev(qkx_ctx* c, const double* prop1_dev, const double* prop2_dev, int Q_sq,
                        const int x_src[4], double* corr) {
  return baryon_2pt(c, prop1_dev, prop2_dev, false, 0, Q_sq, x_src, corr);
}

}  // extern "C"
