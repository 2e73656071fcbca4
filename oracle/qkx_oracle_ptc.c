/*
 * qkx_oracle_ptc.c -- CPU oracle of the learned preconditioner: a linear,
 * gauge-covariant parallel-transport convolution (PTC) network, its loss on a
 * (residual, error) pair and the loss gradient with respect to the weights.
 *
 * TEST INFRASTRUCTURE ONLY (see qkx_oracle.h).  Plain C99, FP64, serial.
 * The network has no counterpart in the reference; this file is the
 * project-written restatement that the GPU's forward and backward kernels are
 * checked against (values and finite-difference gradients).
 *
 * Fields.  A layer activation with C channels is [V][C][3] complex (site LEXIC,
 * channel, colour); a spinor [V][4][3] is the same array with C = 4, so the
 * network maps a spinor to a spinor.
 *
 * Paths.  p = 0 is the identity; p = 1 + 2 mu transports from x + mu,
 * (T a)(x) = U_mu(x) a(x + mu); p = 2 + 2 mu from x - mu,
 * (T a)(x) = U_mu(x - mu)^dag a(x - mu).  U is used as given (with the
 * boundary sign when the caller applied it), and T_{1+2mu}^dag = T_{2+2mu}.
 *
 * Layer l maps C_l to C_{l+1} channels:
 *   a_{l+1}[x][c] = sum_p sum_c' W_l[p][c][c'] (T_p a_l[.][c'])(x)
 * with complex weights W_l [9][C_{l+1}][C_l], layers stored one after another.
 *
 * Loss on a pair (r, e):  L = |N(r) - e|^2 / |e|^2.  The gradient returned is
 * dL/dW^* (Wirtinger): dL = 2 Re sum conj(dL/dW^*) dW, so the derivative of L
 * with respect to Re W is 2 Re(dL/dW^*) and with respect to Im W is 2 Im(dL/dW^*).
 */
#include "qkx_oracle.h"

#include <complex.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

/* Optional BF16 storage of the activations between layers, as the GPU keeps them:
 * when on, every hidden activation (the output of layers 0..nlayers-2) and every
 * activation gradient between layers is rounded to BF16 (round to nearest even,
 * from its FP32 value) after it is computed; the arithmetic stays FP64. */
static int act_bf16 = 0;
void orc_ptc_act_bf16(int on) { act_bf16 = on; }

static double bf16_round(double v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) { /* finite: add half an ulp (ties to even), truncate */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
  }
  memcpy(&f, &u, 4);
  return (double)f;
}

static void round_field(cplx* a, long n) {
  if (!act_bf16) return;
  for (long i = 0; i < n; i++) a[i] = bf16_round(creal(a[i])) + I * bf16_round(cimag(a[i]));
}

static long nbr(const int L[4], long s, int mu, int d) {
  int c[4];
  long t = s;
  c[0] = (int)(t % L[0]); t /= L[0];
  c[1] = (int)(t % L[1]); t /= L[1];
  c[2] = (int)(t % L[2]); t /= L[2];
  c[3] = (int)t;
  c[mu] = (c[mu] + d + L[mu]) % L[mu];
  return (long)c[0] + (long)L[0] * (c[1] + (long)L[1] * (c[2] + (long)L[2] * c[3]));
}

/* s = T_p a for channel c of a [V][C][3] field, at site x */
static void transport(const int L[4], const cplx* U, const cplx* a, int C, int c, long x, int p, cplx s[3]) {
  if (p == 0) {
    for (int i = 0; i < 3; i++) s[i] = a[(x * C + c) * 3 + i];
    return;
  }
  const int mu = (p - 1) / 2;
  if ((p - 1) % 2 == 0) {
    const long y = nbr(L, x, mu, 1);
    const cplx* u = U + (x * 4 + mu) * 9;
    const cplx* v = a + (y * C + c) * 3;
    for (int i = 0; i < 3; i++) s[i] = u[i * 3] * v[0] + u[i * 3 + 1] * v[1] + u[i * 3 + 2] * v[2];
  } else {
    const long y = nbr(L, x, mu, -1);
    const cplx* u = U + (y * 4 + mu) * 9;
    const cplx* v = a + (y * C + c) * 3;
    for (int i = 0; i < 3; i++) s[i] = conj(u[i]) * v[0] + conj(u[3 + i]) * v[1] + conj(u[6 + i]) * v[2];
  }
}

static long weights_per_layer(const int* ch, int l) { return 9L * ch[l + 1] * ch[l]; }

long orc_ptc_nweights(int nlayers, const int* ch) {
  long n = 0;
  for (int l = 0; l < nlayers; l++) n += weights_per_layer(ch, l);
  return n;
}

/* one layer: out [V][Co][3] = sum_p W[p] T_p in [V][Ci][3] */
static void layer(const int L[4], const cplx* U, const cplx* W, int Ci, int Co, const cplx* in, cplx* out) {
  const long V = orc_volume(L);
  for (long x = 0; x < V; x++) {
    cplx* o = out + x * Co * 3;
    memset(o, 0, sizeof(cplx) * Co * 3);
    for (int p = 0; p < 9; p++)
      for (int cp = 0; cp < Ci; cp++) {
        cplx s[3];
        transport(L, U, in, Ci, cp, x, p, s);
        for (int c = 0; c < Co; c++) {
          const cplx w = W[((long)p * Co + c) * Ci + cp];
          for (int i = 0; i < 3; i++) o[c * 3 + i] += w * s[i];
        }
      }
  }
}

/* out = N(in); in and out are spinors [V][4][3] (ch[0] == ch[nlayers] == 4 for a
 * preconditioner, any widths otherwise).  acts, if not NULL, receives every
 * layer's input activation, layer after layer ([V][ch[l]][3] each). */
void orc_ptc_forward(const int L[4], const double* Ud, int nlayers, const int* ch, const double* Wd,
                     const double* in, double* out, double* acts) {
  const long V = orc_volume(L);
  const cplx* U = (const cplx*)Ud;
  const cplx* W = (const cplx*)Wd;
  int cmax = 0;
  for (int l = 0; l <= nlayers; l++) cmax = ch[l] > cmax ? ch[l] : cmax;
  cplx* a = (cplx*)malloc(sizeof(cplx) * V * cmax * 3);
  cplx* b = (cplx*)malloc(sizeof(cplx) * V * cmax * 3);
  memcpy(a, in, sizeof(cplx) * V * ch[0] * 3);
  cplx* store = (cplx*)acts;
  for (int l = 0; l < nlayers; l++) {
    if (store) {
      memcpy(store, a, sizeof(cplx) * V * ch[l] * 3);
      store += V * ch[l] * 3;
    }
    layer(L, U, W, ch[l], ch[l + 1], a, b);
    if (l < nlayers - 1) round_field(b, V * ch[l + 1] * 3);
    W += weights_per_layer(ch, l);
    cplx* t = a;
    a = b;
    b = t;
  }
  memcpy(out, a, sizeof(cplx) * V * ch[nlayers] * 3);
  free(a);
  free(b);
}

/* L = |N(r) - e|^2 / |e|^2 and, if grad is not NULL, dL/dW^* in the layout of W. */
double orc_ptc_loss_grad(const int L[4], const double* Ud, int nlayers, const int* ch, const double* Wd,
                         const double* r, const double* ed, double* grad) {
  const long V = orc_volume(L);
  const cplx* U = (const cplx*)Ud;
  const cplx* W = (const cplx*)Wd;
  const cplx* e = (const cplx*)ed;
  long nact = 0;
  int cmax = 0;
  for (int l = 0; l < nlayers; l++) nact += V * ch[l] * 3;
  for (int l = 0; l <= nlayers; l++) cmax = ch[l] > cmax ? ch[l] : cmax;
  cplx* acts = (cplx*)malloc(sizeof(cplx) * nact);
  cplx* y = (cplx*)malloc(sizeof(cplx) * V * ch[nlayers] * 3);
  orc_ptc_forward(L, Ud, nlayers, ch, Wd, r, (double*)y, (double*)acts);
  double e2 = 0, d2 = 0;
  const long ny = V * ch[nlayers] * 3;
  for (long i = 0; i < ny; i++) {
    e2 += creal(e[i]) * creal(e[i]) + cimag(e[i]) * cimag(e[i]);
    const cplx d = y[i] - e[i];
    d2 += creal(d) * creal(d) + cimag(d) * cimag(d);
  }
  const double loss = d2 / e2;
  if (grad) {
    cplx* g = (cplx*)malloc(sizeof(cplx) * V * cmax * 3);
    cplx* h = (cplx*)malloc(sizeof(cplx) * V * cmax * 3);
    for (long i = 0; i < ny; i++) g[i] = (y[i] - e[i]) / e2;
    long woff = orc_ptc_nweights(nlayers, ch);
    long aoff = nact;
    for (int l = nlayers - 1; l >= 0; l--) {
      const int Ci = ch[l], Co = ch[l + 1];
      woff -= weights_per_layer(ch, l);
      aoff -= V * Ci * 3;
      const cplx* a = acts + aoff;
      const cplx* Wl = W + woff;
      cplx* G = (cplx*)grad + woff;
      memset(G, 0, sizeof(cplx) * weights_per_layer(ch, l));
      for (long x = 0; x < V; x++)
        for (int p = 0; p < 9; p++)
          for (int cp = 0; cp < Ci; cp++) {
            cplx s[3];
            transport(L, U, a, Ci, cp, x, p, s);
            for (int c = 0; c < Co; c++) {
              const cplx* gy = g + (x * Co + c) * 3;
              G[((long)p * Co + c) * Ci + cp] += gy[0] * conj(s[0]) + gy[1] * conj(s[1]) + gy[2] * conj(s[2]);
            }
          }
      if (l == 0) break;
      /* h[c'] = sum_p sum_c conj(W[p][c][c']) (T_{-p} g[c]) */
      for (long x = 0; x < V; x++) {
        cplx* o = h + x * Ci * 3;
        memset(o, 0, sizeof(cplx) * Ci * 3);
        for (int p = 0; p < 9; p++) {
          const int q = p == 0 ? 0 : (p % 2 == 1 ? p + 1 : p - 1);
          for (int c = 0; c < Co; c++) {
            cplx s[3];
            transport(L, U, g, Co, c, x, q, s);
            for (int cp = 0; cp < Ci; cp++) {
              const cplx w = conj(Wl[((long)p * Co + c) * Ci + cp]);
              for (int i = 0; i < 3; i++) o[cp * 3 + i] += w * s[i];
            }
          }
        }
      }
      round_field(h, V * Ci * 3);
      cplx* t = g;
      g = h;
      h = t;
    }
    free(g);
    free(h);
  }
  free(acts);
  free(y);
  return loss;
}
