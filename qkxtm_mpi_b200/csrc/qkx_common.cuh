// qkx_common.cuh -- device building blocks for the twisted-mass Wilson operator
// on sm_100a: complex arithmetic, compile-time gamma tables, half-spinor
// projection/reconstruction, even-odd site geometry and the per-precision
// field accessors.
//
// Device field layouts (all structure-of-arrays, site index fastest so a warp
// reads 32 consecutive sites with one 128-bit load per component group):
//   spinor  [parity][G][Vh] of a 16-byte word, G words per site:
//             FP64: 12 x double2 (one complex each)
//             FP32:  6 x float4  (two complex each)
//             FP16:  3 x uint4   (four complex each as half2) + float norm [parity][Vh]
//   gauge   [parity][dir][W][Vh], dir 0..3 = x y z t, a link U_mu(x) stored with
//           the parity of x.  18-real: the full 3x3; 12-real: rows 0 and 1 with
//           row 2 rebuilt as conj(row0 x row1) (exact for SU(3)).
// Site numbering inside a parity: cb = lex/2 with lex = x + Lx*(y + Ly*(z + Lz*t))
// (LEXIC, include/qkxTM.h:130 of the reference) and parity (x+y+z+t)&1
// (getOddBit, lib/lattice_util.cpp:1148).  Lx must be even.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace qkx {

// ---------------------------------------------------------------- complex
template <typename R>
struct Cx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ Cx<R> operator+(Cx<R> a, Cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R>
__device__ __forceinline__ Cx<R> operator-(Cx<R> a, Cx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R>
__device__ __forceinline__ Cx<R> operator*(R s, Cx<R> a) { return {s * a.re, s * a.im}; }
template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// conj(a) * b
template <typename R>
__device__ __forceinline__ Cx<R> cmulc(Cx<R> a, Cx<R> b) {
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}
template <typename R>
__device__ __forceinline__ Cx<R> conj(Cx<R> a) { return {a.re, -a.im}; }

// f * a + b for a real scale f
template <typename R>
__device__ __forceinline__ Cx<R> fma_s(R f, Cx<R> a, Cx<R> b) {
  return {fma(f, a.re, b.re), fma(f, a.im, b.im)};
}

// multiply by a phase code: 0 -> 1, 1 -> i, 2 -> -1, 3 -> -i
template <int PH, typename R>
__device__ __forceinline__ Cx<R> phase(Cx<R> z) {
  if constexpr ((PH & 3) == 0) return z;
  else if constexpr ((PH & 3) == 1) return {-z.im, z.re};
  else if constexpr ((PH & 3) == 2) return {-z.re, -z.im};
  else return {z.im, -z.re};
}

template <typename R>
struct Spinor {
  Cx<R> c[4][3];
};
template <typename R>
struct HalfSpinor {
  Cx<R> c[2][3];
};
template <typename R>
struct Link {
  Cx<R> m[3][3];
};
// the four spins of one colour of a spinor
template <typename R>
struct Spin4 {
  Cx<R> s[4];
};

// ---------------------------------------------------------------- gamma tables
// Every gamma matrix used here has one non-zero per row: row r has the entry
// phase code gph(...) in column gcol(...).  Basis 0 = UKQCD (reference
// lib/lattice_util.cpp:281-290), basis 1 = the chiral basis of
// include/hopping_term_chiral.h.  mu = 0..3 are gamma_1..gamma_4, mu = 4 is gamma_5.
__host__ __device__ constexpr int gcol(int basis, int mu, int r) {
  if (basis == 0) {
    switch (mu) {
      case 0: return 3 - r;                      // (0,3) (1,2) (2,1) (3,0)
      case 1: return 3 - r;
      case 2: return r < 2 ? r + 2 : r - 2;      // (0,2) (1,3) (2,0) (3,1)
      case 3: return r;                          // diagonal
      default: return r < 2 ? r + 2 : r - 2;     // gamma5
    }
  } else {
    switch (mu) {
      case 0: return 3 - r;
      case 1: return 3 - r;
      case 2: return r < 2 ? r + 2 : r - 2;
      case 3: return r < 2 ? r + 2 : r - 2;
      default: return r;                         // gamma5 diagonal
    }
  }
}

__host__ __device__ constexpr int gph(int basis, int mu, int r) {
  if (basis == 0) {
    switch (mu) {
      case 0: return r < 2 ? 1 : 3;                    // i, i, -i, -i
      case 1: return (r == 0 || r == 3) ? 0 : 2;       // 1, -1, -1, 1
      case 2: return (r == 0 || r == 3) ? 1 : 3;       // i, -i, -i, i
      case 3: return r < 2 ? 0 : 2;                    // 1, 1, -1, -1
      default: return 0;                               // gamma5 all +1
    }
  } else {
    switch (mu) {
      case 0: return r < 2 ? 3 : 1;                    // -i, -i, i, i
      case 1: return (r == 0 || r == 3) ? 2 : 0;       // -1, 1, 1, -1
      case 2: return (r == 0 || r == 3) ? 3 : 1;       // -i, i, i, -i
      case 3: return 2;                                // -1 everywhere
      default: return r < 2 ? 0 : 2;                  // diag(1,1,-1,-1)
    }
  }
}

// (1 + SIGN*gamma_mu) psi has rank 2.  project() gives its two independent rows
// h0, h1; reconstruct() adds the full 4-spinor rebuilt from (a colour-rotated)
// h back into an accumulator.  For an off-diagonal gamma, rows 0 and 1 are
// h0, h1 and row gcol(0) is SIGN*g_{gcol(0)} * h0 (same for row gcol(1));
// the diagonal gamma_4 of the UKQCD basis keeps rows {0,1} or {2,3} doubled.
template <int B, int MU, int SIGN>
struct Proj {
  static constexpr bool diag = (gcol(B, MU, 0) == 0);
  static constexpr int sh = SIGN > 0 ? 0 : 2;
  static constexpr int c0 = gcol(B, MU, 0), c1 = gcol(B, MU, 1);
  static constexpr int p0 = gph(B, MU, 0) + sh, p1 = gph(B, MU, 1) + sh;
  static constexpr int q0 = gph(B, MU, c0) + sh, q1 = gph(B, MU, c1) + sh;
  static constexpr int drow = (gph(B, MU, 0) + sh) % 4 == 0 ? 0 : 2;  // rows kept by diag

  template <typename R>
  __device__ __forceinline__ static void project(const Spinor<R>& s, HalfSpinor<R>& h) {
    if constexpr (diag) {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        h.c[0][a] = R(2) * s.c[drow][a];
        h.c[1][a] = R(2) * s.c[drow + 1][a];
      }
    } else {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        h.c[0][a] = s.c[0][a] + phase<p0>(s.c[c0][a]);
        h.c[1][a] = s.c[1][a] + phase<p1>(s.c[c1][a]);
      }
    }
  }

  // reconstruct() for a single colour: h0, h1 are that colour of the two rows
  template <typename R>
  __device__ __forceinline__ static void reconstruct1(Spin4<R>& acc, Cx<R> h0, Cx<R> h1) {
    if constexpr (diag) {
      acc.s[drow] = acc.s[drow] + h0;
      acc.s[drow + 1] = acc.s[drow + 1] + h1;
    } else {
      acc.s[0] = acc.s[0] + h0;
      acc.s[1] = acc.s[1] + h1;
      acc.s[c0] = acc.s[c0] + phase<q0>(h0);
      acc.s[c1] = acc.s[c1] + phase<q1>(h1);
    }
  }

  // acc += f * (rebuilt spinor): the scale is folded into the accumulating FMAs
  template <typename R>
  __device__ __forceinline__ static void reconstruct_scaled(Spinor<R>& acc, const HalfSpinor<R>& h, R f) {
    if constexpr (diag) {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        acc.c[drow][a] = fma_s(f, h.c[0][a], acc.c[drow][a]);
        acc.c[drow + 1][a] = fma_s(f, h.c[1][a], acc.c[drow + 1][a]);
      }
    } else {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        acc.c[0][a] = fma_s(f, h.c[0][a], acc.c[0][a]);
        acc.c[1][a] = fma_s(f, h.c[1][a], acc.c[1][a]);
        acc.c[c0][a] = fma_s(f, phase<q0>(h.c[0][a]), acc.c[c0][a]);
        acc.c[c1][a] = fma_s(f, phase<q1>(h.c[1][a]), acc.c[c1][a]);
      }
    }
  }

  template <typename R>
  __device__ __forceinline__ static void reconstruct(Spinor<R>& acc, const HalfSpinor<R>& h) {
    if constexpr (diag) {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        acc.c[drow][a] = acc.c[drow][a] + h.c[0][a];
        acc.c[drow + 1][a] = acc.c[drow + 1][a] + h.c[1][a];
      }
    } else {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        acc.c[0][a] = acc.c[0][a] + h.c[0][a];
        acc.c[1][a] = acc.c[1][a] + h.c[1][a];
        acc.c[c0][a] = acc.c[c0][a] + phase<q0>(h.c[0][a]);
        acc.c[c1][a] = acc.c[c1][a] + phase<q1>(h.c[1][a]);
      }
    }
  }
};

// gamma5 applied to a spinor, in the given basis
template <int B, typename R>
__device__ __forceinline__ Spinor<R> gamma5(const Spinor<R>& s) {
  Spinor<R> o;
  if constexpr (B == 0) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      o.c[0][a] = s.c[2][a];
      o.c[1][a] = s.c[3][a];
      o.c[2][a] = s.c[0][a];
      o.c[3][a] = s.c[1][a];
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      o.c[0][a] = s.c[0][a];
      o.c[1][a] = s.c[1][a];
      o.c[2][a] = R(-1) * s.c[2][a];
      o.c[3][a] = R(-1) * s.c[3][a];
    }
  }
  return o;
}

template <int B, typename R>
__device__ __forceinline__ Spin4<R> gamma5_4(const Spin4<R>& v) {
  if constexpr (B == 0) return {{v.s[2], v.s[3], v.s[0], v.s[1]}};
  else return {{v.s[0], v.s[1], R(-1) * v.s[2], R(-1) * v.s[3]}};
}

// U h and U^+ h on a half spinor
template <typename R>
__device__ __forceinline__ void mul_link(const Link<R>& u, const HalfSpinor<R>& h, HalfSpinor<R>& o) {
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int a = 0; a < 3; a++)
      o.c[s][a] = cmul(u.m[a][0], h.c[s][0]) + cmul(u.m[a][1], h.c[s][1]) + cmul(u.m[a][2], h.c[s][2]);
}
template <typename R>
__device__ __forceinline__ void mul_link_dag(const Link<R>& u, const HalfSpinor<R>& h, HalfSpinor<R>& o) {
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int a = 0; a < 3; a++)
      o.c[s][a] = cmulc(u.m[0][a], h.c[s][0]) + cmulc(u.m[1][a], h.c[s][1]) + cmulc(u.m[2][a], h.c[s][2]);
}

// ---------------------------------------------------------------- geometry
struct Geom {
  int L[4];
  int Vh;       // sites per parity
  int bc_sign;  // sign applied to the t-hops that cross t = Lt-1 -> 0
};

// full coordinates of the cb-th site of the given parity
__device__ __forceinline__ void cb_coords(const Geom& g, int cb, int parity, int x[4]) {
  int j = 2 * cb;
  int x0 = j % g.L[0];
  int r = j / g.L[0];
  x[1] = r % g.L[1];
  r /= g.L[1];
  x[2] = r % g.L[2];
  x[3] = r / g.L[2];
  x[0] = x0 + ((x[1] + x[2] + x[3] + parity) & 1);
}

__device__ __forceinline__ int cb_index(const Geom& g, const int x[4]) {
  return (x[0] + g.L[0] * (x[1] + g.L[1] * (x[2] + g.L[2] * x[3]))) >> 1;
}

// cb index of the neighbour one step forward (+1) or backward (-1) along mu
__device__ __forceinline__ int cb_neighbour(const Geom& g, const int x[4], int mu, int step) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  int v = y[mu] + step;
  y[mu] = v < 0 ? v + g.L[mu] : (v >= g.L[mu] ? v - g.L[mu] : v);
  return cb_index(g, y);
}

// ---------------------------------------------------------------- spinor accessors
// Each spinor accessor holds one base pointer per parity (p0 even, p1 odd), so a
// full field is two halves and a single-parity field leaves the other null.
// FP64: [12][Vh] double2 per parity
struct SpinorF64 {
  double2* p0;
  double2* p1;
  int Vh;
  size_t rs = 0;  // words between consecutive right-hand sides of a batch
  __device__ __forceinline__ SpinorF64 shift(int r) const {
    SpinorF64 o = *this;
    if (p0) o.p0 = p0 + rs * r;
    if (p1) o.p1 = p1 + rs * r;
    return o;
  }
  __device__ __forceinline__ Spinor<double> load(int parity, int cb) const {
    const double2* b = (parity ? p1 : p0) + cb;
    Spinor<double> s;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 d = __ldg(b + k * Vh);
      s.c[k / 3][k % 3] = {d.x, d.y};
    }
    return s;
  }
  static constexpr bool has_norm = false;
  __device__ __forceinline__ Spinor<double> load_raw(int parity, int cb, double& n) const {
    n = 1.0;
    return load(parity, cb);
  }
  __device__ __forceinline__ void store(int parity, int cb, const Spinor<double>& s) const {
    double2* b = (parity ? p1 : p0) + cb;
#pragma unroll
    for (int k = 0; k < 12; k++) b[k * Vh] = make_double2(s.c[k / 3][k % 3].re, s.c[k / 3][k % 3].im);
  }
};

// FP32: [6][Vh] float4 per parity
struct SpinorF32 {
  float4* p0;
  float4* p1;
  int Vh;
  size_t rs = 0;
  __device__ __forceinline__ SpinorF32 shift(int r) const {
    SpinorF32 o = *this;
    if (p0) o.p0 = p0 + rs * r;
    if (p1) o.p1 = p1 + rs * r;
    return o;
  }
  __device__ __forceinline__ Spinor<float> load(int parity, int cb) const {
    const float4* b = (parity ? p1 : p0) + cb;
    Spinor<float> s;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      float4 f = __ldg(b + q * Vh);
      s.c[(2 * q) / 3][(2 * q) % 3] = {f.x, f.y};
      s.c[(2 * q + 1) / 3][(2 * q + 1) % 3] = {f.z, f.w};
    }
    return s;
  }
  static constexpr bool has_norm = false;
  __device__ __forceinline__ Spinor<float> load_raw(int parity, int cb, float& n) const {
    n = 1.f;
    return load(parity, cb);
  }
  __device__ __forceinline__ void store(int parity, int cb, const Spinor<float>& s) const {
    float4* b = (parity ? p1 : p0) + cb;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      Cx<float> a = s.c[(2 * q) / 3][(2 * q) % 3], c = s.c[(2 * q + 1) / 3][(2 * q + 1) % 3];
      b[q * Vh] = make_float4(a.re, a.im, c.re, c.im);
    }
  }
};

// FP16 with a per-site FP32 scale: [3][Vh] uint4 (8 halves each) + norm [Vh] per parity.
// Stored value = component / norm, norm = max |real or imaginary part| over the site.
struct SpinorF16 {
  uint4* p0;
  uint4* p1;
  float* n0;
  float* n1;
  int Vh;
  size_t rs = 0;   // uint4 words between right-hand sides
  size_t rsn = 0;  // norms between right-hand sides
  __device__ __forceinline__ SpinorF16 shift(int r) const {
    SpinorF16 o = *this;
    if (p0) o.p0 = p0 + rs * r;
    if (p1) o.p1 = p1 + rs * r;
    if (n0) o.n0 = n0 + rsn * r;
    if (n1) o.n1 = n1 + rsn * r;
    return o;
  }
  __device__ __forceinline__ Spinor<float> load(int parity, int cb) const {
    const uint4* b = (parity ? p1 : p0) + cb;
    float n = __ldg((parity ? n1 : n0) + cb);
    Spinor<float> s;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      uint4 w = __ldg(b + q * Vh);
      uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        __half2 h = *reinterpret_cast<__half2*>(&ws[k]);
        float2 f = __half22float2(h);
        int idx = 4 * q + k;
        s.c[idx / 3][idx % 3] = {f.x * n, f.y * n};
      }
    }
    return s;
  }
  // the stored values without the site scale (the caller multiplies by n later,
  // after the linear projection and link multiplication)
  static constexpr bool has_norm = true;
  __device__ __forceinline__ Spinor<float> load_raw(int parity, int cb, float& n) const {
    const uint4* b = (parity ? p1 : p0) + cb;
    n = __ldg((parity ? n1 : n0) + cb);
    Spinor<float> s;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      uint4 w = __ldg(b + q * Vh);
      uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        float2 f = __half22float2(*reinterpret_cast<__half2*>(&ws[k]));
        int idx = 4 * q + k;
        s.c[idx / 3][idx % 3] = {f.x, f.y};
      }
    }
    return s;
  }
  __device__ __forceinline__ void store(int parity, int cb, const Spinor<float>& s) const {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 12; k++) m = fmaxf(m, fmaxf(fabsf(s.c[k / 3][k % 3].re), fabsf(s.c[k / 3][k % 3].im)));
    // below FLT_MIN the reciprocal would overflow; such a site is stored as zero
    // (its entries are negligible next to any spinor the solver works with)
    if (!(m >= 1.17549435e-38f)) m = 0.f;
    float inv = m > 0.f ? 1.f / m : 0.f;
    uint4* b = (parity ? p1 : p0) + cb;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      uint32_t ws[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        int idx = 4 * q + k;
        __half2 h = __floats2half2_rn(s.c[idx / 3][idx % 3].re * inv, s.c[idx / 3][idx % 3].im * inv);
        ws[k] = *reinterpret_cast<uint32_t*>(&h);
      }
      b[q * Vh] = make_uint4(ws[0], ws[1], ws[2], ws[3]);
    }
    (parity ? n1 : n0)[cb] = m;
  }
};

// ---------------------------------------------------------------- link accessors
// FP64 18-real: [parity][4][9][Vh] double2
struct GaugeF64x18 {
  const double2* p;
  int Vh;
  __device__ __forceinline__ Link<double> load(int parity, int mu, int cb) const {
    const double2* b = p + ((parity * 4 + mu) * 9 * Vh + cb);
    Link<double> u;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 d = __ldg(b + k * Vh);
      u.m[k / 3][k % 3] = {d.x, d.y};
    }
    return u;
  }
};

template <typename R>
__device__ __forceinline__ void rebuild_row2(Link<R>& u) {
  // row2 = conj(row0 x row1)
  u.m[2][0] = conj(cmul(u.m[0][1], u.m[1][2]) - cmul(u.m[0][2], u.m[1][1]));
  u.m[2][1] = conj(cmul(u.m[0][2], u.m[1][0]) - cmul(u.m[0][0], u.m[1][2]));
  u.m[2][2] = conj(cmul(u.m[0][0], u.m[1][1]) - cmul(u.m[0][1], u.m[1][0]));
}

// FP64 12-real: [parity][4][6][Vh] double2
struct GaugeF64x12 {
  const double2* p;
  int Vh;
  __device__ __forceinline__ Link<double> load(int parity, int mu, int cb) const {
    const double2* b = p + ((parity * 4 + mu) * 6 * Vh + cb);
    Link<double> u;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      double2 d = __ldg(b + k * Vh);
      u.m[k / 3][k % 3] = {d.x, d.y};
    }
    rebuild_row2(u);
    return u;
  }
};

// FP32 12-real: [parity][4][3][Vh] float4
struct GaugeF32x12 {
  const float4* p;
  int Vh;
  __device__ __forceinline__ Link<float> load(int parity, int mu, int cb) const {
    const float4* b = p + ((parity * 4 + mu) * 3 * Vh + cb);
    Link<float> u;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      float4 f = __ldg(b + q * Vh);
      u.m[(2 * q) / 3][(2 * q) % 3] = {f.x, f.y};
      u.m[(2 * q + 1) / 3][(2 * q + 1) % 3] = {f.z, f.w};
    }
    rebuild_row2(u);
    return u;
  }
};

// FP16 12-real: [parity][4][Vh] uint4 (complex 0..3) + [parity][4][Vh] uint2 (complex 4..5)
struct GaugeF16x12 {
  const uint4* a;
  const uint2* b;
  int Vh;
  __device__ __forceinline__ Link<float> load(int parity, int mu, int cb) const {
    const int o = (parity * 4 + mu) * Vh + cb;
    uint4 w = __ldg(a + o);
    uint2 v = __ldg(b + o);
    uint32_t ws[6] = {w.x, w.y, w.z, w.w, v.x, v.y};
    Link<float> u;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      float2 f = __half22float2(*reinterpret_cast<__half2*>(&ws[k]));
      u.m[k / 3][k % 3] = {f.x, f.y};
    }
    rebuild_row2(u);
    return u;
  }
};

}  // namespace qkx
