// layout.cuh -- conversions between the reference's host layouts and the
// device layouts, link compression, link checks, and the synthetic link /
// source generators.
//
// Host layouts (reference include/lattice_util.h:90, 198):
//   spinor [V][4][3] complex double   -> here [V][12] double2, lexicographic site order
//   gauge  [V][4][3][3] complex double -> here [V][4][9] double2
// Device layouts are described in qkx_common.cuh.
#pragma once
#include "qkx_common.cuh"

namespace qkx {

__device__ __forceinline__ void lex_coords(const Geom& g, int s, int x[4]) {
  x[0] = s % g.L[0];
  int r = s / g.L[0];
  x[1] = r % g.L[1];
  r /= g.L[1];
  x[2] = r % g.L[2];
  x[3] = r / g.L[2];
}

// host AoS spinor -> device even-odd SoA, FP64
static __global__ void k_spinor_aos_to_eo(const double2* __restrict__ aos, double2* __restrict__ eo, Geom g) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int x[4];
  lex_coords(g, s, x);
  int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  int cb = s >> 1;
  const double2* src = aos + (size_t)s * 12;
  double2* dst = eo + (size_t)par * 12 * g.Vh + cb;
#pragma unroll
  for (int k = 0; k < 12; k++) dst[(size_t)k * g.Vh] = src[k];
}

static __global__ void k_spinor_eo_to_aos(const double2* __restrict__ eo, double2* __restrict__ aos, Geom g) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int x[4];
  lex_coords(g, s, x);
  int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  int cb = s >> 1;
  const double2* src = eo + (size_t)par * 12 * g.Vh + cb;
  double2* dst = aos + (size_t)s * 12;
#pragma unroll
  for (int k = 0; k < 12; k++) dst[k] = src[(size_t)k * g.Vh];
}

// host AoS links -> device even-odd SoA 18-real FP64.  The t-links on the last
// time slice are multiplied by tsign (+1 keeps them, -1 applies or strips the
// antiperiodic sign).
static __global__ void k_gauge_aos_to_eo(const double2* __restrict__ aos, double2* __restrict__ eo, Geom g, int tsign) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int x[4];
  lex_coords(g, s, x);
  int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  int cb = s >> 1;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    double f = (mu == 3 && x[3] == g.L[3] - 1) ? double(tsign) : 1.0;
    const double2* src = aos + ((size_t)s * 4 + mu) * 9;
    double2* dst = eo + ((size_t)par * 4 + mu) * 9 * g.Vh + cb;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 v = src[k];
      dst[(size_t)k * g.Vh] = make_double2(f * v.x, f * v.y);
    }
  }
}

static __global__ void k_gauge_eo_to_aos(const double2* __restrict__ eo, double2* __restrict__ aos, Geom g) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int x[4];
  lex_coords(g, s, x);
  int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  int cb = s >> 1;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    const double2* src = eo + ((size_t)par * 4 + mu) * 9 * g.Vh + cb;
    double2* dst = aos + ((size_t)s * 4 + mu) * 9;
#pragma unroll
    for (int k = 0; k < 9; k++) dst[k] = src[(size_t)k * g.Vh];
  }
}

// Per-block maxima over the links of: [0] |U U^+ - 1|_max, [1] |det - 1| away
// from the last time slice's t-links, [2] |det - 1| and [3] |det + 1| on them.
static __global__ void k_gauge_check(const double2* __restrict__ eo, Geom g, double* __restrict__ part) {
  __shared__ double red[4][8];
  double m[4] = {0, 0, 0, 0};
  int i = blockIdx.x * blockDim.x + threadIdx.x;  // over 2*Vh*4 links
  if (i < 8 * g.Vh) {
    int mu = i % 4;
    int site = i / 4;
    int par = site >= g.Vh ? 1 : 0;
    int cb = site - par * g.Vh;
    int x[4];
    cb_coords(g, cb, par, x);
    const double2* b = eo + ((size_t)par * 4 + mu) * 9 * g.Vh + cb;
    Cx<double> u[3][3];
    for (int k = 0; k < 9; k++) {
      double2 d = b[(size_t)k * g.Vh];
      u[k / 3][k % 3] = {d.x, d.y};
    }
    for (int a = 0; a < 3; a++)
      for (int c = 0; c < 3; c++) {
        Cx<double> acc = {0, 0};
        for (int k = 0; k < 3; k++) acc = acc + cmul(u[a][k], conj(u[c][k]));
        double d = fmax(fabs(acc.re - (a == c ? 1.0 : 0.0)), fabs(acc.im));
        m[0] = fmax(m[0], d);
      }
    Cx<double> det = cmul(u[0][0], cmul(u[1][1], u[2][2]) - cmul(u[1][2], u[2][1])) -
                     cmul(u[0][1], cmul(u[1][0], u[2][2]) - cmul(u[1][2], u[2][0])) +
                     cmul(u[0][2], cmul(u[1][0], u[2][1]) - cmul(u[1][1], u[2][0]));
    double dp = hypot(det.re - 1.0, det.im), dm = hypot(det.re + 1.0, det.im);
    if (mu == 3 && x[3] == g.L[3] - 1) {
      m[2] = dp;
      m[3] = dm;
    } else {
      m[1] = dp;
    }
  }
  for (int q = 0; q < 4; q++) {
    double v = m[q];
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v = fmax(v, red[threadIdx.x][w]);
    part[blockIdx.x * 4 + threadIdx.x] = v;
  }
}

// 18-real FP64 -> 12-real forms; the last slice's t-links are multiplied by
// tsign so the stored rows are those of an SU(3) matrix.
static __global__ void k_gauge_compress(const double2* __restrict__ eo18, Geom g, int tsign, double2* __restrict__ d12,
                                 float4* __restrict__ f12, uint4* __restrict__ h12a, uint2* __restrict__ h12b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;  // link index over [2][4][Vh]
  if (i >= 8 * g.Vh) return;
  int cb = i % g.Vh;
  int pm = i / g.Vh;  // parity*4 + mu
  int par = pm / 4, mu = pm % 4;
  int x[4];
  cb_coords(g, cb, par, x);
  double f = (mu == 3 && x[3] == g.L[3] - 1) ? double(tsign) : 1.0;
  const double2* src = eo18 + (size_t)pm * 9 * g.Vh + cb;
  double2 v[6];
  for (int k = 0; k < 6; k++) {
    double2 t = src[(size_t)k * g.Vh];
    v[k] = make_double2(f * t.x, f * t.y);
  }
  if (d12)
    for (int k = 0; k < 6; k++) d12[(size_t)pm * 6 * g.Vh + (size_t)k * g.Vh + cb] = v[k];
  if (f12)
    for (int q = 0; q < 3; q++)
      f12[(size_t)pm * 3 * g.Vh + (size_t)q * g.Vh + cb] =
          make_float4((float)v[2 * q].x, (float)v[2 * q].y, (float)v[2 * q + 1].x, (float)v[2 * q + 1].y);
  if (h12a) {
    uint32_t w[6];
    for (int k = 0; k < 6; k++) {
      __half2 h = __floats2half2_rn((float)v[k].x, (float)v[k].y);
      w[k] = *reinterpret_cast<uint32_t*>(&h);
    }
    h12a[(size_t)pm * g.Vh + cb] = make_uint4(w[0], w[1], w[2], w[3]);
    h12b[(size_t)pm * g.Vh + cb] = make_uint2(w[4], w[5]);
  }
}

// 18-real FP64 (boundary sign included) -> FP32 18 reals: complex 0..7 as four
// float4 words [parity*4+mu][4][Vh], complex 8 as a float2 [parity*4+mu][Vh]
static __global__ void k_gauge_f32x18(const double2* __restrict__ eo18, int Vh, float4* __restrict__ a,
                                      float2* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // link index over [2][4][Vh]
  if (i >= 8 * Vh) return;
  const int cb = i % Vh, pm = i / Vh;
  const double2* src = eo18 + (size_t)pm * 9 * Vh + cb;
  double2 t[9];
  for (int k = 0; k < 9; k++) t[k] = src[(size_t)k * Vh];
  for (int q = 0; q < 4; q++)
    a[(size_t)(pm * 4 + q) * Vh + cb] =
        make_float4((float)t[2 * q].x, (float)t[2 * q].y, (float)t[2 * q + 1].x, (float)t[2 * q + 1].y);
  b[(size_t)pm * Vh + cb] = make_float2((float)t[8].x, (float)t[8].y);
}

// 18-real FP64 (boundary sign included) -> FP16 18 reals as (re, im) half2 words:
// complex 0..3 and 4..7 as uint4 [parity*4+mu][Vh], complex 8 as uint32
static __global__ void k_gauge_f16x18(const double2* __restrict__ eo18, int Vh, uint4* __restrict__ a,
                                      uint4* __restrict__ b, uint32_t* __restrict__ c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // link index over [2][4][Vh]
  if (i >= 8 * Vh) return;
  const int cb = i % Vh, pm = i / Vh;
  const double2* src = eo18 + (size_t)pm * 9 * Vh + cb;
  uint32_t w[9];
  for (int k = 0; k < 9; k++) {
    const double2 t = src[(size_t)k * Vh];
    __half2 h = __floats2half2_rn((float)t.x, (float)t.y);
    w[k] = *reinterpret_cast<uint32_t*>(&h);
  }
  a[(size_t)pm * Vh + cb] = make_uint4(w[0], w[1], w[2], w[3]);
  b[(size_t)pm * Vh + cb] = make_uint4(w[4], w[5], w[6], w[7]);
  c[(size_t)pm * Vh + cb] = w[8];
}

// ---------------------------------------------------------------- generators
// Counter-based generator shared with the CPU oracle: every (seed, stream,
// counter) hashes to a uniform in (0,1) with the splitmix64 finaliser, and
// normals come from Box-Muller pairs.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t h = mix64(seed ^ mix64(stream ^ mix64(ctr)));
  return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ void normal_pair(uint64_t seed, uint64_t stream, uint64_t ctr, double* g0, double* g1) {
  double u1 = uniform01(seed, stream, 2 * ctr);
  double u2 = uniform01(seed, stream, 2 * ctr + 1);
  double r = sqrt(-2.0 * log(u1));
  double sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  *g0 = r * cs;
  *g1 = r * sn;
}

__device__ __forceinline__ void mat_mul3(const Cx<double>* a, const Cx<double>* b, Cx<double>* c) {
  Cx<double> t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      Cx<double> acc = {0, 0};
      for (int k = 0; k < 3; k++) acc = acc + cmul(a[i * 3 + k], b[k * 3 + j]);
      t[i * 3 + j] = acc;
    }
  for (int k = 0; k < 9; k++) c[k] = t[k];
}

// U = exp(i eps H), H traceless Hermitian from unit complex Gaussians; exp by
// scaling and squaring around a 16-term Taylor series, then rows 0,1
// orthonormalised and row 2 = conj(row0 x row1).
static __global__ void k_gauge_generate(double2* __restrict__ eo18, Geom g, double eps, uint64_t seed) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;  // over V*4 links, lexicographic
  if (i >= 8 * g.Vh) return;
  int mu = i % 4;
  int s = i / 4;
  Cx<double> A[9], X[9], E[9], T[9];
  for (int k = 0; k < 9; k++) {
    double g0, g1;
    normal_pair(seed, 1, (uint64_t)(s * 4 + mu) * 9 + k, &g0, &g1);
    A[k] = {g0 * 0.70710678118654752440, g1 * 0.70710678118654752440};
  }
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      Cx<double> h = A[a * 3 + b] + conj(A[b * 3 + a]);
      X[a * 3 + b] = 0.5 * h;
    }
  Cx<double> tr = (1.0 / 3.0) * (X[0] + X[4] + X[8]);
  X[0] = X[0] - tr;
  X[4] = X[4] - tr;
  X[8] = X[8] - tr;
  for (int k = 0; k < 9; k++) X[k] = {-eps * X[k].im, eps * X[k].re};  // i eps H
  double fn = 0;
  for (int k = 0; k < 9; k++) fn += X[k].re * X[k].re + X[k].im * X[k].im;
  fn = sqrt(fn);
  int sq = 0;
  while (fn > 0.25 && sq < 64) {  // bounded: a non-finite eps cannot spin
    fn *= 0.5;
    sq++;
  }
  double scale = ldexp(1.0, -sq);
  for (int k = 0; k < 9; k++) X[k] = scale * X[k];
  for (int k = 0; k < 9; k++) E[k] = {(k % 4 == 0) ? 1.0 : 0.0, 0.0};
  for (int n = 16; n >= 1; n--) {
    mat_mul3(X, E, T);
    for (int k = 0; k < 9; k++) E[k] = {T[k].re / n + ((k % 4 == 0) ? 1.0 : 0.0), T[k].im / n};
  }
  for (int r = 0; r < sq; r++) mat_mul3(E, E, E);
  // reunitarize
  double n0 = 0;
  for (int b = 0; b < 3; b++) n0 += E[b].re * E[b].re + E[b].im * E[b].im;
  n0 = 1.0 / sqrt(n0);
  for (int b = 0; b < 3; b++) E[b] = n0 * E[b];
  Cx<double> d = {0, 0};
  for (int b = 0; b < 3; b++) d = d + cmulc(E[b], E[3 + b]);
  for (int b = 0; b < 3; b++) E[3 + b] = E[3 + b] - cmul(d, E[b]);
  double n1 = 0;
  for (int b = 0; b < 3; b++) n1 += E[3 + b].re * E[3 + b].re + E[3 + b].im * E[3 + b].im;
  n1 = 1.0 / sqrt(n1);
  for (int b = 0; b < 3; b++) E[3 + b] = n1 * E[3 + b];
  E[6] = conj(cmul(E[1], E[5]) - cmul(E[2], E[4]));
  E[7] = conj(cmul(E[2], E[3]) - cmul(E[0], E[5]));
  E[8] = conj(cmul(E[0], E[4]) - cmul(E[1], E[3]));

  int x[4];
  lex_coords(g, s, x);
  int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  int cb = s >> 1;
  double2* dst = eo18 + ((size_t)par * 4 + mu) * 9 * g.Vh + cb;
  for (int k = 0; k < 9; k++) dst[(size_t)k * g.Vh] = make_double2(E[k].re, E[k].im);
}

// Gaussian spinor (24 unit normals per site) straight into the even-odd FP64 layout
static __global__ void k_spinor_gaussian(double2* __restrict__ eo, Geom g, uint64_t seed) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= 2 * g.Vh) return;
  int x[4];
  lex_coords(g, s, x);
  int par = (x[0] + x[1] + x[2] + x[3]) & 1;
  int cb = s >> 1;
  double2* dst = eo + (size_t)par * 12 * g.Vh + cb;
  for (int k = 0; k < 12; k++) {
    double g0, g1;
    normal_pair(seed, 2, (uint64_t)s * 12 + k, &g0, &g1);
    dst[(size_t)k * g.Vh] = make_double2(g0, g1);
  }
}

}  // namespace qkx
