// ptc.cu -- the learned preconditioner: network object, training on
// (residual, error) pairs from the library's own solves, and the flexible GCR
// solver that uses it (QKX_SOLVER_GCR_PTC).  No reference counterpart.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <random>
#include <vector>

#include "hop_mrhs.cuh"
#include "layout.cuh"
#include "ptc.cuh"
#include "ptc_tc.cuh"
#include "qkx_ctx.cuh"

using namespace qkx;

struct qkx_ptc {
  qkx_ctx* c = nullptr;
  int nl = 0;
  int ch[QKX_PTC_MAX_LAYERS + 1] = {};
  std::vector<long> woff;  // first complex weight of each layer
  long nw = 0;
  float2* w = nullptr;  // FP32 master weights
  float2* m = nullptr;  // Adam moments
  float2* v = nullptr;
  __nv_bfloat162* wb = nullptr;  // BF16 forward weights
  __nv_bfloat162* wt = nullptr;  // BF16 backward weights (reversed paths, conjugate transpose)
  double2* grad = nullptr;
  double2* part = nullptr;  // weight-gradient block partials
  int wg_blocks = 0;
  float4* act[QKX_PTC_MAX_LAYERS + 1] = {};  // layer inputs (act[0] unused: the input field), act[nl] output
  float4* gb[2] = {};                        // gradient ping-pong
  double* red = nullptr;                     // reduction partials
  int red_n = 0;
  int adam_t = 0;
  int use_tc = 0;          // 16 -> 16 inference layers on the tensor cores
  int* tc_err = nullptr;   // device flag set by a timed-out tensor-core wait
};

namespace qkx {
namespace {

int bad(const char* what) {
  set_error("invalid argument: %s", what);
  return QKX_ERR_INVALID;
}

size_t act_words(const qkx_ctx* c, int C) { return (size_t)2 * (3 * C / 2) * c->Vh; }  // float4 per field

template <class T>
int dalloc(T** p, size_t n, const char* what) {
  if (cudaMalloc((void**)p, sizeof(T) * n) != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    set_error("device allocation of %s failed", what);
    return QKX_ERR_NOMEM;
  }
  return QKX_OK;
}

// ---------------------------------------------------------------- layer dispatch
template <int CI, int CO>
void layer_t(qkx_ctx* c, const float4* in, float4* out, const __nv_bfloat162* w) {
  const int nb = 2 * ((c->Vh + PTC_NT - 1) / PTC_NT);
  k_ptc_layer<CI, CO><<<nb, PTC_NT, 0, c->st>>>(in, out, w, GaugeF32x12{c->U12f, c->Vh}, c->geom_raw);
}
template <int CI, int CO>
void wgrad_t(qkx_ctx* c, const float4* a, const float4* gy, double2* part, int nblocks) {
  k_ptc_wgrad<CI, CO><<<nblocks, PTC_NT, 0, c->st>>>(a, gy, GaugeF32x12{c->U12f, c->Vh}, c->geom_raw, part);
}

#define QKX_PTC_WIDTHS(X) X(4, 4) X(4, 8) X(4, 16) X(8, 4) X(8, 8) X(8, 16) X(16, 4) X(16, 8) X(16, 16)

int layer(qkx_ctx* c, int ci, int co, const float4* in, float4* out, const __nv_bfloat162* w) {
#define QKX_L(A, B) \
  if (ci == A && co == B) layer_t<A, B>(c, in, out, w); else
  QKX_PTC_WIDTHS(QKX_L) return bad("channel widths");
#undef QKX_L
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// 16 -> 16 layer on the tensor cores (ptc_tc.cuh)
int layer_tc(qkx_ctx* c, const float4* in, float4* out, const __nv_bfloat162* w, int* err) {
  static bool attr = false;
  if (!attr) {
    QKX_CUDA(cudaFuncSetAttribute(k_ptc_layer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TcSmem)));
    attr = true;
  }
  const int nb = 2 * ((c->Vh + TC_M - 1) / TC_M);
  k_ptc_layer_tc<<<nb, TC_M, sizeof(TcSmem), c->st>>>(in, out, w, GaugeF32x12{c->U12f, c->Vh}, c->geom_raw, err);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

int wgrad(qkx_ctx* c, int ci, int co, const float4* a, const float4* gy, double2* part, int nblocks) {
#define QKX_W(A, B) \
  if (ci == A && co == B) wgrad_t<A, B>(c, a, gy, part, nblocks); else
  QKX_PTC_WIDTHS(QKX_W) return bad("channel widths");
#undef QKX_W
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// ---------------------------------------------------------------- small field kernels
constexpr int FNT = 256;

inline int fgrid(size_t n) {
  size_t b = (n + FNT - 1) / FNT;
  return (int)std::min<size_t>(b ? b : 1, 148 * 8);
}

// FP64 even-odd spinor [2][12][Vh] double2 -> FP32 [2][6][Vh] float4
__global__ void k_f64_to_f32(const double2* __restrict__ a, float4* __restrict__ b, int Vh) {
  const size_t n = (size_t)12 * Vh;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const size_t par = i / ((size_t)6 * Vh), q = (i / Vh) % 6, cb = i % Vh;
    const double2 u = a[(par * 12 + 2 * q) * Vh + cb], v = a[(par * 12 + 2 * q + 1) * Vh + cb];
    b[i] = make_float4((float)u.x, (float)u.y, (float)v.x, (float)v.y);
  }
}

// x (FP64 layout) += e (FP32 layout)
__global__ void k_add_f32_to_f64(const float4* __restrict__ e, double2* __restrict__ x, int Vh) {
  const size_t n = (size_t)12 * Vh;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const size_t par = i / ((size_t)6 * Vh), q = (i / Vh) % 6, cb = i % Vh;
    const float4 f = e[i];
    double2& u = x[(par * 12 + 2 * q) * Vh + cb];
    double2& v = x[(par * 12 + 2 * q + 1) * Vh + cb];
    u.x += f.x;
    u.y += f.y;
    v.x += f.z;
    v.y += f.w;
  }
}

// FP32 layout -> FP64 layout
__global__ void k_f32_to_f64(const float4* __restrict__ e, double2* __restrict__ x, int Vh) {
  const size_t n = (size_t)12 * Vh;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const size_t par = i / ((size_t)6 * Vh), q = (i / Vh) % 6, cb = i % Vh;
    const float4 f = e[i];
    x[(par * 12 + 2 * q) * Vh + cb] = make_double2(f.x, f.y);
    x[(par * 12 + 2 * q + 1) * Vh + cb] = make_double2(f.z, f.w);
  }
}

__device__ __forceinline__ double block_sum_d(double v) { return block_sum<FNT>(v); }

// x += d (FP64)
__global__ void k_add64(const double2* __restrict__ d, double2* __restrict__ x, size_t n) {
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const double2 a = d[i];
    x[i].x += a.x;
    x[i].y += a.y;
  }
}

// r = b - Mx (FP64), partial sums of |r|^2
__global__ void k_res64(const double2* __restrict__ b, const double2* __restrict__ Mx, double2* __restrict__ r,
                        size_t n, double* __restrict__ part) {
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const double2 u = b[i], v = Mx[i];
    const double2 d = make_double2(u.x - v.x, u.y - v.y);
    r[i] = d;
    acc += d.x * d.x + d.y * d.y;
  }
  const double s = block_sum_d(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// partial sums of |a|^2 over n double2
__global__ void k_norm64(const double2* __restrict__ a, size_t n, double* __restrict__ part) {
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const double2 u = a[i];
    acc += u.x * u.x + u.y * u.y;
  }
  const double s = block_sum_d(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// sum part[j][0..nb) for j < nv, fixed order -> out[j]
__global__ void k_sum_parts(const double* __restrict__ part, int nb, int nv, double* __restrict__ out) {
  const int j = blockIdx.x;
  if (j >= nv) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += FNT) acc += part[(size_t)j * nb + i];
  const double s = block_sum_d(acc);
  if (threadIdx.x == 0) out[j] = s;
}

// training residual: g = (y - e) * inv_e2 and partial sums of |y - e|^2
__global__ void k_ptc_residual(const float4* __restrict__ y, const float4* __restrict__ e, float4* __restrict__ g,
                               size_t n4, float inv_e2, double* __restrict__ part) {
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    const float4 a = y[i], b = e[i];
    const float4 d = make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
    acc += (double)d.x * d.x + (double)d.y * d.y + (double)d.z * d.z + (double)d.w * d.w;
    g[i] = make_float4(d.x * inv_e2, d.y * inv_e2, d.z * inv_e2, d.w * inv_e2);
  }
  const double s = block_sum_d(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ---- GCR vector kernels on FP32 fields (float4 = two complex numbers)
constexpr int GCR_M = 16;  // Krylov vectors per inner cycle

struct F4Ptrs {
  const float4* p[GCR_M];
};

// part[j][block] = partial of <a_j, b> = sum conj(a_j) b, complex, j < na
__global__ void k_cdot_multi(F4Ptrs a, int na, const float4* __restrict__ b, size_t n4, double* __restrict__ part) {
  double re[GCR_M], im[GCR_M];
#pragma unroll
  for (int j = 0; j < GCR_M; j++) re[j] = im[j] = 0.0;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    const float4 y = b[i];
#pragma unroll
    for (int j = 0; j < GCR_M; j++) {
      if (j >= na) break;
      const float4 x = a.p[j][i];
      re[j] += (double)x.x * y.x + (double)x.y * y.y + (double)x.z * y.z + (double)x.w * y.w;
      im[j] += (double)x.x * y.y - (double)x.y * y.x + (double)x.z * y.w - (double)x.w * y.z;
    }
  }
  for (int j = 0; j < na; j++) {
    const double sr = block_sum_d(re[j]);
    const double si = block_sum_d(im[j]);
    if (threadIdx.x == 0) {
      part[(size_t)(2 * j) * gridDim.x + blockIdx.x] = sr;
      part[(size_t)(2 * j + 1) * gridDim.x + blockIdx.x] = si;
    }
  }
}

__device__ __forceinline__ float4 cmul4(double2 z, float4 v) {  // z * (two complex numbers)
  const float zr = (float)z.x, zi = (float)z.y;
  return make_float4(zr * v.x - zi * v.y, zr * v.y + zi * v.x, zr * v.z - zi * v.w, zr * v.w + zi * v.z);
}

// wk -= sum_j beta_j W_j, zk -= sum_j beta_j Z_j  (beta[j] complex = dots[2j], dots[2j+1])
__global__ void k_gcr_orth(F4Ptrs W, F4Ptrs Z, int k, const double* __restrict__ dots, float4* __restrict__ wk,
                           float4* __restrict__ zk, size_t n4) {
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    float4 w = wk[i], z = zk[i];
    for (int j = 0; j < k; j++) {
      const double2 b = make_double2(dots[2 * j], dots[2 * j + 1]);
      const float4 a = cmul4(b, W.p[j][i]), c = cmul4(b, Z.p[j][i]);
      w = make_float4(w.x - a.x, w.y - a.y, w.z - a.z, w.w - a.w);
      z = make_float4(z.x - c.x, z.y - c.y, z.z - c.z, z.w - c.w);
    }
    wk[i] = w;
    zk[i] = z;
  }
}

// wk, zk *= 1 / sqrt(n2[0])
__global__ void k_gcr_scale(float4* __restrict__ wk, float4* __restrict__ zk, const double* __restrict__ n2,
                            size_t n4) {
  const float f = (float)(1.0 / sqrt(n2[0]));
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    const float4 a = wk[i], b = zk[i];
    wk[i] = make_float4(f * a.x, f * a.y, f * a.z, f * a.w);
    zk[i] = make_float4(f * b.x, f * b.y, f * b.z, f * b.w);
  }
}

// e += alpha zk, rho -= alpha wk (alpha = al[0] + i al[1]); partial sums of |rho|^2
__global__ void k_gcr_update(const float4* __restrict__ wk, const float4* __restrict__ zk,
                             const double* __restrict__ al, float4* __restrict__ e, float4* __restrict__ rho, size_t n4,
                             double* __restrict__ part) {
  const double2 a = make_double2(al[0], al[1]);
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    const float4 dz = cmul4(a, zk[i]), dw = cmul4(a, wk[i]);
    float4 ee = e[i], r = rho[i];
    ee = make_float4(ee.x + dz.x, ee.y + dz.y, ee.z + dz.z, ee.w + dz.w);
    r = make_float4(r.x - dw.x, r.y - dw.y, r.z - dw.z, r.w - dw.w);
    e[i] = ee;
    rho[i] = r;
    acc += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z + (double)r.w * r.w;
  }
  const double s = block_sum_d(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ---------------------------------------------------------------- network pieces
int ensure_buffers(qkx_ptc* n) {
  qkx_ctx* c = n->c;
  for (int l = 1; l <= n->nl; l++)
    if (!n->act[l]) QKX_TRY(dalloc(&n->act[l], act_words(c, n->ch[l]), "PTC activations"));
  int cmax = 4;
  for (int l = 0; l <= n->nl; l++) cmax = std::max(cmax, n->ch[l]);
  for (int i = 0; i < 2; i++)
    if (!n->gb[i]) QKX_TRY(dalloc(&n->gb[i], act_words(c, cmax), "PTC gradients"));
  if (!n->red) {
    n->red_n = 148 * 8 * 2 * GCR_M;
    QKX_TRY(dalloc(&n->red, (size_t)n->red_n + 64, "PTC reductions"));
  }
  if (!n->part) {
    const int tiles = 2 * ((c->Vh + PTC_TS - 1) / PTC_TS);
    n->wg_blocks = std::min(tiles, 148 * 4);
    QKX_TRY(dalloc(&n->part, (size_t)n->wg_blocks * 9 * 256, "PTC weight-gradient partials"));
  }
  return QKX_OK;
}

int refresh_backward_weights(qkx_ptc* n) {
  for (int l = 0; l < n->nl; l++) {
    const int cnt = 9 * n->ch[l] * n->ch[l + 1];
    k_ptc_wtrans<<<(cnt + 255) / 256, 256, 0, n->c->st>>>(n->wb + n->woff[l], n->wt + n->woff[l], n->ch[l],
                                                           n->ch[l + 1]);
    counted(n->c);
  }
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// out = N(in); the layer outputs are kept in act[1..nl-1] for the backward pass.
// With tc (inference only) the 16 -> 16 layers run on the tensor cores.
int forward(qkx_ptc* n, const float4* in, float4* out, bool tc = false) {
  const float4* src = in;
  for (int l = 0; l < n->nl; l++) {
    float4* dst = (l == n->nl - 1) ? out : n->act[l + 1];
    if (tc && n->ch[l] == 16 && n->ch[l + 1] == 16)
      QKX_TRY(layer_tc(n->c, src, dst, n->wb + n->woff[l], n->tc_err));
    else
      QKX_TRY(layer(n->c, n->ch[l], n->ch[l + 1], src, dst, n->wb + n->woff[l]));
    src = dst;
  }
  return QKX_OK;
}

// the tensor-core error flag, cleared after reading
int check_tc(qkx_ptc* n) {
  if (!n->use_tc) return QKX_OK;
  int h = 0;
  QKX_CUDA(cudaMemcpyAsync(&h, n->tc_err, sizeof(int), cudaMemcpyDeviceToHost, n->c->st));
  QKX_CUDA(cudaStreamSynchronize(n->c->st));
  if (h) {
    QKX_CUDA(cudaMemsetAsync(n->tc_err, 0, sizeof(int), n->c->st));
    set_error("tensor-core PTC layer: an mbarrier wait timed out");
    return QKX_ERR_CUDA;
  }
  return QKX_OK;
}

// dL/dW^* of every layer into n->grad, from gy = dL/dy^* at the output and the
// activations of the last forward(in)
int backward(qkx_ptc* n, const float4* in, const float4* gy) {
  qkx_ctx* c = n->c;
  const float4* g = gy;
  int slot = 0;
  for (int l = n->nl - 1; l >= 0; l--) {
    const int ci = n->ch[l], co = n->ch[l + 1];
    const float4* a = l == 0 ? in : n->act[l];
    QKX_TRY(wgrad(c, ci, co, a, g, n->part, n->wg_blocks));
    const int cnt = 9 * ci * co;
    k_ptc_wgrad_reduce<<<(cnt + 255) / 256, 256, 0, c->st>>>(n->part, n->wg_blocks, cnt, n->grad + n->woff[l]);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    if (l == 0) break;
    float4* h = n->gb[slot];
    QKX_TRY(layer(c, co, ci, g, h, n->wt + n->woff[l]));
    g = h;
    slot ^= 1;
  }
  return QKX_OK;
}

// loss on one pair: returns (on the device, at *loss_dev) |N(r) - e|^2 / |e|^2
// and leaves dL/dy^* in gb-free scratch for backward; y goes to n->act[nl]
int loss_and_output_grad(qkx_ptc* n, const float4* r, const float4* e, double e2, float4* g, double* loss_dev) {
  qkx_ctx* c = n->c;
  QKX_TRY(forward(n, r, n->act[n->nl]));
  const size_t n4 = act_words(c, 4);
  const int gr = fgrid(n4);
  k_ptc_residual<<<gr, FNT, 0, c->st>>>(n->act[n->nl], e, g, n4, (float)(1.0 / e2), n->red);
  counted(c);
  k_sum_parts<<<1, FNT, 0, c->st>>>(n->red, gr, 1, loss_dev);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// |a|^2 of an FP32 spinor field, on the host
int norm2_f32(qkx_ptc* n, const float4* a, double* out) {
  qkx_ctx* c = n->c;
  // reuse the GCR multi-dot with a single vector
  F4Ptrs p{};
  p.p[0] = a;
  const size_t n4 = act_words(c, 4);
  const int gr = fgrid(n4);
  k_cdot_multi<<<gr, FNT, 0, c->st>>>(p, 1, a, n4, n->red);
  counted(c);
  k_sum_parts<<<1, FNT, 0, c->st>>>(n->red, gr, 1, c->dscal);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaMemcpyAsync(c->hscal, c->dscal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  *out = c->hscal[0];
  return QKX_OK;
}

// host Vector::M spinor -> FP32 even-odd field (through the FP64 staging path)
int upload_f32(qkx_ptc* n, const double* host, float4* dst, double2* tmp64) {
  qkx_ctx* c = n->c;
  QKX_TRY(upload_spinor(c, host, tmp64));
  k_f64_to_f32<<<fgrid((size_t)12 * c->Vh), FNT, 0, c->st>>>(tmp64, dst, c->Vh);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

int check_ready(qkx_ctx* c) {
  if (!c->have_gauge) {
    set_error("the learned preconditioner needs a gauge field");
    return QKX_ERR_NOGAUGE;
  }
  if (!c->compressible || !c->U12f) {
    set_error("the learned preconditioner needs SU(3) links (12-real FP32 copy)");
    return QKX_ERR_UNSUPPORTED;
  }
  return QKX_OK;
}

// ---------------------------------------------------------------- FP32 operator
// out = M in on FP32 full fields (both parities), twisted mass mu
int apply_m_f32(qkx_ctx* c, const float4* in, float4* out, double mu) {
  HopArgs<SpinorF32, GaugeF32x12> A{};
  A.in = SpinorF32{};
  A.in.p0 = const_cast<float4*>(in);
  A.in.p1 = const_cast<float4*>(in) + (size_t)6 * c->Vh;
  A.in.Vh = c->Vh;
  A.out = A.in;
  A.out.p0 = out;
  A.out.p1 = out + (size_t)6 * c->Vh;
  A.x = A.in;
  A.gauge = GaugeF32x12{c->U12f, c->Vh};
  A.g = c->geom_raw;
  A.a = -c->p.kappa;
  A.c = 2.0 * c->p.kappa * mu * c->p.twistSign;
  A.s = 1.0;
  A.nrhs = 1;
  A.nblk = mrhs_site_blocks<128>(c->Vh);
  for (int par = 0; par < 2; par++) {
    A.out_parity = par;
    hop_mrhs_kernel<128, 1, SpinorF32, GaugeF32x12, float, 0, false, EPI_XPAY><<<A.nblk, 128, 0, c->st>>>(A);
    counted(c);
  }
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

}  // namespace

// ---------------------------------------------------------------- GCR solver
// Solve M x = b for each right-hand side: FP64 defect correction around a
// flexible GCR(GCR_M) on M in FP32, right-preconditioned by the network (or by
// nothing when net is NULL).  After a cycle x += e in FP64 and the true residual
// b - M x is recomputed in FP64; it is the stopping test.  A right-hand side
// that has not converged after the iteration budget, or stalls, is finished by
// the even-odd mixed-precision CG from the current residual (the fallback).
int invert_gcr_ptc(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b, double2* const* x,
                   qkx_solve_info* info) {
  QKX_TRY(check_ready(c));
  qkx_ptc* net = const_cast<qkx_ptc*>(sp->preconditioner);
  if (net && net->c != c) return bad("the preconditioner belongs to another context");
  const int Vh = c->Vh;
  const size_t n64 = (size_t)12 * c->V;  // double2 per FP64 field
  const size_t n4 = (size_t)12 * Vh;     // float4 per FP32 field
  // scratch: r64, t64, and FP32 rho, e, rf, W[GCR_M], Z[GCR_M]
  double2 *r64 = nullptr, *t64 = nullptr;
  float4* f32 = nullptr;
  double* red = nullptr;
  const int nf = 3 + 2 * GCR_M;
  const int gr = fgrid(n4);
  int rc = QKX_OK;
  auto fail = [&](int code) {
    rc = code;
    return code;
  };
  struct Scratch {  // freed on every return path
    cudaStream_t st;
    void* p[4];
    ~Scratch() {
      cudaStreamSynchronize(st);
      for (void* q : p) cudaFree(q);
    }
  };
  if (dalloc(&r64, n64, "GCR residual") || dalloc(&t64, n64, "GCR scratch") ||
      dalloc(&f32, n4 * nf, "GCR vectors") || dalloc(&red, (size_t)2 * GCR_M * (gr + 1) + 64, "GCR reductions")) {
    cudaFree(r64);
    cudaFree(t64);
    cudaFree(f32);
    cudaFree(red);
    return QKX_ERR_NOMEM;
  }
  Scratch scratch{c->st, {r64, t64, f32, red}};
  if (net) {
    int e = ensure_buffers(net);
    if (e != QKX_OK) fail(e);
  }
  float4 *rho = f32, *ef = f32 + n4, *rf = f32 + 2 * n4;
  float4* Wv[GCR_M];
  float4* Zv[GCR_M];
  for (int j = 0; j < GCR_M; j++) {
    Wv[j] = f32 + (3 + j) * n4;
    Zv[j] = f32 + (3 + GCR_M + j) * n4;
  }
  double* dsc = red + (size_t)2 * GCR_M * gr;  // device scalars
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->st);
  const double mu = c->p.mu;
  int total_it = 0, cycles = 0, fallbacks = 0;
  double worst = 0.0;
  bool all_conv = true;
  auto host_scalar = [&](const double* d, double* h, int cnt) -> int {
    QKX_CUDA(cudaMemcpyAsync(c->hscal, d, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->st));
    QKX_CUDA(cudaStreamSynchronize(c->st));
    for (int i = 0; i < cnt; i++) h[i] = c->hscal[i];
    return QKX_OK;
  };
  auto norm64 = [&](const double2* a, double* out) -> int {
    k_norm64<<<gr, FNT, 0, c->st>>>(a, n64, red);
    counted(c);
    k_sum_parts<<<1, FNT, 0, c->st>>>(red, gr, 1, dsc);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    return host_scalar(dsc, out, 1);
  };
  for (int i = 0; i < nrhs && rc == QKX_OK; i++) {
    double b2 = 0;
    if (norm64(b[i], &b2) != QKX_OK) break;
    cudaMemsetAsync(x[i], 0, sizeof(double2) * n64, c->st);
    cudaMemcpyAsync(r64, b[i], sizeof(double2) * n64, cudaMemcpyDeviceToDevice, c->st);
    double r2 = b2;
    if (b2 == 0) continue;
    int it = 0, stall = 0;
    double prev = 1.0;
    while (rc == QKX_OK) {
      const double rel = sqrt(r2 / b2);
      if (rel <= sp->tol) break;
      if (it >= sp->maxIter || stall >= 3) {
        // fallback: the mixed-precision CG on M d = r, then x += d
        qkx_solver_params fp = *sp;
        fp.method = QKX_SOLVER_CG_EO_MIXED;
        fp.sloppy_precision = QKX_PREC_HALF;
        fp.tol = std::min(0.5, 0.9 * sp->tol / rel);
        fp.maxIter = 100000;  // the GCR's budget is spent; the fallback solves to completion
        fp.mu = nullptr;
        fp.preconditioner = nullptr;
        const double2* bb[1] = {r64};
        double2* xx[1] = {t64};
        qkx_solve_info fi{};
        int frc = invert_eo_mixed(c, &fp, 1, bb, xx, &fi);
        if (frc != QKX_OK && frc != QKX_ERR_NOT_CONVERGED) {
          fail(frc);
          break;
        }
        fallbacks++;
        total_it += fi.iterations;
        k_add64<<<gr, FNT, 0, c->st>>>(t64, x[i], n64);  // x += d
        counted(c);
        QKX_TRY(apply_tm_mu(c, x[i], t64, false, mu));
        k_res64<<<gr, FNT, 0, c->st>>>(b[i], t64, r64, n64, red);
        counted(c);
        k_sum_parts<<<1, FNT, 0, c->st>>>(red, gr, 1, dsc);
        counted(c);
        QKX_TRY(host_scalar(dsc, &r2, 1));
        if (sqrt(r2 / b2) > sp->tol) all_conv = false;
        break;
      }
      // inner flexible GCR on M e = r (FP32)
      k_f64_to_f32<<<gr, FNT, 0, c->st>>>(r64, rf, Vh);
      counted(c);
      cudaMemcpyAsync(rho, rf, sizeof(float4) * n4, cudaMemcpyDeviceToDevice, c->st);
      cudaMemsetAsync(ef, 0, sizeof(float4) * n4, c->st);
      const double target = std::max(0.5 * sp->tol / rel, 1e-5);
      double rho2 = r2;
      for (int k = 0; k < GCR_M && rc == QKX_OK; k++) {
        if (net) {
          if (forward(net, rho, Zv[k], net->use_tc != 0) != QKX_OK) {
            fail(QKX_ERR_CUDA);
            break;
          }
        } else {
          cudaMemcpyAsync(Zv[k], rho, sizeof(float4) * n4, cudaMemcpyDeviceToDevice, c->st);
        }
        if (apply_m_f32(c, Zv[k], Wv[k], mu) != QKX_OK) {
          fail(QKX_ERR_CUDA);
          break;
        }
        F4Ptrs Wp{}, Zp{};
        for (int j = 0; j < GCR_M; j++) {
          Wp.p[j] = Wv[j];
          Zp.p[j] = Zv[j];
        }
        if (k > 0) {
          k_cdot_multi<<<gr, FNT, 0, c->st>>>(Wp, k, Wv[k], n4, red);
          counted(c);
          k_sum_parts<<<2 * k, FNT, 0, c->st>>>(red, gr, 2 * k, dsc);
          counted(c);
          k_gcr_orth<<<gr, FNT, 0, c->st>>>(Wp, Zp, k, dsc, Wv[k], Zv[k], n4);
          counted(c);
        }
        F4Ptrs one{};
        one.p[0] = Wv[k];
        k_cdot_multi<<<gr, FNT, 0, c->st>>>(one, 1, Wv[k], n4, red);
        counted(c);
        k_sum_parts<<<1, FNT, 0, c->st>>>(red, gr, 1, dsc + 2 * GCR_M);
        counted(c);
        k_gcr_scale<<<gr, FNT, 0, c->st>>>(Wv[k], Zv[k], dsc + 2 * GCR_M, n4);
        counted(c);
        k_cdot_multi<<<gr, FNT, 0, c->st>>>(one, 1, rho, n4, red);
        counted(c);
        k_sum_parts<<<2, FNT, 0, c->st>>>(red, gr, 2, dsc + 2 * GCR_M + 2);
        counted(c);
        k_gcr_update<<<gr, FNT, 0, c->st>>>(Wv[k], Zv[k], dsc + 2 * GCR_M + 2, ef, rho, n4, red);
        counted(c);
        k_sum_parts<<<1, FNT, 0, c->st>>>(red, gr, 1, dsc + 2 * GCR_M + 4);
        counted(c);
        if (cudaGetLastError() != cudaSuccess) {
          set_error("GCR kernels failed");
          fail(QKX_ERR_CUDA);
          break;
        }
        if (host_scalar(dsc + 2 * GCR_M + 4, &rho2, 1) != QKX_OK) {
          fail(QKX_ERR_CUDA);
          break;
        }
        it++;
        if (!(rho2 == rho2)) {
          set_error("GCR residual is NaN");
          fail(QKX_ERR_NAN);
          break;
        }
        if (rho2 <= target * target * r2) break;
      }
      if (rc != QKX_OK) break;
      // x += e, true residual in FP64
      k_add_f32_to_f64<<<gr, FNT, 0, c->st>>>(ef, x[i], Vh);
      counted(c);
      QKX_TRY(apply_tm_mu(c, x[i], t64, false, mu));
      k_res64<<<gr, FNT, 0, c->st>>>(b[i], t64, r64, n64, red);
      counted(c);
      k_sum_parts<<<1, FNT, 0, c->st>>>(red, gr, 1, dsc);
      counted(c);
      QKX_TRY(host_scalar(dsc, &r2, 1));
      cycles++;
      const double now = sqrt(r2 / b2);
      stall = (now > 0.5 * prev) ? stall + 1 : 0;
      prev = now;
    }
    total_it += it;
    worst = std::max(worst, sqrt(r2 / b2));
  }
  cudaEventRecord(e1, c->st);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == QKX_OK && net) rc = check_tc(net);
  if (rc != QKX_OK) return rc;
  if (info) {
    info->iterations = total_it;
    info->restarts = cycles;
    info->fallbacks = fallbacks;
    info->true_residual = worst;
    info->normal_residual = worst;
    info->converged = (all_conv && worst <= sp->tol) ? 1 : 0;
    info->seconds = ms * 1e-3;
  }
  return (all_conv && worst <= sp->tol) ? QKX_OK : QKX_ERR_NOT_CONVERGED;
}

}  // namespace qkx

// =================================================================== C ABI
extern "C" {

int qkx_ptc_create(qkx_ctx* c, const qkx_ptc_params* p, qkx_ptc** out) {
  if (!c || !p || !out) return bad("NULL argument");
  *out = nullptr;
  if (p->nlayers < 1 || p->nlayers > QKX_PTC_MAX_LAYERS) return bad("nlayers");
  if (p->channels[0] != 4 || p->channels[p->nlayers] != 4) return bad("the first and last widths must be 4");
  for (int l = 0; l <= p->nlayers; l++)
    if (p->channels[l] != 4 && p->channels[l] != 8 && p->channels[l] != 16) return bad("widths must be 4, 8 or 16");
  if (!(p->init_scale >= 0)) return bad("init_scale");
  QKX_CUDA(cudaSetDevice(c->device));
  qkx_ptc* n = new qkx_ptc;
  n->c = c;
  n->use_tc = p->tensor_cores ? 1 : 0;
  n->nl = p->nlayers;
  for (int l = 0; l <= n->nl; l++) n->ch[l] = p->channels[l];
  for (int l = 0; l < n->nl; l++) {
    n->woff.push_back(n->nw);
    n->nw += 9L * n->ch[l] * n->ch[l + 1];
  }
  int rc = QKX_OK;
  if (dalloc(&n->w, n->nw, "PTC weights") || dalloc(&n->m, n->nw, "Adam moments") ||
      dalloc(&n->v, n->nw, "Adam moments") || dalloc(&n->wb, n->nw, "BF16 weights") ||
      dalloc(&n->wt, n->nw, "BF16 weights") || dalloc(&n->grad, n->nw, "weight gradient") ||
      dalloc(&n->tc_err, 1, "error flag"))
    rc = QKX_ERR_NOMEM;
  if (rc == QKX_OK && cudaMemsetAsync(n->tc_err, 0, sizeof(int), c->st) != cudaSuccess) rc = QKX_ERR_CUDA;
  if (rc != QKX_OK) {
    qkx_ptc_destroy(n);
    return rc;
  }
  // identity path = identity embedding, hop paths ~ N(0, init_scale^2 / C_in)
  std::vector<double> h((size_t)2 * n->nw, 0.0);
  std::mt19937_64 gen(p->seed);
  std::normal_distribution<double> nd(0.0, 1.0);
  for (int l = 0; l < n->nl; l++) {
    const int ci = n->ch[l], co = n->ch[l + 1];
    const double sc = p->init_scale / sqrt((double)ci);
    for (int q = 0; q < 9; q++)
      for (int a = 0; a < co; a++)
        for (int b = 0; b < ci; b++) {
          const long i = n->woff[l] + ((long)q * co + a) * ci + b;
          if (q == 0) {
            h[2 * i] = (a % ci == b && (co >= ci || b % co == a)) ? 1.0 : 0.0;
          } else {
            h[2 * i] = sc * nd(gen);
            h[2 * i + 1] = sc * nd(gen);
          }
        }
  }
  rc = qkx_ptc_set_weights(n, h.data());
  if (rc != QKX_OK) {
    qkx_ptc_destroy(n);
    return rc;
  }
  *out = n;
  return QKX_OK;
}

void qkx_ptc_destroy(qkx_ptc* n) {
  if (!n) return;
  cudaSetDevice(n->c->device);
  cudaStreamSynchronize(n->c->st);
  cudaFree(n->w);
  cudaFree(n->m);
  cudaFree(n->v);
  cudaFree(n->wb);
  cudaFree(n->wt);
  cudaFree(n->grad);
  cudaFree(n->tc_err);
  cudaFree(n->part);
  cudaFree(n->red);
  for (int l = 0; l <= QKX_PTC_MAX_LAYERS; l++) cudaFree(n->act[l]);
  cudaFree(n->gb[0]);
  cudaFree(n->gb[1]);
  delete n;
}

long qkx_ptc_num_weights(const qkx_ptc* n) { return n ? n->nw : -1; }

int qkx_ptc_get_weights(const qkx_ptc* n, int which, double* w) {
  if (!n || !w) return bad("NULL argument");
  if (which != 0 && which != 1) return bad("which");
  QKX_CUDA(cudaSetDevice(n->c->device));
  std::vector<float2> f((size_t)n->nw);
  if (which == 0) {
    QKX_CUDA(cudaMemcpyAsync(f.data(), n->w, sizeof(float2) * n->nw, cudaMemcpyDeviceToHost, n->c->st));
    QKX_CUDA(cudaStreamSynchronize(n->c->st));
  } else {
    std::vector<__nv_bfloat162> bq((size_t)n->nw);
    QKX_CUDA(cudaMemcpyAsync(bq.data(), n->wb, sizeof(__nv_bfloat162) * n->nw, cudaMemcpyDeviceToHost, n->c->st));
    QKX_CUDA(cudaStreamSynchronize(n->c->st));
    for (long i = 0; i < n->nw; i++) f[i] = __bfloat1622float2(bq[i]);
  }
  for (long i = 0; i < n->nw; i++) {
    w[2 * i] = f[i].x;
    w[2 * i + 1] = f[i].y;
  }
  return QKX_OK;
}

int qkx_ptc_set_weights(qkx_ptc* n, const double* w) {
  if (!n || !w) return bad("NULL argument");
  QKX_CUDA(cudaSetDevice(n->c->device));
  std::vector<float2> f((size_t)n->nw);
  std::vector<__nv_bfloat162> bq((size_t)n->nw);
  for (long i = 0; i < n->nw; i++) {
    f[i] = make_float2((float)w[2 * i], (float)w[2 * i + 1]);
    bq[i] = __floats2bfloat162_rn(f[i].x, f[i].y);
  }
  QKX_CUDA(cudaMemcpyAsync(n->w, f.data(), sizeof(float2) * n->nw, cudaMemcpyHostToDevice, n->c->st));
  QKX_CUDA(cudaMemcpyAsync(n->wb, bq.data(), sizeof(__nv_bfloat162) * n->nw, cudaMemcpyHostToDevice, n->c->st));
  QKX_CUDA(cudaMemsetAsync(n->m, 0, sizeof(float2) * n->nw, n->c->st));
  QKX_CUDA(cudaMemsetAsync(n->v, 0, sizeof(float2) * n->nw, n->c->st));
  n->adam_t = 0;
  QKX_TRY(refresh_backward_weights(n));
  QKX_CUDA(cudaStreamSynchronize(n->c->st));
  return QKX_OK;
}

int qkx_ptc_apply(qkx_ptc* n, const double* in_host, double* out_host) {
  if (!n || !in_host || !out_host) return bad("NULL argument");
  qkx_ctx* c = n->c;
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(check_ready(c));
  QKX_TRY(ensure_buffers(n));
  QKX_TRY(ensure_work(c));
  float4 *a = nullptr, *y = nullptr;
  QKX_TRY(dalloc(&a, act_words(c, 4), "PTC input"));
  if (dalloc(&y, act_words(c, 4), "PTC output") != QKX_OK) {
    cudaFree(a);
    return QKX_ERR_NOMEM;
  }
  int rc = upload_f32(n, in_host, a, c->w[0]);
  if (rc == QKX_OK) rc = forward(n, a, y, n->use_tc != 0);
  if (rc == QKX_OK) rc = check_tc(n);
  if (rc == QKX_OK) {
    k_f32_to_f64<<<fgrid((size_t)12 * c->Vh), FNT, 0, c->st>>>(y, c->w[1], c->Vh);
    counted(c);
    rc = download_spinor(c, c->w[1], out_host);
  }
  cudaStreamSynchronize(c->st);
  cudaFree(a);
  cudaFree(y);
  return rc;
}

int qkx_ptc_loss_grad(qkx_ptc* n, const double* r_host, const double* e_host, double* loss, double* grad) {
  if (!n || !r_host || !e_host || !loss) return bad("NULL argument");
  qkx_ctx* c = n->c;
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(check_ready(c));
  QKX_TRY(ensure_buffers(n));
  QKX_TRY(ensure_work(c));
  float4* f = nullptr;
  QKX_TRY(dalloc(&f, 3 * act_words(c, 4), "PTC pair"));
  float4 *r = f, *e = f + act_words(c, 4), *g = f + 2 * act_words(c, 4);
  double e2 = 0;
  int rc = upload_f32(n, r_host, r, c->w[0]);
  if (rc == QKX_OK) rc = upload_f32(n, e_host, e, c->w[0]);
  if (rc == QKX_OK) rc = norm2_f32(n, e, &e2);
  if (rc == QKX_OK && !(e2 > 0)) rc = bad("|e| = 0");
  if (rc == QKX_OK) rc = loss_and_output_grad(n, r, e, e2, g, c->dscal + 1);
  if (rc == QKX_OK && grad) rc = backward(n, r, g);
  if (rc == QKX_OK) {
    double d2 = 0;
    cudaMemcpyAsync(&d2, c->dscal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->st);
    cudaStreamSynchronize(c->st);
    *loss = d2 / e2;
    if (grad) {
      std::vector<double2> gh((size_t)n->nw);
      cudaMemcpyAsync(gh.data(), n->grad, sizeof(double2) * n->nw, cudaMemcpyDeviceToHost, c->st);
      cudaStreamSynchronize(c->st);
      for (long i = 0; i < n->nw; i++) {
        grad[2 * i] = gh[i].x;
        grad[2 * i + 1] = gh[i].y;
      }
    }
  }
  cudaStreamSynchronize(c->st);
  cudaFree(f);
  if (rc == QKX_OK && cudaGetLastError() != cudaSuccess) rc = QKX_ERR_CUDA;
  return rc;
}

int qkx_ptc_train(qkx_ptc* n, const qkx_ptc_train_params* tp, qkx_ptc_train_info* info) {
  if (!n || !tp) return bad("NULL argument");
  if (tp->n_solves < 1 || tp->steps < 0 || !(tp->lr > 0) || !(tp->solve_tol > 0)) return bad("training parameters");
  qkx_ctx* c = n->c;
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(check_ready(c));
  QKX_TRY(ensure_buffers(n));
  const size_t fw = act_words(c, 4);         // float4 per FP32 spinor
  const size_t n64 = (size_t)12 * c->V;      // double2 per FP64 spinor
  // pairs [0, ns): (b, M^-1 b) from the solves; [ns, 2 ns): (M v, v) for Gaussian v, the
  // high-mode part of M^-1 that a network of nlayers hops can represent
  const int ns = tp->n_solves;
  const int np = 2 * ns;
  float4* pairs = nullptr;
  QKX_TRY(dalloc(&pairs, fw * 2 * (size_t)np, "training pairs"));
  std::vector<double> e2(np, 0.0);
  int rc = QKX_OK;
  cudaEvent_t t0, t1, t2;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventCreate(&t2);
  cudaEventRecord(t0, c->st);
  {
    const int B = std::min(ns, 16);
    double2* buf = nullptr;
    if (dalloc(&buf, n64 * 2 * B, "data solves") != QKX_OK) {
      cudaFree(pairs);
      return QKX_ERR_NOMEM;
    }
    for (int i0 = 0; i0 < ns && rc == QKX_OK; i0 += B) {
      const int nb = std::min(B, ns - i0);
      std::vector<const double2*> bp(nb);
      std::vector<double2*> xp(nb);
      for (int k = 0; k < nb; k++) {
        double2* bk = buf + (size_t)k * n64;
        k_spinor_gaussian<<<(unsigned)((c->V + 127) / 128), 128, 0, c->st>>>(bk, c->geom,
                                                                          tp->seed * 1000003ULL + i0 + k);
        counted(c);
        bp[k] = bk;
        xp[k] = buf + (size_t)(B + k) * n64;
      }
      qkx_solver_params sp{};
      sp.method = QKX_SOLVER_CG_EO_MIXED;
      sp.sloppy_precision = QKX_PREC_HALF;
      sp.tol = tp->solve_tol;
      sp.maxIter = 100000;
      sp.use_graphs = 1;
      qkx_solve_info si{};
      rc = invert_eo_mixed(c, &sp, nb, bp.data(), xp.data(), &si);
      if (rc == QKX_ERR_NOT_CONVERGED) rc = QKX_OK;
      for (int k = 0; k < nb && rc == QKX_OK; k++) {
        float4* r = pairs + (size_t)(i0 + k) * 2 * fw;
        k_f64_to_f32<<<fgrid(n64), FNT, 0, c->st>>>(bp[k], r, c->Vh);
        k_f64_to_f32<<<fgrid(n64), FNT, 0, c->st>>>(xp[k], r + fw, c->Vh);
        counted(c, 2);
        rc = norm2_f32(n, r + fw, &e2[i0 + k]);
      }
      // operator pairs: v Gaussian, r = M v (FP64 operator)
      for (int k = 0; k < nb && rc == QKX_OK; k++) {
        double2* v = buf + (size_t)k * n64;
        double2* Mv = buf + (size_t)(B + k) * n64;
        k_spinor_gaussian<<<(unsigned)((c->V + 127) / 128), 128, 0, c->st>>>(
            v, c->geom, (tp->seed * 1000003ULL + i0 + k) ^ 0xA5A5A5A5ULL);
        counted(c);
        rc = apply_tm_mu(c, v, Mv, false, c->p.mu);
        if (rc != QKX_OK) break;
        float4* r = pairs + (size_t)(ns + i0 + k) * 2 * fw;
        k_f64_to_f32<<<fgrid(n64), FNT, 0, c->st>>>(Mv, r, c->Vh);
        k_f64_to_f32<<<fgrid(n64), FNT, 0, c->st>>>(v, r + fw, c->Vh);
        counted(c, 2);
        rc = norm2_f32(n, r + fw, &e2[ns + i0 + k]);
      }
    }
    cudaStreamSynchronize(c->st);
    cudaFree(buf);
  }
  cudaEventRecord(t1, c->st);
  float4* g = nullptr;
  double* losses = nullptr;
  if (rc == QKX_OK && dalloc(&g, fw, "output gradient") != QKX_OK) rc = QKX_ERR_NOMEM;
  std::vector<int> evals;
  for (int k = 0; k < std::min(ns, 4); k++) {
    evals.push_back(k);
    evals.push_back(ns + k);
  }
  const int neval = (int)evals.size();
  if (rc == QKX_OK && dalloc(&losses, (size_t)tp->steps + 2 * neval + 1, "loss history") != QKX_OK)
    rc = QKX_ERR_NOMEM;
  auto mean_loss = [&](int slot0, double* out) -> int {
    for (int k = 0; k < neval; k++) {
      const float4* r = pairs + (size_t)evals[k] * 2 * fw;
      QKX_TRY(loss_and_output_grad(n, r, r + fw, e2[evals[k]], g, losses + slot0 + k));
    }
    std::vector<double> h(neval);
    QKX_CUDA(cudaMemcpyAsync(h.data(), losses + slot0, sizeof(double) * neval, cudaMemcpyDeviceToHost, c->st));
    QKX_CUDA(cudaStreamSynchronize(c->st));
    double s = 0;
    for (int k = 0; k < neval; k++) s += h[k] / e2[evals[k]];
    *out = s / neval;
    return QKX_OK;
  };
  double l0 = 0, l1 = 0;
  if (rc == QKX_OK) rc = mean_loss(tp->steps, &l0);
  // steps: pairs in shuffled epochs
  std::mt19937_64 gen(tp->seed ^ 0x5eedULL);
  std::vector<int> order(np);
  std::iota(order.begin(), order.end(), 0);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int s = 0; s < tp->steps && rc == QKX_OK; s++) {
    if (s % np == 0) std::shuffle(order.begin(), order.end(), gen);
    const int k = order[s % np];
    const float4* r = pairs + (size_t)k * 2 * fw;
    rc = loss_and_output_grad(n, r, r + fw, e2[k], g, losses + s);
    if (rc == QKX_OK) rc = backward(n, r, g);
    if (rc != QKX_OK) break;
    n->adam_t++;
    const double lr = tp->lr * (0.05 + 0.95 * 0.5 * (1.0 + cos(M_PI * s / std::max(1, tp->steps))));
    const float bc1 = 1.0f - powf(b1, (float)n->adam_t), bc2 = 1.0f - powf(b2, (float)n->adam_t);
    k_ptc_adam<<<(unsigned)((n->nw + 255) / 256), 256, 0, c->st>>>(n->w, n->m, n->v, n->grad, n->wb, (int)n->nw,
                                                                (float)lr, b1, b2, bc1, bc2, eps);
    counted(c);
    if (cudaGetLastError() != cudaSuccess) rc = QKX_ERR_CUDA;
    if (rc == QKX_OK) rc = refresh_backward_weights(n);
  }
  cudaEventRecord(t2, c->st);
  if (rc == QKX_OK) rc = mean_loss(tp->steps + neval, &l1);
  cudaStreamSynchronize(c->st);
  float ms_data = 0, ms_train = 0;
  cudaEventElapsedTime(&ms_data, t0, t1);
  cudaEventElapsedTime(&ms_train, t1, t2);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(t2);
  cudaFree(pairs);
  cudaFree(g);
  cudaFree(losses);
  if (rc == QKX_ERR_CUDA) set_error("training: %s", cudaGetErrorString(cudaGetLastError()));
  if (rc != QKX_OK) return rc;
  if (info) {
    info->loss_initial = l0;
    info->loss_final = l1;
    info->seconds_data = ms_data * 1e-3;
    info->seconds_train = ms_train * 1e-3;
    info->steps = tp->steps;
  }
  return QKX_OK;
}

}  // extern "C"
