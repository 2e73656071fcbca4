// ptc.cu -- the learned preconditioner: network object, training on
// (residual, error) pairs from the library's own solves, and the flexible CG
// solver that uses it (QKX_SOLVER_GCR_PTC).  No reference counterpart.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <random>
#include <vector>

#include "hop_c3t.cuh"
#include "hop_mrhs.cuh"
#include "layout.cuh"
#include "ptc.cuh"
#include "ptc_tc.cuh"
#include "qkx_ctx.cuh"
#include "site_ops.cuh"

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
  uint4* hid[QKX_PTC_MAX_LAYERS + 1] = {};  // BF16 hidden activations of layers 1..nl-1 (kept for backward)
  float4* yout = nullptr;                   // FP32 network output of the loss (C = 4, both parities)
  uint4* gb[2] = {};                        // BF16 activation-gradient ping-pong
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

size_t f32_words(const qkx_ctx* c) { return (size_t)12 * c->Vh; }                 // float4, FP32 spinor
size_t bf_words(const qkx_ctx* c, int C) { return (size_t)2 * (3 * C / 4) * c->Vh; }  // uint4, BF16 field

// network fields over contiguous buffers (even parity first)
PtcField f32_field(const float4* base, int Vh) {
  return PtcField{{(void*)base, (void*)(base + (size_t)6 * Vh)}};
}
PtcField bf_field(const uint4* base, int C, int Vh) {
  return PtcField{{(void*)base, (void*)(base + (size_t)(3 * C / 4) * Vh)}};
}

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
template <int CI, int CO, bool I32, bool O32>
void layer_t(qkx_ctx* c, PtcField in, PtcField out, const __nv_bfloat162* w, int par0, int npar) {
  const int nsb = (c->Vh + PTC_SB - 1) / PTC_SB;
  const size_t smem = sizeof(float4) * 9 * CI * CO;  // <= 36 KB: no opt-in needed
  k_ptc_layer<CI, CO, I32, O32><<<nsb * npar, dim3(PTC_SB, 3), smem, c->st>>>(
      in, out, w, GaugeF32x12{c->U12f, c->Vh}, c->geom_raw, par0, npar);
}
template <int CI, int CO, bool A32, bool G32>
void wgrad_t(qkx_ctx* c, PtcField a, PtcField gy, double2* part, int nblocks) {
  k_ptc_wgrad<CI, CO, A32, G32><<<nblocks, PTC_NT, 0, c->st>>>(a, gy, GaugeF32x12{c->U12f, c->Vh}, c->geom_raw,
                                                               part);
}

// (C_in, C_out, FP32 input, FP32 output): FP32 only at the network's 4-channel ends
#define QKX_PTC_KINDS(X)                                                                                    \
  X(4, 4, 0, 0) X(4, 4, 1, 0) X(4, 4, 0, 1) X(4, 4, 1, 1) X(4, 8, 0, 0) X(4, 8, 1, 0) X(4, 16, 0, 0)      \
  X(4, 16, 1, 0) X(8, 4, 0, 0) X(8, 4, 0, 1) X(8, 8, 0, 0) X(8, 16, 0, 0) X(16, 4, 0, 0) X(16, 4, 0, 1)   \
  X(16, 8, 0, 0) X(16, 16, 0, 0)

// one layer on the FP32 pipe; npar = 1 computes the output parity par0 only
int layer(qkx_ctx* c, int ci, int co, PtcField in, bool in32, PtcField out, bool out32, const __nv_bfloat162* w,
          int par0 = 0, int npar = 2) {
#define QKX_L(A, B, I, O) \
  if (ci == A && co == B && in32 == (I != 0) && out32 == (O != 0)) layer_t<A, B, I, O>(c, in, out, w, par0, npar); else
  QKX_PTC_KINDS(QKX_L) return bad("channel widths");
#undef QKX_L
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// 16 -> co layer on the tensor cores (ptc_tc.cuh): BF16 in, BF16 out or (out32, co = 4) the
// FP32 spinor layout; npar = 1 computes the output parity par0 only.  The kernel's shared
// memory (43 KB) is within the default limit.
template <int CI, int CO, bool I32, bool O32>
int layer_tc_t(qkx_ctx* c, PtcField in, PtcField out, const __nv_bfloat162* w, int* err, int par0, int npar) {
  static_assert(sizeof(TcSmem) <= 48 * 1024, "the tensor-core layer's shared memory needs no opt-in");
  const int nb = npar * ((c->Vh + TC_M - 1) / TC_M);
  k_ptc_layer_tc<CI, CO, I32, O32><<<nb, TC_M, sizeof(TcSmem), c->st>>>(
      in, out, w, GaugeF32x12{c->U12f, c->Vh}, c->geom_raw, par0, npar, err);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}
// whether a layer has a tensor-core form: 16 channels on one side, the other 4 or 16
inline bool tc_layer(int ci, int co) { return (ci == 16 && (co == 16 || co == 4)) || (ci == 4 && co == 16); }
int layer_tc(qkx_ctx* c, int ci, int co, bool in32, bool out32, PtcField in, PtcField out, const __nv_bfloat162* w,
             int* err, int par0 = 0, int npar = 2) {
  if (ci == 16 && co == 16 && !in32 && !out32) return layer_tc_t<16, 16, false, false>(c, in, out, w, err, par0, npar);
  if (ci == 16 && co == 4 && !in32) {
    if (out32) return layer_tc_t<16, 4, false, true>(c, in, out, w, err, par0, npar);
    return layer_tc_t<16, 4, false, false>(c, in, out, w, err, par0, npar);
  }
  if (ci == 4 && co == 16 && !out32) {
    if (in32) return layer_tc_t<4, 16, true, false>(c, in, out, w, err, par0, npar);
    return layer_tc_t<4, 16, false, false>(c, in, out, w, err, par0, npar);
  }
  return bad("tensor-core layer widths");
}

int wgrad(qkx_ctx* c, int ci, int co, PtcField a, bool a32, PtcField gy, bool g32, double2* part, int nblocks) {
#define QKX_W(A, B, I, O) \
  if (ci == A && co == B && a32 == (I != 0) && g32 == (O != 0)) wgrad_t<A, B, I, O>(c, a, gy, part, nblocks); else
  QKX_PTC_KINDS(QKX_W) return bad("channel widths");
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

// ---- multi-dot on FP32 fields (float4 = two complex numbers)
constexpr int GCR_M = 16;  // vectors one k_cdot_multi launch takes

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

// ---------------------------------------------------------------- network pieces
int ensure_buffers(qkx_ptc* n) {
  qkx_ctx* c = n->c;
  for (int l = 1; l < n->nl; l++)
    if (!n->hid[l]) QKX_TRY(dalloc(&n->hid[l], bf_words(c, n->ch[l]), "PTC activations"));
  if (!n->yout) QKX_TRY(dalloc(&n->yout, f32_words(c), "PTC output"));
  int cmax = 4;
  for (int l = 0; l <= n->nl; l++) cmax = std::max(cmax, n->ch[l]);
  for (int i = 0; i < 2; i++)
    if (!n->gb[i]) QKX_TRY(dalloc(&n->gb[i], bf_words(c, cmax), "PTC gradients"));
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

// out = N(in) on FP32 4-channel fields; the hidden activations stay in hid[1..nl-1]
// (BF16) for the backward pass.  With tc the layers with 16 channels on one side (4 or 16 on the
// other) run on the tensor cores.
// out_npar = 1 computes the output on parity out_par0 only (the even-odd solver reads
// the even sites of N applied to an even-site input).
int forward(qkx_ptc* n, PtcField in, PtcField out, bool tc = false, int out_par0 = 0, int out_npar = 2) {
  const int Vh = n->c->Vh;
  PtcField src = in;
  bool s32 = true;
  for (int l = 0; l < n->nl; l++) {
    const bool last = l == n->nl - 1;
    const PtcField dst = last ? out : bf_field(n->hid[l + 1], n->ch[l + 1], Vh);
    if (tc && tc_layer(n->ch[l], n->ch[l + 1]))
      QKX_TRY(layer_tc(n->c, n->ch[l], n->ch[l + 1], s32, last, src, dst, n->wb + n->woff[l], n->tc_err,
                       last ? out_par0 : 0, last ? out_npar : 2));
    else
      QKX_TRY(layer(n->c, n->ch[l], n->ch[l + 1], src, s32, dst, last, n->wb + n->woff[l], last ? out_par0 : 0,
                    last ? out_npar : 2));
    src = dst;
    s32 = last;
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

// dL/dW^* of every layer into n->grad, from gy = dL/dy^* at the output (FP32) and the
// activations of the last forward(in).  The activation gradients between layers are
// BF16, like the activations; with tc the layers with a tensor-core form run there.
int backward(qkx_ptc* n, PtcField in, PtcField gy, bool tc = false) {
  qkx_ctx* c = n->c;
  const int Vh = c->Vh;
  PtcField g = gy;
  bool g32 = true;
  int slot = 0;
  for (int l = n->nl - 1; l >= 0; l--) {
    const int ci = n->ch[l], co = n->ch[l + 1];
    const PtcField a = l == 0 ? in : bf_field(n->hid[l], ci, Vh);
    QKX_TRY(wgrad(c, ci, co, a, l == 0, g, g32, n->part, n->wg_blocks));
    const int cnt = 9 * ci * co;
    k_ptc_wgrad_reduce<<<(cnt + 255) / 256, 256, 0, c->st>>>(n->part, n->wg_blocks, cnt, n->grad + n->woff[l]);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    if (l == 0) break;
    const PtcField h = bf_field(n->gb[slot], ci, Vh);
    if (tc && tc_layer(co, ci))
      QKX_TRY(layer_tc(c, co, ci, g32, false, g, h, n->wt + n->woff[l], n->tc_err));
    else
      QKX_TRY(layer(c, co, ci, g, g32, h, false, n->wt + n->woff[l]));
    g = h;
    g32 = false;
    slot ^= 1;
  }
  return QKX_OK;
}

// loss on one pair: returns (on the device, at *loss_dev) |N(r) - e|^2 / |e|^2 and leaves
// dL/dy^* in g for backward; y goes to n->yout.  even_only: the loss of the even sites only
// (the even-odd solver reads N on the even sites), g zero on the odd ones.
int loss_and_output_grad(qkx_ptc* n, const float4* r, const float4* e, double e2, float4* g, double* loss_dev,
                         bool even_only = false) {
  qkx_ctx* c = n->c;
  QKX_TRY(forward(n, f32_field(r, c->Vh), f32_field(n->yout, c->Vh), n->use_tc != 0));
  const size_t n4 = even_only ? f32_words(c) / 2 : f32_words(c);
  const int gr = fgrid(n4);
  if (even_only) QKX_CUDA(cudaMemsetAsync(g + n4, 0, sizeof(float4) * n4, c->st));
  k_ptc_residual<<<gr, FNT, 0, c->st>>>(n->yout, e, g, n4, (float)(1.0 / e2), n->red);
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
  const size_t n4 = f32_words(c);
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

}  // namespace

// ---------------------------------------------------------------- learned-preconditioned solver
// Even-odd, batched, mixed precision.  All right-hand sides of a call are solved as one batch
// on the Schur system of the even sites,
//   Mh x_e = b^_e,   Mh = A_ee - k^2 D_eo A_oo^-1 D_oe,   b^_e = b_e + k D_eo A_oo^-1 b_o
// (A = 1 + i c g5: the operator's normalisation M = A - k D), through its normal equations
// Mh^+ Mh x_e = Mh^+ b^_e, by FP64 defect correction around a flexible CG in FP32.  The
// preconditioner is P = K K^+ with K = the network restricted to the even sites,
// K r = [N (r, 0)]_even: the even-even block of M^-1 is Mh^-1, so a network trained towards
// M^-1 gives K ~ Mh^-1 and P ~ (Mh^+ Mh)^-1.  P is Hermitian and positive by construction,
// whatever the network; K^+ is the network's adjoint (its layers in reverse order with the
// reversed-path, conjugate-transposed weights of the backward pass).  The flexible CG takes
// beta = -<z', A p> / <p, A p> (one-vector truncation), which tolerates the preconditioner's
// BF16 roundings.
// After each inner solve x_e += e in FP64 and the true Schur residual b^_e - Mh x_e is
// recomputed by the batched FP64 hop, whose residual epilogue stores g5 (b^_e - Mh x_e) in
// FP32 (the next normal residual is Mh^+ of it) and sums its norm in FP64.  The full residual
// b - M x equals the Schur one on the even sites and is zero on the odd ones, so a right-hand
// side stops at ||b^_e - Mh x_e|| <= 0.9 tol ||b||; then x_o = A_oo^-1 (b_o + k D_oe x_e) and
// ||b - M x|| is recomputed on the full lattice in FP64 and reported.  A right-hand side that
// spends maxIter iterations, or three outer passes without halving its residual, is finished
// by the even-odd mixed-precision CG from its full residual (the fallback).

// x += a y (real a), over n4 float4
static __global__ void k_f4_axpy(float4* __restrict__ x, float a, const float4* __restrict__ y, size_t n4) {
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    const float4 u = x[i], v = y[i];
    x[i] = make_float4(fmaf(a, v.x, u.x), fmaf(a, v.y, u.y), fmaf(a, v.z, u.z), fmaf(a, v.w, u.w));
  }
}

// x = y + b x (real b), over n4 float4
static __global__ void k_f4_xpby(float4* __restrict__ x, float b, const float4* __restrict__ y, size_t n4) {
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n4; i += (size_t)gridDim.x * FNT) {
    const float4 u = x[i], v = y[i];
    x[i] = make_float4(fmaf(b, u.x, v.x), fmaf(b, u.y, v.y), fmaf(b, u.z, v.z), fmaf(b, u.w, v.w));
  }
}

// single-parity FP64 batch member [12][Vh] += FP32 [6][Vh]
static __global__ void k_eo_add32(const float4* __restrict__ e, double2* __restrict__ x, int Vh) {
  const size_t n = (size_t)6 * Vh;
  for (size_t i = (size_t)blockIdx.x * FNT + threadIdx.x; i < n; i += (size_t)gridDim.x * FNT) {
    const size_t q = i / Vh, cb = i % Vh;
    const float4 f = e[i];
    double2& u = x[(2 * q) * Vh + cb];
    double2& v = x[(2 * q + 1) * Vh + cb];
    u.x += f.x;
    u.y += f.y;
    v.x += f.z;
    v.y += f.w;
  }
}

// one batched FP32 hop on the even-odd single-parity batches [R][6][Vh] (12-real FP32 links)
template <int EPI>
static int hop32(qkx_ctx* c, int R, float4* in, int in_par, float4* out, float4* x, double a, double csign,
                 const double* cvec, const double* svec, const int* active) {
  const int Vh = c->Vh;
  const size_t rs = (size_t)6 * Vh;
  const int op = 1 - in_par;  // output parity
  HopArgs<SpinorF32, GaugeF32x12> A{};
  A.gauge = GaugeF32x12{c->U12f, Vh};
  A.g = c->geom_raw;
  A.nrhs = R;
  A.nblk = mrhs_site_blocks<64>(Vh);
  A.in = in_par ? SpinorF32{nullptr, in, Vh, rs} : SpinorF32{in, nullptr, Vh, rs};
  A.out = op ? SpinorF32{nullptr, out, Vh, rs} : SpinorF32{out, nullptr, Vh, rs};
  A.x = op ? SpinorF32{nullptr, x, Vh, rs} : SpinorF32{x, nullptr, Vh, rs};
  A.out_parity = op;
  A.a = a;
  A.c = csign;
  A.s = 1.0;
  A.cvec = cvec;
  A.svec = svec;
  A.active = active;
  A.norm_part = nullptr;
  hop_mrhs_kernel<64, 1, SpinorF32, GaugeF32x12, float, 0, false, EPI><<<A.nblk * R, 64, 0, c->st>>>(A);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// out = Mh^+ Mh in (FP32 batch): g5 Mh(-c) g5 Mh(c), through te (even) and to (odd)
static int normal32(qkx_ctx* c, int R, float4* in, float4* out, float4* te, float4* to, const double* cvec,
                    const double* svec, const int* active) {
  const double k2 = c->p.kappa * c->p.kappa;
  QKX_TRY(hop32<EPI_TWIST_INV>(c, R, in, 0, to, in, 0.0, +1.0, cvec, svec, active));
  QKX_TRY(hop32<EPI_XPAY_G5>(c, R, to, 1, te, in, -k2, +1.0, cvec, nullptr, active));
  QKX_TRY(hop32<EPI_TWIST_INV>(c, R, te, 0, to, te, 0.0, -1.0, cvec, svec, active));
  return hop32<EPI_XPAY_G5>(c, R, to, 1, out, te, -k2, -1.0, cvec, nullptr, active);
}

// FP64 batch accessor over [R][12][Vh]
static SpinorF64 eo64(double2* base, int par, int Vh) {
  SpinorF64 s{};
  if (par) s.p1 = base;
  else s.p0 = base;
  s.Vh = Vh;
  s.rs = (size_t)12 * Vh;
  return s;
}

// out = N^+ in on FP32 4-channel fields: the layers in reverse order with the backward
// weights (reversed paths, conjugate transposes), hidden activations in gb[]; out_npar = 1
// computes parity out_par0 of the output only
int adjoint(qkx_ptc* n, PtcField in, PtcField out, bool tc, int out_par0, int out_npar) {
  const int Vh = n->c->Vh;
  PtcField src = in;
  bool s32 = true;
  int slot = 0;
  for (int l = n->nl - 1; l >= 0; l--) {
    const int ci = n->ch[l + 1], co = n->ch[l];  // the adjoint of layer l maps ch[l+1] -> ch[l]
    const bool last = l == 0;
    const PtcField dst = last ? out : bf_field(n->gb[slot], co, Vh);
    if (tc && tc_layer(ci, co))
      QKX_TRY(layer_tc(n->c, ci, co, s32, last, src, dst, n->wt + n->woff[l], n->tc_err, last ? out_par0 : 0,
                       last ? out_npar : 2));
    else
      QKX_TRY(layer(n->c, ci, co, src, s32, dst, last, n->wt + n->woff[l], last ? out_par0 : 0,
                    last ? out_npar : 2));
    src = dst;
    s32 = last;
    slot ^= 1;
  }
  return QKX_OK;
}

// device buffers of one solve, freed on every return path
struct EoScratch {
  cudaStream_t st = nullptr;
  std::vector<void*> p;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  template <class T>
  T* get(size_t n, int* rc, const char* what) {
    T* q = nullptr;
    if (*rc == QKX_OK && dalloc(&q, n, what) != QKX_OK) *rc = QKX_ERR_NOMEM;
    p.push_back(q);
    return q;
  }
  ~EoScratch() {
    if (st) cudaStreamSynchronize(st);
    for (void* q : p) cudaFree(q);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

int invert_gcr_ptc(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b, double2* const* x,
                   qkx_solve_info* info) {
  QKX_TRY(check_ready(c));
  qkx_ptc* net = const_cast<qkx_ptc*>(sp->preconditioner);
  if (net && net->c != c) return bad("the preconditioner belongs to another context");
  if (net) QKX_TRY(ensure_buffers(net));
  const int Vh = c->Vh, R = nrhs;
  const size_t n12 = (size_t)12 * Vh, hb = sizeof(double2) * n12;  // one parity, FP64
  const size_t n4e = (size_t)6 * Vh;                                // one parity, FP32 (float4)
  const double k = c->p.kappa;
  const int gr = fgrid(n4e);
  const int nblk_max = 2 * ((Vh + 31) / 32) + c3t_blocks(c->geom, -1) + 1;  // FP64 hop partials per RHS
  int rc = QKX_OK;
  EoScratch S;
  S.st = c->st;
  double2* bE = S.get<double2>(n12 * R, &rc, "solver fields");
  double2* bO = S.get<double2>(n12 * R, &rc, "solver fields");
  double2* g5bh = S.get<double2>(n12 * R, &rc, "solver fields");
  double2* x64 = S.get<double2>(n12 * R, &rc, "solver fields");
  double2* t64 = S.get<double2>(n12 * R, &rc, "solver fields");
  float4* rr = S.get<float4>(n4e * R, &rc, "solver fields");  // normal residual
  float4* zz = S.get<float4>(n4e * R, &rc, "solver fields");  // preconditioned residual
  float4* pp = S.get<float4>(n4e * R, &rc, "solver fields");  // search direction
  float4* qq = S.get<float4>(n4e * R, &rc, "solver fields");  // A p
  float4* ef = S.get<float4>(n4e * R, &rc, "solver fields");  // solution increment
  float4* te = S.get<float4>(n4e * R, &rc, "solver fields");  // even scratch
  float4* to = S.get<float4>(n4e * R, &rc, "solver fields");  // odd scratch
  float4* mid = S.get<float4>(n4e, &rc, "solver fields");     // K^+ r of one RHS
  float4* zero = S.get<float4>(n4e, &rc, "solver fields");
  double* part = S.get<double>((size_t)nblk_max * R, &rc, "partials");
  double* red = S.get<double>((size_t)2 * GCR_M * gr + 64, &rc, "partials");
  double* dsc = S.get<double>((size_t)10 * R, &rc, "scalars");  // [R] + [R] + [R][8]
  double* dtw = S.get<double>((size_t)2 * R, &rc, "twist factors");
  int* dact = S.get<int>((size_t)R, &rc, "masks");
  if (rc != QKX_OK) return rc;
  double* dres = dsc;    // |true residual|^2 per RHS
  double* db2 = dsc + R;  // |b|^2 per RHS
  double* dd = dsc + 2 * R;  // per RHS: up to 4 scalars of the current step (re, im pairs)
  auto F = [&](float4* base, int r) { return base + (size_t)r * n4e; };

  QKX_CUDA(cudaEventCreate(&S.ev[0]));
  QKX_CUDA(cudaEventCreate(&S.ev[1]));
  cudaEvent_t e0 = S.ev[0], e1 = S.ev[1];
  QKX_CUDA(cudaEventRecord(e0, c->st));
  // per-RHS twist factors
  std::vector<double> tw(2 * R), mu(R);
  for (int r = 0; r < R; r++) {
    mu[r] = sp->mu ? sp->mu[r] : c->p.mu;
    tw[r] = 2.0 * k * mu[r] * c->p.twistSign;
    tw[R + r] = 1.0 / (1.0 + tw[r] * tw[r]);
  }
  const double* cvec = dtw;
  const double* svec = dtw + R;
  QKX_CUDA(cudaMemcpyAsync(dtw, tw.data(), sizeof(double) * 2 * R, cudaMemcpyHostToDevice, c->st));
  std::vector<int> act(R, 1), inner(R, 0);
  auto upload_mask = [&](const std::vector<int>& m) -> int {
    QKX_CUDA(cudaMemcpyAsync(dact, m.data(), sizeof(int) * R, cudaMemcpyHostToDevice, c->st));
    QKX_CUDA(cudaStreamSynchronize(c->st));  // m may change before an asynchronous copy would run
    return QKX_OK;
  };
  auto read = [&](const double* d, double* h, int cnt) -> int {
    QKX_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->st));
    QKX_CUDA(cudaStreamSynchronize(c->st));
    return QKX_OK;
  };
  // complex dots <a_j, b> (j < na) of RHS r into dd[r*8 + 2j], dd[r*8 + 2j + 1]
  auto dots = [&](int r, std::initializer_list<const float4*> as, const float4* bv) {
    F4Ptrs A{};
    int na = 0;
    for (const float4* a : as) A.p[na++] = a;
    k_cdot_multi<<<gr, FNT, 0, c->st>>>(A, na, bv, n4e, red);
    k_sum_parts<<<2 * na, FNT, 0, c->st>>>(red, gr, 2 * na, dd + (size_t)r * 8);
    counted(c, 2);
  };
  // z = P r = K (K^+ r) for RHS r, or z = r without a network
  auto precondition = [&](int r) -> int {
    if (!net) {
      QKX_CUDA(cudaMemcpyAsync(F(zz, r), F(rr, r), sizeof(float4) * n4e, cudaMemcpyDeviceToDevice, c->st));
      return QKX_OK;
    }
    const bool tc = net->use_tc != 0;
    QKX_TRY(adjoint(net, PtcField{{F(rr, r), zero}}, PtcField{{mid, nullptr}}, tc, 0, 1));
    return forward(net, PtcField{{mid, zero}}, PtcField{{F(zz, r), nullptr}}, tc, 0, 1);
  };

  // --- set-up (FP64): gather b, |b|^2, b^_e = b_e + k D_eo A_oo^-1 b_o and g5 b^_e; x_e = 0
  QKX_CUDA(cudaMemsetAsync(zero, 0, sizeof(float4) * n4e, c->st));
  for (int r = 0; r < R; r++) {
    QKX_CUDA(cudaMemcpyAsync(bE + r * n12, b[r], hb, cudaMemcpyDeviceToDevice, c->st));
    QKX_CUDA(cudaMemcpyAsync(bO + r * n12, b[r] + n12, hb, cudaMemcpyDeviceToDevice, c->st));
    const int g2 = fgrid(2 * n12);
    k_norm64<<<g2, FNT, 0, c->st>>>(b[r], 2 * n12, red);
    k_sum_parts<<<1, FNT, 0, c->st>>>(red, g2, 1, db2 + r);
    counted(c, 2);
    QKX_TRY(site_op_acc(c, 0, SITE_TWIST_INV, eo64(bO + r * n12, 1, Vh), eo64(t64 + r * n12, 1, Vh), 1, 1, tw[r],
                        tw[R + r]));
  }
  QKX_TRY(upload_mask(act));
  QKX_TRY(hop64_batch(c, EPI_XPAY, R, eo64(t64, 1, Vh), eo64(x64, 0, Vh), eo64(bE, 0, Vh), 0, k, 0.0, cvec, nullptr,
                      dact, nullptr, nullptr));  // b^ into x64 for the moment
  for (int r = 0; r < R; r++)
    QKX_TRY(site_op_acc(c, 0, SITE_GAMMA5, eo64(x64 + r * n12, 0, Vh), eo64(g5bh + r * n12, 0, Vh), 0, 1, 0.0, 1.0));
  QKX_CUDA(cudaMemsetAsync(x64, 0, hb * R, c->st));
  std::vector<double> b2(R), r2(R), prev(R, 0.0), h((size_t)8 * R);
  QKX_TRY(read(db2, b2.data(), R));
  const double target = 0.9 * sp->tol;
  std::vector<int> its(R, 0), stall(R, 0), fb(R, 0);
  for (int r = 0; r < R; r++)
    if (!(b2[r] > 0)) act[r] = 0;  // zero source: x = 0
  int passes = 0;
  for (;;) {
    // --- true Schur residual (FP64): te = g5 (b^ - Mh x_e) in FP32, |.|^2 into dres
    QKX_TRY(upload_mask(act));
    QKX_TRY(hop64_batch(c, EPI_TWIST_INV, R, eo64(x64, 0, Vh), eo64(t64, 1, Vh), eo64(x64, 0, Vh), 1, 0.0, 1.0, cvec,
                        svec, dact, nullptr, nullptr));
    int nb = 0;
    QKX_TRY(hop64_batch_res(c, R, eo64(t64, 1, Vh), eo64(x64, 0, Vh), eo64(g5bh, 0, Vh),
                            SpinorF32{te, nullptr, Vh, n4e}, 0, -k * k, 1.0, cvec, dact, part, &nb, true));
    k_sum_parts<<<R, FNT, 0, c->st>>>(part, nb, R, dres);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    QKX_TRY(read(dres, r2.data(), R));
    int nact = 0;
    for (int r = 0; r < R; r++) {
      if (!act[r]) continue;
      if (!(r2[r] == r2[r])) {
        set_error("learned solver: the residual of right-hand side %d is NaN", r);
        return QKX_ERR_NAN;
      }
      if (r2[r] <= target * target * b2[r]) {
        act[r] = 0;
        continue;
      }
      if (passes > 0) stall[r] = r2[r] > 0.25 * prev[r] ? stall[r] + 1 : 0;
      prev[r] = r2[r];
      if (its[r] >= sp->maxIter || stall[r] >= 3) {
        act[r] = 0;
        fb[r] = 1;
        continue;
      }
      nact++;
    }
    if (nact == 0) break;
    passes++;
    // --- normal residual r = Mh^+ (b^ - Mh x_e) = g5 Mh(-c) te, e = 0, z = P r, p = z
    QKX_TRY(hop32<EPI_TWIST_INV>(c, R, te, 0, to, te, 0.0, -1.0, cvec, svec, dact));
    QKX_TRY(hop32<EPI_XPAY_G5>(c, R, to, 1, rr, te, -k * k, -1.0, cvec, nullptr, dact));
    QKX_CUDA(cudaMemsetAsync(ef, 0, sizeof(float4) * n4e * R, c->st));
    std::vector<double> rz(R), rn0(R), tgt(R);
    for (int r = 0; r < R; r++) {
      inner[r] = act[r];
      if (!act[r]) continue;
      QKX_TRY(precondition(r));
      QKX_CUDA(cudaMemcpyAsync(F(pp, r), F(zz, r), sizeof(float4) * n4e, cudaMemcpyDeviceToDevice, c->st));
      dots(r, {F(rr, r), F(zz, r)}, F(rr, r));  // |r|^2, <z, r>
    }
    QKX_TRY(read(dd, h.data(), 8 * R));
    for (int r = 0; r < R; r++) {
      if (!act[r]) continue;
      rn0[r] = h[(size_t)r * 8];
      rz[r] = h[(size_t)r * 8 + 2];
      // the FP32 inner solve: |r| down by 1e-6 (the recursive FP32 residual keeps falling past
      // that; the pass's FP64 residual then says how far the true one went), or by what the
      // outer target still needs
      const double rel = sqrt(r2[r] / b2[r]);
      const double t = std::max(0.5 * sp->tol / rel, 1e-6);
      tgt[r] = t * t * rn0[r];
    }
    for (;;) {
      int nin = 0;
      for (int r = 0; r < R; r++) nin += inner[r];
      if (nin == 0) break;
      QKX_TRY(upload_mask(inner));
      // q = A p
      QKX_TRY(normal32(c, R, pp, qq, te, to, cvec, svec, dact));
      for (int r = 0; r < R; r++)
        if (inner[r]) dots(r, {F(pp, r)}, F(qq, r));  // <p, A p>
      QKX_TRY(read(dd, h.data(), 8 * R));
      std::vector<double> pq(R, 0.0);
      for (int r = 0; r < R; r++) {
        if (!inner[r]) continue;
        pq[r] = h[(size_t)r * 8];
        if (!(pq[r] > 0)) {  // A p vanished (or NaN): this RHS's inner solve ends here
          inner[r] = 0;
          continue;
        }
        const float al = (float)(rz[r] / pq[r]);
        k_f4_axpy<<<gr, FNT, 0, c->st>>>(F(ef, r), al, F(pp, r), n4e);
        k_f4_axpy<<<gr, FNT, 0, c->st>>>(F(rr, r), -al, F(qq, r), n4e);
        counted(c, 2);
        QKX_TRY(precondition(r));
        dots(r, {F(rr, r), F(zz, r), F(qq, r)}, F(zz, r));  // <r, z>, |z|^2 (unused), <q, z>
        // |r|^2 for the stop: the same kernel on (r, r) into the fourth pair
        F4Ptrs one{};
        one.p[0] = F(rr, r);
        k_cdot_multi<<<gr, FNT, 0, c->st>>>(one, 1, F(rr, r), n4e, red);
        k_sum_parts<<<1, FNT, 0, c->st>>>(red, gr, 1, dd + (size_t)r * 8 + 6);
        counted(c, 2);
      }
      QKX_CUDA(cudaGetLastError());
      QKX_TRY(read(dd, h.data(), 8 * R));
      for (int r = 0; r < R; r++) {
        if (!inner[r]) continue;
        its[r]++;
        const double rz_new = h[(size_t)r * 8], qz = h[(size_t)r * 8 + 4], rn = h[(size_t)r * 8 + 6];
        if (!(rn == rn) || !(rz_new == rz_new)) {
          set_error("learned solver: the inner residual of right-hand side %d is NaN", r);
          return QKX_ERR_NAN;
        }
        if (rn <= tgt[r] || its[r] >= sp->maxIter || !(rz_new > 0)) {
          inner[r] = 0;
          continue;
        }
        // flexible CG: beta = -<z', A p> / <p, A p>, p = z' + beta p
        const float be = (float)(-qz / pq[r]);
        k_f4_xpby<<<gr, FNT, 0, c->st>>>(F(pp, r), be, F(zz, r), n4e);
        counted(c);
        rz[r] = rz_new;
      }
      QKX_CUDA(cudaGetLastError());
    }
    // x_e += e (FP64) on the RHS of this pass
    for (int r = 0; r < R; r++)
      if (act[r]) {
        k_eo_add32<<<fgrid(n4e), FNT, 0, c->st>>>(F(ef, r), x64 + r * n12, Vh);
        counted(c);
      }
    QKX_CUDA(cudaGetLastError());
  }
  // --- odd sites, solutions out
  std::vector<int> all(R, 1);
  QKX_TRY(upload_mask(all));
  QKX_TRY(hop64_batch(c, EPI_XPAY_TWINV, R, eo64(x64, 0, Vh), eo64(t64, 1, Vh), eo64(bO, 1, Vh), 1, k, 1.0, cvec,
                      svec, dact, nullptr, nullptr));
  for (int r = 0; r < R; r++) {
    QKX_CUDA(cudaMemcpyAsync(x[r], x64 + r * n12, hb, cudaMemcpyDeviceToDevice, c->st));
    QKX_CUDA(cudaMemcpyAsync(x[r] + n12, t64 + r * n12, hb, cudaMemcpyDeviceToDevice, c->st));
  }
  // --- fallback: the mixed-precision CG on M d = b - M x, then x += d
  std::vector<int> fbl;
  for (int r = 0; r < R; r++)
    if (fb[r]) fbl.push_back(r);
  int fb_iters = 0;
  if (!fbl.empty()) {
    const int nF = (int)fbl.size();
    double2* rf = S.get<double2>(2 * n12 * nF, &rc, "fallback fields");
    double2* df = S.get<double2>(2 * n12 * nF, &rc, "fallback fields");
    double2* mx = S.get<double2>(2 * n12, &rc, "fallback fields");
    if (rc != QKX_OK) return rc;
    std::vector<const double2*> bb(nF);
    std::vector<double2*> xx(nF);
    double worst_rel = 0.0;
    for (int i = 0; i < nF; i++) {
      const int r = fbl[i];
      QKX_TRY(apply_tm_mu(c, x[r], mx, false, mu[r]));
      const int g2 = fgrid(2 * n12);
      k_res64<<<g2, FNT, 0, c->st>>>(b[r], mx, rf + i * 2 * n12, 2 * n12, red);
      k_sum_parts<<<1, FNT, 0, c->st>>>(red, g2, 1, dres + r);
      counted(c, 2);
      double rr = 0;
      QKX_TRY(read(dres + r, &rr, 1));
      worst_rel = std::max(worst_rel, sqrt(rr / b2[r]));
      bb[i] = rf + i * 2 * n12;
      xx[i] = df + i * 2 * n12;
    }
    qkx_solver_params fp = *sp;
    fp.method = QKX_SOLVER_CG_EO_MIXED;
    fp.sloppy_precision = QKX_PREC_HALF;
    fp.tol = std::min(0.5, 0.9 * sp->tol / std::max(worst_rel, 1e-300));
    fp.maxIter = 100000;  // the learned solver's budget is spent; the fallback solves to completion
    fp.preconditioner = nullptr;
    std::vector<double> fmu(nF);
    for (int i = 0; i < nF; i++) fmu[i] = mu[fbl[i]];
    fp.mu = fmu.data();
    qkx_solve_info fi{};
    const int frc = invert_eo_mixed(c, &fp, nF, bb.data(), xx.data(), &fi);
    if (frc != QKX_OK && frc != QKX_ERR_NOT_CONVERGED) return frc;
    fb_iters = fi.iterations;
    for (int i = 0; i < nF; i++) {
      const int r = fbl[i];
      k_add64<<<fgrid(2 * n12), FNT, 0, c->st>>>(xx[i], x[r], 2 * n12);
      counted(c);
      QKX_CUDA(cudaMemcpyAsync(x64 + r * n12, x[r], hb, cudaMemcpyDeviceToDevice, c->st));
      QKX_CUDA(cudaMemcpyAsync(t64 + r * n12, x[r] + n12, hb, cudaMemcpyDeviceToDevice, c->st));
    }
  }
  // --- ||b - M x||^2 on the full lattice in FP64 (x: even half x64, odd half t64)
  int nbr = 0;
  SpinorF64 xf = eo64(x64, 0, Vh);
  xf.p1 = t64;
  SpinorF64 bf = eo64(bE, 0, Vh);
  bf.p1 = bO;
  QKX_TRY(hop64_batch_res(c, R, xf, xf, bf, SpinorF32{nullptr, nullptr, Vh, 0}, -1, -k, 1.0, cvec, dact, part, &nbr,
                          false));
  k_sum_parts<<<R, FNT, 0, c->st>>>(part, nbr, R, dres);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_TRY(read(dres, r2.data(), R));
  cudaEventRecord(e1, c->st);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (net) QKX_TRY(check_tc(net));
  double worst = 0.0;
  int maxit = 0, nfb = 0;
  for (int r = 0; r < R; r++) {
    worst = std::max(worst, b2[r] > 0 ? sqrt(r2[r] / b2[r]) : 0.0);
    maxit = std::max(maxit, its[r]);
    nfb += fb[r];
  }
  const bool conv = worst <= sp->tol;
  if (info) {
    info->iterations = maxit + fb_iters;
    info->restarts = passes;
    info->fallbacks = nfb;
    info->true_residual = worst;
    info->normal_residual = worst;
    info->converged = conv ? 1 : 0;
    info->seconds = ms * 1e-3;
  }
  if (!conv) set_error("learned solver: true residual %g above tol %g", worst, sp->tol);
  return conv ? QKX_OK : QKX_ERR_NOT_CONVERGED;
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
  for (int l = 0; l <= QKX_PTC_MAX_LAYERS; l++) cudaFree(n->hid[l]);
  cudaFree(n->yout);
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
  QKX_TRY(dalloc(&a, f32_words(c), "PTC input"));
  if (dalloc(&y, f32_words(c), "PTC output") != QKX_OK) {
    cudaFree(a);
    return QKX_ERR_NOMEM;
  }
  int rc = upload_f32(n, in_host, a, c->w[0]);
  if (rc == QKX_OK) rc = forward(n, f32_field(a, c->Vh), f32_field(y, c->Vh), n->use_tc != 0);
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
  QKX_TRY(dalloc(&f, 3 * f32_words(c), "PTC pair"));
  float4 *r = f, *e = f + f32_words(c), *g = f + 2 * f32_words(c);
  double e2 = 0;
  int rc = upload_f32(n, r_host, r, c->w[0]);
  if (rc == QKX_OK) rc = upload_f32(n, e_host, e, c->w[0]);
  if (rc == QKX_OK) rc = norm2_f32(n, e, &e2);
  if (rc == QKX_OK && !(e2 > 0)) rc = bad("|e| = 0");
  if (rc == QKX_OK) rc = loss_and_output_grad(n, r, e, e2, g, c->dscal + 1);
  if (rc == QKX_OK && grad) rc = backward(n, f32_field(r, c->Vh), f32_field(g, c->Vh), n->use_tc != 0);
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
  const size_t fw = f32_words(c);            // float4 per FP32 spinor
  const size_t n64 = (size_t)12 * c->V;      // double2 per FP64 spinor
  // pairs on the even-odd Schur system the solver preconditions (inputs zero on the odd sites,
  // loss on the even sites): [0, ns) r = b^_e, e = x_e = Mh^-1 b^_e from mixed-CG solves of
  // Gaussian b (b^_e = b_e + k D_eo A_oo^-1 b_o, x_e the even half of M^-1 b); [ns, 2 ns)
  // r = Mh v_e, e = v_e for Gaussian v, the short-distance part of Mh^-1
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
    const int Vh = c->Vh;
    const double k = c->p.kappa;
    const double tw = 2.0 * k * c->p.mu * c->p.twistSign, inv = 1.0 / (1.0 + tw * tw);
    const int B = std::min(ns, 16);
    double2* buf = nullptr;
    if (dalloc(&buf, n64 * (2 * B + 2), "data solves") != QKX_OK) {
      cudaFree(pairs);
      return QKX_ERR_NOMEM;
    }
    double2* s1 = buf + (size_t)2 * B * n64;  // FP64 scratch fields
    double2* s2 = s1 + n64;
    // FP32 pair member from the even half of an FP64 field, odd half zero
    auto even32 = [&](const double2* src, float4* dst) {
      k_f64_to_f32<<<fgrid(n64), FNT, 0, c->st>>>(src, dst, Vh);
      counted(c);
      cudaMemsetAsync(dst + fw / 2, 0, sizeof(float4) * (fw / 2), c->st);
    };
    for (int i0 = 0; i0 < ns && rc == QKX_OK; i0 += B) {
      const int nb = std::min(B, ns - i0);
      std::vector<const double2*> bp(nb);
      std::vector<double2*> xp(nb);
      for (int j = 0; j < nb; j++) {
        double2* bk = buf + (size_t)j * n64;
        k_spinor_gaussian<<<(unsigned)((c->V + 127) / 128), 128, 0, c->st>>>(bk, c->geom,
                                                                          tp->seed * 1000003ULL + i0 + j);
        counted(c);
        bp[j] = bk;
        xp[j] = buf + (size_t)(B + j) * n64;
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
      for (int j = 0; j < nb && rc == QKX_OK; j++) {
        // b^_e = b_e + k D_eo A_oo^-1 b_o into s2
        rc = site_op_acc(c, 0, SITE_TWIST_INV, F64(bp[j], Vh), F64(s1, Vh), 1, 1, tw, inv);
        if (rc == QKX_OK)
          rc = hop64a(c, 0, false, EPI_XPAY, F64(s1, Vh), F64(s2, Vh), F64(bp[j], Vh), true, 0, k, 0.0, 1.0, nullptr);
        if (rc != QKX_OK) break;
        float4* r = pairs + (size_t)(i0 + j) * 2 * fw;
        even32(s2, r);
        even32(xp[j], r + fw);
        rc = norm2_f32(n, r + fw, &e2[i0 + j]);
      }
      // operator pairs: v Gaussian, r = Mh v_e (FP64 operator), e = v_e
      for (int j = 0; j < nb && rc == QKX_OK; j++) {
        double2* v = buf + (size_t)j * n64;
        k_spinor_gaussian<<<(unsigned)((c->V + 127) / 128), 128, 0, c->st>>>(
            v, c->geom, (tp->seed * 1000003ULL + i0 + j) ^ 0xA5A5A5A5ULL);
        counted(c);
        rc = hop64a(c, 0, false, EPI_TWIST_INV, F64(v, Vh), F64(s1, Vh), F64(v, Vh), false, 1, 0.0, tw, inv, nullptr);
        if (rc == QKX_OK)
          rc = hop64a(c, 0, false, EPI_XPAY, F64(s1, Vh), F64(s2, Vh), F64(v, Vh), true, 0, -k * k, tw, 1.0, nullptr);
        if (rc != QKX_OK) break;
        float4* r = pairs + (size_t)(ns + i0 + j) * 2 * fw;
        even32(s2, r);
        even32(v, r + fw);
        rc = norm2_f32(n, r + fw, &e2[ns + i0 + j]);
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
      QKX_TRY(loss_and_output_grad(n, r, r + fw, e2[evals[k]], g, losses + slot0 + k, true));
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
    rc = loss_and_output_grad(n, r, r + fw, e2[k], g, losses + s, true);
    if (rc == QKX_OK) rc = backward(n, f32_field(r, c->Vh), f32_field(g, c->Vh), n->use_tc != 0);
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
