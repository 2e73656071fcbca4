// mixed.cu -- even-odd Schur-complement CG with sloppy spinors and links,
// FP64 reliable updates, batched over right-hand sides (and twisted masses),
// the inner iteration replayed from a CUDA graph.
//
// System (reference operator Vector::tm, lib/lattice_util.cpp:1925; its Schur
// form Vector::tm_xx, :2001-2022):
//   M = [[A, -k D_eo], [-k D_oe, A]],  A = 1 + i c g5,  c = 2 kappa mu twistSign
//   b^_e = b_e + k D_eo A^-1 b_o
//   Mh = A - k^2 D_eo A^-1 D_oe   solved on the normal equations Mh^+ Mh x_e = Mh^+ b^_e
//   Mh^+ = g5 Mh(-c) g5           (the reference builds tm_xxDagTm_xx the same way, :2024)
//   x_o = A^-1 (b_o + k D_oe x_e)
// ||b - M x|| = ||b^_e - Mh x_e|| exactly, so the FP64 Schur residual that each
// reliable update computes is the true residual of the full system; the end of
// the solve recomputes ||b - M x|| on the full lattice in FP64 as well.
//
// Inner iterations (all right-hand sides of the batch in lock-step, per-RHS
// scalars in device memory, converged RHS masked off):
//   t_o  = A^-1(c) D_oe p_e                   hop, TWIST_INV
//   y_e  = g5 (A(c) p_e - k^2 D_eo t_o)        hop, XPAY_G5, |y|^2 = <p, Mh^+Mh p> fused
//   t_o  = A^-1(-c) D_oe y_e                  hop, TWIST_INV
//   Ap_e = g5 (A(-c) y_e - k^2 D_eo t_o)       hop, XPAY_G5
//   alpha = r2 / pAp ; r_s -= alpha Ap ; r2' = |r_s|^2 ; beta ; x_s += alpha p ; p = r_s + beta p
// p, t, y, Ap are sloppy (FP16 + per-site norm, or FP32); r_s and x_s are FP32.
// A reliable update (all active right-hand sides together, so the FP64 hops
// share the links) folds x_s into the FP64 solution and recomputes the true
// residual rhat = b^ - Mh x with the FP64 operator on the 18-real links as the
// caller gave them; the residual the sloppy CG restarts from, Mh^+ rhat, is
// built from rhat in FP32.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <type_traits>
#include <vector>

#include "blas.cuh"
#include "hop.cuh"
#include "hop_mrhs.cuh"
#include "hop_pair.cuh"
#include "hop_c3t.cuh"
#include "qkx_ctx.cuh"
#include "site_ops.cuh"

namespace qkx {

// ---------------------------------------------------------------- precision traits
struct PHalf {
  static constexpr int id = QKX_PREC_HALF;
  using SP = SpinorF16;
  using GA = GaugeF16x12;
  using R = float;
  using AC = SpinorF32;
  // delta_min: FP16 storage cannot follow the residual much below 1e-3 of its value at the
  // last update (a 1e-3 threshold diverged on a 32^3x64 batch, 3e-3 converged)
  static constexpr double S = 52.0, G = 24.0, delta = 1e-2, delta_min = 5e-3;
};
struct PSingle {
  static constexpr int id = QKX_PREC_SINGLE;
  using SP = SpinorF32;
  using GA = GaugeF32x12;
  using R = float;
  using AC = SpinorF32;
  static constexpr double S = 96.0, G = 48.0, delta = 1e-5, delta_min = 1e-7;
};
struct PDouble {
  static constexpr int id = QKX_PREC_DOUBLE;
  using SP = SpinorF64;
  using GA = GaugeF64x18;
  using R = double;
  using AC = SpinorF64;
  static constexpr double S = 192.0, G = 144.0, delta = 1e-30, delta_min = 1e-30;
};

// a batch of single-parity fields: data [R][words][Vh] (+ norms [R][Vh] for FP16)
struct BField {
  void* d = nullptr;
  float* n = nullptr;
};

template <class SPT>
struct FieldTraits;
template <>
struct FieldTraits<SpinorF16> {
  static constexpr size_t words = 3;
  static SpinorF16 acc(const BField& f, int par, int Vh) {
    SpinorF16 s{};
    uint4* d = (uint4*)f.d;
    if (par) {
      s.p1 = d;
      s.n1 = f.n;
    } else {
      s.p0 = d;
      s.n0 = f.n;
    }
    s.Vh = Vh;
    s.rs = words * Vh;
    s.rsn = Vh;
    return s;
  }
};
template <>
struct FieldTraits<SpinorF32> {
  static constexpr size_t words = 6;
  static SpinorF32 acc(const BField& f, int par, int Vh) {
    SpinorF32 s{};
    if (par) s.p1 = (float4*)f.d;
    else s.p0 = (float4*)f.d;
    s.Vh = Vh;
    s.rs = words * Vh;
    return s;
  }
};
template <>
struct FieldTraits<SpinorF64> {
  static constexpr size_t words = 12;
  static SpinorF64 acc(const BField& f, int par, int Vh) {
    SpinorF64 s{};
    if (par) s.p1 = (double2*)f.d;
    else s.p0 = (double2*)f.d;
    s.Vh = Vh;
    s.rs = words * Vh;
    return s;
  }
};

// FP64 batch accessor over a raw [R][12][Vh] buffer
static SpinorF64 B64(double2* base, int par, int Vh) {
  SpinorF64 s{};
  if (par) s.p1 = base;
  else s.p0 = base;
  s.Vh = Vh;
  s.rs = 12 * (size_t)Vh;
  return s;
}
// FP64 batch accessor over two [R][12][Vh] buffers holding the even and odd halves
static SpinorF64 B64full(double2* even, double2* odd, int Vh) {
  SpinorF64 s{};
  s.p0 = even;
  s.p1 = odd;
  s.Vh = Vh;
  s.rs = 12 * (size_t)Vh;
  return s;
}

template <class SPT>
static int bfield_alloc(BField& f, int R, int Vh) {
  using T = FieldTraits<SPT>;
  if (cudaMalloc(&f.d, T::words * 16 * (size_t)Vh * R) != cudaSuccess) return QKX_ERR_NOMEM;
  if (std::is_same<SPT, SpinorF16>::value && cudaMalloc(&f.n, sizeof(float) * (size_t)Vh * R) != cudaSuccess)
    return QKX_ERR_NOMEM;
  return QKX_OK;
}
static void bfield_free(BField& f) {
  cudaFree(f.d);
  cudaFree(f.n);
  f.d = nullptr;
  f.n = nullptr;
}

// ---------------------------------------------------------------- kernels
constexpr int MX_NT = 256;
constexpr int MX_GRID = 148 * 2;  // blocks per RHS for the streaming kernels

// x_s += alpha p, then p = r_s + beta p (alpha of this iteration, beta from the new r_s)
template <class SP, class AC, typename R>
__global__ void __launch_bounds__(MX_NT) k_mx_update_p(SP p, AC xs, AC rs, const CgScalars* sc) {
  const int r = blockIdx.y;
  if (!sc->active[r]) return;
  const R alpha = R(sc->alpha[r]);
  const R beta = R(sc->beta[r]);
  const SP pr = p.shift(r);
  const AC xr = xs.shift(r), rr = rs.shift(r);
  for (int cb = blockIdx.x * MX_NT + threadIdx.x; cb < p.Vh; cb += gridDim.x * MX_NT) {
    Spinor<R> pv = pr.load(0, cb), rv = rr.load(0, cb), xv = xr.load(0, cb);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      Cx<R>& X = xv.c[k / 3][k % 3];
      X = X + alpha * pv.c[k / 3][k % 3];
      pv.c[k / 3][k % 3] = rv.c[k / 3][k % 3] + beta * pv.c[k / 3][k % 3];
    }
    xr.store(0, cb, xv);
    pr.store(0, cb, pv);
  }
}

enum { FIN_AUX = 10, FIN_AUX2 = 11, FIN_AUX_ADD = 12 };

// per-RHS finalize of [R][n] partials (one block per RHS)
__global__ void __launch_bounds__(256) k_mx_finalize(const double* part, int n, int mode, CgScalars* sc) {
  const int r = blockIdx.x;
  if (!sc->active[r]) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) acc += part[(size_t)r * n + i];
  double s = block_sum<256>(acc);
  if (threadIdx.x == 0) {
    if (mode == FIN_PAP) {
      sc->pAp[r] = s;
      sc->alpha[r] = sc->r2[r] / s;
    } else if (mode == FIN_R2) {
      sc->r2_old[r] = sc->r2[r];
      sc->r2[r] = s;
      sc->beta[r] = s / sc->r2_old[r];
      sc->iters[r] += 1;
    } else if (mode == FIN_R2_INIT) {
      sc->r2[r] = s;
    } else if (mode == FIN_AUX) {
      sc->aux[r] = s;
    } else if (mode == FIN_AUX2) {
      sc->aux2[r] = s;
    } else {
      sc->aux[r] += s;
    }
  }
}

// dst(rhs r) = convert(src(rhs r)) for the active RHS of a batch of single-parity fields
template <class SOUT, typename ROUT>
__global__ void k_mx_from_f64(SpinorF64 src, SOUT dst, const int* active) {
  const int r = blockIdx.y;
  if (active && !active[r]) return;
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= src.Vh) return;
  Spinor<double> v = src.shift(r).load(0, cb);
  Spinor<ROUT> o;
#pragma unroll
  for (int k = 0; k < 12; k++) o.c[k / 3][k % 3] = {ROUT(v.c[k / 3][k % 3].re), ROUT(v.c[k / 3][k % 3].im)};
  dst.shift(r).store(0, cb, o);
}

// dst(rhs r) = src(rhs r) in dst's precision for the active RHS of a batch of single-parity fields
template <class SIN, class SOUT>
__global__ void k_mx_convert(SIN src, SOUT dst, const int* active) {
  const int r = blockIdx.y;
  if (active && !active[r]) return;
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= src.Vh) return;
  dst.shift(r).store(0, cb, src.shift(r).load(0, cb));
}

// dst(rhs r) = src(rhs r) widened to FP64, every RHS of the batch
template <class SIN, typename RIN>
__global__ void k_mx_to_f64(SIN src, SpinorF64 dst) {
  const int r = blockIdx.y;
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= dst.Vh) return;
  Spinor<RIN> v = src.shift(r).load(0, cb);
  Spinor<double> o;
#pragma unroll
  for (int k = 0; k < 12; k++) o.c[k / 3][k % 3] = {double(v.c[k / 3][k % 3].re), double(v.c[k / 3][k % 3].im)};
  dst.shift(r).store(0, cb, o);
}

// x64(r) += x_s(r) ; x_s(r) = 0   for the active RHS
template <class AC, typename R>
__global__ void k_mx_fold(AC xs, SpinorF64 x64, const int* active) {
  const int r = blockIdx.y;
  if (active && !active[r]) return;
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= x64.Vh) return;
  const AC xr = xs.shift(r);
  const SpinorF64 xo = x64.shift(r);
  Spinor<R> v = xr.load(0, cb);
  Spinor<double> o = xo.load(0, cb);
  Spinor<R> z;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    o.c[k / 3][k % 3] = o.c[k / 3][k % 3] + Cx<double>{double(v.c[k / 3][k % 3].re), double(v.c[k / 3][k % 3].im)};
    z.c[k / 3][k % 3] = {R(0), R(0)};
  }
  xo.store(0, cb, o);
  xr.store(0, cb, z);
}

// z(r) = a(r) - z(r), partial |z(r)|^2 (batch of single-parity FP64 fields)
__global__ void __launch_bounds__(MX_NT) k_mx_sub_norm(SpinorF64 a, SpinorF64 z, const int* active, double* part) {
  const int r = blockIdx.y;
  double* slot = part + (size_t)r * gridDim.x + blockIdx.x;
  if (active && !active[r]) {
    if (threadIdx.x == 0) *slot = 0.0;
    return;
  }
  const SpinorF64 ar = a.shift(r), zr = z.shift(r);
  double acc = 0.0;
  for (int cb = blockIdx.x * MX_NT + threadIdx.x; cb < a.Vh; cb += gridDim.x * MX_NT) {
    Spinor<double> u = ar.load(0, cb), v = zr.load(0, cb);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      Cx<double> d = u.c[k / 3][k % 3] - v.c[k / 3][k % 3];
      v.c[k / 3][k % 3] = d;
      acc += d.re * d.re + d.im * d.im;
    }
    zr.store(0, cb, v);
  }
  double s = block_sum<MX_NT>(acc);
  if (threadIdx.x == 0) *slot = s;
}

// partial |a(r)|^2 (batch of single-parity FP64 fields)
__global__ void __launch_bounds__(MX_NT) k_mx_norm(SpinorF64 a, double* part) {
  const int r = blockIdx.y;
  const SpinorF64 ar = a.shift(r);
  double acc = 0.0;
  for (int cb = blockIdx.x * MX_NT + threadIdx.x; cb < a.Vh; cb += gridDim.x * MX_NT) {
    Spinor<double> u = ar.load(0, cb);
#pragma unroll
    for (int k = 0; k < 12; k++) acc += u.c[k / 3][k % 3].re * u.c[k / 3][k % 3].re + u.c[k / 3][k % 3].im * u.c[k / 3][k % 3].im;
  }
  double s = block_sum<MX_NT>(acc);
  if (threadIdx.x == 0) part[(size_t)r * gridDim.x + blockIdx.x] = s;
}

// site-local FP64 op on a batch of single-parity fields
template <int OP>
__global__ void k_mx_site(SpinorF64 in, SpinorF64 out, int par, const double* cvec, const double* svec) {
  const int r = blockIdx.y;
  int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= in.Vh) return;
  Spinor<double> v = in.shift(r).load(par, cb), o;
  if constexpr (OP == SITE_GAMMA5) {
    o = gamma5<0>(v);
  } else {  // twist inverse with the RHS's own mu
    o = twist_inv<0>(v, cvec[r], svec[r]);
  }
  out.shift(r).store(par, cb, o);
}

// ---------------------------------------------------------------- device-driven iteration loop
// The decisions of the reliable-update CG (when to recompute the FP64 residual, which
// right-hand sides have converged or diverged, where the search direction restarts) are
// taken on the device by one-block kernels, so that the whole iteration loop is one CUDA
// graph launch with two conditional WHILE nodes and the host waits once per solve.
struct MxCtl {
  double bnorm2[MAX_RHS];  // |b|^2
  double best[MAX_RHS];    // smallest FP64 true residual^2 so far (|b^|^2 at x = 0)
  double r2ru[MAX_RHS];    // sloppy r^2 right after the last reliable update
  double ratio[MAX_RHS];   // |rhat|^2 / |Mh^+ rhat|^2 at the last update
  double r2rec[MAX_RHS];   // sloppy r^2 of the last iteration
  double delta2;           // reliable_delta^2
  double target2;          // (0.9 tol)^2
  int nrhs, maxIter;
  int iter, since, n_ru, n_outer, n_restart, diverged;
  int nan_rhs, nan_iter;   // first right-hand side whose r^2 became NaN or inf, and when (0: none)
  int unconverged;         // right-hand sides still active when the loop ended
  unsigned long long t_ru0, ru_ns;  // device clock at the start of the last update; summed update time
  double cv[MAX_RHS], sv[MAX_RHS];  // per-RHS twist factors, staged here (page-locked) for the set-up's copies
};

__device__ __forceinline__ unsigned long long mx_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// start of the loop (one block of MAX_RHS threads): the per-RHS state from the set-up's norms
// (|b|^2 in aux, |b^|^2 in aux2, |Mh^+ b^|^2 in r2); the outer loop runs while any RHS is active
__global__ void __launch_bounds__(MAX_RHS) k_ctl_start(CgScalars* sc, MxCtl* ctl, cudaGraphConditionalHandle h_outer) {
  const int i = threadIdx.x;
  bool act = false;
  if (i < ctl->nrhs) {
    const double bn = sc->aux[i], rh = sc->aux2[i], r2 = sc->r2[i];
    ctl->bnorm2[i] = bn;
    sc->stop[i] = ctl->target2 * bn;
    ctl->best[i] = rh;
    ctl->r2ru[i] = r2;
    ctl->ratio[i] = r2 > 0 ? rh / r2 : 1.0;
    ctl->r2rec[i] = 0.0;
    act = !(bn == 0.0 || r2 == 0.0);
    sc->active[i] = act ? 1 : 0;
  }
  const int any = __syncthreads_or(act);
  if (i == 0) {
    ctl->iter = ctl->since = ctl->n_ru = ctl->n_outer = ctl->n_restart = ctl->diverged = 0;
    ctl->nan_rhs = MAX_RHS;
    ctl->nan_iter = 0;
    ctl->unconverged = 0;
    ctl->ru_ns = 0;
    cudaGraphSetConditional(h_outer, any ? 1u : 0u);
  }
}

// in a reliable update, once the FP64 true residuals are summed (aux): a RHS whose residual meets
// the tolerance stops there, before the FP32 Mh^+ rhat of the update, which then skips it.  The
// decisions after the update apply the same test to the same numbers and stop it too.
__global__ void __launch_bounds__(MAX_RHS) k_mx_stop_converged(CgScalars* sc, int nrhs) {
  const int i = threadIdx.x;
  if (i < nrhs && sc->active[i] && sc->aux[i] <= sc->stop[i]) sc->active[i] = 0;
}

// first node of every outer pass: the inner loop runs at least once
__global__ void k_ctl_inner_begin(cudaGraphConditionalHandle h_inner) { cudaGraphSetConditional(h_inner, 1u); }

// after each inner iteration: the inner loop stops when an RHS asks for a reliable update (its
// sloppy r^2 fell by delta^2 since the last one, or it looks converged), after 200 iterations
// without one, at maxIter, or when an r^2 is not finite
__global__ void __launch_bounds__(MAX_RHS) k_ctl_after_iter(const CgScalars* sc, MxCtl* ctl,
                                                            cudaGraphConditionalHandle h_inner) {
  const int i = threadIdx.x;
  bool act = false, ru = false, bad = false;
  if (i < ctl->nrhs && sc->active[i]) {
    act = true;
    const double r2s = sc->r2[i];
    if (!(r2s == r2s) || isinf(r2s)) bad = true;
    ctl->r2rec[i] = r2s;
    if (r2s < ctl->delta2 * ctl->r2ru[i] || r2s * ctl->ratio[i] <= ctl->target2 * ctl->bnorm2[i]) ru = true;
  }
  if (bad) atomicMin(&ctl->nan_rhs, i);
  const int any_act = __syncthreads_or(act), any_ru = __syncthreads_or(ru), any_bad = __syncthreads_or(bad);
  if (i == 0) {
    const int it = ++ctl->iter;
    const int since = ++ctl->since;
    if (any_bad && ctl->nan_iter == 0) ctl->nan_iter = it;
    const bool go = any_act && !any_ru && !any_bad && since < 200 && it < ctl->maxIter;
    if (!go) ctl->t_ru0 = mx_clock_ns();
    cudaGraphSetConditional(h_inner, go ? 1u : 0u);
  }
}

// after a reliable update (|rhat|^2 in aux, |Mh^+ rhat|^2 in aux2): converged and diverged RHS
// stop, the others restart their sloppy recursion from the new residual; the outer loop goes
// on while any RHS is active, below maxIter, with finite residuals
__global__ void __launch_bounds__(MAX_RHS) k_ctl_after_ru(CgScalars* sc, MxCtl* ctl, cudaGraphConditionalHandle h_outer) {
  const int i = threadIdx.x;
  bool act = false, rst = false, div = false;
  sc->restart[i] = 0;
  if (i < ctl->nrhs && sc->active[i]) {
    const double rhat2 = sc->aux[i], r2 = sc->aux2[i];
    if (rhat2 <= ctl->target2 * ctl->bnorm2[i] || r2 == 0.0) {
      sc->active[i] = 0;
    } else if (!(rhat2 <= 1e6 * ctl->best[i])) {  // the true residual grew 1000x above its best
      sc->active[i] = 0;
      div = true;
    } else {
      ctl->best[i] = fmin(ctl->best[i], rhat2);
      ctl->ratio[i] = rhat2 / r2;
      ctl->r2ru[i] = r2;
      sc->r2[i] = r2;
      // a residual much larger than the sloppy one it replaces restarts the search direction
      if (r2 > 4.0 * ctl->r2rec[i]) {
        sc->restart[i] = 1;
        rst = true;
      }
      act = true;
    }
  }
  const int any_act = __syncthreads_or(act), any_rst = __syncthreads_or(rst), ndiv = __syncthreads_count(div);
  if (i == 0) {
    ctl->n_ru++;
    ctl->n_outer++;
    ctl->since = 0;
    ctl->diverged += ndiv;
    if (any_rst) ctl->n_restart++;
    ctl->ru_ns += mx_clock_ns() - ctl->t_ru0;
    const bool go = any_act && ctl->iter < ctl->maxIter && ctl->nan_iter == 0;
    cudaGraphSetConditional(h_outer, go ? 1u : 0u);
  }
}

// after the loop: count the RHS that did not converge; every RHS takes part in the final phase
__global__ void __launch_bounds__(MAX_RHS) k_ctl_final(CgScalars* sc, MxCtl* ctl) {
  const int i = threadIdx.x;
  const bool act = i < ctl->nrhs && sc->active[i];
  const int n = __syncthreads_count(act);
  if (i < ctl->nrhs) sc->active[i] = 1;
  if (i == 0) ctl->unconverged = n;
}

// Builds the loop graph into `top` (which may already hold other work: the new nodes are roots
// of their own branch): emit(part, h_outer, h_inner) launches the kernels of each part on the
// context's stream while it is being captured (-1: top level, before anything else of the
// branch; 0: top level before the outer loop; 4: top level after it; 1: outer body before the
// inner loop; 2: outer body after it; 3: inner body).  The kernels each level launched come back
// in *kt, *ko, *ki.  Both handles default to 0 at every launch, so a loop whose condition is never
// set does not run.
template <class Emit>
static int build_loop_graph(qkx_ctx* c, cudaGraph_t top, long long* kt, long long* ko, long long* ki, Emit emit) {
  bool capturing = false;
  auto begin = [&](cudaGraph_t g) -> int {
    QKX_CUDA(cudaStreamBeginCaptureToGraph(c->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    c->capturing = 1;
    c->captured = 0;
    return QKX_OK;
  };
  auto end = [&](long long* k) -> int {
    c->capturing = 0;
    capturing = false;
    *k = c->captured;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (e != cudaSuccess) {
      set_error("graph capture: %s", cudaGetErrorString(e));
      return QKX_ERR_CUDA;
    }
    return QKX_OK;
  };
  // a WHILE node on what the capture has issued so far; later work depends on the node
  auto add_while = [&](cudaGraphConditionalHandle h, cudaGraph_t* body) -> int {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    QKX_CUDA(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    QKX_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
    *body = np.conditional.phGraph_out[0];
    QKX_CUDA(cudaStreamUpdateCaptureDependencies(c->st, &node, 1, cudaStreamSetCaptureDependencies));
    return QKX_OK;
  };
  auto run = [&]() -> int {
    cudaGraphConditionalHandle h_outer = 0, h_inner = 0;
    cudaGraph_t outer_body = nullptr, inner_body = nullptr;
    QKX_CUDA(cudaGraphConditionalHandleCreate(&h_outer, top, 0, cudaGraphCondAssignDefault));
    QKX_TRY(begin(top));
    QKX_TRY(emit(-1, h_outer, h_inner));
    QKX_TRY(emit(0, h_outer, h_inner));
    QKX_TRY(add_while(h_outer, &outer_body));
    QKX_TRY(emit(4, h_outer, h_inner));
    QKX_TRY(end(kt));
    QKX_CUDA(cudaGraphConditionalHandleCreate(&h_inner, outer_body, 0, cudaGraphCondAssignDefault));
    QKX_TRY(begin(outer_body));
    QKX_TRY(emit(1, h_outer, h_inner));
    QKX_TRY(add_while(h_inner, &inner_body));
    QKX_TRY(emit(2, h_outer, h_inner));
    QKX_TRY(end(ko));
    QKX_TRY(begin(inner_body));
    QKX_TRY(emit(3, h_outer, h_inner));
    QKX_TRY(end(ki));
    return QKX_OK;
  };
  const int rc = run();
  if (capturing) {  // a failed part: close the capture so the stream is usable again
    c->capturing = 0;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(c->st, &g);
    cudaGetLastError();
  }
  return rc;
}

// ---------------------------------------------------------------- solver state
struct MixedState {
  int prec = -1;
  int R = 0;
  BField p, Ap, t, y, rs, xs;  // sloppy batch fields
  // FP64 batches [R][12][Vh]
  double2 *bE = nullptr, *bO = nullptr, *x64 = nullptr, *g5bh = nullptr, *t64 = nullptr, *z64 = nullptr,
          *r64 = nullptr;
  double* cvec = nullptr;  // per-RHS 2 kappa mu_r twistSign
  double* svec = nullptr;  // per-RHS 1 / (1 + (2 kappa mu_r)^2)
  double* part = nullptr;  // [R][max(nblk, MX_GRID)]
  MxCtl* ctl = nullptr;    // decisions of the device-driven loop
  MxCtl* ctl_h = nullptr;  // page-locked host copy
  cudaGraphExec_t dgraph = nullptr;  // the device-driven iteration loop
  int dgraph_R = 0, dgraph_nr = 0, dgraph_nt = 0, dgraph_kind = 0;
  double dgraph_kappa = 0;
  long long dgraph_k[3] = {};  // kernels of its top level, outer pass, inner pass
  cudaGraphExec_t graph = nullptr;  // one iteration (host-driven loop)
  int graph_R = 0;
  int graph_nr = 0, graph_nt = 0, graph_kind = 0;  // hop tile the graph was captured with
  long long graph_kernels = 0;    // kernel nodes in the graph
  double graph_kappa = 0;         // kappa^2 is a kernel argument inside the graph
  std::vector<cudaEvent_t> gev;   // event pairs captured around the hop kernels
  cudaEvent_t ph[4] = {};         // phase marks: set-up done, reliable update start, its end, final start
};

void mixed_free(qkx_ctx* c) {
  MixedState* m = c->mixed;
  if (!m) return;
  cudaStreamSynchronize(c->st);
  for (BField* f : {&m->p, &m->Ap, &m->t, &m->y, &m->rs, &m->xs}) bfield_free(*f);
  for (double2* f : {m->bE, m->bO, m->x64, m->g5bh, m->t64, m->z64, m->r64}) cudaFree(f);
  cudaFree(m->cvec);
  cudaFree(m->svec);
  cudaFree(m->part);
  if (m->graph) cudaGraphExecDestroy(m->graph);
  if (m->dgraph) cudaGraphExecDestroy(m->dgraph);
  cudaFree(m->ctl);
  if (m->ctl_h) cudaFreeHost(m->ctl_h);
  for (auto e : m->gev) cudaEventDestroy(e);
  for (auto e : m->ph)
    if (e) cudaEventDestroy(e);
  delete m;
  c->mixed = nullptr;
}

// Sloppy hop fields (p, Ap, t, y) for R right-hand sides; with `solver` also
// the accumulators and FP64 batches the solve needs (tuning needs only the former).
template <class P>
static int mixed_alloc(qkx_ctx* c, int R, bool solver) {
  MixedState* m = c->mixed;
  if (m && (m->prec != P::id || m->R < R)) {
    mixed_free(c);
    m = nullptr;
  }
  if (!m) {
    m = new MixedState();
    c->mixed = m;
    m->prec = P::id;
    m->R = R;
  }
  const int Vh = c->Vh;
  int rc = QKX_OK;
  for (BField* f : {&m->p, &m->Ap, &m->t, &m->y})
    if (rc == QKX_OK && !f->d) rc = bfield_alloc<typename P::SP>(*f, m->R, Vh);
  if (rc == QKX_OK && !m->cvec && cudaMalloc(&m->cvec, sizeof(double) * MAX_RHS) != cudaSuccess) rc = QKX_ERR_NOMEM;
  if (rc == QKX_OK && !m->svec && cudaMalloc(&m->svec, sizeof(double) * MAX_RHS) != cudaSuccess) rc = QKX_ERR_NOMEM;
  // partials: the smallest hop block (64 threads) or the FP64 hop's row tiles (whichever is more)
  // over both parities, plus the streaming grid
  const size_t nblk =
      (size_t)std::max(hop_blocks_per_rhs<64>(Vh, -1), c3t_blocks(c->geom, -1)) + MX_GRID;
  if (rc == QKX_OK && !m->part && cudaMalloc(&m->part, sizeof(double) * (size_t)m->R * nblk) != cudaSuccess)
    rc = QKX_ERR_NOMEM;
  if (solver) {
    for (BField* f : {&m->rs, &m->xs})
      if (rc == QKX_OK && !f->d) rc = bfield_alloc<typename P::AC>(*f, m->R, Vh);
    const size_t h64 = sizeof(double2) * 12 * (size_t)Vh * m->R;
    for (double2** f : {&m->bE, &m->bO, &m->x64, &m->g5bh, &m->t64, &m->z64, &m->r64})
      if (rc == QKX_OK && !*f && cudaMalloc(f, h64) != cudaSuccess) rc = QKX_ERR_NOMEM;
    if (rc == QKX_OK && !m->ctl && cudaMalloc(&m->ctl, sizeof(MxCtl)) != cudaSuccess) rc = QKX_ERR_NOMEM;
    if (rc == QKX_OK && !m->ctl_h && cudaMallocHost(&m->ctl_h, sizeof(MxCtl)) != cudaSuccess) rc = QKX_ERR_NOMEM;
  }
  if (rc != QKX_OK) {
    mixed_free(c);
    set_error("mixed solver: device allocation for %d right-hand sides failed", R);
    return rc;
  }
  return QKX_OK;
}

// ---------------------------------------------------------------- multi-RHS sloppy hop
// Tile of the sloppy hop: NR right-hand sides per thread, NT threads per block,
// and the kernel kind.  Kind 0: hop_mrhs_kernel, or for FP16 with NR even the
// packed-pair hop_pair_kernel.  FP16 only, NR = 2 (register bounds are
// launch-bounds hints, 65536 registers / (bound x NT) blocks an SM):
//   1  hop_pair_pf_kernel, next term's loads held in registers, no bound
//   2  the same, 128 registers a thread
//   3  the same, about 100 registers a thread
//   4  hop_pair_kernel (one pair), 128 registers a thread
//   5  hop_pair_as_kernel, cp.async into shared memory, one term ahead, 128 registers
//   6  the same, two terms ahead
//   7  the same as 5, about 100 registers a thread
//   8  hop_pair_hp_kernel: as 5 with the spin projection in FP16 before widening
//   9  the same with 18-real FP32 links (no link conversion or rebuild)
//  10  hop_pair_hm_kernel: as 8 with the link multiply in FP16 on 18-real FP16 links.
//      Its products round to FP16, which costs the solver about one more reliable
//      update on a 32^3x64 batch, so the tuner does not pick it; qkx_set_tile does.
//  11  as 8 with the 18-real FP16 links (boundary sign included): nine half2
//      conversions a link and no third-row rebuild, for 12 more bytes a link.
struct HopTile {
  int nr = 0, nt = 0, kind = 0;
};
static const HopTile kTiles[] = {{1, 64, 0}, {1, 128, 0}, {1, 256, 0}, {2, 64, 0}, {2, 128, 0}, {2, 256, 0},
                                 {3, 64, 0}, {3, 128, 0}, {3, 256, 0}, {4, 64, 0}, {4, 128, 0}, {4, 256, 0},
                                 {2, 64, 1}, {2, 128, 1}, {2, 256, 1}, {2, 64, 2}, {2, 128, 2}, {2, 256, 2},
                                 {2, 64, 3}, {2, 128, 3}, {2, 64, 4}, {2, 128, 4}, {2, 256, 4}, {2, 64, 5},
                                 {2, 128, 5}, {2, 64, 6}, {2, 64, 7}, {2, 128, 7}, {2, 64, 8}, {2, 128, 8},
                                 {2, 64, 9},  {2, 128, 9}, {2, 64, 10}, {2, 128, 10}, {2, 64, 11},
                                 {2, 128, 11}};

template <int NT, int NR, int KIND, class SP, class GA, typename R, int EPI>
static int launch_mrhs(qkx_ctx* c, int R_, const GA& gauge, const Geom& g, SP in, SP out, SP x, int out_parity,
                       double a, double csign, bool with_s, double* norm_part, int prof_slot) {
  MixedState* m = c->mixed;
  HopArgs<SP, GA> A;
  A.out = out;
  A.in = in;
  A.x = x;
  A.gauge = gauge;
  A.g = g;
  A.out_parity = out_parity;
  A.a = a;
  A.c = csign;
  A.s = 1.0;
  A.norm_part = norm_part;
  A.nrhs = R_;
  A.nblk = mrhs_site_blocks<NT>(c->Vh);
  A.cvec = m->cvec;
  A.svec = with_s ? m->svec : nullptr;
  A.active = c->sc->active;
  if constexpr (EPI == EPI_XPAY_G5_CGR) {
    // the CG residual batch (FP32, or FP64 for FP64 sloppy) and the step lengths
    A.alpha = c->sc->alpha;
    if constexpr (std::is_same<R, double>::value) A.racc64 = FieldTraits<SpinorF64>::acc(m->rs, 0, c->Vh);
    else A.racc32 = FieldTraits<SpinorF32>::acc(m->rs, 0, c->Vh);
  }
  const int ngrp = (R_ + NR - 1) / NR;
  if (prof_slot >= 0) QKX_CUDA(cudaEventRecordWithFlags(m->gev[2 * prof_slot], c->st, cudaEventRecordExternal));
  constexpr bool f16 = std::is_same<SP, SpinorF16>::value && std::is_same<GA, GaugeF16x12>::value;
  // blocks an SM must hold: 65536 registers / (128 or about 100 a thread x NT)
  constexpr int B128 = 512 / NT, B100 = 640 / NT;
  if constexpr (KIND >= 1 && KIND <= 3) {
    static_assert(f16 && NR == 2, "pipelined tiles are FP16 pairs");
    constexpr int MINB = KIND == 1 ? 0 : (KIND == 2 ? B128 : B100);
    hop_pair_pf_kernel<NT, MINB, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A);
  } else if constexpr (KIND == 4) {
    static_assert(f16 && NR == 2, "pipelined tiles are FP16 pairs");
    hop_pair_kernel<NT, 1, 0, false, EPI, B128><<<A.nblk * ngrp, NT, 0, c->st>>>(A);
  } else if constexpr (KIND == 8 || KIND == 9 || KIND == 11) {
    static_assert(f16 && NR == 2, "pipelined tiles are FP16 pairs");
    if constexpr (KIND == 8) {
      const HLinks<0> G{gauge.a, gauge.b};
      hop_pair_hp_kernel<NT, 2, B128, 0, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A, G);
    } else if constexpr (KIND == 9) {
      const HLinks<1> G{(const uint4*)c->U18fa, (const uint2*)c->U18fb};
      hop_pair_hp_kernel<NT, 2, B128, 1, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A, G);
    } else {
      const HLinks<2> G{c->U18ha, nullptr, c->U18hb, c->U18hc};
      hop_pair_hp_kernel<NT, 2, B128, 2, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A, G);
    }
  } else if constexpr (KIND == 10) {
    static_assert(f16 && NR == 2, "pipelined tiles are FP16 pairs");
    const HLinks18 G{c->U18ha, c->U18hb, c->U18hc};
    hop_pair_hm_kernel<NT, B128, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A, G);
  } else if constexpr (KIND >= 5) {
    static_assert(f16 && NR == 2, "pipelined tiles are FP16 pairs");
    constexpr int S = KIND == 6 ? 3 : 2;
    constexpr int MINB = KIND == 7 ? B100 : B128;
    hop_pair_as_kernel<NT, S, MINB, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A);
  } else if constexpr (f16 && NR % 2 == 0) {
    hop_pair_kernel<NT, NR / 2, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A);
  } else {
    hop_mrhs_kernel<NT, NR, SP, GA, R, 0, false, EPI><<<A.nblk * ngrp, NT, 0, c->st>>>(A);
  }
  counted(c);
  QKX_CUDA(cudaGetLastError());
  if (prof_slot >= 0)
    QKX_CUDA(cudaEventRecordWithFlags(m->gev[2 * prof_slot + 1], c->st, cudaEventRecordExternal));
  return QKX_OK;
}

template <class SP, class GA, typename R, int EPI>
static int hop_tile(qkx_ctx* c, HopTile t, int R_, const GA& gauge, const Geom& g, SP in, SP out, SP x,
                    int out_parity, double a, double csign, bool with_s, double* norm_part, int prof_slot) {
#define QKX_TILE(NR_, NT_, K_)                                                                              \
  if (t.nr == NR_ && t.nt == NT_ && t.kind == K_)                                                          \
    return launch_mrhs<NT_, NR_, K_, SP, GA, R, EPI>(c, R_, gauge, g, in, out, x, out_parity, a, csign,     \
                                                     with_s, norm_part, prof_slot);
  QKX_TILE(1, 64, 0) QKX_TILE(1, 128, 0) QKX_TILE(1, 256, 0)
  QKX_TILE(2, 64, 0) QKX_TILE(2, 128, 0) QKX_TILE(2, 256, 0)
  QKX_TILE(3, 64, 0) QKX_TILE(3, 128, 0) QKX_TILE(3, 256, 0)
  QKX_TILE(4, 64, 0) QKX_TILE(4, 128, 0) QKX_TILE(4, 256, 0)
  if constexpr (std::is_same<SP, SpinorF16>::value && std::is_same<GA, GaugeF16x12>::value) {
    QKX_TILE(2, 64, 1) QKX_TILE(2, 128, 1) QKX_TILE(2, 256, 1)
    QKX_TILE(2, 64, 2) QKX_TILE(2, 128, 2) QKX_TILE(2, 256, 2)
    QKX_TILE(2, 64, 3) QKX_TILE(2, 128, 3)
    QKX_TILE(2, 64, 4) QKX_TILE(2, 128, 4) QKX_TILE(2, 256, 4)
    QKX_TILE(2, 64, 5) QKX_TILE(2, 128, 5) QKX_TILE(2, 64, 6)
    QKX_TILE(2, 64, 7) QKX_TILE(2, 128, 7)
    QKX_TILE(2, 64, 8) QKX_TILE(2, 128, 8) QKX_TILE(2, 64, 9) QKX_TILE(2, 128, 9)
    QKX_TILE(2, 64, 10) QKX_TILE(2, 128, 10)
    QKX_TILE(2, 64, 11) QKX_TILE(2, 128, 11)
  }
#undef QKX_TILE
  set_error("invalid hop tile (%d, %d, kind %d) for this precision", t.nr, t.nt, t.kind);
  return QKX_ERR_INVALID;
}

template <class P>
struct Sloppy {
  using SP = typename P::SP;
  using GA = typename P::GA;
  using R = typename P::R;
  using AC = typename P::AC;

  static GA gauge(qkx_ctx* c);
  static Geom geom(qkx_ctx* c) { return std::is_same<P, PDouble>::value ? c->geom : c->geom_raw; }

  // one inner CG iteration for all right-hand sides (graph-capturable)
  static int iteration(qkx_ctx* c, int R_, bool prof, HopTile tile) {
    MixedState* m = c->mixed;
    const int Vh = c->Vh;
    using FT = FieldTraits<SP>;
    using FA = FieldTraits<AC>;
    SP p = FT::acc(m->p, 0, Vh), t = FT::acc(m->t, 1, Vh), y = FT::acc(m->y, 0, Vh), Ap = FT::acc(m->Ap, 0, Vh);
    AC xs = FA::acc(m->xs, 0, Vh), rs = FA::acc(m->rs, 0, Vh);
    const double k2 = c->p.kappa * c->p.kappa;
    const int nblk = (Vh + tile.nt - 1) / tile.nt;
    const GA U = gauge(c);
    const Geom g = geom(c);
    QKX_TRY((hop_tile<SP, GA, R, EPI_TWIST_INV>(c, tile, R_, U, g, p, t, p, 1, 0.0, +1.0, true, nullptr,
                                                prof ? 0 : -1)));
    QKX_TRY((hop_tile<SP, GA, R, EPI_XPAY_G5>(c, tile, R_, U, g, t, y, p, 0, -k2, +1.0, false, m->part,
                                              prof ? 1 : -1)));
    k_mx_finalize<<<R_, 256, 0, c->st>>>(m->part, nblk, FIN_PAP, c->sc);
    counted(c);
    QKX_TRY((hop_tile<SP, GA, R, EPI_TWIST_INV>(c, tile, R_, U, g, y, t, y, 1, 0.0, -1.0, true, nullptr,
                                                prof ? 2 : -1)));
    // A p = g5 (A(-c) y - k^2 D t) goes straight into r -= alpha A p and |r|^2 (never stored)
    QKX_TRY((hop_tile<SP, GA, R, EPI_XPAY_G5_CGR>(c, tile, R_, U, g, t, Ap, y, 0, -k2, -1.0, false, m->part,
                                                  prof ? 3 : -1)));
    dim3 gr(MX_GRID, R_);
    k_mx_finalize<<<R_, 256, 0, c->st>>>(m->part, nblk, FIN_R2, c->sc);
    counted(c);
    k_mx_update_p<SP, AC, R><<<gr, MX_NT, 0, c->st>>>(p, xs, rs, c->sc);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    return QKX_OK;
  }

  // algorithmic bytes of one of the four inner hops, averaged, per RHS in a batch of R_:
  // per output site the input spinor and 8 links shared by the batch in the tile's link
  // format, plus the output spinor (hops 1 to 3), the xpay operand (hops 2 and 4) and the
  // CG residual read and written by the fourth hop's epilogue (FP32, or FP64 for FP64 sloppy)
  static double hop_bytes_per_rhs(qkx_ctx* c, int R_, const HopTile& tile) {
    const double S = P::S, Vh = c->Vh;
    const double Sr = std::is_same<AC, SpinorF64>::value ? 192.0 : 96.0;
    double G = P::G;
    if (P::id == QKX_PREC_HALF && tile.kind == 9) G = 72.0;  // 18-real FP32 links
    if (P::id == QKX_PREC_HALF && (tile.kind == 10 || tile.kind == 11)) G = 36.0;  // 18-real FP16 links
    const double hops = (2 * S) + (3 * S) + (2 * S) + (2 * S + 2 * Sr);
    return Vh * (hops / 4.0 + 8 * G / R_);
  }
};

template <>
GaugeF16x12 Sloppy<PHalf>::gauge(qkx_ctx* c) {
  return GaugeF16x12{c->U12ha, c->U12hb, c->Vh};
}
template <>
GaugeF32x12 Sloppy<PSingle>::gauge(qkx_ctx* c) {
  return GaugeF32x12{c->U12f, c->Vh};
}
template <>
GaugeF64x18 Sloppy<PDouble>::gauge(qkx_ctx* c) {
  return GaugeF64x18{c->U18, c->Vh};
}

// ---------------------------------------------------------------- autotuner
// Times the four hops of an inner iteration as the solver runs them (TWIST_INV,
// XPAY_G5 with the fused norm, TWIST_INV, and XPAY_G5 feeding the CG residual
// update) for every tile on this lattice and batch, on the solver's own fields,
// and keeps the fastest.  The result is cached in the context per (precision,
// batch size) and survives gauge reloads.
template <class P>
static int tune_tile(qkx_ctx* c, int R_, HopTile* best, double* best_ms) {
  using SP = typename P::SP;
  using GA = typename P::GA;
  using R = typename P::R;
  using FT = FieldTraits<SP>;
  MixedState* m = c->mixed;
  const int Vh = c->Vh;
  using FA = FieldTraits<typename P::AC>;
  SP p = FT::acc(m->p, 0, Vh), t = FT::acc(m->t, 1, Vh), y = FT::acc(m->y, 0, Vh), Ap = FT::acc(m->Ap, 0, Vh);
  const GA U = Sloppy<P>::gauge(c);
  const Geom g = Sloppy<P>::geom(c);
  CgScalars* sh = c->sc_h;
  for (int i = 0; i < MAX_RHS; i++) sh->active[i] = i < R_ ? 1 : 0;
  QKX_CUDA(cudaMemcpyAsync(c->sc->active, sh->active, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, c->st));
  QKX_CUDA(cudaMemsetAsync(c->sc->alpha, 0, sizeof(double) * MAX_RHS, c->st));
  QKX_CUDA(cudaMemsetAsync(m->p.d, 0, FT::words * 16 * (size_t)Vh * R_, c->st));
  if (m->p.n) QKX_CUDA(cudaMemsetAsync(m->p.n, 0, sizeof(float) * (size_t)Vh * R_, c->st));
  QKX_CUDA(cudaMemsetAsync(m->rs.d, 0, FA::words * 16 * (size_t)Vh * R_, c->st));
  cudaEvent_t e0, e1;
  QKX_CUDA(cudaEventCreate(&e0));
  QKX_CUDA(cudaEventCreate(&e1));
  *best_ms = 1e30;
  const double k2 = c->p.kappa * c->p.kappa;
  int rc = QKX_OK;
  std::vector<std::array<double, 4>> log;
  for (const HopTile& tile : kTiles) {
    if (tile.nr > 1 && tile.nr > R_) continue;
    if (tile.kind != 0 && P::id != QKX_PREC_HALF) continue;
    if (tile.kind == 10) continue;  // changes the rounding of the operator, chosen explicitly only
    for (int rep = 0; rep < 4 && rc == QKX_OK; rep++) {
      if (rep == 1) rc = cudaEventRecord(e0, c->st) == cudaSuccess ? QKX_OK : QKX_ERR_CUDA;
      if (rc == QKX_OK)
        rc = hop_tile<SP, GA, R, EPI_TWIST_INV>(c, tile, R_, U, g, p, t, p, 1, 0.0, 1.0, true, nullptr, -1);
      if (rc == QKX_OK)
        rc = hop_tile<SP, GA, R, EPI_XPAY_G5>(c, tile, R_, U, g, t, y, p, 0, -k2, 1.0, false, m->part, -1);
      if (rc == QKX_OK)
        rc = hop_tile<SP, GA, R, EPI_TWIST_INV>(c, tile, R_, U, g, y, t, y, 1, 0.0, -1.0, true, nullptr, -1);
      if (rc == QKX_OK)
        rc = hop_tile<SP, GA, R, EPI_XPAY_G5_CGR>(c, tile, R_, U, g, t, Ap, y, 0, -k2, -1.0, false, m->part, -1);
    }
    if (rc != QKX_OK) break;
    if (cudaEventRecord(e1, c->st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      rc = QKX_ERR_CUDA;
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double per_hop = ms / 12.0;
    log.push_back({double(tile.nr), double(tile.nt), double(tile.kind), per_hop});
    if (per_hop < *best_ms) {
      *best_ms = per_hop;
      *best = tile;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == QKX_OK) {
    c->tuned[P::id * 1000 + R_] = {best->nr, best->nt, best->kind};
    c->tune_log[P::id * 1000 + R_] = log;
  }
  return rc;
}

template <class P>
static int tile_for(qkx_ctx* c, int R_, HopTile* tile) {
  auto it = c->tuned.find(P::id * 1000 + R_);
  if (it != c->tuned.end()) {
    tile->nr = it->second.nr;
    tile->nt = it->second.nt;
    tile->kind = it->second.kind;
    return QKX_OK;
  }
  double ms;
  return tune_tile<P>(c, R_, tile, &ms);
}

// ---------------------------------------------------------------- batched FP64 pieces
using H18 = GaugeF64x18;

// out(r) = g5 Mh(csign * c_r) v(r) for the active RHS, through t64; optional |out|^2 partials
// (*nblk of them per RHS)
static int schur64_g5_batch(qkx_ctx* c, int R_, double csign, double2* v, double2* out, double* norm_part,
                            int* nblk = nullptr) {
  MixedState* m = c->mixed;
  const int Vh = c->Vh;
  const double k = c->p.kappa;
  QKX_TRY(hop64_batch(c, EPI_TWIST_INV, R_, B64(v, 0, Vh), B64(m->t64, 1, Vh), B64(v, 0, Vh), 1, 0.0, csign, m->cvec,
                      m->svec, c->sc->active, nullptr, nullptr));
  return hop64_batch(c, EPI_XPAY_G5, R_, B64(m->t64, 1, Vh), B64(out, 0, Vh), B64(v, 0, Vh), 0, -k * k, csign,
                     m->cvec, nullptr, c->sc->active, norm_part, nblk);
}

// r = g5 Mh(-c) g5 rhat = Mh^+ rhat for the active RHS, in FP32 on the 12-real FP32 links,
// from the FP64 field z = g5 rhat, into the FP32 field out, with |r|^2 partials per RHS in
// m->part (*nblk of them).  r is the residual the sloppy CG restarts from, so FP32 is enough:
// the true residual rhat it is built from is FP64, and the sloppy iterations that continue
// from r round to FP16 or FP32 themselves.  m->r64 is the scratch (the FP32 copy of z and
// the odd-parity intermediate, 96 B per site and RHS each).
static SpinorF32 scratch32(qkx_ctx* c, int R_, int which) {
  using F32 = FieldTraits<SpinorF32>;
  const BField f{(float4*)c->mixed->r64 + which * F32::words * (size_t)c->Vh * R_, nullptr};
  return F32::acc(f, which, c->Vh);  // 0: even-parity z32, 1: odd-parity t32
}

// the same from z = g5 rhat already in FP32 (the even half of the r64 scratch)
static int normal_residual_from32(qkx_ctx* c, int R_, SpinorF32 out, int* nblk) {
  MixedState* m = c->mixed;
  const int Vh = c->Vh;
  const double k = c->p.kappa;
  const SpinorF32 z32 = scratch32(c, R_, 0), t32 = scratch32(c, R_, 1);
  const GaugeF32x12 U{c->U12f, Vh};
  // the FP32 batch hop's tile with one RHS a thread and 64 threads (the tuner's choice for
  // FP32 at 12 RHS on 24^3x48 and 32^3x64)
  QKX_TRY((launch_mrhs<64, 1, 0, SpinorF32, GaugeF32x12, float, EPI_TWIST_INV>(c, R_, U, c->geom_raw, z32, t32, z32,
                                                                                1, 0.0, -1.0, true, nullptr, -1)));
  QKX_TRY((launch_mrhs<64, 1, 0, SpinorF32, GaugeF32x12, float, EPI_XPAY_G5>(c, R_, U, c->geom_raw, t32, out, z32, 0,
                                                                              -k * k, -1.0, false, m->part, -1)));
  *nblk = mrhs_site_blocks<64>(Vh);
  return QKX_OK;
}

static int normal_residual_f32(qkx_ctx* c, int R_, double2* z, SpinorF32 out, int* nblk) {
  const int Vh = c->Vh;
  const dim3 cg2((Vh + 255) / 256, R_);
  k_mx_from_f64<SpinorF32, float><<<cg2, 256, 0, c->st>>>(B64(z, 0, Vh), scratch32(c, R_, 0), c->sc->active);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return normal_residual_from32(c, R_, out, nblk);
}

// One even-odd mixed solve, in phases, so that a single solve can run them eagerly and a batch of
// lattices can capture the set-up, loop and final phase of each into one graph (qkx_invert_batch).
//   prepare()       allocation, tile, per-RHS twist factors and scalars into page-locked memory
//   setup()         b^, |b|^2, Mh^+ b^ and the starting fields, on the context's stream (capturable)
//   loop_graph()    the device-driven iteration loop added to a graph
//   host_loop()     the host-driven loop (hop kernels timed with events, or graphs off)
//   final_phase()   odd sites, the FP64 true residual, solutions out, scalars to the host (capturable)
//   finish()        solve info and status from the scalars the final phase copied back
template <class P>
struct MixedSolve {
  using SL = Sloppy<P>;
  using SP = typename P::SP;
  using AC = typename P::AC;
  using R = typename P::R;
  using FT = FieldTraits<SP>;
  using FA = FieldTraits<AC>;
  static constexpr bool r32 = std::is_same<AC, SpinorF32>::value;

  qkx_ctx* c;
  const qkx_solver_params* sp;
  int nrhs;
  const double2* const* b;
  double2* const* x;
  MixedState* m = nullptr;
  HopTile tile;
  int Vh = 0;
  size_t n12 = 0, hb = 0;
  double k = 0, delta = 0, target = 0;
  int maxIter = 0;
  dim3 cg2, bg2;
  bool device_loop = false;
  long long kcount[3] = {};  // kernels of the loop graph's top level, outer pass and inner pass
  // results of the host-driven loop (the device loop keeps them in MxCtl)
  int iter = 0, n_ru = 0, n_restart = 0, diverged = 0, nact = 0;
  float ms_ru = 0;
  std::vector<int> active;
  std::vector<double> bnorm2;

  MixedSolve(qkx_ctx* c_, const qkx_solver_params* sp_, int nrhs_, const double2* const* b_, double2* const* x_)
      : c(c_), sp(sp_), nrhs(nrhs_), b(b_), x(x_), active(nrhs_, 1), bnorm2(nrhs_) {}

  int prepare(bool allow_device_loop) {
    QKX_TRY(mixed_alloc<P>(c, nrhs, true));
    m = c->mixed;
    QKX_TRY(tile_for<P>(c, nrhs, &tile));
    Vh = c->Vh;
    n12 = 12 * (size_t)Vh;
    hb = sizeof(double2) * n12;
    k = c->p.kappa;
    const double ts = c->p.twistSign;
    delta = sp->reliable_delta > 0 ? std::max(P::delta_min, std::min(0.5, sp->reliable_delta)) : P::delta;
    target = 0.9 * sp->tol;
    maxIter = std::min(sp->maxIter, 1000000);
    cg2 = dim3((Vh + 255) / 256, nrhs);
    bg2 = dim3(MX_GRID, nrhs);
    // the whole iteration loop on the device (one graph launch) unless the hop kernels are being
    // timed one by one (event records cannot sit inside a conditional graph body) or graphs are off
    device_loop = allow_device_loop && sp->use_graphs != 0 && c->prof == 0;
    MxCtl* hc = m->ctl_h;
    memset(hc, 0, sizeof(MxCtl));
    hc->nrhs = nrhs;
    hc->maxIter = maxIter;
    hc->delta2 = delta * delta;
    hc->target2 = target * target;
    for (int i = 0; i < nrhs; i++) {
      const double mu = sp->mu ? sp->mu[i] : c->p.mu;
      hc->cv[i] = 2.0 * k * mu * ts;
      hc->sv[i] = 1.0 / (1.0 + (2.0 * k * mu) * (2.0 * k * mu));
    }
    CgScalars* sh = c->sc_h;
    memset(sh, 0, sizeof(CgScalars));
    for (int i = 0; i < nrhs; i++) sh->active[i] = 1;
    for (auto& e : m->ph)
      if (!e) QKX_CUDA(cudaEventCreate(&e));
    return QKX_OK;
  }

  // --- set-up, batched FP64: gather b, |b|^2; b^_e = b_e + k D_eo A^-1 b_o; g5 b^_e; r = Mh^+ b^_e
  int setup() {
    MxCtl* hc = m->ctl_h;
    QKX_CUDA(cudaMemcpyAsync(m->cvec, hc->cv, sizeof(double) * nrhs, cudaMemcpyHostToDevice, c->st));
    QKX_CUDA(cudaMemcpyAsync(m->svec, hc->sv, sizeof(double) * nrhs, cudaMemcpyHostToDevice, c->st));
    QKX_CUDA(cudaMemcpyAsync(c->sc, c->sc_h, sizeof(CgScalars), cudaMemcpyHostToDevice, c->st));
    if (device_loop) QKX_CUDA(cudaMemcpyAsync(m->ctl, hc, sizeof(MxCtl), cudaMemcpyHostToDevice, c->st));
    for (int i = 0; i < nrhs; i++) {
      QKX_CUDA(cudaMemcpyAsync(m->bE + i * n12, b[i], hb, cudaMemcpyDeviceToDevice, c->st));
      QKX_CUDA(cudaMemcpyAsync(m->bO + i * n12, b[i] + n12, hb, cudaMemcpyDeviceToDevice, c->st));
    }
    k_mx_norm<<<bg2, MX_NT, 0, c->st>>>(B64(m->bE, 0, Vh), m->part);
    counted(c);
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, MX_GRID, FIN_AUX, c->sc);
    counted(c);
    k_mx_norm<<<bg2, MX_NT, 0, c->st>>>(B64(m->bO, 0, Vh), m->part);
    counted(c);
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, MX_GRID, FIN_AUX_ADD, c->sc);
    counted(c);
    // t_o = A^-1 b_o
    k_mx_site<SITE_TWIST_INV><<<cg2, 256, 0, c->st>>>(B64(m->bO, 1, Vh), B64(m->t64, 1, Vh), 1, m->cvec, m->svec);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    // z = b_e + k D_eo t_o = b^_e, |b^|^2 -> aux2 ; g5bh = g5 b^_e
    int nb64 = 0;
    QKX_TRY(hop64_batch(c, EPI_XPAY, nrhs, B64(m->t64, 1, Vh), B64(m->z64, 0, Vh), B64(m->bE, 0, Vh), 0, k, 0.0,
                        m->cvec, nullptr, c->sc->active, m->part, &nb64));
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, nb64, FIN_AUX2, c->sc);
    counted(c);
    k_mx_site<SITE_GAMMA5><<<cg2, 256, 0, c->st>>>(B64(m->z64, 0, Vh), B64(m->g5bh, 0, Vh), 0, nullptr, nullptr);
    counted(c);
    // r = g5 Mh(-c) g5 b^_e = Mh^+ b^_e, |r|^2 -> r2 (FP32 when the sloppy residual is FP32)
    if constexpr (r32) {
      QKX_TRY(normal_residual_f32(c, nrhs, m->g5bh, FA::acc(m->rs, 0, Vh), &nb64));
    } else {
      QKX_TRY(schur64_g5_batch(c, nrhs, -1.0, m->g5bh, m->r64, m->part, &nb64));
    }
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, nb64, FIN_R2_INIT, c->sc);
    counted(c);
    QKX_CUDA(cudaMemsetAsync(m->x64, 0, hb * nrhs, c->st));
    QKX_CUDA(cudaMemsetAsync(m->xs.d, 0, FA::words * 16 * (size_t)Vh * nrhs, c->st));
    if constexpr (r32) {
      k_mx_convert<AC, SP><<<cg2, 256, 0, c->st>>>(FA::acc(m->rs, 0, Vh), FT::acc(m->p, 0, Vh), nullptr);
      counted(c);
    } else {
      k_mx_from_f64<AC, R><<<cg2, 256, 0, c->st>>>(B64(m->r64, 0, Vh), FA::acc(m->rs, 0, Vh), nullptr);
      counted(c);
      k_mx_from_f64<SP, R><<<cg2, 256, 0, c->st>>>(B64(m->r64, 0, Vh), FT::acc(m->p, 0, Vh), nullptr);
      counted(c);
    }
    QKX_CUDA(cudaGetLastError());
    return QKX_OK;
  }

  // reliable update of the active RHS: x64 += x_s (x_s = 0); the FP64 true residual
  // |rhat|^2 -> aux, after which the RHS that meet the tolerance stop; for the others the residual
  // the sloppy CG restarts from, Mh^+ rhat, with its norm -> aux2
  int reliable_update() {
    k_mx_fold<AC, R><<<cg2, 256, 0, c->st>>>(FA::acc(m->xs, 0, Vh), B64(m->x64, 0, Vh), c->sc->active);
    counted(c);
    int nb = 0;
    if constexpr (r32) {
      // the second FP64 hop of Mh x64 forms z = g5 b^ - g5 Mh x64 itself: |z|^2 from the FP64
      // values, z stored in FP32 for the FP32 Mh^+ that follows (straight into the sloppy residual)
      QKX_TRY(hop64_batch(c, EPI_TWIST_INV, nrhs, B64(m->x64, 0, Vh), B64(m->t64, 1, Vh), B64(m->x64, 0, Vh), 1, 0.0,
                          +1.0, m->cvec, m->svec, c->sc->active, nullptr, nullptr));
      int nbz = 0;
      QKX_TRY(hop64_batch_res(c, nrhs, B64(m->t64, 1, Vh), B64(m->x64, 0, Vh), B64(m->g5bh, 0, Vh),
                              scratch32(c, nrhs, 0), 0, -k * k, +1.0, m->cvec, c->sc->active, m->part, &nbz,
                              true));
      k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, nbz, FIN_AUX, c->sc);
      counted(c);
      k_mx_stop_converged<<<1, MAX_RHS, 0, c->st>>>(c->sc, nrhs);
      counted(c);
      QKX_TRY(normal_residual_from32(c, nrhs, FA::acc(m->rs, 0, Vh), &nb));
    } else {
      QKX_TRY(schur64_g5_batch(c, nrhs, +1.0, m->x64, m->z64, nullptr));
      k_mx_sub_norm<<<bg2, MX_NT, 0, c->st>>>(B64(m->g5bh, 0, Vh), B64(m->z64, 0, Vh), c->sc->active, m->part);
      counted(c);
      k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, MX_GRID, FIN_AUX, c->sc);
      counted(c);
      k_mx_stop_converged<<<1, MAX_RHS, 0, c->st>>>(c->sc, nrhs);
      counted(c);
      QKX_TRY(schur64_g5_batch(c, nrhs, -1.0, m->z64, m->r64, m->part, &nb));
    }
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, nb, FIN_AUX2, c->sc);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    return QKX_OK;
  }

  // after an update's decisions (active and restart flags set): the sloppy residual of the RHS
  // that go on, and p = r where the search direction restarts
  int restart_kernels(bool any_restart) {
    if constexpr (!r32) {
      k_mx_from_f64<AC, R><<<cg2, 256, 0, c->st>>>(B64(m->r64, 0, Vh), FA::acc(m->rs, 0, Vh), c->sc->active);
      counted(c);
    }
    if (any_restart) {
      k_mx_convert<AC, SP><<<cg2, 256, 0, c->st>>>(FA::acc(m->rs, 0, Vh), FT::acc(m->p, 0, Vh), c->sc->restart);
      counted(c);
    }
    QKX_CUDA(cudaGetLastError());
    return QKX_OK;
  }

  // --- the iteration loop as a graph: WHILE (any RHS active) { WHILE (no reliable update asked
  // for) { iteration }; reliable update; decisions }, added to `top`.  Every decision of the host
  // loop is taken by a one-block kernel from the same scalars; both loops are bounded by maxIter
  // because every pass of the outer one runs at least one inner iteration.  pre / post emit work
  // into the top level before and after the loop (the batch's set-up and final phase).
  template <class Pre, class Post>
  int loop_graph(cudaGraph_t top, long long* kt, long long* ko, long long* ki, Pre pre, Post post) {
    return build_loop_graph(c, top, kt, ko, ki,
                            [&](int part, cudaGraphConditionalHandle h_outer, cudaGraphConditionalHandle h_inner) -> int {
                              if (part == -1) return pre();
                              if (part == 4) return post();
                              if (part == 0) {  // per-RHS state from the set-up
                                k_ctl_start<<<1, MAX_RHS, 0, c->st>>>(c->sc, m->ctl, h_outer);
                                counted(c);
                                return cudaGetLastError() == cudaSuccess ? QKX_OK : QKX_ERR_CUDA;
                              }
                              if (part == 1) {  // outer body before the inner loop
                                k_ctl_inner_begin<<<1, 1, 0, c->st>>>(h_inner);
                                counted(c);
                                return cudaGetLastError() == cudaSuccess ? QKX_OK : QKX_ERR_CUDA;
                              }
                              if (part == 2) {  // outer body after the inner loop
                                QKX_TRY(reliable_update());
                                k_ctl_after_ru<<<1, MAX_RHS, 0, c->st>>>(c->sc, m->ctl, h_outer);
                                counted(c);
                                return restart_kernels(true);
                              }
                              // inner body: one iteration and the decision to go on
                              QKX_TRY(SL::iteration(c, nrhs, false, tile));
                              k_ctl_after_iter<<<1, MAX_RHS, 0, c->st>>>(c->sc, m->ctl, h_inner);
                              counted(c);
                              return cudaGetLastError() == cudaSuccess ? QKX_OK : QKX_ERR_CUDA;
                            });
  }

  // the loop graph of this context (cached while the batch size, kappa and tile stay), launched
  int device_loop_launch() {
    if (m->dgraph && (m->dgraph_R != nrhs || m->dgraph_kappa != c->p.kappa || m->dgraph_nr != tile.nr ||
                      m->dgraph_nt != tile.nt || m->dgraph_kind != tile.kind)) {
      QKX_CUDA(cudaStreamSynchronize(c->st));
      cudaGraphExecDestroy(m->dgraph);
      m->dgraph = nullptr;
    }
    if (!m->dgraph) {
      cudaGraph_t top = nullptr;
      QKX_CUDA(cudaGraphCreate(&top, 0));
      long long kt = 0, ko = 0, ki = 0;
      auto none = []() -> int { return QKX_OK; };
      int rc = loop_graph(top, &kt, &ko, &ki, none, none);
      if (rc == QKX_OK) {
        const cudaError_t e = cudaGraphInstantiate(&m->dgraph, top, 0);
        if (e != cudaSuccess) {
          set_error("instantiating the solver graph: %s", cudaGetErrorString(e));
          rc = QKX_ERR_CUDA;
          m->dgraph = nullptr;
        }
      }
      cudaGraphDestroy(top);
      if (rc != QKX_OK) return rc;
      m->dgraph_R = nrhs;
      m->dgraph_kappa = c->p.kappa;
      m->dgraph_nr = tile.nr;
      m->dgraph_nt = tile.nt;
      m->dgraph_kind = tile.kind;
      m->dgraph_k[0] = kt;
      m->dgraph_k[1] = ko;
      m->dgraph_k[2] = ki;
    }
    for (int i = 0; i < 3; i++) kcount[i] = m->dgraph_k[i];
    QKX_CUDA(cudaGraphLaunch(m->dgraph, c->st));
    return QKX_OK;
  }

  // --- host-driven loop: the host reads r^2 after every iteration and takes the decisions
  int host_loop() {
    CgScalars* sh = c->sc_h;
    const bool prof = c->prof != 0;
    const bool graphs = sp->use_graphs != 0;
    float ms_seg = 0;
    QKX_CUDA(cudaMemcpyAsync(sh, c->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->st));
    QKX_CUDA(cudaStreamSynchronize(c->st));
    bool ru_pending = false;  // a reliable update's end mark not yet read

    // r2rec: the sloppy r^2 when a reliable update was asked for; best: the smallest FP64
    // true residual ||rhat||^2 seen so far (||b^||^2 at x = 0)
    std::vector<double> r2ru(nrhs), ratio(nrhs, 1.0), r2rec(nrhs, 0.0), best(nrhs);
    for (int i = 0; i < nrhs; i++) {
      bnorm2[i] = sh->aux[i];
      best[i] = sh->aux2[i];
      r2ru[i] = sh->r2[i];
      ratio[i] = sh->r2[i] > 0 ? sh->aux2[i] / sh->r2[i] : 1.0;  // ||rhat||^2 / ||Mh^+ rhat||^2 at x = 0
      if (bnorm2[i] == 0.0 || sh->r2[i] == 0.0) active[i] = 0;
      sh->active[i] = active[i];
      sh->stop[i] = target * target * bnorm2[i];
    }
    QKX_CUDA(cudaMemcpyAsync(c->sc->active, sh->active, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, c->st));
    QKX_CUDA(cudaMemcpyAsync(c->sc->stop, sh->stop, sizeof(double) * MAX_RHS, cudaMemcpyHostToDevice, c->st));

    // --- graph of one inner iteration
    if (prof && m->gev.size() < 8) {
      for (int e = (int)m->gev.size(); e < 8; e++) {
        cudaEvent_t ev;
        QKX_CUDA(cudaEventCreate(&ev));
        m->gev.push_back(ev);
      }
    }
    if (m->graph && (m->graph_R != nrhs || m->graph_kappa != c->p.kappa || m->graph_nr != tile.nr ||
                     m->graph_nt != tile.nt || m->graph_kind != tile.kind || !graphs || prof)) {
      cudaGraphExecDestroy(m->graph);
      m->graph = nullptr;
    }
    if (graphs && !m->graph) {
      cudaGraph_t gr;
      QKX_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      c->capturing = 1;
      c->captured = 0;
      int rc = SL::iteration(c, nrhs, prof, tile);
      c->capturing = 0;
      m->graph_kernels = c->captured;
      cudaError_t e = cudaStreamEndCapture(c->st, &gr);
      if (rc != QKX_OK) return rc;
      if (e != cudaSuccess) {
        set_error("graph capture: %s", cudaGetErrorString(e));
        return QKX_ERR_CUDA;
      }
      QKX_CUDA(cudaGraphInstantiate(&m->graph, gr, 0));
      cudaGraphDestroy(gr);
      m->graph_R = nrhs;
      m->graph_kappa = c->p.kappa;
      m->graph_nr = tile.nr;
      m->graph_nt = tile.nt;
      m->graph_kind = tile.kind;
    }

    int since = 0;
    while (iter < maxIter) {
      int na = 0;
      for (int i = 0; i < nrhs; i++) na += active[i];
      if (!na) break;
      if (m->graph) {
        QKX_CUDA(cudaGraphLaunch(m->graph, c->st));
        counted(c, (int)m->graph_kernels);
      } else {
        QKX_TRY(SL::iteration(c, nrhs, prof, tile));
      }
      iter++;
      since++;
      QKX_CUDA(cudaMemcpyAsync(sh->r2, c->sc->r2, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, c->st));
      QKX_CUDA(cudaStreamSynchronize(c->st));
      if (ru_pending) {
        QKX_CUDA(cudaEventElapsedTime(&ms_seg, m->ph[1], m->ph[2]));
        ms_ru += ms_seg;
        ru_pending = false;
      }
      if (prof) {
        for (int h = 0; h < 4; h++) {
          float ms = 0;
          QKX_CUDA(cudaEventElapsedTime(&ms, m->gev[2 * h], m->gev[2 * h + 1]));
          c->prof_ms += ms;
          c->prof_launches++;
          c->prof_bytes += SL::hop_bytes_per_rhs(c, nrhs, tile) * na;
        }
      }
      // reliable update of every active RHS when one of them asks for it
      bool ru = since >= 200;
      for (int i = 0; i < nrhs; i++) {
        if (!active[i]) continue;
        const double r2s = sh->r2[i];
        if (!(r2s == r2s) || isinf(r2s)) {
          set_error("mixed CG: r2 of right-hand side %d became %g at iteration %d", i, r2s, iter);
          return QKX_ERR_NAN;
        }
        r2rec[i] = r2s;
        if (r2s < delta * delta * r2ru[i] || r2s * ratio[i] <= target * target * bnorm2[i]) ru = true;
      }
      if (!ru) continue;
      n_ru++;
      since = 0;
      QKX_CUDA(cudaEventRecord(m->ph[1], c->st));
      QKX_TRY(reliable_update());
      QKX_CUDA(cudaMemcpyAsync(sh->aux, c->sc->aux, 2 * sizeof(double) * MAX_RHS, cudaMemcpyDeviceToHost, c->st));
      QKX_CUDA(cudaStreamSynchronize(c->st));
      bool any_restart = false;
      for (int i = 0; i < nrhs; i++) {
        sh->restart[i] = 0;
        if (!active[i]) continue;
        const double rhat2 = sh->aux[i], r2 = sh->aux2[i];
        if (rhat2 <= target * target * bnorm2[i] || r2 == 0.0) {
          active[i] = 0;
          sh->active[i] = 0;
          continue;
        }
        if (!(rhat2 <= 1e6 * best[i])) {  // the true residual grew 1000x above its best: diverged
          active[i] = 0;
          sh->active[i] = 0;
          diverged++;
          continue;
        }
        best[i] = std::min(best[i], rhat2);
        ratio[i] = rhat2 / r2;
        r2ru[i] = r2;
        sh->r2[i] = r2;
        // The search direction was built from the sloppy residual.  When the residual that
        // replaces it is much larger, alpha = r^2 / <p, A p> of the next step would be too,
        // so the direction restarts from the new residual.
        if (r2 > 4.0 * r2rec[i]) {
          sh->restart[i] = 1;
          any_restart = true;
        }
      }
      // restart the sloppy residual from the new one for the RHS that go on
      QKX_CUDA(cudaMemcpyAsync(c->sc->active, sh->active, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, c->st));
      QKX_CUDA(cudaMemcpyAsync(c->sc->r2, sh->r2, sizeof(double) * MAX_RHS, cudaMemcpyHostToDevice, c->st));
      if (any_restart) {
        n_restart++;
        QKX_CUDA(cudaMemcpyAsync(c->sc->restart, sh->restart, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, c->st));
      }
      QKX_TRY(restart_kernels(any_restart));
      QKX_CUDA(cudaEventRecord(m->ph[2], c->st));
      ru_pending = true;
    }
    if (ru_pending) {
      QKX_CUDA(cudaEventSynchronize(m->ph[2]));
      QKX_CUDA(cudaEventElapsedTime(&ms_seg, m->ph[1], m->ph[2]));
      ms_ru += ms_seg;
    }
    for (int i = 0; i < nrhs; i++) nact += active[i];
    // every RHS takes part in the final phase
    for (int i = 0; i < nrhs; i++) sh->active[i] = 1;
    QKX_CUDA(cudaMemcpyAsync(c->sc->active, sh->active, sizeof(int) * MAX_RHS, cudaMemcpyHostToDevice, c->st));
    return QKX_OK;
  }

  // --- odd parity and the FP64 true residual of the full system, batched, for every RHS;
  // the solutions to x[] and the scalars to the host mirrors
  int final_phase() {
    if (device_loop) {
      k_ctl_final<<<1, MAX_RHS, 0, c->st>>>(c->sc, m->ctl);
      counted(c);
    }
    // fold what the unconverged RHS accumulated since their last update (x_s is zero for the others)
    if (device_loop || nact) {
      k_mx_fold<AC, R><<<cg2, 256, 0, c->st>>>(FA::acc(m->xs, 0, Vh), B64(m->x64, 0, Vh), c->sc->active);
      counted(c);
    }
    // x_o = A^-1 (b_o + k D_oe x_e) into t64; the same kernel sums the odd half of ||b - M x||^2,
    // |v - A_oo x_o|^2 with v = b_o + k D_oe x_e, from the D_oe x_e it has just computed
    int nbo = 0;
    QKX_TRY(hop64_batch(c, EPI_XPAY_TWINV_RES, nrhs, B64(m->x64, 0, Vh), B64(m->t64, 1, Vh), B64(m->bO, 1, Vh), 1, k,
                        1.0, m->cvec, m->svec, c->sc->active, m->part, &nbo));
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, nbo, FIN_AUX, c->sc);
    counted(c);
    // the even half, ||b_e - (A_ee x_e - k D_eo x_o)||^2 (x: even half in x64, odd half in t64),
    // summed in FP64 by the hop's epilogue; nothing is stored
    int nbe = 0;
    QKX_TRY(hop64_batch_res(c, nrhs, B64full(m->x64, m->t64, Vh), B64full(m->x64, m->t64, Vh),
                            B64full(m->bE, m->bO, Vh), SpinorF32{nullptr, nullptr, Vh}, 0, -k, 1.0, m->cvec,
                            c->sc->active, m->part, &nbe, false));
    k_mx_finalize<<<nrhs, 256, 0, c->st>>>(m->part, nbe, FIN_AUX_ADD, c->sc);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    for (int i = 0; i < nrhs; i++) {
      QKX_CUDA(cudaMemcpyAsync(x[i], m->x64 + i * n12, hb, cudaMemcpyDeviceToDevice, c->st));
      QKX_CUDA(cudaMemcpyAsync(x[i] + n12, m->t64 + i * n12, hb, cudaMemcpyDeviceToDevice, c->st));
    }
    QKX_CUDA(cudaMemcpyAsync(c->sc_h, c->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, c->st));
    if (device_loop) QKX_CUDA(cudaMemcpyAsync(m->ctl_h, m->ctl, sizeof(MxCtl), cudaMemcpyDeviceToHost, c->st));
    return QKX_OK;
  }

  // status and solve info once the final phase's copies are in host memory; rel (optional) gets
  // every RHS's true residual ||b - M x|| / ||b||.  Device times: the phase marks when given.
  int finish(qkx_solve_info* info, double* rel, const float* ms_total, const float* ms_setup, const float* ms_final) {
    CgScalars* sh = c->sc_h;
    if (device_loop) {
      MxCtl* hc = m->ctl_h;
      iter = hc->iter;
      n_ru = hc->n_ru;
      n_restart = hc->n_restart;
      diverged = hc->diverged;
      nact = hc->unconverged;
      ms_ru = float(hc->ru_ns * 1e-6);
      for (int i = 0; i < nrhs; i++) bnorm2[i] = hc->bnorm2[i];
      counted(c, (int)(kcount[0] + (long long)hc->n_outer * kcount[1] + (long long)hc->iter * kcount[2]));
      if (hc->nan_iter > 0) {
        set_error("mixed CG: r2 of right-hand side %d became non-finite at iteration %d", hc->nan_rhs, hc->nan_iter);
        return QKX_ERR_NAN;
      }
    }
    int rc = nact ? QKX_ERR_NOT_CONVERGED : QKX_OK;
    double worst = 0.0;
    int it = 0;
    for (int i = 0; i < nrhs; i++) {
      const double r = bnorm2[i] > 0 ? sqrt(sh->aux[i] / bnorm2[i]) : 0.0;
      if (rel) rel[i] = r;
      worst = std::max(worst, r);
      it = std::max(it, sh->iters[i]);
    }
    if (rc == QKX_OK && worst > sp->tol) rc = QKX_ERR_NOT_CONVERGED;
    if (info) {
      info->iterations = it;
      info->reliable_updates = n_ru;
      info->restarts = n_restart;
      info->converged = rc == QKX_OK;
      info->true_residual = worst;
      info->normal_residual = 0.0;
      info->seconds = ms_total ? *ms_total * 1e-3 : 0.0;
      info->seconds_setup = ms_setup ? *ms_setup * 1e-3 : 0.0;
      info->seconds_reliable = ms_ru * 1e-3;
      info->seconds_final = ms_final ? *ms_final * 1e-3 : 0.0;
    }
    if (rc == QKX_ERR_NOT_CONVERGED && diverged)
      set_error("mixed solve: %d right-hand side(s) diverged (FP64 true residual 1000x above its best) after %d "
                "iterations; a larger reliable_delta keeps the sloppy recursion closer to the true residual",
                diverged, iter);
    else if (rc == QKX_ERR_NOT_CONVERGED)
      set_error("mixed solve: true residual %g above tol %g after %d iterations", worst, sp->tol, iter);
    return rc;
  }
};

template <class P>
static int invert_eo_mixed_t(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b,
                             double2* const* x, qkx_solve_info* info) {
  MixedSolve<P> s(c, sp, nrhs, b, x);
  QKX_TRY(s.prepare(true));
  MixedState* m = c->mixed;
  QKX_CUDA(cudaEventRecord(c->t0, c->st));
  QKX_TRY(s.setup());
  QKX_CUDA(cudaEventRecord(m->ph[0], c->st));  // set-up done
  if (s.device_loop) {
    QKX_TRY(s.device_loop_launch());
  } else {
    QKX_TRY(s.host_loop());
  }
  QKX_CUDA(cudaEventRecord(m->ph[3], c->st));  // the final phase starts where the loop ended
  QKX_TRY(s.final_phase());
  QKX_CUDA(cudaEventRecord(c->t1, c->st));
  QKX_CUDA(cudaEventSynchronize(c->t1));
  float ms = 0, ms_setup = 0, ms_final = 0;
  cudaEventElapsedTime(&ms, c->t0, c->t1);
  cudaEventElapsedTime(&ms_setup, c->t0, m->ph[0]);
  cudaEventElapsedTime(&ms_final, m->ph[3], c->t1);
  return s.finish(info, nullptr, &ms, &ms_setup, &ms_final);
}

// ---------------------------------------------------------------- many lattices in one graph launch
// The jobs of qkx_invert_batch, grouped by context: the jobs of a context become one batch of
// right-hand sides (each with its own twisted mass), and every context's solve -- set-up,
// device-driven loop, final phase -- is one branch of a single CUDA graph.  One launch runs
// all lattices; their kernels share the SMs as the branches go, so the small lattices' blocks
// fill the gaps around the large one's.  Each branch ends with an event that dates it.
struct BatchGroup {
  qkx_ctx* c;
  std::vector<int> jobs;        // job indices, in order
  std::vector<int> first;       // first right-hand side of each job in the merged batch
  std::vector<const double2*> b;
  std::vector<double2*> x;
  std::vector<double> mu;
  qkx_solver_params p;
  cudaEvent_t done = nullptr;
};

static double steady_seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class P>
static int batch_graph_t(std::vector<BatchGroup>& groups, qkx_batch_job* jobs, const qkx_solver_params* sp,
                         double t0) {
  std::vector<std::unique_ptr<MixedSolve<P>>> solves;
  for (BatchGroup& g : groups) {
    solves.emplace_back(new MixedSolve<P>(g.c, &g.p, (int)g.b.size(), g.b.data(), g.x.data()));
    QKX_TRY(solves.back()->prepare(true));
    if (!solves.back()->device_loop) {
      set_error("internal: the batch graph needs the device-driven loop");
      return QKX_ERR_INVALID;
    }
  }
  cudaStream_t master = groups[0].c->st;
  cudaGraph_t top = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t start = nullptr;
  QKX_CUDA(cudaGraphCreate(&top, 0));
  // Each lattice's branch is captured on a stream of its own priority, the smallest lattice the
  // highest, and the graph runs its kernel nodes at those priorities: the branches still share the
  // SMs, but the small lattices' blocks go first, so their jobs finish early instead of all jobs
  // finishing together at the end of the largest one.
  int prio_least = 0, prio_greatest = 0;
  QKX_CUDA(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
  std::vector<cudaStream_t> pstreams(groups.size(), nullptr);
  int rc = QKX_OK;
  for (size_t j = 0; j < groups.size() && rc == QKX_OK; j++) {
    MixedSolve<P>& s = *solves[j];
    BatchGroup& g = groups[j];
    if (cudaEventCreate(&g.done) != cudaSuccess) {
      set_error("batch: cudaEventCreate failed");
      rc = QKX_ERR_CUDA;
      break;
    }
    const int prio = std::max(prio_greatest, prio_least - (int)j);  // groups come largest first
    if (cudaStreamCreateWithPriority(&pstreams[j], cudaStreamNonBlocking, prio) != cudaSuccess) {
      set_error("batch: cudaStreamCreateWithPriority failed");
      rc = QKX_ERR_CUDA;
      break;
    }
    cudaStream_t own = g.c->st;
    g.c->st = pstreams[j];  // the capture records the branch on the prioritised stream
    long long kt = 0, ko = 0, ki = 0;
    rc = s.loop_graph(
        top, &kt, &ko, &ki, [&]() { return s.setup(); },
        [&]() -> int {
          QKX_TRY(s.final_phase());
          QKX_CUDA(cudaEventRecordWithFlags(g.done, g.c->st, cudaEventRecordExternal));
          return QKX_OK;
        });
    g.c->st = own;
    s.kcount[0] = kt;
    s.kcount[1] = ko;
    s.kcount[2] = ki;
  }
  for (cudaStream_t ps : pstreams)
    if (ps) cudaStreamDestroy(ps);
  if (rc == QKX_OK && cudaGraphInstantiate(&exec, top, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) {
    set_error("batch: instantiating the graph failed: %s", cudaGetErrorString(cudaGetLastError()));
    rc = QKX_ERR_CUDA;
  }
  cudaGraphDestroy(top);
  // work queued earlier on any context's stream comes first
  for (size_t j = 1; j < groups.size() && rc == QKX_OK; j++) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess || cudaEventRecord(e, groups[j].c->st) != cudaSuccess ||
        cudaStreamWaitEvent(master, e, 0) != cudaSuccess) {
      set_error("batch: stream ordering failed");
      rc = QKX_ERR_CUDA;
    }
    cudaEventDestroy(e);
  }
  const double t_host = steady_seconds() - t0;  // set-up and capture before the launch
  if (rc == QKX_OK && (cudaEventCreate(&start) != cudaSuccess || cudaEventRecord(start, master) != cudaSuccess ||
                       cudaGraphLaunch(exec, master) != cudaSuccess || cudaStreamSynchronize(master) != cudaSuccess)) {
    set_error("batch: graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    rc = QKX_ERR_CUDA;
  }
  if (rc == QKX_OK) {
    for (size_t j = 0; j < groups.size(); j++) {
      BatchGroup& g = groups[j];
      MixedSolve<P>& s = *solves[j];
      float ms = 0;
      cudaEventElapsedTime(&ms, start, g.done);
      std::vector<double> rel(s.nrhs, 0.0);
      qkx_solve_info info{};
      int src = s.finish(&info, rel.data(), &ms, nullptr, nullptr);
      const int st = device_status(g.c);  // a bounded device wait that gave up voids the solution
      if (st != QKX_OK) src = st;
      const char* msg = src == QKX_OK ? "" : qkx_last_error();
      for (size_t q = 0; q < g.jobs.size(); q++) {
        qkx_batch_job& jb = jobs[g.jobs[q]];
        jb.info = info;
        double worst = 0.0;
        for (int r = g.first[q]; r < g.first[q] + jb.nrhs; r++) worst = std::max(worst, rel[r]);
        jb.info.true_residual = worst;
        jb.info.converged = src == QKX_OK || (src == QKX_ERR_NOT_CONVERGED && worst <= sp->tol) ? 1 : 0;
        jb.status = src == QKX_ERR_NOT_CONVERGED && worst <= sp->tol ? QKX_OK : src;
        jb.latency = t_host + ms * 1e-3;
        snprintf(jb.message, sizeof jb.message, "%s", jb.status == QKX_OK ? "" : msg);
      }
    }
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (start) cudaEventDestroy(start);
  for (BatchGroup& g : groups)
    if (g.done) {
      cudaEventDestroy(g.done);
      g.done = nullptr;
    }
  return rc;
}

// qkx_invert_batch for CG_EO_MIXED with graphs on: 0 = done (each job's status set), 1 = not
// applicable (the caller runs the jobs one context per thread), < 0 = error.  Latencies count
// from t0 (seconds of the steady clock).
int invert_batch_graph(qkx_batch_job* jobs, int njobs, const qkx_solver_params* sp, double t0) {
  if (sp->method != QKX_SOLVER_CG_EO_MIXED || sp->use_graphs == 0) return 1;
  std::vector<BatchGroup> groups;
  for (int i = 0; i < njobs; i++) {
    qkx_ctx* c = jobs[i].ctx;
    if (c->prof || (sp->sloppy_precision != QKX_PREC_DOUBLE && !c->compressible) || !c->have_gauge) return 1;
    auto it = std::find_if(groups.begin(), groups.end(), [&](const BatchGroup& g) { return g.c == c; });
    if (it == groups.end()) {
      groups.emplace_back();
      it = groups.end() - 1;
      it->c = c;
    }
    it->jobs.push_back(i);
    it->first.push_back((int)it->b.size());
    for (int r = 0; r < jobs[i].nrhs; r++) {
      it->b.push_back((const double2*)jobs[i].b_dev[r]);
      it->x.push_back((double2*)jobs[i].x_dev[r]);
      it->mu.push_back(jobs[i].mu ? jobs[i].mu[r] : c->p.mu);
    }
  }
  int dev0 = groups[0].c->device;
  for (BatchGroup& g : groups) {
    if ((int)g.b.size() > MAX_RHS || g.c->device != dev0) return 1;
    g.p = *sp;
    g.p.mu = g.mu.data();
  }
  // the largest lattice's branch first
  std::stable_sort(groups.begin(), groups.end(), [](const BatchGroup& a, const BatchGroup& b) { return a.c->V > b.c->V; });
  QKX_CUDA(cudaSetDevice(dev0));
  if (sp->sloppy_precision == QKX_PREC_HALF) return batch_graph_t<PHalf>(groups, jobs, sp, t0);
  if (sp->sloppy_precision == QKX_PREC_SINGLE) return batch_graph_t<PSingle>(groups, jobs, sp, t0);
  if (sp->sloppy_precision == QKX_PREC_DOUBLE) return batch_graph_t<PDouble>(groups, jobs, sp, t0);
  set_error("invalid argument: sloppy_precision");
  return QKX_ERR_INVALID;
}

// the captured graph holds gauge geometry: drop it when the gauge changes
// out_r = g5 Mh(-) g5 Mh(+) in_r on the even sites (Vector::tm_xxDagTm_xx(.., EE)),
// computed as one inner iteration of the mixed solver computes A p: the input
// rounded to the sloppy precision, then the four sloppy hops with the given tile.
template <class P>
static int sloppy_normal_t(qkx_ctx* c, int R_, HopTile tile, const double* const* in_host, double* const* out_host) {
  using SL = Sloppy<P>;
  using SP = typename P::SP;
  using GA = typename P::GA;
  using R = typename P::R;
  using FT = FieldTraits<SP>;
  QKX_TRY(mixed_alloc<P>(c, R_, true));
  MixedState* m = c->mixed;
  if (tile.nr == 0) QKX_TRY(tile_for<P>(c, R_, &tile));
  const int Vh = c->Vh;
  const size_t n12 = 12 * (size_t)Vh;
  const double k = c->p.kappa, cc = 2.0 * k * c->p.mu * c->p.twistSign;
  std::vector<double> cv(R_, cc), sv(R_, 1.0 / (1.0 + cc * cc));
  CgScalars* sh = c->sc_h;
  memset(sh, 0, sizeof(CgScalars));
  for (int i = 0; i < R_; i++) sh->active[i] = 1;
  QKX_CUDA(cudaMemcpyAsync(m->cvec, cv.data(), sizeof(double) * R_, cudaMemcpyHostToDevice, c->st));
  QKX_CUDA(cudaMemcpyAsync(m->svec, sv.data(), sizeof(double) * R_, cudaMemcpyHostToDevice, c->st));
  QKX_CUDA(cudaMemcpyAsync(c->sc, sh, sizeof(CgScalars), cudaMemcpyHostToDevice, c->st));
  double2* full = nullptr;
  QKX_CUDA(cudaMallocAsync(&full, sizeof(double2) * 2 * n12, c->st));
  int rc = QKX_OK;
  for (int i = 0; i < R_ && rc == QKX_OK; i++) {
    rc = upload_spinor(c, in_host[i], full);
    if (rc == QKX_OK && cudaMemcpyAsync(m->bE + i * n12, full, sizeof(double2) * n12, cudaMemcpyDeviceToDevice,
                                        c->st) != cudaSuccess)
      rc = QKX_ERR_CUDA;
  }
  const dim3 cg2((Vh + 255) / 256, R_);
  const double k2 = k * k;
  const GA U = SL::gauge(c);
  const Geom g = SL::geom(c);
  SP p = FT::acc(m->p, 0, Vh), t = FT::acc(m->t, 1, Vh), y = FT::acc(m->y, 0, Vh), Ap = FT::acc(m->Ap, 0, Vh);
  if (rc == QKX_OK) {
    k_mx_from_f64<SP, R><<<cg2, 256, 0, c->st>>>(B64(m->bE, 0, Vh), p, nullptr);
    counted(c);
    rc = hop_tile<SP, GA, R, EPI_TWIST_INV>(c, tile, R_, U, g, p, t, p, 1, 0.0, +1.0, true, nullptr, -1);
  }
  if (rc == QKX_OK) rc = hop_tile<SP, GA, R, EPI_XPAY_G5>(c, tile, R_, U, g, t, y, p, 0, -k2, +1.0, false, nullptr, -1);
  if (rc == QKX_OK) rc = hop_tile<SP, GA, R, EPI_TWIST_INV>(c, tile, R_, U, g, y, t, y, 1, 0.0, -1.0, true, nullptr, -1);
  if (rc == QKX_OK) rc = hop_tile<SP, GA, R, EPI_XPAY_G5>(c, tile, R_, U, g, t, Ap, y, 0, -k2, -1.0, false, nullptr, -1);
  if (rc == QKX_OK) {
    k_mx_to_f64<SP, R><<<cg2, 256, 0, c->st>>>(Ap, B64(m->z64, 0, Vh));
    counted(c);
    if (cudaGetLastError() != cudaSuccess) rc = QKX_ERR_CUDA;
  }
  for (int i = 0; i < R_ && rc == QKX_OK; i++) {
    if (cudaMemcpyAsync(full, m->z64 + i * n12, sizeof(double2) * n12, cudaMemcpyDeviceToDevice, c->st) !=
            cudaSuccess ||
        cudaMemsetAsync(full + n12, 0, sizeof(double2) * n12, c->st) != cudaSuccess)
      rc = QKX_ERR_CUDA;
    if (rc == QKX_OK) rc = download_spinor(c, full, out_host[i]);
    if (rc == QKX_OK && cudaStreamSynchronize(c->st) != cudaSuccess) rc = QKX_ERR_CUDA;
  }
  cudaFreeAsync(full, c->st);
  if (rc == QKX_ERR_CUDA) set_error("sloppy normal operator: %s", cudaGetErrorString(cudaGetLastError()));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return rc;
}

static bool known_tile(int precision, int nr, int nt, int kind) {
  for (const HopTile& t : kTiles)
    if (t.nr == nr && t.nt == nt && t.kind == kind && (kind == 0 || precision == QKX_PREC_HALF)) return true;
  set_error("invalid argument: tile (%d, %d, kind %d) is not one of the tuner's tiles for this precision", nr, nt,
            kind);
  return false;
}

int set_tile(qkx_ctx* c, int precision, int nrhs, int nr, int nt, int kind) {
  if (precision != QKX_PREC_HALF && precision != QKX_PREC_SINGLE && precision != QKX_PREC_DOUBLE) {
    set_error("invalid argument: precision");
    return QKX_ERR_INVALID;
  }
  if (!known_tile(precision, nr, nt, kind)) return QKX_ERR_INVALID;
  c->tuned[precision * 1000 + nrhs] = {nr, nt, kind};
  return QKX_OK;
}

int tune_table(qkx_ctx* c, int precision, int nrhs, int max, int* count, int* nr, int* nt, int* kind, double* ms) {
  auto it = c->tune_log.find(precision * 1000 + nrhs);
  const int n = it == c->tune_log.end() ? 0 : (int)it->second.size();
  if (count) *count = n;
  for (int i = 0; i < n && i < max; i++) {
    const auto& e = it->second[i];
    if (nr) nr[i] = (int)e[0];
    if (nt) nt[i] = (int)e[1];
    if (kind) kind[i] = (int)e[2];
    if (ms) ms[i] = e[3];
  }
  return QKX_OK;
}

int sloppy_normal(qkx_ctx* c, int precision, int nrhs, int nr, int nt, int kind, const double* const* in_host,
                  double* const* out_host) {
  HopTile tile;
  if (nr != 0 || nt != 0 || kind != 0) {
    if (!known_tile(precision, nr, nt, kind)) return QKX_ERR_INVALID;
    tile.nr = nr;
    tile.nt = nt;
    tile.kind = kind;
  }
  if (precision != QKX_PREC_DOUBLE && !c->compressible) {
    set_error("the sloppy operator needs SU(3) links (12-real reconstruction)");
    return QKX_ERR_UNSUPPORTED;
  }
  if (precision == QKX_PREC_HALF) return sloppy_normal_t<PHalf>(c, nrhs, tile, in_host, out_host);
  if (precision == QKX_PREC_SINGLE) return sloppy_normal_t<PSingle>(c, nrhs, tile, in_host, out_host);
  if (precision == QKX_PREC_DOUBLE) return sloppy_normal_t<PDouble>(c, nrhs, tile, in_host, out_host);
  set_error("invalid argument: precision");
  return QKX_ERR_INVALID;
}

void mixed_invalidate(qkx_ctx* c) {
  MixedState* m = c->mixed;
  if (m && (m->graph || m->dgraph)) {
    cudaStreamSynchronize(c->st);
    if (m->graph) cudaGraphExecDestroy(m->graph);
    if (m->dgraph) cudaGraphExecDestroy(m->dgraph);
    m->graph = nullptr;
    m->dgraph = nullptr;
  }
}

int tune(qkx_ctx* c, int precision, int nrhs, int* nr, int* nt, double* ms) {
  HopTile t;
  double best = 0;
  int rc;
  if (precision == QKX_PREC_HALF || precision == QKX_PREC_SINGLE) {
    if (!c->compressible) {
      set_error("tuning the sloppy hop needs SU(3) links (12-real reconstruction)");
      return QKX_ERR_UNSUPPORTED;
    }
  }
  if (precision == QKX_PREC_HALF) {
    QKX_TRY(mixed_alloc<PHalf>(c, nrhs, true));
    rc = tune_tile<PHalf>(c, nrhs, &t, &best);
  } else if (precision == QKX_PREC_SINGLE) {
    QKX_TRY(mixed_alloc<PSingle>(c, nrhs, true));
    rc = tune_tile<PSingle>(c, nrhs, &t, &best);
  } else if (precision == QKX_PREC_DOUBLE) {
    QKX_TRY(mixed_alloc<PDouble>(c, nrhs, true));
    rc = tune_tile<PDouble>(c, nrhs, &t, &best);
  } else {
    set_error("invalid argument: precision");
    return QKX_ERR_INVALID;
  }
  if (rc != QKX_OK) return rc;
  if (nr) *nr = t.nr;
  if (nt) *nt = t.nt;
  if (ms) *ms = best;
  return QKX_OK;
}

int invert_eo_mixed(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b, double2* const* x,
                    qkx_solve_info* info) {
  if (sp->sloppy_precision == QKX_PREC_DOUBLE) return invert_eo_mixed_t<PDouble>(c, sp, nrhs, b, x, info);
  if (!c->compressible) {
    set_error("mixed precision needs SU(3) links (12-real reconstruction); these links are not unitary "
              "to 1e-6 (max |UU^+-1| = %g)", c->link_unitarity);
    return QKX_ERR_UNSUPPORTED;
  }
  if (sp->sloppy_precision == QKX_PREC_SINGLE) return invert_eo_mixed_t<PSingle>(c, sp, nrhs, b, x, info);
  if (sp->sloppy_precision == QKX_PREC_HALF) return invert_eo_mixed_t<PHalf>(c, sp, nrhs, b, x, info);
  set_error("invalid argument: sloppy_precision");
  return QKX_ERR_INVALID;
}

}  // namespace qkx
