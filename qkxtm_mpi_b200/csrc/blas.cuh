// blas.cuh -- qkxTM BLAS on device fields (reference lib/blas_qkxTM.cpp:4-56,
// Vector::norm2 lib/lattice_util.cpp:464-477), plus the fused CG updates.
//
// Reductions are deterministic: a fixed grid writes one partial per block and
// a one-block finalize sums the partials in a fixed order, so repeated runs
// give bit-identical scalars.  Scalars that drive the solvers (alpha, beta,
// r2) live in device memory so an iteration needs no host round trip.
#pragma once
#include "qkx_common.cuh"

namespace qkx {

constexpr int BLAS_NT = 256;

// Solver scalars for up to QKX_MAX_RHS right-hand sides.
constexpr int MAX_RHS = 64;
struct CgScalars {
  double r2[MAX_RHS];
  double r2_old[MAX_RHS];
  double pAp[MAX_RHS];
  double alpha[MAX_RHS];
  double beta[MAX_RHS];
  double stop[MAX_RHS];   // FP64 true residual^2 at which the RHS has converged ((0.9 tol)^2 |b|^2)
  int active[MAX_RHS];   // 1 while the RHS still iterates
  int iters[MAX_RHS];
  double aux[MAX_RHS];   // per-RHS results of the batched FP64 residual steps
  double aux2[MAX_RHS];
  int restart[MAX_RHS];  // 1: restart the search direction from the residual (p = r)
};

template <int NT>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[NT / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double w = 0.0;
  if (threadIdx.x < 32) {
    w = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
  }
  __syncthreads();
  return w;  // valid in thread 0
}

// Re <x, y> over n complex numbers (partials per block)
static __global__ void __launch_bounds__(BLAS_NT) k_redot(const double2* __restrict__ x, const double2* __restrict__ y,
                                                   size_t n, double* __restrict__ part) {
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLAS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * BLAS_NT) {
    double2 a = x[i], b = y[i];
    acc += a.x * b.x + a.y * b.y;
  }
  double s = block_sum<BLAS_NT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// finalize modes
enum { FIN_STORE = 0, FIN_PAP = 1, FIN_R2 = 2, FIN_R2_INIT = 3 };

// Sum part[0..n) in a fixed order and act on the solver scalars of one RHS:
//   FIN_STORE    *dst = sum
//   FIN_PAP      pAp = sum, alpha = r2 / pAp
//   FIN_R2       r2_old = r2, r2 = sum, beta = r2 / r2_old
//   FIN_R2_INIT  r2 = sum
static __global__ void __launch_bounds__(1024) k_finalize(const double* __restrict__ part, int n, double* dst,
                                                   int mode, CgScalars* sc, int rhs) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += 1024) acc += part[i];
  double s = block_sum<1024>(acc);
  if (threadIdx.x == 0) {
    if (mode == FIN_STORE) {
      *dst = s;
    } else if (mode == FIN_PAP) {
      sc->pAp[rhs] = s;
      sc->alpha[rhs] = sc->r2[rhs] / s;
    } else if (mode == FIN_R2) {
      sc->r2_old[rhs] = sc->r2[rhs];
      sc->r2[rhs] = s;
      sc->beta[rhs] = s / sc->r2_old[rhs];
    } else {
      sc->r2[rhs] = s;
    }
    if (dst && mode != FIN_STORE) *dst = s;
  }
}

// y = y + a x with a = sign * (*a_dev)       (X_eq_X_p_aY, lib/blas_qkxTM.cpp:31)
static __global__ void __launch_bounds__(BLAS_NT) k_axpy(const double* __restrict__ a_dev, double sign,
                                                  const double2* __restrict__ x, double2* __restrict__ y,
                                                  size_t n) {
  const double a = sign * *a_dev;
  for (size_t i = (size_t)blockIdx.x * BLAS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * BLAS_NT) {
    double2 xv = x[i], yv = y[i];
    y[i] = make_double2(yv.x + a * xv.x, yv.y + a * xv.y);
  }
}

// y = a y + x with a = *a_dev                (X_eq_aX_p_Y, lib/blas_qkxTM.cpp:45)
static __global__ void __launch_bounds__(BLAS_NT) k_xpay(const double2* __restrict__ x, const double* __restrict__ a_dev,
                                                  double2* __restrict__ y, size_t n) {
  const double a = *a_dev;
  for (size_t i = (size_t)blockIdx.x * BLAS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * BLAS_NT) {
    double2 xv = x[i], yv = y[i];
    y[i] = make_double2(a * yv.x + xv.x, a * yv.y + xv.y);
  }
}

// y = y + a x with a host scalar
static __global__ void __launch_bounds__(BLAS_NT) k_axpy_h(double a, const double2* __restrict__ x,
                                                    double2* __restrict__ y, size_t n) {
  for (size_t i = (size_t)blockIdx.x * BLAS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * BLAS_NT) {
    double2 xv = x[i], yv = y[i];
    y[i] = make_double2(yv.x + a * xv.x, yv.y + a * xv.y);
  }
}

// y = a y + x with a host scalar
static __global__ void __launch_bounds__(BLAS_NT) k_xpay_h(const double2* __restrict__ x, double a,
                                                    double2* __restrict__ y, size_t n) {
  for (size_t i = (size_t)blockIdx.x * BLAS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * BLAS_NT) {
    double2 xv = x[i], yv = y[i];
    y[i] = make_double2(a * yv.x + xv.x, a * yv.y + xv.y);
  }
}

// z = x - y, with partial sums of |z|^2 (true-residual helper)
static __global__ void __launch_bounds__(BLAS_NT) k_sub_norm(const double2* __restrict__ x, const double2* __restrict__ y,
                                                      double2* __restrict__ z, size_t n, double* __restrict__ part) {
  double acc = 0.0;
  for (size_t i = (size_t)blockIdx.x * BLAS_NT + threadIdx.x; i < n; i += (size_t)gridDim.x * BLAS_NT) {
    double2 a = x[i], b = y[i];
    double2 d = make_double2(a.x - b.x, a.y - b.y);
    z[i] = d;
    acc += d.x * d.x + d.y * d.y;
  }
  double s = block_sum<BLAS_NT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

}  // namespace qkx
