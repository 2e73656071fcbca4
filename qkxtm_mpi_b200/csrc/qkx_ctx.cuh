// qkx_ctx.cuh -- the context behind the C ABI (internal to libqkx_b200.so).
#pragma once
#include <stdarg.h>
#include <stdio.h>

#include <array>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "qkx_b200.h"
#include "blas.cuh"
#include "qkx_common.cuh"

namespace qkx {
void set_error(const char* fmt, ...);
struct MixedState;
}  // namespace qkx

#define QKX_CUDA(call)                                                                                \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess) {                                                                          \
      qkx::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);     \
      return QKX_ERR_CUDA;                                                                            \
    }                                                                                                 \
  } while (0)

#define QKX_TRY(expr)        \
  do {                       \
    int rc_ = (expr);        \
    if (rc_ != QKX_OK) return rc_; \
  } while (0)

struct qkx_tile_rec {
  int nr = 0, nt = 0, kind = 0;
};

struct qkx_ctx {
  qkx_params p;
  int device = 0;
  cudaStream_t st = nullptr;
  int Vh = 0;
  size_t V = 0;
  qkx::Geom geom{};      // links exactly as the operator uses them (bc_sign +1)
  qkx::Geom geom_raw{};  // compressed SU(3) links, boundary sign applied in the kernels
  int have_gauge = 0;
  int compressible = 0;
  int raw_sign = 1;
  double link_unitarity = 0;  // max |U U^+ - 1|
  double2* U18 = nullptr;     // [2][4][9][Vh] FP64, as the operator uses them
  float4* U12f = nullptr;     // [2][4][3][Vh] FP32 12-real, SU(3)
  uint4* U12ha = nullptr;     // [2][4][Vh]  FP16 12-real complex 0..3
  uint2* U12hb = nullptr;     // [2][4][Vh]  FP16 12-real complex 4..5
  float4* U18fa = nullptr;    // [2][4][4][Vh] FP32 18-real complex 0..7 (boundary sign included)
  float2* U18fb = nullptr;    // [2][4][Vh]  FP32 18-real complex 8
  uint4* U18ha = nullptr;     // [2][4][Vh]  FP16 18-real complex 0..3 (boundary sign included)
  uint4* U18hb = nullptr;     // [2][4][Vh]  FP16 18-real complex 4..7
  uint32_t* U18hc = nullptr;  // [2][4][Vh]  FP16 18-real complex 8
  double2* Usm = nullptr;     // [2][4][9][Vh] FP64 links of the Gaussian smearing (APE-smeared)
  int have_smear = 0;
  double2* stage = nullptr;   // one host-layout spinor (V*12 double2)
  static constexpr int NW = 8;
  double2* w[NW] = {};        // FP64 full-lattice work fields
  double* part = nullptr;     // reduction partials
  int npart = 0;
  qkx::CgScalars* sc = nullptr;    // device solver scalars
  qkx::CgScalars* sc_h = nullptr;  // pinned host mirror
  double* dscal = nullptr;         // device scratch scalars [64]
  double* hscal = nullptr;         // pinned host scalars [64]
  int* dstat = nullptr;            // device status word: non-zero after a bounded device wait gave up
  int* hstat = nullptr;            // pinned host copy
  int smem_optin = 0;              // shared memory a block may opt in to on this device
  int c3t = 0;                     // the TMA-tiled FP64 hop where the lattice allows it (opt-in)
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  // profiling of the hopping kernels
  int prof = 0;
  std::vector<cudaEvent_t> ev_a, ev_b;
  std::vector<double> ev_bytes;
  size_t ev_used = 0;
  long long prof_launches = 0;
  double prof_ms = 0, prof_bytes = 0;
  qkx::MixedState* mixed = nullptr;
  // kernel launches issued by this context (graph launches count their kernel nodes)
  long long kernels = 0;
  int capturing = 0;          // set while a CUDA graph is being captured
  long long captured = 0;     // kernels recorded into the graph being captured
  // tuned tiles: (precision*1000 + nrhs) -> (RHS per thread, threads per block, kernel kind)
  std::map<int, qkx_tile_rec> tuned;
  // every tile timed by the last tuning of a key: (nr, nt, kind, ms per hop)
  std::map<int, std::vector<std::array<double, 4>>> tune_log;
};

namespace qkx {

// count one kernel launch (during graph capture it is counted once per replay instead)
inline void counted(qkx_ctx* c, int n = 1) {
  if (c->capturing) c->captured += n;
  else c->kernels += n;
}

inline SpinorF64 F64(const double2* base, int Vh) {
  double2* b = const_cast<double2*>(base);
  return SpinorF64{b, b ? b + (size_t)12 * Vh : nullptr, Vh};
}

// profiling brackets around one hopping-kernel launch
int prof_begin(qkx_ctx* c);
int prof_end(qkx_ctx* c, double bytes);
int prof_collect(qkx_ctx* c);

// grid for the grid-stride BLAS kernels
inline int blas_grid(size_t n) {
  size_t b = (n + BLAS_NT - 1) / BLAS_NT;
  return (int)(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

// Re<x,y> over n double2, finalized into the solver scalars / dst (see FIN_*)
int redot(qkx_ctx* c, const double2* x, const double2* y, size_t n, int mode, double* dst, int rhs);
int finalize(qkx_ctx* c, int nparts, int mode, double* dst, int rhs);

// FP64 operator on full even-odd fields (out != in)
int run_op(qkx_ctx* c, int op, const double2* in, double2* out);
// M (tm) or M^+ on full FP64 fields with the 18-real links, fused twist
int apply_tm(qkx_ctx* c, const double2* in, double2* out, bool dagger);
int apply_tm_mu(qkx_ctx* c, const double2* in, double2* out, bool dagger, double mu);
// FP64 hopping kernel on accessors (one parity or both), see hop.cuh for the epilogues
int hop64a(qkx_ctx* c, int basis, bool dag, int epi, SpinorF64 in, SpinorF64 out, SpinorF64 x, bool x_distinct,
           int out_parity, double a, double cc, double s, double* norm_part);
// batched FP64 hop (UKQCD, D): nrhs fields [rhs][12][Vh] per parity; *nblk = norm partials per RHS
int hop64_batch(qkx_ctx* c, int epi, int nrhs, SpinorF64 in, SpinorF64 out, SpinorF64 x, int out_parity, double a,
                double csign, const double* cvec, const double* svec, const int* active, double* norm_part,
                int* nblk);
// batched FP64 hop with a residual epilogue: res32(rhs) = w - g5 (a D in + x + i c g5 x) (g5, EPI_XPAY_G5_RES)
// or w - (a D in + x + i c g5 x) (EPI_XPAY_RES) in FP32 on out_parity (-1: both; a null res32 stores
// nothing), |res|^2 partials (FP64) per RHS into norm_part (*nblk of them)
int hop64_batch_res(qkx_ctx* c, int nrhs, SpinorF64 in, SpinorF64 x, SpinorF64 w, SpinorF32 res32, int out_parity,
                    double a, double csign, const double* cvec, const int* active, double* norm_part, int* nblk,
                    bool g5);
// site-local operator (site_ops.cuh) on parities [par_first, par_first + npar)
int site_op_acc(qkx_ctx* c, int basis, int op, SpinorF64 in, SpinorF64 out, int par_first, int npar, double cc,
                double s);
// FP64 accessor for a single-parity field [12][Vh]
inline SpinorF64 H64(const double2* base, int parity, int Vh) {
  double2* b = const_cast<double2*>(base);
  return parity ? SpinorF64{nullptr, b, Vh} : SpinorF64{b, nullptr, Vh};
}

// mixed-precision solver entry (mixed.cu)
int invert_eo_mixed(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b,
                    double2* const* x, qkx_solve_info* info);
void mixed_free(qkx_ctx* c);
// qkx_invert_batch as one graph launch for all lattices (CG_EO_MIXED, graphs on): 0 done,
// 1 not applicable, < 0 error; t0 is the batch's start on the steady clock, in seconds
int invert_batch_graph(qkx_batch_job* jobs, int njobs, const qkx_solver_params* sp, double t0);
// the learned solver: batched even-odd flexible CG preconditioned by the network (ptc.cu)
int invert_gcr_ptc(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b, double2* const* x,
                   qkx_solve_info* info);
void mixed_invalidate(qkx_ctx* c);
int tune(qkx_ctx* c, int precision, int nrhs, int* nr, int* nt, double* ms);
int set_tile(qkx_ctx* c, int precision, int nrhs, int nr, int nt, int kind);
int tune_table(qkx_ctx* c, int precision, int nrhs, int max, int* count, int* nr, int* nt, int* kind, double* ms);
int sloppy_normal(qkx_ctx* c, int precision, int nrhs, int nr, int nt, int kind, const double* const* in_host,
                  double* const* out_host);

// the device status word: QKX_ERR_CUDA (and the word cleared) if a kernel's bounded wait gave
// up since the last check; synchronizes the context's stream
int device_status(qkx_ctx* c);

// lazy buffers and context-level helpers (api.cu)
int ensure_stage(qkx_ctx* c);
int ensure_links(qkx_ctx* c);
int ensure_work(qkx_ctx* c);
// after U18 changed: link checks, 12-real compression, solver caches invalidated
int gauge_finish(qkx_ctx* c);
// host Vector::M layout <-> device even-odd FP64 field, through the staging buffer
int upload_spinor(qkx_ctx* c, const double* host, double2* dev);
int download_spinor(qkx_ctx* c, const double2* dev, double* host);

}  // namespace qkx
