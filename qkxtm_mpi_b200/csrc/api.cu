// api.cu -- C ABI of libqkx_b200.so: context, gauge upload and compression,
// the FP64 operators of the reference's qkxTM::Vector, the qkxTM BLAS and
// the reference's CG (lib/solvers.cpp:16-81) on one B200.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "blas.cuh"
#include "hop.cuh"
#include "hop_c3.cuh"
#include "hop_c3t.cuh"
#include "layout.cuh"
#include "qkx_ctx.cuh"
#include "site_ops.cuh"

using namespace qkx;

namespace qkx {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

static int invalid(const char* what) {
  set_error("invalid argument: %s", what);
  return QKX_ERR_INVALID;
}

// ---------------------------------------------------------------- profiling
int prof_begin(qkx_ctx* c) {
  if (!c->prof) return QKX_OK;
  if (c->ev_used == c->ev_a.size()) {
    cudaEvent_t a, b;
    QKX_CUDA(cudaEventCreate(&a));
    QKX_CUDA(cudaEventCreate(&b));
    c->ev_a.push_back(a);
    c->ev_b.push_back(b);
    c->ev_bytes.push_back(0);
  }
  QKX_CUDA(cudaEventRecord(c->ev_a[c->ev_used], c->st));
  return QKX_OK;
}

int prof_end(qkx_ctx* c, double bytes) {
  if (!c->prof) return QKX_OK;
  QKX_CUDA(cudaEventRecord(c->ev_b[c->ev_used], c->st));
  c->ev_bytes[c->ev_used] = bytes;
  c->ev_used++;
  if (c->ev_used >= 4096) return prof_collect(c);
  return QKX_OK;
}

int prof_collect(qkx_ctx* c) {
  if (c->ev_used == 0) return QKX_OK;
  QKX_CUDA(cudaStreamSynchronize(c->st));
  for (size_t i = 0; i < c->ev_used; i++) {
    float ms = 0;
    QKX_CUDA(cudaEventElapsedTime(&ms, c->ev_a[i], c->ev_b[i]));
    c->prof_ms += ms;
    c->prof_bytes += c->ev_bytes[i];
    c->prof_launches++;
  }
  c->ev_used = 0;
  return QKX_OK;
}

// ---------------------------------------------------------------- lazy buffers
// The host-layout staging buffer and the FP64 work fields are allocated when a
// call first needs them, so a context that only tunes or runs the batched
// solver on device fields does not hold them.
int ensure_stage(qkx_ctx* c) {
  if (c->stage) return QKX_OK;
  cudaError_t e = cudaMalloc(&c->stage, sizeof(double2) * 12 * c->V);
  if (e != cudaSuccess) {
    set_error("staging buffer: %s", cudaGetErrorString(e));
    return QKX_ERR_NOMEM;
  }
  return QKX_OK;
}

int ensure_links(qkx_ctx* c) {
  if (c->U18) return QKX_OK;
  cudaError_t e = cudaMalloc(&c->U18, sizeof(double2) * 36 * c->V);
  if (e != cudaSuccess) {
    set_error("gauge field: %s", cudaGetErrorString(e));
    return QKX_ERR_NOMEM;
  }
  return QKX_OK;
}

int ensure_work(qkx_ctx* c) {
  for (int i = 0; i < qkx_ctx::NW; i++) {
    if (c->w[i]) continue;
    cudaError_t e = cudaMalloc(&c->w[i], sizeof(double2) * 12 * c->V);
    if (e != cudaSuccess) {
      set_error("work field: %s", cudaGetErrorString(e));
      return QKX_ERR_NOMEM;
    }
  }
  return QKX_OK;
}

// ---------------------------------------------------------------- reductions
int finalize(qkx_ctx* c, int nparts, int mode, double* dst, int rhs) {
  k_finalize<<<1, 1024, 0, c->st>>>(c->part, nparts, dst, mode, c->sc, rhs);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

int redot(qkx_ctx* c, const double2* x, const double2* y, size_t n, int mode, double* dst, int rhs) {
  int g = blas_grid(n);
  k_redot<<<g, BLAS_NT, 0, c->st>>>(x, y, n, c->part);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return finalize(c, g, mode, dst, rhs);
}

// ---------------------------------------------------------------- hopping term, FP64 18-real
// Algorithmic bytes of one launch: per output site the input spinor once, the
// output once, the links touching the site (8 for one parity, 4 per site when
// both parities are covered since the halves share them) and, for an xpay
// epilogue on a field other than the hop input, that field once.
static double hop_bytes(size_t nout, double S, double G, bool both, bool extra_x) {
  return (double)nout * (2 * S + (both ? 4 : 8) * G + (extra_x ? S : 0));
}

// FP64 sites per block of the colour-split kernel (x 3 colour threads)
constexpr int C3_NS = 64;

// cuTensorMapEncodeTiled of the driver, looked up once (the library links the runtime only)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  });
  return fn;
}

// A 2D TMA map over `rows` rows of Vh double2 (row stride Vh x 16 bytes) with boxes of `sites`
// sites x `comps` rows, as FP64 elements (two per site and row).
static bool map2d(CUtensorMap* m, const void* base, int Vh, int rows, int sites, int comps) {
  const EncodeTiledFn f = encode_tiled();
  if (!f || !base || ((uintptr_t)base & 15u)) return false;
  const cuuint64_t dim[2] = {(cuuint64_t)2 * Vh, (cuuint64_t)rows};
  const cuuint64_t stride[1] = {(cuuint64_t)Vh * 16};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * sites), (cuuint32_t)comps};
  const cuuint32_t es[2] = {1, 1};
  return f(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dim, stride, box, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the TMA-tiled kernel for this launch, when the lattice and the fields allow it (else false)
template <int B, bool DAG, int EPI>
static bool launch_hop64_tiled(qkx_ctx* c, HopArgs<SpinorF64, GaugeF64x18>& A, const HopRes& Rz) {
  const Geom& g = A.g;
  if (!c->c3t || !c3t_supported(g, c->smem_optin)) return false;
  if (A.nrhs > 1 && A.in.rs != (size_t)12 * g.Vh) return false;  // the batch must be [rhs][12][Vh]
  const int W = g.L[0] / 2, Vh = g.Vh, rows = 12 * A.nrhs;
  C3tMaps M;
  memset(&M, 0, sizeof M);
  for (int par = 0; par < 2; par++) {
    const double2* base = par ? A.in.p1 : A.in.p0;
    if (!base) continue;  // this input parity is not read by the launch
    if (!map2d(&M.in4[par], base, Vh, rows, C3T_ROWS * W, 12) || !map2d(&M.in1[par], base, Vh, rows, W, 12))
      return false;
  }
  const bool need0 = A.out_parity != 0, need1 = A.out_parity != 1;  // input parities: the other one
  if ((need0 && !A.in.p0) || (need1 && !A.in.p1)) return false;
  if (!map2d(&M.l4, A.gauge.p, Vh, 72, C3T_ROWS * W, 9) || !map2d(&M.l1, A.gauge.p, Vh, 72, W, 9) ||
      !map2d(&M.l3, A.gauge.p, Vh, 72, (C3T_ROWS - 1) * W, 9))
    return false;
  // opt in once per device, to all the shared memory a block may have, so that concurrent
  // contexts of different lattice sizes never lower one another's limit
  const int smem = C3tLayout(W).bytes + 128;
  static std::atomic<uint64_t> opted{0};
  const uint64_t bit = 1ull << (c->device & 63);
  if (!(opted.load() & bit)) {
    if (cudaFuncSetAttribute(hop_c3t_kernel<B, DAG, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             c->smem_optin) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    opted.fetch_or(bit);
  }
  A.nblk = c3t_blocks(g, A.out_parity);
  hop_c3t_kernel<B, DAG, EPI><<<A.nblk, dim3(C3T_ROWS * W, 3), smem, c->st>>>(A, Rz, M, W, c->dstat);
  counted(c);
  return true;
}

// one FP64 18-real hop launch over A.nrhs right-hand sides (Rz: operands of EPI_XPAY_G5_RES)
template <int B, bool DAG, int EPI>
static int launch_hop64(qkx_ctx* c, HopArgs<SpinorF64, GaugeF64x18>& A, const HopRes& Rz = HopRes{}) {
  if (launch_hop64_tiled<B, DAG, EPI>(c, A, Rz)) return QKX_OK;
  A.nblk = c3_blocks_per_rhs<C3_NS>(c->Vh, A.out_parity);
  hop_c3_kernel<C3_NS, SpinorF64, B, DAG, EPI><<<A.nblk * A.nrhs, dim3(C3_NS, 3), 0, c->st>>>(A, Rz);
  counted(c);
  return QKX_OK;
}

int device_status(qkx_ctx* c) {
  QKX_CUDA(cudaMemcpyAsync(c->hstat, c->dstat, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  if (*c->hstat == 0) return QKX_OK;
  const int code = *c->hstat;
  *c->hstat = 0;
  QKX_CUDA(cudaMemsetAsync(c->dstat, 0, sizeof(int), c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  set_error("a kernel's bounded wait for its shared-memory staging gave up (code %d): the results of the calls "
            "since the last check are not valid",
            code);
  return QKX_ERR_CUDA;
}

template <int B, bool DAG, int EPI>
static int hop64_t(qkx_ctx* c, SpinorF64 in, SpinorF64 out, SpinorF64 x, bool x_distinct, int out_parity,
                   double a, double cc, double s, double* norm_part) {
  HopArgs<SpinorF64, GaugeF64x18> A;
  A.out = out;
  A.in = in;
  A.x = x;
  A.gauge = GaugeF64x18{c->U18, c->Vh};
  A.g = c->geom;
  A.out_parity = out_parity;
  A.a = a;
  A.c = cc;
  A.s = s;
  A.norm_part = norm_part;
  A.nrhs = 1;
  A.cvec = nullptr;
  A.svec = nullptr;
  A.active = nullptr;
  const int n = out_parity < 0 ? 2 * c->Vh : c->Vh;
  QKX_TRY(prof_begin(c));
  QKX_TRY((launch_hop64<B, DAG, EPI>(c, A)));
  QKX_CUDA(cudaGetLastError());
  bool extra = (EPI == EPI_XPAY || EPI == EPI_XPAY_G5 || EPI == EPI_XPAY_TWINV) && x_distinct;
  return prof_end(c, hop_bytes(n, 192.0, 144.0, out_parity < 0, extra));
}

// Batched FP64 hop (UKQCD basis, D not D^+) over nrhs right-hand sides stored
// [rhs][12][Vh] per parity, per-RHS twist factors and mask; returns the
// number of norm partials per RHS in *nblk.
template <int EPI>
static int hop64_batch_t(qkx_ctx* c, int nrhs, SpinorF64 in, SpinorF64 out, SpinorF64 x, int out_parity, double a,
                         double csign, const double* cvec, const double* svec, const int* active, double* norm_part,
                         int* nblk) {
  HopArgs<SpinorF64, GaugeF64x18> A;
  A.out = out;
  A.in = in;
  A.x = x;
  A.gauge = GaugeF64x18{c->U18, c->Vh};
  A.g = c->geom;
  A.out_parity = out_parity;
  A.a = a;
  A.c = csign;
  A.s = 1.0;
  A.norm_part = norm_part;
  A.nrhs = nrhs;
  A.cvec = cvec;
  A.svec = svec;
  A.active = active;
  QKX_TRY((launch_hop64<0, false, EPI>(c, A)));
  QKX_CUDA(cudaGetLastError());
  if (nblk) *nblk = A.nblk;
  return QKX_OK;
}

int hop64_batch_res(qkx_ctx* c, int nrhs, SpinorF64 in, SpinorF64 x, SpinorF64 w, SpinorF32 res32, int out_parity,
                    double a, double csign, const double* cvec, const int* active, double* norm_part, int* nblk,
                    bool g5) {
  HopArgs<SpinorF64, GaugeF64x18> A;
  A.out = SpinorF64{nullptr, nullptr, c->Vh};
  A.in = in;
  A.x = x;
  A.gauge = GaugeF64x18{c->U18, c->Vh};
  A.g = c->geom;
  A.out_parity = out_parity;
  A.a = a;
  A.c = csign;
  A.s = 1.0;
  A.norm_part = norm_part;
  A.nrhs = nrhs;
  A.cvec = cvec;
  A.svec = nullptr;
  A.active = active;
  if (g5) QKX_TRY((launch_hop64<0, false, EPI_XPAY_G5_RES>(c, A, HopRes{w, res32})));
  else QKX_TRY((launch_hop64<0, false, EPI_XPAY_RES>(c, A, HopRes{w, res32})));
  QKX_CUDA(cudaGetLastError());
  if (nblk) *nblk = A.nblk;
  return QKX_OK;
}

int hop64_batch(qkx_ctx* c, int epi, int nrhs, SpinorF64 in, SpinorF64 out, SpinorF64 x, int out_parity, double a,
                double csign, const double* cvec, const double* svec, const int* active, double* norm_part,
                int* nblk) {
  switch (epi) {
    case EPI_PLAIN:
      return hop64_batch_t<EPI_PLAIN>(c, nrhs, in, out, x, out_parity, a, csign, cvec, svec, active, norm_part, nblk);
    case EPI_XPAY:
      return hop64_batch_t<EPI_XPAY>(c, nrhs, in, out, x, out_parity, a, csign, cvec, svec, active, norm_part, nblk);
    case EPI_XPAY_G5:
      return hop64_batch_t<EPI_XPAY_G5>(c, nrhs, in, out, x, out_parity, a, csign, cvec, svec, active, norm_part,
                                        nblk);
    case EPI_TWIST_INV:
      return hop64_batch_t<EPI_TWIST_INV>(c, nrhs, in, out, x, out_parity, a, csign, cvec, svec, active, norm_part,
                                          nblk);
    case EPI_XPAY_TWINV:
      return hop64_batch_t<EPI_XPAY_TWINV>(c, nrhs, in, out, x, out_parity, a, csign, cvec, svec, active,
                                           norm_part, nblk);
    case EPI_XPAY_TWINV_RES:
      return hop64_batch_t<EPI_XPAY_TWINV_RES>(c, nrhs, in, out, x, out_parity, a, csign, cvec, svec, active,
                                               norm_part, nblk);
  }
  return invalid("epilogue");
}

// runtime -> compile-time dispatch, on accessors (single-parity fields allowed)
int hop64a(qkx_ctx* c, int basis, bool dag, int epi, SpinorF64 in, SpinorF64 out, SpinorF64 x, bool x_distinct,
           int out_parity, double a, double cc, double s, double* norm_part) {
#define QKX_HOP_CASE(B_, D_, E_) \
  if (basis == B_ && dag == D_ && epi == E_)   \
    return hop64_t<B_, D_, E_>(c, in, out, x, x_distinct, out_parity, a, cc, s, norm_part);
#define QKX_HOP_EPIS(B_, D_) \
  QKX_HOP_CASE(B_, D_, EPI_PLAIN) QKX_HOP_CASE(B_, D_, EPI_XPAY) QKX_HOP_CASE(B_, D_, EPI_XPAY_G5) \
  QKX_HOP_CASE(B_, D_, EPI_TWIST_INV) QKX_HOP_CASE(B_, D_, EPI_XPAY_TWINV)
  QKX_HOP_EPIS(0, false)
  QKX_HOP_EPIS(0, true)
  QKX_HOP_EPIS(1, false)
  QKX_HOP_EPIS(1, true)
#undef QKX_HOP_EPIS
#undef QKX_HOP_CASE
  return invalid("hop variant");
}

// the same on full (both-parity) fields
static int hop64(qkx_ctx* c, int basis, bool dag, int epi, const double2* in, double2* out, const double2* x,
                 int out_parity, double a, double cc, double s, double* norm_part = nullptr) {
  return hop64a(c, basis, dag, epi, F64(in, c->Vh), F64(out, c->Vh), F64(x ? x : in, c->Vh), x && x != in,
                out_parity, a, cc, s, norm_part);
}

int site_op_acc(qkx_ctx* c, int basis, int op, SpinorF64 in, SpinorF64 out, int par_first, int npar, double cc,
                double s) {
  const int n = npar * c->Vh;
  const int nb = (n + 255) / 256;
  if (basis == 0)
    {
      k_site_op<0><<<nb, 256, 0, c->st>>>(in, out, par_first, npar, op, cc, s);
      counted(c);
    }
  else
    {
      k_site_op<1><<<nb, 256, 0, c->st>>>(in, out, par_first, npar, op, cc, s);
      counted(c);
    }
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

static int site_op(qkx_ctx* c, int basis, int op, const double2* in, double2* out, double cc, double s) {
  return site_op_acc(c, basis, op, F64(in, c->Vh), F64(out, c->Vh), 0, 2, cc, s);
}

static int zero_parity(qkx_ctx* c, double2* f, int parity) {
  QKX_CUDA(cudaMemsetAsync(f + (size_t)parity * 12 * c->Vh, 0, sizeof(double2) * 12 * c->Vh, c->st));
  return QKX_OK;
}

int apply_tm_mu(qkx_ctx* c, const double2* in, double2* out, bool dagger, double mu) {
  const double tw = 2.0 * c->p.kappa * mu * c->p.twistSign;
  return hop64(c, 0, dagger, EPI_XPAY, in, out, in, -1, -c->p.kappa, dagger ? -tw : tw, 1.0);
}

int apply_tm(qkx_ctx* c, const double2* in, double2* out, bool dagger) {
  return apply_tm_mu(c, in, out, dagger, c->p.mu);
}

// M_xx psi for output parity `par` (0 = EE, 1 = OO) with twist sign `sgn`:
//   t = A^-1 D_{1-par <- par} psi ;  out_par = A psi - kappa^2 D_{par <- 1-par} t
// (Vector::tm_xx, lib/lattice_util.cpp:2001-2022).  With g5out the result is
// multiplied by gamma5, which is how tm_xxDagTm_xx chains two of them.
static int tm_xx(qkx_ctx* c, int basis, int par, double sgn, const double2* in, double2* out, double2* tmp,
                 bool g5out) {
  const double k = c->p.kappa, mu = c->p.mu;
  const double cc = 2.0 * k * mu * sgn;
  const double inv = 1.0 / (1.0 + (2.0 * k * mu) * (2.0 * k * mu));
  QKX_TRY(hop64(c, basis, false, EPI_TWIST_INV, in, tmp, nullptr, 1 - par, 0.0, cc, inv));
  return hop64(c, basis, false, g5out ? EPI_XPAY_G5 : EPI_XPAY, tmp, out, in, par, -k * k, cc, 1.0);
}

int run_op(qkx_ctx* c, int op, const double2* in, double2* out) {
  QKX_TRY(ensure_work(c));
  if (!c->have_gauge && op != QKX_OP_GAMMA5 && op != QKX_OP_GAMMA5_CHIRAL && op != QKX_OP_TWIST &&
      op != QKX_OP_TWIST_INV && op != QKX_OP_TWIST_DAG && op != QKX_OP_TWIST_DAG_INV &&
      op != QKX_OP_TWIST_INV_CHIRAL && op != QKX_OP_ROTATE_CHIRAL_TO_UKQCD) {
    set_error("operator %d needs a gauge field: call qkx_load_gauge first", op);
    return QKX_ERR_NOGAUGE;
  }
  const double k = c->p.kappa, mu = c->p.mu, s = c->p.twistSign;
  const double tw = 2.0 * k * mu * s;
  const double inv = 1.0 / (1.0 + (2.0 * k * mu) * (2.0 * k * mu));
  double2* t1 = c->w[6];
  double2* t2 = c->w[7];
  if (in == t1 || in == t2 || out == t1 || out == t2) return invalid("operator fields alias the work fields");
  switch (op) {
    case QKX_OP_DSLASH: return hop64(c, 0, false, EPI_PLAIN, in, out, nullptr, -1, 0, 0, 1);
    case QKX_OP_DSLASH_DAG: return hop64(c, 0, true, EPI_PLAIN, in, out, nullptr, -1, 0, 0, 1);
    case QKX_OP_DSLASH_CHIRAL: return hop64(c, 1, false, EPI_PLAIN, in, out, nullptr, -1, 0, 0, 1);
    case QKX_OP_TM: return hop64(c, 0, false, EPI_XPAY, in, out, in, -1, -k, tw, 1);
    case QKX_OP_TM_DAG: return hop64(c, 0, true, EPI_XPAY, in, out, in, -1, -k, -tw, 1);
    case QKX_OP_TM_CHIRAL: return hop64(c, 1, false, EPI_XPAY, in, out, in, -1, -k, tw, 1);
    case QKX_OP_TM_DAG_CHIRAL: return hop64(c, 1, true, EPI_XPAY, in, out, in, -1, -k, -tw, 1);
    case QKX_OP_WILSON: return hop64(c, 0, false, EPI_XPAY, in, out, in, -1, -k, 0.0, 1);
    case QKX_OP_TM_DAGTM:
      QKX_TRY(hop64(c, 0, false, EPI_XPAY, in, t1, in, -1, -k, tw, 1));
      return hop64(c, 0, true, EPI_XPAY, t1, out, t1, -1, -k, -tw, 1);
    case QKX_OP_TM_DAGTM_CHIRAL:
      QKX_TRY(hop64(c, 1, false, EPI_XPAY, in, t1, in, -1, -k, tw, 1));
      return hop64(c, 1, true, EPI_XPAY, t1, out, t1, -1, -k, -tw, 1);
    case QKX_OP_DSLASH_XX_EO:
    case QKX_OP_DSLASH_XX_OE:
    case QKX_OP_DSLASH_XX_CHIRAL_EO:
    case QKX_OP_DSLASH_XX_CHIRAL_OE: {
      int basis = (op == QKX_OP_DSLASH_XX_CHIRAL_EO || op == QKX_OP_DSLASH_XX_CHIRAL_OE) ? 1 : 0;
      int par = (op == QKX_OP_DSLASH_XX_EO || op == QKX_OP_DSLASH_XX_CHIRAL_EO) ? 0 : 1;
      QKX_TRY(hop64(c, basis, false, EPI_PLAIN, in, out, nullptr, par, 0, 0, 1));
      return zero_parity(c, out, 1 - par);
    }
    case QKX_OP_TM_XX_EE:
    case QKX_OP_TM_XX_OO:
    case QKX_OP_TM_XX_CHIRAL_EE:
    case QKX_OP_TM_XX_CHIRAL_OO: {
      int basis = (op == QKX_OP_TM_XX_CHIRAL_EE || op == QKX_OP_TM_XX_CHIRAL_OO) ? 1 : 0;
      int par = (op == QKX_OP_TM_XX_EE || op == QKX_OP_TM_XX_CHIRAL_EE) ? 0 : 1;
      QKX_TRY(tm_xx(c, basis, par, s, in, out, t1, false));
      return zero_parity(c, out, 1 - par);
    }
    case QKX_OP_TM_XX_DAGTM_XX_EE:
    case QKX_OP_TM_XX_DAGTM_XX_OO:
    case QKX_OP_TM_XX_DAGTM_XX_CHIRAL_EE:
    case QKX_OP_TM_XX_DAGTM_XX_CHIRAL_OO: {
      // g5 M_xx(-s) g5 M_xx(s) psi  (Vector::tm_xxDagTm_xx, lib/lattice_util.cpp:2024-2035)
      int basis = (op == QKX_OP_TM_XX_DAGTM_XX_CHIRAL_EE || op == QKX_OP_TM_XX_DAGTM_XX_CHIRAL_OO) ? 1 : 0;
      int par = (op == QKX_OP_TM_XX_DAGTM_XX_EE || op == QKX_OP_TM_XX_DAGTM_XX_CHIRAL_EE) ? 0 : 1;
      QKX_TRY(tm_xx(c, basis, par, s, in, t2, t1, true));
      QKX_TRY(tm_xx(c, basis, par, -s, t2, out, t1, true));
      return zero_parity(c, out, 1 - par);
    }
    case QKX_OP_GAMMA5: return site_op(c, 0, SITE_GAMMA5, in, out, 0, 1);
    case QKX_OP_GAMMA5_CHIRAL: return site_op(c, 1, SITE_GAMMA5, in, out, 0, 1);
    case QKX_OP_TWIST: return site_op(c, 0, SITE_TWIST, in, out, tw, 1);
    case QKX_OP_TWIST_DAG: return site_op(c, 0, SITE_TWIST, in, out, -tw, 1);
    case QKX_OP_TWIST_INV: return site_op(c, 0, SITE_TWIST_INV, in, out, tw, inv);
    case QKX_OP_TWIST_DAG_INV: return site_op(c, 0, SITE_TWIST_INV, in, out, -tw, inv);
    case QKX_OP_TWIST_INV_CHIRAL: return site_op(c, 1, SITE_TWIST_INV, in, out, tw, inv);
    case QKX_OP_ROTATE_CHIRAL_TO_UKQCD: return site_op(c, 0, SITE_ROTATE_CH2UK, in, out, 0, 1);
    default: return invalid("operator id");
  }
}

int upload_spinor(qkx_ctx* c, const double* host, double2* dev) {
  QKX_TRY(ensure_stage(c));
  QKX_CUDA(cudaMemcpyAsync(c->stage, host, sizeof(double2) * 12 * c->V, cudaMemcpyHostToDevice, c->st));
  k_spinor_aos_to_eo<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(c->stage, dev, c->geom);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

int download_spinor(qkx_ctx* c, const double2* dev, double* host) {
  QKX_TRY(ensure_stage(c));
  k_spinor_eo_to_aos<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(dev, c->stage, c->geom);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaMemcpyAsync(host, c->stage, sizeof(double2) * 12 * c->V, cudaMemcpyDeviceToHost, c->st));
  return QKX_OK;
}

// ---------------------------------------------------------------- gauge
// Check the links the operator uses and, if they are SU(3) up to one global
// sign on the last time slice's t-links, build the sloppy copies: 12-real
// FP32 and FP16 with that sign stripped (the kernels then apply it from the
// coordinate), and 18-real FP32 and FP16 with the sign kept (for the FP16 hop
// variants that skip the third-row rebuild).
int gauge_finish(qkx_ctx* c) {
  const int nl = 8 * c->Vh;
  const int nb = (nl + 255) / 256;
  double* part = nullptr;
  QKX_CUDA(cudaMallocAsync(&part, sizeof(double) * 4 * nb, c->st));
  k_gauge_check<<<nb, 256, 0, c->st>>>(c->U18, c->geom, part);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  std::vector<double> h((size_t)4 * nb);
  QKX_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * 4 * nb, cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaFreeAsync(part, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  double m[4] = {0, 0, 0, 0};
  for (int b = 0; b < nb; b++)
    for (int q = 0; q < 4; q++) m[q] = std::max(m[q], h[(size_t)b * 4 + q]);
  c->link_unitarity = m[0];
  const double thr = 1e-6;
  c->compressible = 0;
  if (m[0] < thr && m[1] < thr && (m[2] < thr || m[3] < thr)) {
    c->compressible = 1;
    c->raw_sign = (m[2] < thr) ? 1 : -1;
  }
  c->geom_raw = c->geom;
  c->geom_raw.bc_sign = c->raw_sign;
  if (c->compressible) {
    if (!c->U12f) {
      QKX_CUDA(cudaMalloc(&c->U12f, sizeof(float4) * 8 * 3 * (size_t)c->Vh));
      QKX_CUDA(cudaMalloc(&c->U12ha, sizeof(uint4) * 8 * (size_t)c->Vh));
      QKX_CUDA(cudaMalloc(&c->U12hb, sizeof(uint2) * 8 * (size_t)c->Vh));
    }
    k_gauge_compress<<<nb, 256, 0, c->st>>>(c->U18, c->geom, c->raw_sign, nullptr, c->U12f, c->U12ha, c->U12hb);
    counted(c);
    if (!c->U18fa) {
      QKX_CUDA(cudaMalloc(&c->U18fa, sizeof(float4) * 8 * 4 * (size_t)c->Vh));
      QKX_CUDA(cudaMalloc(&c->U18fb, sizeof(float2) * 8 * (size_t)c->Vh));
    }
    k_gauge_f32x18<<<nb, 256, 0, c->st>>>(c->U18, c->Vh, c->U18fa, c->U18fb);
    counted(c);
    if (!c->U18ha) {
      QKX_CUDA(cudaMalloc(&c->U18ha, sizeof(uint4) * 8 * (size_t)c->Vh));
      QKX_CUDA(cudaMalloc(&c->U18hb, sizeof(uint4) * 8 * (size_t)c->Vh));
      QKX_CUDA(cudaMalloc(&c->U18hc, sizeof(uint32_t) * 8 * (size_t)c->Vh));
    }
    k_gauge_f16x18<<<nb, 256, 0, c->st>>>(c->U18, c->Vh, c->U18ha, c->U18hb, c->U18hc);
    counted(c);
    QKX_CUDA(cudaGetLastError());
  }
  c->have_gauge = 1;
  mixed_invalidate(c);
  return QKX_OK;
}

}  // namespace qkx

// =================================================================== C ABI
extern "C" {

const char* qkx_version(void) { return "qkx_b200 0.1 (sm_100a)"; }
const char* qkx_last_error(void) { return qkx::g_err.c_str(); }

static int check_params(const qkx_params* p) {
  if (!p) return invalid("params is NULL");
  for (int i = 0; i < 4; i++)
    if (p->L[i] < 2) return invalid("lattice extents must be >= 2");
  if (p->L[0] % 2) return invalid("L[0] must be even for the even-odd layout");
  long long V = (long long)p->L[0] * p->L[1] * p->L[2] * p->L[3];
  if (V > (1LL << 28)) return invalid("lattice volume above 2^28 sites (32-bit site-word indexing)");
  if (p->twistSign != 1 && p->twistSign != -1) return invalid("twistSign must be +1 or -1");
  if (p->boundaryT != 1 && p->boundaryT != -1) return invalid("boundaryT must be +1 or -1");
  if (!(p->kappa == p->kappa) || !(p->mu == p->mu)) return invalid("kappa/mu is NaN");
  return QKX_OK;
}

int qkx_create(const qkx_params* p, int device, qkx_ctx** out) {
  if (!out) return invalid("out is NULL");
  *out = nullptr;
  QKX_TRY(check_params(p));
  int ndev = 0;
  QKX_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return invalid("device index");
  QKX_CUDA(cudaSetDevice(device));
  qkx_ctx* c = new qkx_ctx();
  c->p = *p;
  c->device = device;
  c->V = (size_t)p->L[0] * p->L[1] * p->L[2] * p->L[3];
  c->Vh = (int)(c->V / 2);
  for (int i = 0; i < 4; i++) c->geom.L[i] = p->L[i];
  c->geom.Vh = c->Vh;
  c->geom.bc_sign = 1;
  c->geom_raw = c->geom;
  int rc = QKX_OK;
  auto fail = [&](cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    rc = (e == cudaErrorMemoryAllocation) ? QKX_ERR_NOMEM : QKX_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) != cudaSuccess) fail(e, "stream");
  // The host-buffer entry points stage their device copies through the
  // stream-ordered allocator; keep freed blocks in this process's pool instead
  // of returning them to the driver at every synchronisation, so repeated
  // calls do not pay for fresh allocations.
  if (rc == QKX_OK) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  const size_t fbytes = sizeof(double2) * 12 * c->V;
  (void)fbytes;  // the staging buffer and the FP64 work fields are allocated on first use
  // room for any hop block size >= 32 and for the FP64 hop's row tiles
  c->npart = std::max(std::max(148 * 8, 2 * (int)((c->Vh + 31) / 32)), c3t_blocks(c->geom, -1)) + 1;
  if (rc == QKX_OK && (e = cudaMalloc(&c->part, sizeof(double) * c->npart)) != cudaSuccess) fail(e, "partials");
  if (rc == QKX_OK && (e = cudaMalloc(&c->sc, sizeof(CgScalars))) != cudaSuccess) fail(e, "scalars");
  if (rc == QKX_OK && (e = cudaHostAlloc(&c->sc_h, sizeof(CgScalars), cudaHostAllocDefault)) != cudaSuccess)
    fail(e, "pinned scalars");
  if (rc == QKX_OK && (e = cudaMalloc(&c->dscal, sizeof(double) * 64)) != cudaSuccess) fail(e, "scalars");
  if (rc == QKX_OK && (e = cudaHostAlloc(&c->hscal, sizeof(double) * 64, cudaHostAllocDefault)) != cudaSuccess)
    fail(e, "pinned scalars");
  if (rc == QKX_OK && (e = cudaMalloc(&c->dstat, sizeof(int))) != cudaSuccess) fail(e, "status word");
  if (rc == QKX_OK && (e = cudaMemset(c->dstat, 0, sizeof(int))) != cudaSuccess) fail(e, "status word");
  if (rc == QKX_OK && (e = cudaHostAlloc(&c->hstat, sizeof(int), cudaHostAllocDefault)) != cudaSuccess)
    fail(e, "pinned status word");
  if (rc == QKX_OK &&
      (e = cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device)) != cudaSuccess)
    fail(e, "device attribute");
  {
    // QKX_FP64_TILED=1 puts the FP64 hop on the TMA row tiles (hop_c3t.cuh) where the lattice
    // allows them; the direct kernel is the default, as it is the faster of the two on B200
    const char* v = getenv("QKX_FP64_TILED");
    c->c3t = (v && v[0] == '1') ? 1 : 0;
  }
  if (rc == QKX_OK && (e = cudaEventCreate(&c->t0)) != cudaSuccess) fail(e, "event");
  if (rc == QKX_OK && (e = cudaEventCreate(&c->t1)) != cudaSuccess) fail(e, "event");
  if (rc != QKX_OK) {
    std::string msg = qkx::g_err;
    qkx_destroy(c);
    qkx::g_err = msg;
    return rc;
  }
  *out = c;
  return QKX_OK;
}

void qkx_destroy(qkx_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  mixed_free(c);
  cudaFree(c->U18);
  cudaFree(c->U12f);
  cudaFree(c->U12ha);
  cudaFree(c->U12hb);
  cudaFree(c->U18fa);
  cudaFree(c->U18fb);
  cudaFree(c->U18ha);
  cudaFree(c->U18hb);
  cudaFree(c->U18hc);
  cudaFree(c->Usm);
  cudaFree(c->stage);
  cudaFree(c->dstat);
  if (c->hstat) cudaFreeHost(c->hstat);
  for (int i = 0; i < qkx_ctx::NW; i++) cudaFree(c->w[i]);
  cudaFree(c->part);
  cudaFree(c->sc);
  cudaFree(c->dscal);
  if (c->sc_h) cudaFreeHost(c->sc_h);
  if (c->hscal) cudaFreeHost(c->hscal);
  for (auto ev : c->ev_a) cudaEventDestroy(ev);
  for (auto ev : c->ev_b) cudaEventDestroy(ev);
  if (c->t0) cudaEventDestroy(c->t0);
  if (c->t1) cudaEventDestroy(c->t1);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

int qkx_set_params(qkx_ctx* c, const qkx_params* p) {
  if (!c) return invalid("ctx is NULL");
  QKX_TRY(check_params(p));
  for (int i = 0; i < 4; i++)
    if (p->L[i] != c->p.L[i]) return invalid("L differs from the context's lattice");
  c->p = *p;
  return QKX_OK;
}

int qkx_get_params(const qkx_ctx* c, qkx_params* p) {
  if (!c || !p) return invalid("NULL argument");
  *p = c->p;
  return QKX_OK;
}

int qkx_sync(qkx_ctx* c) {
  if (!c) return invalid("ctx is NULL");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

void* qkx_stream(qkx_ctx* c) { return c ? (void*)c->st : nullptr; }
size_t qkx_spinor_bytes(const qkx_ctx* c) { return c ? sizeof(double2) * 12 * c->V : 0; }
size_t qkx_volume(const qkx_ctx* c) { return c ? c->V : 0; }

int qkx_load_gauge(qkx_ctx* c, const double* U_host, int bc_mode) {
  if (!c || !U_host) return invalid("NULL argument");
  if (bc_mode != QKX_LINKS_AS_GIVEN && bc_mode != QKX_LINKS_APPLY_BC) return invalid("bc_mode");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_links(c));
  double2* tmp = nullptr;
  const size_t bytes = sizeof(double2) * 36 * c->V;
  QKX_CUDA(cudaMallocAsync(&tmp, bytes, c->st));
  QKX_CUDA(cudaMemcpyAsync(tmp, U_host, bytes, cudaMemcpyHostToDevice, c->st));
  int tsign = (bc_mode == QKX_LINKS_APPLY_BC && c->p.boundaryT == -1) ? -1 : 1;
  k_gauge_aos_to_eo<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(tmp, c->U18, c->geom, tsign);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaFreeAsync(tmp, c->st));
  return gauge_finish(c);
}

int qkx_gauge_generate(qkx_ctx* c, double eps, unsigned long long seed, int bc_mode) {
  if (!c) return invalid("ctx is NULL");
  if (bc_mode != QKX_LINKS_AS_GIVEN && bc_mode != QKX_LINKS_APPLY_BC) return invalid("bc_mode");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_links(c));
  const int nl = 8 * c->Vh;
  k_gauge_generate<<<(nl + 127) / 128, 128, 0, c->st>>>(c->U18, c->geom, eps, seed);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  if (bc_mode == QKX_LINKS_APPLY_BC && c->p.boundaryT == -1) {
    // multiply the last slice's t-links by -1 in place (the aos->eo kernel
    // reads and writes different buffers, so go through the stream allocator)
    double2* tmp = nullptr;
    const size_t bytes = sizeof(double2) * 36 * c->V;
    QKX_CUDA(cudaMallocAsync(&tmp, bytes, c->st));
    k_gauge_eo_to_aos<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(c->U18, tmp, c->geom);
    counted(c);
    k_gauge_aos_to_eo<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(tmp, c->U18, c->geom, -1);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    QKX_CUDA(cudaFreeAsync(tmp, c->st));
  }
  return gauge_finish(c);
}

int qkx_download_gauge(qkx_ctx* c, double* U_host) {
  if (!c || !U_host) return invalid("NULL argument");
  if (!c->have_gauge) {
    set_error("no gauge field loaded");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  double2* tmp = nullptr;
  const size_t bytes = sizeof(double2) * 36 * c->V;
  QKX_CUDA(cudaMallocAsync(&tmp, bytes, c->st));
  k_gauge_eo_to_aos<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(c->U18, tmp, c->geom);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaMemcpyAsync(U_host, tmp, bytes, cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaFreeAsync(tmp, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

int qkx_gauge_compressible(const qkx_ctx* c) {
  if (!c) return invalid("ctx is NULL");
  return c->compressible;
}

// ---------------------------------------------------------------- operators
int qkx_apply_dev(qkx_ctx* c, int op, const double* in_dev, double* out_dev) {
  if (!c || !in_dev || !out_dev) return invalid("NULL argument");
  if (in_dev == out_dev) return invalid("in and out must differ for qkx_apply_dev");
  QKX_CUDA(cudaSetDevice(c->device));
  return run_op(c, op, (const double2*)in_dev, (double2*)out_dev);
}

int qkx_apply(qkx_ctx* c, int op, const double* in_host, double* out_host) {
  if (!c || !in_host || !out_host) return invalid("NULL argument");
  if (op < 0 || op >= QKX_OP_COUNT) return invalid("operator id");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_work(c));
  QKX_TRY(upload_spinor(c, in_host, c->w[0]));
  QKX_TRY(run_op(c, op, c->w[0], c->w[1]));
  QKX_TRY(download_spinor(c, c->w[1], out_host));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return device_status(c);
}

int qkx_spinor_upload(qkx_ctx* c, const double* host, double* dev) {
  if (!c || !host || !dev) return invalid("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  return upload_spinor(c, host, (double2*)dev);
}

int qkx_spinor_download(qkx_ctx* c, const double* dev, double* host) {
  if (!c || !host || !dev) return invalid("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(download_spinor(c, (const double2*)dev, host));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

// ---------------------------------------------------------------- BLAS
int qkx_reCdotXdagY(qkx_ctx* c, const double* x, const double* y, double* result) {
  if (!c || !x || !y || !result) return invalid("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(redot(c, (const double2*)x, (const double2*)y, 12 * c->V, FIN_STORE, c->dscal, 0));
  QKX_CUDA(cudaMemcpyAsync(c->hscal, c->dscal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  *result = c->hscal[0];
  return QKX_OK;
}

int qkx_norm2(qkx_ctx* c, const double* x, double* result) { return qkx_reCdotXdagY(c, x, x, result); }

int qkx_X_eq_X_p_aY(qkx_ctx* c, double* x, double a, const double* y) {
  if (!c || !x || !y) return invalid("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  size_t n = 12 * c->V;
  k_axpy_h<<<blas_grid(n), BLAS_NT, 0, c->st>>>(a, (const double2*)y, (double2*)x, n);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

int qkx_X_eq_aX_p_Y(qkx_ctx* c, double* x, double a, const double* y) {
  if (!c || !x || !y) return invalid("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  size_t n = 12 * c->V;
  k_xpay_h<<<blas_grid(n), BLAS_NT, 0, c->st>>>((const double2*)y, a, (double2*)x, n);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// ---------------------------------------------------------------- CG (lib/solvers.cpp:16-81)
// One run of the reference's CG recurrence on device fields, continuing from
// the state in (r, p, sc->r2[0]) until r2 <= stop or *k reaches maxIter.
static int cg_fp64_loop(qkx_ctx* c, double2* x, double2* r, double2* p, double2* Ap, double2* tmp, double stop,
                        int maxIter, int* k, double* r2_host) {
  const size_t n = 12 * c->V;
  const int g = blas_grid(n);
  double r2 = *r2_host;
  while (r2 > stop && *k < maxIter) {
    QKX_TRY(apply_tm(c, p, tmp, false));                     // Ap.tmDagtm(p, tmp, ...)
    QKX_TRY(apply_tm(c, tmp, Ap, true));
    QKX_TRY(redot(c, p, Ap, n, FIN_PAP, nullptr, 0));         // pAp, alpha = r2 / pAp
    k_axpy<<<g, BLAS_NT, 0, c->st>>>(c->sc->alpha, 1.0, p, x, n);
    counted(c);    // x = x + alpha p
    k_axpy<<<g, BLAS_NT, 0, c->st>>>(c->sc->alpha, -1.0, Ap, r, n);
    counted(c);  // r = r - alpha Ap
    QKX_CUDA(cudaGetLastError());
    QKX_TRY(redot(c, r, r, n, FIN_R2, nullptr, 0));           // r2, beta = r2 / r2_old
    k_xpay<<<g, BLAS_NT, 0, c->st>>>(r, c->sc->beta, p, n);
    counted(c);          // p = r + beta p
    QKX_CUDA(cudaGetLastError());
    (*k)++;
    QKX_CUDA(cudaMemcpyAsync(c->hscal, c->sc->r2, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    QKX_CUDA(cudaStreamSynchronize(c->st));
    r2 = c->hscal[0];
    if (!(r2 == r2) || isinf(r2)) {
      *r2_host = r2;
      set_error("CG: r2 became %g at iteration %d", r2, *k);
      return QKX_ERR_NAN;
    }
  }
  *r2_host = r2;
  return QKX_OK;
}

static int cg_fp64_start(qkx_ctx* c, const double2* in, double2* r, double2* p, double* r2, double* src) {
  const size_t n = 12 * c->V;
  QKX_CUDA(cudaMemcpyAsync(r, in, sizeof(double2) * n, cudaMemcpyDeviceToDevice, c->st));
  QKX_CUDA(cudaMemcpyAsync(p, in, sizeof(double2) * n, cudaMemcpyDeviceToDevice, c->st));
  QKX_TRY(redot(c, r, r, n, FIN_R2_INIT, nullptr, 0));
  QKX_TRY(redot(c, in, in, n, FIN_STORE, c->dscal, 0));
  QKX_CUDA(cudaMemcpyAsync(c->hscal, c->sc->r2, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaMemcpyAsync(c->hscal + 1, c->dscal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  *r2 = c->hscal[0];
  *src = c->hscal[1];
  return QKX_OK;
}

int qkx_cg_dev(qkx_ctx* c, const double* in_dev, double* x_dev, qkx_solve_info* info) {
  if (!c || !in_dev || !x_dev) return invalid("NULL argument");
  if (!c->have_gauge) {
    set_error("CG needs a gauge field");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_work(c));
  double2 *r = c->w[2], *p = c->w[3], *Ap = c->w[4], *tmp = c->w[5];
  const double2* in = (const double2*)in_dev;
  double2* x = (double2*)x_dev;
  for (double2* f : {r, p, Ap, tmp})
    if ((const double2*)in == f || x == f) return invalid("CG fields alias the context's work fields");
  QKX_CUDA(cudaEventRecord(c->t0, c->st));
  double r2, src;
  QKX_TRY(cg_fp64_start(c, in, r, p, &r2, &src));
  const double stop = src * c->p.tol * c->p.tol;
  int k = 0;
  int rc = cg_fp64_loop(c, x, r, p, Ap, tmp, stop, c->p.maxIter, &k, &r2);
  QKX_CUDA(cudaEventRecord(c->t1, c->st));
  QKX_CUDA(cudaEventSynchronize(c->t1));
  QKX_TRY(device_status(c));
  if (info) {
    memset(info, 0, sizeof *info);
    info->iterations = k;
    info->converged = (rc == QKX_OK && r2 <= stop) ? 1 : 0;
    info->normal_residual = src > 0 ? sqrt(r2 / src) : 0.0;
    info->true_residual = -1.0;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    info->seconds = ms * 1e-3;
  }
  if (rc != QKX_OK) return rc;
  if (r2 > stop) {
    set_error("CG reached maxIter = %d (r2 = %g > %g)", c->p.maxIter, r2, stop);
    return QKX_ERR_NOT_CONVERGED;
  }
  return QKX_OK;
}

int qkx_cg(qkx_ctx* c, const double* in_host, double* x_host, qkx_solve_info* info) {
  if (!c || !in_host || !x_host) return invalid("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_work(c));
  QKX_TRY(upload_spinor(c, in_host, c->w[0]));
  QKX_TRY(upload_spinor(c, x_host, c->w[1]));
  int rc = qkx_cg_dev(c, (const double*)c->w[0], (double*)c->w[1], info);
  if (rc != QKX_OK && rc != QKX_ERR_NOT_CONVERGED) return rc;
  QKX_TRY(download_spinor(c, c->w[1], x_host));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return rc;
}

// ---------------------------------------------------------------- invert
// ||b - M x||^2 and ||b||^2 in FP64 (uses w[6] for M x)
static int true_residual(qkx_ctx* c, const double2* b, const double2* x, double* rel) {
  const size_t n = 12 * c->V;
  QKX_TRY(apply_tm(c, x, c->w[6], false));
  int g = blas_grid(n);
  k_sub_norm<<<g, BLAS_NT, 0, c->st>>>(b, c->w[6], c->w[6], n, c->part);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_TRY(finalize(c, g, FIN_STORE, c->dscal + 2, 0));
  QKX_TRY(redot(c, b, b, n, FIN_STORE, c->dscal + 3, 0));
  QKX_CUDA(cudaMemcpyAsync(c->hscal + 2, c->dscal + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  *rel = c->hscal[3] > 0 ? sqrt(c->hscal[2] / c->hscal[3]) : 0.0;
  return QKX_OK;
}

// Plain FP64 method: in = M^+ b, then the reference CG on M^+M; when the
// normal-equation stop leaves ||b - Mx||/||b|| above tol the same recurrence
// continues with a proportionally tighter stop.
static int invert_cg_fp64(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double2* const* b,
                          double2* const* x, qkx_solve_info* info) {
  QKX_TRY(ensure_work(c));
  double2 *in = c->w[0], *r = c->w[2], *p = c->w[3], *Ap = c->w[4], *tmp = c->w[5];
  const size_t n = 12 * c->V;
  for (int i = 0; i < nrhs; i++) {
    if (b[i] == in || x[i] == in || b[i] == r || x[i] == r || b[i] == p || x[i] == p || b[i] == Ap ||
        x[i] == Ap || b[i] == tmp || x[i] == tmp || b[i] == c->w[6] || x[i] == c->w[6])
      return invalid("invert fields alias the context's work fields");
  }
  QKX_CUDA(cudaEventRecord(c->t0, c->st));
  int worst = QKX_OK;
  for (int i = 0; i < nrhs; i++) {
    QKX_TRY(apply_tm(c, b[i], in, true));
    QKX_CUDA(cudaMemsetAsync(x[i], 0, sizeof(double2) * n, c->st));
    double r2, src;
    QKX_TRY(cg_fp64_start(c, in, r, p, &r2, &src));
    double stop = src * sp->tol * sp->tol;
    int k = 0, restarts = 0;
    double rel = 0;
    int rc = QKX_OK;
    for (;;) {
      rc = cg_fp64_loop(c, x[i], r, p, Ap, tmp, stop, sp->maxIter, &k, &r2);
      if (rc != QKX_OK) break;
      QKX_TRY(true_residual(c, b[i], x[i], &rel));
      if (rel <= sp->tol || k >= sp->maxIter || restarts >= 20) break;
      double f = sp->tol / rel;
      stop = std::min(stop, r2) * f * f * 0.5;
      restarts++;
    }
    if (rc == QKX_OK && rel > sp->tol) rc = QKX_ERR_NOT_CONVERGED;
    if (info) {
      info->iterations = std::max(info->iterations, k);
      info->restarts += restarts;
      info->true_residual = std::max(info->true_residual, rel);
      info->normal_residual = std::max(info->normal_residual, src > 0 ? sqrt(r2 / src) : 0.0);
    }
    if (rc != QKX_OK && worst == QKX_OK) worst = rc;
    if (rc == QKX_ERR_NAN || rc == QKX_ERR_CUDA) return rc;
  }
  QKX_CUDA(cudaEventRecord(c->t1, c->st));
  QKX_CUDA(cudaEventSynchronize(c->t1));
  if (info) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->t0, c->t1);
    info->seconds = ms * 1e-3;
    info->converged = worst == QKX_OK;
  }
  if (worst == QKX_ERR_NOT_CONVERGED) set_error("solve did not reach tol = %g", sp->tol);
  return worst;
}

int qkx_invert_dev(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double* const* b_dev,
                   double* const* x_dev, qkx_solve_info* info) {
  if (!c || !sp || !b_dev || !x_dev) return invalid("NULL argument");
  if (nrhs < 1 || nrhs > MAX_RHS) return invalid("nrhs must be in 1..64");
  for (int i = 0; i < nrhs; i++)
    if (!b_dev[i] || !x_dev[i]) return invalid("NULL field");
  if (!(sp->tol > 0) || sp->maxIter < 1) return invalid("tol/maxIter");
  if (!c->have_gauge) {
    set_error("invert needs a gauge field");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  const double2* const* b = (const double2* const*)b_dev;
  double2* const* x = (double2* const*)x_dev;
  int rc;
  if (sp->method == QKX_SOLVER_CG_FP64) rc = invert_cg_fp64(c, sp, nrhs, b, x, info);
  else if (sp->method == QKX_SOLVER_CG_EO_MIXED) rc = invert_eo_mixed(c, sp, nrhs, b, x, info);
  else if (sp->method == QKX_SOLVER_GCR_PTC) rc = invert_gcr_ptc(c, sp, nrhs, b, x, info);
  else return invalid("solver method");
  const int st = device_status(c);  // a bounded device wait that gave up voids the solution
  return st != QKX_OK ? st : rc;
}

int qkx_invert(qkx_ctx* c, const qkx_solver_params* sp, int nrhs, const double* const* b_host,
               double* const* x_host, qkx_solve_info* info) {
  if (!c || !sp || !b_host || !x_host) return invalid("NULL argument");
  if (nrhs < 1 || nrhs > MAX_RHS) return invalid("nrhs must be in 1..64");
  for (int i = 0; i < nrhs; i++)
    if (!b_host[i] || !x_host[i]) return invalid("NULL field");
  QKX_CUDA(cudaSetDevice(c->device));
  // device copies of every b and x (released when the call returns)
  const size_t fb = qkx_spinor_bytes(c);
  std::vector<double2*> bd(nrhs, nullptr), xd(nrhs, nullptr);
  int rc = QKX_OK;
  for (int i = 0; i < nrhs && rc == QKX_OK; i++) {
    if (cudaMallocAsync(&bd[i], fb, c->st) != cudaSuccess || cudaMallocAsync(&xd[i], fb, c->st) != cudaSuccess) {
      set_error("device allocation of %d right-hand sides failed", nrhs);
      rc = QKX_ERR_NOMEM;
    }
  }
  for (int i = 0; i < nrhs && rc == QKX_OK; i++) rc = upload_spinor(c, b_host[i], bd[i]);
  if (rc == QKX_OK) {
    rc = qkx_invert_dev(c, sp, nrhs, (const double* const*)bd.data(), (double* const*)xd.data(), info);
    if (rc == QKX_OK || rc == QKX_ERR_NOT_CONVERGED) {
      int rc2 = QKX_OK;
      for (int i = 0; i < nrhs && rc2 == QKX_OK; i++) rc2 = download_spinor(c, xd[i], x_host[i]);
      if (rc2 != QKX_OK) rc = rc2;
    }
  }
  for (int i = 0; i < nrhs; i++) {
    if (bd[i]) cudaFreeAsync(bd[i], c->st);
    if (xd[i]) cudaFreeAsync(xd[i], c->st);
  }
  cudaError_t e = cudaStreamSynchronize(c->st);
  if (rc == QKX_OK && e != cudaSuccess) {
    set_error("invert: %s", cudaGetErrorString(e));
    rc = QKX_ERR_CUDA;
  }
  return rc;
}

// ---------------------------------------------------------------- memory helpers
void* qkx_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}
void qkx_host_free(void* p) {
  if (p) cudaFreeHost(p);
}
void* qkx_device_alloc(qkx_ctx* c, size_t bytes) {
  if (!c) return nullptr;
  void* p = nullptr;
  if (cudaSetDevice(c->device) != cudaSuccess || cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}
void qkx_device_free(qkx_ctx* c, void* p) {
  if (c && p) {
    cudaSetDevice(c->device);
    cudaFree(p);
  }
}
int qkx_memcpy_h2d(qkx_ctx* c, void* dst, const void* src, size_t bytes) {
  if (!c || !dst || !src) return invalid("NULL argument");
  QKX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}
int qkx_memcpy_d2h(qkx_ctx* c, void* dst, const void* src, size_t bytes) {
  if (!c || !dst || !src) return invalid("NULL argument");
  QKX_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

// ---------------------------------------------------------------- profiling
int qkx_profile_enable(qkx_ctx* c, int on) {
  if (!c) return invalid("ctx is NULL");
  if (!on) QKX_TRY(prof_collect(c));
  c->prof = on ? 1 : 0;
  return QKX_OK;
}
int qkx_profile_read(qkx_ctx* c, long long* launches, double* ms, double* bytes) {
  if (!c) return invalid("ctx is NULL");
  QKX_TRY(prof_collect(c));
  if (launches) *launches = c->prof_launches;
  if (ms) *ms = c->prof_ms;
  if (bytes) *bytes = c->prof_bytes;
  return QKX_OK;
}
long long qkx_kernel_launches(const qkx_ctx* c) { return c ? c->kernels : -1; }

int qkx_tune(qkx_ctx* c, int precision, int nrhs, int* rhs_per_thread, int* threads_per_block,
             double* ms_per_hop) {
  if (!c) return invalid("ctx is NULL");
  if (nrhs < 1 || nrhs > MAX_RHS) return invalid("nrhs must be in 1..64");
  if (!c->have_gauge) {
    set_error("tuning needs a gauge field");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  return tune(c, precision, nrhs, rhs_per_thread, threads_per_block, ms_per_hop);
}

int qkx_set_tile(qkx_ctx* c, int precision, int nrhs, int rhs_per_thread, int threads_per_block, int kind) {
  if (!c) return invalid("ctx is NULL");
  if (nrhs < 1 || nrhs > MAX_RHS) return invalid("nrhs must be in 1..64");
  return set_tile(c, precision, nrhs, rhs_per_thread, threads_per_block, kind);
}

int qkx_tune_table(qkx_ctx* c, int precision, int nrhs, int max, int* count, int* rhs_per_thread,
                   int* threads_per_block, int* kind, double* ms_per_hop) {
  if (!c) return invalid("ctx is NULL");
  if (max < 0) return invalid("max must be >= 0");
  return tune_table(c, precision, nrhs, max, count, rhs_per_thread, threads_per_block, kind, ms_per_hop);
}

int qkx_sloppy_normal(qkx_ctx* c, int precision, int nrhs, int rhs_per_thread, int threads_per_block, int kind,
                      const double* const* in_host, double* const* out_host) {
  if (!c) return invalid("ctx is NULL");
  if (nrhs < 1 || nrhs > MAX_RHS) return invalid("nrhs must be in 1..64");
  if (!in_host || !out_host) return invalid("in_host/out_host is NULL");
  for (int i = 0; i < nrhs; i++)
    if (!in_host[i] || !out_host[i]) return invalid("a spinor pointer is NULL");
  if (!c->have_gauge) {
    set_error("the operator needs a gauge field");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  return sloppy_normal(c, precision, nrhs, rhs_per_thread, threads_per_block, kind, in_host, out_host);
}

int qkx_profile_reset(qkx_ctx* c) {
  if (!c) return invalid("ctx is NULL");
  QKX_TRY(prof_collect(c));
  c->prof_launches = 0;
  c->prof_ms = 0;
  c->prof_bytes = 0;
  return QKX_OK;
}

}  // extern "C"
