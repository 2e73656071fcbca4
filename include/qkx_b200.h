/*
 * qkx_b200.h -- C ABI of the B200 twisted-mass Dslash / CG library
 * (libqkx_b200.so).  Plain pointers and sizes only.
 *
 * It replaces the hot path of khadjiyiannakou/qkxTM_MPI: the operators that
 * are member functions of qkxTM::Vector (include/lattice_util.h:80-156), the
 * CG solver (include/solvers.h:3-22) and the qkxTM BLAS
 * (include/blas_qkxTM.h:3-5).  Each declaration names the reference
 * interface it stands in for.
 *
 * Host field layouts are the reference's own (so a caller hands over
 * Vector::M / Gauge::M unchanged):
 *   spinor  double[V][4][3][2]     (Vector::M,  include/lattice_util.h:90)
 *   gauge   double[V][4][3][3][2]  (Gauge::M,   include/lattice_util.h:198)
 *   site    x + Lx*(y + Ly*(z + Lz*t))  (LEXIC, include/qkxTM.h:130)
 * Device-resident fields (the *_dev entry points) use the library's even-odd
 * layout: double2 [parity][12][V/2], parity = (x+y+z+t)&1, site within a
 * parity = lexicographic index / 2.  qkx_spinor_bytes() gives the size.
 *
 * Errors: every call returns an int status (QKX_OK = 0, negative on error)
 * where the reference aborted the MPI job (errorQKXTM, include/qkxTM.h:137).
 * qkx_last_error() returns a message for the calling thread.
 * A context is not thread-safe; use one per thread.  All work of a context
 * runs on its own CUDA stream; calls that take host buffers return after the
 * results are in host memory.  The *_dev entry points are asynchronous on
 * that stream (qkx_sync waits).
 *
 * Lx must be even (the even-odd layout pairs x and x+1).
 */
#ifndef QKX_B200_H
#define QKX_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define QKX_API __attribute__((visibility("default")))
#else
#define QKX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define QKX_OK 0
#define QKX_ERR_INVALID (-1)        /* bad argument: null pointer, size, enum value */
#define QKX_ERR_CUDA (-2)           /* a CUDA call failed */
#define QKX_ERR_NOMEM (-3)          /* device or pinned allocation failed */
#define QKX_ERR_NOGAUGE (-4)        /* operator used before qkx_load_gauge */
#define QKX_ERR_NOT_CONVERGED (-5)  /* solver stopped at maxIter; the iterate is still written */
#define QKX_ERR_NAN (-6)            /* a solver scalar became NaN or Inf */
#define QKX_ERR_UNSUPPORTED (-7)    /* e.g. 12-real links requested for non-SU(3) links */

/* Mirrors the hot-path fields of struct LatticeInfo (include/qkxTM.h:156-204).
 * The process grid P is absent: one GPU holds the whole lattice. */
typedef struct qkx_params {
  int L[4];             /* LatticeInfo::L, x y z t */
  double kappa;         /* LatticeInfo::kappa */
  double mu;            /* LatticeInfo::mu */
  int twistSign;        /* LatticeInfo::twistSign, +1 or -1 */
  int boundaryT;        /* LatticeInfo::boundaryT, +1 periodic, -1 antiperiodic */
  double tol;           /* LatticeInfo::tol */
  int maxIter;          /* LatticeInfo::maxIter */
  double reliableDelta; /* LatticeInfo::reliableDelta (used by the mixed-precision solvers) */
} qkx_params;

typedef struct qkx_ctx qkx_ctx;

/* Library version string. */
QKX_API const char* qkx_version(void);
/* Message of the last failing call on this thread ("" if none). */
QKX_API const char* qkx_last_error(void);

/* Create a context on a CUDA device: allocates the device work fields for the
 * lattice L.  Replaces the construction of LatticeGeometry / Vector / Gauge
 * (lib/lattice_util.cpp:44-380) for the hot path. */
QKX_API int qkx_create(const qkx_params* p, int device, qkx_ctx** out);
QKX_API void qkx_destroy(qkx_ctx* ctx);
/* Change kappa, mu, twistSign, boundaryT, tol, maxIter, reliableDelta
 * (L must stay the same).  A changed boundaryT takes effect at the next
 * qkx_load_gauge / qkx_gauge_generate. */
QKX_API int qkx_set_params(qkx_ctx* ctx, const qkx_params* p);
QKX_API int qkx_get_params(const qkx_ctx* ctx, qkx_params* p);
/* Wait for all work queued on the context's stream. */
QKX_API int qkx_sync(qkx_ctx* ctx);
/* The context's cudaStream_t, as void*. */
QKX_API void* qkx_stream(qkx_ctx* ctx);
/* Bytes of a device spinor field in the even-odd layout (both parities). */
QKX_API size_t qkx_spinor_bytes(const qkx_ctx* ctx);
QKX_API size_t qkx_volume(const qkx_ctx* ctx);

/* ---------------------------------------------------------------- gauge */
/* How the links passed to qkx_load_gauge relate to the boundary condition. */
#define QKX_LINKS_AS_GIVEN 0  /* the operator uses the links exactly as passed, like
                                 Vector::tm does (the caller may already have run
                                 Gauge::applyBoundaryCondition, lib/lattice_util.cpp:708) */
#define QKX_LINKS_APPLY_BC 1  /* the operator applies boundaryT itself, as if
                                 Gauge::applyBoundaryCondition had been called */

/* Upload a gauge field in Gauge::M layout.  Replaces filling Gauge::M plus
 * Gauge::applyBoundaryCondition (lib/lattice_util.cpp:708-724) and the halo
 * exchange Gauge::communicateToPlus (:726-774), which has no counterpart on
 * one GPU.  The library also builds the compressed (12-real) copies used by
 * the mixed-precision solvers when the links are SU(3) up to a global sign on
 * the last time slice; otherwise those solvers return QKX_ERR_UNSUPPORTED. */
QKX_API int qkx_load_gauge(qkx_ctx* ctx, const double* U_host, int bc_mode);
/* Generate U_mu(x) = exp(i eps H) on the device (H traceless Hermitian from
 * unit complex Gaussians, counter-based generator keyed by seed) and use it
 * with bc_mode as in qkx_load_gauge.  No reference counterpart: the reference
 * reads ILDG files (lib/read_conf_lime.cpp). */
QKX_API int qkx_gauge_generate(qkx_ctx* ctx, double eps, unsigned long long seed, int bc_mode);
/* Download the links the operator uses (boundary sign included), Gauge::M layout. */
QKX_API int qkx_download_gauge(qkx_ctx* ctx, double* U_host);
/* 1 if 12-real compressed links are available, 0 if not, <0 on error. */
QKX_API int qkx_gauge_compressible(const qkx_ctx* ctx);

/* ---------------------------------------------------------------- operators */
/* Operator ids.  Each names the reference member function it reproduces
 * (all in lib/lattice_util.cpp); out = op(in) on full-lattice fields, with the
 * parity the reference zero-fills written as zero. */
enum qkx_op {
  QKX_OP_DSLASH = 0,                  /* Vector::applyDslash                 :1158 */
  QKX_OP_DSLASH_DAG = 1,              /* Vector::applyDslashDag              :1643 */
  QKX_OP_TM = 2,                      /* Vector::tm                          :1925 */
  QKX_OP_TM_DAG = 3,                  /* Vector::tmDag                       :1935 */
  QKX_OP_TM_DAGTM = 4,                /* Vector::tmDagtm                     :1940 */
  QKX_OP_WILSON = 5,                  /* Vector::Wilson                      :1949 */
  QKX_OP_TM_XX_EE = 6,                /* Vector::tm_xx(.., EE)               :2001 */
  QKX_OP_TM_XX_OO = 7,                /* Vector::tm_xx(.., OO)               :2001 */
  QKX_OP_TM_XX_DAGTM_XX_EE = 8,       /* Vector::tm_xxDagTm_xx(.., EE)       :2024 */
  QKX_OP_TM_XX_DAGTM_XX_OO = 9,       /* Vector::tm_xxDagTm_xx(.., OO)       :2024 */
  QKX_OP_DSLASH_CHIRAL = 10,          /* Vector::applyDslash_chiral          :1215 */
  QKX_OP_TM_CHIRAL = 11,              /* Vector::tm_chiral                   :1930 */
  QKX_OP_TM_XX_CHIRAL_EE = 12,        /* Vector::tm_xx_chiral(.., EE)        :2037 */
  QKX_OP_TM_XX_CHIRAL_OO = 13,        /* Vector::tm_xx_chiral(.., OO)        :2037 */
  QKX_OP_TM_XX_DAGTM_XX_CHIRAL_EE = 14, /* Vector::tm_xxDagTm_xx_chiral(..EE) :2060 */
  QKX_OP_TM_XX_DAGTM_XX_CHIRAL_OO = 15, /* Vector::tm_xxDagTm_xx_chiral(..OO) :2060 */
  QKX_OP_GAMMA5 = 16,                 /* Vector::applyGamma5                 :1778 */
  QKX_OP_GAMMA5_CHIRAL = 17,          /* Vector::applyGamma5_chiral          :1800 */
  QKX_OP_TWIST = 18,                  /* Vector::applyTwist                  :1563 */
  QKX_OP_TWIST_INV = 19,              /* Vector::applyTwistInv               :1588 */
  QKX_OP_TWIST_DAG = 20,              /* Vector::applyTwistDag               :1726 */
  QKX_OP_TWIST_DAG_INV = 21,          /* Vector::applyTwistDagInv            :1751 */
  QKX_OP_TWIST_INV_CHIRAL = 22,       /* Vector::applyTwistInv_chiral        :1615 */
  QKX_OP_DSLASH_XX_EO = 23,           /* Vector::applyDslash_xx(.., EO)      :1272 */
  QKX_OP_DSLASH_XX_OE = 24,           /* Vector::applyDslash_xx(.., OE)      :1272 */
  QKX_OP_ROTATE_CHIRAL_TO_UKQCD = 25, /* Vector::rotateFromChiralToUKQCD     :1834 */
  QKX_OP_DSLASH_XX_CHIRAL_EO = 26,    /* Vector::applyDslash_xx_chiral(.., EO) :1346 */
  QKX_OP_DSLASH_XX_CHIRAL_OE = 27,    /* Vector::applyDslash_xx_chiral(.., OE) :1346 */
  QKX_OP_TM_DAG_CHIRAL = 28,          /* tmDag in the chiral basis (no reference member; D^+ of :1215) */
  QKX_OP_TM_DAGTM_CHIRAL = 29,        /* tmDagtm in the chiral basis (no reference member) */
  QKX_OP_COUNT = 30
};

/* out = op(in), host buffers in Vector::M layout.  in and out may alias. */
QKX_API int qkx_apply(qkx_ctx* ctx, int op, const double* in_host, double* out_host);
/* out = op(in), device fields in the even-odd layout (in != out). */
QKX_API int qkx_apply_dev(qkx_ctx* ctx, int op, const double* in_dev, double* out_dev);
/* Host Vector::M layout <-> device even-odd layout (both on the context stream). */
QKX_API int qkx_spinor_upload(qkx_ctx* ctx, const double* host, double* dev);
QKX_API int qkx_spinor_download(qkx_ctx* ctx, const double* dev, double* host);

/* ---------------------------------------------------------------- BLAS */
/* Device fields in the even-odd layout, FP64, whole lattice. */
/* reCdotXdagY (lib/blas_qkxTM.cpp:4-28): Re sum conj(x) y */
QKX_API int qkx_reCdotXdagY(qkx_ctx* ctx, const double* x_dev, const double* y_dev, double* result);
/* X_eq_X_p_aY (lib/blas_qkxTM.cpp:31-42): x = x + a y */
QKX_API int qkx_X_eq_X_p_aY(qkx_ctx* ctx, double* x_dev, double a, const double* y_dev);
/* X_eq_aX_p_Y (lib/blas_qkxTM.cpp:45-56): x = a x + y */
QKX_API int qkx_X_eq_aX_p_Y(qkx_ctx* ctx, double* x_dev, double a, const double* y_dev);
/* Vector::norm2 (lib/lattice_util.cpp:464-477) */
QKX_API int qkx_norm2(qkx_ctx* ctx, const double* x_dev, double* result);

/* Allocation-free Re sum conj(x) y over n_sites sites (12 complex numbers each)
 * of two device fields, FP64, result written to *result (host memory) after
 * the work on `stream` (a cudaStream_t, NULL for the legacy default stream)
 * has finished.  No counterpart in the reference: it is reCdotXdagY for
 * callers that cannot allocate device memory -- code running under a fixed
 * device-memory budget that another allocator already owns, or that must not
 * enter the allocator on its path -- and therefore cannot create a qkx_ctx.
 * It calls no cudaMalloc/cudaFree: its scratch (the per-block partial sums)
 * is a fixed 512 KB array compiled into the library, resident on every GPU
 * that loads it until the process exits.  Inputs above QKX_NOALLOC_MAX_SITES
 * sites are rejected with QKX_ERR_INVALID, and so are field pointers that are
 * not 16-byte aligned or not device (or managed) memory of the current device,
 * before anything is launched.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it; after a
 * cudaDeviceReset of that device the kept address is stale, so do not call
 * again in that process.  The call waits for its result (a synchronizing copy
 * to host memory), so it cannot be made on a capturing stream: it returns
 * QKX_ERR_INVALID there.  All calls on a device share the array: calls whose
 * GPU work overlaps (other streams or host threads) race. */
#define QKX_NOALLOC_MAX_SITES 11184810ULL
QKX_API int qkx_reCdotXdagY_noalloc(const double* x_dev, const double* y_dev, size_t n_sites, double* result,
                                    void* stream);

/* ---------------------------------------------------------------- solvers */
typedef struct qkx_solve_info {
  int iterations;          /* CG iterations (max over right-hand sides) */
  int reliable_updates;    /* FP64 residual recomputations (mixed precision) */
  int converged;           /* 1 if every right-hand side met its target */
  int restarts;            /* CG_FP64: outer restarts made to reach the true-residual target;
                              CG_EO_MIXED: reliable updates after which a search direction
                              restarted from the new residual (it had grown more than 2x) */
  double true_residual;    /* max over RHS of ||b - M x|| / ||b||, recomputed in FP64 */
  double normal_residual;  /* max over RHS of the final CG residual ||r|| / ||in|| */
  double seconds;          /* device time of the solve (CUDA events) */
  int fallbacks;           /* right-hand sides that QKX_SOLVER_GCR_PTC handed to the plain solver */
  /* device time of the phases of a CG_EO_MIXED solve (0 for the other methods);
   * the inner iterations take seconds - setup - reliable - final */
  double seconds_setup;     /* gathering b, the Schur source b^ and Mh^+ b^ (FP64) */
  double seconds_reliable;  /* the FP64 reliable updates */
  double seconds_final;     /* odd sites, the FP64 true residual and the copies out */
} qkx_solve_info;

/* CG::operator()(out, in, param) (lib/solvers.cpp:16-81), FP64, full lattice:
 * solves M^+M out = in with the reference's algorithm and stopping rule
 * (r2 <= tol^2 |in|^2 or maxIter).  Like the reference, the result is ADDED
 * to the incoming content of x (callers zero it first) and the initial
 * residual is in.  Host buffers in Vector::M layout. */
QKX_API int qkx_cg(qkx_ctx* ctx, const double* in_host, double* x_host, qkx_solve_info* info);
QKX_API int qkx_cg_dev(qkx_ctx* ctx, const double* in_dev, double* x_dev, qkx_solve_info* info);

/* Solver methods for qkx_invert. */
#define QKX_SOLVER_CG_FP64 0        /* plain FP64 CG on M^+M, full lattice (the reference's method) */
#define QKX_SOLVER_CG_EO_MIXED 1    /* even-odd Schur CG, sloppy spinors/links, FP64 reliable updates */
#define QKX_SOLVER_GCR_PTC 2        /* the learned solver: all right-hand sides in one batch on the
                                       even-odd Schur system, flexible CG on its normal equations in
                                       FP32 preconditioned by K K^+ (K the network sp->preconditioner
                                       on the even sites; NULL = none), FP64 defect correction, and
                                       CG_EO_MIXED as the fallback */

#define QKX_PREC_DOUBLE 0
#define QKX_PREC_SINGLE 1
#define QKX_PREC_HALF 2

typedef struct qkx_solver_params {
  int method;              /* QKX_SOLVER_* */
  int sloppy_precision;    /* QKX_PREC_* for the inner iterations (CG_EO_MIXED) */
  double tol;              /* target for the true residual ||b - M x|| / ||b|| */
  int maxIter;             /* total iteration cap */
  double reliable_delta;   /* FP64 residual recomputation when |r| drops by this factor;
                              <= 0 picks the default of the sloppy precision (1e-2 half, 1e-5 single);
                              clamped to [5e-3, 0.5] for half and [1e-7, 0.5] for single: below that
                              the sloppy recursion drifts from the true residual and the solve
                              diverges (a right-hand side whose FP64 true residual grows 1000x
                              above its best is stopped with QKX_ERR_NOT_CONVERGED) */
  int use_graphs;          /* replay the inner iteration from a CUDA graph */
  const double* mu;        /* NULL, or nrhs twisted masses (one per right-hand side, the
                              multi-mass solve of CG_EO_MIXED); NULL = the context's mu */
  const struct qkx_ptc* preconditioner;  /* QKX_SOLVER_GCR_PTC: the trained network, or NULL */
} qkx_solver_params;

/* Solve M x_i = b_i for nrhs right-hand sides (host buffers, Vector::M layout),
 * each to ||b - M x|| / ||b|| <= sp->tol recomputed in FP64.  x is overwritten
 * (no initial guess).  This is the drop-in for the reference's solve sequence
 * vec_in.tmDag(b) ; CG(x, vec_in) (bin/test_invert.cpp:95-117).  info receives
 * the aggregate. */
QKX_API int qkx_invert(qkx_ctx* ctx, const qkx_solver_params* sp, int nrhs, const double* const* b_host,
               double* const* x_host, qkx_solve_info* info);
/* The same on device fields in the even-odd layout. */
QKX_API int qkx_invert_dev(qkx_ctx* ctx, const qkx_solver_params* sp, int nrhs, const double* const* b_dev,
                   double* const* x_dev, qkx_solve_info* info);

/* Many solves on several lattices at once (no reference counterpart).  Each
 * job is a batch of right-hand sides on its context (a lattice with its own
 * links, parameters and stream); sp applies to every job (its mu replaced by
 * the job's).  For QKX_SOLVER_CG_EO_MIXED with use_graphs, the jobs of a
 * context are merged into one batch (each right-hand side keeps its twisted
 * mass) and every context's whole solve is one branch of a single CUDA graph:
 * all lattices run from one launch and share the GPU, each branch at a stream
 * priority that grows as the lattice's volume falls (small lattices finish
 * first); a job's latency is when its lattice's branch ended, and its info is its
 * lattice's (true_residual the worst of the job's own right-hand sides; the
 * phase times are 0).  Otherwise the jobs of a context run in order on one
 * host thread and different contexts on different threads, so their kernels
 * overlap on the GPU; contexts start in order of decreasing volume. */
typedef struct qkx_batch_job {
  qkx_ctx* ctx;                /* the job's lattice */
  int nrhs;                    /* right-hand sides of this job */
  const double* const* b_dev;  /* nrhs device fields in the context's even-odd layout */
  double* const* x_dev;        /* nrhs device fields for the solutions */
  const double* mu;            /* NULL, or nrhs twisted masses */
  int status;                  /* out: QKX_OK or the job's error code */
  double latency;              /* out: seconds from the start of the batch to this job's results */
  qkx_solve_info info;         /* out */
  char message[160];           /* out: the error message when status != QKX_OK */
} qkx_batch_job;
QKX_API int qkx_invert_batch(qkx_batch_job* jobs, int njobs, const qkx_solver_params* sp);

/* Autotune the inner hop of CG_EO_MIXED for this lattice, precision and batch
 * size: times every tile (right-hand sides per thread x threads per block) on
 * the device and keeps the fastest for later solves (a solve with an untuned
 * (precision, nrhs) tunes itself first, outside its timed region).  No
 * reference counterpart. */
QKX_API int qkx_tune(qkx_ctx* ctx, int precision, int nrhs, int* rhs_per_thread, int* threads_per_block,
                     double* ms_per_hop);

/* A tile of the sloppy hop is (rhs_per_thread, threads_per_block, kind).
 * kind 0 is the plain kernel for any precision; kinds 1-7 are FP16-only
 * variants for two right-hand sides a thread: loads of the next neighbour term
 * held in registers (1-3: no / a 128 / a ~100 registers-a-thread launch
 * bound), the plain pair kernel with a 128-register bound (4), and loads staged
 * in shared memory by cp.async one (5, 7) or two (6) terms ahead with a 128
 * (5, 6) or ~100 (7) register bound, and as 5 with the spin projection done in
 * FP16 before widening to FP32 (8) and also 18-real FP32 links (9), or also
 * the link multiply in FP16 on 18-real FP16 links (10; rounds the products to
 * FP16, so qkx_tune never picks it: only qkx_set_tile selects it), or as 8
 * on 18-real FP16 links (11: no third-row rebuild).
 *
 * Use this tile (one of the tuner's) for later CG_EO_MIXED solves and
 * qkx_sloppy_normal calls with this precision and batch size, instead of the
 * tuned one.  No reference counterpart. */
QKX_API int qkx_set_tile(qkx_ctx* ctx, int precision, int nrhs, int rhs_per_thread, int threads_per_block,
                         int kind);

/* The per-tile timings of the last tuning of (precision, nrhs): *count tiles,
 * the first min(*count, max) written to the arrays (any may be NULL).  0 tiles
 * if that key was never tuned.  No reference counterpart. */
QKX_API int qkx_tune_table(qkx_ctx* ctx, int precision, int nrhs, int max, int* count, int* rhs_per_thread,
                           int* threads_per_block, int* kind, double* ms_per_hop);

/* out_r = Vector::tm_xxDagTm_xx(.., EE) in_r (lib/lattice_util.cpp:2024) for a
 * batch, computed the way one inner iteration of CG_EO_MIXED computes A p: the
 * even sites of in_r rounded to the sloppy precision, then the four sloppy hops
 * with the given tile (one of the tuner's; 0, 0, 0 = the tuned tile).  Odd sites of out_r are zero.  Host buffers in
 * Vector::M layout.  A hook for checking every tile against the FP64 operator;
 * no reference counterpart. */
QKX_API int qkx_sloppy_normal(qkx_ctx* ctx, int precision, int nrhs, int rhs_per_thread, int threads_per_block,
                              int kind, const double* const* in_host, double* const* out_host);

/* ---------------------------------------------------------------- gauge-side stencils
 * The smearing links are a second FP64 gauge field held by the context, used
 * only by the Gaussian smearing: they are set by qkx_ape_smear or
 * qkx_load_smearing_gauge and are independent of the operator's links. */
#define QKX_LINKS_OPERATOR 0   /* the links of qkx_load_gauge / qkx_gauge_generate, as stored */
#define QKX_LINKS_SMEARING 1   /* the smearing links */

/* Gauge::calculatePlaquette() (lib/lattice_util.cpp:923-946): the mean over
 * sites and the six planes of Re tr U_mu U_nu U_mu^+ U_nu^+ / 3, for the host
 * links U_host (Gauge::M layout, taken as given). */
QKX_API int qkx_plaquette(qkx_ctx* ctx, const double* U_host, double* plaquette);
/* The same for a field the context holds (QKX_LINKS_OPERATOR includes the
 * boundary sign when it was applied at load time). */
QKX_API int qkx_plaquette_loaded(qkx_ctx* ctx, int which, double* plaquette);

/* qcd_projectSU33d(Gauge&) (lib/blas.cpp:6-404): projects the spatial links
 * (mu = 0, 1, 2) of the host field U_host to SU(3) in place; t-links unchanged. */
QKX_API int qkx_project_su3(qkx_ctx* ctx, double* U_host);

/* this->APE_smearing(U_tmp, &li) (lib/lattice_util.cpp:948-1078) with U_tmp =
 * U_in, li.NsmearAPE = nsmear, li.alphaAPE = alpha: nsmear iterations of
 * U_mu <- P_SU3[U_mu + alpha * (sum of the four spatial staples)] on the
 * spatial links; the t-links are those of U_in.  The result becomes the
 * context's smearing links and, if U_out is not NULL, is written to U_out.
 * U_in is left unchanged (the reference overwrites U_tmp).  nsmear == 0 does
 * nothing, as in the reference. */
QKX_API int qkx_ape_smear(qkx_ctx* ctx, const double* U_in, double* U_out, int nsmear, double alpha);
/* Set the smearing links from host links (Gauge::M layout, as given). */
QKX_API int qkx_load_smearing_gauge(qkx_ctx* ctx, const double* U_host);

/* this->Gaussian_smearing(vec_tmp, gauge, &li) (lib/lattice_util.cpp:1080-1145)
 * for nrhs vectors at once, vec_tmp = in[i], gauge = the smearing links:
 * nsmear iterations of psi <- (psi + alpha sum_{mu<3} [U_mu(x) psi(x+mu) +
 * U_mu(x-mu)^+ psi(x-mu)]) / (1 + 6 alpha).  Host buffers in Vector::M layout.
 * The inputs are left unchanged (the reference overwrites vec_tmp).  nsmear
 * == 0 leaves out untouched, as in the reference. */
QKX_API int qkx_gaussian_smear(qkx_ctx* ctx, int nrhs, const double* const* in_host, double* const* out_host,
                               int nsmear, double alpha);
/* The same on device fields in the even-odd layout; in[i] != out[j] for all i, j. */
QKX_API int qkx_gaussian_smear_dev(qkx_ctx* ctx, int nrhs, const double* const* in_dev, double* const* out_dev,
                                   int nsmear, double alpha);

/* ---------------------------------------------------------------- two-point functions
 * From propagators in the Propagator::M layout (host, or device memory for the
 * _dev forms, e.g. the output of qkx_propagator_dev).  Momenta p = 2 pi n / L
 * are those of createMomenta (lib/contractions.cpp:37): every integer n with
 * |n|^2 = q for q = 0..Q_sq, each component running from +q down to -q; the
 * Fourier transform is sum_x C(x) exp(-i p.(x - x_src)) over each time slice,
 * with the reference's pi = 3.14159265359 and x - x_src not wrapped. */
#define QKX_NUM_MESONS 10   /* MESONS_OPERATOR order: ONE G5 G1 G2 G3 G4 G5G1 G5G2 G5G3 G5G4 */
#define QKX_BARYON_NTN 0    /* BARYON_OPERATOR order */
#define QKX_BARYON_NTR 1
#define QKX_BARYON_RTN 2
#define QKX_BARYON_RTR 3

/* createMomenta: writes up to max momenta as mom[i][3] and returns their number */
QKX_API int qkx_momenta(int Q_sq, int* mom, int max);
/* Meson::contract(prop, op) + Meson::fourier(FORWARD) (lib/contractions.cpp:251,
 * :121) for nop operators: corr[op][t][imom] complex (Meson::F per operator). */
QKX_API int qkx_meson_2pt(qkx_ctx* ctx, const double* prop_host, int nop, const int* ops, int Q_sq,
                          const int x_src[4], double* corr);
QKX_API int qkx_meson_2pt_dev(qkx_ctx* ctx, const double* prop_dev, int nop, const int* ops, int Q_sq,
                              const int x_src[4], double* corr);
/* Baryon::contract(prop1, prop2, op) + Baryon::fourier(FORWARD) (lib/contractions.cpp:494,
 * :356): corr[t][imom][gamma][gamma'] complex (Baryon::F). */
QKX_API int qkx_baryon_2pt(qkx_ctx* ctx, const double* prop1_host, const double* prop2_host, int op, int Q_sq,
                           const int x_src[4], double* corr);
QKX_API int qkx_baryon_2pt_dev(qkx_ctx* ctx, const double* prop1_dev, const double* prop2_dev, int op, int Q_sq,
                               const int x_src[4], double* corr);
#define QKX_DELTA_ISO1 0    /* BARYON_DEC_OPERATOR order */
#define QKX_DELTA_ISO1O2 1
/* Baryon_Dec::contract(prop1, prop2, op) + Baryon_Dec::fourier(FORWARD)
 * (lib/contractions.cpp:768-866, :703-741): the decuplet with the three spatial
 * C gamma_i; corr[t][imom][i][gamma][gamma'] complex (Baryon_Dec::F). */
QKX_API int qkx_delta_2pt(qkx_ctx* ctx, const double* prop1_host, const double* prop2_host, int op, int Q_sq,
                          const int x_src[4], double* corr);
QKX_API int qkx_delta_2pt_dev(qkx_ctx* ctx, const double* prop1_dev, const double* prop2_dev, int op, int Q_sq,
                              const int x_src[4], double* corr);
/* contractNucleon(prop1, prop2, output, Q_sq, x_src) (lib/lattice_util.cpp:3374):
 * corr[t][imom][gamma][gamma1] complex, the numbers that function prints per time
 * slice (the C++ layer's contractNucleon writes them in its text format). */
QKX_API int qkx_nucleon_2pt(qkx_ctx* ctx, const double* prop1_host, const double* prop2_host, int Q_sq,
                            const int x_src[4], double* corr);
QKX_API int qkx_nucleon_2pt_dev(qkx_ctx* ctx, const double* prop1_dev, const double* prop2_dev, int Q_sq,
                                const int x_src[4], double* corr);

/* ---------------------------------------------------------------- ILDG / LIME configurations
 * A LIME file is a sequence of records, each a 144-byte big-endian header
 * (magic 0x456789ab, version, MB/ME flags, data length, 128-byte type string)
 * followed by its data padded to a multiple of 8 bytes.  An ILDG gauge
 * configuration has an "ildg-format" XML record (<precision>, <lx> .. <lt>)
 * and an "ildg-binary-data" record: V x 4 x 3 x 3 big-endian complex numbers,
 * sites with x fastest and t slowest, directions x y z t -- the Gauge::M
 * layout once byte-swapped. */
typedef struct qkx_lime_info {
  int precision;            /* 64 or 32 (bits per real), from the ildg-format record (64 if absent) */
  int L[4];                 /* lattice extents from the ildg-format record (0 if absent) */
  long long data_offset;    /* byte offset of the binary data in the file */
  long long data_bytes;     /* its length */
  int records;              /* records scanned */
} qkx_lime_info;

/* qkxTM_MPI_getGaugeLime(fname, u) (lib/read_conf_lime.cpp:111-245): read the
 * ildg-binary-data record of an ILDG file into the context as its operator
 * links (bc_mode as in qkx_load_gauge) and, if U_host is not NULL, into U_host
 * (Gauge::M layout).  The file is streamed through two page-locked buffers, so
 * disk reads overlap the host-to-device copies; the byte swap and the layout
 * change run on the GPU.  Beyond the reference: 32-bit files are accepted
 * (converted to FP64), and the extents in the ildg-format record must match
 * the context's lattice. */
QKX_API int qkx_read_gauge_lime(qkx_ctx* ctx, const char* path, int bc_mode, double* U_host, qkx_lime_info* info);
/* qkxTM_writeGaugeLime(fname, u, message) (lib/write_conf_lime.cpp:49-199):
 * write an ILDG file with the records ildg-format (64-bit), xlf-info (message)
 * and ildg-binary-data.  U_host (Gauge::M layout) is written, or the context's
 * operator links as stored when U_host is NULL. */
QKX_API int qkx_write_gauge_lime(qkx_ctx* ctx, const char* path, const double* U_host, const char* message);

/* ---------------------------------------------------------------- propagators
 * A propagator is double[V][4 mu][4 nu][3 c1][3 c2][2] (Propagator::M,
 * include/lattice_util.h:168), site order LEXIC; V*2304 bytes. */

/* Propagator::absorbVector(phi, nu, c2) (lib/lattice_util.cpp:2073-2081):
 * prop[x][mu][nu][c1][c2] = phi[x][mu][c1] for every x, mu, c1 (host buffers). */
QKX_API int qkx_propagator_absorb(qkx_ctx* ctx, const double* phi_host, int nu, int c2, double* prop_host);

/* The smeared-source propagator of bin/test_invert_prop.cpp:83-97 in one call:
 * for the 12 spin-colour point sources at x_src (coordinates x y z t) it
 * Gaussian-smears the sources (nsmear, alpha, with the smearing links), solves
 * M x = b for all 12 at once with sp, smears the 12 solutions and assembles
 * them as prop[.][.][nu][.][c2] = solution of source (nu, c2).  The reference
 * solves each source with tmDag + CG; here sp->method picks the solver and
 * sp->tol bounds the true residual.  nsmear == 0 uses unsmeared sources and
 * sinks.  info receives the solve's aggregate. */
QKX_API int qkx_propagator(qkx_ctx* ctx, const qkx_solver_params* sp, int nsmear, double alpha, const int x_src[4],
                           double* prop_host, qkx_solve_info* info);
/* The same with the propagator written to device memory (V*2304 bytes, host layout). */
QKX_API int qkx_propagator_dev(qkx_ctx* ctx, const qkx_solver_params* sp, int nsmear, double alpha,
                               const int x_src[4], double* prop_dev, qkx_solve_info* info);

/* ---------------------------------------------------------------- learned preconditioner
 * No reference counterpart.  A linear, gauge-covariant parallel-transport
 * convolution network N approximating M^-1: layer l maps channels[l] to
 * channels[l+1] colour vectors per site,
 *   out(x)[c] = sum_{p=0..8} sum_c' W[p][c][c'] (T_p in)(x)[c'],
 * T_0 = 1, T_{1+2mu} a(x) = U_mu(x) a(x+mu), T_{2+2mu} a(x) = U_mu(x-mu)^+ a(x-mu),
 * with the context's links (boundary sign included).  channels[0] =
 * channels[nlayers] = 4 (the spins), so N maps a spinor to a spinor.  Weights
 * are complex, [9][channels[l+1]][channels[l]] per layer, layers concatenated;
 * the kernels use BF16 copies with FP32 arithmetic.  Widths are 4, 8 or 16. */
typedef struct qkx_ptc qkx_ptc;
#define QKX_PTC_MAX_LAYERS 8

typedef struct qkx_ptc_params {
  int nlayers;                               /* 1..QKX_PTC_MAX_LAYERS */
  int channels[QKX_PTC_MAX_LAYERS + 1];      /* widths, 4/8/16, first and last 4 */
  unsigned long long seed;                   /* random initial weights */
  double init_scale;                         /* std of the initial hop-path weights (identity path starts
                                                as the identity, so N starts close to 1) */
  int tensor_cores;                          /* 1: the 16 -> 16 layers of qkx_ptc_apply and of the solver
                                                run on the tensor cores (tcgen05, BF16 activations and
                                                weights, FP32 accumulation); training always uses the
                                                FP32-activation kernels */
} qkx_ptc_params;

typedef struct qkx_ptc_train_params {
  int n_solves;            /* (residual, error) pairs on the even-odd Schur system Mh x_e = b^_e
                              that QKX_SOLVER_GCR_PTC preconditions: from as many mixed-precision
                              CG solves of Gaussian sources b, r = b^_e and e = x_e, plus as many
                              pairs r = Mh v_e, e = v_e for Gaussian v (the short-distance part of
                              Mh^-1); inputs are zero on the odd sites, the loss counts the even
                              sites */
  int steps;               /* Adam steps, one pair each, pairs in a seeded shuffled order */
  double lr;               /* peak learning rate (cosine decay to lr/20) */
  double solve_tol;        /* true-residual tolerance of the data solves */
  unsigned long long seed; /* sources and pair order */
} qkx_ptc_train_params;

typedef struct qkx_ptc_train_info {
  double loss_initial;     /* mean |N(r) - e|^2 / |e|^2 (even sites) over up to 4 pairs of each
                              kind, before */
  double loss_final;       /* the same after training */
  double seconds_data;     /* device time of the data solves */
  double seconds_train;    /* device time of the training steps */
  int steps;
} qkx_ptc_train_info;

QKX_API int qkx_ptc_create(qkx_ctx* ctx, const qkx_ptc_params* p, qkx_ptc** out);
QKX_API void qkx_ptc_destroy(qkx_ptc* net);
/* number of complex weights */
QKX_API long qkx_ptc_num_weights(const qkx_ptc* net);
/* weights as [n][2] doubles: which = 0 the FP32 master copy, 1 the BF16 copy the kernels use */
QKX_API int qkx_ptc_get_weights(const qkx_ptc* net, int which, double* w);
QKX_API int qkx_ptc_set_weights(qkx_ptc* net, const double* w);
/* out = N(in), host spinors (Vector::M layout) */
QKX_API int qkx_ptc_apply(qkx_ptc* net, const double* in_host, double* out_host);
/* loss |N(r) - e|^2 / |e|^2 on one pair and its gradient dL/dW^* ([n][2] doubles, may be NULL),
 * computed by the training kernels with the BF16 weights */
QKX_API int qkx_ptc_loss_grad(qkx_ptc* net, const double* r_host, const double* e_host, double* loss,
                              double* grad);
/* make the training pairs with the context's solver and train with Adam */
QKX_API int qkx_ptc_train(qkx_ptc* net, const qkx_ptc_train_params* tp, qkx_ptc_train_info* info);

/* ---------------------------------------------------------------- memory helpers */
/* Page-locked host memory for fast transfers (cudaHostAlloc); NULL on failure. */
QKX_API void* qkx_host_alloc(size_t bytes);
QKX_API void qkx_host_free(void* p);
/* Device memory on the context's device (cudaMalloc); NULL on failure. */
QKX_API void* qkx_device_alloc(qkx_ctx* ctx, size_t bytes);
QKX_API void qkx_device_free(qkx_ctx* ctx, void* p);
QKX_API int qkx_memcpy_h2d(qkx_ctx* ctx, void* dst, const void* src, size_t bytes);
QKX_API int qkx_memcpy_d2h(qkx_ctx* ctx, void* dst, const void* src, size_t bytes);

/* ---------------------------------------------------------------- profiling */
/* When enabled, every launch of the hopping kernels is bracketed by CUDA
 * events on the context stream; qkx_profile_read returns the count and the
 * summed device milliseconds and bytes of algorithmic traffic since the last reset. */
QKX_API int qkx_profile_enable(qkx_ctx* ctx, int on);
QKX_API int qkx_profile_read(qkx_ctx* ctx, long long* launches, double* ms, double* bytes);
QKX_API int qkx_profile_reset(qkx_ctx* ctx);
/* Kernels this context has launched since creation (a replayed CUDA graph
 * counts each of its kernel nodes); -1 for a NULL context. */
QKX_API long long qkx_kernel_launches(const qkx_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
