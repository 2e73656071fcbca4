// smear.cu -- C ABI of the gauge-side stencils (plaquette, SU(3) projection,
// APE smearing), the Gaussian smearing and the smeared-source propagator of
// the reference's bin/test_invert_prop.cpp, on one B200.
#include <math.h>
#include <string.h>

#include <vector>

#include "layout.cuh"
#include "qkx_ctx.cuh"
#include "smear.cuh"

using namespace qkx;

namespace qkx {
namespace {

constexpr int SM_NT = 128;  // block size of the link kernels

int bad(const char* what) {
  set_error("invalid argument: %s", what);
  return QKX_ERR_INVALID;
}

ProjConst proj_const() { return {pow(18., 1. / 3.), pow(12., 1. / 3.), pow(2. / 3., 1. / 3.), sqrt(3.)}; }

// A device temporary on the context stream's allocator, released on scope exit.
struct Tmp {
  cudaStream_t st;
  void* p = nullptr;
  explicit Tmp(cudaStream_t s) : st(s) {}
  ~Tmp() {
    if (p) cudaFreeAsync(p, st);
  }
  int alloc(size_t bytes, const char* what) {
    if (cudaMallocAsync(&p, bytes, st) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      set_error("device allocation of %s (%zu bytes) failed", what, bytes);
      return QKX_ERR_NOMEM;
    }
    return QKX_OK;
  }
  double2* d() const { return (double2*)p; }
};

size_t gauge_words(const qkx_ctx* c) { return (size_t)36 * c->V; }  // double2 per gauge field
size_t field_words(const qkx_ctx* c) { return (size_t)12 * c->V; }  // double2 per spinor field

// host Gauge::M links (as given) -> even-odd FP64 device field
int upload_links(qkx_ctx* c, const double* U_host, double2* eo) {
  Tmp t(c->st);
  QKX_TRY(t.alloc(sizeof(double2) * gauge_words(c), "link staging"));
  QKX_CUDA(cudaMemcpyAsync(t.p, U_host, sizeof(double2) * gauge_words(c), cudaMemcpyHostToDevice, c->st));
  k_gauge_aos_to_eo<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(t.d(), eo, c->geom, 1);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

int download_links(qkx_ctx* c, const double2* eo, double* U_host) {
  Tmp t(c->st);
  QKX_TRY(t.alloc(sizeof(double2) * gauge_words(c), "link staging"));
  k_gauge_eo_to_aos<<<(unsigned)((c->V + 255) / 256), 256, 0, c->st>>>(eo, t.d(), c->geom);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaMemcpyAsync(U_host, t.p, sizeof(double2) * gauge_words(c), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

int ensure_smear_links(qkx_ctx* c) {
  if (c->Usm) return QKX_OK;
  if (cudaMalloc(&c->Usm, sizeof(double2) * gauge_words(c)) != cudaSuccess) {
    c->Usm = nullptr;
    cudaGetLastError();
    set_error("smearing links: device allocation failed");
    return QKX_ERR_NOMEM;
  }
  return QKX_OK;
}

int plaquette_of(qkx_ctx* c, const double2* eo, double* out) {
  const int nblk = (c->Vh + SM_NT - 1) / SM_NT;
  k_plaquette<SM_NT><<<2 * nblk, SM_NT, 0, c->st>>>(GaugeF64x18{eo, c->Vh}, c->geom, c->part);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  QKX_TRY(finalize(c, 2 * nblk, FIN_STORE, c->dscal, 0));
  QKX_CUDA(cudaMemcpyAsync(c->hscal, c->dscal, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  *out = c->hscal[0] / ((double)c->V * 3.0 * 6.0);
  return QKX_OK;
}

// nsmear APE steps from the spatial links of `in`; the result lands in R (its
// t-links copied from `in`), T is scratch.  Algorithmic traffic per step: the
// three spatial links of every site read once and written once.
int ape_run(qkx_ctx* c, const double2* in, double2* R, double2* T, int nsmear, double alpha) {
  const size_t tl = (size_t)9 * c->Vh;
  for (int par = 0; par < 2; par++)
    QKX_CUDA(cudaMemcpyAsync(R + (size_t)(par * 4 + 3) * tl, in + (size_t)(par * 4 + 3) * tl, sizeof(double2) * tl,
                             cudaMemcpyDeviceToDevice, c->st));
  const ProjConst pc = proj_const();
  const int nblk = (c->Vh + SM_NT - 1) / SM_NT;
  const double2* src = in;
  double2* dst = (nsmear & 1) ? R : T;
  for (int it = 0; it < nsmear; it++) {
    QKX_TRY(prof_begin(c));
    k_ape_step<SM_NT><<<6 * nblk, SM_NT, 0, c->st>>>(GaugeF64x18{src, c->Vh}, dst, c->geom, alpha, pc);
    counted(c);
    QKX_CUDA(cudaGetLastError());
    QKX_TRY(prof_end(c, 864.0 * c->V));
    src = dst;
    dst = (dst == R) ? T : R;
  }
  return QKX_OK;
}

// ---------------------------------------------------------------- Gaussian smearing
struct GaussTile {
  int nr, nt;
};
constexpr GaussTile kGaussTiles[] = {{1, 64}, {1, 128}, {1, 256}, {2, 64}, {2, 128}, {2, 256}};

template <int NT, int NR>
void launch_gauss_t(qkx_ctx* c, const FieldPtrs& in, const FieldPtrs& out, int nrhs, int cb0, int ncb, double alpha,
                    double norm) {
  const int nblk = (ncb + NT - 1) / NT;
  const int ngrp = (nrhs + NR - 1) / NR;
  k_gauss_step<NT, NR><<<(unsigned)nblk * 2 * ngrp, NT, 0, c->st>>>(in, out, GaugeF64x18{c->Usm, c->Vh}, c->geom,
                                                                     nrhs, cb0, ncb, alpha, norm);
}

int launch_gauss(qkx_ctx* c, GaussTile t, const FieldPtrs& in, const FieldPtrs& out, int nrhs, int cb0, int ncb,
                 double alpha, double norm) {
  switch (t.nr * 1000 + t.nt) {
    case 1064: launch_gauss_t<64, 1>(c, in, out, nrhs, cb0, ncb, alpha, norm); break;
    case 1128: launch_gauss_t<128, 1>(c, in, out, nrhs, cb0, ncb, alpha, norm); break;
    case 1256: launch_gauss_t<256, 1>(c, in, out, nrhs, cb0, ncb, alpha, norm); break;
    case 2064: launch_gauss_t<64, 2>(c, in, out, nrhs, cb0, ncb, alpha, norm); break;
    case 2128: launch_gauss_t<128, 2>(c, in, out, nrhs, cb0, ncb, alpha, norm); break;
    case 2256: launch_gauss_t<256, 2>(c, in, out, nrhs, cb0, ncb, alpha, norm); break;
    default: set_error("internal: no smearing tile %d/%d", t.nr, t.nt); return QKX_ERR_INVALID;
  }
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return QKX_OK;
}

// The tile (right-hand sides per thread, threads per block) of the smearing
// step for a batch size, timed once per context on a full-lattice step from
// `in` into `scratch` (the caller's data are not changed).
int gauss_tile(qkx_ctx* c, int nrhs, const FieldPtrs& in, const FieldPtrs& scratch, double alpha, double norm,
               GaussTile* out) {
  const int key = 900000 + nrhs;
  auto it = c->tuned.find(key);
  if (it != c->tuned.end()) {
    *out = {it->second.nr, it->second.nt};
    return QKX_OK;
  }
  cudaEvent_t a, b;
  QKX_CUDA(cudaEventCreate(&a));
  QKX_CUDA(cudaEventCreate(&b));
  GaussTile best = kGaussTiles[0];
  float best_ms = 1e30f;
  int rc = QKX_OK;
  for (const GaussTile& t : kGaussTiles) {
    if (t.nr > 1 && nrhs < t.nr) continue;
    float ms = 0;
    for (int rep = 0; rep < 3 && rc == QKX_OK; rep++) {  // first run warms up
      if (cudaEventRecord(a, c->st) != cudaSuccess) rc = QKX_ERR_CUDA;
      if (rc == QKX_OK) rc = launch_gauss(c, t, in, scratch, nrhs, 0, c->Vh, alpha, norm);
      if (rc == QKX_OK && cudaEventRecord(b, c->st) != cudaSuccess) rc = QKX_ERR_CUDA;
      if (rc == QKX_OK && cudaEventSynchronize(b) != cudaSuccess) rc = QKX_ERR_CUDA;
      float m = 0;
      if (rc == QKX_OK && cudaEventElapsedTime(&m, a, b) != cudaSuccess) rc = QKX_ERR_CUDA;
      if (rep > 0) ms += m;
    }
    if (rc != QKX_OK) break;
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc == QKX_ERR_CUDA) set_error("smearing tile timing: %s", cudaGetErrorString(cudaGetLastError()));
  if (rc != QKX_OK) return rc;
  c->tuned[key] = {best.nr, best.nt, 0};
  *out = best;
  return QKX_OK;
}

// nsmear Gaussian smearing steps of nrhs fields on the sites cb in [cb0, cb0 +
// ncb) of both parities (the whole lattice, or whole time slices: the stencil
// is spatial, so slices do not mix).  The result lands in `out`; `tmp` is
// scratch; `in` is read only.
int gauss_run(qkx_ctx* c, int nrhs, const FieldPtrs& in, const FieldPtrs& out, const FieldPtrs& tmp, int nsmear,
              double alpha, int cb0, int ncb) {
  const double norm = 1.0 / (1.0 + 6.0 * alpha);
  GaussTile tile;
  QKX_TRY(gauss_tile(c, nrhs, in, tmp, alpha, norm, &tile));
  const double bytes = 2.0 * ncb * (384.0 * nrhs + 432.0);
  const FieldPtrs* src = &in;
  const FieldPtrs* dst = (nsmear & 1) ? &out : &tmp;
  for (int it = 0; it < nsmear; it++) {
    QKX_TRY(prof_begin(c));
    QKX_TRY(launch_gauss(c, tile, *src, *dst, nrhs, cb0, ncb, alpha, norm));
    QKX_TRY(prof_end(c, bytes));
    src = dst;
    dst = (dst == &out) ? &tmp : &out;
  }
  return QKX_OK;
}

FieldPtrs batch_ptrs(double2* base, int n, size_t words) {
  FieldPtrs f{};
  for (int i = 0; i < n; i++) f.p[i] = base + (size_t)i * words;
  return f;
}

}  // namespace
}  // namespace qkx

// =================================================================== C ABI
extern "C" {

int qkx_plaquette(qkx_ctx* c, const double* U_host, double* plaquette) {
  if (!c || !U_host || !plaquette) return bad("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  Tmp eo(c->st);
  QKX_TRY(eo.alloc(sizeof(double2) * gauge_words(c), "links"));
  QKX_TRY(upload_links(c, U_host, eo.d()));
  return plaquette_of(c, eo.d(), plaquette);
}

int qkx_plaquette_loaded(qkx_ctx* c, int which, double* plaquette) {
  if (!c || !plaquette) return bad("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  if (which == QKX_LINKS_OPERATOR) {
    if (!c->have_gauge) {
      set_error("no gauge field loaded");
      return QKX_ERR_NOGAUGE;
    }
    return plaquette_of(c, c->U18, plaquette);
  }
  if (which == QKX_LINKS_SMEARING) {
    if (!c->have_smear) {
      set_error("no smearing links set");
      return QKX_ERR_NOGAUGE;
    }
    return plaquette_of(c, c->Usm, plaquette);
  }
  return bad("which");
}

int qkx_project_su3(qkx_ctx* c, double* U_host) {
  if (!c || !U_host) return bad("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  Tmp eo(c->st);
  QKX_TRY(eo.alloc(sizeof(double2) * gauge_words(c), "links"));
  QKX_TRY(upload_links(c, U_host, eo.d()));
  const int nblk = (c->Vh + SM_NT - 1) / SM_NT;
  k_project_su3<SM_NT><<<6 * nblk, SM_NT, 0, c->st>>>(eo.d(), c->geom, proj_const());
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return download_links(c, eo.d(), U_host);
}

int qkx_ape_smear(qkx_ctx* c, const double* U_in, double* U_out, int nsmear, double alpha) {
  if (!c || !U_in) return bad("NULL argument");
  if (nsmear < 0) return bad("nsmear < 0");
  if (nsmear == 0) return QKX_OK;
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_smear_links(c));
  Tmp in(c->st), T(c->st);
  QKX_TRY(in.alloc(sizeof(double2) * gauge_words(c), "links"));
  QKX_TRY(T.alloc(sizeof(double2) * gauge_words(c), "APE scratch"));
  QKX_TRY(upload_links(c, U_in, in.d()));
  c->have_smear = 0;
  QKX_TRY(ape_run(c, in.d(), c->Usm, T.d(), nsmear, alpha));
  c->have_smear = 1;
  if (U_out) return download_links(c, c->Usm, U_out);
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

int qkx_load_smearing_gauge(qkx_ctx* c, const double* U_host) {
  if (!c || !U_host) return bad("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_smear_links(c));
  QKX_TRY(upload_links(c, U_host, c->Usm));
  c->have_smear = 1;
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

int qkx_gaussian_smear_dev(qkx_ctx* c, int nrhs, const double* const* in_dev, double* const* out_dev, int nsmear,
                           double alpha) {
  if (!c || !in_dev || !out_dev) return bad("NULL argument");
  if (nrhs < 1 || nrhs > MAX_RHS) return bad("nrhs must be in 1..64");
  if (nsmear < 0) return bad("nsmear < 0");
  for (int i = 0; i < nrhs; i++) {
    if (!in_dev[i] || !out_dev[i]) return bad("NULL field");
    for (int j = 0; j < nrhs; j++)
      if (in_dev[i] == out_dev[j]) return bad("an input field is also an output field");
  }
  if (nsmear == 0) return QKX_OK;
  if (!c->have_smear) {
    set_error("Gaussian smearing needs the smearing links (qkx_ape_smear or qkx_load_smearing_gauge)");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  Tmp tmp(c->st);
  QKX_TRY(tmp.alloc(sizeof(double2) * field_words(c) * nrhs, "smearing scratch"));
  FieldPtrs in{}, out{};
  for (int i = 0; i < nrhs; i++) {
    in.p[i] = (const double2*)in_dev[i];
    out.p[i] = (const double2*)out_dev[i];
  }
  return gauss_run(c, nrhs, in, out, batch_ptrs(tmp.d(), nrhs, field_words(c)), nsmear, alpha, 0, c->Vh);
}

int qkx_gaussian_smear(qkx_ctx* c, int nrhs, const double* const* in_host, double* const* out_host, int nsmear,
                       double alpha) {
  if (!c || !in_host || !out_host) return bad("NULL argument");
  if (nrhs < 1 || nrhs > MAX_RHS) return bad("nrhs must be in 1..64");
  if (nsmear < 0) return bad("nsmear < 0");
  for (int i = 0; i < nrhs; i++)
    if (!in_host[i] || !out_host[i]) return bad("NULL field");
  if (nsmear == 0) return QKX_OK;
  if (!c->have_smear) {
    set_error("Gaussian smearing needs the smearing links (qkx_ape_smear or qkx_load_smearing_gauge)");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  const size_t fw = field_words(c);
  Tmp bin(c->st), bout(c->st);
  QKX_TRY(bin.alloc(sizeof(double2) * fw * nrhs, "smearing inputs"));
  QKX_TRY(bout.alloc(sizeof(double2) * fw * nrhs, "smearing outputs"));
  for (int i = 0; i < nrhs; i++) QKX_TRY(upload_spinor(c, in_host[i], bin.d() + i * fw));
  std::vector<const double*> pi(nrhs);
  std::vector<double*> po(nrhs);
  for (int i = 0; i < nrhs; i++) {
    pi[i] = (const double*)(bin.d() + i * fw);
    po[i] = (double*)(bout.d() + i * fw);
  }
  QKX_TRY(qkx_gaussian_smear_dev(c, nrhs, pi.data(), po.data(), nsmear, alpha));
  for (int i = 0; i < nrhs; i++) QKX_TRY(download_spinor(c, bout.d() + i * fw, out_host[i]));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

int qkx_propagator_absorb(qkx_ctx* c, const double* phi_host, int nu, int c2, double* prop_host) {
  if (!c || !phi_host || !prop_host) return bad("NULL argument");
  if (nu < 0 || nu > 3 || c2 < 0 || c2 > 2) return bad("nu must be in 0..3 and c2 in 0..2");
  QKX_CUDA(cudaSetDevice(c->device));
  QKX_TRY(ensure_stage(c));
  QKX_CUDA(cudaMemcpyAsync(c->stage, phi_host, sizeof(double2) * field_words(c), cudaMemcpyHostToDevice, c->st));
  // element (mu, c1) of every site: a strided column of the staged vector
  // (site pitch 192 bytes) into a strided column of the propagator (2304 bytes)
  for (int mu = 0; mu < 4; mu++)
    for (int c1 = 0; c1 < 3; c1++)
      QKX_CUDA(cudaMemcpy2DAsync(prop_host + 2 * (mu * 36 + nu * 9 + c1 * 3 + c2), sizeof(double2) * 144,
                                 c->stage + (mu * 3 + c1), sizeof(double2) * 12, sizeof(double2), c->V,
                                 cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return QKX_OK;
}

int qkx_propagator_dev(qkx_ctx* c, const qkx_solver_params* sp, int nsmear, double alpha, const int x_src[4],
                       double* prop_dev, qkx_solve_info* info) {
  if (!c || !sp || !x_src || !prop_dev) return bad("NULL argument");
  if (nsmear < 0) return bad("nsmear < 0");
  for (int i = 0; i < 4; i++)
    if (x_src[i] < 0 || x_src[i] >= c->p.L[i]) return bad("source coordinate outside the lattice");
  if (!c->have_gauge) {
    set_error("the propagator needs a gauge field");
    return QKX_ERR_NOGAUGE;
  }
  if (nsmear > 0 && !c->have_smear) {
    set_error("smeared sources need the smearing links (qkx_ape_smear or qkx_load_smearing_gauge)");
    return QKX_ERR_NOGAUGE;
  }
  QKX_CUDA(cudaSetDevice(c->device));
  const size_t fw = field_words(c);
  Tmp S(c->st), X(c->st), T(c->st);
  QKX_TRY(S.alloc(sizeof(double2) * fw * 12, "sources"));
  QKX_TRY(X.alloc(sizeof(double2) * fw * 12, "smeared fields"));
  if (nsmear > 0) QKX_TRY(T.alloc(sizeof(double2) * fw * 12, "smearing scratch"));
  const FieldPtrs s = batch_ptrs(S.d(), 12, fw), x = batch_ptrs(X.d(), 12, fw);
  const FieldPtrs t = nsmear > 0 ? batch_ptrs(T.d(), 12, fw) : FieldPtrs{};

  // 12 unit point sources at x_src
  const int lex = x_src[0] + c->p.L[0] * (x_src[1] + c->p.L[1] * (x_src[2] + c->p.L[2] * x_src[3]));
  const int par = (x_src[0] + x_src[1] + x_src[2] + x_src[3]) & 1;
  QKX_CUDA(cudaMemsetAsync(S.p, 0, sizeof(double2) * fw * 12, c->st));
  k_point_sources<<<1, 32, 0, c->st>>>(s, c->Vh, par, lex >> 1);
  counted(c);
  QKX_CUDA(cudaGetLastError());

  // smeared sources in X: only the source's time slice is non-zero
  const FieldPtrs* b = &s;
  const FieldPtrs* sol = &x;
  if (nsmear > 0) {
    const int half_slice = c->p.L[0] * c->p.L[1] * c->p.L[2] / 2;
    QKX_CUDA(cudaMemsetAsync(X.p, 0, sizeof(double2) * fw * 12, c->st));
    QKX_TRY(gauss_run(c, 12, s, x, t, nsmear, alpha, x_src[3] * half_slice, half_slice));
    b = &x;
    sol = &s;
  }

  // M x = b for the 12 right-hand sides at once
  std::vector<const double*> bp(12);
  std::vector<double*> xp(12);
  for (int i = 0; i < 12; i++) {
    bp[i] = (const double*)b->p[i];
    xp[i] = (double*)sol->p[i];
  }
  const int rc = qkx_invert_dev(c, sp, 12, bp.data(), xp.data(), info);
  if (rc != QKX_OK && rc != QKX_ERR_NOT_CONVERGED) return rc;

  // smeared sinks, then the propagator columns
  const FieldPtrs* fin = sol;
  if (nsmear > 0) {
    QKX_TRY(gauss_run(c, 12, *sol, x, t, nsmear, alpha, 0, c->Vh));
    fin = &x;
  }
  const size_t n = c->V * 144;
  k_prop_assemble<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(*fin, (double2*)prop_dev, c->geom);
  counted(c);
  QKX_CUDA(cudaGetLastError());
  return rc;
}

int qkx_propagator(qkx_ctx* c, const qkx_solver_params* sp, int nsmear, double alpha, const int x_src[4],
                   double* prop_host, qkx_solve_info* info) {
  if (!c || !sp || !x_src || !prop_host) return bad("NULL argument");
  QKX_CUDA(cudaSetDevice(c->device));
  Tmp P(c->st);
  QKX_TRY(P.alloc(sizeof(double2) * c->V * 144, "propagator"));
  const int rc = qkx_propagator_dev(c, sp, nsmear, alpha, x_src, (double*)P.p, info);
  if (rc != QKX_OK && rc != QKX_ERR_NOT_CONVERGED) return rc;
  QKX_CUDA(cudaMemcpyAsync(prop_host, P.p, sizeof(double2) * c->V * 144, cudaMemcpyDeviceToHost, c->st));
  QKX_CUDA(cudaStreamSynchronize(c->st));
  return rc;
}

}  // extern "C"
