// qkxTM_b200.hpp -- header-only C++ layer over libqkx_b200 (include/qkx_b200.h)
// that keeps the reference's hot-path interface: the names, argument order
// and meaning of qkxTM::Vector / qkxTM::Gauge members (include/lattice_util.h),
// class CG (include/solvers.h) and the qkxTM BLAS (include/blas_qkxTM.h).
//
// Host fields keep the reference layout (Vector::M [V][4][3], Gauge::M
// [V][4][3][3] complex<double>), so driver code that fills or reads M keeps
// working.  Each Gauge owns one device context: the links go to the GPU on
// first use (and again after zero/copy/applyBoundaryCondition, or an explicit
// upload() after writing M directly).  Operators upload their input, run on
// the GPU and write the result into this->M.
//
// Error behaviour: the reference aborts the MPI job (errorQKXTM,
// include/qkxTM.h:137); here every failing library call throws
// qkxTM_b200::Error carrying the status code and message, which terminates the
// program the same way when not caught.
//
// Link with -lqkx_b200 (qkxtm_mpi_b200/libqkx_b200.so).
#ifndef QKXTM_B200_HPP
#define QKXTM_B200_HPP

#include <complex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "qkx_b200.h"

namespace qkxTM_b200 {

typedef std::complex<double> Complex;

// qkxTM::PARITY (include/lattice_util.h:22): EO/OE select the output parity of
// the parity-restricted hop, OO/EE the parity of the Schur operator.
enum PARITY { EO, OE, OO, EE };

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}
  int code;
};

inline void check(int rc) {
  if (rc != QKX_OK) throw Error(rc, std::string("qkx_b200: ") + qkx_last_error());
}

// struct LatticeInfo (include/qkxTM.h:156-204) with the reference's defaults.
// P, Nprocs and rank are kept for source compatibility; one GPU holds the lattice.
struct LatticeInfo {
  int L[4];
  int P[4];
  int x_src[4];
  int Nprocs;
  int rank;
  double kappa;
  double csw;
  double mu;
  int twistSign;
  double tol;
  double maxIter;
  double reliableDelta;
  int NsmearAPE;
  int NsmearGauss;
  double alphaAPE;
  double alphaGauss;
  int boundaryT;
  int Q_sq;
  int device;  // CUDA device of the contexts created with this LatticeInfo

  LatticeInfo()
      : Nprocs(1), rank(0), kappa(0.16), csw(1.57551), mu(0.008), twistSign(+1), tol(1e-1), maxIter(1000),
        reliableDelta(0.1), NsmearAPE(20), NsmearGauss(50), alphaAPE(0.5), alphaGauss(4.0), boundaryT(-1), Q_sq(0),
        device(0) {
    for (int i = 0; i < 4; i++) L[i] = P[i] = x_src[i] = 0;
  }

  qkx_params params() const {
    qkx_params p;
    for (int i = 0; i < 4; i++) p.L[i] = L[i];
    p.kappa = kappa;
    p.mu = mu;
    p.twistSign = twistSign;
    p.boundaryT = boundaryT;
    p.tol = tol;
    p.maxIter = (int)maxIter;
    p.reliableDelta = reliableDelta;
    return p;
  }
  long volume() const { return (long)L[0] * L[1] * L[2] * L[3]; }
};

namespace detail {
struct Ctx {
  qkx_ctx* c = nullptr;
  explicit Ctx(const LatticeInfo& li) {
    qkx_params p = li.params();
    check(qkx_create(&p, li.device, &c));
  }
  ~Ctx() { qkx_destroy(c); }
  Ctx(const Ctx&) = delete;
  Ctx& operator=(const Ctx&) = delete;
};
}  // namespace detail

class Gauge;

// qkxTM::Vector (include/lattice_util.h:80-156), hot-path members.
class Vector {
 public:
  long size, size_total, lV4d;
  Complex (*M)[4][3];

  explicit Vector(LatticeInfo* li) : info_(*li) {
    lV4d = size = size_total = li->volume();
    storage_.assign((size_t)lV4d * 12, Complex(0, 0));
    M = reinterpret_cast<Complex(*)[4][3]>(storage_.data());
  }
  virtual ~Vector() {}

  void zero() { std::fill(storage_.begin(), storage_.end(), Complex(0, 0)); }
  void copy(Vector& src) { std::memcpy(M, src.M, sizeof(Complex) * 12 * lV4d); }
  double norm2() const {
    double r = 0;
    for (const Complex& z : storage_) r += std::norm(z);
    return r;
  }
  double* data() { return reinterpret_cast<double*>(storage_.data()); }
  const LatticeInfo& info() const { return info_; }
  const double* data() const { return reinterpret_cast<const double*>(storage_.data()); }

  // lib/lattice_util.cpp:1158 applyDslash, :1643 applyDslashDag, :1215 applyDslash_chiral
  void applyDslash(Vector& psi, Gauge& u);
  void applyDslashDag(Vector& psi, Gauge& u);
  void applyDslash_chiral(Vector& psi, Gauge& u);
  // :1272 applyDslash_xx (EO: output even, OE: output odd), :1346 chiral
  void applyDslash_xx(Vector& psi, Gauge& u, PARITY parity);
  void applyDslash_xx_chiral(Vector& psi, Gauge& u, PARITY parity);
  // site operators :1563-1820
  void applyTwist(Vector& psi, LatticeInfo* li) { site(QKX_OP_TWIST, psi, li); }
  void applyTwistInv(Vector& psi, LatticeInfo* li) { site(QKX_OP_TWIST_INV, psi, li); }
  void applyTwistDag(Vector& psi, LatticeInfo* li) { site(QKX_OP_TWIST_DAG, psi, li); }
  void applyTwistDagInv(Vector& psi, LatticeInfo* li) { site(QKX_OP_TWIST_DAG_INV, psi, li); }
  void applyTwistInv_chiral(Vector& psi, LatticeInfo* li) { site(QKX_OP_TWIST_INV_CHIRAL, psi, li); }
  void applyGamma5(Vector& psi, LatticeInfo* li) { site(QKX_OP_GAMMA5, psi, li); }
  void applyGamma5_chiral(Vector& psi, LatticeInfo* li) { site(QKX_OP_GAMMA5_CHIRAL, psi, li); }
  void rotateFromChiralToUKQCD() { site(QKX_OP_ROTATE_CHIRAL_TO_UKQCD, *this, &info_); }
  // composite operators :1925-2071
  void tm(Vector& psi, Gauge& u, LatticeInfo* li);
  void tm_chiral(Vector& psi, Gauge& u, LatticeInfo* li);
  void tmDag(Vector& psi, Gauge& u, LatticeInfo* li);
  void tmDagtm(Vector& psi, Vector& vec_tmp, Gauge& u, LatticeInfo* li);
  void Wilson(Vector& psi, Gauge& u, LatticeInfo* li);
  void tm_xx(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity);
  void tm_xxDagTm_xx(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity);
  void tm_xx_chiral(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity);
  void tm_xxDagTm_xx_chiral(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity);

  // lib/lattice_util.cpp:1080-1145: *this = nsmear Gaussian smearing steps of
  // vec_tmp with the links of gauge (li->NsmearGauss, li->alphaGauss).  vec_tmp
  // is left unchanged (the reference overwrites it); nsmear == 0 leaves *this.
  void Gaussian_smearing(Vector& vec_tmp, Gauge& gauge, LatticeInfo* li);

 private:
  friend class Gauge;
  void site(int op, Vector& psi, LatticeInfo* li);
  LatticeInfo info_;
  std::vector<Complex> storage_;
};

// qkxTM::Gauge (include/lattice_util.h:186-212), hot-path members.
class Gauge {
 public:
  long size, size_total, lV4d;
  bool constGauge;
  Complex (*M)[4][3][3];

  explicit Gauge(LatticeInfo* li) : constGauge(false), info_(*li), ctx_(new detail::Ctx(*li)) {
    lV4d = size = size_total = li->volume();
    storage_.assign((size_t)lV4d * 36, Complex(0, 0));
    M = reinterpret_cast<Complex(*)[4][3][3]>(storage_.data());
  }
  virtual ~Gauge() {}

  void zero() {
    std::fill(storage_.begin(), storage_.end(), Complex(0, 0));
    dirty_ = smear_dirty_ = true;
  }
  void copy(Gauge& src) {
    std::memcpy(M, src.M, sizeof(Complex) * 36 * lV4d);
    dirty_ = smear_dirty_ = true;
  }
  // lib/lattice_util.cpp:708-724: t-links on the last time slice change sign when boundaryT == -1
  void applyBoundaryCondition(LatticeInfo* li) {
    if (li->boundaryT != -1) return;
    const long V3 = (long)li->L[0] * li->L[1] * li->L[2];
    for (long iv = lV4d - V3; iv < lV4d; iv++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) M[iv][3][a][b] = -M[iv][3][a][b];
    dirty_ = smear_dirty_ = true;
  }
  // push M to the device now (needed after writing M directly once the field was used)
  void upload() {
    check(qkx_load_gauge(ctx_->c, reinterpret_cast<const double*>(storage_.data()), QKX_LINKS_AS_GIVEN));
    dirty_ = false;
    smear_dirty_ = true;
  }

  // lib/lattice_util.cpp:923-946, on the GPU
  double calculatePlaquette() {
    double r = 0;
    check(qkx_plaquette_loaded(ctx(&info_), QKX_LINKS_OPERATOR, &r));
    return r;
  }
  // lib/lattice_util.cpp:948-1078: *this = APE smearing of U_tmp (li->NsmearAPE,
  // li->alphaAPE), spatial links projected to SU(3), t-links of U_tmp.  U_tmp is
  // left unchanged (the reference overwrites it); nsmear == 0 leaves *this.
  void APE_smearing(Gauge& U_tmp, LatticeInfo* li) {
    if (li->NsmearAPE == 0) return;
    check(qkx_ape_smear(ctx_->c, U_tmp.data(), data(), li->NsmearAPE, li->alphaAPE));
    dirty_ = true;          // operator links are re-uploaded on next use
    smear_dirty_ = false;   // the context's smearing links are this result
  }
  // the library context with M as its smearing links (for Gaussian smearing)
  qkx_ctx* smear_ctx() {
    if (smear_dirty_) {
      check(qkx_load_smearing_gauge(ctx_->c, data()));
      smear_dirty_ = false;
    }
    return ctx_->c;
  }
  double* data() { return reinterpret_cast<double*>(storage_.data()); }
  // the library context of this gauge field, with the parameters of li
  qkx_ctx* ctx(const LatticeInfo* li) {
    if (dirty_) upload();
    qkx_params p = li->params();
    check(qkx_set_params(ctx_->c, &p));
    return ctx_->c;
  }
  const LatticeInfo& info() const { return info_; }
  // M was written outside the class: upload it again before the next use
  void mark_modified() { dirty_ = smear_dirty_ = true; }

 private:
  LatticeInfo info_;
  std::unique_ptr<detail::Ctx> ctx_;
  std::vector<Complex> storage_;
  bool dirty_ = true;
  bool smear_dirty_ = true;
};

// ---- Vector members that need a gauge field
inline void Vector::applyDslash(Vector& psi, Gauge& u) {
  check(qkx_apply(u.ctx(&info_), QKX_OP_DSLASH, psi.data(), data()));
}
inline void Vector::applyDslashDag(Vector& psi, Gauge& u) {
  check(qkx_apply(u.ctx(&info_), QKX_OP_DSLASH_DAG, psi.data(), data()));
}
inline void Vector::applyDslash_chiral(Vector& psi, Gauge& u) {
  check(qkx_apply(u.ctx(&info_), QKX_OP_DSLASH_CHIRAL, psi.data(), data()));
}
inline void Vector::applyDslash_xx(Vector& psi, Gauge& u, PARITY parity) {
  if (parity != EO && parity != OE) throw Error(QKX_ERR_INVALID, "Error wrong parity for hopping term");
  check(qkx_apply(u.ctx(&info_), parity == EO ? QKX_OP_DSLASH_XX_EO : QKX_OP_DSLASH_XX_OE, psi.data(), data()));
}
inline void Vector::applyDslash_xx_chiral(Vector& psi, Gauge& u, PARITY parity) {
  if (parity != EO && parity != OE) throw Error(QKX_ERR_INVALID, "Error wrong parity for hopping term");
  check(qkx_apply(u.ctx(&info_), parity == EO ? QKX_OP_DSLASH_XX_CHIRAL_EO : QKX_OP_DSLASH_XX_CHIRAL_OE,
                  psi.data(), data()));
}
inline void Vector::tm(Vector& psi, Gauge& u, LatticeInfo* li) {
  check(qkx_apply(u.ctx(li), QKX_OP_TM, psi.data(), data()));
}
inline void Vector::tm_chiral(Vector& psi, Gauge& u, LatticeInfo* li) {
  check(qkx_apply(u.ctx(li), QKX_OP_TM_CHIRAL, psi.data(), data()));
}
inline void Vector::tmDag(Vector& psi, Gauge& u, LatticeInfo* li) {
  check(qkx_apply(u.ctx(li), QKX_OP_TM_DAG, psi.data(), data()));
}
inline void Vector::tmDagtm(Vector& psi, Vector& vec_tmp, Gauge& u, LatticeInfo* li) {
  (void)vec_tmp;  // the library keeps its own device temporary
  check(qkx_apply(u.ctx(li), QKX_OP_TM_DAGTM, psi.data(), data()));
}
inline void Vector::Wilson(Vector& psi, Gauge& u, LatticeInfo* li) {
  check(qkx_apply(u.ctx(li), QKX_OP_WILSON, psi.data(), data()));
}
inline void Vector::tm_xx(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity) {
  if (parity != EE && parity != OO) throw Error(QKX_ERR_INVALID, "Error wrong parity choise");
  check(qkx_apply(u.ctx(li), parity == EE ? QKX_OP_TM_XX_EE : QKX_OP_TM_XX_OO, psi.data(), data()));
}
inline void Vector::tm_xxDagTm_xx(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity) {
  if (parity != EE && parity != OO) throw Error(QKX_ERR_INVALID, "Error wrong parity choise");
  check(qkx_apply(u.ctx(li), parity == EE ? QKX_OP_TM_XX_DAGTM_XX_EE : QKX_OP_TM_XX_DAGTM_XX_OO, psi.data(),
                  data()));
}
inline void Vector::tm_xx_chiral(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity) {
  if (parity != EE && parity != OO) throw Error(QKX_ERR_INVALID, "Error wrong parity choise");
  check(qkx_apply(u.ctx(li), parity == EE ? QKX_OP_TM_XX_CHIRAL_EE : QKX_OP_TM_XX_CHIRAL_OO, psi.data(), data()));
}
inline void Vector::tm_xxDagTm_xx_chiral(Vector& psi, Gauge& u, LatticeInfo* li, PARITY parity) {
  if (parity != EE && parity != OO) throw Error(QKX_ERR_INVALID, "Error wrong parity choise");
  check(qkx_apply(u.ctx(li), parity == EE ? QKX_OP_TM_XX_DAGTM_XX_CHIRAL_EE : QKX_OP_TM_XX_DAGTM_XX_CHIRAL_OO,
                  psi.data(), data()));
}

namespace detail {
// a gauge-less context per lattice shape for the site operators and the BLAS
inline qkx_ctx* plain_ctx(const LatticeInfo& li) {
  static std::vector<std::unique_ptr<Ctx>> pool;
  static std::vector<LatticeInfo> keys;
  for (size_t i = 0; i < keys.size(); i++)
    if (std::memcmp(keys[i].L, li.L, sizeof li.L) == 0 && keys[i].device == li.device) {
      qkx_params p = li.params();
      check(qkx_set_params(pool[i]->c, &p));
      return pool[i]->c;
    }
  pool.emplace_back(new Ctx(li));
  keys.push_back(li);
  return pool.back()->c;
}

// a device copy of a host Vector for the BLAS
struct DevField {
  qkx_ctx* c;
  double* p;
  DevField(qkx_ctx* c, const Vector& v) : c(c), p((double*)qkx_device_alloc(c, qkx_spinor_bytes(c))) {
    if (!p) throw Error(QKX_ERR_NOMEM, "qkx_b200: device allocation failed");
    check(qkx_spinor_upload(c, v.data(), p));
  }
  ~DevField() { qkx_device_free(c, p); }
};
}  // namespace detail

inline void Vector::site(int op, Vector& psi, LatticeInfo* li) {
  check(qkx_apply(detail::plain_ctx(*li), op, psi.data(), data()));
}

// ---- qkxTM BLAS (lib/blas_qkxTM.cpp:4-56 and Vector::norm2), on the GPU,
// with the reference's signatures
inline double reCdotXdagY(Vector& x, Vector& y) {
  qkx_ctx* c = detail::plain_ctx(x.info());
  detail::DevField dx(c, x), dy(c, y);
  double r = 0;
  check(qkx_reCdotXdagY(c, dx.p, dy.p, &r));
  return r;
}
inline void X_eq_X_p_aY(Vector& x, double a, Vector& y) {
  qkx_ctx* c = detail::plain_ctx(x.info());
  detail::DevField dx(c, x), dy(c, y);
  check(qkx_X_eq_X_p_aY(c, dx.p, a, dy.p));
  check(qkx_spinor_download(c, dx.p, x.data()));
}
inline void X_eq_aX_p_Y(Vector& x, double a, Vector& y) {
  qkx_ctx* c = detail::plain_ctx(x.info());
  detail::DevField dx(c, x), dy(c, y);
  check(qkx_X_eq_aX_p_Y(c, dx.p, a, dy.p));
  check(qkx_spinor_download(c, dx.p, x.data()));
}

inline void Vector::Gaussian_smearing(Vector& vec_tmp, Gauge& gauge, LatticeInfo* li) {
  if (li->NsmearGauss == 0) return;
  const double* in[1] = {vec_tmp.data()};
  double* out[1] = {data()};
  check(qkx_gaussian_smear(gauge.smear_ctx(), 1, in, out, li->NsmearGauss, li->alphaGauss));
}

// qkxTM::Propagator (include/lattice_util.h:158-183), hot-path members.
class Propagator {
 public:
  long size, size_total, lV4d;
  Complex (*M)[4][4][3][3];

  explicit Propagator(LatticeInfo* li) : info_(*li) {
    lV4d = size = size_total = li->volume();
    storage_.assign((size_t)lV4d * 144, Complex(0, 0));
    M = reinterpret_cast<Complex(*)[4][4][3][3]>(storage_.data());
  }
  virtual ~Propagator() {}
  void zero() { std::fill(storage_.begin(), storage_.end(), Complex(0, 0)); }
  void copy(Propagator& src) { std::memcpy(M, src.M, sizeof(Complex) * 144 * lV4d); }
  // lib/lattice_util.cpp:2073-2081: M[x][mu][nu][c1][c2] = phi.M[x][mu][c1],
  // moved by the GPU's copy engines
  void absorbVector(Vector& phi, int nu, int c2) {
    check(qkx_propagator_absorb(detail::plain_ctx(info_), phi.data(), nu, c2, data()));
  }
  double* data() { return reinterpret_cast<double*>(storage_.data()); }
  const LatticeInfo& info() const { return info_; }

 private:
  LatticeInfo info_;
  std::vector<Complex> storage_;
};

// ---- ILDG configurations (lib/read_conf_lime.cpp:111, lib/write_conf_lime.cpp:49)
// qkxTM_MPI_getGaugeLime: fill u.M from an ILDG file (read and byte-swapped on the GPU).
inline int qkxTM_MPI_getGaugeLime(char* fname, Gauge& u) {
  check(qkx_read_gauge_lime(detail::plain_ctx(u.info()), fname, QKX_LINKS_AS_GIVEN, u.data(), nullptr));
  u.mark_modified();
  return 0;
}
// qkxTM_writeGaugeLime: write u.M as an ILDG file with message as its xlf-info record.
inline int qkxTM_writeGaugeLime(char* fname, Gauge& u, char* message) {
  check(qkx_write_gauge_lime(detail::plain_ctx(u.info()), fname, u.data(), message));
  return 0;
}

// ---- two-point functions (lib/contractions.cpp:873-914), on the GPU, written
// in the reference's text format (Meson::dumpData :149, Baryon::dumpData :641)
inline void contractMesons(Propagator* prop1, Propagator* prop2, char* twop_filename, LatticeInfo* latInfo) {
  qkx_ctx* c = detail::plain_ctx(*latInfo);
  const int nmom = qkx_momenta(latInfo->Q_sq, nullptr, 0);
  std::vector<int> mom((size_t)3 * nmom);
  qkx_momenta(latInfo->Q_sq, mom.data(), nmom);
  const int ops[QKX_NUM_MESONS] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9};
  const int Lt = latInfo->L[3];
  std::vector<double> F((size_t)QKX_NUM_MESONS * Lt * nmom * 2);
  FILE* f = std::fopen(twop_filename, "w");
  if (!f) throw Error(QKX_ERR_INVALID, "qkx_b200: cannot open the meson output file");
  for (Propagator* p : {prop1, prop2}) {
    check(qkx_meson_2pt(c, p->data(), QKX_NUM_MESONS, ops, latInfo->Q_sq, latInfo->x_src, F.data()));
    for (int op = 0; op < QKX_NUM_MESONS; op++)
      for (int t = 0; t < Lt; t++)
        for (int im = 0; im < nmom; im++) {
          const double* v = &F[(((size_t)op * Lt + t) * nmom + im) * 2];
          std::fprintf(f, "%d \t %d \t %+d %+d %+d \t %+e %+e\n", op, t, mom[3 * im], mom[3 * im + 1],
                       mom[3 * im + 2], v[0], v[1]);
        }
  }
  std::fclose(f);
}

inline void contractBaryons(Propagator* prop1, Propagator* prop2, char* twop_filename, LatticeInfo* latInfo) {
  qkx_ctx* c = detail::plain_ctx(*latInfo);
  const int nmom = qkx_momenta(latInfo->Q_sq, nullptr, 0);
  std::vector<int> mom((size_t)3 * nmom);
  qkx_momenta(latInfo->Q_sq, mom.data(), nmom);
  const int Lt = latInfo->L[3];
  std::vector<double> F((size_t)Lt * nmom * 16 * 2);
  FILE* f = std::fopen(twop_filename, "w");
  if (!f) throw Error(QKX_ERR_INVALID, "qkx_b200: cannot open the baryon output file");
  Propagator* pairs[2][2] = {{prop1, prop2}, {prop2, prop1}};
  for (auto& pr : pairs)
    for (int op = 0; op < 4; op++) {
      check(qkx_baryon_2pt(c, pr[0]->data(), pr[1]->data(), op, latInfo->Q_sq, latInfo->x_src, F.data()));
      for (int t = 0; t < Lt; t++)
        for (int im = 0; im < nmom; im++)
          for (int g = 0; g < 4; g++)
            for (int gp = 0; gp < 4; gp++) {
              const double* v = &F[((((size_t)t * nmom + im) * 4 + g) * 4 + gp) * 2];
              std::fprintf(f, "%d \t %d \t %+d %+d %+d \t %d %d \t %+e %+e\n", op, t, mom[3 * im],
                           mom[3 * im + 1], mom[3 * im + 2], g, gp, v[0], v[1]);
            }
    }
  std::fclose(f);
}

// contractBaryonsDec (lib/contractions.cpp:916-936): DELTA_ISO1 and DELTA_ISO1O2 for (prop1, prop2)
// then (prop2, prop1), in Baryon_Dec::dumpData's text format (:869)
inline void contractBaryonsDec(Propagator* prop1, Propagator* prop2, char* twop_filename, LatticeInfo* latInfo) {
  qkx_ctx* c = detail::plain_ctx(*latInfo);
  const int nmom = qkx_momenta(latInfo->Q_sq, nullptr, 0);
  std::vector<int> mom((size_t)3 * nmom);
  qkx_momenta(latInfo->Q_sq, mom.data(), nmom);
  const int Lt = latInfo->L[3];
  std::vector<double> F((size_t)Lt * nmom * 48 * 2);
  FILE* f = std::fopen(twop_filename, "w");
  if (!f) throw Error(QKX_ERR_INVALID, "qkx_b200: cannot open the decuplet output file");
  Propagator* pairs[2][2] = {{prop1, prop2}, {prop2, prop1}};
  for (auto& pr : pairs)
    for (int op = 0; op < 2; op++) {
      check(qkx_delta_2pt(c, pr[0]->data(), pr[1]->data(), op, latInfo->Q_sq, latInfo->x_src, F.data()));
      for (int t = 0; t < Lt; t++)
        for (int im = 0; im < nmom; im++)
          for (int i = 0; i < 3; i++)
            for (int g = 0; g < 4; g++)
              for (int gp = 0; gp < 4; gp++) {
                const double* v = &F[(((((size_t)t * nmom + im) * 3 + i) * 4 + g) * 4 + gp) * 2];
                std::fprintf(f, "%d \t %d \t %+d %+d %+d \t %d \t %d %d \t %+e %+e\n", op, t, mom[3 * im],
                             mom[3 * im + 1], mom[3 * im + 2], i, g, gp, v[0], v[1]);
              }
    }
  std::fclose(f);
}

// contractNucleon (lib/lattice_util.cpp:3374): the nucleon correlator of (prop1, prop2), per time
// slice in that function's text format
inline void contractNucleon(Propagator& prop1, Propagator& prop2, char* output, int Q_sq, int x_src[4]) {
  qkx_ctx* c = detail::plain_ctx(prop1.info());
  const int nmom = qkx_momenta(Q_sq, nullptr, 0);
  std::vector<int> mom((size_t)3 * nmom);
  qkx_momenta(Q_sq, mom.data(), nmom);
  const int Lt = prop1.info().L[3];
  std::vector<double> F((size_t)Lt * nmom * 16 * 2);
  check(qkx_nucleon_2pt(c, prop1.data(), prop2.data(), Q_sq, x_src, F.data()));
  FILE* f = std::fopen(output, "w");
  if (!f) throw Error(QKX_ERR_INVALID, "qkx_b200: cannot open the nucleon output file");
  for (int t = 0; t < Lt; t++)
    for (int im = 0; im < nmom; im++)
      for (int g = 0; g < 4; g++)
        for (int g1 = 0; g1 < 4; g1++) {
          const double* v = &F[((((size_t)t * nmom + im) * 4 + g) * 4 + g1) * 2];
          std::fprintf(f, "%d   %+d %+d %+d   %d %d  \t %+e %+e\n", t, mom[3 * im], mom[3 * im + 1], mom[3 * im + 2],
                       g, g1, v[0], v[1]);
        }
  std::fclose(f);
}

// ---- class CG (include/solvers.h:3-22, lib/solvers.cpp)
class CG {
 public:
  CG(LatticeInfo* param, Gauge& gauge)
      : maxIter_((int)param->maxIter), tol_(param->tol), reliableDelta_(param->reliableDelta), u_(gauge) {}
  int MaxIter() { return maxIter_; }
  double Tol() { return tol_; }
  double ReliableDelta() { return reliableDelta_; }

  // CG::operator()(out, in, param): solves M^+M out = in with the reference's
  // algorithm and stopping rule; adds the solution to out, as the reference does.
  // Reaching maxIter is not an error (the reference only prints a warning).
  qkx_solve_info operator()(Vector& out, Vector& in, LatticeInfo* param) {
    qkx_solve_info info;
    int rc = qkx_cg(u_.ctx(param), in.data(), out.data(), &info);
    if (rc != QKX_ERR_NOT_CONVERGED) check(rc);
    return info;
  }

  // B200 solve of M x_i = b_i to ||b - M x|| / ||b|| <= tol for a batch of
  // right-hand sides (no reference counterpart; replaces tmDag + CG of
  // bin/test_invert.cpp:95-117 and the 12 sequential solves of
  // bin/test_invert_prop.cpp:72-96).
  qkx_solve_info invert(std::vector<Vector*>& b, std::vector<Vector*>& x, LatticeInfo* param,
                        int method = QKX_SOLVER_CG_EO_MIXED, int precision = QKX_PREC_HALF, double tol = 1e-10) {
    std::vector<const double*> bp;
    std::vector<double*> xp;
    for (Vector* v : b) bp.push_back(v->data());
    for (Vector* v : x) xp.push_back(v->data());
    qkx_solver_params sp;
    sp.method = method;
    sp.sloppy_precision = precision;
    sp.tol = tol;
    sp.maxIter = 100000;
    sp.reliable_delta = 0.0;
    sp.use_graphs = 1;
    sp.mu = nullptr;
    sp.preconditioner = nullptr;
    qkx_solve_info info;
    check(qkx_invert(u_.ctx(param), &sp, (int)bp.size(), bp.data(), xp.data(), &info));
    return info;
  }

  // B200 smeared-source propagator (no reference counterpart; replaces the
  // loop of bin/test_invert_prop.cpp:83-97): 12 point sources at
  // param->x_src, Gaussian smearing with the links of smear_gauge
  // (param->NsmearGauss, param->alphaGauss) at source and sink, one batched
  // solve, the columns assembled into prop.
  qkx_solve_info propagator(Propagator& prop, Gauge& smear_gauge, LatticeInfo* param,
                            int method = QKX_SOLVER_CG_EO_MIXED, int precision = QKX_PREC_HALF, double tol = 1e-10) {
    qkx_ctx* c = u_.ctx(param);
    if (param->NsmearGauss > 0) check(qkx_load_smearing_gauge(c, smear_gauge.data()));
    qkx_solver_params sp;
    sp.method = method;
    sp.sloppy_precision = precision;
    sp.tol = tol;
    sp.maxIter = 100000;
    sp.reliable_delta = 0.0;
    sp.use_graphs = 1;
    sp.mu = nullptr;
    sp.preconditioner = nullptr;
    qkx_solve_info info;
    check(qkx_propagator(c, &sp, param->NsmearGauss, param->alphaGauss, param->x_src, prop.data(), &info));
    return info;
  }

 private:
  int maxIter_;
  double tol_;
  double reliableDelta_;
  Gauge& u_;
};

}  // namespace qkxTM_b200

#endif
