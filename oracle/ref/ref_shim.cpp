/*
 * ref_shim.cpp -- C entry points around the reference's own classes, compiled
 * together with the unmodified reference sources into oracle/_ref/libqkxref.so.
 * TEST INFRASTRUCTURE ONLY: it lets the tests run the reference's Vector::tm,
 * tm_xx, chiral variants, BLAS, CG::operator(), the plaquette, APE and
 * Gaussian smearing, Propagator::absorbVector and the propagator loop of
 * bin/test_invert_prop.cpp on plain arrays so the CPU
 * restatement (oracle/qkx_oracle.c) and the golden vectors are pinned to the
 * reference itself.  Single rank, P = (1,1,1,1), the MPI calls go to ref/mpi.h.
 *
 * Arrays use the reference layouts: spinor Vector::M [V][4][3] complex,
 * gauge Gauge::M [V][4][3][3] complex (include/lattice_util.h:90, 198).
 */
#include <qkxTM.h>
#include <lattice_util.h>
#include <blas_qkxTM.h>
#include <solvers.h>

#include <fcntl.h>
#include <unistd.h>

using namespace qkxTM;

namespace {

LatticeInfo make_info(const int L[4], double kappa, double mu, int twistSign, int boundaryT,
                      double tol, int maxIter) {
  LatticeInfo li;
  for (int i = 0; i < 4; i++) {
    li.L[i] = L[i];
    li.P[i] = 1;
  }
  li.Nprocs = 1;
  li.rank = 0;
  li.kappa = kappa;
  li.mu = mu;
  li.twistSign = twistSign;
  li.boundaryT = boundaryT;
  li.tol = tol;
  li.maxIter = maxIter;
  return li;
}

long volume(const int L[4]) { return (long)L[0] * L[1] * L[2] * L[3]; }

void load_vec(Vector& v, const double* a) {
  memcpy(&(v.M[0][0][0]), a, sizeof(double) * 24 * v.lV4d);
}
void store_vec(const Vector& v, double* a) {
  memcpy(a, &(v.M[0][0][0]), sizeof(double) * 24 * v.lV4d);
}

/* silence the reference's per-iteration prints (lib/solvers.cpp:49) */
struct QuietStdout {
  int saved;
  QuietStdout() {
    fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    dup2(devnull, 1);
    close(devnull);
  }
  ~QuietStdout() {
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

}  // namespace

extern "C" {

enum {
  REF_DSLASH = 0,
  REF_DSLASH_DAG = 1,
  REF_TM = 2,
  REF_TM_DAG = 3,
  REF_TM_DAGTM = 4,
  REF_WILSON = 5,
  REF_TM_XX_EE = 6,
  REF_TM_XX_OO = 7,
  REF_TM_XX_DAGTM_XX_EE = 8,
  REF_TM_XX_DAGTM_XX_OO = 9,
  REF_DSLASH_CHIRAL = 10,
  REF_TM_CHIRAL = 11,
  REF_TM_XX_CHIRAL_EE = 12,
  REF_TM_XX_CHIRAL_OO = 13,
  REF_TM_XX_DAGTM_XX_CHIRAL_EE = 14,
  REF_TM_XX_DAGTM_XX_CHIRAL_OO = 15,
  REF_GAMMA5 = 16,
  REF_GAMMA5_CHIRAL = 17,
  REF_TWIST = 18,
  REF_TWIST_INV = 19,
  REF_TWIST_DAG = 20,
  REF_TWIST_DAG_INV = 21,
  REF_TWIST_INV_CHIRAL = 22,
  REF_DSLASH_XX_EO = 23,
  REF_DSLASH_XX_OE = 24,
  REF_ROTATE_CHIRAL_TO_UKQCD = 25,
  REF_DSLASH_XX_CHIRAL_EO = 26,
  REF_DSLASH_XX_CHIRAL_OE = 27,
  REF_NUM_OPS = 28
};

int ref_num_ops(void) { return REF_NUM_OPS; }

/* Apply one reference operator: out = op(in).  Returns 0, or -1 for an unknown op. */
int ref_apply(int op, const int L[4], double kappa, double mu, int twistSign, const double* U,
              const double* in, double* out) {
  LatticeInfo li = make_info(L, kappa, mu, twistSign, -1, 1e-10, 1000);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  Vector psi(&li), res(&li), tmp(&li);
  load_vec(psi, in);
  res.zero();
  tmp.zero();
  switch (op) {
    case REF_DSLASH: res.applyDslash(psi, u); break;
    case REF_DSLASH_DAG: res.applyDslashDag(psi, u); break;
    case REF_TM: res.tm(psi, u, &li); break;
    case REF_TM_DAG: res.tmDag(psi, u, &li); break;
    case REF_TM_DAGTM: res.tmDagtm(psi, tmp, u, &li); break;
    case REF_WILSON: res.Wilson(psi, u, &li); break;
    case REF_TM_XX_EE: res.tm_xx(psi, u, &li, EE); break;
    case REF_TM_XX_OO: res.tm_xx(psi, u, &li, OO); break;
    case REF_TM_XX_DAGTM_XX_EE: res.tm_xxDagTm_xx(psi, u, &li, EE); break;
    case REF_TM_XX_DAGTM_XX_OO: res.tm_xxDagTm_xx(psi, u, &li, OO); break;
    case REF_DSLASH_CHIRAL: res.applyDslash_chiral(psi, u); break;
    case REF_TM_CHIRAL: res.tm_chiral(psi, u, &li); break;
    case REF_TM_XX_CHIRAL_EE: res.tm_xx_chiral(psi, u, &li, EE); break;
    case REF_TM_XX_CHIRAL_OO: res.tm_xx_chiral(psi, u, &li, OO); break;
    case REF_TM_XX_DAGTM_XX_CHIRAL_EE: res.tm_xxDagTm_xx_chiral(psi, u, &li, EE); break;
    case REF_TM_XX_DAGTM_XX_CHIRAL_OO: res.tm_xxDagTm_xx_chiral(psi, u, &li, OO); break;
    case REF_GAMMA5: res.applyGamma5(psi, &li); break;
    case REF_GAMMA5_CHIRAL: res.applyGamma5_chiral(psi, &li); break;
    case REF_TWIST: res.applyTwist(psi, &li); break;
    case REF_TWIST_INV: res.applyTwistInv(psi, &li); break;
    case REF_TWIST_DAG: res.applyTwistDag(psi, &li); break;
    case REF_TWIST_DAG_INV: res.applyTwistDagInv(psi, &li); break;
    case REF_TWIST_INV_CHIRAL: res.applyTwistInv_chiral(psi, &li); break;
    case REF_DSLASH_XX_EO: res.applyDslash_xx(psi, u, EO); break;
    case REF_DSLASH_XX_OE: res.applyDslash_xx(psi, u, OE); break;
    case REF_ROTATE_CHIRAL_TO_UKQCD:
      res.copy(psi);
      res.rotateFromChiralToUKQCD();
      break;
    case REF_DSLASH_XX_CHIRAL_EO: res.applyDslash_xx_chiral(psi, u, EO); break;
    case REF_DSLASH_XX_CHIRAL_OE: res.applyDslash_xx_chiral(psi, u, OE); break;
    default: return -1;
  }
  store_vec(res, out);
  return 0;
}

/* Gauge::applyBoundaryCondition on a plain array. */
void ref_apply_bc(const int L[4], int boundaryT, double* U) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, boundaryT, 1e-10, 1000);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  {
    QuietStdout q;
    u.applyBoundaryCondition(&li);
  }
  memcpy(U, &(u.M[0][0][0][0]), sizeof(double) * 72 * volume(L));
}

/* BLAS of lib/blas_qkxTM.cpp on plain arrays.  which: 0 reCdotXdagY(x,y),
 * 1 X_eq_X_p_aY (x updated), 2 X_eq_aX_p_Y (x updated), 3 Vector::norm2(x). */
double ref_blas(int which, const int L[4], double a, double* x, const double* y) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Vector vx(&li), vy(&li);
  load_vec(vx, x);
  load_vec(vy, y);
  double r = 0;
  switch (which) {
    case 0: r = reCdotXdagY(vx, vy); break;
    case 1: X_eq_X_p_aY(vx, a, vy); break;
    case 2: X_eq_aX_p_Y(vx, a, vy); break;
    case 3: r = vx.norm2(); break;
  }
  store_vec(vx, x);
  return r;
}

/* CG::operator()(out, in) with the links as given (the caller applies the
 * boundary condition beforehand, as bin/test_invert.cpp:106 does).  x is both
 * the initial content of `out` and the result. */
void ref_cg(const int L[4], double kappa, double mu, int twistSign, double tol, int maxIter,
            const double* U, const double* in, double* x) {
  LatticeInfo li = make_info(L, kappa, mu, twistSign, -1, tol, maxIter);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  u.constGauge = true;
  Vector vin(&li), vout(&li);
  load_vec(vin, in);
  load_vec(vout, x);
  {
    QuietStdout q;
    CG cg(&li, u);
    cg(vout, vin, &li);
  }
  store_vec(vout, x);
}

/* CG::operator() as above, returning the wall seconds of the solver call
 * alone (set-up and copies excluded).  Used for the timed CPU baseline with
 * maxIter set to a bounded number of iterations. */
double ref_cg_timed(const int L[4], double kappa, double mu, int twistSign, double tol, int maxIter,
                    const double* U, const double* in, double* x) {
  LatticeInfo li = make_info(L, kappa, mu, twistSign, -1, tol, maxIter);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  u.constGauge = true;
  Vector vin(&li), vout(&li);
  load_vec(vin, in);
  load_vec(vout, x);
  double t0, t1;
  {
    QuietStdout q;
    CG cg(&li, u);
    t0 = MPI_Wtime();
    cg(vout, vin, &li);
    t1 = MPI_Wtime();
  }
  store_vec(vout, x);
  return t1 - t0;
}

/* qkxTM_MPI_getGaugeLime (lib/read_conf_lime.cpp:111-245): the links of an ILDG file into U.
 * Returns the reference's status (0). */
int ref_read_gauge_lime(const char* path, const int L[4], double* U) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Gauge u(&li);
  const int rc = qkxTM_MPI_getGaugeLime(const_cast<char*>(path), u);
  memcpy(U, &(u.M[0][0][0][0]), sizeof(double) * 72 * volume(L));
  return rc;
}

/* qkxTM_writeGaugeLime (lib/write_conf_lime.cpp:49-199): U as an ILDG file with the message as
 * its xlf-info record.  Returns the reference's status (0). */
int ref_write_gauge_lime(const char* path, const int L[4], const double* U, const char* message) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  return qkxTM_writeGaugeLime(const_cast<char*>(path), u, const_cast<char*>(message));
}

/* Gauge::calculatePlaquette (lib/lattice_util.cpp:923) of the links as given. */
double ref_plaquette(const int L[4], const double* U) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  return u.calculatePlaquette();
}

/* qcd_projectSU33d (lib/blas.cpp:6) on the spatial links of U, in place. */
void ref_project_su3(const int L[4], double* U) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  qcd_projectSU33d(u);
  memcpy(U, &(u.M[0][0][0][0]), sizeof(double) * 72 * volume(L));
}

/* this->APE_smearing(U_tmp) (lib/lattice_util.cpp:948) with U_tmp = U_in and
 * *this = U_out on entry; U_out receives *this afterwards. */
void ref_ape_smear(const int L[4], const double* U_in, double* U_out, int nsmear, double alpha) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  li.NsmearAPE = nsmear;
  li.alphaAPE = alpha;
  Gauge tmp(&li), out(&li);
  memcpy(&(tmp.M[0][0][0][0]), U_in, sizeof(double) * 72 * volume(L));
  memcpy(&(out.M[0][0][0][0]), U_out, sizeof(double) * 72 * volume(L));
  {
    QuietStdout q;
    out.APE_smearing(tmp, &li);
  }
  memcpy(U_out, &(out.M[0][0][0][0]), sizeof(double) * 72 * volume(L));
}

/* this->Gaussian_smearing(vec_tmp, gauge) (lib/lattice_util.cpp:1080) with
 * vec_tmp = in and *this = out on entry; out receives *this afterwards. */
void ref_gaussian_smear(const int L[4], const double* U, const double* in, double* out, int nsmear,
                        double alpha) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  li.NsmearGauss = nsmear;
  li.alphaGauss = alpha;
  Gauge u(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  Vector vin(&li), vout(&li);
  load_vec(vin, in);
  load_vec(vout, out);
  {
    QuietStdout q;
    vout.Gaussian_smearing(vin, u, &li);
  }
  store_vec(vout, out);
}

/* Propagator::absorbVector (lib/lattice_util.cpp:2073) into prop in place. */
void ref_absorb_vector(const int L[4], const double* phi, int nu, int c2, double* prop) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Propagator p(&li);
  memcpy(&(p.M[0][0][0][0][0]), prop, sizeof(double) * 288 * volume(L));
  Vector v(&li);
  load_vec(v, phi);
  p.absorbVector(v, nu, c2);
  memcpy(prop, &(p.M[0][0][0][0][0]), sizeof(double) * 288 * volume(L));
}

/* The propagator loop of bin/test_invert_prop.cpp:83-97: for each source
 * spin-colour (mu, ic), a point source at site `src` is Gaussian-smeared with
 * U_smear, the system M x = b is solved as tmDag + CG::operator() with the
 * operator links U (boundary condition already applied), the solution is
 * smeared and absorbed as column (mu, ic) of prop. */
void ref_propagator(const int L[4], double kappa, double mu, int twistSign, double tol, int maxIter,
                    const double* U, const double* U_smear, int nsmear, double alpha, long src, double* prop) {
  LatticeInfo li = make_info(L, kappa, mu, twistSign, -1, tol, maxIter);
  li.NsmearGauss = nsmear;
  li.alphaGauss = alpha;
  Gauge u(&li), us(&li);
  memcpy(&(u.M[0][0][0][0]), U, sizeof(double) * 72 * volume(L));
  memcpy(&(us.M[0][0][0][0]), U_smear, sizeof(double) * 72 * volume(L));
  u.constGauge = true;
  Vector vec_out(&li), vec_tmp(&li), vec_in(&li);
  Propagator p(&li);
  p.zero();
  {
    QuietStdout q;
    CG cg(&li, u);
    for (int sp = 0; sp < 4; sp++)
      for (int ic = 0; ic < 3; ic++) {
        vec_tmp.zero();
        vec_out.zero();
        vec_tmp.M[src][sp][ic].real() = 1.;
        vec_out.Gaussian_smearing(vec_tmp, us, &li);
        vec_in.tmDag(vec_out, u, &li);
        vec_out.zero();
        cg(vec_out, vec_in, &li);
        vec_in.Gaussian_smearing(vec_out, us, &li);
        p.absorbVector(vec_in, sp, ic);
      }
  }
  memcpy(prop, &(p.M[0][0][0][0][0]), sizeof(double) * 288 * volume(L));
}

/* Meson::contract(prop, op) and fourier(FORWARD) (lib/contractions.cpp:251, :121)
 * with Q_sq and x_src; corr receives Meson::F ([Lt][Nmom] complex).  Returns Nmom. */
int ref_meson_2pt(const int L[4], const double* prop, int op, int Q_sq, const int x_src[4], double* corr) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  li.Q_sq = Q_sq;
  for (int i = 0; i < 4; i++) li.x_src[i] = x_src[i];
  Propagator p(&li);
  memcpy(&(p.M[0][0][0][0][0]), prop, sizeof(double) * 288 * volume(L));
  char devnull[] = "/dev/null";
  int nmom;
  {
    QuietStdout q;
    Meson m(&li, devnull);
    m.contract(p, (MESONS_OPERATOR)op);
    m.fourier(FORWARD);
    nmom = m.Nmom;
    memcpy(corr, m.F, sizeof(double) * 2 * L[3] * nmom);
  }
  return nmom;
}

/* Baryon::contract(prop1, prop2, op) and fourier(FORWARD) (lib/contractions.cpp:494,
 * :356); corr receives Baryon::F ([Lt][Nmom][4][4] complex).  Returns Nmom. */
int ref_baryon_2pt(const int L[4], const double* prop1, const double* prop2, int op, int Q_sq, const int x_src[4],
                   double* corr) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  li.Q_sq = Q_sq;
  for (int i = 0; i < 4; i++) li.x_src[i] = x_src[i];
  Propagator p1(&li), p2(&li);
  memcpy(&(p1.M[0][0][0][0][0]), prop1, sizeof(double) * 288 * volume(L));
  memcpy(&(p2.M[0][0][0][0][0]), prop2, sizeof(double) * 288 * volume(L));
  char devnull[] = "/dev/null";
  int nmom;
  {
    QuietStdout q;
    Baryon b(&li, devnull);
    b.contract(p1, p2, (BARYON_OPERATOR)op);
    b.fourier(FORWARD);
    nmom = b.Nmom;
    memcpy(corr, b.F, sizeof(double) * 32 * L[3] * nmom);
  }
  return nmom;
}

/* Baryon_Dec::contract(prop1, prop2, op) and fourier(FORWARD) (lib/contractions.cpp:703-870);
 * corr receives Baryon_Dec::F ([Lt][Nmom][3][4][4] complex).  Returns Nmom. */
int ref_delta_2pt(const int L[4], const double* prop1, const double* prop2, int op, int Q_sq, const int x_src[4],
                  double* corr) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  li.Q_sq = Q_sq;
  for (int i = 0; i < 4; i++) li.x_src[i] = x_src[i];
  Propagator p1(&li), p2(&li);
  memcpy(&(p1.M[0][0][0][0][0]), prop1, sizeof(double) * 288 * volume(L));
  memcpy(&(p2.M[0][0][0][0][0]), prop2, sizeof(double) * 288 * volume(L));
  char devnull[] = "/dev/null";
  int nmom;
  {
    QuietStdout q;
    Baryon_Dec d(&li, devnull);
    d.contract(p1, p2, (BARYON_DEC_OPERATOR)op);
    d.fourier(FORWARD);
    nmom = d.Nmom;
    memcpy(corr, d.F, sizeof(double) * 96 * L[3] * nmom);
  }
  return nmom;
}

/* contractNucleon(prop1, prop2, output, Q_sq, x_src) (lib/lattice_util.cpp:3374): the
 * reference writes its correlator as text to `output`. */
void ref_contract_nucleon(const int L[4], const double* prop1, const double* prop2, int Q_sq, const int x_src[4],
                          const char* output) {
  LatticeInfo li = make_info(L, 0.1, 0.0, 1, -1, 1e-10, 1000);
  Propagator p1(&li), p2(&li);
  memcpy(&(p1.M[0][0][0][0][0]), prop1, sizeof(double) * 288 * volume(L));
  memcpy(&(p2.M[0][0][0][0][0]), prop2, sizeof(double) * 288 * volume(L));
  int xs[4] = {x_src[0], x_src[1], x_src[2], x_src[3]};
  QuietStdout q;
  contractNucleon(p1, p2, const_cast<char*>(output), Q_sq, xs);
}

}  // extern "C"
