/*
 * qkx_oracle.h -- CPU oracle for the twisted-mass Dslash / CG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the
 * reference algorithm (khadjiyiannakou/qkxTM_MPI, lib/lattice_util.cpp,
 * lib/blas_qkxTM.cpp, lib/solvers.cpp).  Only the tests, the smoke check and
 * the CPU-baseline leg of the benchmark may load it, and only as the checker.
 * The product library never links or calls it.
 *
 * Parity of this restatement is pinned against the reference's own sources,
 * compiled unmodified by oracle/ref/Makefile into oracle/_ref/, and against the
 * golden vectors in tests/golden/ that were produced from that build.
 *
 * Field layouts are those of the reference's host containers:
 *   spinor  [V][4 spin][3 colour] complex double   (Vector::M, include/lattice_util.h:90)
 *   gauge   [V][4 dir][3][3]      complex double   (Gauge::M,  include/lattice_util.h:198)
 *   site    x + Lx*(y + Ly*(z + Lz*t))             (LEXIC,     include/qkxTM.h:130)
 *   dir     0=x 1=y 2=z 3=t
 * Arrays are passed as interleaved (re,im) doubles.
 */
#ifndef QKX_ORACLE_H
#define QKX_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_UKQCD = 0, ORC_CHIRAL = 1 };
/* parity selectors, same meaning as qkxTM::PARITY (include/lattice_util.h:22) */
enum { ORC_EO = 0, ORC_OE = 1, ORC_OO = 2, ORC_EE = 3 };

typedef struct {
  int L[4];
  double kappa;
  double mu;
  int twistSign;
  int boundaryT;
  double tol;
  int maxIter;
} orc_params;

long orc_volume(const int L[4]);

/* synthetic inputs (no reference counterpart: the reference reads ILDG files) */
void orc_gauge_random(const int L[4], double eps, unsigned long long seed, double* U);
void orc_gauge_unit(const int L[4], double* U);
void orc_spinor_gaussian(const int L[4], unsigned long long seed, double* psi);
void orc_spinor_point(const int L[4], const int x[4], int spin, int colour, double* psi);
double orc_plaquette(const int L[4], const double* U);
void orc_apply_bc(const int L[4], int boundaryT, double* U);

/* operators: basis = ORC_UKQCD or ORC_CHIRAL */
void orc_dslash(const int L[4], const double* U, const double* psi, double* out, int dagger, int basis);
void orc_dslash_xx(const int L[4], const double* U, const double* psi, double* out, int parity, int basis);
void orc_twist(const orc_params* p, const double* psi, double* out, int dagger, int inverse, int basis);
void orc_gamma5(const int L[4], const double* psi, double* out, int basis);
void orc_tm(const orc_params* p, const double* U, const double* psi, double* out, int basis);
void orc_tm_dag(const orc_params* p, const double* U, const double* psi, double* out, int basis);
void orc_tm_dagtm(const orc_params* p, const double* U, const double* psi, double* out, int basis);
void orc_wilson(const orc_params* p, const double* U, const double* psi, double* out);
void orc_tm_xx(const orc_params* p, const double* U, const double* psi, double* out, int parity, int basis);
void orc_tm_xx_dagtm_xx(const orc_params* p, const double* U, const double* psi, double* out, int parity, int basis);
void orc_rotate_chiral_to_ukqcd(const int L[4], double* psi);

/* BLAS (lib/blas_qkxTM.cpp) */
double orc_re_dot(long V, const double* x, const double* y);
void orc_axpy(long V, double a, const double* y, double* x);   /* x = x + a*y */
void orc_xpay(long V, double a, const double* y, double* x);   /* x = a*x + y */
double orc_norm2(long V, const double* x);

/* CG on M^dag M exactly as CG::operator() (lib/solvers.cpp:16-81).
 * x is accumulated into (the reference never zeroes it).  r2_trace, if not
 * NULL, receives r2 at the top of every iteration (max_trace entries).
 * Returns the iteration count. */
int orc_cg(const orc_params* p, const double* U, const double* in, double* x,
           double* r2_trace, int max_trace);

/* gauge-side stencils and propagator workflow (qkx_oracle_smear.c):
 * Gauge::calculatePlaquette (lib/lattice_util.cpp:923), qcd_projectSU33d
 * (lib/blas.cpp:6) on n matrices in place, Gauge::APE_smearing (:948),
 * Vector::Gaussian_smearing (:1080), Propagator::absorbVector (:2073).
 * A propagator is [V][4 mu][4 nu][3 c1][3 c2] complex double
 * (Propagator::M, include/lattice_util.h:168). */
double orc_plaquette_ref(const int L[4], const double* U);
void orc_su3_project_many(long n, double* m);
void orc_ape_smear(const int L[4], const double* U_in, double* U_out, int nsmear, double alpha);
void orc_gaussian_smear(const int L[4], const double* U, const double* in, double* out, int nsmear,
                        double alpha);
void orc_absorb_vector(long V, const double* phi, int nu, int c2, double* prop);

/* two-point contractions (qkx_oracle_contract.c): createMomenta
 * (lib/contractions.cpp:37), Meson::contract + fourier(FORWARD) (:251, :121),
 * Baryon::contract + fourier(FORWARD) (:494, :356).  Return the number of
 * momenta; corr is [Lt][Nmom] (meson) or [Lt][Nmom][4][4] (baryon) complex. */
int orc_momenta(int Q_sq, int* mom, int max);
int orc_meson_2pt(const int L[4], const double* prop, int op, int Q_sq, const int x_src[4], double* corr);
int orc_baryon_2pt(const int L[4], const double* prop1, const double* prop2, int op, int Q_sq, const int x_src[4],
                   double* corr);
/* Baryon_Dec::contract + fourier(FORWARD) (lib/contractions.cpp:703-870): corr is
 * [Lt][Nmom][3][4][4]; op 0 DELTA_ISO1, 1 DELTA_ISO1O2. */
int orc_delta_2pt(const int L[4], const double* prop1, const double* prop2, int op, int Q_sq, const int x_src[4],
                  double* corr);
/* contractNucleon (lib/lattice_util.cpp:3374): corr is [Lt][Nmom][4][4]. */
int orc_nucleon_2pt(const int L[4], const double* prop1, const double* prop2, int Q_sq, const int x_src[4],
                    double* corr);

/* learned preconditioner (qkx_oracle_ptc.c; no reference counterpart): a linear
 * parallel-transport convolution network with nlayers layers of channel widths
 * ch[0..nlayers]; weights [9][ch[l+1]][ch[l]] complex per layer, concatenated. */
long orc_ptc_nweights(int nlayers, const int* ch);
void orc_ptc_forward(const int L[4], const double* U, int nlayers, const int* ch, const double* W,
                     const double* in, double* out, double* acts);
double orc_ptc_loss_grad(const int L[4], const double* U, int nlayers, const int* ch, const double* W,
                         const double* r, const double* e, double* grad);
/* 1: hidden activations and activation gradients stored as BF16 (as on the GPU); 0: FP64 */
void orc_ptc_act_bf16(int on);

#ifdef __cplusplus
}
#endif
#endif
