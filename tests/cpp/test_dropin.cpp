// test_dropin.cpp -- the reference's driver flow (bin/test_applyTM.cpp,
// bin/test_invert.cpp, bin/test_invert_prop.cpp) written against
// include/qkxTM_b200.hpp, checked against the CPU oracle.  Built and run by
// tests/test_gpu_dropin.py.
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/qkxTM_b200.hpp"
#include "../../oracle/qkx_oracle.h"

using namespace qkxTM_b200;

static double rel(const double* a, const double* b, long n) {
  double d = 0, s = 0;
  for (long i = 0; i < n; i++) {
    d += (a[i] - b[i]) * (a[i] - b[i]);
    s += b[i] * b[i];
  }
  return std::sqrt(d / (s > 0 ? s : 1));
}

int main() {
  LatticeInfo latInfo;
  latInfo.L[0] = 8;
  latInfo.L[1] = 8;
  latInfo.L[2] = 8;
  latInfo.L[3] = 16;
  latInfo.kappa = 0.16;
  latInfo.mu = 0.01;
  latInfo.twistSign = +1;
  latInfo.tol = 1e-10;
  latInfo.maxIter = 1000;
  latInfo.boundaryT = -1;

  Gauge* gauge = new Gauge(&latInfo);
  Vector* vec = new Vector(&latInfo);
  Vector* vecIn = new Vector(&latInfo);
  Vector* tmp = new Vector(&latInfo);
  const long V = vec->lV4d;
  int fails = 0;

  orc_gauge_random(latInfo.L, 0.3, 1234, reinterpret_cast<double*>(gauge->M));
  gauge->applyBoundaryCondition(&latInfo);
  orc_spinor_gaussian(latInfo.L, 42, vecIn->data());

  orc_params op = {{8, 8, 8, 16}, latInfo.kappa, latInfo.mu, latInfo.twistSign, latInfo.boundaryT, latInfo.tol, 1000};
  std::vector<double> ref(24 * V);
  const double* U = reinterpret_cast<const double*>(gauge->M);

  vec->tm(*vecIn, *gauge, &latInfo);
  orc_tm(&op, U, vecIn->data(), ref.data(), ORC_UKQCD);
  double e = rel(vec->data(), ref.data(), 24 * V);
  printf("tm            rel err %.2e\n", e);
  fails += e > 1e-13;

  vec->tm_xxDagTm_xx(*vecIn, *gauge, &latInfo, OO);
  orc_tm_xx_dagtm_xx(&op, U, vecIn->data(), ref.data(), ORC_OO, ORC_UKQCD);
  e = rel(vec->data(), ref.data(), 24 * V);
  printf("tm_xxDagTm_xx rel err %.2e\n", e);
  fails += e > 1e-13;

  vec->tm_xx_chiral(*vecIn, *gauge, &latInfo, EE);
  orc_tm_xx(&op, U, vecIn->data(), ref.data(), ORC_EE, ORC_CHIRAL);
  e = rel(vec->data(), ref.data(), 24 * V);
  printf("tm_xx_chiral  rel err %.2e\n", e);
  fails += e > 1e-13;

  // BLAS with the reference signatures
  double d = reCdotXdagY(*vecIn, *vecIn);
  double dref = orc_re_dot(V, vecIn->data(), vecIn->data());
  printf("reCdotXdagY   rel err %.2e\n", std::fabs(d - dref) / dref);
  fails += std::fabs(d - dref) > 1e-12 * dref;

  // bin/test_invert.cpp:95-117: in = M^+ b ; CG on M^+M with x zeroed
  Vector* vec_out = new Vector(&latInfo);
  tmp->tmDag(*vecIn, *gauge, &latInfo);
  vec_out->zero();
  CG cg(&latInfo, *gauge);
  qkx_solve_info info = cg(*vec_out, *tmp, &latInfo);
  std::vector<double> xo(24 * V, 0.0);
  orc_tm_dag(&op, U, vecIn->data(), ref.data(), ORC_UKQCD);
  int it = orc_cg(&op, U, ref.data(), xo.data(), nullptr, 0);
  e = rel(vec_out->data(), xo.data(), 24 * V);
  printf("CG            iterations %d (oracle %d), solution rel err %.2e\n", info.iterations, it, e);
  fails += e > 1e-9 || std::abs(info.iterations - it) > 1;

  // the batched B200 solve of M x = b
  std::vector<Vector*> bs = {vecIn}, xs = {vec};
  qkx_solve_info inv = cg.invert(bs, xs, &latInfo);
  vec_out->tm(*vec, *gauge, &latInfo);
  double r2 = 0, b2 = 0;
  for (long i = 0; i < 24 * V; i++) {
    double dv = vecIn->data()[i] - vec_out->data()[i];
    r2 += dv * dv;
    b2 += vecIn->data()[i] * vecIn->data()[i];
  }
  printf("invert        true residual %.2e (library %.2e)\n", std::sqrt(r2 / b2), inv.true_residual);
  fails += std::sqrt(r2 / b2) > 1e-10;

  // errors are exceptions carrying the status code
  try {
    vec->tm_xx(*vecIn, *gauge, &latInfo, EO);
    fails++;
  } catch (const Error& err) {
    printf("wrong parity  -> Error %d\n", err.code);
  }

  // bin/test_invert_prop.cpp: plaquettes, APE smearing, the smeared-source
  // propagator loop with the drop-in classes, and the batched B200 call
  {
    LatticeInfo li;
    li.L[0] = li.L[1] = li.L[2] = 4;
    li.L[3] = 8;
    li.kappa = 0.16;
    li.mu = 0.01;
    li.tol = 1e-12;
    li.maxIter = 5000;
    li.NsmearAPE = 20;
    li.alphaAPE = 0.5;
    li.NsmearGauss = 5;
    li.alphaGauss = 4.0;
    li.x_src[0] = 1;
    li.x_src[1] = 2;
    li.x_src[2] = 3;
    li.x_src[3] = 5;
    Gauge* g = new Gauge(&li);
    Gauge* g_tmp = new Gauge(&li);
    Gauge* g_ape = new Gauge(&li);
    const long Vs = g->lV4d;
    orc_gauge_random(li.L, 0.3, 51, g->data());
    g_tmp->copy(*g);
    double plaq = g->calculatePlaquette();
    double pref = orc_plaquette_ref(li.L, g->data());
    printf("plaquette     %.12f (oracle %.12f)\n", plaq, pref);
    fails += std::fabs(plaq - pref) > 1e-13;
    g_ape->APE_smearing(*g_tmp, &li);
    std::vector<double> ape(72 * Vs);
    orc_ape_smear(li.L, g->data(), ape.data(), li.NsmearAPE, li.alphaAPE);
    e = rel(g_ape->data(), ape.data(), 72 * Vs);
    double pa = g_ape->calculatePlaquette();
    printf("APE smearing  rel err %.2e, smeared plaquette %.12f\n", e, pa);
    fails += e > 1e-10 || std::fabs(pa - orc_plaquette_ref(li.L, ape.data())) > 1e-12;
    g->applyBoundaryCondition(&li);

    Vector v_out(&li), v_tmp(&li), v_in(&li);
    Propagator prop(&li), prop2(&li);
    CG cgp(&li, *g);
    const long src = li.x_src[0] + 4 * (li.x_src[1] + 4 * (li.x_src[2] + 4 * li.x_src[3]));
    for (int mu = 0; mu < 4; mu++)
      for (int ic = 0; ic < 3; ic++) {
        v_tmp.zero();
        v_out.zero();
        v_tmp.M[src][mu][ic] = 1.0;
        v_out.Gaussian_smearing(v_tmp, *g_ape, &li);
        v_in.tmDag(v_out, *g, &li);
        v_out.zero();
        cgp(v_out, v_in, &li);
        v_in.Gaussian_smearing(v_out, *g_ape, &li);
        prop.absorbVector(v_in, mu, ic);
      }
    qkx_solve_info pi = cgp.propagator(prop2, *g_ape, &li, QKX_SOLVER_CG_EO_MIXED, QKX_PREC_HALF, 1e-12);
    e = rel(prop2.data(), prop.data(), 288 * Vs);
    printf("propagator    batched vs loop rel err %.2e (true residual %.2e)\n", e, pi.true_residual);
    fails += e > 1e-8;

    // ILDG round trip (lib/write_conf_lime.cpp, lib/read_conf_lime.cpp) and the
    // contraction drivers (lib/contractions.cpp:873-914)
    std::string tag = "/tmp/qkx_dropin_" + std::to_string(getpid());
    std::string conf = tag + ".lime", twop = tag + "_mesons.dat", twob = tag + "_baryons.dat";
    char msg[] = "drop-in test";
    qkxTM_writeGaugeLime(&conf[0], *g, msg);
    Gauge* g2 = new Gauge(&li);
    qkxTM_MPI_getGaugeLime(&conf[0], *g2);
    const bool same = std::memcmp(g2->data(), g->data(), sizeof(double) * 72 * Vs) == 0;
    printf("ILDG          write + read %s\n", same ? "identical" : "DIFFERENT");
    fails += !same;
    li.Q_sq = 1;
    contractMesons(&prop, &prop2, &twop[0], &li);
    contractBaryons(&prop, &prop2, &twob[0], &li);
    int mom[7 * 3];
    const int nmom = orc_momenta(1, mom, 7);
    std::vector<double> cref((size_t)2 * li.L[3] * nmom), bref((size_t)32 * li.L[3] * nmom);
    orc_meson_2pt(li.L, prop.data(), 0, 1, li.x_src, cref.data());
    orc_baryon_2pt(li.L, prop2.data(), prop.data(), 3, 1, li.x_src, bref.data());
    // line 0: ONE of prop, t = 0, first momentum; the baryon file's last block: RTR of (prop2, prop)
    FILE* fm = fopen(twop.c_str(), "r");
    int op, t, n0, n1, n2;
    double re = 0, im = 0;
    int lines = 0, ok_line = fscanf(fm, "%d %d %d %d %d %lf %lf", &op, &t, &n0, &n1, &n2, &re, &im) == 7;
    fseek(fm, 0, SEEK_SET);
    for (int ch; (ch = fgetc(fm)) != EOF;) lines += ch == '\n';
    fclose(fm);
    double em = std::hypot(re - cref[0], im - cref[1]) / std::hypot(cref[0], cref[1]);
    FILE* fb = fopen(twob.c_str(), "r");
    int blines = 0, g0, g1;
    double br = 0, bi = 0, eb = 0;
    for (int k = 0; fscanf(fb, "%d %d %d %d %d %d %d %lf %lf", &op, &t, &n0, &n1, &n2, &g0, &g1, &br, &bi) == 9; k++) {
      blines++;
      if (k >= 7 * li.L[3] * nmom * 16) {  // the second propagator pair's RTR block
        const int j = k - 7 * li.L[3] * nmom * 16;
        eb = std::max(eb, std::hypot(br - bref[2 * j], bi - bref[2 * j + 1]));
      }
    }
    fclose(fb);
    double bmax = 0;
    for (double v : bref) bmax = std::max(bmax, std::fabs(v));
    printf("contractions  %d meson lines (rel err %.1e), %d baryon lines (max err %.1e of %.1e)\n", lines, em,
           blines, eb, bmax);
    fails += !ok_line || lines != 2 * 10 * li.L[3] * nmom || em > 1e-6;  // the text keeps 7 digits
    fails += blines != 8 * li.L[3] * nmom * 16 || eb > 1e-6 * bmax;
    unlink(conf.c_str());
    unlink(twop.c_str());
    unlink(twob.c_str());
    delete g2;
    delete g_ape;
    delete g_tmp;
    delete g;
  }

  delete vec_out;
  delete tmp;
  delete vecIn;
  delete vec;
  delete gauge;
  printf(fails ? "FAILED %d\n" : "OK\n", fails);
  return fails ? 1 : 0;
}
