// The CPU oracle (oracle/exo_oracle.cpp) under AddressSanitizer and
// UndefinedBehaviorSanitizer, built by tests/test_sanitizers_host.py: a few
// steps of the shallow-water case, of the dry gas with the full and the
// partial vertical correction (LMARS and HLLC, gravity, the 3D Coriolis
// force and the Held-Suarez forcing), the column corrections and the
// decomposition hooks.  Exit status 0 when every result is finite.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/exo_b200.h"

extern "C" {
void* ora_create(const exo_config* cfg);
void ora_destroy(void* h);
int ora_set_primitive(void* h, const double* w);
void ora_get_conserved(void* h, double* out);
void ora_get_primitive(void* h, double* out);
void ora_step(void* h, int nsteps, double dt_fixed);
void ora_get_mesh(void* h, int panel, double* x1f, double* x2f, double* x3f);
void ora_change_to_perturbation(void* h, double* w);
void ora_restore_from_perturbation(void* h, double* w, double* wl, double* wr);
void ora_correction_columns(int full, int ncol, int L, const double* w, double* du,
                            const double* colgeo, const double* x1f, const double* x1v,
                            const double* dx1f, double dt, double gamma, double grav);
}

static uint64_t rng = 12345;
static double noise() {  // uniform in [-1, 1)
  rng = rng * 6364136223846793005ull + 1442695040888963407ull;
  return (double)(rng >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

static int finite(const std::vector<double>& a) {
  for (double x : a)
    if (!std::isfinite(x)) return 0;
  return 1;
}

static int run(exo_config c, int steps) {
  const int G = 3, N = c.N, L = c.L, nc1 = L + 2 * G, nc2 = N + 2 * G;
  const int nv = c.eqn == EXO_EQN_SHALLOW_YZ ? 4 : 5;
  const size_t cells = (size_t)nc2 * nc2 * nc1, tot = 6 * nv * cells;
  void* h = ora_create(&c);
  if (!h) return 1;
  std::vector<double> w(tot, 0.), x1f(nc1 + 1), x2f(nc2 + 1), x3f(nc2 + 1);
  ora_get_mesh(h, 0, x1f.data(), x2f.data(), x3f.data());
  auto at = [&](int p, int n, int k, int j, int i) {
    return (((size_t)p * nv + n) * nc2 + k) * nc2 * nc1 + (size_t)j * nc1 + i;
  };
  for (int p = 0; p < 6; ++p)
    for (int k = G; k < G + N; ++k)
      for (int j = G; j < G + N; ++j)
        for (int i = G; i < G + L; ++i) {
          if (nv == 4) {
            w[at(p, 0, k, j, i)] = 2.94e4 * (1. + 0.01 * noise());
            w[at(p, 2, k, j, i)] = 10. * noise();
            w[at(p, 3, k, j, i)] = 10. * noise();
          } else {
            double z = 0.5 * (x1f[i] + x1f[i + 1]) - c.x1min, T = 250. + noise();
            double pr = 1e5 * std::exp(-9.81 * z / (287. * 250.));
            w[at(p, 0, k, j, i)] = pr / (287. * T);
            w[at(p, 1, k, j, i)] = 0.1 * noise();
            w[at(p, 2, k, j, i)] = 5. * noise();
            w[at(p, 3, k, j, i)] = 5. * noise();
            w[at(p, 4, k, j, i)] = pr;
          }
        }
  int ok = ora_set_primitive(h, w.data()) == 0;
  ora_step(h, steps, 0.);
  std::vector<double> u(tot);
  ora_get_conserved(h, u.data());
  ok &= finite(u);
  if (nv == 5 && c.grav != 0.) {
    std::vector<double> wp(tot), wl(tot), wr(tot);
    ora_get_primitive(h, wp.data());
    wl = wp;
    wr = wp;
    ora_change_to_perturbation(h, wp.data());
    ora_restore_from_perturbation(h, wp.data(), wl.data(), wr.data());
    ok &= finite(wp) & finite(wl) & finite(wr);
  }
  ora_destroy(h);
  return ok ? 0 : 1;
}

int main() {
  int rc = 0;
  exo_config sw = {};
  sw.N = 6; sw.L = 3; sw.eqn = EXO_EQN_SHALLOW_YZ; sw.rsolver = EXO_RS_ROE_SHALLOW;
  sw.coriolis = EXO_CORIOLIS_W92; sw.x1min = 6371000.; sw.x1max = 6371001.;
  sw.gamma = 1.4; sw.Rd = 287.; sw.cfl = 0.4; sw.omega = 7.292e-5;
  rc |= run(sw, 2);
  sw.rsolver = EXO_RS_LMARS_SHALLOW;
  rc |= run(sw, 2);
  exo_config d = {};
  d.N = 6; d.L = 8; d.eqn = EXO_EQN_IDEAL; d.rsolver = EXO_RS_LMARS; d.implicit_flag = 9;
  d.x1min = 6.371e6; d.x1max = 6.371e6 + 3.0e4; d.gamma = 1.4; d.Rd = 287.; d.grav = -9.81;
  d.cfl = 0.4; d.omega = 7.292e-5;
  rc |= run(d, 2);
  d.rsolver = EXO_RS_HLLC; d.implicit_flag = 1; d.coriolis = EXO_CORIOLIS_3D;
  rc |= run(d, 2);
  d.coriolis = EXO_CORIOLIS_NONE; d.forcing = EXO_FORCING_HS94;
  d.hs_p0 = 1e5; d.hs_Ts = 315.; d.hs_dT = 60.; d.hs_dtheta = 10.; d.hs_Kf = 1.;
  d.hs_Ka = 0.025; d.hs_Ks = 0.25; d.hs_sigmab = 0.7;
  rc |= run(d, 2);
  // column corrections on a few synthetic columns
  const int ncol = 3, L = 6, nc1 = L + 6;
  std::vector<double> x1f(nc1 + 1), x1v(nc1), dx1f(nc1), w(ncol * 5 * nc1), du(ncol * 5 * L),
      colgeo(ncol * 4);
  for (int i = 0; i <= nc1; ++i) x1f[i] = 6.371e6 + 1000. * (i - 3);
  for (int i = 0; i < nc1; ++i) {
    x1v[i] = 0.5 * (x1f[i] + x1f[i + 1]);
    dx1f[i] = 1000.;
  }
  for (int c = 0; c < ncol; ++c) {
    for (int i = 0; i < nc1; ++i) {
      double pr = 1e5 * std::exp(-9.81 * 1000. * (i - 3) / (287. * 250.));
      w[(c * 5 + 0) * nc1 + i] = pr / (287. * 250.);
      w[(c * 5 + 1) * nc1 + i] = 0.1 * noise();
      w[(c * 5 + 2) * nc1 + i] = 5. * noise();
      w[(c * 5 + 3) * nc1 + i] = 5. * noise();
      w[(c * 5 + 4) * nc1 + i] = pr;
    }
    for (int n = 0; n < 5 * L; ++n) du[c * 5 * L + n] = 1e-4 * noise();
    colgeo[c * 4 + 0] = 0.2;
    colgeo[c * 4 + 1] = std::sqrt(1. - 0.04);
    colgeo[c * 4 + 2] = colgeo[c * 4 + 3] = 0.1;
  }
  for (int full = 0; full < 2; ++full) {
    std::vector<double> d2 = du;
    ora_correction_columns(full, ncol, L, w.data(), d2.data(), colgeo.data(), x1f.data(),
                           x1v.data(), dx1f.data(), 200., 1.4, -9.81);
    rc |= finite(d2) ? 0 : 1;
  }
  std::printf(rc ? "oracle: FAIL\n" : "oracle: ok\n");
  return rc;
}
