// Host bounds check of the cubed-sphere tables (exo::build_tables,
// exocubed_b200/csrc/geometry.cpp), built with AddressSanitizer and
// UndefinedBehaviorSanitizer by tests/test_sanitizers_host.py: every ghost
// and edge entry must name cells inside the arrays the kernels index with
// it, and every metric value must be finite.  Exit status 0 when all hold.
#include <cmath>
#include <cstdio>
#include <string>

#include "../../exocubed_b200/csrc/exo_internal.h"

static int check(int N, int L, int eqn) {
  exo_config c = {};
  c.N = N;
  c.L = L;
  c.eqn = eqn;
  c.x1min = 6.371e6;
  c.x1max = 6.371e6 + 2.5e4;
  c.gamma = 1.4;
  c.Rd = 287.;
  c.cfl = 0.4;
  c.omega = 7.292e-5;
  exo::HostTables t;
  std::string err;
  if (!exo::build_tables(c, t, &err)) {
    std::printf("N=%d L=%d: %s\n", N, L, err.c_str());
    return 1;
  }
  int bad = 0;
  for (size_t n = 0; n < t.geo.size(); ++n)
    if (!std::isfinite(t.geo[n])) ++bad;
  if ((int)t.ghost_map.size() != 6 * t.nc3 * t.nc2) ++bad;
  for (int m : t.ghost_map)
    if (m < -1 || m >= (int)t.ghost.size()) ++bad;
  for (const exo::GhostEntry& g : t.ghost) {
    if (g.src_panel < 0 || g.src_panel >= 6) ++bad;
    if (g.k0 < 0 || g.k0 >= t.nc3 || g.k1 < 0 || g.k1 >= t.nc3) ++bad;
    if (g.j0 < 0 || g.j0 >= t.nc2 || g.j1 < 0 || g.j1 >= t.nc2) ++bad;
    if (!(g.C != 0.) || !std::isfinite(g.A) || !std::isfinite(g.B)) ++bad;
  }
  if ((int)t.edge.size() != 6 * 4 * N) ++bad;
  for (const exo::EdgeEntry& e : t.edge) {
    if (e.src_panel < 0 || e.src_panel >= 6 || e.src_side < 0 || e.src_side >= 4) ++bad;
    if (e.src_along < 0 || e.src_along >= N) ++bad;
  }
  if ((int)t.x1f.size() != t.nc1 + 1 || (int)t.x1v.size() != t.nc1) ++bad;
  if (bad) std::printf("N=%d L=%d: %d entries out of range\n", N, L, bad);
  return bad ? 1 : 0;
}

int main() {
  int rc = 0;
  const int sizes[][2] = {{6, 1}, {8, 3}, {12, 16}, {40, 40}, {96, 8}};
  for (const auto& s : sizes) {
    rc |= check(s[0], s[1], EXO_EQN_IDEAL);
    rc |= check(s[0], s[1], EXO_EQN_SHALLOW_YZ);
  }
  std::printf(rc ? "tables: FAIL\n" : "tables: ok\n");
  return rc;
}
