// geometry.cpp -- host-side tables of the gnomonic equiangular cubed sphere.
//
// Everything that needs a transcendental function (tan, acos, atan, sin) is
// evaluated here once, in FP64, with the expressions of the reference, and
// uploaded to the device.  The kernels then use only +, -, *, / and sqrt, so
// a device step reproduces a CPU step bit for bit when both avoid fused
// multiply-add.
//
// Reference (cshsgy/ExoCubed):
//   cell faces      patches/27.coordinates.patch:21,40; src/exo3/cubed_sphere.cpp:37-73
//   metric          src/exo3/gnomonic_equiangle.cpp:154-221
//   flux projection src/snap/riemann/hllc_transform.cpp:235-262
//   Coriolis        examples/2023-Chen-exo3/W92.cpp:48-70; cubed_sphere.cpp:78-162,226-262
//   ghost bands     src/exo3/cubed_sphere_utility.cpp:18-619
//   edge states     src/exo3/cubed_sphere.cpp:326-688
//   adjacency       src/exo3/cs_transform_ox.cpp:11-229
#include <algorithm>
#include <cmath>
#include <cstring>

#include "exo_internal.h"

namespace exo {

namespace {

constexpr double PI = 3.1415926535897932;  // Athena++ PI

// neighbour across each side of each panel and the side it arrives at
const int kNbrPanel[6][4] = {{6, 2, 3, 4}, {1, 5, 3, 4}, {1, 5, 6, 2},
                             {1, 5, 2, 6}, {2, 6, 3, 4}, {1, 5, 4, 3}};
const int kNbrSide[6][4] = {{UP, UP, UP, UP},         {DOWN, UP, RIGHT, LEFT},
                            {LEFT, LEFT, RIGHT, LEFT}, {RIGHT, RIGHT, RIGHT, LEFT},
                            {DOWN, DOWN, DOWN, DOWN},   {UP, DOWN, RIGHT, LEFT}};
// direction inversion and touching-side tables (cubed_sphere_utility.cpp:378-390)
const int kDinv[6][4] = {{1, 0, 0, 1}, {0, 0, 0, 0}, {0, 1, 0, 0},
                         {1, 0, 0, 0}, {0, 1, 1, 0}, {1, 1, 0, 0}};
const int kTgSide[6][4] = {{-1, -1, -1, -1}, {1, -1, 1, -1}, {-1, -1, 1, -1},
                           {1, 1, 1, -1},    {1, 1, 1, 1},   {-1, 1, 1, -1}};
// traversal used to pack each (panel, side): PackDataR0..R3
const int kPackOrder[6][4] = {{2, 0, 3, 1}, {0, 0, 0, 0}, {1, 3, 0, 0},
                              {3, 1, 0, 0}, {0, 2, 1, 3}, {2, 2, 0, 0}};

int side_ox2(int s) { return s == UP ? -1 : (s == DOWN ? 1 : 0); }
int side_ox3(int s) { return s == LEFT ? -1 : (s == RIGHT ? 1 : 0); }

// Athena++ ComputeMeshGeneratorX, symmetric interval
double mesh_gen_x(int64_t index, int64_t nrange) {
  int64_t noffset = index - nrange / 2;
  int64_t noffset_ceil = index - (nrange + 1) / 2;
  return static_cast<double>(noffset + noffset_ceil) / (2.0 * nrange);
}

double gen_mesh_x2(double x, int lx2) {
  double x_l = lx2 == 0 ? -0.5 : 0.0, x_u = lx2 == 0 ? 0.0 : 0.5;
  return (0.5 * (x - x_l) / (x_u - x_l) - 0.25) * PI;
}

double gen_mesh_x3(double x, int lx3) {
  double x_l, x_u;
  if (lx3 == 0) { x_l = -0.5; x_u = -1.0 / 6.0; }
  else if (lx3 == 1) { x_l = -1.0 / 6.0; x_u = 1.0 / 6.0; }
  else { x_l = 1.0 / 6.0; x_u = 0.5; }
  return (0.5 * (x - x_l) / (x_u - x_l) - 0.25) * PI;
}

// CalculateInterpLocations: angular position of a cell seen across the edge
double interp_loc(int loc_n, int N_blk, int k, bool ghost) {
  double temp0 = tan((double)1.0 * (N_blk - 1 - 2 * k) / (N_blk * 4) * PI);
  if (ghost) {
    temp0 = 1.0 / temp0;
    temp0 = 1.0 + temp0 * temp0;
  } else {
    temp0 = 1.0 + temp0 * temp0;
  }
  double t = pow(tan((double)1.0 * (2 * loc_n + 1) / (N_blk * 4) * PI), 2.0);
  if (loc_n < 0) return -acos(sqrt(temp0 / (temp0 + t)));
  return acos(sqrt(temp0 / (temp0 + t)));
}

}  // namespace

void rll_from_abp_coef(double X, double Y, int blockID, double c[4]) {
  double C = sqrt(1 + X * X), D = sqrt(1 + Y * Y), E = sqrt(X * X + Y * Y);
  double delta = sqrt(1 + X * X + Y * Y);
  switch (blockID) {
    case 1:
      c[0] = -delta * Y / (D * E);
      c[1] = delta * X / (C * E);
      c[2] = -X / (D * E);
      c[3] = -(Y / (C * E));
      break;
    case 5:
      c[0] = delta * Y / (D * E);
      c[1] = -(delta * X / (C * E));
      c[2] = X / (D * E);
      c[3] = Y / (C * E);
      break;
    default:  // 2, 3, 4, 6
      c[0] = 0.;
      c[1] = delta / (C * D);
      c[2] = -1.;
      c[3] = X * Y / (C * D);
      break;
  }
}

void abp_from_rll_coef(double X, double Y, int blockID, double c[4]) {
  double C = sqrt(1 + X * X), D = sqrt(1 + Y * Y), E = sqrt(X * X + Y * Y);
  double delta = sqrt(1 + X * X + Y * Y);
  switch (blockID) {
    case 1:
      c[0] = -D * Y / (delta * E);
      c[1] = -(D * X / E);
      c[2] = C * X / (delta * E);
      c[3] = -(C * Y / E);
      break;
    case 5:
      c[0] = D * Y / (delta * E);
      c[1] = D * X / E;
      c[2] = -C * X / (delta * E);
      c[3] = C * Y / E;
      break;
    default:
      c[0] = X * Y / delta;
      c[1] = -1.;
      c[2] = C * D / delta;
      c[3] = 0.;
      break;
  }
}

void rll_from_xyp(double dX, double dY, int nP, double& lon, double& lat) {
  const double eps = 1.0e-10;
  switch (nP) {
    case 1: lon = atan(dX); lat = atan(dY / sqrt(1.0 + dX * dX)); break;
    case 3: lon = atan(dX) + 0.5 * M_PI; lat = atan(dY / sqrt(1.0 + dX * dX)); break;
    case 5: lon = atan(dX) + M_PI; lat = atan(dY / sqrt(1.0 + dX * dX)); break;
    case 2: lon = atan(dX) + 1.5 * M_PI; lat = atan(dY / sqrt(1.0 + dX * dX)); break;
    case 0:
      if (fabs(dX) > eps) lon = atan2(dX, -dY);
      else if (dY <= 0.0) lon = 0.0;
      else lon = M_PI;
      lat = 0.5 * M_PI - atan(sqrt(dX * dX + dY * dY));
      break;
    default:  // 4
      if (fabs(dX) > eps) lon = atan2(dX, dY);
      else if (dY > 0.0) lon = 0.0;
      else lon = M_PI;
      lat = -0.5 * M_PI + atan(sqrt(dX * dX + dY * dY));
      break;
  }
  if (lon < 0.0) lon += 2.0 * M_PI;
}

static void build_mesh(const exo_config& cfg, HostTables& t) {
  int N = t.N, L = t.L, is = G, ie = G + L - 1;
  t.x1f.assign(t.nc1 + 1, 0.);
  t.dx1f.assign(t.nc1, 0.);
  t.x1v.assign(t.nc1, 0.);
  for (int i = 0; i <= t.nc1; ++i) {
    double rx = mesh_gen_x(i - is, L);
    t.x1f[i] = 0.5 * (cfg.x1min + cfg.x1max) + (rx * cfg.x1max - rx * cfg.x1min);
  }
  t.x1f[is] = cfg.x1min;
  t.x1f[ie + 1] = cfg.x1max;
  for (int i = 0; i < t.nc1; ++i) t.dx1f[i] = t.x1f[i + 1] - t.x1f[i];
  for (int i = 1; i <= G; ++i) {
    t.dx1f[is - i] = t.dx1f[is + i - 1];
    t.x1f[is - i] = t.x1f[is - i + 1] - t.dx1f[is - i];
  }
  for (int i = 1; i <= G; ++i) {
    t.dx1f[ie + i] = t.dx1f[ie - i + 1];
    t.x1f[ie + i + 1] = t.x1f[ie + i] + t.dx1f[ie + i];
  }
  for (int i = 0; i < t.nc1; ++i) t.x1v[i] = 0.5 * (t.x1f[i + 1] + t.x1f[i]);
  for (int p = 0; p < 6; ++p) {
    int lx2 = p % 2, lx3 = p / 2;
    t.x2f[p].assign(t.nc2 + 1, 0.);
    t.x3f[p].assign(t.nc3 + 1, 0.);
    t.x2v[p].assign(t.nc2, 0.);
    t.x3v[p].assign(t.nc3, 0.);
    for (int j = 0; j <= t.nc2; ++j)
      t.x2f[p][j] = gen_mesh_x2(mesh_gen_x((j - G) + (int64_t)lx2 * N, 2 * N), lx2);
    for (int k = 0; k <= t.nc3; ++k)
      t.x3f[p][k] = gen_mesh_x3(mesh_gen_x((k - G) + (int64_t)lx3 * N, 3 * N), lx3);
    for (int j = 0; j < t.nc2; ++j) t.x2v[p][j] = 0.5 * (t.x2f[p][j + 1] + t.x2f[p][j]);
    for (int k = 0; k < t.nc3; ++k) t.x3v[p][k] = 0.5 * (t.x3f[p][k + 1] + t.x3f[p][k]);
  }
}

static void build_metric(const exo_config& cfg, HostTables& t) {
  t.geo.assign((size_t)NGEO2D * 6 * t.nc3 * t.nc2, 0.);
  for (int p = 0; p < 6; ++p)
    for (int k = 0; k < t.nc3; ++k)
      for (int j = 0; j < t.nc2; ++j) {
        auto G2 = [&](int f) -> double& { return t.geo[t.g2(f, p, k, j)]; };
        const std::vector<double>& x2f = t.x2f[p];
        const std::vector<double>& x3f = t.x3f[p];
        double x = tan(t.x2v[p][j]), xf = tan(x2f[j]);
        double y = tan(t.x3v[p][k]), yf = tan(x3f[k]);
        double C = sqrt(1.0 + x * x), Cf = sqrt(1.0 + xf * xf);
        double D = sqrt(1.0 + y * y), Df = sqrt(1.0 + yf * yf);
        G2(GCOSC) = -x * y / (C * D);
        G2(GSINC) = sqrt(1.0 + x * x + y * y) / (C * D);
        G2(GCOSF2) = -xf * y / (Cf * D);
        G2(GSINF2) = sqrt(1.0 + xf * xf + y * y) / (Cf * D);
        G2(GCOSF3) = -x * yf / (C * Df);
        G2(GSINF3) = sqrt(1.0 + x * x + yf * yf) / (C * Df);
        double x1 = tan(x2f[j]), x2 = tan(x2f[j + 1]);
        double delta1 = sqrt(1.0 + x1 * x1 + y * y), delta2 = sqrt(1.0 + x2 * x2 + y * y);
        double delta1f = sqrt(1.0 + x1 * x1 + yf * yf), delta2f = sqrt(1.0 + x2 * x2 + yf * yf);
        G2(GDX2A) = acos((1 + x1 * x2 + y * y) / (delta1 * delta2));
        G2(GDX2A_F3) = acos((1 + x1 * x2 + yf * yf) / (delta1f * delta2f));
        double y1 = tan(x3f[k]), y2 = tan(x3f[k + 1]);
        delta1 = sqrt(1.0 + x * x + y1 * y1);
        delta2 = sqrt(1.0 + x * x + y2 * y2);
        delta1f = sqrt(1.0 + xf * xf + y1 * y1);
        delta2f = sqrt(1.0 + xf * xf + y2 * y2);
        G2(GDX3A) = acos((1 + x * x + y1 * y2) / (delta1 * delta2));
        G2(GDX3A_F2) = acos((1 + xf * xf + y1 * y2) / (delta1f * delta2f));
        // projection angle of contravariant fluxes onto covariant components
        double xx = tan(t.x2v[p][j]), yy = tan(t.x3v[p][k]);
        double CC = sqrt(1. + xx * xx), DD = sqrt(1. + yy * yy);
        G2(GCTHP1) = -xx * yy / CC / DD;
        xx = tan(x2f[j]); yy = tan(t.x3v[p][k]);
        CC = sqrt(1. + xx * xx); DD = sqrt(1. + yy * yy);
        G2(GCTHP2) = -xx * yy / CC / DD;
        xx = tan(t.x2v[p][j]); yy = tan(x3f[k]);
        CC = sqrt(1. + xx * xx); DD = sqrt(1. + yy * yy);
        G2(GCTHP3) = -xx * yy / CC / DD;
        // Coriolis (W92 Forcing2): f at the cell centre and the cell's
        // panel <-> lat-lon vector maps
        double dX = tan(t.x2v[p][j]), dY = tan(t.x3v[p][k]);
        double lat, lon;
        rll_from_xyp(dY, -dX, p, lon, lat);
        G2(GFCOR) = 2. * cfg.omega * sin(lat);
        // Held-Suarez forcing: hs94.cpp:130-138 (_sqr, _qur of sin/cos(lat))
        {
          double sl = sin(lat), cl = cos(lat);
          G2(GSLAT2) = sl * sl;
          G2(GCLAT2) = cl * cl;
          G2(GCLAT4) = cl * cl * cl * cl;
        }
        // CalculateCoriolisForce3 (cubed_sphere.cpp:197-231): A = 2 Omega C D
        // / delta / delta, times the density on the device
        {
          double C = sqrt(dX * dX + 1), D = sqrt(dY * dY + 1);
          double delta = sqrt(dX * dX + dY * dY + 1);
          G2(GTANX) = dX;
          G2(GTANY) = dY;
          G2(GC3C) = C;
          G2(GC3D) = D;
          G2(GC3A) = 2 * cfg.omega * C * D / delta / delta;
        }
        double c[4];
        rll_from_abp_coef(dX, dY, p + 1, c);
        G2(GCR0) = c[0]; G2(GCR1) = c[1]; G2(GCR2) = c[2]; G2(GCR3) = c[3];
        abp_from_rll_coef(dX, dY, p + 1, c);
        G2(GCQ0) = c[0]; G2(GCQ1) = c[1]; G2(GCQ2) = c[2]; G2(GCQ3) = c[3];
      }
}

// Ghost bands: emulate PackData (interpolate + traversal) and the plain
// unpack of the receiver, recording coefficients instead of values.
static void build_ghost_table(HostTables& t) {
  int N = t.N;
  int js = G, je = G + N - 1, ks = G, ke = G + N - 1;
  t.ghost_map.assign((size_t)6 * t.nc3 * t.nc2, -1);
  t.ghost.clear();
  for (int p = 0; p < 6; ++p)
    for (int s = 0; s < 4; ++s) {
      int blockID = p + 1;
      int ox2 = side_ox2(s), ox3 = side_ox3(s);
      int sj = (ox2 > 0) ? (je - G + 1) : js;
      int ej = (ox2 < 0) ? (js + G - 1) : je;
      int sk = (ox3 > 0) ? (ke - G + 1) : ks;
      int ek = (ox3 < 0) ? (ks + G - 1) : ke;
      bool along_x2 = (ox3 != 0);
      int DirInv = kDinv[p][s], TgtSide = kTgSide[p][s], TgtID = kNbrPanel[p][s];
      int N_blk = along_x2 ? (ej - sj + 1) : (ek - sk + 1);
      int n_start = -N_blk / 2;
      int K = ek - sk + 1, J = ej - sj + 1;
      std::vector<GhostEntry> arr((size_t)K * J);
      std::vector<double> src_x(N_blk), src_coord(N_blk), tgt_x(N_blk), tgt_coord(N_blk);
      int rows_lo = along_x2 ? sk : sj, rows_hi = along_x2 ? ek : ej;
      int other_hi = along_x2 ? ej : ek;
      int lo_along = along_x2 ? sj : sk;
      for (int r = rows_lo; r <= rows_hi; ++r) {
        int k_now, SrcSide;
        if (rows_lo < other_hi - G) { k_now = r - rows_lo; SrcSide = -1; }
        else { k_now = rows_hi - r; SrcSide = 1; }
        for (int m = 0; m < N_blk; ++m) {
          src_x[m] = interp_loc(m - N_blk / 2, N_blk, k_now, false);
          src_coord[m] = PI / 2.0 / N_blk * (m + 0.5) - PI / 4.0;
        }
        for (int m = 0; m < N_blk; ++m) {
          tgt_x[m] = interp_loc(n_start + m, N_blk, k_now, true);
          tgt_coord[m] = DirInv == 1 ? -src_coord[n_start + N_blk / 2 + m]
                                     : src_coord[n_start + N_blk / 2 + m];
        }
        int ptr = 0;
        for (int m = 0; m < N_blk; ++m) {
          while (tgt_x[m] > src_x[ptr + 1]) ptr++;
          double y1 = src_x[ptr], y2 = src_x[ptr + 1], yq = tgt_x[m];
          int a0 = ptr - n_start - N_blk / 2 + lo_along;
          int a1 = ptr + 1 - n_start - N_blk / 2 + lo_along;
          GhostEntry e;
          std::memset(&e, 0, sizeof(e));
          e.src_panel = p;
          if (along_x2) { e.k0 = r; e.j0 = a0; e.k1 = r; e.j1 = a1; }
          else { e.k0 = a0; e.j0 = r; e.k1 = a1; e.j1 = r; }
          e.A = y2 - yq;
          e.B = yq - y1;
          e.C = y2 - y1;
          double tgt_cy, tgt_cz, src_cy, src_cz;
          double scoord = ((y2 - yq) * src_coord[ptr] + (yq - y1) * src_coord[ptr + 1]) / (y2 - y1);
          if (along_x2) {
            tgt_cy = tan(tgt_coord[m]);
            tgt_cz = tan(TgtSide * (PI / 2.0 / (N_blk) * (k_now + 0.5) + PI / 4.0));
            src_cz = tan(SrcSide * (-PI / 2.0 / (N_blk) * (k_now + 0.5) + PI / 4.0));
            src_cy = tan(scoord);
          } else {
            tgt_cz = tan(tgt_coord[m]);
            tgt_cy = tan(TgtSide * (PI / 2.0 / (N_blk) * (k_now + 0.5) + PI / 4.0));
            src_cy = tan(SrcSide * (-PI / 2.0 / (N_blk) * (k_now + 0.5) + PI / 4.0));
            src_cz = tan(scoord);
          }
          e.ss = sqrt(1 + src_cy * src_cy + src_cz * src_cz) / sqrt(1 + src_cy * src_cy) /
                 sqrt(1 + src_cz * src_cz);
          e.cs = -src_cy * src_cz / sqrt(1 + src_cy * src_cy) / sqrt(1 + src_cz * src_cz);
          rll_from_abp_coef(src_cy, src_cz, blockID, e.r);
          if (!along_x2) {
            bool swap = ((TgtID == 1 || TgtID == 5) && (blockID == 3 || blockID == 4)) ||
                        ((TgtID == 3 || TgtID == 4) && (blockID == 1 || blockID == 5));
            if (swap) std::swap(tgt_cy, tgt_cz);
          }
          abp_from_rll_coef(tgt_cy, tgt_cz, TgtID, e.q);
          e.ct = -tgt_cy * tgt_cz / sqrt(1 + tgt_cy * tgt_cy) / sqrt(1 + tgt_cz * tgt_cz);
          int kk = along_x2 ? (r - sk) : m;
          int jj = along_x2 ? m : (r - sj);
          arr[(size_t)kk * J + jj] = e;
        }
      }
      // traversal of the packed buffer
      std::vector<int> seq;
      seq.reserve(arr.size());
      switch (kPackOrder[p][s]) {
        case 0: for (int k = 0; k < K; ++k) for (int j = 0; j < J; ++j) seq.push_back(k * J + j); break;
        case 1: for (int j = J - 1; j >= 0; --j) for (int k = 0; k < K; ++k) seq.push_back(k * J + j); break;
        case 2: for (int k = K - 1; k >= 0; --k) for (int j = J - 1; j >= 0; --j) seq.push_back(k * J + j); break;
        default: for (int j = 0; j < J; ++j) for (int k = K - 1; k >= 0; --k) seq.push_back(k * J + j); break;
      }
      // receiver unpacks in plain (k, j) order into its ghost band
      int tp = kNbrPanel[p][s] - 1, ts = kNbrSide[p][s];
      int tox2 = side_ox2(ts), tox3 = side_ox3(ts);
      int rsj, rej, rsk, rek;
      if (tox2 < 0) { rsj = js - G; rej = js - 1; } else if (tox2 > 0) { rsj = je + 1; rej = je + G; } else { rsj = js; rej = je; }
      if (tox3 < 0) { rsk = ks - G; rek = ks - 1; } else if (tox3 > 0) { rsk = ke + 1; rek = ke + G; } else { rsk = ks; rek = ke; }
      size_t q = 0;
      for (int k = rsk; k <= rek; ++k)
        for (int j = rsj; j <= rej; ++j) {
          t.ghost_map[((size_t)tp * t.nc3 + k) * t.nc2 + j] = (int)t.ghost.size();
          t.ghost.push_back(arr[seq[q++]]);
        }
    }
}

// Edge face states: emulate sendNeighborBlocks / recvNeighborBlocks.
static void build_edge_table(HostTables& t) {
  int N = t.N;
  t.edge.assign((size_t)6 * 4 * N, EdgeEntry());
  for (int p = 0; p < 6; ++p)
    for (int s = 0; s < 4; ++s) {
      int blockID = p + 1;
      int ox2 = side_ox2(s), ox3 = side_ox3(s);
      int tp = kNbrPanel[p][s] - 1, ts = kNbrSide[p][s];
      int tox2 = side_ox2(ts), tox3 = side_ox3(ts);
      int dinv = kDinv[p][s];
      for (int b = 0; b < N; ++b) {
        int a_s = dinv ? (N - 1 - b) : b;  // sender's along index
        double x2s, x3s, x2d, x3d, pos_along;
        if (ox2 == 1) { x2s = PI / 4.0; x3s = t.x3v[p][G + a_s]; pos_along = x3s; }
        else if (ox2 == -1) { x2s = -PI / 4.0; x3s = t.x3v[p][G + a_s]; pos_along = x3s; }
        else if (ox3 == 1) { x2s = t.x2v[p][G + a_s]; x3s = PI / 4.0; pos_along = x2s; }
        else { x2s = t.x2v[p][G + a_s]; x3s = -PI / 4.0; pos_along = x2s; }
        double pa = dinv ? -pos_along : pos_along;
        if (tox2 == 1) { x2d = PI / 4.0; x3d = pa; }
        else if (tox2 == -1) { x2d = -PI / 4.0; x3d = pa; }
        else if (tox3 == 1) { x2d = pa; x3d = PI / 4.0; }
        else { x2d = pa; x3d = -PI / 4.0; }
        x2d = tan(x2d); x3d = tan(x3d); x2s = tan(x2s); x3s = tan(x3s);
        EdgeEntry& e = t.edge[((size_t)tp * 4 + ts) * N + b];
        e.src_panel = p;
        e.src_side = s;
        e.src_along = a_s;
        e.pad = 0;
        rll_from_abp_coef(x2s, x3s, blockID, e.r);
        abp_from_rll_coef(x2d, x3d, kNbrPanel[p][s], e.q);
      }
    }
}

void panel_neighbor(int p, int s, int* tp, int* ts) {
  *tp = kNbrPanel[p][s] - 1;
  *ts = kNbrSide[p][s];
}

bool build_tables(const exo_config& cfg, HostTables& t, std::string* err) {
  if (cfg.N < 6 || (cfg.N % 2) != 0) {
    if (err) *err = "N must be even and >= 6 (one block per panel, even edge count)";
    return false;
  }
  if (cfg.L < 1) {
    if (err) *err = "L must be >= 1";
    return false;
  }
  t.N = cfg.N;
  t.L = cfg.L;
  t.nc1 = cfg.L + 2 * G;
  t.nc2 = t.nc3 = cfg.N + 2 * G;
  build_mesh(cfg, t);
  build_metric(cfg, t);
  build_ghost_table(t);
  build_edge_table(t);
  // every ghost-band cell is mapped once and every source cell is interior
  // (the kernels index with these values unchecked)
  int lo = G, hi = G + cfg.N - 1;
  for (int p = 0; p < 6; ++p)
    for (int k = 0; k < t.nc3; ++k)
      for (int j = 0; j < t.nc2; ++j) {
        bool kin = k >= lo && k <= hi, jin = j >= lo && j <= hi;
        int e = t.ghost_map[((size_t)p * t.nc3 + k) * t.nc2 + j];
        bool band = kin != jin;
        if (band != (e >= 0) || e >= (int)t.ghost.size()) {
          if (err) *err = "internal: ghost table does not cover the ghost bands";
          return false;
        }
        if (e < 0) continue;
        const GhostEntry& g = t.ghost[e];
        if (g.src_panel < 0 || g.src_panel > 5 || g.k0 < lo || g.k0 > hi || g.k1 < lo ||
            g.k1 > hi || g.j0 < lo || g.j0 > hi || g.j1 < lo || g.j1 > hi || !(g.C != 0.)) {
          if (err) *err = "internal: ghost source cell outside the neighbour's interior";
          return false;
        }
      }
  for (const EdgeEntry& e : t.edge)
    if (e.src_panel < 0 || e.src_panel > 5 || e.src_side < 0 || e.src_side > 3 ||
        e.src_along < 0 || e.src_along >= cfg.N) {
      if (err) *err = "internal: edge table entry out of range";
      return false;
    }
  return true;
}

}  // namespace exo
