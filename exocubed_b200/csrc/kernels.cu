// kernels.cu -- sm_100a kernels of the cubed-sphere finite-volume step (FP64).
//
// One stage of SSPRK(3,3) is five launches:
//   k_flux_x1     per radial column: hydrostatic decomposition, WENO5 in x1,
//                 restore, Riemann solve -> x1 face fluxes         (exo3 only)
//   k_flux_x23    per horizontal face: WENO5 on both sides; at panel edges the
//                 outer state is the neighbour panel's own reconstruction,
//                 rotated into this panel's basis; Riemann solve -> x2/x3 fluxes
//   k_update      per cell: RK register average, flux divergence, geometric
//                 source, gravity / Coriolis -> u (exo2) or du (exo3)
//   k_implicit    per radial column: 5x5 block-tridiagonal vertical correction,
//                 u += du, AirParcel round trip on the last stage (exo3)
//   k_prim_ghost  per cell incl. ghosts: ConservedToPrimitive of the interior,
//                 of the ghost bands interpolated from the neighbour panels and
//                 of the reflected x1 ghosts; CFL time-step candidate
// Every arithmetic expression is written in the order of the reference so the
// parity build (--fmad=false) reproduces the CPU restatement bit for bit where
// no transcendental function is involved.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "exo_internal.h"

namespace exo {

namespace {

constexpr double TINY_NUMBER = 1.0e-20;
constexpr double WENO_EPS = 1.0e-7;

__device__ __forceinline__ double sqr(double x) { return x * x; }

__device__ __forceinline__ size_t idx(const DevView& v, int p, int n, int k, int j, int i) {
  return ((((size_t)p * v.nv + n) * v.nc3 + k) * v.nc2 + j) * v.nc1 + i;
}
__device__ __forceinline__ double geo(const DevView& v, int f, int p, int k, int j) {
  return v.geo[(((size_t)f * 6 + p) * v.nc3 + k) * v.nc2 + j];
}

// interp_weno5(phip2, phip1, phi, phim1, phim2): the face value between the
// 2nd and 3rd argument (Jiang & Shu 1996; orientation of tests/test_weno.cpp)
__device__ __forceinline__ double weno5(double phip2, double phip1, double phi,
                                        double phim1, double phim2) {
  double p0 = (1.0 / 3.0) * phim2 - (7.0 / 6.0) * phim1 + (11.0 / 6.0) * phi;
  double p1 = (-1.0 / 6.0) * phim1 + (5.0 / 6.0) * phi + (1.0 / 3.0) * phip1;
  double p2 = (1.0 / 3.0) * phi + (5.0 / 6.0) * phip1 - (1.0 / 6.0) * phip2;
  double b0 = 13. / 12. * sqr(phim2 - 2. * phim1 + phi) +
              .25 * sqr(phim2 - 4. * phim1 + 3. * phi);
  double b1 = 13. / 12. * sqr(phim1 - 2. * phi + phip1) + .25 * sqr(phim1 - phip1);
  double b2 = 13. / 12. * sqr(phi - 2. * phip1 + phip2) +
              .25 * sqr(3. * phi - 4. * phip1 + phip2);
  double a0 = 0.1 / ((b0 + WENO_EPS) * (b0 + WENO_EPS));
  double a1 = 0.6 / ((b1 + WENO_EPS) * (b1 + WENO_EPS));
  double a2 = 0.3 / ((b2 + WENO_EPS) * (b2 + WENO_EPS));
  return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}

// right-face value (face c+1) and left-face value (face c) of cell c on a
// strided line q[c*s]
__device__ __forceinline__ double weno_r(const double* q, long s, int c) {
  return weno5(q[(c + 2) * s], q[(c + 1) * s], q[c * s], q[(c - 1) * s], q[(c - 2) * s]);
}
__device__ __forceinline__ double weno_l(const double* q, long s, int c) {
  return weno5(q[(c - 2) * s], q[(c - 1) * s], q[c * s], q[(c + 1) * s], q[(c + 2) * s]);
}

// ------------------------------------------------------------------ EOS ----
// CubedSphereUtility::CovariantToContravariant (cubed_sphere_utility.hpp:22-31)
__device__ __forceinline__ void cov_to_contra(double* a, double cth) {
  double v = a[IVY], w = a[IVZ];
  double sth2 = 1. - cth * cth;
  a[IVY] = v / sth2 - w * cth / sth2;
  a[IVZ] = -v * cth / sth2 + w / sth2;
}
__device__ __forceinline__ void contra_to_cov(double* a, double cth) {
  double v = a[IVY], w = a[IVZ];
  a[IVY] = v + w * cth;
  a[IVZ] = w + v * cth;
}

// ConservedToPrimitive of one cell (shallow_yz_hydro.cpp:42-67,
// ideal_moist_hydro.cpp:77-159); returns 1 if the state is invalid
__device__ __forceinline__ int cons_to_prim(const DevView& v, const double* c, double* w,
                                            double cth) {
  int bad = 0;
  if (v.eqn == EXO_EQN_SHALLOW_YZ) {
    double dfloor = (double)sqrtf(1024 * FLT_MIN);
    double ud = c[IDN];
    ud = (ud > dfloor) ? ud : dfloor;
    w[IDN] = ud;
    w[IVX] = 0.;
    w[IVY] = c[IVY];
    w[IVZ] = c[IVZ];
    double di = 1. / ud;
    cov_to_contra(w, cth);
    w[IVY] *= di;
    w[IVZ] *= di;
  } else {
    double gm1 = v.gamma - 1.0;
    double density = 0.;
    density += c[IDN];
    w[IDN] = density;
    double di = 1. / density;
    if ((w[IDN] < 0.) || isnan(w[IDN])) bad = 1;
    double fsig = 1., feps = 1.;
    w[IVX] = c[IVX] * di;
    w[IVY] = c[IVY] * di;
    w[IVZ] = c[IVZ] * di;
    cov_to_contra(w, cth);
    double KE = 0.5 * (c[IVX] * w[IVX] + c[IVY] * w[IVY] + c[IVZ] * w[IVZ]);
    w[IPR] = gm1 * (c[IEN] - KE) * feps / fsig;
    if ((w[IPR] < 0.) || isnan(w[IPR])) bad = 1;
  }
  return bad;
}

__device__ __forceinline__ void prim_to_cons(const DevView& v, const double* w, double* c,
                                             double cth) {
  if (v.eqn == EXO_EQN_SHALLOW_YZ) {
    double wd = w[IDN];
    c[IDN] = wd;
    c[IVX] = 0.;
    c[IVY] = w[IVY];
    c[IVZ] = w[IVZ];
    contra_to_cov(c, cth);
    c[IVY] *= wd;
    c[IVZ] *= wd;
  } else {
    double igm1 = 1.0 / (v.gamma - 1.0);
    double wd = w[IDN];
    c[IDN] = wd;
    c[IVX] = w[IVX] * wd;
    c[IVY] = w[IVY] * wd;
    c[IVZ] = w[IVZ] * wd;
    contra_to_cov(c, cth);
    double KE = 0.5 * (c[IVX] * w[IVX] + c[IVY] * w[IVY] + c[IVZ] * w[IVZ]);
    double fsig = 1., feps = 1.;
    c[IEN] = igm1 * w[IPR] * fsig / feps + KE;
  }
}

// ------------------------------------------------------ Riemann solvers ----
struct FaceGeo {
  double cosf, sinf, cthp, cthc;
};

__device__ __forceinline__ void prim_to_local(int ivx, const FaceGeo& fg, double* w) {
  if (ivx == IVY) {  // PrimToLocal2, gnomonic_equiangle.cpp:604-660
    double g23 = fg.cosf, g33 = 1.0, gi22 = 1.0 / (fg.sinf * fg.sinf);
    double T11 = 1.0, T22 = 1.0 / sqrt(gi22), T32 = g23 / sqrt(g33), T33 = sqrt(g33);
    double uu1 = w[IVX], uu2 = w[IVY], uu3 = w[IVZ];
    w[IVX] = T11 * uu1;
    w[IVY] = T22 * uu2;
    w[IVZ] = T32 * uu2 + T33 * uu3;
  } else if (ivx == IVZ) {  // PrimToLocal3, :662-718
    double g23 = fg.cosf, g22 = 1.0, gi33 = 1.0 / (fg.sinf * fg.sinf);
    double T11 = 1.0, T22 = sqrt(g22), T23 = g23 / sqrt(g22), T33 = 1.0 / sqrt(gi33);
    double uu1 = w[IVX], uu2 = w[IVY], uu3 = w[IVZ];
    w[IVX] = T11 * uu1;
    w[IVY] = T22 * uu2 + T23 * uu3;
    w[IVZ] = T33 * uu3;
  }
}

__device__ __forceinline__ void flux_to_global(int ivx, const FaceGeo& fg, double* f) {
  if (ivx == IVY) {  // FluxToGlobal2, :752-791
    double g23 = fg.cosf, g33 = 1.0, gi22 = 1.0 / (fg.sinf * fg.sinf);
    double T11 = 1.0, T22 = sqrt(gi22), T32 = -sqrt(gi22) * g23 / g33, T33 = 1.0 / sqrt(g33);
    double txx = f[IVX], txy = f[IVY], txz = f[IVZ];
    f[IVX] = T11 * txx;
    f[IVY] = T22 * txy;
    f[IVZ] = T32 * txy + T33 * txz;
  } else if (ivx == IVZ) {  // FluxToGlobal3, :793-832
    double g23 = fg.cosf, g22 = 1.0, gi33 = 1.0 / (fg.sinf * fg.sinf);
    double T11 = 1.0, T22 = 1.0 / sqrt(g22), T23 = -g23 / g22 * sqrt(gi33), T33 = sqrt(gi33);
    double txx = f[IVX], txy = f[IVY], txz = f[IVZ];
    f[IVX] = T11 * txx;
    f[IVY] = T22 * txy + T23 * txz;
    f[IVZ] = T33 * txz;
  }
}

// roe_shallow_yz.cpp:18-122
__device__ void riemann_roe_shallow(int ivx, const FaceGeo& fg, double* wli, double* wri,
                                    double* flx) {
  int ivy = ivx == IVY ? IVZ : IVY;
  prim_to_local(ivx, fg, wli);
  prim_to_local(ivx, fg, wri);
  double ubar = (wli[ivx] * sqrt(wli[IDN]) + wri[ivx] * sqrt(wri[IDN])) /
                (sqrt(wli[IDN]) + sqrt(wri[IDN]));
  double vbar = (wli[ivy] * sqrt(wli[IDN]) + wri[ivy] * sqrt(wri[IDN])) /
                (sqrt(wli[IDN]) + sqrt(wri[IDN]));
  double cbar = sqrt(0.5 * (wli[IDN] + wri[IDN]));
  double delh = wri[IDN] - wli[IDN];
  double delu = wri[ivx] - wli[ivx];
  double delv = wri[ivy] - wli[ivy];
  double hbar = sqrt(wli[IDN] * wri[IDN]);
  double a1 = 0.5 * (cbar * delh - hbar * delu) / cbar;
  double a2 = hbar * delv;
  double a3 = 0.5 * (cbar * delh + hbar * delu) / cbar;
  double w00 = a1, w01 = a1 * (ubar - cbar), w02 = a1 * vbar;
  double w10 = 0., w11 = 0., w12 = a2;
  double w20 = a3, w21 = a3 * (ubar + cbar), w22 = a3 * vbar;
  double s0 = fabs(ubar - cbar), s1 = fabs(ubar), s2 = fabs(ubar + cbar);
  flx[IVZ] = 0.;
  flx[IDN] = 0.5 * (wli[IDN] * wli[ivx] + wri[IDN] * wri[ivx]);
  flx[ivx] = 0.5 * (wli[IDN] * wli[ivx] * wli[ivx] + 0.5 * wli[IDN] * wli[IDN] +
                    wri[IDN] * wri[ivx] * wri[ivx] + 0.5 * wri[IDN] * wri[IDN]);
  flx[ivy] = 0.5 * (wli[IDN] * wli[ivx] * wli[ivy] + wri[IDN] * wri[ivx] * wri[ivy]);
  flx[IVX] = 0.;
  flx[IDN] -= 0.5 * s0 * w00;
  flx[ivx] -= 0.5 * s0 * w01;
  flx[ivy] -= 0.5 * s0 * w02;
  flx[IDN] -= 0.5 * s1 * w10;
  flx[ivx] -= 0.5 * s1 * w11;
  flx[ivy] -= 0.5 * s1 * w12;
  flx[IDN] -= 0.5 * s2 * w20;
  flx[ivx] -= 0.5 * s2 * w21;
  flx[ivy] -= 0.5 * s2 * w22;
  if (ivx == IVX) {
    flx[IVX] = 0.;
    return;
  }
  flux_to_global(ivx, fg, flx);
  double ty = flx[ivx], tz = flx[ivy];
  flx[ivx] = ty + tz * fg.cthp;
  flx[ivy] = tz + ty * fg.cthp;
}

// lmars.cpp:24-110 (NVAPOR = NCLOUD = 0), no projection
__device__ void riemann_lmars(double gamma, int ivx, const double* wli, const double* wri,
                              double* flx) {
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
  double fsig = 1., feps = 1.;
  double kappal = 1. / (gamma - 1.) * fsig / feps;
  double kappar = 1. / (gamma - 1.) * fsig / feps;
  double hl = wli[IPR] / wli[IDN] * (kappal + 1.) +
              0.5 * (sqr(wli[ivx]) + sqr(wli[ivy]) + sqr(wli[ivz]));
  double hr = wri[IPR] / wri[IDN] * (kappar + 1.) +
              0.5 * (sqr(wri[ivx]) + sqr(wri[ivy]) + sqr(wri[ivz]));
  double rhobar = 0.5 * (wli[IDN] + wri[IDN]);
  double cbar = sqrt(0.5 * (1. + (1. / kappar + 1. / kappal) / 2.) *
                     (wli[IPR] + wri[IPR]) / rhobar);
  double pbar = 0.5 * (wli[IPR] + wri[IPR]) + 0.5 * (rhobar * cbar) * (wli[ivx] - wri[ivx]);
  double ubar = 0.5 * (wli[ivx] + wri[ivx]) + 0.5 / (rhobar * cbar) * (wli[IPR] - wri[IPR]);
  double rdl = 1., rdr = 1.;
  if (ubar > 0.) {
    flx[IDN] = ubar * wli[IDN] * rdl;
    flx[ivx] = ubar * wli[IDN] * wli[ivx] + pbar;
    flx[ivy] = ubar * wli[IDN] * wli[ivy];
    flx[ivz] = ubar * wli[IDN] * wli[ivz];
    flx[IEN] = ubar * wli[IDN] * hl;
  } else {
    flx[IDN] = ubar * wri[IDN] * rdr;
    flx[ivx] = ubar * wri[IDN] * wri[ivx] + pbar;
    flx[ivy] = ubar * wri[IDN] * wri[ivy];
    flx[ivz] = ubar * wri[IDN] * wri[ivz];
    flx[IEN] = ubar * wri[IDN] * hr;
  }
}

// hllc_transform.cpp:24-263
__device__ void riemann_hllc(double gamma, int ivx, const FaceGeo& fg, double* wl, double* wr,
                             double* flx) {
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
  double gm1 = gamma - 1.0, igm1 = 1.0 / gm1;
  prim_to_local(ivx, fg, wl);
  prim_to_local(ivx, fg, wr);
  double wli[5], wri[5], fl[5], fr[5];
  wli[IDN] = wl[IDN]; wli[IVX] = wl[ivx]; wli[IVY] = wl[ivy]; wli[IVZ] = wl[ivz]; wli[IPR] = wl[IPR];
  wri[IDN] = wr[IDN]; wri[IVX] = wr[ivx]; wri[IVY] = wr[ivy]; wri[IVZ] = wr[ivz]; wri[IPR] = wr[IPR];
  double fsig = 1., feps = 1.;
  double cl = sqrt((1. + (gamma - 1) * feps / fsig) * wli[IPR] / wli[IDN]);
  double cr = sqrt((1. + (gamma - 1) * feps / fsig) * wri[IPR] / wri[IDN]);
  double KE_l, KE_r;
  if (ivx == IVX) {
    double cth = fg.cthc, vy, vz;
    vy = wli[IVY] + wli[IVZ] * cth;
    vz = wli[IVZ] + wli[IVY] * cth;
    KE_l = 0.5 * wli[IDN] * (sqr(wli[IVX]) + wli[IVY] * vy + wli[IVZ] * vz);
    vy = wri[IVY] + wri[IVZ] * cth;
    vz = wri[IVZ] + wri[IVY] * cth;
    KE_r = 0.5 * wri[IDN] * (sqr(wri[IVX]) + wri[IVY] * vy + wri[IVZ] * vz);
  } else {
    KE_l = 0.5 * wli[IDN] * (sqr(wli[IVX]) + sqr(wli[IVY]) + sqr(wli[IVZ]));
    KE_r = 0.5 * wri[IDN] * (sqr(wri[IVX]) + sqr(wri[IVY]) + sqr(wri[IVZ]));
  }
  double el = wli[IPR] * igm1 + KE_l;
  double er = wri[IPR] * igm1 + KE_r;
  double rhoa = .5 * (wli[IDN] + wri[IDN]);
  double ca = .5 * (cl + cr);
  double pmid = .5 * (wli[IPR] + wri[IPR] + (wli[IVX] - wri[IVX]) * rhoa * ca);
  double ql = (pmid <= wli[IPR]) ? 1.0
              : sqrt(1.0 + (gamma + 1) / (2 * gamma) * (pmid / wli[IPR] - 1.0));
  double qr = (pmid <= wri[IPR]) ? 1.0
              : sqrt(1.0 + (gamma + 1) / (2 * gamma) * (pmid / wri[IPR] - 1.0));
  double al = wli[IVX] - cl * ql;
  double ar = wri[IVX] + cr * qr;
  double bp = ar > 0.0 ? ar : (TINY_NUMBER);
  double bm = al < 0.0 ? al : -(TINY_NUMBER);
  double vxl = wli[IVX] - al;
  double vxr = wri[IVX] - ar;
  double tl = wli[IPR] + vxl * wli[IDN] * wli[IVX];
  double tr = wri[IPR] + vxr * wri[IDN] * wri[IVX];
  double ml = wli[IDN] * vxl;
  double mr = -(wri[IDN] * vxr);
  double am = (tl - tr) / (ml + mr);
  double cp = (ml * tr + mr * tl) / (ml + mr);
  cp = cp > 0.0 ? cp : 0.0;
  vxl = wli[IVX] - bm;
  vxr = wri[IVX] - bp;
  fl[IDN] = wli[IDN] * vxl;
  fr[IDN] = wri[IDN] * vxr;
  fl[IVX] = wli[IDN] * wli[IVX] * vxl + wli[IPR];
  fr[IVX] = wri[IDN] * wri[IVX] * vxr + wri[IPR];
  fl[IVY] = wli[IDN] * wli[IVY] * vxl;
  fr[IVY] = wri[IDN] * wri[IVY] * vxr;
  fl[IVZ] = wli[IDN] * wli[IVZ] * vxl;
  fr[IVZ] = wri[IDN] * wri[IVZ] * vxr;
  fl[IEN] = el * vxl + wli[IPR] * wli[IVX];
  fr[IEN] = er * vxr + wri[IPR] * wri[IVX];
  double sl, sr, sm;
  if (am >= 0.0) {
    sl = am / (am - bm);
    sr = 0.0;
    sm = -bm / (am - bm);
  } else {
    sl = 0.0;
    sr = -am / (bp - am);
    sm = bp / (bp - am);
  }
  flx[IDN] = sl * fl[IDN] + sr * fr[IDN];
  flx[ivx] = sl * fl[IVX] + sr * fr[IVX] + sm * cp;
  flx[ivy] = sl * fl[IVY] + sr * fr[IVY];
  flx[ivz] = sl * fl[IVZ] + sr * fr[IVZ];
  flx[IEN] = sl * fl[IEN] + sr * fr[IEN] + sm * cp * am;
  flux_to_global(ivx, fg, flx);
  double ty = flx[IVY], tz = flx[IVZ];
  flx[IVY] = ty + tz * fg.cthp;
  flx[IVZ] = tz + ty * fg.cthp;
}

// lmars_shallow_yz.cpp:18-93
__device__ void riemann_lmars_shallow(int ivx, const FaceGeo& fg, double* wli, double* wri,
                                      double* flx) {
  int ivy = ivx == IVY ? IVZ : IVY;
  prim_to_local(ivx, fg, wli);
  prim_to_local(ivx, fg, wri);
  double cbar = sqrt(0.5 * (wli[IDN] + wri[IDN]));
  double hbar = 0.5 * (wli[IDN] + wri[IDN]) + 0.5 * cbar * (wli[ivx] - wri[ivx]);
  double ubar = 0.5 * (wli[ivx] + wri[ivx]) + 0.5 / cbar * (wli[IDN] - wri[IDN]);
  flx[IVZ] = 0.;
  if (ubar > 0.) {
    flx[IDN] = ubar * wli[IDN];
    flx[ivx] = ubar * wli[IDN] * wli[ivx] + 0.5 * hbar * hbar;
    flx[ivy] = ubar * wli[IDN] * wli[ivy];
  } else {
    flx[IDN] = ubar * wri[IDN];
    flx[ivx] = ubar * wri[IDN] * wri[ivx] + 0.5 * hbar * hbar;
    flx[ivy] = ubar * wri[IDN] * wri[ivy];
  }
  flx[IVX] = 0.;
  if (ivx == IVX) return;
  flux_to_global(ivx, fg, flx);
  double ty = flx[ivx], tz = flx[ivy];
  flx[ivx] = ty + tz * fg.cthp;
  flx[ivy] = tz + ty * fg.cthp;
}

__device__ __forceinline__ void riemann(int rsolver, double gamma, int ivx, const FaceGeo& fg,
                                        double* wl, double* wr, double* flx) {
  switch (rsolver) {
    case EXO_RS_ROE_SHALLOW: riemann_roe_shallow(ivx, fg, wl, wr, flx); break;
    case EXO_RS_LMARS: riemann_lmars(gamma, ivx, wl, wr, flx); break;
    case EXO_RS_HLLC: riemann_hllc(gamma, ivx, fg, wl, wr, flx); break;
    default: riemann_lmars_shallow(ivx, fg, wl, wr, flx); break;
  }
}

// ----------------------------------------------------- k_prim_ghost ------
// Conserved value of variable n at cell (p,k,j,i) where (k,j) is interior or
// in a ghost band; vectors (IVY, IVZ) come back together.
__device__ __forceinline__ void load_cons(const DevView& v, int p, int k, int j, int i,
                                          bool interior, double* c) {
  if (interior) {
    for (int n = 0; n < v.nv; ++n) c[n] = v.u[idx(v, p, n, k, j, i)];
    return;
  }
  const GhostEntry& e = v.ghost[v.ghost_map[((size_t)p * v.nc3 + k) * v.nc2 + j]];
  int sp = e.src_panel;
  for (int n = 0; n < v.nv; ++n) {
    if (n == IVY || n == IVZ) continue;
    double v1 = v.u[idx(v, sp, n, e.k0, e.j0, i)];
    double v2 = v.u[idx(v, sp, n, e.k1, e.j1, i)];
    c[n] = (e.A * v1 + e.B * v2) / e.C;
  }
  double v1y = v.u[idx(v, sp, IVY, e.k0, e.j0, i)], v1z = v.u[idx(v, sp, IVZ, e.k0, e.j0, i)];
  double v2y = v.u[idx(v, sp, IVY, e.k1, e.j1, i)], v2z = v.u[idx(v, sp, IVZ, e.k1, e.j1, i)];
  double vy = (e.A * v1y + e.B * v2y) / e.C;
  double vz = (e.A * v1z + e.B * v2z) / e.C;
  double sth = e.ss, cth = e.cs;
  double vyt = vy, vzt = vz;
  vy = vyt / sth / sth - vzt * cth / sth / sth;
  vz = vzt / sth / sth - vyt * cth / sth / sth;
  double U = e.r[0] * vy + e.r[1] * vz;
  double V = e.r[2] * vy + e.r[3] * vz;
  vy = e.q[0] * U + e.q[1] * V;
  vz = e.q[2] * U + e.q[3] * V;
  vyt = vy;
  vzt = vz;
  c[IVY] = vyt + vzt * e.ct;
  c[IVZ] = vzt + vyt * e.ct;
}

__global__ void k_prim_ghost(DevView v, int compute_dt) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)6 * v.cells;
  if (tid >= total) return;
  int i = (int)(tid % v.nc1);
  size_t r = tid / v.nc1;
  int j = (int)(r % v.nc2);
  r /= v.nc2;
  int k = (int)(r % v.nc3);
  int p = (int)(r / v.nc3);
  bool kin = (k >= v.ks && k <= v.ke), jin = (j >= v.js && j <= v.je);
  if (!kin && !jin) return;  // corner: never read on the path
  int ii = i;
  bool mirror = false;
  if (i < v.is) { ii = 2 * v.is - 1 - i; mirror = true; }
  else if (i > v.ie) { ii = 2 * v.ie + 1 - i; mirror = true; }
  double c[5], w[5];
  load_cons(v, p, k, j, ii, kin && jin, c);
  double cth = geo(v, GCOSC, p, k, j);
  int bad = cons_to_prim(v, c, w, cth);
  if (mirror) w[IVX] = -w[IVX];
  for (int n = 0; n < v.nv; ++n) v.w[idx(v, p, n, k, j, i)] = w[n];
  if (!(kin && jin) || mirror) return;
  if (bad) atomicOr(&v.sc->invalid, 1);
  if (compute_dt) {
    // Hydro::NewBlockTimeStep with patches/21.new_blockdt.patch:23-35
    bool shallow = (v.eqn == EXO_EQN_SHALLOW_YZ);
    double cs;
    if (shallow) cs = sqrt(w[IDN]);
    else {
      double fsig = 1., feps = 1.;
      cs = sqrt((1. + (v.gamma - 1) * feps / fsig) * w[IPR] / w[IDN]);
    }
    double dt1 = v.dx1f[i], dt2 = v.x1v[i] * geo(v, GDX2A, p, k, j);
    double dt3 = v.x1v[i] * geo(v, GDX3A, p, k, j);
    double speed1 = fmax(0., (fabs(w[IVX]) + cs));
    double speed2 = fmax(0., (fabs(w[IVY]) + cs));
    double speed3 = fmax(0., (fabs(w[IVZ]) + cs));
    if ((v.implicit_flag & 1) && (v.N > 1)) dt1 /= v.cfl * fabs(w[IVX]);
    else dt1 /= speed1;
    if (v.implicit_flag & 2) dt2 /= v.cfl * fabs(w[IVY]);
    else dt2 /= speed2;
    if (v.implicit_flag & 4) dt3 /= v.cfl * fabs(w[IVZ]);
    else dt3 /= speed3;
    double m = fmin(dt2, dt3);
    if (!shallow) m = fmin(dt1, m);
    if (m >= 0.) atomicMin(&v.sc->dtmin_bits, (unsigned long long)__double_as_longlong(m));
  }
}

// ------------------------------------------------------------ k_flux_x1 ---
// One CTA per interior radial column.
__global__ void k_flux_x1(DevView v) {
  extern __shared__ double sm[];
  int col = blockIdx.x;
  int j = v.js + col % v.N;
  int k = v.ks + (col / v.N) % v.N;
  int p = col / (v.N * v.N);
  int nc1 = v.nc1, nv = v.nv;
  double* wc = sm;              // [nv][nc1]
  double* psf = sm + nv * nc1;  // [nc1+1]
  __shared__ double s_gam, s_expf;
  for (int t = threadIdx.x; t < nv * nc1; t += blockDim.x)
    wc[t] = v.w[idx(v, p, t / nc1, k, j, t % nc1)];
  __syncthreads();
  bool decomp = (v.grav != 0.);
  if (decomp) {
    // Decomposition::ChangeToPerturbation (change_to_perturbation.cpp:39-157)
    if (threadIdx.x == 0) {
      double grav = -v.grav;
      int is = v.is, ie = v.ie;
      double* wd = wc + IDN * nc1;
      double* wp = wc + IPR * nc1;
      double RdTv = wp[ie] / wd[ie];
      psf[ie + 1] = wp[ie] * exp(-grav * v.dx1f[ie] / (2 * RdTv));
      for (int i = ie; i >= is; --i) psf[i] = psf[i + 1] + grav * wd[i] * v.dx1f[i];
      for (int i = 1; i <= G; ++i) psf[is - i] = psf[is + i];
      for (int i = 1; i <= G; ++i) psf[ie + i + 1] = psf[ie + 1 - i];
      double gammad = v.gamma, fsig = 1., feps = 1.;
      double gam = 1. + (gammad - 1.) * feps / fsig;
      double ent = log(wp[is]) - gam * log(wd[is]);
      s_gam = gam;
      s_expf = exp(-ent / gam);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nc1; i += blockDim.x) {
      double psv, dsv;
      if (fabs(psf[i] - psf[i + 1]) < 1.E-6)
        psv = (psf[i] + psf[i + 1]) / 2.;
      else
        psv = (psf[i] - psf[i + 1]) / log(psf[i] / psf[i + 1]);
      dsv = pow(psv, 1. / s_gam) * s_expf;
      wc[IPR * nc1 + i] -= psv;
      wc[IDN * nc1 + i] -= dsv;
    }
    __syncthreads();
  }
  FaceGeo fg{0., 1., geo(v, GCTHP1, p, k, j), geo(v, GCOSC, p, k, j)};
  for (int f = threadIdx.x; f <= v.L; f += blockDim.x) {
    int i = v.is + f;
    double wl[5], wr[5], fx[5] = {0., 0., 0., 0., 0.};
    for (int n = 0; n < nv; ++n) {
      const double* q = wc + n * nc1;
      wl[n] = weno_r(q, 1, i - 1);
      wr[n] = weno_l(q, 1, i);
    }
    if (decomp) {
      // RestoreFromPerturbation (change_to_perturbation.cpp:159-222)
      double ps = psf[i];
      wr[IPR] += ps;
      if (wr[IPR] < 0.) wr[IPR] = ps;
      wl[IPR] += ps;
      if (wl[IPR] < 0.) wl[IPR] = ps;
      double dsf = pow(ps, 1. / s_gam) * s_expf;
      wr[IDN] += dsf;
      if (wr[IDN] < 0.) wr[IDN] = dsf;
      wl[IDN] += dsf;
      if (wl[IDN] < 0.) wl[IDN] = dsf;
    }
    riemann(v.rsolver, v.gamma, IVX, fg, wl, wr, fx);
    for (int n = 0; n < nv; ++n) v.flux[0][idx(v, p, n, k, j, i)] = fx[n];
  }
}

// ----------------------------------------------------------- k_flux_x23 --
// Interior-side reconstruction of panel p at its own edge face (side s,
// along index a) for radial index i: the state CubedSphere::sendNeighborBlocks
// sends (L at Down/Right edges, R at Up/Left edges).
__device__ __forceinline__ void edge_interior_state(const DevView& v, int p, int s, int a,
                                                    int i, double* st) {
  long s2 = v.nc1, s3 = (long)v.nc1 * v.nc2;
  for (int n = 0; n < v.nv; ++n) {
    if (s == UP || s == DOWN) {
      const double* q = v.w + idx(v, p, n, v.ks + a, 0, i);
      st[n] = (s == DOWN) ? weno_r(q, s2, v.je) : weno_l(q, s2, v.js);
    } else {
      const double* q = v.w + idx(v, p, n, 0, v.js + a, i);
      st[n] = (s == RIGHT) ? weno_r(q, s3, v.ke) : weno_l(q, s3, v.ks);
    }
  }
}

__device__ __forceinline__ void edge_outer_state(const DevView& v, int p, int side, int a,
                                                 int i, double* st) {
  const EdgeEntry& e = v.edge[((size_t)p * 4 + side) * v.N + a];
  edge_interior_state(v, e.src_panel, e.src_side, e.src_along, i, st);
  double V2 = st[IVY], V3 = st[IVZ];
  double U = e.r[0] * V2 + e.r[1] * V3;
  double V = e.r[2] * V2 + e.r[3] * V3;
  st[IVY] = e.q[0] * U + e.q[1] * V;
  st[IVZ] = e.q[2] * U + e.q[3] * V;
}

__global__ void k_flux_x23(DevView v) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t nface = (size_t)6 * v.N * (v.N + 1) * v.L;  // per direction
  if (tid >= 2 * nface) return;
  int dir = tid < nface ? 1 : 2;
  size_t r = dir == 1 ? tid : tid - nface;
  int i = v.is + (int)(r % v.L);
  r /= v.L;
  int k, j;
  int p;
  if (dir == 1) {  // x2 faces: j in [js, je+1], k in [ks, ke]
    j = v.js + (int)(r % (v.N + 1));
    r /= (v.N + 1);
    k = v.ks + (int)(r % v.N);
    p = (int)(r / v.N);
  } else {  // x3 faces: j in [js, je], k in [ks, ke+1]
    j = v.js + (int)(r % v.N);
    r /= v.N;
    k = v.ks + (int)(r % (v.N + 1));
    p = (int)(r / (v.N + 1));
  }
  double wl[5], wr[5], fx[5] = {0., 0., 0., 0., 0.};
  long s2 = v.nc1, s3 = (long)v.nc1 * v.nc2;
  FaceGeo fg;
  int ivx;
  if (dir == 1) {
    for (int n = 0; n < v.nv; ++n) {
      const double* q = v.w + idx(v, p, n, k, 0, i);
      wl[n] = weno_r(q, s2, j - 1);
      wr[n] = weno_l(q, s2, j);
    }
    if (j == v.js) edge_outer_state(v, p, UP, k - v.ks, i, wl);
    else if (j == v.je + 1) edge_outer_state(v, p, DOWN, k - v.ks, i, wr);
    fg = FaceGeo{geo(v, GCOSF2, p, k, j), geo(v, GSINF2, p, k, j), geo(v, GCTHP2, p, k, j),
                 geo(v, GCOSC, p, k, j)};
    ivx = IVY;
  } else {
    for (int n = 0; n < v.nv; ++n) {
      const double* q = v.w + idx(v, p, n, 0, j, i);
      wl[n] = weno_r(q, s3, k - 1);
      wr[n] = weno_l(q, s3, k);
    }
    if (k == v.ks) edge_outer_state(v, p, LEFT, j - v.js, i, wl);
    else if (k == v.ke + 1) edge_outer_state(v, p, RIGHT, j - v.js, i, wr);
    fg = FaceGeo{geo(v, GCOSF3, p, k, j), geo(v, GSINF3, p, k, j), geo(v, GCTHP3, p, k, j),
                 geo(v, GCOSC, p, k, j)};
    ivx = IVZ;
  }
  riemann(v.rsolver, v.gamma, ivx, fg, wl, wr, fx);
  double* F = v.flux[dir];
  for (int n = 0; n < v.nv; ++n) F[idx(v, p, n, k, j, i)] = fx[n];
}

// --------------------------------------------------------------- k_update -
__global__ void k_update(DevView v, int stage) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)6 * v.N * v.N * v.L;
  if (tid >= total) return;
  int i = v.is + (int)(tid % v.L);
  size_t r = tid / v.L;
  int j = v.js + (int)(r % v.N);
  r /= v.N;
  int k = v.ks + (int)(r % v.N);
  int p = (int)(r / v.N);
  const double kBeta[3] = {1.0, 0.25, 2.0 / 3.0};
  double wght = kBeta[stage] * v.sc->dt;
  bool shallow = (v.eqn == EXO_EQN_SHALLOW_YZ);
  int nv = v.nv;
  double un[5];
  // WeightedAve(u1, u, ...) then WeightedAve(u, u1, ...) (SSPRK(3,3) registers)
  for (int n = 0; n < nv; ++n) {
    size_t q = idx(v, p, n, k, j, i);
    double uu = v.u[q];
    if (stage == 0) {
      v.u1[q] = uu;
      un[n] = 0. + 1.0 * uu;
    } else if (stage == 1) {
      un[n] = 0.25 * uu + 0.75 * v.u1[q];
    } else {
      un[n] = (2.0 / 3.0) * uu + (1.0 / 3.0) * v.u1[q];
    }
  }
  // AddFluxDivergence
  double s = geo(v, GSINC, p, k, j);
  double d2 = geo(v, GDX2A, p, k, j), d3 = geo(v, GDX3A, p, k, j);
  double a1 = d2 * d3 * v.x1f[i] * v.x1f[i] * s;
  double a1p = d2 * d3 * v.x1f[i + 1] * v.x1f[i + 1] * s;
  double a2 = v.x1v[i] * geo(v, GDX3A_F2, p, k, j) * v.dx1f[i];
  double a2p = v.x1v[i] * geo(v, GDX3A_F2, p, k, j + 1) * v.dx1f[i];
  double a3 = v.x1v[i] * geo(v, GDX2A_F3, p, k, j) * v.dx1f[i];
  double a3p = v.x1v[i] * geo(v, GDX2A_F3, p, k + 1, j) * v.dx1f[i];
  double vol = v.dx1f[i] * d2 * d3 * v.x1v[i] * v.x1v[i] * s;
  double du[5];
  for (int n = 0; n < nv; ++n) {
    double dflx;
    if (shallow) {
      dflx = (a1p * 0. - a1 * 0.);
    } else {
      dflx = (a1p * v.flux[0][idx(v, p, n, k, j, i + 1)] - a1 * v.flux[0][idx(v, p, n, k, j, i)]);
    }
    dflx += (a2p * v.flux[1][idx(v, p, n, k, j + 1, i)] - a2 * v.flux[1][idx(v, p, n, k, j, i)]);
    dflx += (a3p * v.flux[2][idx(v, p, n, k + 1, j, i)] - a3 * v.flux[2][idx(v, p, n, k, j, i)]);
    if (shallow) {
      un[n] -= wght * dflx / vol;
    } else {
      du[n] = 0.;
      du[n] -= wght * dflx / vol;
    }
  }
  double* out = shallow ? un : du;
  // AddCoordTermsDivergence (gnomonic_equiangle.cpp:834-879)
  {
    double cosine = geo(v, GCOSC, p, k, j);
    double sine2 = s * s;
    double x_ov_rD = (v.x1v[i] * geo(v, GDX3A_F2, p, k, j) * v.dx1f[i] * geo(v, GSINF2, p, k, j) -
                      v.x1v[i] * geo(v, GDX3A_F2, p, k, j + 1) * v.dx1f[i] *
                          geo(v, GSINF2, p, k, j + 1)) / vol;
    double y_ov_rC = (v.x1v[i] * geo(v, GDX2A_F3, p, k, j) * v.dx1f[i] * geo(v, GSINF3, p, k, j) -
                      v.x1v[i] * geo(v, GDX2A_F3, p, k + 1, j) * v.dx1f[i] *
                          geo(v, GSINF3, p, k + 1, j)) / vol;
    double rho = v.w[idx(v, p, IDN, k, j, i)];
    double v1 = v.w[idx(v, p, IVX, k, j, i)], v2 = v.w[idx(v, p, IVY, k, j, i)];
    double v3 = v.w[idx(v, p, IVZ, k, j, i)];
    double radius = v.x1v[i];
    double pr;
    double v_2 = v2 + v3 * cosine;
    double v_3 = v3 + v2 * cosine;
    if (shallow) {
      pr = 0.5 * rho * rho;
    } else {
      pr = v.w[idx(v, p, IPR, k, j, i)];
      double src1 = (2.0 * pr + rho * (v2 * v_2 + v3 * v_3)) / radius;
      out[IVX] += wght * src1;
    }
    double src2 = -x_ov_rD * (pr + rho * v3 * v3 * sine2) - rho * v1 * v_2 / radius;
    out[IVY] += wght * src2;
    double src3 = -y_ov_rC * (pr + rho * v2 * v2 * sine2) - rho * v1 * v_3 / radius;
    out[IVZ] += wght * src3;
    // constant gravity (patches/25.constant_acc.patch:35-53)
    if (v.grav != 0.) {
      double src = wght * rho * v.grav;
      out[IVX] += src;
      if (!shallow) out[IEN] += src * v1;
    }
    // W92 Coriolis (examples/2023-Chen-exo3/W92.cpp:48-70)
    if (v.coriolis == EXO_CORIOLIS_W92) {
      double f = geo(v, GFCOR, p, k, j);
      double U = geo(v, GCR0, p, k, j) * v2 + geo(v, GCR1, p, k, j) * v3;
      double V = geo(v, GCR2, p, k, j) * v2 + geo(v, GCR3, p, k, j) * v3;
      U = -U;
      double llU = f * V, llV = -f * U;
      double mU = -llU;
      double acc2 = geo(v, GCQ0, p, k, j) * mU + geo(v, GCQ1, p, k, j) * llV;
      double acc3 = geo(v, GCQ2, p, k, j) * mU + geo(v, GCQ3, p, k, j) * llV;
      double a2c = acc2 + acc3 * cosine, a3c = acc3 + acc2 * cosine;
      out[IVY] += wght * rho * a2c;
      out[IVZ] += wght * rho * a3c;
    }
  }
  if (shallow) {
    for (int n = 0; n < nv; ++n) v.u[idx(v, p, n, k, j, i)] = un[n];
  } else if (v.implicit_flag & 1) {
    for (int n = 0; n < nv; ++n) {
      v.u[idx(v, p, n, k, j, i)] = un[n];
      v.du[idx(v, p, n, k, j, i)] = du[n];
    }
  } else {
    for (int n = 0; n < nv; ++n) v.u[idx(v, p, n, k, j, i)] = un[n] + 1. * du[n];
  }
}

// ------------------------------------------------------------- k_implicit -
struct M5 { double a[5][5]; };
struct V5 { double a[5]; };

__device__ __forceinline__ void mzero(M5& m) {
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) m.a[r][c] = 0.;
}
__device__ __forceinline__ M5 mmul(const M5& A, const M5& B) {
  M5 C;
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double s = A.a[r][0] * B.a[0][c];
#pragma unroll
      for (int k = 1; k < 5; ++k) s += A.a[r][k] * B.a[k][c];
      C.a[r][c] = s;
    }
  return C;
}
__device__ __forceinline__ V5 mvmul(const M5& A, const V5& x) {
  V5 y;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double s = A.a[r][0] * x.a[0];
#pragma unroll
    for (int k = 1; k < 5; ++k) s += A.a[r][k] * x.a[k];
    y.a[r] = s;
  }
  return y;
}
// Gauss-Jordan with partial pivoting on [A | I]
__device__ M5 minv(const M5& A0) {
  M5 A = A0, B;
  mzero(B);
#pragma unroll
  for (int r = 0; r < 5; ++r) B.a[r][r] = 1.;
  for (int c = 0; c < 5; ++c) {
    int piv = c;
    double best = fabs(A.a[c][c]);
    for (int r = c + 1; r < 5; ++r)
      if (fabs(A.a[r][c]) > best) { best = fabs(A.a[r][c]); piv = r; }
    if (piv != c) {
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double t = A.a[c][q]; A.a[c][q] = A.a[piv][q]; A.a[piv][q] = t;
        t = B.a[c][q]; B.a[c][q] = B.a[piv][q]; B.a[piv][q] = t;
      }
    }
    double d = 1.0 / A.a[c][c];
#pragma unroll
    for (int q = 0; q < 5; ++q) { A.a[c][q] *= d; B.a[c][q] *= d; }
    for (int r = 0; r < 5; ++r) {
      if (r == c) continue;
      double f = A.a[r][c];
#pragma unroll
      for (int q = 0; q < 5; ++q) { A.a[r][q] -= f * A.a[c][q]; B.a[r][q] -= f * B.a[c][q]; }
    }
  }
  return B;
}

// flux_decomposition.hpp:34-120, X1 direction
__device__ __forceinline__ void roe_average(double* prim, double gm1, const double* wl,
                                            const double* wr) {
  double sqrtdl = sqrt(wl[IDN]), sqrtdr = sqrt(wr[IDN]);
  double isdlpdr = 1.0 / (sqrtdl + sqrtdr);
  prim[IDN] = sqrtdl * sqrtdr;
  prim[IVX] = (sqrtdl * wl[IVX] + sqrtdr * wr[IVX]) * isdlpdr;
  prim[IVY] = (sqrtdl * wl[IVY] + sqrtdr * wr[IVY]) * isdlpdr;
  prim[IVZ] = (sqrtdl * wl[IVZ] + sqrtdr * wr[IVZ]) * isdlpdr;
  double el = wl[IPR] / gm1 + 0.5 * wl[IDN] * (sqr(wl[IVX]) + sqr(wl[IVY]) + sqr(wl[IVZ]));
  double er = wr[IPR] / gm1 + 0.5 * wr[IDN] * (sqr(wr[IVX]) + sqr(wr[IVY]) + sqr(wr[IVZ]));
  double hbar = ((el + wl[IPR]) / sqrtdl + (er + wr[IPR]) / sqrtdr) * isdlpdr;
  prim[IPR] = (hbar - 0.5 * (sqr(prim[IVX]) + sqr(prim[IVY]) + sqr(prim[IVZ]))) * gm1 /
              (gm1 + 1.) * prim[IDN];
}

__device__ M5 abs_jacobian(const double* prim, double cs, double gm1) {
  double r = prim[IDN], u = prim[IVX], v = prim[IVY], w = prim[IVZ], p = prim[IPR];
  double ke = 0.5 * (u * u + v * v + w * w);
  double hp = (gm1 + 1.) / gm1 * p / r;
  double h = hp + ke;
  M5 R = {{{1., 1., 1., 0., 0.},
           {u - cs, u, u + cs, 0., 0.},
           {v, v, v, 1., 0.},
           {w, w, w, 0., 1.},
           {h - u * cs, ke, h + u * cs, v, w}}};
  M5 Ri = {{{(cs * ke + u * hp) / (2. * cs * hp), (-hp - cs * u) / (2. * cs * hp), -v / (2. * hp),
             -w / (2. * hp), 1. / (2. * hp)},
            {(hp - ke) / hp, u / hp, v / hp, w / hp, -1. / hp},
            {(cs * ke - u * hp) / (2. * cs * hp), (hp - cs * u) / (2. * cs * hp), -v / (2. * hp),
             -w / (2. * hp), 1. / (2. * hp)},
            {-v, 0., 1., 0., 0.},
            {-w, 0., 0., 1., 0.}}};
  M5 Lam;
  mzero(Lam);
  Lam.a[0][0] = fabs(u - cs);
  Lam.a[1][1] = fabs(u);
  Lam.a[2][2] = fabs(u + cs);
  Lam.a[3][3] = fabs(u);
  Lam.a[4][4] = fabs(u);
  return mmul(mmul(R, Lam), Ri);
}

__device__ M5 flux_jacobian(double gm1, const double* w) {
  double v1 = w[IVX], v2 = w[IVY], v3 = w[IVZ], rho = w[IDN], pres = w[IPR];
  double s2 = v1 * v1 + v2 * v2 + v3 * v3;
  double c1 = ((gm1 - 1) * s2 / 2 - (gm1 + 1) / gm1 * pres / rho) * v1;
  double c2 = (gm1 + 1) / gm1 * pres / rho + s2 / 2 - gm1 * v1 * v1;
  M5 J = {{{0, 1., 0., 0., 0.},
           {gm1 * s2 / 2 - v1 * v1, (2. - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1},
           {-v1 * v2, v2, v1, 0., 0.},
           {-v1 * v3, v3, 0., v1, 0.},
           {c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + 1) * v1}}};
  return J;
}

// The vertical 5x5 block-tridiagonal correction of one radial column
// (ImplicitSolver::SolveImplicit3D X1 branch, solve_implicit_3d.cpp:102-179,
// with FullCorrection, full_correction.cpp:32-165, and ForwardSweep /
// BackwardSubstitution, forward_backward.hpp:15-126).
//   W(i, w5)      loads the primitive state of level i (i in [is-2, ie+1])
//   DU(i, n)      the explicit update of level i, variable n (read)
//   SCR(lev, e)   30 scratch doubles per level: the forward-sweep products
//                 A_i*c_i (25) and delta_i (5), read back by the back substitution
//   OUT(i, dl)    receives the corrected update of level i (ie down to is)
// geo: cos/sin of the cell metric and the angular widths dx2f_ang, dx3f_ang.
template <class WF, class DUF, class SCRF, class OUTF>
__device__ __forceinline__ void implicit_column(WF W, DUF DU, SCRF SCR, OUTF OUT, double cos_theta,
                                                double sin_theta, double d2, double d3,
                                                const double* x1f, const double* x1v,
                                                const double* dx1f, int is, int ie, double dt,
                                                double gamma, double grav) {
  double s = sin_theta;
  auto load = [&](int i, double* out) {
    W(i, out);
    out[IVY] += out[IVZ] * cos_theta;
    out[IVZ] *= sin_theta;
  };
  double fsig = 1., feps = 1.;
  double gmm1 = (gamma - 1.) * feps / fsig;  // the same for every level (NVAPOR = 0)
  double wl[5], wr[5], prim[5];
  double gm1 = 0.5 * (gmm1 + gmm1);
  double cs;
  // window at i = is: Am on the face between is-1 and is, dfdq[is-1], dfdq[is]
  load(is - 1, wl);
  load(is, wr);
  M5 dfm = flux_jacobian(gmm1, wl);
  M5 df0 = flux_jacobian(gmm1, wr);
  roe_average(prim, gm1, wl, wr);
  cs = sqrt((1. + (gamma - 1) * feps / fsig) * prim[IPR] / prim[IDN]);
  M5 Am = abs_jacobian(prim, cs, gm1);
  M5 Aprev;
  V5 dprev;
  for (int i = is; i <= ie; ++i) {
    load(i, wl);
    load(i + 1, wr);
    M5 dfp = flux_jacobian(gmm1, wr);
    roe_average(prim, gm1, wl, wr);
    cs = sqrt((1. + (gamma - 1) * feps / fsig) * prim[IPR] / prim[IDN]);
    M5 Ap = abs_jacobian(prim, cs, gm1);
    double aleft = d2 * d3 * x1f[i] * x1f[i] * s;
    double aright = d2 * d3 * x1f[i + 1] * x1f[i + 1] * s;
    double vol = dx1f[i] * d2 * d3 * x1v[i] * x1v[i] * s;
    M5 a, b, c;
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double Dt = (r == q) ? 1. / dt : 0.;
        double Phi = ((r == IVX && q == IDN) || (r == IEN && q == IVX)) ? grav : 0.;
        a.a[r][q] = (Am.a[r][q] * aleft + Ap.a[r][q] * aright +
                     (aright - aleft) * df0.a[r][q]) / (2. * vol) + Dt - Phi;
        b.a[r][q] = -(Am.a[r][q] + dfm.a[r][q]) * aleft / (2. * vol);
        c.a[r][q] = -(Ap.a[r][q] - dfp.a[r][q]) * aright / (2. * vol);
      }
    // reflecting boundaries: Bnds = Bnde = diag(1,-1,1,1,1)
    M5 B;
    mzero(B);
#pragma unroll
    for (int r = 0; r < 5; ++r) B.a[r][r] = 1.;
    B.a[IVX][IVX] = -1;
    if (i == is) {
      M5 t = mmul(b, B);
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) a.a[r][q] += t.a[r][q];
    }
    if (i == ie) {
      M5 t = mmul(c, B);
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) a.a[r][q] += t.a[r][q];
    }
    V5 rhs;
    rhs.a[0] = DU(i, IDN);
    rhs.a[0] /= dt;
    rhs.a[1] = DU(i, IVX) / dt;
    rhs.a[2] = DU(i, IVY) / dt;
    rhs.a[3] = DU(i, IVZ) / dt;
    rhs.a[4] = DU(i, IEN) / dt;
    M5 A;
    V5 dl;
    if (i == is) {
      A = minv(a);
      dl = mvmul(A, rhs);
    } else {
      M5 ba = mmul(b, Aprev);
      M5 t;
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) t.a[r][q] = a.a[r][q] - ba.a[r][q];
      A = minv(t);
      V5 bd = mvmul(b, dprev), x;
#pragma unroll
      for (int r = 0; r < 5; ++r) x.a[r] = rhs.a[r] - bd.a[r];
      dl = mvmul(A, x);
    }
    Aprev = mmul(A, c);
    dprev = dl;
    int lev = i - is;
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) SCR(lev, r * 5 + q) = Aprev.a[r][q];
#pragma unroll
    for (int r = 0; r < 5; ++r) SCR(lev, 25 + r) = dl.a[r];
    Am = Ap;
    dfm = df0;
    df0 = dfp;
  }
  V5 dnext;
  for (int i = ie; i >= is; --i) {
    int lev = i - is;
    V5 dl;
#pragma unroll
    for (int r = 0; r < 5; ++r) dl.a[r] = SCR(lev, 25 + r);
    if (i < ie) {
      M5 Ai;
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) Ai.a[r][q] = SCR(lev, r * 5 + q);
      V5 ad = mvmul(Ai, dnext);
#pragma unroll
      for (int r = 0; r < 5; ++r) dl.a[r] -= ad.a[r];
    }
    dnext = dl;
    OUT(i, dl.a);
  }
}

// UpdateAllConserved on the last stage with NVAPOR = NCLOUD = 0: the
// AirParcel round trip MassConc -> MoleFrac -> MassConc of one cell
// (impl.cpp:138-304, air_parcel.cpp:190-278)
__device__ __forceinline__ void airparcel_round_trip(double* uu, double Rd, double gammad) {
  const double Rgas = 8.314462;  // src/constants.hpp:5
  double mu0 = Rgas / Rd;
  double inv_mu0 = 1. / (mu0 * 1.);
  double cv0 = 1. * (Rd / (gammad - 1.));
  double w[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) w[n] = uu[n];
  double rho = 0., cvt = 0.;
  rho += w[0];
  cvt += w[0] * cv0;
  double KE = 0.5 / rho * (sqr(w[IVX]) + sqr(w[IVY]) + sqr(w[IVZ]));
  double tem = (w[IEN] - KE) / cvt;
  w[IEN] = cvt * tem;
  {
    double r2 = 0., cv = 0., rhoR = 0.;
    r2 += w[0];
    cv += w[0] * cv0;
    rhoR += w[0] * Rgas * inv_mu0;
    double di = 1. / r2;
    w[IDN] = w[IEN] / cv;
    w[IPR] = rhoR * w[IDN];
    w[IVX] *= di; w[IVY] *= di; w[IVZ] *= di;
  }
  {
    double tt = w[IDN], sum = 1., gg = 1.;
    double r2 = w[IPR] * sum / (Rd * tt * gg);
    w[IDN] = r2;
    w[IEN] = 0.;
    w[IEN] += w[IDN] * cv0 * tt;
    w[IVX] *= r2; w[IVY] *= r2; w[IVZ] *= r2;
  }
  double r2 = 0.;
  r2 += w[0];
  double vx = w[IVX] / r2, vy = w[IVY] / r2, vz = w[IVZ] / r2;
  double e = w[IEN] + 0.5 * w[0] * (sqr(vx) + sqr(vy) + sqr(vz));
#pragma unroll
  for (int n = 0; n < 4; ++n) uu[n] = w[n];
  uu[IEN] = e;
}

// One radial column of the stepping context: solve, then u += du and, on
// the last stage, the AirParcel round trip.  scratch is interleaved over
// columns so neighbouring threads touch neighbouring words.
__global__ void k_implicit(DevView v, int stage, double* scratch) {
  int ncol = 6 * v.N * v.N;
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  int j = v.js + col % v.N;
  int k = v.ks + (col / v.N) % v.N;
  int p = col / (v.N * v.N);
  const double kBeta[3] = {1.0, 0.25, 2.0 / 3.0};
  double dt = kBeta[stage] * v.sc->dt;
  auto W = [&](int i, double* out) {
    for (int n = 0; n < 5; ++n) out[n] = v.w[idx(v, p, n, k, j, i)];
  };
  auto DU = [&](int i, int n) { return v.du[idx(v, p, n, k, j, i)]; };
  auto SCR = [&](int lev, int e) -> double& { return scratch[((size_t)lev * 30 + e) * ncol + col]; };
  auto OUT = [&](int i, const double* dl) {
    double uu[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) uu[n] = v.u[idx(v, p, n, k, j, i)] + 1. * dl[n];
    if (stage == 2) airparcel_round_trip(uu, v.Rd, v.gamma);
#pragma unroll
    for (int n = 0; n < 5; ++n) v.u[idx(v, p, n, k, j, i)] = uu[n];
  };
  implicit_column(W, DU, SCR, OUT, geo(v, GCOSC, p, k, j), geo(v, GSINC, p, k, j),
                  geo(v, GDX2A, p, k, j), geo(v, GDX3A, p, k, j), v.x1f, v.x1v, v.dx1f, v.is,
                  v.ie, dt, v.gamma, v.grav);
}

// ImplicitSolver::FullCorrection over a batch of independent columns given
// as plain arrays: w [ncol][5][L+6] primitives with ghosts, du [ncol][5][L]
// explicit update (overwritten by the corrected one), colgeo [ncol][4] =
// (cos, sin, dx2f_ang, dx3f_ang), scratch ncol*L*30 doubles.
__global__ void k_implicit_columns(int ncol, int L, const double* w, double* du,
                                   const double* colgeo, const double* x1f, const double* x1v,
                                   const double* dx1f, double dt, double gamma, double grav,
                                   double* scratch) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  int nc1 = L + 2 * G;
  const double* wc = w + (size_t)col * 5 * nc1;
  double* duc = du + (size_t)col * 5 * L;
  auto W = [&](int i, double* out) {
    for (int n = 0; n < 5; ++n) out[n] = wc[n * nc1 + i];
  };
  auto DU = [&](int i, int n) { return duc[n * L + (i - G)]; };
  auto SCR = [&](int lev, int e) -> double& { return scratch[((size_t)lev * 30 + e) * ncol + col]; };
  auto OUT = [&](int i, const double* dl) {
#pragma unroll
    for (int n = 0; n < 5; ++n) duc[n * L + (i - G)] = dl[n];
  };
  const double* g4 = colgeo + (size_t)col * 4;
  implicit_column(W, DU, SCR, OUT, g4[0], g4[1], g4[2], g4[3], x1f, x1v, dx1f, G, G + L - 1, dt,
                  gamma, grav);
}

// last-stage round trip when the implicit solver is off
__global__ void k_roundtrip(DevView v) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)6 * v.N * v.N * v.L;
  if (tid >= total) return;
  int i = v.is + (int)(tid % v.L);
  size_t r = tid / v.L;
  int j = v.js + (int)(r % v.N);
  r /= v.N;
  int k = v.ks + (int)(r % v.N);
  int p = (int)(r / v.N);
  double uu[5];
  for (int n = 0; n < 5; ++n) uu[n] = v.u[idx(v, p, n, k, j, i)];
  airparcel_round_trip(uu, v.Rd, v.gamma);
  for (int n = 0; n < 5; ++n) v.u[idx(v, p, n, k, j, i)] = uu[n];
}

__global__ void k_p2c(DevView v, const double* wsrc) {
  size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)6 * v.N * v.N * v.L;
  if (tid >= total) return;
  int i = v.is + (int)(tid % v.L);
  size_t r = tid / v.L;
  int j = v.js + (int)(r % v.N);
  r /= v.N;
  int k = v.ks + (int)(r % v.N);
  int p = (int)(r / v.N);
  double w[5], c[5];
  for (int n = 0; n < v.nv; ++n) w[n] = wsrc[idx(v, p, n, k, j, i)];
  prim_to_cons(v, w, c, geo(v, GCOSC, p, k, j));
  for (int n = 0; n < v.nv; ++n) v.u[idx(v, p, n, k, j, i)] = c[n];
}

__global__ void k_set_dt(DevScalars* sc, double dt) { sc->dt = dt; }

__global__ void k_dt_reset(DevScalars* sc) {
  sc->dtmin_bits = 0x7FEFFFFFFFFFFFFFull;  // DBL_MAX
}

// Mesh::NewTimeStep: dt = min(2 dt, cfl * min over cells); advance time
__global__ void k_dt_finalize(DevScalars* sc, double cfl, double dt_fixed, int advance,
                              int first) {
  if (advance) {
    sc->time += sc->dt;
    sc->ncycle += 1;
  }
  if (dt_fixed > 0.) {
    sc->dt = dt_fixed;
    return;
  }
  double nd = cfl * __longlong_as_double((long long)sc->dtmin_bits);
  sc->dt = first ? nd : fmin(2.0 * sc->dt, nd);
}

__global__ void k_riemann_rows(int rsolver, int eqn, int ivx, int n, double gamma,
                               const double* wl, const double* wr, double* flx,
                               const double* cosf, const double* sinf, const double* cthp,
                               const double* cthc) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  int nv = eqn == EXO_EQN_SHALLOW_YZ ? 4 : 5;
  double a[5] = {0, 0, 0, 0, 0}, b[5] = {0, 0, 0, 0, 0}, f[5] = {0, 0, 0, 0, 0};
  for (int q = 0; q < nv; ++q) { a[q] = wl[(size_t)q * n + m]; b[q] = wr[(size_t)q * n + m]; }
  FaceGeo fg{cosf ? cosf[m] : 0., sinf ? sinf[m] : 1., cthp ? cthp[m] : 0., cthc ? cthc[m] : 0.};
  riemann(rsolver, gamma, ivx, fg, a, b, f);
  for (int q = 0; q < nv; ++q) flx[(size_t)q * n + m] = f[q];
}

__global__ void k_weno5(int n, const double* a, const double* b, const double* c,
                        const double* d, const double* e, double* out) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) out[m] = weno5(a[m], b[m], c[m], d[m], e[m]);
}

inline int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : EXO_ERR_CUDA;
}

inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

int launch_prim_ghost(const DevView& v, bool compute_dt, void* stream) {
  size_t total = (size_t)6 * v.cells;
  k_prim_ghost<<<nblk(total, 256), 256, 0, (cudaStream_t)stream>>>(v, compute_dt ? 1 : 0);
  return check_launch();
}

int launch_flux_x1(const DevView& v, void* stream) {
  if (v.eqn == EXO_EQN_SHALLOW_YZ) return 0;
  int threads = ((v.L + 1 + 31) / 32) * 32;
  if (threads > 256) threads = 256;
  size_t smem = ((size_t)v.nv * v.nc1 + v.nc1 + 1) * sizeof(double);
  k_flux_x1<<<6 * v.N * v.N, threads, smem, (cudaStream_t)stream>>>(v);
  return check_launch();
}

int launch_flux_x23(const DevView& v, void* stream) {
  size_t total = (size_t)2 * 6 * v.N * (v.N + 1) * v.L;
  k_flux_x23<<<nblk(total, 128), 128, 0, (cudaStream_t)stream>>>(v);
  return check_launch();
}

int launch_update(const DevView& v, int stage, void* stream) {
  size_t total = (size_t)6 * v.N * v.N * v.L;
  k_update<<<nblk(total, 128), 128, 0, (cudaStream_t)stream>>>(v, stage);
  int rc = check_launch();
  if (rc) return rc;
  if (v.eqn != EXO_EQN_SHALLOW_YZ && !(v.implicit_flag & 1) && stage == 2) {
    k_roundtrip<<<nblk(total, 128), 128, 0, (cudaStream_t)stream>>>(v);
    rc = check_launch();
  }
  return rc;
}

int launch_implicit(const DevView& v, int stage, void* stream) {
  if (v.eqn == EXO_EQN_SHALLOW_YZ || !(v.implicit_flag & 1)) return 0;
  int ncol = 6 * v.N * v.N;
  k_implicit<<<nblk(ncol, 64), 64, 0, (cudaStream_t)stream>>>(v, stage, v.scratch);
  return check_launch();
}

int launch_implicit_columns(int ncol, int L, const double* w, double* du, const double* colgeo,
                            const double* x1f, const double* x1v, const double* dx1f, double dt,
                            double gamma, double grav, double* scratch, void* stream) {
  if (ncol <= 0) return 0;
  k_implicit_columns<<<nblk(ncol, 64), 64, 0, (cudaStream_t)stream>>>(
      ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, scratch);
  return check_launch();
}

// ---------------------------------------------------------------------------
// Allocation-free variant of exo_implicit_columns.  Its scratch is this
// file-scope device array instead of caller memory, so the entry point never
// calls cudaMalloc or cudaFree.  Every GPU that loads the library holds the
// 8 MiB until the process exits.  The array name is only a host-side handle:
// kernels get the device address that cudaGetSymbolAddress returns, looked up
// once per device with that device current (on the first call made there).
static __device__ __align__(256) double g_noalloc_scratch[EXO_NOALLOC_SCRATCH_DOUBLES];

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {};
}  // namespace

int launch_implicit_columns_noalloc(int ncol, int L, const double* w, double* du,
                                    const double* colgeo, const double* x1f, const double* x1v,
                                    const double* dx1f, double dt, double gamma, double grav,
                                    void* stream, std::string* err) {
  if ((size_t)ncol * (size_t)L * 30 > (size_t)EXO_NOALLOC_SCRATCH_DOUBLES) {
    *err = "ncol*L*30 = " + std::to_string((size_t)ncol * (size_t)L * 30) +
           " exceeds the fixed scratch of " + std::to_string((size_t)EXO_NOALLOC_SCRATCH_DOUBLES) +
           " doubles (ncol*L must be <= " + std::to_string(EXO_NOALLOC_SCRATCH_DOUBLES / 30) + ")";
    return EXO_ERR_CAPACITY;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  double* scratch;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr) {
        *err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
        return EXO_ERR_CUDA;
      }
      g_noalloc_addr[dev] = static_cast<double*>(ptr);
    }
    scratch = g_noalloc_addr[dev];
  }
  if (ncol <= 0) return 0;
  k_implicit_columns<<<nblk(ncol, 64), 64, 0, (cudaStream_t)stream>>>(
      ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    *err = std::string("k_implicit_columns: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  return 0;
}

int launch_dt_reset(const DevView& v, void* stream) {
  k_dt_reset<<<1, 1, 0, (cudaStream_t)stream>>>(v.sc);
  return check_launch();
}

int launch_dt_finalize(const DevView& v, double dt_fixed, bool advance_time, void* stream) {
  k_dt_finalize<<<1, 1, 0, (cudaStream_t)stream>>>(v.sc, v.cfl, dt_fixed, advance_time ? 1 : 0,
                                                   advance_time ? 0 : 1);
  return check_launch();
}

int launch_set_dt(const DevView& v, double dt, void* stream) {
  k_set_dt<<<1, 1, 0, (cudaStream_t)stream>>>(v.sc, dt);
  return check_launch();
}

int launch_p2c_interior(const DevView& v, const double* w_src, void* stream) {
  size_t total = (size_t)6 * v.N * v.N * v.L;
  k_p2c<<<nblk(total, 128), 128, 0, (cudaStream_t)stream>>>(v, w_src);
  return check_launch();
}

int launch_riemann_rows(int rsolver, int eqn, int ivx, int n, double gamma, const double* wl,
                        const double* wr, double* flx, const double* cosf, const double* sinf,
                        const double* cthp, const double* cthc, void* stream) {
  if (n <= 0) return 0;
  k_riemann_rows<<<nblk(n, 128), 128, 0, (cudaStream_t)stream>>>(
      rsolver, eqn, ivx, n, gamma, wl, wr, flx, cosf, sinf, cthp, cthc);
  return check_launch();
}

int launch_weno5(int n, const double* a, const double* b, const double* c, const double* d,
                 const double* e, double* out, void* stream) {
  if (n <= 0) return 0;
  k_weno5<<<nblk(n, 128), 128, 0, (cudaStream_t)stream>>>(n, a, b, c, d, e, out);
  return check_launch();
}

}  // namespace exo
