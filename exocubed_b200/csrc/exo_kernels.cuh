// exo_kernels.cuh -- the device code of one arithmetic build of the step.
//
// Included by kernels.cu (EXO_MIXED 0: everything in FP64, compiled without
// fused multiply-add so it reproduces the CPU restatement bit for bit) and by
// kernels_mixed.cu (EXO_MIXED 1: WENO5, the Riemann solvers and the flux
// divergence in FP32 -- EXO_FLUX_T -- while the hydrostatic decomposition, the
// implicit solve, the equation of state and the conserved state stay FP64;
// compiled with FMA).  EXO_KNS names the namespace of the build.
//
// One stage of SSPRK(3,3) is five launches, each one kernel over every
// member of a batch (a single atmosphere is a batch of one):
//   kb_flux_x1    per radial column: hydrostatic decomposition, WENO5 in x1,
//                 restore, Riemann solve -> x1 face fluxes         (exo3 only)
//   kb_flux_x23   per line of horizontal faces (per face on grids of few
//                 levels): WENO5 on both sides; at panel edges the outer state
//                 is the neighbour panel's own reconstruction, rotated into
//                 this panel's basis; Riemann solve -> x2/x3 fluxes
//   kb_update     per cell: RK register average, flux divergence, geometric
//                 source, gravity / Coriolis -> u (exo2) or du (exo3)
//   kb_implicit   per radial column: 5x5 block-tridiagonal vertical correction,
//                 u += du, AirParcel round trip on the last stage (exo3)
//   kb_prim_ghost per cell incl. ghosts: ConservedToPrimitive of the interior,
//                 of the ghost bands interpolated from the neighbour panels and
//                 of the reflected x1 ghosts; CFL time-step candidate
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <utility>

#include <cuda_runtime.h>

#include "exo_internal.h"
#include "exo_mbarrier.cuh"

// x2/x3 fluxes: EXO_X23_TILES 1 = a block per line of faces, cells staged
// through shared memory (flux_x23_pipe), and one thread per face for grids
// of few levels; otherwise EXO_X23_LINES 1 = one thread per line of faces
// (sliding stencil window), 0 = one thread per face
#ifndef EXO_X23_TILES
#define EXO_X23_TILES 1
#endif
#ifndef EXO_X23_LINES
#define EXO_X23_LINES EXO_MIXED
#endif
// 1: the x1 (radial) Riemann flux, its storage and its divergence stay FP64
// in the mixed build (the reconstruction of the perturbations stays FP32):
// the radial momentum flux carries the full hydrostatic pressure, whose
// difference across a cell is a few per cent of it, so FP32 storage of the
// flux loses the balance against gravity to cancellation
#ifndef EXO_X1_FLUX64
#define EXO_X1_FLUX64 EXO_MIXED
#endif
// 1: the sliding window computes each cell's WENO smoothness indicators once
// for both of its faces (mixed build; the FP64 build keeps weno5's order)
#ifndef EXO_X23_SHARED_BETA
#define EXO_X23_SHARED_BETA EXO_MIXED
#endif
// 1: the same in the x1 kernel, whose cells' face values go through shared
// memory (mixed build)
#ifndef EXO_X1_SHARED_BETA
#define EXO_X1_SHARED_BETA EXO_MIXED
#endif
// 1: the implicit solve keeps (A c)_{i-1} in shared memory instead of registers
#ifndef EXO_IMPL_AP_SMEM
#define EXO_IMPL_AP_SMEM 0
#endif

namespace exo {
namespace EXO_KNS {
namespace {

// the implicit solve's block arithmetic is FP64 or FP32 (template argument
// R): EXO_PREC_MIXED_F32_SOLVE builds and factors its blocks and keeps its
// back-substitution factors in FP32, EXO_PREC_MIXED and the FP64 build in
// FP64.  The state, the explicit update it corrects and the corrected state
// are FP64 in every case.  At the solver's time steps (vertical acoustic
// Courant numbers of tens) FP32 blocks change a corrected update by a few
// 1e-7 of itself.
__device__ __forceinline__ float abs_r(float x) { return fabsf(x); }
__device__ __forceinline__ double abs_r(double x) { return fabs(x); }
// EXO_IMPL_RCP_NR 1: the mixed build's FP64 implicit blocks take 1/x as PTX
// rcp.approx.ftz.f64 refined by two Newton-Raphson steps, r <- r + r (1 - x r)
// (Newton's method for 1/x: the relative error squares each step, so a
// seed good to 2^-14 or better ends within an ulp or two of 1/x), instead of
// the IEEE division sequence: 3.6 % less implicit time at 6x192^2x96, on
// the LU pivots and the divisions of |A|.  The mixed build's primitive and
// update kernels take their reciprocals (density, sin^2, volume, radius)
// the same way.  The FP64 build divides.
#ifndef EXO_IMPL_RCP_NR
#define EXO_IMPL_RCP_NR 1
#endif
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ float inv_r(float x) { return 1.f / x; }
__device__ __forceinline__ double inv_r(double x) {
  if constexpr (EXO_IMPL_RCP_NR && EXO_MIXED) return rcp_nr(x);
  else return 1. / x;
}
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }

constexpr double TINY_NUMBER = 1.0e-20;
constexpr double WENO_EPS = 1.0e-7;

__device__ __forceinline__ double sqr(double x) { return x * x; }
__device__ __forceinline__ float sqr(float x) { return x * x; }

// SSPRK(3,3) stage weights beta = 1, 1/4, 2/3
__device__ __forceinline__ double rk_beta(int stage) {
  return stage == 0 ? 1.0 : (stage == 1 ? 0.25 : 2.0 / 3.0);
}

__device__ __forceinline__ size_t idx(const DevView& v, int p, int n, int k, int j, int i) {
  return ((((size_t)p * v.nv + n) * v.nc3 + k) * v.nc2 + j) * v.nc1 + i;
}
__device__ __forceinline__ double geo(const DevView& v, int f, int p, int k, int j) {
  return v.geo[(((size_t)f * 6 + p) * v.nc3 + k) * v.nc2 + j];
}

// face-flux and primitive arrays in the type the flux kernels work in
template <class T> __device__ __forceinline__ T* flux_array(const DevView& v, int d);
template <> __device__ __forceinline__ double* flux_array<double>(const DevView& v, int d) {
  return v.flux[d];
}
template <> __device__ __forceinline__ float* flux_array<float>(const DevView& v, int d) {
  return v.flux32[d];
}
// the type of the x1 face fluxes for a build whose flux type is T
template <class T>
using X1Flux = std::conditional_t<(EXO_X1_FLUX64 != 0), double, T>;
template <class T> __device__ __forceinline__ const T* prim_array(const DevView& v);
template <> __device__ __forceinline__ const double* prim_array<double>(const DevView& v) {
  return v.w;
}
template <> __device__ __forceinline__ const float* prim_array<float>(const DevView& v) {
  return v.w32;
}

// interp_weno5(phip2, phip1, phi, phim1, phim2): the face value between the
// 2nd and 3rd argument (Jiang & Shu 1996; orientation of tests/test_weno.cpp)
template <class T>
__device__ __forceinline__ T weno5(T phip2, T phip1, T phi, T phim1, T phim2) {
  const T eps = T(WENO_EPS);
  T p0 = T(1.0 / 3.0) * phim2 - T(7.0 / 6.0) * phim1 + T(11.0 / 6.0) * phi;
  T p1 = T(-1.0 / 6.0) * phim1 + T(5.0 / 6.0) * phi + T(1.0 / 3.0) * phip1;
  T p2 = T(1.0 / 3.0) * phi + T(5.0 / 6.0) * phip1 - T(1.0 / 6.0) * phip2;
  T b0 = T(13. / 12.) * sqr(phim2 - T(2.) * phim1 + phi) +
         T(.25) * sqr(phim2 - T(4.) * phim1 + T(3.) * phi);
  T b1 = T(13. / 12.) * sqr(phim1 - T(2.) * phi + phip1) + T(.25) * sqr(phim1 - phip1);
  T b2 = T(13. / 12.) * sqr(phi - T(2.) * phip1 + phip2) +
         T(.25) * sqr(T(3.) * phi - T(4.) * phip1 + phip2);
  T a0 = T(0.1) / ((b0 + eps) * (b0 + eps));
  T a1 = T(0.6) / ((b1 + eps) * (b1 + eps));
  T a2 = T(0.3) / ((b2 + eps) * (b2 + eps));
  return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}

// The same reconstruction split so that a cell's smoothness indicators serve
// both of its faces: the right-face value of cell c uses the weights
// 1/(beta_k + eps)^2 of its left, centre and right candidate stencils in that
// order, the left-face value the same three in mirror order.  a..e are the
// cells c-2..c+2.  (A sliding window over a line of faces computes each
// cell's indicators once instead of twice; the indicators of the mirrored
// stencils are the same sums taken in the other order, so results agree
// with weno5 to rounding.)
template <class T>
struct WenoCell {
  T i0, i1, i2;  // 1/(beta+eps)^2 of the stencils {c-2..c}, {c-1..c+1}, {c..c+2}
};
template <class T>
__device__ __forceinline__ WenoCell<T> weno_cell(T a, T b, T c, T d, T e) {
  const T eps = T(WENO_EPS);
  T b0 = T(13. / 12.) * sqr(a - T(2.) * b + c) + T(.25) * sqr(a - T(4.) * b + T(3.) * c);
  T b1 = T(13. / 12.) * sqr(b - T(2.) * c + d) + T(.25) * sqr(b - d);
  T b2 = T(13. / 12.) * sqr(c - T(2.) * d + e) + T(.25) * sqr(T(3.) * c - T(4.) * d + e);
  return {T(1.) / ((b0 + eps) * (b0 + eps)), T(1.) / ((b1 + eps) * (b1 + eps)),
          T(1.) / ((b2 + eps) * (b2 + eps))};
}
template <class T>
__device__ __forceinline__ T weno_right(const WenoCell<T>& w, T a, T b, T c, T d, T e) {
  T p0 = T(1.0 / 3.0) * a - T(7.0 / 6.0) * b + T(11.0 / 6.0) * c;
  T p1 = T(-1.0 / 6.0) * b + T(5.0 / 6.0) * c + T(1.0 / 3.0) * d;
  T p2 = T(1.0 / 3.0) * c + T(5.0 / 6.0) * d - T(1.0 / 6.0) * e;
  T a0 = T(0.1) * w.i0, a1 = T(0.6) * w.i1, a2 = T(0.3) * w.i2;
  return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}
template <class T>
__device__ __forceinline__ T weno_left(const WenoCell<T>& w, T a, T b, T c, T d, T e) {
  T p0 = T(1.0 / 3.0) * e - T(7.0 / 6.0) * d + T(11.0 / 6.0) * c;
  T p1 = T(-1.0 / 6.0) * d + T(5.0 / 6.0) * c + T(1.0 / 3.0) * b;
  T p2 = T(1.0 / 3.0) * c + T(5.0 / 6.0) * b - T(1.0 / 6.0) * a;
  T a0 = T(0.1) * w.i2, a1 = T(0.6) * w.i1, a2 = T(0.3) * w.i0;
  return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}

// right-face value (face c+1) and left-face value (face c) of cell c on a
// strided line q[c*s]
// (the stencil values are converted to the reconstruction type T first)
template <class T, class S>
__device__ __forceinline__ T weno_r(const S* q, long s, int c) {
  return weno5<T>(T(q[(c + 2) * s]), T(q[(c + 1) * s]), T(q[c * s]), T(q[(c - 1) * s]),
                  T(q[(c - 2) * s]));
}
template <class T, class S>
__device__ __forceinline__ T weno_l(const S* q, long s, int c) {
  return weno5<T>(T(q[(c - 2) * s]), T(q[(c - 1) * s]), T(q[c * s]), T(q[(c + 1) * s]),
                  T(q[(c + 2) * s]));
}

// ------------------------------------------------------------------ EOS ----
// CubedSphereUtility::CovariantToContravariant (cubed_sphere_utility.hpp:22-31)
// (the mixed build multiplies by one reciprocal instead of four divisions)
__device__ __forceinline__ void cov_to_contra(double* a, double cth) {
  double v = a[IVY], w = a[IVZ];
  double sth2 = 1. - cth * cth;
#if EXO_MIXED
  const double is2 = inv_r(sth2);
  a[IVY] = (v - w * cth) * is2;
  a[IVZ] = (w - v * cth) * is2;
#else
  a[IVY] = v / sth2 - w * cth / sth2;
  a[IVZ] = -v * cth / sth2 + w / sth2;
#endif
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
    double di = inv_r(density);
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
template <class T>
struct FaceGeo {
  T cosf, sinf, cthp, cthc;
};

template <class T>
__device__ __forceinline__ void prim_to_local(int ivx, const FaceGeo<T>& fg, T* w) {
  if (ivx == IVY) {  // PrimToLocal2, gnomonic_equiangle.cpp:604-660
    T g23 = fg.cosf, g33 = T(1.0), gi22 = T(1.0) / (fg.sinf * fg.sinf);
    T T11 = T(1.0), T22 = T(1.0) / sqrt(gi22), T32 = g23 / sqrt(g33), T33 = sqrt(g33);
    T uu1 = w[IVX], uu2 = w[IVY], uu3 = w[IVZ];
    w[IVX] = T11 * uu1;
    w[IVY] = T22 * uu2;
    w[IVZ] = T32 * uu2 + T33 * uu3;
  } else if (ivx == IVZ) {  // PrimToLocal3, :662-718
    T g23 = fg.cosf, g22 = T(1.0), gi33 = T(1.0) / (fg.sinf * fg.sinf);
    T T11 = T(1.0), T22 = sqrt(g22), T23 = g23 / sqrt(g22), T33 = T(1.0) / sqrt(gi33);
    T uu1 = w[IVX], uu2 = w[IVY], uu3 = w[IVZ];
    w[IVX] = T11 * uu1;
    w[IVY] = T22 * uu2 + T23 * uu3;
    w[IVZ] = T33 * uu3;
  }
}

template <class T>
__device__ __forceinline__ void flux_to_global(int ivx, const FaceGeo<T>& fg, T* f) {
  if (ivx == IVY) {  // FluxToGlobal2, :752-791
    T g23 = fg.cosf, g33 = T(1.0), gi22 = T(1.0) / (fg.sinf * fg.sinf);
    T T11 = T(1.0), T22 = sqrt(gi22), T32 = -sqrt(gi22) * g23 / g33, T33 = T(1.0) / sqrt(g33);
    T txx = f[IVX], txy = f[IVY], txz = f[IVZ];
    f[IVX] = T11 * txx;
    f[IVY] = T22 * txy;
    f[IVZ] = T32 * txy + T33 * txz;
  } else if (ivx == IVZ) {  // FluxToGlobal3, :793-832
    T g23 = fg.cosf, g22 = T(1.0), gi33 = T(1.0) / (fg.sinf * fg.sinf);
    T T11 = T(1.0), T22 = T(1.0) / sqrt(g22), T23 = -g23 / g22 * sqrt(gi33), T33 = sqrt(gi33);
    T txx = f[IVX], txy = f[IVY], txz = f[IVZ];
    f[IVX] = T11 * txx;
    f[IVY] = T22 * txy + T23 * txz;
    f[IVZ] = T33 * txz;
  }
}

// roe_shallow_yz.cpp:18-122
template <class T>
__device__ __forceinline__ void riemann_roe_shallow(int ivx, const FaceGeo<T>& fg, T* wli, T* wri, T* flx) {
  const T h = T(0.5);
  int ivy = ivx == IVY ? IVZ : IVY;
  prim_to_local(ivx, fg, wli);
  prim_to_local(ivx, fg, wri);
  T ubar = (wli[ivx] * sqrt(wli[IDN]) + wri[ivx] * sqrt(wri[IDN])) /
           (sqrt(wli[IDN]) + sqrt(wri[IDN]));
  T vbar = (wli[ivy] * sqrt(wli[IDN]) + wri[ivy] * sqrt(wri[IDN])) /
           (sqrt(wli[IDN]) + sqrt(wri[IDN]));
  T cbar = sqrt(h * (wli[IDN] + wri[IDN]));
  T delh = wri[IDN] - wli[IDN];
  T delu = wri[ivx] - wli[ivx];
  T delv = wri[ivy] - wli[ivy];
  T hbar = sqrt(wli[IDN] * wri[IDN]);
  T a1 = h * (cbar * delh - hbar * delu) / cbar;
  T a2 = hbar * delv;
  T a3 = h * (cbar * delh + hbar * delu) / cbar;
  T w00 = a1, w01 = a1 * (ubar - cbar), w02 = a1 * vbar;
  T w10 = T(0.), w11 = T(0.), w12 = a2;
  T w20 = a3, w21 = a3 * (ubar + cbar), w22 = a3 * vbar;
  T s0 = fabs(ubar - cbar), s1 = fabs(ubar), s2 = fabs(ubar + cbar);
  flx[IVZ] = T(0.);
  flx[IDN] = h * (wli[IDN] * wli[ivx] + wri[IDN] * wri[ivx]);
  flx[ivx] = h * (wli[IDN] * wli[ivx] * wli[ivx] + h * wli[IDN] * wli[IDN] +
                  wri[IDN] * wri[ivx] * wri[ivx] + h * wri[IDN] * wri[IDN]);
  flx[ivy] = h * (wli[IDN] * wli[ivx] * wli[ivy] + wri[IDN] * wri[ivx] * wri[ivy]);
  flx[IVX] = T(0.);
  flx[IDN] -= h * s0 * w00;
  flx[ivx] -= h * s0 * w01;
  flx[ivy] -= h * s0 * w02;
  flx[IDN] -= h * s1 * w10;
  flx[ivx] -= h * s1 * w11;
  flx[ivy] -= h * s1 * w12;
  flx[IDN] -= h * s2 * w20;
  flx[ivx] -= h * s2 * w21;
  flx[ivy] -= h * s2 * w22;
  if (ivx == IVX) {
    flx[IVX] = T(0.);
    return;
  }
  flux_to_global(ivx, fg, flx);
  T ty = flx[ivx], tz = flx[ivy];
  flx[ivx] = ty + tz * fg.cthp;
  flx[ivy] = tz + ty * fg.cthp;
}

// lmars.cpp:24-110 (NVAPOR = NCLOUD = 0), no projection
template <class T>
__device__ __forceinline__ void riemann_lmars(double gamma_d, int ivx, const T* wli, const T* wri, T* flx) {
  const T h = T(0.5), one = T(1.);
  T gamma = T(gamma_d);
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
  T fsig = one, feps = one;
  T kappal = one / (gamma - one) * fsig / feps;
  T kappar = one / (gamma - one) * fsig / feps;
  T hl = wli[IPR] / wli[IDN] * (kappal + one) +
         h * (sqr(wli[ivx]) + sqr(wli[ivy]) + sqr(wli[ivz]));
  T hr = wri[IPR] / wri[IDN] * (kappar + one) +
         h * (sqr(wri[ivx]) + sqr(wri[ivy]) + sqr(wri[ivz]));
  T rhobar = h * (wli[IDN] + wri[IDN]);
  T cbar = sqrt(h * (one + (one / kappar + one / kappal) / T(2.)) *
                (wli[IPR] + wri[IPR]) / rhobar);
  T pbar = h * (wli[IPR] + wri[IPR]) + h * (rhobar * cbar) * (wli[ivx] - wri[ivx]);
  T ubar = h * (wli[ivx] + wri[ivx]) + h / (rhobar * cbar) * (wli[IPR] - wri[IPR]);
  T rdl = one, rdr = one;
  if (ubar > T(0.)) {
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
template <class T>
__device__ __forceinline__ void riemann_hllc(double gamma_d, int ivx, const FaceGeo<T>& fg, T* wl, T* wr, T* flx) {
  const T h = T(.5), one = T(1.0), zero = T(0.0);
  T gamma = T(gamma_d);
  int ivy = IVX + ((ivx - IVX) + 1) % 3;
  int ivz = IVX + ((ivx - IVX) + 2) % 3;
  T gm1 = gamma - one, igm1 = one / gm1;
  prim_to_local(ivx, fg, wl);
  prim_to_local(ivx, fg, wr);
  T wli[5], wri[5], fl[5], fr[5];
  wli[IDN] = wl[IDN]; wli[IVX] = wl[ivx]; wli[IVY] = wl[ivy]; wli[IVZ] = wl[ivz]; wli[IPR] = wl[IPR];
  wri[IDN] = wr[IDN]; wri[IVX] = wr[ivx]; wri[IVY] = wr[ivy]; wri[IVZ] = wr[ivz]; wri[IPR] = wr[IPR];
  T fsig = one, feps = one;
  T cl = sqrt((one + (gamma - one) * feps / fsig) * wli[IPR] / wli[IDN]);
  T cr = sqrt((one + (gamma - one) * feps / fsig) * wri[IPR] / wri[IDN]);
  T KE_l, KE_r;
  if (ivx == IVX) {
    T cth = fg.cthc, vy, vz;
    vy = wli[IVY] + wli[IVZ] * cth;
    vz = wli[IVZ] + wli[IVY] * cth;
    KE_l = h * wli[IDN] * (sqr(wli[IVX]) + wli[IVY] * vy + wli[IVZ] * vz);
    vy = wri[IVY] + wri[IVZ] * cth;
    vz = wri[IVZ] + wri[IVY] * cth;
    KE_r = h * wri[IDN] * (sqr(wri[IVX]) + wri[IVY] * vy + wri[IVZ] * vz);
  } else {
    KE_l = h * wli[IDN] * (sqr(wli[IVX]) + sqr(wli[IVY]) + sqr(wli[IVZ]));
    KE_r = h * wri[IDN] * (sqr(wri[IVX]) + sqr(wri[IVY]) + sqr(wri[IVZ]));
  }
  T el = wli[IPR] * igm1 + KE_l;
  T er = wri[IPR] * igm1 + KE_r;
  T rhoa = h * (wli[IDN] + wri[IDN]);
  T ca = h * (cl + cr);
  T pmid = h * (wli[IPR] + wri[IPR] + (wli[IVX] - wri[IVX]) * rhoa * ca);
  T ql = (pmid <= wli[IPR]) ? one
         : sqrt(one + (gamma + one) / (T(2) * gamma) * (pmid / wli[IPR] - one));
  T qr = (pmid <= wri[IPR]) ? one
         : sqrt(one + (gamma + one) / (T(2) * gamma) * (pmid / wri[IPR] - one));
  T al = wli[IVX] - cl * ql;
  T ar = wri[IVX] + cr * qr;
  T bp = ar > zero ? ar : T(TINY_NUMBER);
  T bm = al < zero ? al : -T(TINY_NUMBER);
  T vxl = wli[IVX] - al;
  T vxr = wri[IVX] - ar;
  T tl = wli[IPR] + vxl * wli[IDN] * wli[IVX];
  T tr = wri[IPR] + vxr * wri[IDN] * wri[IVX];
  T ml = wli[IDN] * vxl;
  T mr = -(wri[IDN] * vxr);
  T am = (tl - tr) / (ml + mr);
  T cp = (ml * tr + mr * tl) / (ml + mr);
  cp = cp > zero ? cp : zero;
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
  T sl, sr, sm;
  if (am >= zero) {
    sl = am / (am - bm);
    sr = zero;
    sm = -bm / (am - bm);
  } else {
    sl = zero;
    sr = -am / (bp - am);
    sm = bp / (bp - am);
  }
  flx[IDN] = sl * fl[IDN] + sr * fr[IDN];
  flx[ivx] = sl * fl[IVX] + sr * fr[IVX] + sm * cp;
  flx[ivy] = sl * fl[IVY] + sr * fr[IVY];
  flx[ivz] = sl * fl[IVZ] + sr * fr[IVZ];
  flx[IEN] = sl * fl[IEN] + sr * fr[IEN] + sm * cp * am;
  flux_to_global(ivx, fg, flx);
  T ty = flx[IVY], tz = flx[IVZ];
  flx[IVY] = ty + tz * fg.cthp;
  flx[IVZ] = tz + ty * fg.cthp;
}

// lmars_shallow_yz.cpp:18-93
template <class T>
__device__ __forceinline__ void riemann_lmars_shallow(int ivx, const FaceGeo<T>& fg, T* wli, T* wri, T* flx) {
  const T h = T(0.5);
  int ivy = ivx == IVY ? IVZ : IVY;
  prim_to_local(ivx, fg, wli);
  prim_to_local(ivx, fg, wri);
  T cbar = sqrt(h * (wli[IDN] + wri[IDN]));
  T hbar = h * (wli[IDN] + wri[IDN]) + h * cbar * (wli[ivx] - wri[ivx]);
  T ubar = h * (wli[ivx] + wri[ivx]) + h / cbar * (wli[IDN] - wri[IDN]);
  flx[IVZ] = T(0.);
  if (ubar > T(0.)) {
    flx[IDN] = ubar * wli[IDN];
    flx[ivx] = ubar * wli[IDN] * wli[ivx] + h * hbar * hbar;
    flx[ivy] = ubar * wli[IDN] * wli[ivy];
  } else {
    flx[IDN] = ubar * wri[IDN];
    flx[ivx] = ubar * wri[IDN] * wri[ivx] + h * hbar * hbar;
    flx[ivy] = ubar * wri[IDN] * wri[ivy];
  }
  flx[IVX] = T(0.);
  if (ivx == IVX) return;
  flux_to_global(ivx, fg, flx);
  T ty = flx[ivx], tz = flx[ivy];
  flx[ivx] = ty + tz * fg.cthp;
  flx[ivy] = tz + ty * fg.cthp;
}

template <class T>
__device__ __forceinline__ void riemann(int rsolver, double gamma, int ivx, const FaceGeo<T>& fg,
                                        T* wl, T* wr, T* flx) {
  switch (rsolver) {
    case EXO_RS_ROE_SHALLOW: riemann_roe_shallow(ivx, fg, wl, wr, flx); break;
    case EXO_RS_LMARS: riemann_lmars(gamma, ivx, wl, wr, flx); break;
    case EXO_RS_HLLC: riemann_hllc(gamma, ivx, fg, wl, wr, flx); break;
    default: riemann_lmars_shallow(ivx, fg, wl, wr, flx); break;
  }
}

// ----------------------------------------------------- k_prim_ghost ------
// The conserved state a ghost-band cell gets from the neighbour panel
// (CubedSphereUtility::PackData with InteprolateX2/X3, cubed_sphere_utility.
// cpp:92-369, as the ghost table e precomputes it): linear interpolation
// along the edge between two source cells, vectors (IVY, IVZ) raised,
// rotated to the receiver's basis through latitude-longitude and lowered.
// src is the source panel's (nv, nc3, nc2, nc1) array.
__device__ __forceinline__ void ghost_interp(const DevView& v, const GhostEntry& e,
                                             const double* src, int i, double* c) {
  auto S = [&](int n, int k, int j) {
    return src[(((size_t)n * v.nc3 + k) * v.nc2 + j) * v.nc1 + i];
  };
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    if (n == IVY || n == IVZ) continue;
    double v1 = S(n, e.k0, e.j0);
    double v2 = S(n, e.k1, e.j1);
    c[n] = (e.A * v1 + e.B * v2) / e.C;
  }
  double v1y = S(IVY, e.k0, e.j0), v1z = S(IVZ, e.k0, e.j0);
  double v2y = S(IVY, e.k1, e.j1), v2z = S(IVZ, e.k1, e.j1);
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

// Conserved value of variable n at cell (p,k,j,i) where (k,j) is interior or
// in a ghost band; vectors (IVY, IVZ) come back together.
__device__ __forceinline__ void load_cons(const DevView& v, int p, int k, int j, int i,
                                          bool interior, double* c) {
  if (interior) {
    #pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= v.nv) break;
      c[n] = v.u[idx(v, p, n, k, j, i)];
    }
    return;
  }
  const GhostEntry& e = v.ghost[v.ghost_map[((size_t)p * v.nc3 + k) * v.nc2 + j]];
  ghost_interp(v, e, v.u + idx(v, e.src_panel, 0, 0, 0, 0), i, c);
}

// the CFL candidate of the block's cells is reduced in shared memory first,
// so one atomic per block reaches the global minimum
__device__ __forceinline__ void block_min_atomic(unsigned long long* target, unsigned long long x) {
  __shared__ unsigned long long warp_min[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long y = __shfl_down_sync(0xffffffffu, x, o);
    x = y < x ? y : x;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_min[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = (blockDim.x + 31) >> 5;
    x = lane < nw ? warp_min[lane] : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long y = __shfl_down_sync(0xffffffffu, x, o);
      x = y < x ? y : x;
    }
    if (lane == 0 && x != ~0ull) atomicMin(target, x);
  }
}

// Hydro::NewBlockTimeStep with patches/21.new_blockdt.patch:23-35 at an
// interior cell with primitives w: the candidate as the bits of a
// non-negative double, or ~0 when there is none
__device__ __forceinline__ unsigned long long cfl_candidate(const DevView& v, const double* w,
                                                            int p, int k, int j, int i) {
  const bool shallow = (v.eqn == EXO_EQN_SHALLOW_YZ);
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
  if (m >= 0.) return (unsigned long long)__double_as_longlong(m);
  return ~0ull;
}

__device__ __forceinline__ unsigned long long prim_ghost_cell(const DevView& v, unsigned tid,
                                                              int compute_dt) {
  const unsigned long long none = ~0ull;
  unsigned total = 6u * (unsigned)v.cells;
  if (tid >= total) return none;
  unsigned r = v.div_nc1(tid);
  unsigned i = tid - r * (unsigned)v.nc1;
  unsigned r2 = v.div_nc2(r);
  int j = (int)(r - r2 * (unsigned)v.nc2);
  unsigned r3 = v.div_nc3(r2);
  int k = (int)(r2 - r3 * (unsigned)v.nc3);
  int p = (int)r3;
  bool kin = (k >= v.ks && k <= v.ke), jin = (j >= v.js && j <= v.je);
  if (!kin && !jin) return none;  // corner: never read on the path
  int ii = i;
  bool mirror = false;
  if (i < v.is) { ii = 2 * v.is - 1 - i; mirror = true; }
  else if (i > v.ie) { ii = 2 * v.ie + 1 - i; mirror = true; }
  double c[5], w[5];
  load_cons(v, p, k, j, ii, kin && jin, c);
  double cth = geo(v, GCOSC, p, k, j);
  int bad = cons_to_prim(v, c, w, cth);
  if (mirror) w[IVX] = -w[IVX];
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    v.w[idx(v, p, n, k, j, i)] = w[n];
  }
#if EXO_MIXED
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    v.w32[idx(v, p, n, k, j, i)] = (float)w[n];
  }
#endif
  if (!(kin && jin) || mirror) return none;
  if (bad) atomicOr(&v.sc->invalid, 1);
  if (compute_dt) return cfl_candidate(v, w, p, k, j, (int)i);
  return none;
}


__device__ __forceinline__ void prim_ghost_block(const DevView& v, unsigned blk, int compute_dt) {
  unsigned tid = blk * blockDim.x + threadIdx.x;
  unsigned long long m = prim_ghost_cell(v, tid, compute_dt);
  if (compute_dt) block_min_atomic(&v.sc->dtmin_bits, m);
}

// ------------------------------------------------------------ k_flux_x1 ---
// One CTA per interior radial column.
// Several radial columns per block (the x1 tile): each column's faces,
// cells and hydrostatic scan are spread over the block's threads, so the
// block's lanes stay busy (one column of L+1 faces leaves most of a warp
// idle) and the columns' serial scans run side by side.
__device__ __forceinline__ int x1_columns_per_block(const DevView& v) {
  return v.tiles[BK_X1] > 0 ? v.tiles[BK_X1] : 1;
}

// q = t / d, r = t - q d for small non-negative t (< 2^20) through a float
// reciprocal, corrected by one step either way
__device__ __forceinline__ void divmod_small(int t, int d, float inv_d, int& q, int& r) {
  q = (int)((float)t * inv_d);
  r = t - q * d;
  if (r < 0) { --q; r += d; }
  else if (r >= d) { ++q; r -= d; }
}

// ln(sinh x / x) for |x| <= 0.25: its Taylor series sum_n c_n x^{2n} with
// c_n = 2^{2n} B_{2n} / (2n (2n)!) (B the Bernoulli numbers), seven terms
// (truncation error below 4e-19 there)
__device__ __forceinline__ double ln_sinhc(double x) {
  const double z = x * x;
  return z * (1. / 6 +
              z * (-1. / 180 +
                   z * (1. / 2835 +
                        z * (-1. / 37800 +
                             z * (1. / 467775 +
                                  z * (-691. / 3831077250. + z * (2. / 127702575.)))))));
}
// e^y for |y| <= 0.25: its Taylor series to y^13 (truncation below 5e-20)
__device__ __forceinline__ double exp_small(double y) {
  constexpr double inv_fact[14] = {1.,
                                   1.,
                                   1. / 2,
                                   1. / 6,
                                   1. / 24,
                                   1. / 120,
                                   1. / 720,
                                   1. / 5040,
                                   1. / 40320,
                                   1. / 362880,
                                   1. / 3628800,
                                   1. / 39916800,
                                   1. / 479001600,
                                   1. / 6227020800.};
  double s = inv_fact[13];
#pragma unroll
  for (int k = 12; k >= 0; --k) s = s * y + inv_fact[k];
  return s;
}

template <class T>
__device__ __forceinline__ void flux_x1_block(const DevView& v, unsigned blk) {
  extern __shared__ double sm[];
  __shared__ double s_gam[X1_MAX_COLUMNS], s_expf[X1_MAX_COLUMNS];
  __shared__ double s_cthp[X1_MAX_COLUMNS], s_cosc[X1_MAX_COLUMNS];
  __shared__ long long s_base[X1_MAX_COLUMNS];  // idx(p, 0, k, j, 0) of each column
  const int cpb = x1_columns_per_block(v);
  const int ncol_total = 6 * v.N * v.N;
  const int col0 = (int)blk * cpb;
  const int ncb = min(cpb, ncol_total - col0);  // columns of this block
  const int nc1 = v.nc1, nv = v.nv, L = v.L;
  const int cstride = x1_column_doubles(v);    // shared doubles per column
  const size_t vs = v.cells;
  // shared memory of column c: w [nv][nc1], psf [nc1+1] (mixed: ln psf, dsf)
  auto WC = [&](int c) { return sm + (size_t)c * cstride; };
  auto PSF = [&](int c) { return sm + (size_t)c * cstride + nv * nc1; };
  if ((int)threadIdx.x < ncb) {
    const int c = threadIdx.x, col = col0 + c;
    const int j = v.js + col % v.N;
    const int k = v.ks + (col / v.N) % v.N;
    const int p = col / (v.N * v.N);
    s_base[c] = (long long)idx(v, p, 0, k, j, 0);
    s_cthp[c] = geo(v, GCTHP1, p, k, j);
    s_cosc[c] = geo(v, GCOSC, p, k, j);
  }
  __syncthreads();
  {
    const int per = nv * nc1;
    const float inv_per = 1.f / (float)per, inv_nc1 = 1.f / (float)nc1;
    for (int t = threadIdx.x; t < ncb * per; t += blockDim.x) {
      int c, r, n, i;
      divmod_small(t, per, inv_per, c, r);
      divmod_small(r, nc1, inv_nc1, n, i);
      WC(c)[r] = v.w[(size_t)s_base[c] + n * vs + i];
    }
  }
  __syncthreads();
  const bool decomp = (v.grav != 0.);
  if (decomp) {
    // Decomposition::ChangeToPerturbation (change_to_perturbation.cpp:39-157).
#if EXO_MIXED
    // The downward scan psf[i] = psf[i+1] + g rho_i dx1f_i as a suffix sum,
    // one warp per column: each lane sums a chunk of levels, the lanes'
    // sums are scanned with shuffles, then each lane fills its chunk (FP64
    // throughout; only the order of the additions differs from the serial
    // scan of the FP64 build)
    {
      const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
      const int nwarps = (int)blockDim.x >> 5;
      const int is = v.is, ie = v.ie;
      const int chunk = (L + 31) >> 5;
      const double grav = -v.grav;
      for (int c = warp; c < ncb; c += nwarps) {
        double* wc = WC(c);
        double* psf = PSF(c);
        const double* wd = wc + IDN * nc1;
        const double* wp = wc + IPR * nc1;
        const int m0 = is + lane * chunk, m1 = min(m0 + chunk, ie + 1);
        double part = 0.;
        for (int m = m0; m < m1; ++m) part += grav * wd[m] * v.dx1f[m];
        // sum of the parts of the lanes above this one
        double above = part;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const double y = __shfl_down_sync(0xffffffffu, above, off);
          if (lane + off < 32) above += y;
        }
        above = __shfl_down_sync(0xffffffffu, above, 1);
        if (lane == 31) above = 0.;
        double top = 0.;
        if (lane == 0) {
          const double RdTv = wp[ie] / wd[ie];
          top = wp[ie] * exp(-grav * v.dx1f[ie] / (2 * RdTv));
          psf[ie + 1] = top;
        }
        top = __shfl_sync(0xffffffffu, top, 0);
        double run = top + above;
        for (int m = m1 - 1; m >= m0; --m) {
          run += grav * wd[m] * v.dx1f[m];
          psf[m] = run;
        }
        __syncwarp();
        if (lane == 0) {
          for (int i = 1; i <= G; ++i) psf[is - i] = psf[is + i];
          for (int i = 1; i <= G; ++i) psf[ie + i + 1] = psf[ie + 1 - i];
          double gammad = v.gamma, fsig = 1., feps = 1.;
          double gam = 1. + (gammad - 1.) * feps / fsig;
          double ent = log(wp[is]) - gam * log(wd[is]);
          s_gam[c] = gam;
          s_expf[c] = exp(-ent / gam);
        }
      }
    }
#else
    // one thread per column for the downward scan
    if ((int)threadIdx.x < ncb) {
      const int c = threadIdx.x;
      double* wc = WC(c);
      double* psf = PSF(c);
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
      s_gam[c] = gam;
      s_expf[c] = exp(-ent / gam);
    }
#endif
    __syncthreads();
    const float inv_nc1 = 1.f / (float)nc1;
#if EXO_MIXED
    // FP64 still, with the powers as exp(log(x) / gamma) and one log per face
    // shared by its two cells: ln psf and the face density of the isentropic
    // reference go to shared memory for the cells and for the restore
    const float inv_f = 1.f / (float)(nc1 + 1);
    for (int t = threadIdx.x; t < ncb * (nc1 + 1); t += blockDim.x) {
      int c, i;
      divmod_small(t, nc1 + 1, inv_f, c, i);
      double* psf = PSF(c);
      const double l = log(psf[i]);
      psf[nc1 + 1 + i] = l;
      psf[2 * (nc1 + 1) + i] = exp(l * (1. / s_gam[c])) * s_expf[c];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < ncb * nc1; t += blockDim.x) {
      int c, i;
      divmod_small(t, nc1, inv_nc1, c, i);
      double* wc = WC(c);
      const double* psf = PSF(c);
      const double* lpsf = psf + nc1 + 1;
      const double* dsf = psf + 2 * (nc1 + 1);
      const double igam = 1. / s_gam[c];
      double psv, dsv;
      if (fabs(psf[i] - psf[i + 1]) < 1.E-6) {
        psv = (psf[i] + psf[i + 1]) * 0.5;
        dsv = exp(log(psv) * igam) * s_expf[c];
      } else {
        // psv, the log-mean of the face pressures, is psf[i+1] (e^d - 1) / d
        // with d = ln psf[i] - ln psf[i+1], so ln psv = ln psf[i+1] + x +
        // ln(sinh x / x) (x = d/2) and psv^(1/gamma) = psf[i+1]^(1/gamma)
        // e^((x + ln(sinh x / x)) / gamma): the face density times two short
        // series instead of a log and an exp (layers thinner than 0.4 scale
        // heights; thicker ones take the log and the exp)
        const double d = lpsf[i] - lpsf[i + 1];
        psv = (psf[i] - psf[i + 1]) / d;
        const double x = 0.5 * d;
        if (fabs(x) <= 0.2) dsv = dsf[i + 1] * exp_small((x + ln_sinhc(x)) * igam);
        else dsv = exp(log(psv) * igam) * s_expf[c];
      }
      wc[IPR * nc1 + i] -= psv;
      wc[IDN * nc1 + i] -= dsv;
    }
#else
    for (int t = threadIdx.x; t < ncb * nc1; t += blockDim.x) {
      int c, i;
      divmod_small(t, nc1, inv_nc1, c, i);
      double* wc = WC(c);
      const double* psf = PSF(c);
      double psv, dsv;
      if (fabs(psf[i] - psf[i + 1]) < 1.E-6)
        psv = (psf[i] + psf[i + 1]) / 2.;
      else
        psv = (psf[i] - psf[i + 1]) / log(psf[i] / psf[i + 1]);
      dsv = pow(psv, 1. / s_gam[c]) * s_expf[c];
      wc[IPR * nc1 + i] -= psv;
      wc[IDN * nc1 + i] -= dsv;
    }
#endif
    __syncthreads();
  }
  using TF = X1Flux<T>;
  TF* F = flux_array<TF>(v, 0);
#if EXO_X1_SHARED_BETA
  // both face values of every cell is-1 .. ie+1, the cell's WENO5
  // smoothness indicators computed once for the two (as the x2/x3 kernel
  // does): rec [2][nv][L+2] floats of each column, after its psf arrays
  const int ncell = L + 2;
  auto REC = [&](int c) {
    return reinterpret_cast<T*>(sm + (size_t)c * cstride + nv * nc1 + 3 * (nc1 + 1));
  };
  {
    const float inv_nc = 1.f / (float)ncell;
    for (int t = threadIdx.x; t < ncb * ncell; t += blockDim.x) {
      int c, m;
      divmod_small(t, ncell, inv_nc, c, m);
      const int cell = v.is - 1 + m;
      const double* wc = WC(c);
      T* rec = REC(c);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        if (n >= nv) break;
        const double* q = wc + n * nc1 + cell;
        const T q0 = T(q[-2]), q1 = T(q[-1]), q2 = T(q[0]), q3 = T(q[1]), q4 = T(q[2]);
        const WenoCell<T> wcl = weno_cell<T>(q0, q1, q2, q3, q4);
        rec[n * ncell + m] = weno_right<T>(wcl, q0, q1, q2, q3, q4);
        rec[(nv + n) * ncell + m] = weno_left<T>(wcl, q0, q1, q2, q3, q4);
      }
    }
  }
  __syncthreads();
#endif
  const float inv_faces = 1.f / (float)(L + 1);
  for (int t = threadIdx.x; t < ncb * (L + 1); t += blockDim.x) {
    int c, f;
    divmod_small(t, L + 1, inv_faces, c, f);
    const double* wc = WC(c);
    const double* psf = PSF(c);
    const int i = v.is + f;
    FaceGeo<TF> fg{TF(0.), TF(1.), TF(s_cthp[c]), TF(s_cosc[c])};
    // perturbations are formed in FP64 above; WENO5 runs in T, the restore in
    // FP64 and the Riemann solve in TF
    TF wl[5], wr[5], fx[5] = {TF(0.), TF(0.), TF(0.), TF(0.), TF(0.)};
#if EXO_X1_SHARED_BETA
    {
      const T* rec = REC(c);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        if (n >= nv) break;
        wl[n] = TF(rec[n * ncell + f]);             // the upper face of cell i-1
        wr[n] = TF(rec[(nv + n) * ncell + f + 1]);  // the lower face of cell i
      }
    }
#else
    #pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= nv) break;
      const double* q = wc + n * nc1;
      wl[n] = TF(weno_r<T>(q, 1, i - 1));
      wr[n] = TF(weno_l<T>(q, 1, i));
    }
#endif
    if (decomp) {
      // RestoreFromPerturbation (change_to_perturbation.cpp:159-222), in FP64
      double ps = psf[i];
      double xr = wr[IPR], xl = wl[IPR];
      xr += ps;
      if (xr < 0.) xr = ps;
      xl += ps;
      if (xl < 0.) xl = ps;
#if EXO_MIXED
      const double dsf = psf[2 * (nc1 + 1) + i];
#else
      double dsf = pow(ps, 1. / s_gam[c]) * s_expf[c];
#endif
      double dr = wr[IDN], dl = wl[IDN];
      dr += dsf;
      if (dr < 0.) dr = dsf;
      dl += dsf;
      if (dl < 0.) dl = dsf;
      wr[IPR] = TF(xr);
      wl[IPR] = TF(xl);
      wr[IDN] = TF(dr);
      wl[IDN] = TF(dl);
    }
    // x1 runs for the ideal gas only: LMARS or HLLC
    if (v.rsolver == EXO_RS_HLLC) riemann_hllc<TF>(v.gamma, IVX, fg, wl, wr, fx);
    else riemann_lmars<TF>(v.gamma, IVX, wl, wr, fx);
    TF* Fc = F + (size_t)s_base[c] + i;
    #pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= nv) break;
      Fc[n * vs] = fx[n];
    }
  }
}

// ----------------------------------------------------------- k_flux_x23 --
// Interior-side reconstruction of panel p at its own edge face (side s,
// along index a) for radial index i: the state CubedSphere::sendNeighborBlocks
// sends (L at Down/Right edges, R at Up/Left edges).
template <class T>
__device__ __forceinline__ void edge_interior_state(const DevView& v, int p, int s, int a,
                                                    int i, T* st) {
  long s2 = v.nc1, s3 = (long)v.nc1 * v.nc2;
  const T* W = prim_array<T>(v);
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    if (s == UP || s == DOWN) {
      const T* q = W + idx(v, p, n, v.ks + a, 0, i);
      st[n] = (s == DOWN) ? weno_r<T>(q, s2, v.je) : weno_l<T>(q, s2, v.js);
    } else {
      const T* q = W + idx(v, p, n, 0, v.js + a, i);
      st[n] = (s == RIGHT) ? weno_r<T>(q, s3, v.ke) : weno_l<T>(q, s3, v.ks);
    }
  }
}

template <class T>
__device__ __forceinline__ void edge_outer_state(const DevView& v, int p, int side, int a,
                                                 int i, T* st) {
  const EdgeEntry& e = v.edge[((size_t)p * 4 + side) * v.N + a];
  edge_interior_state<T>(v, e.src_panel, e.src_side, e.src_along, i, st);
  T V2 = st[IVY], V3 = st[IVZ];
  T U = T(e.r[0]) * V2 + T(e.r[1]) * V3;
  T V = T(e.r[2]) * V2 + T(e.r[3]) * V3;
  st[IVY] = T(e.q[0]) * U + T(e.q[1]) * V;
  st[IVZ] = T(e.q[2]) * U + T(e.q[3]) * V;
}

// One thread per face: grids whose level count leaves too many of a line's
// lanes idle (x23_uses_lines).
template <class T>
__device__ __forceinline__ void flux_x23_faces(const DevView& v, unsigned blk) {
  unsigned tid = blk * blockDim.x + threadIdx.x;
  unsigned nface = 6u * v.N * (v.N + 1) * v.L;  // per direction
  if (tid >= 2 * nface) return;
  int dir = tid < nface ? 1 : 2;
  unsigned r = dir == 1 ? tid : tid - nface;
  unsigned L = v.L, N = v.N;
  int i = v.is + (int)(r % L);
  r /= L;
  int k, j;
  int p;
  if (dir == 1) {  // x2 faces: j in [js, je+1], k in [ks, ke]
    j = v.js + (int)(r % (N + 1));
    r /= (N + 1);
    k = v.ks + (int)(r % N);
    p = (int)(r / N);
  } else {  // x3 faces: j in [js, je], k in [ks, ke+1]
    j = v.js + (int)(r % N);
    r /= N;
    k = v.ks + (int)(r % (N + 1));
    p = (int)(r / (N + 1));
  }
  T wl[5], wr[5], fx[5] = {T(0.), T(0.), T(0.), T(0.), T(0.)};
  long s2 = v.nc1, s3 = (long)v.nc1 * v.nc2;
  const T* W = prim_array<T>(v);
  FaceGeo<T> fg;
  int ivx;
  if (dir == 1) {
    #pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= v.nv) break;
      const T* q = W + idx(v, p, n, k, 0, i);
      wl[n] = weno_r<T>(q, s2, j - 1);
      wr[n] = weno_l<T>(q, s2, j);
    }
    if (j == v.js) edge_outer_state<T>(v, p, UP, k - v.ks, i, wl);
    else if (j == v.je + 1) edge_outer_state<T>(v, p, DOWN, k - v.ks, i, wr);
    fg = FaceGeo<T>{T(geo(v, GCOSF2, p, k, j)), T(geo(v, GSINF2, p, k, j)),
                    T(geo(v, GCTHP2, p, k, j)), T(geo(v, GCOSC, p, k, j))};
    ivx = IVY;
  } else {
    #pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= v.nv) break;
      const T* q = W + idx(v, p, n, 0, j, i);
      wl[n] = weno_r<T>(q, s3, k - 1);
      wr[n] = weno_l<T>(q, s3, k);
    }
    if (k == v.ks) edge_outer_state<T>(v, p, LEFT, j - v.js, i, wl);
    else if (k == v.ke + 1) edge_outer_state<T>(v, p, RIGHT, j - v.js, i, wr);
    fg = FaceGeo<T>{T(geo(v, GCOSF3, p, k, j)), T(geo(v, GSINF3, p, k, j)),
                    T(geo(v, GCTHP3, p, k, j)), T(geo(v, GCOSC, p, k, j))};
    ivx = IVZ;
  }
  // the velocity index as a literal, so the solvers index registers only
  if (ivx == IVY) riemann<T>(v.rsolver, v.gamma, IVY, fg, wl, wr, fx);
  else riemann<T>(v.rsolver, v.gamma, IVZ, fg, wl, wr, fx);
  T* F = flux_array<T>(v, dir);
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    F[idx(v, p, n, k, j, i)] = fx[n];
  }
}


// One thread per line of faces (the mixed build): for x2 faces the line (p, k, i) runs over
// j = js .. je+1, for x3 faces the line (p, j, i) over k = ks .. ke+1.  The
// six cells of the face's WENO5 stencils slide along the line in
// registers, so every cell is read once per line instead of six times; each
// face's reconstruction, edge replacement and Riemann solve are those of a
// face on its own (same values, same operations).
template <class T>
__device__ __forceinline__ void flux_x23_lines(const DevView& v, unsigned blk) {
  const unsigned tid = blk * blockDim.x + threadIdx.x;
  const unsigned L = v.L, N = v.N;
  const unsigned nline = 6u * N * L;  // per direction
  if (tid >= 2 * nline) return;
  const int dir = tid < nline ? 1 : 2;
  unsigned r = dir == 1 ? tid : tid - nline;
  const unsigned rl = v.div_L(r);
  const int i = v.is + (int)(r - rl * L);
  const unsigned rn = v.div_N(rl);
  const int a = (int)(rl - rn * N);  // position across the line: k - ks (x2) or j - js (x3)
  const int p = (int)rn;
  const int nv = v.nv;
  const size_t vs = v.cells;
  const long s = dir == 1 ? (long)v.nc1 : (long)v.nc1 * v.nc2;  // stride along the line
  const size_t base = dir == 1 ? idx(v, p, 0, v.ks + a, 0, i) : idx(v, p, 0, 0, v.js + a, i);
  const T* __restrict__ W = prim_array<T>(v) + base;
  const int c0 = dir == 1 ? v.js : v.ks, c1 = dir == 1 ? v.je : v.ke;
  T* F = flux_array<T>(v, dir);
  // window q[n][m] = cell (c - 3 + m) of the line for face c (cells c-1 | c)
  T q[5][6];
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= nv) break;
#pragma unroll
    for (int m = 0; m < 6; ++m) q[n][m] = T(__ldg(W + n * vs + (long)(c0 - 3 + m) * s));
  }
#if EXO_X23_SHARED_BETA
  WenoCell<T> wprev[5];  // indicators of cell c - 1
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= nv) break;
    wprev[n] = weno_cell<T>(q[n][0], q[n][1], q[n][2], q[n][3], q[n][4]);
  }
#endif
  for (int c = c0; c <= c1 + 1; ++c) {
    T wl[5], wr[5], fx[5] = {T(0.), T(0.), T(0.), T(0.), T(0.)};
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= nv) break;
#if EXO_X23_SHARED_BETA
      const WenoCell<T> wcur = weno_cell<T>(q[n][1], q[n][2], q[n][3], q[n][4], q[n][5]);
      wl[n] = weno_right<T>(wprev[n], q[n][0], q[n][1], q[n][2], q[n][3], q[n][4]);
      wr[n] = weno_left<T>(wcur, q[n][1], q[n][2], q[n][3], q[n][4], q[n][5]);
      wprev[n] = wcur;
#else
      wl[n] = weno5<T>(q[n][4], q[n][3], q[n][2], q[n][1], q[n][0]);  // weno_r of cell c-1
      wr[n] = weno5<T>(q[n][1], q[n][2], q[n][3], q[n][4], q[n][5]);  // weno_l of cell c
#endif
    }
    const int k = dir == 1 ? v.ks + a : c;
    const int j = dir == 1 ? c : v.js + a;
    if (dir == 1) {
      if (c == c0) edge_outer_state<T>(v, p, UP, a, i, wl);
      else if (c == c1 + 1) edge_outer_state<T>(v, p, DOWN, a, i, wr);
      FaceGeo<T> fg{T(geo(v, GCOSF2, p, k, j)), T(geo(v, GSINF2, p, k, j)),
                    T(geo(v, GCTHP2, p, k, j)), T(geo(v, GCOSC, p, k, j))};
      riemann<T>(v.rsolver, v.gamma, IVY, fg, wl, wr, fx);
    } else {
      if (c == c0) edge_outer_state<T>(v, p, LEFT, a, i, wl);
      else if (c == c1 + 1) edge_outer_state<T>(v, p, RIGHT, a, i, wr);
      FaceGeo<T> fg{T(geo(v, GCOSF3, p, k, j)), T(geo(v, GSINF3, p, k, j)),
                    T(geo(v, GCTHP3, p, k, j)), T(geo(v, GCOSC, p, k, j))};
      riemann<T>(v.rsolver, v.gamma, IVZ, fg, wl, wr, fx);
    }
    const size_t f0 = idx(v, p, 0, k, j, i);
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      if (n >= nv) break;
      F[f0 + n * vs] = fx[n];
    }
    if (c <= c1) {  // slide: the next face needs cell c + 3
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        if (n >= nv) break;
#pragma unroll
        for (int m = 0; m < 5; ++m) q[n][m] = q[n][m + 1];
        q[n][5] = T(__ldg(W + n * vs + (long)(c + 3) * s));
      }
    }
  }
}

// asynchronous 8-byte global -> shared copies (the next level's inputs)
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_one() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Faces staged through shared memory: a block of X23_THREADS threads takes
// 32 consecutive radial indices i (one per lane, so every global access of a
// warp is a coalesced row) of one line of one panel and direction, and walks
// the line in chunks of x23_chunk<T>() faces:
//   0. the chunk's cells (with the three-cell halos of its stencils) are in
//      shared memory, each cell copied once;
//   1. one thread per cell computes both face values of the cell's WENO5
//      reconstruction (the right-face value for the face above it, the
//      left-face value for the face below; the mixed build shares the
//      cell's smoothness indicators between the two, the FP64 build calls
//      weno5 for each as the reference does);
//   2. one thread per face takes the right-face value of the cell below
//      and the left-face value of the cell above -- the neighbour panel's
//      rotated state at a panel edge -- and solves the Riemann problem.
// Each face gets the values and operations it gets in the per-face and
// per-line kernels; phases 1 and 2 each keep few registers, so many warps
// are resident.
#ifndef EXO_X23_THREADS
#define EXO_X23_THREADS 128
#endif
constexpr int X23_THREADS = EXO_X23_THREADS;
// A line's 32 lanes are its radial indices, so the line form keeps
// L / (32 ceil(L / 32)) of its lanes busy: 3 of 32 at the exo2
// shallow-water grid's 3 levels, 62.5 % at HS94's 40.  Below a busy
// fraction the per-face form (X23_THREADS threads a block) is faster:
// measured at 40 and 64 levels, the FP64 build's crossover lies near 85 %
// (its line form is 16 % faster at 100 %, 2x slower at 62.5 %), the mixed
// build's near 65 % (line form 1.7x faster at 100 %).
#ifndef EXO_X23_LINE_BUSY_PCT
#define EXO_X23_LINE_BUSY_PCT (EXO_MIXED ? 65 : 85)
#endif
__host__ __device__ constexpr bool x23_uses_lines(int L) {
  return L * 100 >= EXO_X23_LINE_BUSY_PCT * 32 * ((L + 31) / 32);
}
template <class T>
__host__ __device__ constexpr int x23_chunk() {
  return sizeof(T) == 4 ? 15 : 7;
}
// blocks of the tiled x2/x3 kernel for one atmosphere: one per line of 32
// radial indices of one row of one panel and direction
__host__ __device__ constexpr unsigned x23_tile_blocks(int N, int L) {
  return 2u * 6u * (unsigned)N * (unsigned)((L + 31) / 32);
}

// cp.async of 4 or 8 bytes, zero-filled when src_bytes is 0
template <int B>
__device__ __forceinline__ void cp_async_zfill(void* smem_dst, const void* gsrc, int src_bytes) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gsrc), "n"(B),
               "r"(src_bytes)
               : "memory");
}

// The x2/x3 faces of one line (32 radial indices of one row of one panel
// and direction) chunk by chunk, with the same phases, values and
// operations per face as the per-face form.  Cell c of the line sits in ring
// slot (c - c0 + 3) mod XR; the copies of chunk q + 1's new cells are in
// flight while chunk q is finished.  Slots written for chunk q + 1 held
// cells at least XR = 2 CF + 5 below them, which chunk q no longer reads;
// the copies for chunk q + 2 start after the barrier that ends chunk q's
// reconstruction.
template <class T>
__device__ __forceinline__ void flux_x23_pipe(const DevView& v, unsigned blk) {
  constexpr int CF = x23_chunk<T>();
  constexpr int NC = CF + 1;
  constexpr int XR = 2 * CF + 5;
  __shared__ __align__(16) T ring[5][XR][32];
  __shared__ T srec[2][5][NC][32];
  const int N = v.N, L = v.L, nv = v.nv;
  const unsigned nit = (unsigned)((L + 31) / 32);
  unsigned r = blk;
  const int itile = (int)(r % nit);
  r /= nit;
  const int a = (int)(r % (unsigned)N);
  r /= (unsigned)N;
  const int p = (int)(r % 6u);
  const int dir = (int)(r / 6u) + 1;
  const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
  constexpr int NW = X23_THREADS / 32;
  const int il = itile * 32 + lane;
  const bool active = il < L;
  const int i = v.is + il;
  const size_t vs = v.cells;
  const long s = dir == 1 ? (long)v.nc1 : (long)v.nc1 * v.nc2;
  const size_t base = dir == 1 ? idx(v, p, 0, v.ks + a, 0, active ? i : v.is)
                               : idx(v, p, 0, 0, v.js + a, active ? i : v.is);
  const T* __restrict__ W = prim_array<T>(v) + base;
  const int c0 = dir == 1 ? v.js : v.ks, c1 = dir == 1 ? v.je : v.ke;
  const int nch = (N + 1 + CF - 1) / CF;
  // copies of cells [from, to] (line indices), rows (variable, cell) over the warps
  auto issue = [&](int from, int to) {
    const int nc = to - from + 1;
    for (int row = warp; row < nc * nv; row += NW) {
      const int n = row / nc, c = from + row % nc;
      int slot = c - c0 + 3;
      slot -= (slot >= XR) ? XR * (slot / XR) : 0;
      const bool ok = active && c <= c1 + 3;
      cp_async_zfill<sizeof(T)>(&ring[n][slot][lane], W + n * vs + (long)(ok ? c : c0) * s,
                                ok ? (int)sizeof(T) : 0);
    }
    cp_async_commit();
  };
  issue(c0 - 3, c0 + CF + 1);
  T* F = flux_array<T>(v, dir);
  for (int q = 0; q < nch; ++q) {
    const int cb = c0 + q * CF;
    if (q + 1 < nch) {
      issue(cb + CF + 2, cb + 2 * CF + 1);
      cp_async_wait_one();
    } else {
      cp_async_wait_all();
    }
    __syncthreads();
    // 1. both face values of the cells cb-1 .. cb+CF-1
    for (int mc = warp; mc < NC; mc += NW) {
      int s0 = cb - 1 - c0 + 3 + mc - 2;  // slot of cell cb-1+mc-2
      s0 -= (s0 >= XR) ? XR * (s0 / XR) : 0;
      int sl[5];
#pragma unroll
      for (int m = 0; m < 5; ++m) sl[m] = (s0 + m >= XR) ? s0 + m - XR : s0 + m;
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        if (n >= nv) break;
        const T q0 = ring[n][sl[0]][lane], q1 = ring[n][sl[1]][lane], q2 = ring[n][sl[2]][lane];
        const T q3 = ring[n][sl[3]][lane], q4 = ring[n][sl[4]][lane];
#if EXO_X23_SHARED_BETA
        const WenoCell<T> wc = weno_cell<T>(q0, q1, q2, q3, q4);
        srec[0][n][mc][lane] = weno_right<T>(wc, q0, q1, q2, q3, q4);
        srec[1][n][mc][lane] = weno_left<T>(wc, q0, q1, q2, q3, q4);
#else
        srec[0][n][mc][lane] = weno5<T>(q4, q3, q2, q1, q0);
        srec[1][n][mc][lane] = weno5<T>(q0, q1, q2, q3, q4);
#endif
      }
    }
    __syncthreads();
    if (!active) continue;
    // 2. the faces cb .. cb+CF-1 (up to c1+1)
    for (int mf = warp; mf < CF; mf += NW) {
      const int c = cb + mf;
      if (c > c1 + 1) break;
      T wl[5], wr[5], fx[5] = {T(0.), T(0.), T(0.), T(0.), T(0.)};
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        if (n >= nv) break;
        wl[n] = srec[0][n][mf][lane];
        wr[n] = srec[1][n][mf + 1][lane];
      }
      const int k = dir == 1 ? v.ks + a : c;
      const int j = dir == 1 ? c : v.js + a;
      if (dir == 1) {
        if (c == c0) edge_outer_state<T>(v, p, UP, a, i, wl);
        else if (c == c1 + 1) edge_outer_state<T>(v, p, DOWN, a, i, wr);
        FaceGeo<T> fg{T(geo(v, GCOSF2, p, k, j)), T(geo(v, GSINF2, p, k, j)),
                      T(geo(v, GCTHP2, p, k, j)), T(geo(v, GCOSC, p, k, j))};
        riemann<T>(v.rsolver, v.gamma, IVY, fg, wl, wr, fx);
      } else {
        if (c == c0) edge_outer_state<T>(v, p, LEFT, a, i, wl);
        else if (c == c1 + 1) edge_outer_state<T>(v, p, RIGHT, a, i, wr);
        FaceGeo<T> fg{T(geo(v, GCOSF3, p, k, j)), T(geo(v, GSINF3, p, k, j)),
                      T(geo(v, GCTHP3, p, k, j)), T(geo(v, GCOSC, p, k, j))};
        riemann<T>(v.rsolver, v.gamma, IVZ, fg, wl, wr, fx);
      }
      const size_t f0 = idx(v, p, 0, k, j, i);
#pragma unroll
      for (int n = 0; n < 5; ++n) {
        if (n >= nv) break;
        F[f0 + n * vs] = fx[n];
      }
    }
  }
}

template <class T>
__device__ __forceinline__ void flux_x23_block(const DevView& v, unsigned blk) {
  if constexpr (EXO_X23_TILES) {
    if (x23_uses_lines(v.L)) flux_x23_pipe<T>(v, blk);
    else flux_x23_faces<T>(v, blk);
  } else if constexpr (EXO_X23_LINES) {
    flux_x23_lines<T>(v, blk);
  } else {
    flux_x23_faces<T>(v, blk);
  }
}

// --------------------------------------------------------------- k_update -
template <class T>
__device__ __forceinline__ void update_block(const DevView& v, unsigned blk, int stage) {
  const unsigned tid = blk * blockDim.x + threadIdx.x;
  const unsigned L = v.L, N = v.N;
  if (tid >= 6u * N * N * L) return;
  const unsigned r1 = v.div_L(tid), r2 = v.div_N(r1), r3 = v.div_N(r2);
  const int i = v.is + (int)(tid - r1 * L);
  const int j = v.js + (int)(r1 - r2 * N);
  const int k = v.ks + (int)(r2 - r3 * N);
  const int p = (int)r3;
  const double wght = rk_beta(stage) * v.sc->dt;
  const bool shallow = (v.eqn == EXO_EQN_SHALLOW_YZ);
  const int nv = v.nv;
  // offsets: this cell (variable 0), variable stride, +1 in j and in k
  const size_t c0 = idx(v, p, 0, k, j, i), vs = v.cells;
  const size_t sj = (size_t)v.nc1, sk = (size_t)v.nc2 * v.nc1;
  // geometry of the column (k,j) and of its upper x2/x3 neighbours
  const size_t g0 = ((size_t)p * v.nc3 + k) * v.nc2 + j, gs = (size_t)6 * v.nc3 * v.nc2;
  auto G2 = [&](int f, size_t off) { return __ldg(v.geo + f * gs + g0 + off); };
  const double* uin = v.u + c0;  // read here, written below
  const double* u1in = v.u1 + c0;
  const double* __restrict__ win = v.w + c0;
  const X1Flux<T>* __restrict__ F0 = flux_array<X1Flux<T>>(v, 0) + c0;
  const T* __restrict__ F1 = flux_array<T>(v, 1) + c0;
  const T* __restrict__ F2 = flux_array<T>(v, 2) + c0;
  // every input of the cell is requested before any is used
  double uu[5], u1v[5], wv[5];
  X1Flux<T> f0l[5], f0r[5];
  T f1l[5], f1r[5], f2l[5], f2r[5];
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= nv) break;
    uu[n] = uin[n * vs];
    u1v[n] = stage ? u1in[n * vs] : 0.;
    wv[n] = __ldg(win + n * vs);
    f0l[n] = shallow ? X1Flux<T>(0.) : __ldg(F0 + n * vs);
    f0r[n] = shallow ? X1Flux<T>(0.) : __ldg(F0 + n * vs + 1);
    f1l[n] = __ldg(F1 + n * vs);
    f1r[n] = __ldg(F1 + n * vs + sj);
    f2l[n] = __ldg(F2 + n * vs);
    f2r[n] = __ldg(F2 + n * vs + sk);
  }
  const double x1fi = __ldg(v.x1f + i), x1fp = __ldg(v.x1f + i + 1);
  const double x1vi = __ldg(v.x1v + i), dx1fi = __ldg(v.dx1f + i);
  double un[5];
  // WeightedAve(u1, u, ...) then WeightedAve(u, u1, ...) (SSPRK(3,3) registers)
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= nv) break;
    if (stage == 0) {
      v.u1[c0 + n * vs] = uu[n];
      un[n] = 0. + 1.0 * uu[n];
    } else if (stage == 1) {
      un[n] = 0.25 * uu[n] + 0.75 * u1v[n];
    } else {
      un[n] = (2.0 / 3.0) * uu[n] + (1.0 / 3.0) * u1v[n];
    }
  }
  // AddFluxDivergence
  const double s = G2(GSINC, 0);
  const double d2 = G2(GDX2A, 0), d3 = G2(GDX3A, 0);
  const double dx3f2 = G2(GDX3A_F2, 0), dx3f2p = G2(GDX3A_F2, 1);
  const double dx2f3 = G2(GDX2A_F3, 0), dx2f3p = G2(GDX2A_F3, v.nc2);
  const double a1 = d2 * d3 * x1fi * x1fi * s;
  const double a1p = d2 * d3 * x1fp * x1fp * s;
  const double a2 = x1vi * dx3f2 * dx1fi;
  const double a2p = x1vi * dx3f2p * dx1fi;
  const double a3 = x1vi * dx2f3 * dx1fi;
  const double a3p = x1vi * dx2f3p * dx1fi;
  const double vol = dx1fi * d2 * d3 * x1vi * x1vi * s;
  // the mixed build multiplies by reciprocals of the volume and the radius
  // (one division each instead of eight; the FP64 build divides as the
  // reference does)
  [[maybe_unused]] const double ivol = inv_r(vol), irad = inv_r(x1vi);
  double du[5];
  // flux divergence in T (the x1 part in FP64 where its fluxes are); the
  // conserved state accumulates in FP64
  const T A1 = T(a1), A1p = T(a1p), A2 = T(a2), A2p = T(a2p), A3 = T(a3), A3p = T(a3p);
#pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= nv) break;
    double change;
    if constexpr (sizeof(T) == sizeof(double)) {
      T dflx = (A1p * f0r[n] - A1 * f0l[n]);
      dflx += (A2p * f1r[n] - A2 * f1l[n]);
      dflx += (A3p * f2r[n] - A3 * f2l[n]);
      change = wght * dflx / vol;
    } else if constexpr (sizeof(X1Flux<T>) == sizeof(double)) {
      T d23 = (A2p * f1r[n] - A2 * f1l[n]);
      d23 += (A3p * f2r[n] - A3 * f2l[n]);
      const double d1 = a1p * f0r[n] - a1 * f0l[n];
      change = wght * ((d1 + (double)d23) * ivol);
    } else {
      T dflx = (A1p * f0r[n] - A1 * f0l[n]);
      dflx += (A2p * f1r[n] - A2 * f1l[n]);
      dflx += (A3p * f2r[n] - A3 * f2l[n]);
      change = wght * (double)(dflx / T(vol));
    }
    if (shallow) {
      un[n] -= change;
    } else {
      du[n] = 0.;
      du[n] -= change;
    }
  }
  double* out = shallow ? un : du;
  // AddCoordTermsDivergence (gnomonic_equiangle.cpp:834-879)
  {
    const double cosine = G2(GCOSC, 0);
    const double sine2 = s * s;
#if EXO_MIXED
    const double x_ov_rD = (x1vi * dx3f2 * dx1fi * G2(GSINF2, 0) -
                            x1vi * dx3f2p * dx1fi * G2(GSINF2, 1)) * ivol;
    const double y_ov_rC = (x1vi * dx2f3 * dx1fi * G2(GSINF3, 0) -
                            x1vi * dx2f3p * dx1fi * G2(GSINF3, v.nc2)) * ivol;
#else
    const double x_ov_rD = (x1vi * dx3f2 * dx1fi * G2(GSINF2, 0) -
                            x1vi * dx3f2p * dx1fi * G2(GSINF2, 1)) / vol;
    const double y_ov_rC = (x1vi * dx2f3 * dx1fi * G2(GSINF3, 0) -
                            x1vi * dx2f3p * dx1fi * G2(GSINF3, v.nc2)) / vol;
#endif
    const double rho = wv[IDN], v1 = wv[IVX], v2 = wv[IVY], v3 = wv[IVZ];
    [[maybe_unused]] const double radius = x1vi;
    double pr;
    const double v_2 = v2 + v3 * cosine;
    const double v_3 = v3 + v2 * cosine;
    if (shallow) {
      pr = 0.5 * rho * rho;
    } else {
      pr = wv[IPR];
#if EXO_MIXED
      double src1 = (2.0 * pr + rho * (v2 * v_2 + v3 * v_3)) * irad;
#else
      double src1 = (2.0 * pr + rho * (v2 * v_2 + v3 * v_3)) / radius;
#endif
      out[IVX] += wght * src1;
    }
#if EXO_MIXED
    double src2 = -x_ov_rD * (pr + rho * v3 * v3 * sine2) - rho * v1 * v_2 * irad;
    out[IVY] += wght * src2;
    double src3 = -y_ov_rC * (pr + rho * v2 * v2 * sine2) - rho * v1 * v_3 * irad;
#else
    double src2 = -x_ov_rD * (pr + rho * v3 * v3 * sine2) - rho * v1 * v_2 / radius;
    out[IVY] += wght * src2;
    double src3 = -y_ov_rC * (pr + rho * v2 * v2 * sine2) - rho * v1 * v_3 / radius;
#endif
    out[IVZ] += wght * src3;
    // constant gravity (patches/25.constant_acc.patch:35-53)
    if (v.grav != 0.) {
      double src = wght * rho * v.grav;
      out[IVX] += src;
      if (!shallow) out[IEN] += src * v1;
    }
    // W92 Coriolis (examples/2023-Chen-exo3/W92.cpp:48-70)
    if (v.coriolis == EXO_CORIOLIS_W92) {
      double f = G2(GFCOR, 0);
      double U = G2(GCR0, 0) * v2 + G2(GCR1, 0) * v3;
      double V = G2(GCR2, 0) * v2 + G2(GCR3, 0) * v3;
      U = -U;
      double llU = f * V, llV = -f * U;
      double mU = -llU;
      double acc2 = G2(GCQ0, 0) * mU + G2(GCQ1, 0) * llV;
      double acc3 = G2(GCQ2, 0) * mU + G2(GCQ3, 0) * llV;
      double a2c = acc2 + acc3 * cosine, a3c = acc3 + acc2 * cosine;
      out[IVY] += wght * rho * a2c;
      out[IVZ] += wght * rho * a3c;
    }
    // CubedSphere::CalculateCoriolisForce3 (cubed_sphere.cpp:197-231): blocks
    // 1 and 5 (panels 0 and 4) carry the rotation axis through their centre
    if (v.coriolis == EXO_CORIOLIS_3D) {
      const double A = G2(GC3A, 0) * rho;
      const double x = G2(GTANX, 0), y = G2(GTANY, 0), C = G2(GC3C, 0), D = G2(GC3D, 0);
      double cF1, cF2, cF3;
      if (p == 0 || p == 4) {
        cF1 = A * (y * C * v2 - x * D * v3);
        cF2 = A * (-y * C * v1 - v3);
        cF3 = A * (x * D * v1 + v2);
      } else {
        cF1 = -A * D * v3;
        cF2 = A * x * v3;
        cF3 = A * (D * v1 - x * v2);
      }
      out[IVX] += wght * cF1;
      out[IVY] += wght * cF2;
      out[IVZ] += wght * cF3;
    }
    // Held-Suarez forcing (examples/2023-Chen-exo3/hs94.cpp:59-155)
    if (v.forcing == EXO_FORCING_HS94) {
      // Coriolis on the momenta in latitude-longitude (hs94.cpp:82-104)
      {
        double f = G2(GFCOR, 0);
        double U = G2(GCR0, 0) * v2 + G2(GCR1, 0) * v3;
        double V = G2(GCR2, 0) * v2 + G2(GCR3, 0) * v3;
        U = -U;
        double m2 = rho * U, m3 = rho * V;
        double llU = f * m3, llV = -f * m2;
        double mU = -llU;
        double acc2 = G2(GCQ0, 0) * mU + G2(GCQ1, 0) * llV;
        double acc3 = G2(GCQ2, 0) * mU + G2(GCQ3, 0) * llV;
        double a2c = acc2 + acc3 * cosine, a3c = acc3 + acc2 * cosine;
        out[IVY] += wght * a2c;
        out[IVZ] += wght * a3c;
      }
      // Rayleigh drag and Newtonian cooling (hs94.cpp:110-153)
      {
        const double* hs = v.hs;
        double scaled_z = pr / hs[HS_P0];
        double sigma = pr / hs[HS_P0];
        double sigma_p = (sigma - hs[HS_SIGMAB]) / (1. - hs[HS_SIGMAB]);
        double Kv = (sigma_p < 0.0) ? 0.0 : sigma_p * hs[HS_KF];
        double Teq_p = hs[HS_TS] - hs[HS_DT] * G2(GSLAT2, 0) -
                       hs[HS_DTHETA] * log(scaled_z) * G2(GCLAT2, 0);
        Teq_p *= pow(scaled_z, hs[HS_KAPPA]);
        double Teq = (Teq_p > 200.) ? Teq_p : 200.;
        double temp = pr / rho / v.Rd;
        sigma_p = (sigma_p < 0.0) ? 0.0 : sigma_p * G2(GCLAT4, 0);
        double Kt = hs[HS_KA] + (hs[HS_KS] - hs[HS_KA]) * sigma_p;
        double m1 = rho * v1, m2 = rho * v2, m3 = rho * v3;
        double m2c = m2 + m3 * cosine, m3c = m3 + m2 * cosine;
        out[IVX] += -wght * Kv * m1;
        out[IVY] += -wght * Kv * m2c;
        out[IVZ] += -wght * Kv * m3c;
        out[IEN] += -wght * hs[HS_CVM] * rho * Kt * (temp - Teq);
      }
    }
  }
  double* uout = v.u + c0;
  if (shallow) {
#pragma unroll
    for (int n = 0; n < 4; ++n) uout[n * vs] = un[n];
  } else if (v.implicit_flag & 1) {
    double* duout = v.du + c0;
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      uout[n * vs] = un[n];
      duout[n * vs] = du[n];
    }
  } else {
#pragma unroll
    for (int n = 0; n < 5; ++n) uout[n * vs] = un[n] + 1. * du[n];
  }
}

// ------------------------------------------------------------- k_implicit -
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

// Structural non-zeros of the X1 flux Jacobian dF/dq (flux_decomposition.hpp:
// 100-120): row 0 = e_1; rows 2 and 3 carry three entries each.
__host__ __device__ constexpr bool fj_nz(int r, int q) {
  return r == 1 || r == 4 || (r == 0 && q == 1) || (r == 2 && q <= 2) ||
         (r == 3 && (q <= 1 || q == 3));
}
// structural non-zeros of R (right eigenvectors, columns) and R^-1 (rows)
__host__ __device__ constexpr bool r_nz(int r, int c) {
  return c < 3 || (r == 2 && c == 3) || (r == 3 && c == 4) || r == 4;
}
__host__ __device__ constexpr bool ri_nz(int r, int c) {
  return r < 3 || c == 0 || (r == 3 && c == 2) || (r == 4 && c == 3);
}

// One cell of a column, velocities projected (v2 += v3 cos, v3 *= sin): the
// primitives and the two derived quantities of its flux Jacobian.
template <class R>
struct ColCell {
  R rho, v1, v2, v3, p, s2, hr;  // s2 = |v|^2, hr = (g+1)/g * p/rho (g = gamma-1)
  R sq, isq;                     // sqrt(rho), 1/sqrt(rho) (FP32 blocks)
};

// entry (r, q) of dF/dq at a cell, in the reference's expression order
template <int r, int q, class R>
__device__ __forceinline__ R fj_entry(const ColCell<R>& c, R gm1) {
  if constexpr (r == 0) return R(1);
  else if constexpr (r == 1) {
    if constexpr (q == 0) return gm1 * c.s2 / 2 - c.v1 * c.v1;
    else if constexpr (q == 1) return (R(2) - gm1) * c.v1;
    else if constexpr (q == 2) return -gm1 * c.v2;
    else if constexpr (q == 3) return -gm1 * c.v3;
    else return gm1;
  } else if constexpr (r == 2) {
    if constexpr (q == 0) return -c.v1 * c.v2;
    else if constexpr (q == 1) return c.v2;
    else return c.v1;
  } else if constexpr (r == 3) {
    if constexpr (q == 0) return -c.v1 * c.v3;
    else if constexpr (q == 1) return c.v3;
    else return c.v1;
  } else {
    if constexpr (q == 0) return ((gm1 - 1) * c.s2 / 2 - c.hr) * c.v1;
    else if constexpr (q == 1) return c.hr + c.s2 / 2 - gm1 * c.v1 * c.v1;
    else if constexpr (q == 2) return -gm1 * c.v2 * c.v1;
    else if constexpr (q == 3) return -gm1 * c.v3 * c.v1;
    else return (gm1 + 1) * c.v1;
  }
}

// compile-time loops (the matrix entries live in registers, so every index
// has to be a constant)
template <int N, class F, int... I>
__device__ __forceinline__ void unroll_impl(F&& f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void unroll(F&& f) {
  unroll_impl<N>(f, std::make_integer_sequence<int, N>{});
}

// |A| = R |Lambda| R^-1 at the Roe average of a face (flux_decomposition.hpp:
// 34-98).  Exact build: the reference's products R*Lambda and (R*Lambda)*R^-1
// summed in its order, skipping only terms that are structurally zero (the
// value is the same; at most the sign of an exact zero differs).  Mixed
// build: the same matrix as |u| I + (|u-c|-|u|) r0 l0^T + (|u+c|-|u|) r2 l2^T
// (the three |u| eigenvalues coincide), with shared reciprocals.  FP32
// blocks take sqrt(rho) and 1/sqrt(rho) from the cells and the sound speed
// and its reciprocal from one rsqrt (one rsqrt and two reciprocals a face;
// 1.6 % faster); FP64 blocks keep sqrt and division, which measured 3 %
// faster than the same rewrite in FP64.
template <class R>
__device__ __forceinline__ void abs_jacobian(const ColCell<R>& L, const ColCell<R>& R_, R gm1,
                                             R gamma, R A[5][5]) {
  R wl[5] = {L.rho, L.v1, L.v2, L.v3, L.p};
  R wr[5] = {R_.rho, R_.v1, R_.v2, R_.v3, R_.p};
#if EXO_MIXED
  // FP32 blocks take the cells' sqrt(rho) and 1/sqrt(rho); the same scheme
  // in FP64 (with a Newton-refined rsqrt) measured 0.5 % slower
  constexpr bool f32 = sizeof(R) == 4;
  const R one = R(1), half = R(0.5);
  R sqrtdl, sqrtdr, isl, isr, isdlpdr;
  if constexpr (f32) {
    sqrtdl = L.sq;
    sqrtdr = R_.sq;
    isdlpdr = inv_r(sqrtdl + sqrtdr);
    isl = isdlpdr * L.isq;
    isr = isdlpdr * R_.isq;
  } else {
    sqrtdl = sqrt_r(wl[IDN]);
    sqrtdr = sqrt_r(wr[IDN]);
    isdlpdr = inv_r(sqrtdl + sqrtdr);
    if constexpr (EXO_IMPL_RCP_NR) {
      isl = isdlpdr * inv_r(sqrtdl);
      isr = isdlpdr * inv_r(sqrtdr);
    } else {
      isl = isdlpdr / sqrtdl;
      isr = isdlpdr / sqrtdr;
    }
  }
  R rr = sqrtdl * sqrtdr;
  R u = (sqrtdl * wl[IVX] + sqrtdr * wr[IVX]) * isdlpdr;
  R v = (sqrtdl * wl[IVY] + sqrtdr * wr[IVY]) * isdlpdr;
  R w = (sqrtdl * wl[IVZ] + sqrtdr * wr[IVZ]) * isdlpdr;
  R inv_gm1 = one / gm1;
  R el = wl[IPR] * inv_gm1 + half * wl[IDN] * L.s2;
  R er = wr[IPR] * inv_gm1 + half * wr[IDN] * R_.s2;
  R hbar = (el + wl[IPR]) * isl + (er + wr[IPR]) * isr;
  R ke = half * (u * u + v * v + w * w);
  R p = (hbar - ke) * (gm1 / (gm1 + one)) * rr;
  R irr, cs, i2cshp;
  if constexpr (f32) {
    irr = L.isq * R_.isq;
    const R cs2 = gamma * p * irr;
    const R ics = rsqrt_r(cs2);
    cs = cs2 * ics;
    i2cshp = ics;  // times 1/(2 hp) below
  } else {
    irr = inv_r(rr);
    cs = sqrt_r(gamma * p * irr);
  }
  R hp = (gm1 + one) * inv_gm1 * p * irr;
  R h = hp + ke;
  R ihp = inv_r(hp), i2hp = half * ihp;
  if constexpr (f32)
    i2cshp *= i2hp;
  else if constexpr (EXO_IMPL_RCP_NR)
    i2cshp = i2hp * inv_r(cs);
  else
    i2cshp = i2hp / cs;
  R au = abs_r(u), al = abs_r(u - cs) - au, ar = abs_r(u + cs) - au;
  R l0[5] = {al * (cs * ke + u * hp) * i2cshp, al * (-hp - cs * u) * i2cshp, -al * v * i2hp,
              -al * w * i2hp, al * i2hp};
  R l2[5] = {ar * (cs * ke - u * hp) * i2cshp, ar * (hp - cs * u) * i2cshp, -ar * v * i2hp,
              -ar * w * i2hp, ar * i2hp};
  R r0[5] = {one, u - cs, v, w, h - u * cs};
  R r2[5] = {one, u + cs, v, w, h + u * cs};
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) A[r][c] = (r == c ? au : R(0)) + r0[r] * l0[c] + r2[r] * l2[c];
#else
  double prim[5];
  roe_average(prim, gm1, wl, wr);
  double fsig = 1., feps = 1.;
  double cs = sqrt((1. + (gamma - 1) * feps / fsig) * prim[IPR] / prim[IDN]);
  double rr = prim[IDN], u = prim[IVX], v = prim[IVY], w = prim[IVZ], p = prim[IPR];
  double ke = 0.5 * (u * u + v * v + w * w);
  double hp = (gm1 + 1.) / gm1 * p / rr;
  double h = hp + ke;
  const double Rm[5][5] = {{1., 1., 1., 0., 0.},
                           {u - cs, u, u + cs, 0., 0.},
                           {v, v, v, 1., 0.},
                           {w, w, w, 0., 1.},
                           {h - u * cs, ke, h + u * cs, v, w}};
  double mv2 = -v / (2. * hp), mw2 = -w / (2. * hp), i2 = 1. / (2. * hp);
  const double Ri[5][5] = {
      {(cs * ke + u * hp) / (2. * cs * hp), (-hp - cs * u) / (2. * cs * hp), mv2, mw2, i2},
      {(hp - ke) / hp, u / hp, v / hp, w / hp, -1. / hp},
      {(cs * ke - u * hp) / (2. * cs * hp), (hp - cs * u) / (2. * cs * hp), mv2, mw2, i2},
      {-v, 0., 1., 0., 0.},
      {-w, 0., 0., 1., 0.}};
  const double lam[5] = {fabs(u - cs), fabs(u), fabs(u + cs), fabs(u), fabs(u)};
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double s = 0.;
      bool first = true;
#pragma unroll
      for (int k = 0; k < 5; ++k)
        if (r_nz(r, k) && ri_nz(k, c)) {
          double term = (Rm[r][k] * lam[k]) * Ri[k][c];
          s = first ? term : s + term;
          first = false;
        }
      A[r][c] = s;
    }
#endif
}

// Solve with the LU factors of implicit_column's mixed build (rows taken in
// the order 1, 4, 2, 3, 0, threshold row swaps packed 3 bits per step): y
// holds the right-hand side with its rows in natural order on entry and the
// solution, unknowns in order, on exit.
template <class R>
__device__ __forceinline__ void lu_solve_rows(const R (&t)[5][5], const R (&idg)[5],
                                              unsigned perm, bool swapped, R* y) {
  constexpr int O[5] = {1, 4, 2, 3, 0};
  if (swapped) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const unsigned pk = (perm >> (3 * k)) & 7u;
#pragma unroll
      for (int r = k + 1; r < 5; ++r) {
        const bool sw = (pk == (unsigned)r);
        const R a = y[O[k]], b = y[O[r]];
        y[O[k]] = sw ? b : a;
        y[O[r]] = sw ? a : b;
      }
    }
  }
#pragma unroll
  for (int r = 1; r < 5; ++r)
#pragma unroll
    for (int k = 0; k < r; ++k) y[O[r]] -= t[O[r]][k] * y[O[k]];
  R z[5];
#pragma unroll
  for (int r = 4; r >= 0; --r) {
    R acc = y[O[r]];
#pragma unroll
    for (int q = r + 1; q < 5; ++q) acc -= t[O[r]][q] * z[q];
    z[r] = acc * idg[r];
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) y[r] = z[r];
}

// BackwardSubstitution of the full correction (forward_backward.hpp:90-126):
// delta_i -= (A c)_i delta_{i+1} from level ie (delta_ie given in dp) down
// to is, each corrected update stored through io.  kPipe: software-pipelined,
// the next level's factors and state in flight while a level finishes (for
// the few resident columns of the solve kernel); otherwise one level at a
// time, leaving the latency to the many columns of the back-substitution
// kernel.
template <class IO, bool kPipe = true>
__device__ __forceinline__ void implicit_backward_full(IO& io, int is, int ie,
                                                       typename IO::Real* dp) {
  using R = typename IO::Real;
  auto store = [&](int i, const double* u) {
    double d[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) d[n] = dp[n];
    io.ustore(i, u, d);
  };
  if constexpr (!kPipe) {
    {
      double u[5];
      io.uload(ie, u);
      store(ie, u);
    }
#pragma unroll 1
    for (int i = ie - 1; i >= is; --i) {
      R cs[30];
      double u[5];
#pragma unroll
      for (int e = 0; e < 30; ++e) cs[e] = io.scr(i - is, e);
      io.uload(i, u);
      R dl[5];
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        R ad = cs[r * 5] * dp[0];
#pragma unroll
        for (int k = 1; k < 5; ++k) ad += cs[r * 5 + k] * dp[k];
        dl[r] = cs[25 + r] - ad;
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) dp[r] = dl[r];
      store(i, u);
    }
    return;
  }
  R cur_s[30];
  double cur_u[5];
  io.uload(ie, cur_u);
  store(ie, cur_u);
  if (ie > is) {
#pragma unroll
    for (int e = 0; e < 30; ++e) cur_s[e] = io.scr(ie - 1 - is, e);
    io.uload(ie - 1, cur_u);
  }
#pragma unroll 1
  for (int i = ie - 1; i >= is; --i) {
    R nxt_s[30];
    double nxt_u[5];
    if (i > is) {
#pragma unroll
      for (int e = 0; e < 30; ++e) nxt_s[e] = io.scr(i - 1 - is, e);
      io.uload(i - 1, nxt_u);
    }
    R dl[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      R ad = cur_s[r * 5] * dp[0];
#pragma unroll
      for (int k = 1; k < 5; ++k) ad += cur_s[r * 5 + k] * dp[k];
      dl[r] = cur_s[25 + r] - ad;
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) dp[r] = dl[r];
    store(i, cur_u);
    if (i > is) {
#pragma unroll
      for (int e = 0; e < 30; ++e) cur_s[e] = nxt_s[e];
#pragma unroll
      for (int n = 0; n < 5; ++n) cur_u[n] = nxt_u[n];
    }
  }
}

// The back substitution of the stepping kernel's FP64 blocks (mixed build)
// with the state u moved through shared memory by the warp: the warp's 32
// columns go down BWD_TL levels at a time; each lane copies four levels of
// a column for one variable in one 32-byte run (the per-lane accesses of
// one level are 816 bytes apart, a sector each), the next chunk's copies in
// flight while a chunk is corrected.  The factors are read per lane, one
// level ahead, as in implicit_backward_full (they are contiguous across the
// warp).  io.live: the lanes of the warp with a column.  wtile: 2 x 5 x 32 x
// (BWD_TL + 1) doubles of shared memory for the warp alone.
constexpr int BWD_TL = 4;
// the two u tiles of a warp's back substitution (5 variables x 32 columns x
// BWD_TL levels, padded)
constexpr int WARP_TILE_DOUBLES = 2 * 5 * 32 * (BWD_TL + 1);
// levels of look-ahead of the factor loads (1 or 2): two in the FP64 build
// (implicit 8.63 -> 8.39 ms per 6x192^2x96 launch), one in the mixed build,
// where two measured 2.6 % slower
#ifndef EXO_BWD_AHEAD
#define EXO_BWD_AHEAD (EXO_MIXED ? 1 : 2)
#endif
__device__ __forceinline__ void airparcel_round_trip(double* u, double Rd, double gamma);
// the stepping solve's shared doubles per thread
constexpr int IMPL_SM_STRIDE = EXO_IMPL_AP_SMEM ? 87 : 61;
static_assert(32 * IMPL_SM_STRIDE >= WARP_TILE_DOUBLES,
              "the tiled back substitution's buffers fit in the warp's slices");
// NB = 5: the full correction (30 factors per level, delta on every
// variable); NB = 3: the partial one (12 factors per level, delta on rho,
// m1 and E, the explicit du on m2 and m3, read per lane one level ahead).
template <int NB, class IO>
__device__ __forceinline__ void implicit_backward_tiled(IO& io, int is, int ie,
                                                        typename IO::Real* dp, double* wtile) {
  static_assert(BWD_TL == 4, "the lane -> (column, level) split below assumes 4 levels");
  static_assert(NB == 5 || NB == 3, "5x5 or 3x3 blocks");
  constexpr int NF = NB * NB + NB;  // factors per level: (A c)_i and delta_i
  constexpr int TS = BWD_TL + 1;
  constexpr int TW = 5 * 32 * TS;
  const unsigned live = io.live;
  const int lane = (int)(threadIdx.x & 31);
  __syncwarp(live);
  // lane copies level (lane & 3) of columns (lane >> 2) + 8 m, m = 0..3
  // (in a warp with a column in every lane)
  double* ub[4];
#pragma unroll
  for (int m = 0; m < 4; ++m)
    ub[m] = reinterpret_cast<double*>(__shfl_sync(
        live, reinterpret_cast<unsigned long long>(io.uc), ((lane >> 2) + 8 * m) & 31));
  const int l = lane & 3;
  const int nch = (ie - is + BWD_TL) / BWD_TL;
  auto range = [&](int c, int& lo, int& hi) {
    hi = ie - c * BWD_TL;
    lo = max(is, hi - BWD_TL + 1);
  };
  // a warp with a column in every lane copies in 32-byte runs; the last warp
  // of a member may have fewer, and there each lane copies its own column
  const bool full = live == 0xffffffffu;
  auto load = [&](int c) {
    double* t = wtile + (c & 1) * TW;
    int lo, hi;
    range(c, lo, hi);
    if (full) {
      if (lo + l <= hi) {
#pragma unroll
        for (int e = 0; e < 20; ++e) {
          const int m = e & 3, n = e >> 2;
          cp_async8(&t[(n * 32 + (lane >> 2) + 8 * m) * TS + l], ub[m] + n * io.vs + lo + l);
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < 20; ++e) {
        const int ll = e & 3, n = e >> 2;
        if (lo + ll <= hi) cp_async8(&t[(n * 32 + lane) * TS + ll], io.uc + n * io.vs + lo + ll);
      }
    }
    cp_async_commit();
  };
  load(0);
  if (nch > 1) load(1);
  using R = typename IO::Real;
  // the factors of the next level (cur_s) and, with EXO_BWD_AHEAD 2, of the
  // one after (ahd_s): their loads are in flight for two levels (the
  // registers of the finished forward sweep are free)
  R cur_s[NF], ahd_s[NF];
  if (ie > is) {
#pragma unroll
    for (int e = 0; e < NF; ++e) cur_s[e] = io.scr(ie - 1 - is, e);
  }
  if constexpr (EXO_BWD_AHEAD == 2) {
    if (ie - 1 > is) {
#pragma unroll
      for (int e = 0; e < NF; ++e) ahd_s[e] = io.scr(ie - 2 - is, e);
    }
  }
  // the partial correction's explicit du of m2 and m3, one level ahead
  double cur_du[2] = {0., 0.};
  if constexpr (NB == 3) {
    cur_du[0] = *io.duptr(ie, IVY);
    cur_du[1] = *io.duptr(ie, IVZ);
  }
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) cp_async_wait_one();
    else cp_async_wait_all();
    __syncwarp(live);
    double* t = wtile + (c & 1) * TW;
    int lo, hi;
    range(c, lo, hi);
    for (int i = hi; i >= lo; --i) {
      double nxt_du[2] = {0., 0.};
      if constexpr (NB == 3) {
        if (i > is) {
          nxt_du[0] = *io.duptr(i - 1, IVY);
          nxt_du[1] = *io.duptr(i - 1, IVZ);
        }
      }
      if (i < ie) {
        R nxt_s[NF];
        const int ahead = i - EXO_BWD_AHEAD;  // the level whose factors load now
        if (ahead >= is) {
#pragma unroll
          for (int e = 0; e < NF; ++e) nxt_s[e] = io.scr(ahead - is, e);
        }
        R dl[NB];
#pragma unroll
        for (int r = 0; r < NB; ++r) {
          R ad = cur_s[r * NB] * dp[0];
#pragma unroll
          for (int k = 1; k < NB; ++k) ad += cur_s[r * NB + k] * dp[k];
          dl[r] = cur_s[NB * NB + r] - ad;
        }
#pragma unroll
        for (int r = 0; r < NB; ++r) dp[r] = dl[r];
        if constexpr (EXO_BWD_AHEAD == 2) {
#pragma unroll
          for (int e = 0; e < NF; ++e) {
            cur_s[e] = ahd_s[e];
            ahd_s[e] = nxt_s[e];
          }
        } else {
#pragma unroll
          for (int e = 0; e < NF; ++e) cur_s[e] = nxt_s[e];
        }
      }
      // the corrected update of every variable
      double d[5];
      if constexpr (NB == 5) {
#pragma unroll
        for (int n = 0; n < 5; ++n) d[n] = dp[n];
      } else {
        d[IDN] = dp[0];
        d[IVX] = dp[1];
        d[IVY] = cur_du[0];
        d[IVZ] = cur_du[1];
        d[IEN] = dp[2];
        cur_du[0] = nxt_du[0];
        cur_du[1] = nxt_du[1];
      }
      double uu[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) uu[n] = t[(n * 32 + lane) * TS + (i - lo)] + 1. * d[n];
      if (io.stage == 2) airparcel_round_trip(uu, io.Rd, io.gamma);
#pragma unroll
      for (int n = 0; n < 5; ++n) t[(n * 32 + lane) * TS + (i - lo)] = uu[n];
    }
    __syncwarp(live);
    if (full) {
      if (lo + l <= hi) {
#pragma unroll
        for (int e = 0; e < 20; ++e) {
          const int m = e & 3, n = e >> 2;
          ub[m][n * io.vs + lo + l] = t[(n * 32 + (lane >> 2) + 8 * m) * TS + l];
        }
      }
    } else {
#pragma unroll
      for (int e = 0; e < 20; ++e) {
        const int ll = e & 3, n = e >> 2;
        if (lo + ll <= hi) io.uc[n * io.vs + lo + ll] = t[(n * 32 + lane) * TS + ll];
      }
    }
    __syncwarp(live);
    if (c + 2 < nch) load(c + 2);
  }
}

// The vertical 5x5 block-tridiagonal correction of one radial column
// (ImplicitSolver::SolveImplicit3D X1 branch, solve_implicit_3d.cpp:102-179,
// with FullCorrection, full_correction.cpp:32-165, and ForwardSweep /
// BackwardSubstitution, forward_backward.hpp:15-126), one thread per column.
//
// Per level the forward sweep builds the rows of a_i, b_i, c_i from the two
// face Jacobians |A|(i-1/2), |A|(i+1/2) and the three cell Jacobians, forms
// t = a_i - b_i (A c)_{i-1} and x = du_i/dt - b_i delta_{i-1} row by row,
// then
//   exact build: inverts t by Gauss-Jordan with partial pivoting (the
//                reference's inverse) and multiplies, every sum in the
//                reference's order: the result is the CPU restatement's to
//                the bit;
//   mixed build: solves t [X | y] = [c_i | x] by LU with partial pivoting.
// (A c)_i (25) and delta_i (5) go to scratch for the back substitution.  The
// face Jacobian |A|(i+1/2) waits in this thread's slice of shared memory
// until it becomes |A|(i-1/2) of the next level.
//   io.w(i, out[5])  primitives of level i (is-1 .. ie+2), unprojected
//   io.scr(lev, e)   scratch double e (0..29) of level lev = i - is
//   io.uload(i, u[5]), io.ustore(i, u[5], d[5])  the corrected update d of
//                    level i, from ie down to is, with the state u loaded
//                    for it beforehand (callers that only need d load nothing)
//   io.wptr(i, n), io.duptr(i, n)  addresses of w and of the explicit update
//                    du of level i (the inputs are prefetched through shared memory)
//   sa, sp, ss       this thread's shared memory: entry e (0..49) of the two
//                    face blocks at sa[e * ss], prefetch slot n (0..9) at
//                    sp[n * ss]
// kBwd false: the forward sweep only, with delta_ie stored as scratch
// entries 25..29 of the last level (implicit_backward_full finishes it).
template <class IO, bool kBwd = true>
__device__ __forceinline__ void implicit_column(IO& io, typename IO::Real* sa, double* sp, int ss,
                                                double cos_theta, double sin_theta, double d2,
                                                double d3, const double* x1f, const double* x1v,
                                                const double* dx1f, int is, int ie, double dt,
                                                double gamma, double grav,
                                                double* wt = nullptr) {
  using R = typename IO::Real;
  using ColCell = exo::EXO_KNS::ColCell<R>;
  const double s = sin_theta;
  // gmm1 of every cell; the face average equals it
  const R gm1 = R((gamma - 1.) * 1. / 1.);
  const R gp = (gm1 + R(1)) / gm1;
  const R gam = R(gamma);
#if EXO_MIXED
  const R grv = R(grav);
#endif
  // the reference's Dt = 1/dt, the same value every time
  const R rdt = R(1. / dt);
  auto cell = [&](const double* w) {
    ColCell c;
    c.rho = R(w[IDN]);
    c.v1 = R(w[IVX]);
    c.v2 = R(w[IVY] + w[IVZ] * cos_theta);
    c.v3 = R(w[IVZ] * sin_theta);
    c.p = R(w[IPR]);
    c.s2 = c.v1 * c.v1 + c.v2 * c.v2 + c.v3 * c.v3;
#if EXO_MIXED
    if constexpr (sizeof(R) == 4) {
      c.isq = rsqrt_r(c.rho);
      c.sq = c.rho * c.isq;
      c.hr = gp * c.p * (c.isq * c.isq);
    } else {
      c.hr = gp * c.p * inv_r(c.rho);
    }
#else
    c.hr = gp * c.p / c.rho;
#endif
    return c;
  };
  auto AMs = [&](int slot, int r, int q) -> R& { return sa[(slot * 25 + r * 5 + q) * ss]; };

  // prefetch slots: w(i+1) and du(i) of the next level, copied asynchronously
  auto pw = [&](int n) -> double& { return sp[n * ss]; };
  auto pdu = [&](int n) -> double& { return sp[(5 + n) * ss]; };
  auto prefetch = [&](int iw, int idu) {
#pragma unroll
    for (int n = 0; n < 5; ++n) cp_async8(&pw(n), io.wptr(iw, n));
    if (idu >= 0) {
#pragma unroll
      for (int n = 0; n < 5; ++n) cp_async8(&pdu(n), io.duptr(idu, n));
    }
    cp_async_commit();
  };
  double raw[5];
  io.w(is - 1, raw);
  ColCell cm = cell(raw);
  io.w(is, raw);
  ColCell c0 = cell(raw);
  prefetch(is + 1, is);
  {
    R A[5][5];
    abs_jacobian(cm, c0, gm1, gam, A);
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) AMs(0, r, q) = A[r][q];
  }
  // (A c)_{i-1} lives in registers, or in this thread's shared memory when
  // EXO_IMPL_AP_SMEM (fewer registers, more resident warps)
#if EXO_IMPL_AP_SMEM
  static_assert(sizeof(R) == 8, "(A c)_{i-1} in shared memory takes the FP64 slice layout");
  double* const aps = sa + 60;
#define EXO_AP(r, q) aps[(r) * 5 + (q)]
#else
  R Ap[5][5];
#define EXO_AP(r, q) Ap[r][q]
#endif
  R dp[5];  // delta_{i-1}
  int cur = 0;
  for (int i = is; i <= ie; ++i) {
    cp_async_wait_all();
    double rhs[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      raw[n] = pw(n);
      rhs[n] = pdu(n);
    }
    ColCell cp = cell(raw);
    prefetch(i + 2, i < ie ? i + 1 : -1);
    const int nxt = cur ^ 1;
    {
      R A[5][5];
      abs_jacobian(c0, cp, gm1, gam, A);
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) AMs(nxt, r, q) = A[r][q];
    }
    const double aleft = d2 * d3 * x1f[i] * x1f[i] * s;
    const double aright = d2 * d3 * x1f[i + 1] * x1f[i + 1] * s;
    const double vol = dx1f[i] * d2 * d3 * x1v[i] * x1v[i] * s;
#if EXO_MIXED
    const double i2v = 0.5 / vol;
    const R bl = R(aleft * i2v), cr = R(aright * i2v), dd = R((aright - aleft) * i2v);
#endif
    const bool first = (i == is), last = (i == ie);
    R x[5];
    // rows of a, b (and c at the top boundary), then of t = a - b (A c)_{i-1},
    // written over row r of |A|(i-1/2) once that row has been read; and x
    unroll<5>([&](auto Row) {
      constexpr int r = decltype(Row)::value;
      R brow[5], trow[5];
      unroll<5>([&](auto Q) {
        constexpr int q = decltype(Q)::value;
        const R am = AMs(cur, r, q), ap = AMs(nxt, r, q);
#if EXO_MIXED
        R a = am * bl + ap * cr;
        if constexpr (fj_nz(r, q)) a += dd * fj_entry<r, q>(c0, gm1);
        if constexpr (r == q) a += rdt;
        if constexpr ((r == IVX && q == IDN) || (r == IEN && q == IVX)) a -= grv;
        R bm = am;
        if constexpr (fj_nz(r, q)) bm += fj_entry<r, q>(cm, gm1);
        R b = -bm * bl;
        if (first) a += (q == IVX) ? -b : b;
        if (last) {
          R cmv = ap;
          if constexpr (fj_nz(r, q)) cmv -= fj_entry<r, q>(cp, gm1);
          R c = -cmv * cr;
          a += (q == IVX) ? -c : c;
        }
#else
        double num = am * aleft + ap * aright;
        if constexpr (fj_nz(r, q)) num = num + (aright - aleft) * fj_entry<r, q>(c0, gm1);
        double a = num / (2. * vol);
        if constexpr (r == q) a = a + rdt;
        if constexpr ((r == IVX && q == IDN) || (r == IEN && q == IVX)) a = a - grav;
        double bm = am;
        if constexpr (fj_nz(r, q)) bm = am + fj_entry<r, q>(cm, gm1);
        double b = -bm * aleft / (2. * vol);
        if (first) a = a + ((q == IVX) ? -b : b);
        if (last) {
          double cmv = ap;
          if constexpr (fj_nz(r, q)) cmv = ap - fj_entry<r, q>(cp, gm1);
          double c = -cmv * aright / (2. * vol);
          a = a + ((q == IVX) ? -c : c);
        }
#endif
        brow[q] = b;
        trow[q] = a;
      });
#if EXO_MIXED
      x[r] = R(rhs[r]) * rdt;
#else
      x[r] = rhs[r] / dt;
#endif
      if (!first) {
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          R ba = brow[0] * EXO_AP(0, q);
#pragma unroll
          for (int k = 1; k < 5; ++k) ba += brow[k] * EXO_AP(k, q);
          trow[q] = trow[q] - ba;
        }
        R bd = brow[0] * dp[0];
#pragma unroll
        for (int k = 1; k < 5; ++k) bd += brow[k] * dp[k];
        x[r] = x[r] - bd;
      }
#pragma unroll
      for (int q = 0; q < 5; ++q) AMs(cur, r, q) = trow[q];
    });
    R t[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) t[r][q] = AMs(cur, r, q);
    // c_i column by column, from |A|(i+1/2) in shared memory and the upper cell
    auto ccol = [&](auto Q, R* c) {
      constexpr int q = decltype(Q)::value;
      unroll<5>([&](auto Row) {
        constexpr int r = decltype(Row)::value;
        R cmv = AMs(nxt, r, q);
#if EXO_MIXED
        if constexpr (fj_nz(r, q)) cmv -= fj_entry<r, q>(cp, gm1);
        c[r] = -cmv * cr;
#else
        if constexpr (fj_nz(r, q)) cmv = cmv - fj_entry<r, q>(cp, gm1);
        c[r] = -cmv * aright / (2. * vol);
#endif
      });
    };
#if EXO_MIXED
    // LU with the rows taken in the order 1, 4, 2, 3, 0 -- the order partial
    // pivoting ends with for nearly every block of this solve (density last,
    // energy and x1 momentum first) -- and threshold partial pivoting on top:
    // a row swap only where the diagonal falls below a tenth of the largest
    // entry of its column, so the swap code is skipped almost always.
    constexpr int O[5] = {1, 4, 2, 3, 0};
    unsigned perm = 0;  // 3 bits per step: the position swapped in
    bool swapped = false;
    R idg[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      if (k < 4) {
        const R dk = abs_r(t[O[k]][k]);
        R best = dk;
        int piv = k;
#pragma unroll
        for (int r = k + 1; r < 5; ++r) {
          const R m = abs_r(t[O[r]][k]);
          if (m > best) { best = m; piv = r; }
        }
        if (dk < R(0.1) * best) {
          swapped = true;
          perm |= (unsigned)piv << (3 * k);
#pragma unroll
          for (int r = k + 1; r < 5; ++r) {
            const bool sw = (piv == r);
#pragma unroll
            for (int q = 0; q < 5; ++q) {
              const R a = t[O[k]][q], b = t[O[r]][q];
              t[O[k]][q] = sw ? b : a;
              t[O[r]][q] = sw ? a : b;
            }
          }
        } else {
          perm |= (unsigned)k << (3 * k);
        }
      }
      idg[k] = inv_r(t[O[k]][k]);
#pragma unroll
      for (int r = k + 1; r < 5; ++r) {
        const R l = t[O[r]][k] * idg[k];
        t[O[r]][k] = l;
#pragma unroll
        for (int q = k + 1; q < 5; ++q) t[O[r]][q] -= l * t[O[k]][q];
      }
    }
    auto solve = [&](R* y) { lu_solve_rows(t, idg, perm, swapped, y); };
    solve(x);
    unroll<5>([&](auto Q) {
      constexpr int q = decltype(Q)::value;
      R c[5];
      ccol(Q, c);
      solve(c);
#pragma unroll
      for (int r = 0; r < 5; ++r) EXO_AP(r, q) = c[r];
    });
#pragma unroll
    for (int r = 0; r < 5; ++r) dp[r] = x[r];
#else
    // Gauss-Jordan with partial pivoting on [t | I]; columns of t left of the
    // pivot are never read again and are not updated
    double B[5][5];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) B[r][q] = (r == q) ? 1. : 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      int piv = k;
      double best = fabs(t[k][k]);
#pragma unroll
      for (int r = k + 1; r < 5; ++r)
        if (fabs(t[r][k]) > best) { best = fabs(t[r][k]); piv = r; }
#pragma unroll
      for (int r = k + 1; r < 5; ++r) {
        bool sw = (piv == r);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          if (q >= k) {
            double a = t[k][q], b = t[r][q];
            t[k][q] = sw ? b : a;
            t[r][q] = sw ? a : b;
          }
          double a = B[k][q], b = B[r][q];
          B[k][q] = sw ? b : a;
          B[r][q] = sw ? a : b;
        }
      }
      double d = 1.0 / t[k][k];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        if (q > k) t[k][q] *= d;
        B[k][q] *= d;
      }
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        if (r == k) continue;
        double f = t[r][k];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          if (q > k) t[r][q] -= f * t[k][q];
          B[r][q] -= f * B[k][q];
        }
      }
    }
    // delta_i = B x, (A c)_i = B c_i
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double acc = B[r][0] * x[0];
#pragma unroll
      for (int k = 1; k < 5; ++k) acc += B[r][k] * x[k];
      dp[r] = acc;
    }
    unroll<5>([&](auto Q) {
      constexpr int q = decltype(Q)::value;
      double c[5];
      ccol(Q, c);
#pragma unroll
      for (int r = 0; r < 5; ++r) {
        double acc = B[r][0] * c[0];
#pragma unroll
        for (int k = 1; k < 5; ++k) acc += B[r][k] * c[k];
        EXO_AP(r, q) = acc;
      }
    });
#endif
    const int lev = i - is;
    if (!last) {
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int q = 0; q < 5; ++q) io.scr(lev, r * 5 + q) = EXO_AP(r, q);
#pragma unroll
      for (int r = 0; r < 5; ++r) io.scr(lev, 25 + r) = dp[r];
    }
    if constexpr (!kBwd) {
      if (last) {
#pragma unroll
        for (int r = 0; r < 5; ++r) io.scr(lev, 25 + r) = dp[r];
      }
    }
    cm = c0;
    c0 = cp;
    cur = nxt;
  }
  // the last level's prefetch (unused) must land before the back substitution
  // reuses this thread's slots of shared memory
  cp_async_wait_all();
  if constexpr (!kBwd) return;
  if constexpr (IO::kLoadsU && sizeof(R) == 8) {
    if (io.stage >= 0) {
      // the warp's tiles (FP64 blocks: its 32 shared slices, free once every
      // lane has finished its forward sweep)
      implicit_backward_tiled<5>(io, is, ie, dp, wt);
      return;
    }
  }
  implicit_backward_full(io, is, ie, dp);
}
#undef EXO_AP

// ImplicitSolver::PartialCorrection (partial_correction.cpp:26-173) of one
// radial column, one thread per column: the 3x3 block-tridiagonal system of
// (rho, m1, E) -- the rows and columns IDN, IVX, IEN of FullCorrection's
// matrices, the same face and cell Jacobians -- solved by ForwardSweep /
// BackwardSubstitution with 3-row blocks (forward_backward.hpp:15-126).  The
// tangential momenta keep their explicit update; the reference's flux
// correction corr is zero (its computation is commented out there).  Each
// 3x3 block is inverted as its adjugate over its determinant, the closed form
// a fixed-size 3x3 inverse takes.  Scratch per level: (A c)_i (9) and
// delta_i (3).  IO and arguments as for implicit_column; the shared slices
// hold the two face blocks (18 entries of sa) and the prefetched w (5) and
// du (3) of a level (sp).
// BackwardSubstitution of the partial correction: delta_i -= (A c)_i
// delta_{i+1} for (rho, m1, E) from level ie (delta_ie in dp) down to is;
// the update of level i takes delta for rho, m1, E and the explicit du for
// m2, m3.
template <class IO>
__device__ __forceinline__ void implicit_backward_partial(IO& io, int is, int ie,
                                                          typename IO::Real* dp) {
  using R = typename IO::Real;
  auto store = [&](int i, const double* u) {
    double dl[5];
    dl[IDN] = dp[0];
    dl[IVX] = dp[1];
    dl[IVY] = *io.duptr(i, IVY);
    dl[IVZ] = *io.duptr(i, IVZ);
    dl[IEN] = dp[2];
    io.ustore(i, u, dl);
  };
  {
    double u_ie[5];
    io.uload(ie, u_ie);
    store(ie, u_ie);
  }
#pragma unroll 1
  for (int i = ie - 1; i >= is; --i) {
    R cs[12];
    double u[5];
#pragma unroll
    for (int e = 0; e < 12; ++e) cs[e] = io.scr(i - is, e);
    io.uload(i, u);
    R dl[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      R ad = cs[r * 3] * dp[0];
#pragma unroll
      for (int k = 1; k < 3; ++k) ad += cs[r * 3 + k] * dp[k];
      dl[r] = cs[9 + r] - ad;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) dp[r] = dl[r];
    store(i, u);
  }
}

// kBwd false: the forward sweep only, with delta_ie stored as scratch
// entries 9..11 of the last level (implicit_backward_partial finishes it).
template <class IO, bool kBwd = true>
__device__ __forceinline__ void implicit_column_partial(IO& io, typename IO::Real* sa, double* sp, int ss,
                                                        double cos_theta, double sin_theta,
                                                        double d2, double d3, const double* x1f,
                                                        const double* x1v, const double* dx1f,
                                                        int is, int ie, double dt, double gamma,
                                                        double grav, double* wt = nullptr) {
  using R = typename IO::Real;
  using ColCell = exo::EXO_KNS::ColCell<R>;
  constexpr int P[3] = {IDN, IVX, IEN};
  const double s = sin_theta;
  const R gm1 = R((gamma - 1.) * 1. / 1.);
  const R gp = (gm1 + R(1)) / gm1;
  const R gam = R(gamma);
#if EXO_MIXED
  const R grv = R(grav);
#endif
  const R rdt = R(1. / dt);
  auto cell = [&](const double* w) {
    ColCell c;
    c.rho = R(w[IDN]);
    c.v1 = R(w[IVX]);
    c.v2 = R(w[IVY] + w[IVZ] * cos_theta);
    c.v3 = R(w[IVZ] * sin_theta);
    c.p = R(w[IPR]);
    c.s2 = c.v1 * c.v1 + c.v2 * c.v2 + c.v3 * c.v3;
#if EXO_MIXED
    if constexpr (sizeof(R) == 4) {
      c.isq = rsqrt_r(c.rho);
      c.sq = c.rho * c.isq;
      c.hr = gp * c.p * (c.isq * c.isq);
    } else {
      c.hr = gp * c.p * inv_r(c.rho);
    }
#else
    c.hr = gp * c.p / c.rho;
#endif
    return c;
  };
  auto AMs = [&](int slot, int r, int q) -> R& { return sa[(slot * 9 + r * 3 + q) * ss]; };
  auto face = [&](const ColCell& lo, const ColCell& hi, int slot) {
    R A[5][5];
    abs_jacobian(lo, hi, gm1, gam, A);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q) AMs(slot, r, q) = A[P[r]][P[q]];
  };
  auto pw = [&](int n) -> double& { return sp[n * ss]; };
  auto pdu = [&](int m) -> double& { return sp[(5 + m) * ss]; };
  auto prefetch = [&](int iw, int idu) {
#pragma unroll
    for (int n = 0; n < 5; ++n) cp_async8(&pw(n), io.wptr(iw, n));
    if (idu >= 0) {
#pragma unroll
      for (int m = 0; m < 3; ++m) cp_async8(&pdu(m), io.duptr(idu, P[m]));
    }
    cp_async_commit();
  };
  double raw[5];
  io.w(is - 1, raw);
  ColCell cm = cell(raw);
  io.w(is, raw);
  ColCell c0 = cell(raw);
  prefetch(is + 1, is);
  face(cm, c0, 0);
  R Ap[3][3];  // (A c)_{i-1}
  R dp[3];     // delta_{i-1}
  int cur = 0;
  for (int i = is; i <= ie; ++i) {
    cp_async_wait_all();
    double rhs[3];
#pragma unroll
    for (int n = 0; n < 5; ++n) raw[n] = pw(n);
#pragma unroll
    for (int m = 0; m < 3; ++m) rhs[m] = pdu(m);
    ColCell cp = cell(raw);
    prefetch(i + 2, i < ie ? i + 1 : -1);
    const int nxt = cur ^ 1;
    face(c0, cp, nxt);
    const double aleft = d2 * d3 * x1f[i] * x1f[i] * s;
    const double aright = d2 * d3 * x1f[i + 1] * x1f[i + 1] * s;
    const double vol = dx1f[i] * d2 * d3 * x1v[i] * x1v[i] * s;
#if EXO_MIXED
    const double i2v = 0.5 / vol;
    const R bl = R(aleft * i2v), cr = R(aright * i2v), dd = R((aright - aleft) * i2v);
#endif
    const bool first = (i == is), last = (i == ie);
    R t[3][3], cc[3][3], x[3];
    unroll<3>([&](auto Row) {
      constexpr int r = decltype(Row)::value;
      constexpr int pr = P[r];
      R brow[3];
      unroll<3>([&](auto Q) {
        constexpr int q = decltype(Q)::value;
        constexpr int pq = P[q];
        const R am = AMs(cur, r, q), ap = AMs(nxt, r, q);
        // Phi << 0,0,0, grav,0,0, 0,grav,0 and Bnd = diag(1,-1,1)
        constexpr bool phi = (r == 1 && q == 0) || (r == 2 && q == 1);
#if EXO_MIXED
        R a = am * bl + ap * cr;
        if constexpr (fj_nz(pr, pq)) a += dd * fj_entry<pr, pq>(c0, gm1);
        if constexpr (r == q) a += rdt;
        if constexpr (phi) a -= grv;
        R bm = am;
        if constexpr (fj_nz(pr, pq)) bm += fj_entry<pr, pq>(cm, gm1);
        R b = -bm * bl;
        R cmv = ap;
        if constexpr (fj_nz(pr, pq)) cmv -= fj_entry<pr, pq>(cp, gm1);
        R c = -cmv * cr;
        if (first) a += (q == 1) ? -b : b;
        if (last) a += (q == 1) ? -c : c;
#else
        double num = am * aleft + ap * aright;
        if constexpr (fj_nz(pr, pq)) num = num + (aright - aleft) * fj_entry<pr, pq>(c0, gm1);
        double a = num / (2. * vol);
        if constexpr (r == q) a = a + rdt;
        if constexpr (phi) a = a - grav;
        double bm = am;
        if constexpr (fj_nz(pr, pq)) bm = am + fj_entry<pr, pq>(cm, gm1);
        double b = -bm * aleft / (2. * vol);
        double cmv = ap;
        if constexpr (fj_nz(pr, pq)) cmv = ap - fj_entry<pr, pq>(cp, gm1);
        double c = -cmv * aright / (2. * vol);
        if (first) a = a + ((q == 1) ? -b : b);
        if (last) a = a + ((q == 1) ? -c : c);
#endif
        brow[q] = b;
        t[r][q] = a;
        cc[r][q] = c;
      });
#if EXO_MIXED
      x[r] = R(rhs[r]) * rdt;
#else
      x[r] = rhs[r] / dt;
#endif
      if (!first) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          R ba = brow[0] * Ap[0][q];
#pragma unroll
          for (int k = 1; k < 3; ++k) ba += brow[k] * Ap[k][q];
          t[r][q] = t[r][q] - ba;
        }
        R bd = brow[0] * dp[0];
#pragma unroll
        for (int k = 1; k < 3; ++k) bd += brow[k] * dp[k];
        x[r] = x[r] - bd;
      }
    });
    // B = t^-1 = adj(t) / det(t): cofactor (i,j) from the cyclic neighbours
    // of row i and column j (which carries its sign), det along column 0
    auto cof = [&](int i0, int j0) {
      const int i1 = (i0 + 1) % 3, i2 = (i0 + 2) % 3, j1 = (j0 + 1) % 3, j2 = (j0 + 2) % 3;
      return t[i1][j1] * t[i2][j2] - t[i1][j2] * t[i2][j1];
    };
    R B[3][3];
    {
      const R c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
      const R det = c00 * t[0][0] + c10 * t[1][0] + c20 * t[2][0];
      const R id = R(1) / det;
      B[0][0] = c00 * id;
      B[0][1] = c10 * id;
      B[0][2] = c20 * id;
#pragma unroll
      for (int r = 1; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) B[r][q] = cof(q, r) * id;
    }
    // delta_i = B x, (A c)_i = B c_i
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      R acc = B[r][0] * x[0];
#pragma unroll
      for (int k = 1; k < 3; ++k) acc += B[r][k] * x[k];
      dp[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        R acc = B[r][0] * cc[0][q];
#pragma unroll
        for (int k = 1; k < 3; ++k) acc += B[r][k] * cc[k][q];
        Ap[r][q] = acc;
      }
    if (!last) {
      const int lev = i - is;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) io.scr(lev, r * 3 + q) = Ap[r][q];
#pragma unroll
      for (int r = 0; r < 3; ++r) io.scr(lev, 9 + r) = dp[r];
    }
    if constexpr (!kBwd) {
      if (last) {
#pragma unroll
        for (int r = 0; r < 3; ++r) io.scr(i - is, 9 + r) = dp[r];
      }
    }
    cm = c0;
    c0 = cp;
    cur = nxt;
  }
  cp_async_wait_all();  // the last level's prefetch (unused) lands before the slice is reused
  if constexpr (!kBwd) return;
  if constexpr (IO::kLoadsU && sizeof(R) == 8) {
    if (io.stage >= 0) {
      implicit_backward_tiled<3>(io, is, ie, dp, wt);
      return;
    }
  }
  implicit_backward_partial(io, is, ie, dp);
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

// Launch shape of the implicit kernels: one thread per radial column, 64
// columns per block, 60 doubles of shared memory per thread (the face
// Jacobians |A|(i-1/2) and |A|(i+1/2), the next level's w and du).
constexpr int IMPL_THREADS = 64;      // default; 32 and 128 are the other tiles
constexpr int IMPL_MAX_THREADS = 128;
#ifndef EXO_IMPL_MINB
#define EXO_IMPL_MINB 2  // resident 128-thread blocks per SM the register budget is sized for
#endif
// the mixed build's solve is capped at 204 registers (8 bytes of spill),
// measured 18 % faster at 6x192^2x96 than uncapped; with the per-warp
// register rounding that still leaves 4 blocks of 64 columns per SM (8 warps).
// 200 registers fit a fifth block but measured 1-3 % slower, so the forward
// sweep is bound by its FP64 dependency chains, not by resident warps.  The
// FP64 build spills below 254 registers and keeps the full register file.
#if !defined(EXO_IMPL_MAXNREG) && EXO_MIXED
#define EXO_IMPL_MAXNREG 204
#endif
#ifdef EXO_IMPL_MAXNREG
#define EXO_IMPL_BOUNDS __maxnreg__(EXO_IMPL_MAXNREG)
#else
#define EXO_IMPL_BOUNDS __launch_bounds__(IMPL_MAX_THREADS, EXO_IMPL_MINB)
#endif
// FP64 solve: each thread's doubles are contiguous (60, or 85 with
// (A c)_{i-1} kept there), threads IMPL_SM_STRIDE doubles apart (defined
// with the back substitution): an odd stride keeps a half-warp's 8-byte
// accesses on distinct banks.
// FP32 solve: structure of arrays, the 10 prefetch doubles of every thread
// first, then the 50 FP32 face-block entries, entry e of thread t at
// [e * threads + t], so a warp's accesses are consecutive words.
template <class R>
__host__ __device__ constexpr int impl_slice_doubles() {
  return sizeof(R) == 4 ? 10 + 50 / 2 : IMPL_SM_STRIDE;
}
// per block: the threads' slices, then x1f (nc1+1), x1v (nc1), dx1f (nc1)
template <class R>
__host__ __device__ constexpr size_t impl_smem(int threads, int nc1) {
  return ((size_t)impl_slice_doubles<R>() * threads + 3 * (size_t)(nc1 + 1)) * sizeof(double);
}
// this thread's slices of the block's shared memory (arguments sa, sp, ss of
// implicit_column and implicit_column_partial)
template <class R>
struct ImplSlices {
  R* sa;
  double* sp;
  int ss;
  double* wt;  // FP64 blocks: the warp's back-substitution tiles (WARP_TILE_DOUBLES)
};
template <class R>
__device__ __forceinline__ ImplSlices<R> impl_slices(double* ism, bool full) {
  if constexpr (sizeof(R) == 4) {
    const int nt = (int)blockDim.x, t = (int)threadIdx.x;
    return {reinterpret_cast<R*>(ism + 10 * nt) + t, ism + t, nt, nullptr};
  } else {
    double* sm = ism + threadIdx.x * IMPL_SM_STRIDE;
    return {sm, sm + (full ? 50 : 18), 1, ism + (threadIdx.x & ~31u) * IMPL_SM_STRIDE};
  }
}
// where the block's copy of the radial geometry starts
template <class R>
__device__ __forceinline__ double* impl_radial(double* ism) {
  return ism + blockDim.x * impl_slice_doubles<R>();
}
// the largest dynamic shared memory a launch may ask for
constexpr int IMPL_SMEM_MAX = 160 * 1024;

// copies the radial geometry of the member into shared memory (all threads
// of the block take part; returns the shared copies)
__device__ __forceinline__ void stage_radial(double* sg, int nc1, const double* x1f,
                                             const double* x1v, const double* dx1f,
                                             const double*& sx1f, const double*& sx1v,
                                             const double*& sdx1f) {
  double* a = sg;
  double* b = sg + nc1 + 1;
  double* c = b + nc1 + 1;
  for (int t = threadIdx.x; t <= nc1; t += blockDim.x) {
    a[t] = x1f[t];
    if (t < nc1) {
      b[t] = x1v[t];
      c[t] = dx1f[t];
    }
  }
  __syncthreads();
  sx1f = a;
  sx1v = b;
  sdx1f = c;
}

// A column of the stepping context: primitives and update from the state
// arrays, the corrected update added to u (with the AirParcel round trip on
// the last stage).
template <class R>
struct StepColumnIO {
  using Real = R;
  const double* wc;
  const double* duc;
  double* uc;
  size_t vs;       // stride between variables
  R* scr0;         // scratch of this column: [level][entry][32 lanes] per warp of columns
  int stage;            // < 0: write the corrected update into du, leave u alone
  double Rd, gamma;
  double* duw;          // du of this column, for stage < 0
  __device__ __forceinline__ void w(int i, double* out) const {
#pragma unroll
    for (int n = 0; n < 5; ++n) out[n] = wc[n * vs + i];
  }
  __device__ __forceinline__ const double* wptr(int i, int n) const { return wc + n * vs + i; }
  __device__ __forceinline__ const double* duptr(int i, int n) const { return duc + n * vs + i; }
  __device__ __forceinline__ R& scr(int lev, int e) const {
    return scr0[(lev * 30 + e) * 32];
  }
  static constexpr bool kLoadsU = true;
  unsigned live = 0xffffffffu;  // the lanes of the warp with a column
  __device__ __forceinline__ void uload(int i, double* u) const {
    if (stage < 0) return;
#pragma unroll
    for (int n = 0; n < 5; ++n) u[n] = uc[n * vs + i];
  }
  __device__ __forceinline__ void ustore(int i, const double* u, const double* dl) const {
    if (stage < 0) {
#pragma unroll
      for (int n = 0; n < 5; ++n) duw[n * vs + i] = dl[n];
      return;
    }
    double uu[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) uu[n] = u[n] + 1. * dl[n];
    if (stage == 2) airparcel_round_trip(uu, Rd, gamma);
#pragma unroll
    for (int n = 0; n < 5; ++n) uc[n * vs + i] = uu[n];
  }
};

// One radial column of the stepping context: solve, then u += du and, on
// the last stage, the AirParcel round trip.
// stage 0..2: a stage of the step (dt = beta_stage * the CFL step, u += du);
// stage -1: ImplicitSolver::SolveImplicit3D alone (dt given, du corrected in
// place)
template <class R>
__device__ __forceinline__ void implicit_block(const DevView& v, unsigned blk, int stage,
                                               double dt_given = 0.) {
  extern __shared__ double ism[];
  const int ncol = 6 * v.N * v.N;
  const int col = (int)(blk * blockDim.x + threadIdx.x);
  // the radial geometry, read every level by every column, staged once per
  // block: kept out of L1, which the columns' strided loads churn each level
  const double* x1f;
  const double* x1v;
  const double* dx1f;
  stage_radial(impl_radial<R>(ism), v.nc1, v.x1f, v.x1v, v.dx1f, x1f, x1v, dx1f);
  const unsigned live = __ballot_sync(0xffffffffu, col < ncol);
  if (col >= ncol) return;
  const int j = v.js + col % v.N;
  const int k = v.ks + (col / v.N) % v.N;
  const int p = col / (v.N * v.N);
  const double dt = stage < 0 ? dt_given : rk_beta(stage) * v.sc->dt;
  const size_t base = idx(v, p, 0, k, j, 0);
  // scratch in blocks of 32 columns: a warp's 32 entries are 128 (FP32) or
  // 256 (FP64) contiguous bytes
  R* scr0 = reinterpret_cast<R*>(v.scratch) + (size_t)(col >> 5) * v.L * 30 * 32 + (col & 31);
  StepColumnIO<R> io{v.w + base, v.du + base, v.u + base, v.cells, scr0, stage, v.Rd, v.gamma,
                     v.du + base};
  io.live = live;
  const bool full = (v.implicit_flag & 8) != 0;
  const ImplSlices<R> sl = impl_slices<R>(ism, full);
  using IO = StepColumnIO<R>;
  // FP32 blocks: the back substitution of the full correction is
  // kb_implicit_bwd's (split_bwd; the lighter partial one stays here: split,
  // it measured slower)
  constexpr bool kBwd = sizeof(R) == 8;
  if (full)
    implicit_column<IO, kBwd>(io, sl.sa, sl.sp, sl.ss, geo(v, GCOSC, p, k, j),
                                         geo(v, GSINC, p, k, j), geo(v, GDX2A, p, k, j),
                                         geo(v, GDX3A, p, k, j), x1f, x1v, dx1f, v.is, v.ie,
                                         dt, v.gamma, v.grav, sl.wt);
  else
    implicit_column_partial<IO, true>(io, sl.sa, sl.sp, sl.ss,
                                                 geo(v, GCOSC, p, k, j), geo(v, GSINC, p, k, j),
                                                 geo(v, GDX2A, p, k, j), geo(v, GDX3A, p, k, j),
                                                 x1f, x1v, dx1f, v.is, v.ie, dt, v.gamma, v.grav,
                                                 sl.wt);
}

// ---------------------------------------------------- kb_implicit_bwd ---
// The back substitution of the full correction, delta_i -= (A c)_i
// delta_{i+1} from the top level down, u += delta (with the AirParcel round
// trip on the last stage), as a kernel of its own after the forward sweep
// (kb_implicit, which leaves (A c)_i and delta_i of every level in scratch),
// for FP32 blocks.  It streams 120 bytes of scratch and 80 bytes of u per
// cell and computes little, so it is built to keep HBM busy: one
// warp per group of 32 columns, whose scratch is one contiguous run per
// chunk of BWD_LEV levels ([group][level][entry][32]); the chunk below the
// one being finished is already on its way into the other shared-memory
// buffer, by one bulk TMA copy (cp.async.bulk, completion counted by an
// mbarrier) for the factors and by 8-byte cp.async copies for u (four lanes
// read one column's four levels: a 32-byte run per column and variable).
// u is updated in the shared tile and written back the same way.
constexpr int BWD_LEV = 4;  // levels per chunk
// the shared memory of one warp: two buffers, each the factor chunk and the
// u tile [5][32][BWD_LEV + 1] (padded: a warp's column-wise accesses of one
// level fall on distinct banks), then the two mbarriers
template <class R>
__host__ __device__ constexpr size_t bwd_chunk_bytes() {
  return (size_t)BWD_LEV * 30 * 32 * sizeof(R);
}
constexpr int BWD_TILE_DOUBLES = 5 * 32 * (BWD_LEV + 1);
template <class R>
__host__ __device__ constexpr size_t bwd_buffer_bytes() {
  return bwd_chunk_bytes<R>() + BWD_TILE_DOUBLES * sizeof(double);
}
template <class R>
__host__ __device__ constexpr size_t impl_bwd_smem() {
  return 2 * bwd_buffer_bytes<R>() + 16;
}
static_assert(bwd_chunk_bytes<float>() % 16 == 0 && bwd_buffer_bytes<float>() % 16 == 0,
              "bulk copies move multiples of 16 bytes to 16-byte aligned addresses");
static_assert(bwd_chunk_bytes<double>() % 16 == 0 && bwd_buffer_bytes<double>() % 16 == 0,
              "bulk copies move multiples of 16 bytes to 16-byte aligned addresses");

template <class R>
__device__ __forceinline__ void implicit_bwd_warp(const DevView& v, int group, int stage) {
  extern __shared__ __align__(128) unsigned char bws[];
  const int lane = (int)(threadIdx.x & 31);
  const int ncol = 6 * v.N * v.N;
  const int col0 = group * 32, col = col0 + lane;
  const bool active = col < ncol;
  const int ncb = min(32, ncol - col0);
  const int L = v.L;
  const size_t vs = v.cells;
  size_t base = 0;
  if (active) {
    const int j = v.js + col % v.N;
    const int k = v.ks + (col / v.N) % v.N;
    const int p = col / (v.N * v.N);
    base = idx(v, p, 0, k, j, 0);
  }
  // this column's scratch: entry e of level lev at sg[(lev * 30 + e) * 32 + lane]
  const R* sg = reinterpret_cast<const R*>(v.scratch) + (size_t)group * L * 30 * 32;
  unsigned long long* mb = reinterpret_cast<unsigned long long*>(bws + 2 * bwd_buffer_bytes<R>());
  auto chunk_scr = [&](int b) { return reinterpret_cast<R*>(bws + b * bwd_buffer_bytes<R>()); };
  auto chunk_tile = [&](int b) {
    return reinterpret_cast<double*>(bws + b * bwd_buffer_bytes<R>() + bwd_chunk_bytes<R>());
  };
  if (lane == 0) {
    mbar_init(&mb[0], 1);
    mbar_init(&mb[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncwarp();
  // the column bases of the group, for the tile copies
  const long long cb_lane = active ? (long long)base : 0;
  const int nch = (L + BWD_LEV - 1) / BWD_LEV;
  double* const u = v.u;
  // chunk c holds levels [c * BWD_LEV, min(L, (c + 1) * BWD_LEV)) (level
  // index i - is); a tile element e is (variable n, column c, level l)
  auto issue = [&](int c, int b) {
    const int lo = c * BWD_LEV, nl = min(L, lo + BWD_LEV) - lo;
    if (lane == 0) {
      const unsigned bytes = (unsigned)(nl * 30 * 32 * sizeof(R));
      mbar_expect_tx(&mb[b], bytes);
      bulk_g2s(chunk_scr(b), sg + (size_t)lo * 30 * 32, bytes, &mb[b]);
    }
    double* tile = chunk_tile(b);
    for (int e = lane; e < 5 * 32 * BWD_LEV; e += 32) {
      const int l = e & (BWD_LEV - 1), cc = (e / BWD_LEV) & 31, n = e / (BWD_LEV * 32);
      const long long cbase = __shfl_sync(0xffffffffu, cb_lane, cc);
      if (cc < ncb && l < nl)
        cp_async8(&tile[(n * 32 + cc) * (BWD_LEV + 1) + l], u + cbase + n * vs + v.is + lo + l);
    }
    cp_async_commit();
  };
  unsigned phases = 0u;   // bit b: the phase buffer b's mbarrier completes next
  unsigned pending = 0u;  // bit b: buffer b's bulk copy is still outstanding
  bool ok = true;
  R dp[5] = {R(0), R(0), R(0), R(0), R(0)};
  issue(nch - 1, 0);
  pending |= 1u;
  int b = 0;
  for (int c = nch - 1; c >= 0; --c) {
    if (c > 0) {
      issue(c - 1, b ^ 1);
      pending |= 1u << (b ^ 1);
    }
    // the factors of chunk c (bounded wait; the whole warp agrees) and its u tile
    const bool got = mbar_wait(&mb[b], (phases >> b) & 1u);
    if (!__all_sync(0xffffffffu, got)) {
      ok = false;
      break;
    }
    phases ^= 1u << b;
    pending &= ~(1u << b);
    if (c > 0) cp_async_wait_one();
    else cp_async_wait_all();
    __syncwarp();
    const R* cs = chunk_scr(b);
    double* tile = chunk_tile(b);
    const int lo = c * BWD_LEV, nl = min(L, lo + BWD_LEV) - lo;
    if (active) {
      for (int l = nl - 1; l >= 0; --l) {
        const int lev = lo + l;
        const R* f = cs + (size_t)l * 30 * 32 + lane;
        if (lev == L - 1) {
#pragma unroll
          for (int r = 0; r < 5; ++r) dp[r] = f[(25 + r) * 32];  // delta_ie
        } else {
          R dl[5];
#pragma unroll
          for (int r = 0; r < 5; ++r) {
            R ad = f[(r * 5) * 32] * dp[0];
#pragma unroll
            for (int k = 1; k < 5; ++k) ad += f[(r * 5 + k) * 32] * dp[k];
            dl[r] = f[(25 + r) * 32] - ad;
          }
#pragma unroll
          for (int r = 0; r < 5; ++r) dp[r] = dl[r];
        }
        // StepColumnIO::ustore with u in the tile
        double uu[5];
#pragma unroll
        for (int n = 0; n < 5; ++n)
          uu[n] = tile[(n * 32 + lane) * (BWD_LEV + 1) + l] + 1. * (double)dp[n];
        if (stage == 2) airparcel_round_trip(uu, v.Rd, v.gamma);
#pragma unroll
        for (int n = 0; n < 5; ++n) tile[(n * 32 + lane) * (BWD_LEV + 1) + l] = uu[n];
      }
    }
    __syncwarp();
    for (int e = lane; e < 5 * 32 * BWD_LEV; e += 32) {
      const int l = e & (BWD_LEV - 1), cc = (e / BWD_LEV) & 31, n = e / (BWD_LEV * 32);
      const long long cbase = __shfl_sync(0xffffffffu, cb_lane, cc);
      if (cc < ncb && l < nl)
        u[cbase + n * vs + v.is + lo + l] = tile[(n * 32 + cc) * (BWD_LEV + 1) + l];
    }
    __syncwarp();
    b ^= 1;
  }
  if (!ok) {
    // a bulk copy did not complete in time: record it, and give every copy
    // still outstanding a bounded wait before this warp's shared memory is
    // released (the columns keep the forward sweep's state)
    if (lane == 0) atomicOr(&v.sc->timeout, 1);
    for (int bb = 0; bb < 2; ++bb)
      if ((pending >> bb) & 1u) mbar_wait(&mb[bb], (phases >> bb) & 1u);
    cp_async_wait_all();
  }
}

// SolveImplicit3D alone (stage < 0): du corrected in place, column by column
template <class R>
__device__ __forceinline__ void implicit_bwd_du(const DevView& v, int col) {
  if (col >= 6 * v.N * v.N) return;
  const int j = v.js + col % v.N;
  const int k = v.ks + (col / v.N) % v.N;
  const int p = col / (v.N * v.N);
  const size_t base = idx(v, p, 0, k, j, 0);
  R* scr0 = reinterpret_cast<R*>(v.scratch) + (size_t)(col >> 5) * v.L * 30 * 32 + (col & 31);
  StepColumnIO<R> io{v.w + base, v.du + base, v.u + base, v.cells, scr0, -1, v.Rd, v.gamma,
                     v.du + base};
  R dp[5];
#pragma unroll
  for (int r = 0; r < 5; ++r) dp[r] = io.scr(v.L - 1, 25 + r);
  implicit_backward_full<StepColumnIO<R>, false>(io, v.is, v.ie, dp);
}

// last-stage round trip when the implicit solver is off
__device__ __forceinline__ void roundtrip_block(const DevView& v, unsigned blk) {
  unsigned tid = blk * blockDim.x + threadIdx.x;
  unsigned L = v.L, N = v.N;
  if (tid >= 6u * N * N * L) return;
  const unsigned r1 = v.div_L(tid), r2 = v.div_N(r1), r3 = v.div_N(r2);
  int i = v.is + (int)(tid - r1 * L);
  int j = v.js + (int)(r1 - r2 * N);
  int k = v.ks + (int)(r2 - r3 * N);
  int p = (int)r3;
  double uu[5];
  for (int n = 0; n < 5; ++n) uu[n] = v.u[idx(v, p, n, k, j, i)];
  airparcel_round_trip(uu, v.Rd, v.gamma);
  for (int n = 0; n < 5; ++n) v.u[idx(v, p, n, k, j, i)] = uu[n];
}

__device__ __forceinline__ void p2c_block(const DevView& v, unsigned blk, const double* wsrc) {
  unsigned tid = blk * blockDim.x + threadIdx.x;
  unsigned L = v.L, N = v.N;
  if (tid >= 6u * N * N * L) return;
  const unsigned r1 = v.div_L(tid), r2 = v.div_N(r1), r3 = v.div_N(r2);
  int i = v.is + (int)(tid - r1 * L);
  int j = v.js + (int)(r1 - r2 * N);
  int k = v.ks + (int)(r2 - r3 * N);
  int p = (int)r3;
  double w[5], c[5];
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    w[n] = wsrc[idx(v, p, n, k, j, i)];
  }
  prim_to_cons(v, w, c, geo(v, GCOSC, p, k, j));
  #pragma unroll
  for (int n = 0; n < 5; ++n) {
    if (n >= v.nv) break;
    v.u[idx(v, p, n, k, j, i)] = c[n];
  }
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

// ------------------------------------------------------------ wrappers ----
// Each kernel body above works on one atmosphere and one block index of it.
// The single-atmosphere kernels take the DevView by value; the batched ones
// take a table of DevViews and, per launch, the first block of every member
// (start[m], start[n] = total): block b belongs to the member m with
// start[m] <= b < start[m+1] and works on its block b - start[m].  One
// batched launch per kernel advances every member of an ensemble.
struct Batch {
  const DevView* views;
  const unsigned* start;
  int n;
};

__device__ __forceinline__ int batch_member(const Batch& bt, unsigned b) {
  int lo = 0, hi = bt.n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (bt.start[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// copies the member's view into shared memory, 16 bytes per thread; returns
// the block's index within the member
__device__ __forceinline__ unsigned batch_enter(const Batch& bt, DevView& sv) {
  static_assert(sizeof(DevView) % 16 == 0, "DevView is copied in 16-byte words");
  const int m = batch_member(bt, blockIdx.x);  // the same for every thread
  const int4* src = reinterpret_cast<const int4*>(bt.views + m);
  int4* dst = reinterpret_cast<int4*>(&sv);
  for (int t = threadIdx.x; t < (int)(sizeof(DevView) / 16); t += blockDim.x) dst[t] = src[t];
  const unsigned local = blockIdx.x - bt.start[m];
  __syncthreads();
  return local;
}

// 64 registers (32 warps per SM, 8 bytes of spill): 9 % faster at
// 6x192^2x96 than 48 (which spills 80 bytes), 56 and 74 (no spill)
#ifndef EXO_PRIM_MAXNREG
#define EXO_PRIM_MAXNREG 64
#endif
#ifdef EXO_PRIM_MAXNREG
#define EXO_PRIM_BOUNDS __maxnreg__(EXO_PRIM_MAXNREG)
#else
#define EXO_PRIM_BOUNDS
#endif
__global__ void EXO_PRIM_BOUNDS kb_prim_ghost(Batch bt, int compute_dt) {
  __shared__ __align__(16) DevView sv;
  unsigned b = batch_enter(bt, sv);
  prim_ghost_block(sv, b, compute_dt);
}

// The x1 kernel is latency bound (a thread per column walks the hydrostatic
// scan while the others wait): occupancy beats registers, measured
#ifndef EXO_X1_MAXNREG
#define EXO_X1_MAXNREG 48
#endif
#define EXO_X1_BOUNDS __maxnreg__(EXO_X1_MAXNREG)
template <class T>
__global__ void EXO_X1_BOUNDS kb_flux_x1(Batch bt) {
  __shared__ __align__(16) DevView sv;
  unsigned b = batch_enter(bt, sv);
  if (sv.eqn == EXO_EQN_SHALLOW_YZ) return;
  flux_x1_block<T>(sv, b);
}

// the mixed build's sliding-window kernel: 168 registers (3 blocks of 128
// threads per SM) measured 16 % faster than its natural 208 at 6x192^2x96;
// the FP64 per-face kernel needs fewer
#if !defined(EXO_X23_MAXNREG) && EXO_MIXED && !EXO_X23_TILES
#define EXO_X23_MAXNREG 168
#endif
// the pipelined line kernel of the mixed build at 128 registers (4 blocks of
// 128 threads per SM): 1.64 ms per launch at 6x192^2x96 against 1.75 at its
// natural 148 and 1.91 for one block per chunk
#if EXO_X23_TILES && EXO_MIXED && !defined(EXO_X23_MINB)
#define EXO_X23_MINB 4
#endif
#if EXO_X23_TILES && defined(EXO_X23_MINB)
#define EXO_X23_BOUNDS __launch_bounds__(X23_THREADS, EXO_X23_MINB)
#elif EXO_X23_TILES
#define EXO_X23_BOUNDS __launch_bounds__(X23_THREADS)
#elif defined(EXO_X23_MAXNREG)
#define EXO_X23_BOUNDS __maxnreg__(EXO_X23_MAXNREG)
#else
#define EXO_X23_BOUNDS
#endif
template <class T>
__global__ void EXO_X23_BOUNDS kb_flux_x23(Batch bt) {
  __shared__ __align__(16) DevView sv;
  unsigned b = batch_enter(bt, sv);
  flux_x23_block<T>(sv, b);
}

#ifdef EXO_UPD_MAXNREG
#define EXO_UPD_BOUNDS __maxnreg__(EXO_UPD_MAXNREG)
#else
#define EXO_UPD_BOUNDS
#endif
template <class T>
__global__ void EXO_UPD_BOUNDS kb_update(Batch bt, int stage) {
  __shared__ __align__(16) DevView sv;
  unsigned b = batch_enter(bt, sv);
  update_block<T>(sv, b, stage);
}

template <class R>
__global__ void EXO_IMPL_BOUNDS kb_implicit(Batch bt, int stage, double dt_given) {
  __shared__ __align__(16) DevView sv;
  unsigned b = batch_enter(bt, sv);
  if (sv.eqn == EXO_EQN_SHALLOW_YZ || !(sv.implicit_flag & 1)) return;
  implicit_block<R>(sv, b, stage, dt_given);
}

// One warp per group of 32 columns: implicit block b of a member (its
// columns b*T .. b*T+T-1 at T = the implicit tile) is T/32 blocks here.
template <class R>
__global__ void __launch_bounds__(32) kb_implicit_bwd(Batch bt, int stage, int warps_per_iblock) {
  __shared__ __align__(16) DevView sv;
  const unsigned ib = blockIdx.x / (unsigned)warps_per_iblock;
  {
    static_assert(sizeof(DevView) % 16 == 0, "DevView is copied in 16-byte words");
    const int m = batch_member(bt, ib);
    const int4* src = reinterpret_cast<const int4*>(bt.views + m);
    int4* dst = reinterpret_cast<int4*>(&sv);
    for (int t = threadIdx.x; t < (int)(sizeof(DevView) / 16); t += blockDim.x) dst[t] = src[t];
    __syncwarp();
  }
  const int m = batch_member(bt, ib);
  const unsigned local = ib - bt.start[m];
  // members with the partial correction finished in kb_implicit
  if (sv.eqn == EXO_EQN_SHALLOW_YZ || !(sv.implicit_flag & 1) || !(sv.implicit_flag & 8)) return;
  const int group = (int)(local * (unsigned)warps_per_iblock + blockIdx.x % (unsigned)warps_per_iblock);
  if (group * 32 >= 6 * sv.N * sv.N) return;
  if (stage < 0) {
    implicit_bwd_du<R>(sv, group * 32 + (int)threadIdx.x);
    return;
  }
  implicit_bwd_warp<R>(sv, group, stage);
}

__global__ void kb_roundtrip(Batch bt) {
  __shared__ __align__(16) DevView sv;
  unsigned b = batch_enter(bt, sv);
  if (sv.eqn == EXO_EQN_SHALLOW_YZ || (sv.implicit_flag & 1)) return;
  roundtrip_block(sv, b);
}

__global__ void k_p2c(DevView v, const double* wsrc) { p2c_block(v, blockIdx.x, wsrc); }

// time-step bookkeeping of every member (one thread per member)
__global__ void kb_dt_reset(const DevView* views, int n) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) views[m].sc->dtmin_bits = 0x7FEFFFFFFFFFFFFFull;
}
__global__ void kb_dt_finalize(const DevView* views, int n, int advance) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  DevScalars* sc = views[m].sc;
  if (advance) {
    sc->time += sc->dt;
    sc->ncycle += 1;
  }
  double nd = views[m].cfl * __longlong_as_double((long long)sc->dtmin_bits);
  sc->dt = advance ? fmin(2.0 * sc->dt, nd) : nd;
}

inline int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : EXO_ERR_CUDA;
}

inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

// the implicit kernel of a precision: FP32 blocks for
// EXO_PREC_MIXED_F32_SOLVE, FP64 for EXO_PREC_MIXED and the FP64 build
// the forward sweep, then (when some member has the full correction) the
// back substitution
template <class R>
inline void launch_kb_implicit(unsigned blocks, int threads, int nc1, cudaStream_t st, Batch b,
                               int stage, double dt_given, bool any_full) {
  kb_implicit<R><<<blocks, threads, impl_smem<R>(threads, nc1), st>>>(b, stage, dt_given);
  if constexpr (sizeof(R) == 4) {
    if (any_full)
      kb_implicit_bwd<R><<<blocks * (unsigned)(threads / 32), 32, impl_bwd_smem<R>(), st>>>(
          b, stage, threads / 32);
  }
}
inline void launch_kb_implicit(int precision, unsigned blocks, int threads, int nc1,
                               cudaStream_t st, Batch b, int stage, double dt_given,
                               bool any_full) {
#if EXO_MIXED
  if (precision == EXO_PREC_MIXED_F32_SOLVE) {
    launch_kb_implicit<float>(blocks, threads, nc1, st, b, stage, dt_given, any_full);
    return;
  }
#endif
  (void)precision;
  launch_kb_implicit<double>(blocks, threads, nc1, st, b, stage, dt_given, any_full);
}

}  // namespace

// The single-atmosphere launches run the batched kernels on a batch of one
// (the view's own device copy and block table), so an atmosphere advanced
// alone executes exactly the code it executes inside an ensemble.
inline Batch one(const DevView& v, int kind) { return Batch{v.self, v.starts + 2 * kind, 1}; }

// threads per block of the x2/x3 kernel: the tiled form is fixed at X23_THREADS
inline int x23_threads(int tile) { return EXO_X23_TILES ? X23_THREADS : tile; }

inline unsigned member_block_count(const DevView& v, int kind) {
  unsigned b[BK_COUNT];
  member_blocks(v, v.tiles, b);
  return b[kind];
}

// 1/x as the FP64 implicit blocks of this compilation take it (inv_r),
// element-wise
__global__ void k_reciprocal(int n, const double* x, double* out) {
  const int m = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (m < n) out[m] = inv_r(x[m]);
}
int launch_reciprocal(int n, const double* x, double* out, void* stream) {
  if (n <= 0) return 0;
  k_reciprocal<<<nblk((size_t)n, 128), 128, 0, (cudaStream_t)stream>>>(n, x, out);
  return check_launch();
}

unsigned x23_blocks(const DevView& v, int tile) {
  const bool lines = EXO_X23_TILES ? x23_uses_lines(v.L) : (bool)EXO_X23_LINES;
  if (EXO_X23_TILES && lines) return x23_tile_blocks(v.N, v.L);
  if (EXO_X23_TILES) tile = X23_THREADS;  // the per-face form of the tiled build
  const size_t n = lines ? (size_t)2 * 6 * v.N * v.L : (size_t)2 * 6 * v.N * (v.N + 1) * v.L;
  return (unsigned)((n + tile - 1) / tile);
}

int prepare_kernels() {
  cudaError_t e = cudaFuncSetAttribute(kb_implicit<double>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, IMPL_SMEM_MAX);
#if EXO_MIXED
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kb_implicit<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             IMPL_SMEM_MAX);
#endif
#if EXO_MIXED
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kb_implicit_bwd<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)impl_bwd_smem<float>());
#endif
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kb_flux_x1<EXO_FLUX_T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             X1_SMEM_MAX);
  return e == cudaSuccess ? 0 : EXO_ERR_CUDA;
}

int launch_prim_ghost(const DevView& v, bool compute_dt, void* stream) {
  kb_prim_ghost<<<member_block_count(v, BK_PRIM), v.tiles[BK_PRIM], 0, (cudaStream_t)stream>>>(
      one(v, BK_PRIM), compute_dt ? 1 : 0);
  return check_launch();
}

int launch_flux_x1(const DevView& v, void* stream) {
  if (v.eqn == EXO_EQN_SHALLOW_YZ) return 0;
  const int threads = x1_threads(v);
  size_t smem = x1_smem_bytes(v);
  kb_flux_x1<EXO_FLUX_T><<<member_block_count(v, BK_X1), threads, smem, (cudaStream_t)stream>>>(
      one(v, BK_X1));
  return check_launch();
}

int launch_flux_x23(const DevView& v, void* stream) {
  kb_flux_x23<EXO_FLUX_T><<<member_block_count(v, BK_X23), x23_threads(v.tiles[BK_X23]), 0,
                            (cudaStream_t)stream>>>(
      one(v, BK_X23));
  return check_launch();
}

int launch_update(const DevView& v, int stage, void* stream) {
  kb_update<EXO_FLUX_T><<<member_block_count(v, BK_UPDATE), v.tiles[BK_UPDATE], 0,
                          (cudaStream_t)stream>>>(
      one(v, BK_UPDATE), stage);
  int rc = check_launch();
  if (rc) return rc;
  if (v.eqn != EXO_EQN_SHALLOW_YZ && !(v.implicit_flag & 1) && stage == 2) {
    kb_roundtrip<<<member_block_count(v, BK_ROUNDTRIP), v.tiles[BK_ROUNDTRIP], 0,
                   (cudaStream_t)stream>>>(
        one(v, BK_ROUNDTRIP));
    rc = check_launch();
  }
  return rc;
}

int launch_implicit(const DevView& v, int stage, void* stream) {
  if (v.eqn == EXO_EQN_SHALLOW_YZ || !(v.implicit_flag & 1)) return 0;
  launch_kb_implicit(v.precision, member_block_count(v, BK_IMPLICIT), v.tiles[BK_IMPLICIT], v.nc1,
                     (cudaStream_t)stream, one(v, BK_IMPLICIT), stage, 0.,
                     (v.implicit_flag & 8) != 0);
  return check_launch();
}

int launch_implicit_du(const DevView& v, double dt, void* stream) {
  if (v.eqn == EXO_EQN_SHALLOW_YZ || !(v.implicit_flag & 1)) return 0;
  launch_kb_implicit(v.precision, member_block_count(v, BK_IMPLICIT), v.tiles[BK_IMPLICIT], v.nc1,
                     (cudaStream_t)stream, one(v, BK_IMPLICIT), -1, dt,
                     (v.implicit_flag & 8) != 0);
  return check_launch();
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

// One SSPRK(3,3) step of every member of a batch: the stage sequence of
// one_step() (capi.cpp) with each kernel launched once for all members.
int launch_batched_step(const BatchPlan& pl, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (pl.n <= 0) return 0;
  auto B = [&](int kind) { return Batch{pl.views, pl.start[kind], pl.n}; };
  int rc;
  for (int s = 0; s < 3; ++s) {
    if (pl.total[BK_X1]) {
      kb_flux_x1<EXO_FLUX_T><<<pl.total[BK_X1], pl.x1_threads, pl.x1_smem, st>>>(B(BK_X1));
      if ((rc = check_launch())) return rc;
    }
    kb_flux_x23<EXO_FLUX_T><<<pl.total[BK_X23], x23_threads(pl.threads[BK_X23]), 0, st>>>(
        B(BK_X23));
    if ((rc = check_launch())) return rc;
    kb_update<EXO_FLUX_T><<<pl.total[BK_UPDATE], pl.threads[BK_UPDATE], 0, st>>>(B(BK_UPDATE), s);
    if ((rc = check_launch())) return rc;
    if (s == 2 && pl.total[BK_ROUNDTRIP]) {
      kb_roundtrip<<<pl.total[BK_ROUNDTRIP], pl.threads[BK_ROUNDTRIP], 0, st>>>(B(BK_ROUNDTRIP));
      if ((rc = check_launch())) return rc;
    }
    if (pl.total[BK_IMPLICIT]) {
      launch_kb_implicit(pl.precision, pl.total[BK_IMPLICIT], pl.threads[BK_IMPLICIT],
                         pl.max_nc1, st, B(BK_IMPLICIT), s, 0., pl.any_full_correction);
      if ((rc = check_launch())) return rc;
    }
    if (s == 2) {
      kb_dt_reset<<<nblk(pl.n, 128), 128, 0, st>>>(pl.views, pl.n);
      if ((rc = check_launch())) return rc;
    }
    kb_prim_ghost<<<pl.total[BK_PRIM], pl.threads[BK_PRIM], 0, st>>>(B(BK_PRIM), s == 2 ? 1 : 0);
    if ((rc = check_launch())) return rc;
  }
  kb_dt_finalize<<<nblk(pl.n, 128), 128, 0, st>>>(pl.views, pl.n, 1);
  return check_launch();
}

}  // namespace EXO_KNS
}  // namespace exo
