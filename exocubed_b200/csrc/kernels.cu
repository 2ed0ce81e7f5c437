// kernels.cu -- the FP64 build of the step (no fused multiply-add: it
// reproduces the CPU restatement bit for bit wherever no transcendental
// function is involved) plus the row-level hooks that exist only in FP64:
// exo_riemann, exo_weno5, exo_implicit_columns and its allocation-free form.
#define EXO_KNS fp64
#define EXO_MIXED 0
#define EXO_FLUX_T double
#include "exo_kernels.cuh"

#include <mutex>
#include <string>

namespace exo {
namespace fp64 {
namespace {

// ImplicitSolver::FullCorrection (full != 0) or PartialCorrection over a
// batch of independent columns given as plain arrays: w [ncol][5][L+6] primitives with ghosts, du [ncol][5][L]
// explicit update (overwritten by the corrected one), colgeo [ncol][4] =
// (cos, sin, dx2f_ang, dx3f_ang), scratch ncol*L*30 doubles.
// A column of exo_implicit_columns: w [5][L+6] and du [5][L] of this column,
// the corrected update written back into du.
struct HookColumnIO {
  using Real = double;
  const double* wc;
  double* duc;
  int nc1, L;
  double* scr0;
  size_t nslot;
  __device__ __forceinline__ void w(int i, double* out) const {
#pragma unroll
    for (int n = 0; n < 5; ++n) out[n] = wc[n * nc1 + i];
  }
  __device__ __forceinline__ const double* wptr(int i, int n) const { return wc + n * nc1 + i; }
  __device__ __forceinline__ const double* duptr(int i, int n) const {
    return duc + n * L + (i - G);
  }
  __device__ __forceinline__ double& scr(int lev, int e) const {
    return scr0[((size_t)lev * 30 + e) * nslot];
  }
  static constexpr bool kLoadsU = false;
  __device__ __forceinline__ const double* uptr(int, int) const { return nullptr; }
  __device__ __forceinline__ void uload(int, double*) const {}
  __device__ __forceinline__ void ustore(int i, const double*, const double* dl) const {
#pragma unroll
    for (int n = 0; n < 5; ++n) duc[n * L + (i - G)] = dl[n];
  }
};

__global__ void EXO_IMPL_BOUNDS k_implicit_columns(
    int ncol, int L, const double* w, double* du, const double* colgeo, const double* x1f,
    const double* x1v, const double* dx1f, double dt, double gamma, double grav,
    double* scratch, int full) {
  extern __shared__ double ism[];
  const int col = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int nc1 = L + 2 * G;
  const double *sx1f, *sx1v, *sdx1f;
  stage_radial(impl_radial<double>(ism), nc1, x1f, x1v, dx1f, sx1f, sx1v, sdx1f);
  if (col >= ncol) return;
  HookColumnIO io{w + (size_t)col * 5 * nc1, du + (size_t)col * 5 * L, nc1, L, scratch + col,
                  (size_t)ncol};
  const double* g4 = colgeo + (size_t)col * 4;
  const ImplSlices<double> sl = impl_slices<double>(ism, full != 0);
  if (full)
    implicit_column(io, sl.sa, sl.sp, sl.ss, g4[0], g4[1], g4[2], g4[3], sx1f, sx1v, sdx1f, G,
                    G + L - 1, dt, gamma, grav);
  else
    implicit_column_partial(io, sl.sa, sl.sp, sl.ss, g4[0], g4[1], g4[2], g4[3], sx1f, sx1v,
                            sdx1f, G, G + L - 1, dt, gamma, grav);
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
  FaceGeo<double> fg{cosf ? cosf[m] : 0., sinf ? sinf[m] : 1., cthp ? cthp[m] : 0., cthc ? cthc[m] : 0.};
  riemann<double>(rsolver, gamma, ivx, fg, a, b, f);
  for (int q = 0; q < nv; ++q) flx[(size_t)q * n + m] = f[q];
}

__global__ void k_weno5(int n, const double* a, const double* b, const double* c,
                        const double* d, const double* e, double* out) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) out[m] = weno5<double>(a[m], b[m], c[m], d[m], e[m]);
}

// Decomposition::ChangeToPerturbation (change_to_perturbation.cpp:39-157) on
// one interior radial column of w (in place), one thread per column: the
// original pressure and density are kept in orig, the face pressures in psf,
// the column's gamma and entropy in colc, for RestoreFromPerturbation.
struct DecompRefs {
  double* psf;   // [6][nc3][nc2][nc1+1]
  double* pres;  // [6][nc3][nc2][nc1]
  double* dens;  // [6][nc3][nc2][nc1]
  double* colc;  // [6][nc3][nc2][2]: gamma, entropy
};

__device__ __forceinline__ bool decomp_column(const DevView& v, int col, int& p, int& k, int& j) {
  if (col >= 6 * v.N * v.N) return false;
  j = v.js + col % v.N;
  k = v.ks + (col / v.N) % v.N;
  p = col / (v.N * v.N);
  return true;
}

__global__ void k_change_to_perturbation(DevView v, double* w, DecompRefs r) {
  int p, k, j;
  if (!decomp_column(v, blockIdx.x * blockDim.x + threadIdx.x, p, k, j)) return;
  const int nc1 = v.nc1, is = v.is, ie = v.ie;
  const size_t q = ((size_t)p * v.nc3 + k) * v.nc2 + j;
  double* wd = w + idx(v, p, IDN, k, j, 0);
  double* wp = w + idx(v, p, IPR, k, j, 0);
  double* psf = r.psf + q * (nc1 + 1);
  for (int i = 0; i < nc1; ++i) {
    r.pres[q * nc1 + i] = wp[i];
    r.dens[q * nc1 + i] = wd[i];
  }
  const double grav = -v.grav;
  const double RdTv = wp[ie] / wd[ie];
  psf[ie + 1] = wp[ie] * exp(-grav * v.dx1f[ie] / (2 * RdTv));
  for (int i = ie; i >= is; --i) psf[i] = psf[i + 1] + grav * wd[i] * v.dx1f[i];
  for (int i = 1; i <= G; ++i) psf[is - i] = psf[is + i];
  for (int i = 1; i <= G; ++i) psf[ie + i + 1] = psf[ie + 1 - i];
  // PopulateBotEntropy (decomposition.cpp:341-388), no bottom neighbour
  const double gammad = v.gamma, fsig = 1., feps = 1.;
  const double gam = 1. + (gammad - 1.) * feps / fsig;
  const double ent = log(wp[is]) - gam * log(wd[is]);
  r.colc[2 * q] = gam;
  r.colc[2 * q + 1] = ent;
  const double expf = exp(-ent / gam);
  for (int i = 0; i < nc1; ++i) {
    double psv;
    if (fabs(psf[i] - psf[i + 1]) < 1.E-6)
      psv = (psf[i] + psf[i + 1]) / 2.;
    else
      psv = (psf[i] - psf[i + 1]) / log(psf[i] / psf[i + 1]);
    const double dsv = pow(psv, 1. / gam) * expf;
    wp[i] -= psv;
    wd[i] -= dsv;
  }
}

// Decomposition::RestoreFromPerturbation (:159-222): the column's pressure
// and density back in w, the face pressure and isentropic face density added
// to the x1 face states wl, wr (same layout as w, faces is..ie+1)
__global__ void k_restore_from_perturbation(DevView v, double* w, double* wl, double* wr,
                                            DecompRefs r) {
  int p, k, j;
  if (!decomp_column(v, blockIdx.x * blockDim.x + threadIdx.x, p, k, j)) return;
  const int nc1 = v.nc1;
  const size_t q = ((size_t)p * v.nc3 + k) * v.nc2 + j;
  const size_t bp = idx(v, p, IPR, k, j, 0), bd = idx(v, p, IDN, k, j, 0);
  for (int i = 0; i < nc1; ++i) {
    w[bp + i] = r.pres[q * nc1 + i];
    w[bd + i] = r.dens[q * nc1 + i];
  }
  const double* psf = r.psf + q * (nc1 + 1);
  const double gam = r.colc[2 * q], ent = r.colc[2 * q + 1];
  for (int i = v.is; i <= v.ie + 1; ++i) {
    wr[bp + i] += psf[i];
    if (wr[bp + i] < 0.) wr[bp + i] = psf[i];
    wl[bp + i] += psf[i];
    if (wl[bp + i] < 0.) wl[bp + i] = psf[i];
    const double dsf = pow(psf[i], 1. / gam) * exp(-ent / gam);
    wr[bd + i] += dsf;
    if (wr[bd + i] < 0.) wr[bd + i] = dsf;
    wl[bd + i] += dsf;
    if (wl[bd + i] < 0.) wl[bd + i] = dsf;
  }
}

}  // namespace
}  // namespace fp64

int launch_change_to_perturbation(const DevView& v, double* w, double* refs, void* stream) {
  const size_t nq = (size_t)6 * v.nc3 * v.nc2;
  fp64::DecompRefs r{refs, refs + nq * (v.nc1 + 1), refs + nq * (v.nc1 + 1) + nq * v.nc1,
                     refs + nq * (v.nc1 + 1) + 2 * nq * v.nc1};
  const int ncol = 6 * v.N * v.N;
  fp64::k_change_to_perturbation<<<fp64::nblk(ncol, 64), 64, 0, (cudaStream_t)stream>>>(v, w, r);
  return fp64::check_launch();
}

int launch_restore_from_perturbation(const DevView& v, double* w, double* wl, double* wr,
                                     double* refs, void* stream) {
  const size_t nq = (size_t)6 * v.nc3 * v.nc2;
  fp64::DecompRefs r{refs, refs + nq * (v.nc1 + 1), refs + nq * (v.nc1 + 1) + nq * v.nc1,
                     refs + nq * (v.nc1 + 1) + 2 * nq * v.nc1};
  const int ncol = 6 * v.N * v.N;
  fp64::k_restore_from_perturbation<<<fp64::nblk(ncol, 64), 64, 0, (cudaStream_t)stream>>>(
      v, w, wl, wr, r);
  return fp64::check_launch();
}

size_t decomposition_refs_doubles(const DevView& v) {
  const size_t nq = (size_t)6 * v.nc3 * v.nc2;
  return nq * (v.nc1 + 1) + 2 * nq * v.nc1 + 2 * nq;
}

// the column kernel's shared memory grows with L (the radial tables); the
// attribute lets a launch go past the 48 KB default
static cudaError_t allow_column_smem() {
  return cudaFuncSetAttribute(fp64::k_implicit_columns,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, fp64::IMPL_SMEM_MAX);
}

int launch_implicit_columns(int ncol, int L, const double* w, double* du, const double* colgeo,
                            const double* x1f, const double* x1v, const double* dx1f, double dt,
                            double gamma, double grav, double* scratch, void* stream, int full) {
  if (ncol <= 0) return 0;
  if (allow_column_smem() != cudaSuccess) return EXO_ERR_CUDA;
  fp64::k_implicit_columns<<<fp64::nblk(ncol, fp64::IMPL_THREADS), fp64::IMPL_THREADS,
                              fp64::impl_smem<double>(fp64::IMPL_THREADS, L + 2 * G),
                              (cudaStream_t)stream>>>(
      ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, scratch, full);
  return fp64::check_launch();
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
  if (e != cudaSuccess) {
    *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) {
    *err = "device index " + std::to_string(dev) +
           " is not supported by the no-alloc scratch table (devices 0..63)";
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
  e = allow_column_smem();
  if (e != cudaSuccess) {
    *err = std::string("cudaFuncSetAttribute(k_implicit_columns): ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  fp64::k_implicit_columns<<<fp64::nblk(ncol, fp64::IMPL_THREADS), fp64::IMPL_THREADS,
                              fp64::impl_smem<double>(fp64::IMPL_THREADS, L + 2 * G),
                              (cudaStream_t)stream>>>(
      ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, scratch, 1);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    *err = std::string("k_implicit_columns: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  return 0;
}

int launch_riemann_rows(int rsolver, int eqn, int ivx, int n, double gamma, const double* wl,
                        const double* wr, double* flx, const double* cosf, const double* sinf,
                        const double* cthp, const double* cthc, void* stream) {
  if (n <= 0) return 0;
  fp64::k_riemann_rows<<<fp64::nblk(n, 128), 128, 0, (cudaStream_t)stream>>>(
      rsolver, eqn, ivx, n, gamma, wl, wr, flx, cosf, sinf, cthp, cthc);
  return fp64::check_launch();
}

int launch_weno5(int n, const double* a, const double* b, const double* c, const double* d,
                 const double* e, double* out, void* stream) {
  if (n <= 0) return 0;
  fp64::k_weno5<<<fp64::nblk(n, 128), 128, 0, (cudaStream_t)stream>>>(n, a, b, c, d, e, out);
  return fp64::check_launch();
}

}  // namespace exo
