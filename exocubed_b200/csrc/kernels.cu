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

// ImplicitSolver::FullCorrection over a batch of independent columns given
// as plain arrays: w [ncol][5][L+6] primitives with ghosts, du [ncol][5][L]
// explicit update (overwritten by the corrected one), colgeo [ncol][4] =
// (cos, sin, dx2f_ang, dx3f_ang), scratch ncol*L*30 doubles.
__global__ void __launch_bounds__(128) k_implicit_columns(int ncol, int L, const double* w,
                                                          double* du, const double* colgeo,
                                                          const double* x1f, const double* x1v,
                                                          const double* dx1f, double dt,
                                                          double gamma, double grav,
                                                          double* scratch) {
  ColumnLanes cl = column_lanes(ncol, blockIdx.x);
  int col = cl.col, r = cl.r;
  int nc1 = L + 2 * G;
  const double* wc = w + (size_t)col * 5 * nc1;
  double* duc = du + (size_t)col * 5 * L;
  size_t nslot = (size_t)ncol * 5;
  size_t slot = (size_t)col * 5 + r;
  double dummy = 0.;
  auto W = [&](int i, double* out) {
    for (int n = 0; n < 5; ++n) out[n] = wc[n * nc1 + i];
  };
  auto DU = [&](int i, int n) { return n < 5 ? duc[n * L + (i - G)] : 0.; };
  auto SCR = [&](int lev, int e) -> double& {
    return cl.active ? scratch[((size_t)lev * 6 + e) * nslot + slot] : dummy;
  };
  auto OUT = [&](int i, const double* dl) {
    if (cl.active) duc[r * L + (i - G)] = dl[r];
  };
  const double* g4 = colgeo + (size_t)col * 4;
  implicit_column_rows(cl.base, r, W, DU, SCR, OUT, g4[0], g4[1], g4[2], g4[3], x1f, x1v, dx1f,
                       G, G + L - 1, dt, gamma, grav);
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

}  // namespace
}  // namespace fp64

int launch_implicit_columns(int ncol, int L, const double* w, double* du, const double* colgeo,
                            const double* x1f, const double* x1v, const double* dx1f, double dt,
                            double gamma, double grav, double* scratch, void* stream) {
  if (ncol <= 0) return 0;
  size_t threads = (size_t)((ncol + 5) / 6) * 32;
  fp64::k_implicit_columns<<<fp64::nblk(threads, 128), 128, 0, (cudaStream_t)stream>>>(
      ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, scratch);
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
  size_t threads = (size_t)((ncol + 5) / 6) * 32;
  fp64::k_implicit_columns<<<fp64::nblk(threads, 128), 128, 0, (cudaStream_t)stream>>>(
      ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, scratch);
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
