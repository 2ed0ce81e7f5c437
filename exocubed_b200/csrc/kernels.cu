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

namespace fp64 {
namespace {

// CubedSphereUtility::PackData of one face: panel src's edge band
// interpolated onto the neighbour's ghost band (target panel tp, rows
// [rsk, rsk+K) x [rsj, rsj+J)), packed in the band's plain (n, k, j, i) order
// -- the order the receiver unpacks, which PackDataR0..R3 produce on the
// sender's side
__global__ void k_panel_pack(DevView v, const double* src, double* buf, int tp, int rsk, int rsj,
                             int K, int J) {
  const int L = v.L;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)K * J * L) return;
  const int ii = (int)(tid % L);
  const int r = (int)(tid / L);
  const int jj = r % J, kk = r / J;
  const int k = rsk + kk, j = rsj + jj, i = v.is + ii;
  const GhostEntry& e = v.ghost[v.ghost_map[((size_t)tp * v.nc3 + k) * v.nc2 + j]];
  double c[5];
  ghost_interp(v, e, src, i, c);
  for (int n = 0; n < v.nv; ++n) buf[(((size_t)n * K + kk) * J + jj) * L + ii] = c[n];
}

// The face position of along index `along` of a panel side: direction (1: x2
// faces, 2: x3 faces) and (k, j)
__device__ __forceinline__ void edge_face(const DevView& v, int side, int along, int& dir, int& k,
                                          int& j) {
  if (side == UP) { dir = 1; j = v.js; k = v.ks + along; }
  else if (side == DOWN) { dir = 1; j = v.je + 1; k = v.ks + along; }
  else if (side == LEFT) { dir = 2; k = v.ks; j = v.js + along; }
  else { dir = 2; k = v.ke + 1; j = v.js + along; }
}

// CubedSphere::SynchronizeFluxesSend/Recv/Wait (cubed_sphere.cpp:289-688) on
// the face-state stores: every receiving edge face takes the sender's
// interior-side state (L at the sender's Down/Right edges, R at Up/Left),
// rotated into the receiver's basis, as its outer state (L at the
// receiver's Up/Left edges, R at Down/Right); faces i = is-1 .. ie+1.
// Senders are never receivers of the same store, so one pass suffices.
__global__ void k_face_sync(DevView v, double* L2, double* R2, double* L3, double* R3) {
  const int ni = v.L + 2, N = v.N;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)6 * 4 * N * ni) return;
  const int ii = (int)(tid % ni);
  long long r = tid / ni;
  const int b = (int)(r % N);
  r /= N;
  const int ts = (int)(r % 4), tp = (int)(r / 4);
  const int i = v.is - 1 + ii;
  const EdgeEntry& e = v.edge[((size_t)tp * 4 + ts) * N + b];
  int sd, sk, sj, td, tk, tj;
  edge_face(v, e.src_side, e.src_along, sd, sk, sj);
  edge_face(v, ts, b, td, tk, tj);
  const double* S = sd == 1 ? (e.src_side == DOWN ? L2 : R2) : (e.src_side == RIGHT ? L3 : R3);
  double* D = td == 1 ? (ts == UP ? L2 : R2) : (ts == LEFT ? L3 : R3);
  double st[5];
  for (int n = 0; n < v.nv; ++n) st[n] = S[idx(v, e.src_panel, n, sk, sj, i)];
  const double V2 = st[IVY], V3 = st[IVZ];
  const double U = e.r[0] * V2 + e.r[1] * V3;
  const double V = e.r[2] * V2 + e.r[3] * V3;
  st[IVY] = e.q[0] * U + e.q[1] * V;
  st[IVZ] = e.q[2] * U + e.q[3] * V;
  for (int n = 0; n < v.nv; ++n) D[idx(v, tp, n, tk, tj, i)] = st[n];
}

// EquationOfState::ConservedToPrimitive (to_prim != 0) or PrimitiveToConserved
// over cells [il, iu] x [jl, ju] x [kl, ku] of every panel (whole arrays in
// the context's layout); an invalid density or pressure sets the sticky flag
__global__ void k_eos_range(DevView v, int to_prim, const double* in, double* out, int il,
                            int jl, int kl, int ni, int nj, int nk) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)6 * ni * nj * nk) return;
  const int i = il + (int)(tid % ni);
  long long r = tid / ni;
  const int j = jl + (int)(r % nj);
  r /= nj;
  const int k = kl + (int)(r % nk);
  const int p = (int)(r / nk);
  double a[5], b[5];
  for (int n = 0; n < v.nv; ++n) a[n] = in[idx(v, p, n, k, j, i)];
  const double cth = geo(v, GCOSC, p, k, j);
  if (to_prim) {
    if (cons_to_prim(v, a, b, cth)) atomicOr(&v.sc->invalid, 1);
  } else {
    prim_to_cons(v, a, b, cth);
  }
  for (int n = 0; n < v.nv; ++n) out[idx(v, p, n, k, j, i)] = b[n];
}

// EquationOfState::SoundSpeed of n cells, prim (NHYDRO, n)
__global__ void k_sound_speed(DevView v, int n, const double* prim, double* cs) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  double w[5];
  for (int q = 0; q < v.nv; ++q) w[q] = prim[(size_t)q * n + m];
  if (v.eqn == EXO_EQN_SHALLOW_YZ) {
    cs[m] = sqrt(w[IDN]);
  } else {
    double fsig = 1., feps = 1.;
    cs[m] = sqrt((1. + (v.gamma - 1) * feps / fsig) * w[IPR] / w[IDN]);
  }
}

// element copy between two strided 4-D views of doubles (strides in elements)
struct Strides4 {
  long long s[4];
};
__global__ void k_view_copy(const double* src, Strides4 ss, double* dst, Strides4 ds, int n4,
                            int n3, int n2, int n1) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)n4 * n3 * n2 * n1) return;
  const int i = (int)(tid % n1);
  long long r = tid / n1;
  const int j = (int)(r % n2);
  r /= n2;
  const int k = (int)(r % n3);
  const int n = (int)(r / n3);
  dst[n * ds.s[0] + k * ds.s[1] + j * ds.s[2] + i * ds.s[3]] =
      src[n * ss.s[0] + k * ss.s[1] + j * ss.s[2] + i * ss.s[3]];
}

}  // namespace
}  // namespace fp64

int launch_panel_pack(const DevView& v, const double* src, double* buf, int tp, int rsk, int rsj,
                      int K, int J, void* stream) {
  const long long n = (long long)K * J * v.L;
  if (n <= 0) return 0;
  fp64::k_panel_pack<<<fp64::nblk((size_t)n, 128), 128, 0, (cudaStream_t)stream>>>(
      v, src, buf, tp, rsk, rsj, K, J);
  return fp64::check_launch();
}

int launch_face_sync(const DevView& v, double* L2, double* R2, double* L3, double* R3,
                     void* stream) {
  const size_t n = (size_t)6 * 4 * v.N * (v.L + 2);
  fp64::k_face_sync<<<fp64::nblk(n, 128), 128, 0, (cudaStream_t)stream>>>(v, L2, R2, L3, R3);
  return fp64::check_launch();
}

int launch_eos_range(const DevView& v, int to_prim, const double* in, double* out, int il, int iu,
                     int jl, int ju, int kl, int ku, void* stream) {
  const int ni = iu - il + 1, nj = ju - jl + 1, nk = ku - kl + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return 0;
  const size_t n = (size_t)6 * ni * nj * nk;
  fp64::k_eos_range<<<fp64::nblk(n, 128), 128, 0, (cudaStream_t)stream>>>(
      v, to_prim, in, out, il, jl, kl, ni, nj, nk);
  return fp64::check_launch();
}

int launch_sound_speed(const DevView& v, int n, const double* prim, double* cs, void* stream) {
  if (n <= 0) return 0;
  fp64::k_sound_speed<<<fp64::nblk((size_t)n, 128), 128, 0, (cudaStream_t)stream>>>(v, n, prim,
                                                                                     cs);
  return fp64::check_launch();
}

int launch_view_copy(const void* src, const int64_t* sstride, void* dst, const int64_t* dstride,
                     const int* size, void* stream) {
  const size_t n = (size_t)size[0] * size[1] * size[2] * size[3];
  if (n == 0) return 0;
  fp64::Strides4 ss, ds;
  for (int q = 0; q < 4; ++q) {
    ss.s[q] = sstride[q];
    ds.s[q] = dstride[q];
  }
  fp64::k_view_copy<<<fp64::nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(
      (const double*)src, ss, (double*)dst, ds, size[0], size[1], size[2], size[3]);
  return fp64::check_launch();
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
