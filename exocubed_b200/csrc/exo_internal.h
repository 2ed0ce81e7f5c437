// exo_internal.h -- shared definitions of the host geometry builder, the
// CUDA kernels and the C ABI layer.
#ifndef EXO_INTERNAL_H_
#define EXO_INTERNAL_H_

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/exo_b200.h"

namespace exo {

// NVTX range for the host side of a call (steps, stages, redos, checkpoints):
// visible in Nsight Systems and Nsight Compute timelines, free when no
// profiler is attached.  Defined in capi.cpp.
struct Range {
  explicit Range(const char* name);
  ~Range();
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

constexpr int G = EXO_NGHOST;
constexpr int IDN = 0, IVX = 1, IVY = 2, IVZ = 3, IPR = 4, IEN = 4;
enum Side { UP = 0, DOWN = 1, LEFT = 2, RIGHT = 3 };

// Fields of the per-panel (k,j) metric table, each nc3*nc2 doubles per panel.
enum Geo2D {
  GCOSC = 0, GSINC, GCOSF2, GSINF2, GCOSF3, GSINF3,  // cell / face metric
  GDX2A, GDX3A, GDX2A_F3, GDX3A_F2,                // angular widths
  GCTHP1, GCTHP2, GCTHP3,                          // flux projection angles
  GFCOR,                                           // Coriolis parameter 2*Omega*sin(lat)
  GCR0, GCR1, GCR2, GCR3,                          // cell (V2,V3) -> (U,V)
  GCQ0, GCQ1, GCQ2, GCQ3,                          // cell (U,V) -> (V2,V3)
  GSLAT2, GCLAT2, GCLAT4,                          // sin^2, cos^2, cos^4 of the latitude
  GTANX, GTANY, GC3C, GC3D, GC3A,                  // CalculateCoriolisForce3: x, y, C, D,
                                                   // 2 Omega C D / delta^2
  NGEO2D
};

// Held-Suarez forcing constants of a DevView (host-computed, hs94.cpp:212-243)
enum HsParam {
  HS_P0 = 0, HS_TS, HS_DT, HS_DTHETA, HS_KF, HS_KA, HS_KS, HS_SIGMAB,  // Kf, Ka, Ks in 1/s
  HS_KAPPA,                                                            // Rd / cp
  HS_CVM,                                                              // cp - Rd
  NHS
};

// One ghost-band cell of a receiving panel (independent of i and n).  Its
// value is interpolated along the shared edge from two interior cells of
// the neighbour panel: (A*v0 + B*v1)/C, and momenta are rotated through
// latitude-longitude (cubed_sphere_utility.cpp:92-369).
struct GhostEntry {
  int src_panel;
  int k0, j0, k1, j1;        // the two source cells
  int pad;
  double A, B, C;
  double ss, cs;             // source-point metric (raise to contravariant)
  double r[4];               // (V2,V3) -> (U,V) at the source point
  double q[4];               // (U,V) -> (V2,V3) at the target point
  double ct;                 // target-point metric (lower to covariant)
};

// One edge face of a receiving panel: the outer face state comes from the
// neighbour's interior-side reconstruction at its own edge face, rotated into
// this panel's basis (cubed_sphere.cpp:326-688).
struct EdgeEntry {
  int src_panel;
  int src_side;
  int src_along;
  int pad;
  double r[4];               // (V2,V3) -> (U,V) at the sender's edge point
  double q[4];               // (U,V) -> (V2,V3) in the receiver's basis
};

// Everything the host computes once per context.
struct HostTables {
  int N, L, nc1, nc2, nc3;
  std::vector<double> x1f, x1v, dx1f;             // nc1+1, nc1, nc1
  std::vector<double> x2f[6], x2v[6], x3f[6], x3v[6];
  std::vector<double> geo;                        // [NGEO2D][6][nc3][nc2]
  std::vector<int> ghost_map;                     // [6][nc3][nc2] -> entry or -1
  std::vector<GhostEntry> ghost;
  std::vector<EdgeEntry> edge;                    // [6][4][N]
  size_t g2(int f, int p, int k, int j) const {
    return (((size_t)f * 6 + p) * nc3 + k) * nc2 + j;
  }
};

// geometry.cpp
bool build_tables(const exo_config& cfg, HostTables& t, std::string* err);
// the panel (0-based) across side s (0 Up, 1 Down, 2 Left, 3 Right) of panel
// p and the side of it that edge is (CubedSphere::TransformOX)
void panel_neighbor(int p, int s, int* tp, int* ts);

// Device-side scalars of one atmosphere (time step bookkeeping and flags).
struct DevScalars {
  double dt;                       // step in use
  double time;                     // simulated time
  unsigned long long dtmin_bits;   // running min of the CFL candidate (bits of a positive double)
  int invalid;                     // sticky: rho/p negative or NaN
  int timeout;                     // sticky: a kernel's bounded wait gave up
  long long ncycle;
};

// n / d for 0 <= n < 2^40 / (d - 1) as floor(n m / 2^40), m = ceil(2^40 / d):
// with n = q d + t, n m / 2^40 = q + t / d + n r / (d 2^40) for some r < d,
// which stays below q + 1 in that range (the kernels' flat indices are
// 32-bit and their divisors at most a few thousand).  n m needs up to 72
// bits (m < 2^41), so it is formed from the two 32-bit halves of m, each
// product within 64 bits: floor(n m / 2^40) = (n mh + floor(n ml / 2^32)) >> 8.
struct FastDiv {
  unsigned long long m;
#ifdef __CUDACC__
  __host__ __device__
#endif
  unsigned operator()(unsigned n) const {
    const unsigned long long lo = (unsigned long long)n * (unsigned)(m & 0xffffffffull);
    const unsigned long long hi = (unsigned long long)n * (unsigned)(m >> 32);
    return (unsigned)((hi + (lo >> 32)) >> 8);
  }
};
inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f;
  f.m = ((1ull << 40) + d - 1) / d;
  return f;
}

// Sizes, parameters and device pointers of one atmosphere; passed by value
// to every kernel.
struct alignas(16) DevView {
  int N, L, nv, nc1, nc2, nc3;
  FastDiv div_L, div_N, div_nc1, div_nc2, div_nc3;  // divisions by L, N, nc1, nc2, nc3
  int is, ie, js, je, ks, ke;
  int eqn, rsolver, implicit_flag, coriolis;
  int precision, forcing;
  double gamma, Rd, grav, cfl;
  double hs[NHS];                  // Held-Suarez constants (forcing == EXO_FORCING_HS94)
  size_t cells;                    // nc3*nc2*nc1 (one variable of one panel)
  // state
  double* u;
  double* w;
  double* u1;
  double* du;
  double* flux[3];                 // face fluxes, same layout as u
  float* w32;                      // mixed precision: FP32 copy of w for the flux kernels
  float* flux32[3];                // mixed precision: FP32 face fluxes
  double* scratch;                 // implicit solver: per column L*(25+5) doubles
  // tables
  const double* x1f;
  const double* x1v;
  const double* dx1f;
  const double* geo;               // [NGEO2D][6][nc3][nc2]
  const int* ghost_map;            // [6][nc3][nc2]
  const GhostEntry* ghost;
  const EdgeEntry* edge;           // [6][4][N]
  DevScalars* sc;
  // device copy of this view and its block table [BK_COUNT][2] = {0, blocks}:
  // the single-atmosphere launches are batches of one
  const DevView* self;
  const unsigned* starts;
  int tiles[6];                    // threads per block by BatchKind (see Tiles)
};

// A batched step: every member's DevView in device memory and, per kernel
// kind, the first block of every member (start[k][n] = total blocks).
enum BatchKind { BK_X1 = 0, BK_X23, BK_UPDATE, BK_IMPLICIT, BK_PRIM, BK_ROUNDTRIP, BK_COUNT };
struct BatchPlan {
  const DevView* views;          // device, n entries
  int n;
  const unsigned* start[BK_COUNT];  // device, n+1 entries each
  unsigned total[BK_COUNT];
  int x1_threads;                // block size of the x1 flux kernel
  size_t x1_smem;                // its dynamic shared memory
  int threads[BK_COUNT];         // tiles of the other kernels
  int max_nc1;                   // largest nc1 of the members (radial tables in shared memory)
  int precision;                 // EXO_PREC_* of every member
  bool any_full_correction;      // some member takes the 5x5 solve (kb_implicit_bwd runs)
};
// Threads per block ("tile") of each batched kernel by BatchKind.  BK_X1
// takes one radial column per block (its size follows L) and ignores its
// entry; the others may be any multiple of 32 in [32, 512], BK_IMPLICIT one of
// 32, 64, 128.  The per-cell arithmetic does not depend on them.
struct Tiles {
  int t[BK_COUNT];
};
Tiles default_tiles();
bool valid_tiles(const int* t, std::string* err);
// The x1 kernel takes tiles[BK_X1] radial columns per block (1..X1_MAX_COLUMNS).
// Shared memory per column: the primitives and the face pressures, and in
// the mixed build ln psf and the face densities.
constexpr int X1_MAX_COLUMNS = 8;
// the x1 kernel's dynamic shared memory limit (the mixed build's 8 columns
// of 250 levels take 212 KB)
constexpr int X1_SMEM_MAX = 224 * 1024;
#ifdef __CUDACC__
#define EXO_HD __host__ __device__
#else
#define EXO_HD
#endif
// the precisions stepped by the mixed build (exo::mixed)
EXO_HD inline bool mixed_build(int precision) {
  return precision == EXO_PREC_MIXED || precision == EXO_PREC_MIXED_F32_SOLVE;
}
// The implicit solve with the full (5x5) correction: FP64 blocks solve and
// back-substitute each column in kb_implicit (a column's back substitution
// overlaps other columns' forward sweeps); FP32 blocks run the forward sweep
// in kb_implicit and the back substitution in kb_implicit_bwd (memory-bound,
// fed by bulk copies).  The partial (3x3) correction does both in kb_implicit.
EXO_HD inline bool split_bwd(int precision) { return precision == EXO_PREC_MIXED_F32_SOLVE; }
inline int implicit_launches(int implicit_flag, int precision) {
  return ((implicit_flag & 8) && split_bwd(precision)) ? 2 : 1;
}
// shared doubles of one x1 column: w [nv][nc1] and psf [nc1+1]; the mixed
// build adds ln psf and the face densities [2][nc1+1] and the cells' two
// WENO5 face values [2][nv][L+2] in FP32 (nv (L+2) doubles)
EXO_HD inline int x1_column_doubles(const DevView& v) {
  int faces = v.nc1 + 1;
  return v.nv * v.nc1 +
         (mixed_build(v.precision) ? 3 * faces + v.nv * (v.L + 2) : faces);
}
inline int x1_cols(const DevView& v) { return v.tiles[BK_X1] > 0 ? v.tiles[BK_X1] : 1; }
inline size_t x1_smem_bytes(const DevView& v) {
  return (size_t)x1_cols(v) * x1_column_doubles(v) * sizeof(double);
}
// threads: the block's faces in whole warps, at most 1024
inline int x1_threads(const DevView& v) {
  int t = ((x1_cols(v) * (v.L + 1) + 31) / 32) * 32;
  return t > 1024 ? 1024 : t;
}
// Columns per block of a member of a batch whose x1 blocks run `threads`
// threads: as many as the member's faces fill (a member with fewer levels
// than the batch's deepest takes more columns per block rather than leave
// threads idle), 1 to X1_MAX_COLUMNS, within the kernel's shared memory.
inline int x1_member_columns(const DevView& v, int threads, size_t smem_max) {
  int c = threads / (v.L + 1);
  c = c < 1 ? 1 : (c > X1_MAX_COLUMNS ? X1_MAX_COLUMNS : c);
  const size_t per = (size_t)x1_column_doubles(v) * sizeof(double);
  while (c > 1 && (size_t)c * per > smem_max) --c;
  return c;
}
// block counts of one member for the given tiles
void member_blocks(const DevView& v, const int* tiles, unsigned blocks[BK_COUNT]);
// re-uploads the view's own device copy (tiles and block table)
int view_refresh_self(DevView& v, void* stream, std::string* err);

// Launchers of one arithmetic build (exo_kernels.cuh): fp64 (kernels.cu) and
// mixed (kernels_mixed.cu) provide the same set.
#define EXO_DECLARE_STEP_LAUNCHERS                                                   \
  int launch_prim_ghost(const DevView& v, bool compute_dt, void* stream);            \
  int launch_flux_x1(const DevView& v, void* stream);                                \
  int launch_flux_x23(const DevView& v, void* stream);                               \
  int launch_update(const DevView& v, int stage, void* stream);                      \
  int launch_implicit(const DevView& v, int stage, void* stream);                    \
  int launch_implicit_du(const DevView& v, double dt, void* stream);                 \
  int launch_dt_reset(const DevView& v, void* stream);                               \
  int launch_dt_finalize(const DevView& v, double dt_fixed, bool advance_time, void* stream); \
  int launch_set_dt(const DevView& v, double dt, void* stream);                      \
  int launch_p2c_interior(const DevView& v, const double* w_src, void* stream);          \
  int launch_batched_step(const BatchPlan& plan, void* stream);                     \
  int prepare_kernels();                                                            \
  int launch_reciprocal(int n, const double* x, double* out, void* stream);         \
  unsigned x23_blocks(const DevView& v, int tile);
namespace fp64 { EXO_DECLARE_STEP_LAUNCHERS }
namespace mixed { EXO_DECLARE_STEP_LAUNCHERS }
#undef EXO_DECLARE_STEP_LAUNCHERS

// kernels.cu: FP64 row-level hooks
int launch_riemann_rows(int rsolver, int eqn, int ivx, int n, double gamma,
                        const double* wl, const double* wr, double* flx,
                        const double* cosf, const double* sinf, const double* cthp,
                        const double* cthc, void* stream);
int launch_weno5(int n, const double* a, const double* b, const double* c,
                 const double* d, const double* e, double* out, void* stream);
int launch_implicit_columns(int ncol, int L, const double* w, double* du, const double* colgeo,
                            const double* x1f, const double* x1v, const double* dx1f, double dt,
                            double gamma, double grav, double* scratch, void* stream, int full);
// Decomposition hooks on whole arrays of one atmosphere (refs: face
// pressures, original pressure and density, column constants)
int launch_change_to_perturbation(const DevView& v, double* w, double* refs, void* stream);
int launch_restore_from_perturbation(const DevView& v, double* w, double* wl, double* wr,
                                     double* refs, void* stream);
size_t decomposition_refs_doubles(const DevView& v);
int launch_implicit_columns_noalloc(int ncol, int L, const double* w, double* du,
                                    const double* colgeo, const double* x1f, const double* x1v,
                                    const double* dx1f, double dt, double gamma, double grav,
                                    void* stream, std::string* err);
// kernels.cu: the boundary's panel and equation-of-state hooks (FP64)
int launch_panel_pack(const DevView& v, const double* src, double* buf, int tp, int rsk, int rsj,
                      int K, int J, void* stream);
int launch_face_sync(const DevView& v, double* L2, double* R2, double* L3, double* R3,
                     void* stream);
int launch_eos_range(const DevView& v, int to_prim, const double* in, double* out, int il, int iu,
                     int jl, int ju, int kl, int ku, void* stream);
int launch_sound_speed(const DevView& v, int n, const double* prim, double* cs, void* stream);
int launch_view_copy(const void* src, const int64_t* sstride, void* dst, const int64_t* dstride,
                     const int* size, void* stream);
// peaks.cu: best FMA rate (flops/s) of independent chains on all SMs
int measure_fma_peak(bool fp64, int repeats, double* flops_per_s, std::string* err);
// peaks.cu: a bounded mbarrier wait that nothing completes, run once
int bounded_wait_selftest(int* gave_up, double* waited_ms, std::string* err);


// checkpoint.cpp: images of one atmosphere (exo_checkpoint_header, u, w)
size_t checkpoint_bytes(const DevView& v);
bool same_config_but_precision(const exo_config& a, const exo_config& b);
int checkpoint_save(const exo_config& cfg, const DevView& v, void* stream, void* image,
                    size_t bytes, std::string* err);
// checks magic, version, configuration and size; copies the header out
int checkpoint_parse(const void* image, size_t bytes, exo_checkpoint_header* h,
                     std::string* err);
// u, w and the clock of an image already parsed into the atmosphere v
int checkpoint_restore(const DevView& v, void* stream, const void* image, std::string* err);

// capi.cpp: shared by the single-atmosphere context and the ensemble
bool validate_config(const exo_config& cfg, std::string* err);
size_t view_footprint(const exo_config& cfg);
int view_allocate(const exo_config& cfg, const HostTables& t, DevView& v,
                  std::vector<void*>& owned, void* stream, void* pool, std::string* err);
int set_error(int code, const std::string& msg);
void view_free(std::vector<void*>& owned, void* stream);

// cell (U,V) <-> panel vector transforms of cubed_sphere_transform.cpp:11-61
// written as coefficient quadruples: out0 = c0*in0 + c1*in1, out1 = c2*in0 + c3*in1
void rll_from_abp_coef(double X, double Y, int blockID, double c[4]);
void abp_from_rll_coef(double X, double Y, int blockID, double c[4]);
void rll_from_xyp(double dX, double dY, int nP, double& lon, double& lat);

}  // namespace exo

#endif  // EXO_INTERNAL_H_
