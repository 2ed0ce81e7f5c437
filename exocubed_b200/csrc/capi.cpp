// capi.cpp -- the extern "C" boundary (include/exo_b200.h): context
// lifecycle, device memory, the stage sequence and the operator hooks.
//
// The stage sequence is ImplicitHydroTasks / TimeIntegratorTaskList of the
// reference (src/tasklist/implicit_hydro_tasks.cpp:40-102,
// patches/24.time_integrator.patch:22-60) with every MPI exchange replaced by
// a device read of the neighbour panel:
//   CALC_HYDFLX -> INT_HYD -> SRC_TERM -> IMPLICIT_CORR -> UPDATE_ALLCONS ->
//   ghost exchange -> CONS2PRIM -> PHY_BVAL -> NEW_DT
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "exo_internal.h"
#include "nvtx3/nvToolsExt.h"

exo::Range::Range(const char* name) { nvtxRangePushA(name); }
exo::Range::~Range() { nvtxRangePop(); }

using exo::DevScalars;
using exo::DevView;

// the step launchers of the context's arithmetic build
#define STEP(name, ...) \
  (exo::mixed_build(c->v.precision) ? exo::mixed::name(__VA_ARGS__) : exo::fp64::name(__VA_ARGS__))

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return EXO_ERR_CUDA;
}

#define CK(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

#define RK(call)                                               \
  do {                                                         \
    int r_ = (call);                                           \
    if (r_) {                                                  \
      cudaError_t e_ = cudaGetLastError();                     \
      return cuda_fail(e_ == cudaSuccess ? cudaErrorUnknown : e_, #call); \
    }                                                          \
  } while (0)

template <typename T>
int upload(T** dst, const std::vector<T>& src, std::vector<void*>& owned) {
  size_t bytes = src.size() * sizeof(T);
  if (bytes == 0) bytes = sizeof(T);
  CK(cudaMalloc((void**)dst, bytes));
  owned.push_back(*dst);
  if (!src.empty()) CK(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

}  // namespace

struct ProfEvent {
  cudaEvent_t a, b;
  int kernel;
};

struct exo_ctx {
  exo_config cfg;
  bool profiling = false;
  std::vector<ProfEvent> prof_used;
  std::vector<ProfEvent> prof_pool;
  int64_t launches = 0;
  exo::HostTables tab;
  DevView v;
  cudaStream_t stream = nullptr;
  std::vector<void*> owned;
  size_t state_elems = 0;  // 6*nv*cells
  bool has_state = false;
  int device = 0;
  // one CFL step captured as a graph (profiling off): exo_step replays it
  cudaGraphExec_t step_graph = nullptr;
  int64_t graph_launches = 0;
  // Decomposition hooks: face pressures, original pressure and density and
  // column constants between the two calls (allocated on the first call)
  double* dec_refs = nullptr;
  bool dec_done = false;
  // Redo of failed steps: budget, redos taken, the pre-step copy of u, w and
  // the clock (allocated by exo_set_max_redo)
  int max_redo = 0;
  int64_t redo_attempts = 0;
  double* redo_state = nullptr;
  exo::DevScalars* redo_sc = nullptr;
  // face-state stores of the SaveLR3DValues / LoadLR3DValues hooks: x2 L, R,
  // x3 L, R in the context's layout (allocated on first use)
  double* lr3d = nullptr;
};


// Run one launch, bracketed by events when profiling.  `nlaunch` is the
// number of kernels the launcher issues.
template <typename F>
static int timed(exo_ctx* c, int kernel, int nlaunch, F&& f) {
  ProfEvent ev;
  if (c->profiling) {
    if (c->prof_pool.empty()) {
      ProfEvent n;
      CK(cudaEventCreate(&n.a));
      CK(cudaEventCreate(&n.b));
      c->prof_pool.push_back(n);
    }
    ev = c->prof_pool.back();
    c->prof_pool.pop_back();
    ev.kernel = kernel;
    CK(cudaEventRecord(ev.a, c->stream));
  }
  int rc = f();
  if (rc) {
    cudaError_t e = cudaGetLastError();
    return cuda_fail(e == cudaSuccess ? cudaErrorUnknown : e, "kernel launch");
  }
  c->launches += nlaunch;
  if (c->profiling) {
    CK(cudaEventRecord(ev.b, c->stream));
    c->prof_used.push_back(ev);
  }
  return 0;
}

// ghost exchange + ConservedToPrimitive + x1 boundary (+ CFL candidate)
static int boundary_and_prim(exo_ctx* c, bool dt) {
  int rc;
  if (dt && (rc = timed(c, EXO_K_OTHER, 1, [&] { return STEP(launch_dt_reset, c->v, c->stream); })))
    return rc;
  return timed(c, EXO_K_PRIM_GHOST, 1,
               [&] { return STEP(launch_prim_ghost, c->v, dt, c->stream); });
}

// One stage of SSPRK(3,3) (DoTaskListOneStage): fluxes, update, implicit
// correction, boundaries and primitives (with the CFL candidate on the last
// stage unless the step is fixed).
static int one_stage(exo_ctx* c, int s, bool cfl) {
  static const char* kStage[3] = {"exo stage 0", "exo stage 1", "exo stage 2"};
  exo::Range range(kStage[s]);
  const DevView& v = c->v;
  bool shallow = v.eqn == EXO_EQN_SHALLOW_YZ;
  bool implicit = !shallow && (v.implicit_flag & 1);
  int rc;
  if (!shallow &&
      (rc = timed(c, EXO_K_FLUX_X1, 1, [&] { return STEP(launch_flux_x1, v, c->stream); })))
    return rc;
  if ((rc = timed(c, EXO_K_FLUX_X23, 1, [&] { return STEP(launch_flux_x23, v, c->stream); })))
    return rc;
  int nup = (!shallow && !implicit && s == 2) ? 2 : 1;
  if ((rc = timed(c, EXO_K_UPDATE, nup, [&] { return STEP(launch_update, v, s, c->stream); })))
    return rc;
  if (implicit && (rc = timed(c, EXO_K_IMPLICIT, exo::implicit_launches(v.implicit_flag, v.precision),
                              [&] { return STEP(launch_implicit, v, s, c->stream); })))
    return rc;
  return boundary_and_prim(c, s == 2 && cfl);
}

static int one_step(exo_ctx* c, double dt_fixed) {
  const DevView& v = c->v;
  int rc;
  if (dt_fixed > 0. &&
      (rc = timed(c, EXO_K_OTHER, 1, [&] { return STEP(launch_set_dt, v, dt_fixed, c->stream); })))
    return rc;
  for (int s = 0; s < 3; ++s)
    if ((rc = one_stage(c, s, dt_fixed <= 0.))) return rc;
  return timed(c, EXO_K_OTHER, 1,
               [&] { return STEP(launch_dt_finalize, v, dt_fixed, true, c->stream); });
}

static_assert((int)exo::BK_X1 == (int)EXO_K_FLUX_X1 && (int)exo::BK_X23 == (int)EXO_K_FLUX_X23 &&
                  (int)exo::BK_UPDATE == (int)EXO_K_UPDATE &&
                  (int)exo::BK_IMPLICIT == (int)EXO_K_IMPLICIT &&
                  (int)exo::BK_PRIM == (int)EXO_K_PRIM_GHOST &&
                  (int)exo::BK_ROUNDTRIP == (int)EXO_K_OTHER && (int)exo::BK_COUNT == EXO_TILE_COUNT,
              "tile slots follow the EXO_K_* kernel ids");

// Captures one CFL step (the launches of one_step) into a graph, once.
static int capture_step(exo_ctx* c) {
  if (c->step_graph) return 0;
  const int64_t l0 = c->launches;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = one_step(c, 0.);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    c->launches = l0;
    return rc;
  }
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
  ce = cudaGraphInstantiate(&c->step_graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    c->step_graph = nullptr;
    return cuda_fail(ce, "cudaGraphInstantiate");
  }
  c->graph_launches = c->launches - l0;
  c->launches = l0;
  return 0;
}

static void drop_step_graph(exo_ctx* c) {
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
}

namespace exo {

// the view's device copy and its one-member block table
struct SelfBlock {
  DevView view;
  unsigned start[BK_COUNT][2];
};


bool validate_config(const exo_config& c, std::string* err) {
  auto bad = [&](const char* m) { *err = m; return false; };
  if (c.eqn != EXO_EQN_SHALLOW_YZ && c.eqn != EXO_EQN_IDEAL) return bad("unknown equation set");
  bool shallow = c.eqn == EXO_EQN_SHALLOW_YZ;
  if (shallow && c.rsolver != EXO_RS_ROE_SHALLOW && c.rsolver != EXO_RS_LMARS_SHALLOW)
    return bad("shallow water needs the Roe or LMARS shallow-water solver");
  if (!shallow && c.rsolver != EXO_RS_LMARS && c.rsolver != EXO_RS_HLLC)
    return bad("the ideal gas needs the LMARS or HLLC solver");
  if (c.precision != EXO_PREC_FP64 && !mixed_build(c.precision))
    return bad("precision must be EXO_PREC_FP64, EXO_PREC_MIXED or EXO_PREC_MIXED_F32_SOLVE");
  if (!shallow && (c.implicit_flag & ~9))
    return bad("implicit_flag: only bits 1 (x1) and 8 (full 5x5 instead of partial 3x3) are supported");
  if (!(c.cfl > 0.) || !(c.gamma > 1.) || !(c.x1max > c.x1min))
    return bad("cfl, gamma or x1 range out of range");
  if (c.coriolis < EXO_CORIOLIS_NONE || c.coriolis > EXO_CORIOLIS_3D)
    return bad("unknown Coriolis source");
  if (shallow && c.coriolis == EXO_CORIOLIS_3D)
    return bad("the 3D Coriolis source needs the ideal gas");
  if (c.forcing != EXO_FORCING_NONE && c.forcing != EXO_FORCING_HS94)
    return bad("unknown forcing");
  if (c.forcing == EXO_FORCING_HS94 &&
      (shallow || !(c.hs_p0 > 0.) || !(c.hs_sigmab < 1.) || !(c.Rd > 0.)))
    return bad("HS94 forcing needs the ideal gas, hs_p0 > 0, hs_sigmab < 1 and Rd > 0");
  if (c.N < 6 || (c.N % 2) != 0) return bad("N must be even and >= 6");
  if (c.L < 1 || c.L > 250) return bad("L must be in [1, 250]");
  return true;
}

// the implicit solve's factors: 30 doubles per column level, columns in
// blocks of 32 (the last block padded)
size_t implicit_scratch_doubles(int N, int L) {
  size_t ncol = (size_t)6 * N * N;
  return (ncol + 31) / 32 * 32 * (size_t)L * 30;
}

size_t view_footprint(const exo_config& c) {
  bool shallow = c.eqn == EXO_EQN_SHALLOW_YZ;
  size_t nv = shallow ? 4 : 5;
  size_t nc1 = c.L + 2 * G, nc2 = c.N + 2 * G;
  size_t elems = 6 * nv * nc1 * nc2 * nc2;
  size_t nd = shallow ? 5 : 7;  // u, w, u1, flux x2, x3 (+ du, flux x1)
  size_t bytes = nd * elems * sizeof(double);
  if (!shallow && (c.implicit_flag & 1)) bytes += implicit_scratch_doubles(c.N, c.L) * sizeof(double);
  if (mixed_build(c.precision)) bytes += (shallow ? 3 : 4) * elems * sizeof(float);
  bytes += (size_t)NGEO2D * 6 * nc2 * nc2 * sizeof(double);       // metric
  bytes += (size_t)6 * nc2 * nc2 * sizeof(int);                   // ghost map
  bytes += (size_t)6 * 12 * c.N * sizeof(GhostEntry) + (size_t)24 * c.N * sizeof(EdgeEntry);
  bytes += 3 * (nc1 + 1) * sizeof(double) + sizeof(DevScalars);
  return bytes;
}

// Allocates and fills the device side of one atmosphere.  stream == nullptr:
// cudaMalloc; otherwise stream-ordered allocation on that stream, from `pool`
// when given (the ensemble's pool).
int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int view_allocate(const exo_config& cfg, const HostTables& t, DevView& v,
                  std::vector<void*>& owned, void* stream_v, void* pool_v, std::string* err) {
  cudaStream_t stream = (cudaStream_t)stream_v;
  cudaMemPool_t pool = (cudaMemPool_t)pool_v;
  bool shallow = cfg.eqn == EXO_EQN_SHALLOW_YZ;
  std::memset(&v, 0, sizeof(v));
  v.N = cfg.N;
  v.L = cfg.L;
  v.nv = shallow ? 4 : 5;
  v.nc1 = t.nc1;
  v.nc2 = t.nc2;
  v.nc3 = t.nc3;
  v.div_L = make_fastdiv((unsigned)v.L);
  v.div_N = make_fastdiv((unsigned)v.N);
  v.div_nc1 = make_fastdiv((unsigned)v.nc1);
  v.div_nc2 = make_fastdiv((unsigned)v.nc2);
  v.div_nc3 = make_fastdiv((unsigned)v.nc3);
  v.is = v.js = v.ks = G;
  v.ie = G + cfg.L - 1;
  v.je = v.ke = G + cfg.N - 1;
  v.eqn = cfg.eqn;
  v.rsolver = cfg.rsolver;
  v.implicit_flag = shallow ? 0 : cfg.implicit_flag;
  v.coriolis = cfg.coriolis;
  v.precision = cfg.precision;
  v.forcing = shallow ? EXO_FORCING_NONE : cfg.forcing;
  if (v.forcing == EXO_FORCING_HS94) {
    // Mesh::InitUserMeshData (hs94.cpp:212-243): cp from gamma, rates per day
    const double day_to_s = 8.64E4;
    const double cp = cfg.gamma / (cfg.gamma - 1.) * cfg.Rd;
    v.hs[HS_P0] = cfg.hs_p0;
    v.hs[HS_TS] = cfg.hs_Ts;
    v.hs[HS_DT] = cfg.hs_dT;
    v.hs[HS_DTHETA] = cfg.hs_dtheta;
    v.hs[HS_KF] = cfg.hs_Kf / day_to_s;
    v.hs[HS_KA] = cfg.hs_Ka / day_to_s;
    v.hs[HS_KS] = cfg.hs_Ks / day_to_s;
    v.hs[HS_SIGMAB] = cfg.hs_sigmab;
    v.hs[HS_KAPPA] = cfg.Rd / cp;
    v.hs[HS_CVM] = cp - cfg.Rd;
  }
  v.gamma = cfg.gamma;
  v.Rd = cfg.Rd;
  v.grav = shallow ? 0. : cfg.grav;
  v.cfl = cfg.cfl;
  v.cells = (size_t)t.nc3 * t.nc2 * t.nc1;
  size_t elems = (size_t)6 * v.nv * v.cells;
  auto alloc = [&](void** p, size_t bytes, bool zero) -> bool {
    cudaError_t e = stream ? (pool ? cudaMallocFromPoolAsync(p, bytes, pool, stream)
                                   : cudaMallocAsync(p, bytes, stream))
                           : cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
      *err = std::string("device allocation: ") + cudaGetErrorString(e);
      return false;
    }
    owned.push_back(*p);
    if (zero) {
      e = stream ? cudaMemsetAsync(*p, 0, bytes, stream) : cudaMemset(*p, 0, bytes);
      if (e != cudaSuccess) {
        *err = std::string("cudaMemset: ") + cudaGetErrorString(e);
        return false;
      }
    }
    return true;
  };
  auto put = [&](void** p, const void* src, size_t bytes) -> bool {
    if (!alloc(p, bytes ? bytes : 8, false)) return false;
    if (!bytes) return true;
    cudaError_t e = stream ? cudaMemcpyAsync(*p, src, bytes, cudaMemcpyHostToDevice, stream)
                           : cudaMemcpy(*p, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      *err = std::string("table upload: ") + cudaGetErrorString(e);
      return false;
    }
    return true;
  };
  size_t db = elems * sizeof(double), fb = elems * sizeof(float);
  if (!alloc((void**)&v.u, db, true) || !alloc((void**)&v.w, db, true) ||
      !alloc((void**)&v.u1, db, true) || !alloc((void**)&v.flux[1], db, true) ||
      !alloc((void**)&v.flux[2], db, true))
    return EXO_ERR_CAPACITY;
  if (!shallow) {
    if (!alloc((void**)&v.du, db, true) || !alloc((void**)&v.flux[0], db, true))
      return EXO_ERR_CAPACITY;
    if ((v.implicit_flag & 1) &&
        !alloc((void**)&v.scratch, implicit_scratch_doubles(cfg.N, cfg.L) * sizeof(double), false))
      return EXO_ERR_CAPACITY;
  }
  if (mixed_build(cfg.precision)) {
    if (!alloc((void**)&v.w32, fb, true) || !alloc((void**)&v.flux32[1], fb, true) ||
        !alloc((void**)&v.flux32[2], fb, true))
      return EXO_ERR_CAPACITY;
    if (!shallow && !alloc((void**)&v.flux32[0], fb, true)) return EXO_ERR_CAPACITY;
  }
  void *x1f, *x1v, *dx1f, *geo, *gmap, *gh, *ed;
  if (!put(&x1f, t.x1f.data(), t.x1f.size() * sizeof(double)) ||
      !put(&x1v, t.x1v.data(), t.x1v.size() * sizeof(double)) ||
      !put(&dx1f, t.dx1f.data(), t.dx1f.size() * sizeof(double)) ||
      !put(&geo, t.geo.data(), t.geo.size() * sizeof(double)) ||
      !put(&gmap, t.ghost_map.data(), t.ghost_map.size() * sizeof(int)) ||
      !put(&gh, t.ghost.data(), t.ghost.size() * sizeof(GhostEntry)) ||
      !put(&ed, t.edge.data(), t.edge.size() * sizeof(EdgeEntry)))
    return EXO_ERR_CAPACITY;
  v.x1f = (const double*)x1f;
  v.x1v = (const double*)x1v;
  v.dx1f = (const double*)dx1f;
  v.geo = (const double*)geo;
  v.ghost_map = (const int*)gmap;
  v.ghost = (const GhostEntry*)gh;
  v.edge = (const EdgeEntry*)ed;
  if (!alloc((void**)&v.sc, sizeof(DevScalars), true)) return EXO_ERR_CAPACITY;
  // the view's own device copy and its one-member block table: the stepping
  // kernels are the batched ones, launched on a batch of one, so an
  // atmosphere runs the same machine code alone as in an ensemble
  SelfBlock* dself = nullptr;
  if (!alloc((void**)&dself, sizeof(SelfBlock), false)) return EXO_ERR_CAPACITY;
  v.self = &dself->view;
  v.starts = &dself->start[0][0];
  Tiles dt = default_tiles();
  for (int k = 0; k < BK_COUNT; ++k) v.tiles[k] = dt.t[k];
  // tables must stay alive until the (possibly asynchronous) uploads finish
  cudaError_t e = stream ? cudaStreamSynchronize(stream) : cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    *err = std::string("upload: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  return view_refresh_self(v, stream, err);
}

void view_free(std::vector<void*>& owned, void* stream_v) {
  cudaStream_t stream = (cudaStream_t)stream_v;
  for (void* p : owned) {
    if (stream) cudaFreeAsync(p, stream);
    else cudaFree(p);
  }
  owned.clear();
}

Tiles default_tiles() {
  Tiles t;
  t.t[BK_X1] = 4;  // radial columns per block
  t.t[BK_X23] = 128;
  t.t[BK_UPDATE] = 128;
  t.t[BK_IMPLICIT] = 64;
  t.t[BK_PRIM] = 256;
  t.t[BK_ROUNDTRIP] = 128;
  return t;
}

bool valid_tiles(const int* t, std::string* err) {
  for (int k = 0; k < BK_COUNT; ++k) {
    bool ok = t[k] >= 32 && t[k] <= 512 && t[k] % 32 == 0;
    if (k == BK_X1) ok = t[k] >= 1 && t[k] <= X1_MAX_COLUMNS;
    if (k == BK_IMPLICIT) ok = t[k] == 32 || t[k] == 64 || t[k] == 128;
    if (!ok) {
      *err = "tile " + std::to_string(k) + " = " + std::to_string(t[k]) +
             ": threads per block must be a multiple of 32 in [32, 512] (implicit: 32, 64, "
             "128; x1: columns per block, 1 to " + std::to_string(X1_MAX_COLUMNS) + ")";
      return false;
    }
  }
  return true;
}

void member_blocks(const DevView& v, const int* t, unsigned b[BK_COUNT]) {
  bool shallow = v.eqn == EXO_EQN_SHALLOW_YZ;
  bool implicit = !shallow && (v.implicit_flag & 1);
  auto nb = [](size_t n, int th) { return (unsigned)((n + th - 1) / th); };
  b[BK_X1] = shallow ? 0u : nb((size_t)6 * v.N * v.N, t[BK_X1]);  // t[BK_X1] columns per block
  // tiles of faces, or one thread per line of faces or per face, as the build chose
  b[BK_X23] = mixed_build(v.precision) ? mixed::x23_blocks(v, t[BK_X23])
                                        : fp64::x23_blocks(v, t[BK_X23]);
  b[BK_UPDATE] = nb((size_t)6 * v.N * v.N * v.L, t[BK_UPDATE]);
  b[BK_IMPLICIT] = implicit ? nb((size_t)6 * v.N * v.N, t[BK_IMPLICIT]) : 0u;  // thread per column
  b[BK_PRIM] = nb((size_t)6 * v.cells, t[BK_PRIM]);
  b[BK_ROUNDTRIP] = (!shallow && !implicit) ? nb((size_t)6 * v.N * v.N * v.L, t[BK_ROUNDTRIP]) : 0u;
}

int view_refresh_self(DevView& v, void* stream_v, std::string* err) {
  cudaStream_t stream = (cudaStream_t)stream_v;
  SelfBlock h;
  std::memset(&h, 0, sizeof(h));
  h.view = v;
  unsigned b[BK_COUNT];
  member_blocks(v, v.tiles, b);
  for (int k = 0; k < BK_COUNT; ++k) h.start[k][1] = b[k];
  SelfBlock* d = (SelfBlock*)const_cast<DevView*>(v.self);
  cudaError_t e = stream ? cudaMemcpyAsync(d, &h, sizeof(h), cudaMemcpyHostToDevice, stream)
                         : cudaMemcpy(d, &h, sizeof(h), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && stream) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    *err = std::string("view upload: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  return 0;
}

}  // namespace exo

extern "C" {

const char* exo_last_error(void) { return g_err.c_str(); }

int exo_config_default(exo_config* cfg, int eqn) {
  if (!cfg) return fail(EXO_ERR_ARG, "cfg is NULL");
  std::memset(cfg, 0, sizeof(*cfg));
  if (eqn == EXO_EQN_SHALLOW_YZ) {
    // exo2 shallow water: examples/2023-Chen-exo3/W92.inp
    cfg->N = 48;
    cfg->L = 3;
    cfg->eqn = EXO_EQN_SHALLOW_YZ;
    cfg->rsolver = EXO_RS_ROE_SHALLOW;
    cfg->implicit_flag = 0;
    cfg->coriolis = EXO_CORIOLIS_W92;
    cfg->x1min = 6371000.;
    cfg->x1max = 6371001.;
    cfg->gamma = 1.4;
    cfg->Rd = 287.;
    cfg->grav = 0.;
    cfg->cfl = 0.4;
    cfg->omega = 7.292e-5;
  } else if (eqn == EXO_EQN_IDEAL) {
    // exo3 dry ideal gas: 96^2 x 64, LMARS, implicit_flag 9
    cfg->N = 96;
    cfg->L = 64;
    cfg->eqn = EXO_EQN_IDEAL;
    cfg->rsolver = EXO_RS_LMARS;
    cfg->implicit_flag = 9;
    cfg->coriolis = EXO_CORIOLIS_NONE;
    cfg->gamma = 1.4;
    cfg->Rd = 287.;
    cfg->grav = -9.81;
    cfg->x1min = 6.371e6;
    cfg->x1max = 6.371e6 + 287. * 250. / 9.81 * 4.605170185988092;  // 1e5 -> 1e3 Pa
    cfg->cfl = 0.4;
    cfg->omega = 0.;
  } else {
    return fail(EXO_ERR_ARG, "unknown equation set");
  }
  // Held-Suarez parameters of examples/2023-Chen-exo3/hs94.inp (used only
  // with forcing = EXO_FORCING_HS94)
  cfg->forcing = EXO_FORCING_NONE;
  cfg->hs_p0 = 1.E5;
  cfg->hs_Ts = 315.;
  cfg->hs_dT = 60.;
  cfg->hs_dtheta = 10.;
  cfg->hs_Kf = 1.;
  cfg->hs_Ka = 0.025;
  cfg->hs_Ks = 0.25;
  cfg->hs_sigmab = 0.7;
  return EXO_OK;
}

int exo_create(const exo_config* cfg, exo_ctx** out) {
  if (!cfg || !out) return fail(EXO_ERR_ARG, "NULL argument");
  *out = nullptr;
  {
    std::string verr;
    if (!exo::validate_config(*cfg, &verr)) return fail(EXO_ERR_ARG, verr);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(EXO_ERR_NOGPU, "no CUDA device");

  exo_ctx* c = new exo_ctx();
  c->cfg = *cfg;
  std::string err;
  if (!exo::build_tables(*cfg, c->tab, &err)) {
    delete c;
    return fail(EXO_ERR_ARG, err);
  }
  cudaGetDevice(&c->device);
  if (exo::fp64::prepare_kernels() || exo::mixed::prepare_kernels()) {
    delete c;
    return fail(EXO_ERR_CUDA, "kernel attributes could not be set");
  }
  auto cleanup = [&](int rc) {
    for (void* p : c->owned) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return rc;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(EXO_ERR_CUDA, "cudaStreamCreate failed"));

  std::string aerr;
  int rc = exo::view_allocate(*cfg, c->tab, c->v, c->owned, nullptr, nullptr, &aerr);
  if (rc) return cleanup(fail(rc, aerr));
  c->state_elems = (size_t)6 * c->v.nv * c->v.cells;
  cudaError_t e;
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "exo_create"));
  *out = c;
  return EXO_OK;
}

void exo_destroy(exo_ctx* c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  drop_step_graph(c);
  for (auto& e : c->prof_used) c->prof_pool.push_back(e);
  for (auto& e : c->prof_pool) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  for (void* p : c->owned) cudaFree(p);
  if (c->dec_refs) cudaFree(c->dec_refs);
  cudaStreamDestroy(c->stream);
  cudaSetDevice(prev);
  delete c;
}

int exo_cell_geometry(const exo_config* cfg, double* lat, double* lon, double* uv_to_v23,
                      double* x1v) {
  if (!cfg) return fail(EXO_ERR_ARG, "cfg is NULL");
  exo::HostTables t;
  std::string err;
  if (!exo::build_tables(*cfg, t, &err)) return fail(EXO_ERR_ARG, err);
  int N = cfg->N;
  for (int p = 0; p < 6; ++p)
    for (int k = 0; k < N; ++k)
      for (int j = 0; j < N; ++j) {
        size_t q = ((size_t)p * N + k) * N + j;
        double dX = tan(t.x2v[p][exo::G + j]), dY = tan(t.x3v[p][exo::G + k]);
        double la, lo;
        exo::rll_from_xyp(dY, -dX, p, lo, la);
        if (lat) lat[q] = la;
        if (lon) lon[q] = 2.0 * 3.1415926535897932 - lo;
        if (uv_to_v23) {
          double c[4];
          exo::abp_from_rll_coef(dX, dY, p + 1, c);
          uv_to_v23[4 * q + 0] = -c[0];
          uv_to_v23[4 * q + 1] = c[1];
          uv_to_v23[4 * q + 2] = -c[2];
          uv_to_v23[4 * q + 3] = c[3];
        }
      }
  if (x1v)
    for (int i = 0; i < cfg->L; ++i) x1v[i] = t.x1v[exo::G + i];
  return EXO_OK;
}

int exo_mesh(const exo_config* cfg, int panel, double* x1f, double* x2f, double* x3f) {
  if (!cfg) return fail(EXO_ERR_ARG, "cfg is NULL");
  if (panel < 0 || panel > 5) return fail(EXO_ERR_ARG, "panel must be 0..5");
  exo::HostTables t;
  std::string err;
  if (!exo::build_tables(*cfg, t, &err)) return fail(EXO_ERR_ARG, err);
  if (x1f) std::memcpy(x1f, t.x1f.data(), t.x1f.size() * sizeof(double));
  if (x2f) std::memcpy(x2f, t.x2f[panel].data(), t.x2f[panel].size() * sizeof(double));
  if (x3f) std::memcpy(x3f, t.x3f[panel].data(), t.x3f[panel].size() * sizeof(double));
  return EXO_OK;
}

int exo_shape(const exo_ctx* c, int* nvar, int* nc3, int* nc2, int* nc1) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (nvar) *nvar = c->v.nv;
  if (nc3) *nc3 = c->v.nc3;
  if (nc2) *nc2 = c->v.nc2;
  if (nc1) *nc1 = c->v.nc1;
  return EXO_OK;
}

int exo_set_primitive(exo_ctx* c, const double* w_host) {
  if (!c || !w_host) return fail(EXO_ERR_ARG, "NULL argument");
  size_t bytes = c->state_elems * sizeof(double);
  // stage through the w array, then P2C of the interior into u
  CK(cudaMemcpyAsync(c->v.w, w_host, bytes, cudaMemcpyHostToDevice, c->stream));
  RK(STEP(launch_p2c_interior, c->v, c->v.w, c->stream));
  int rc = boundary_and_prim(c, true);
  if (rc) return rc;
  RK(STEP(launch_dt_finalize, c->v, 0., false, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->has_state = true;
  return EXO_OK;
}

int exo_get_conserved(exo_ctx* c, double* u_host) {
  if (!c || !u_host) return fail(EXO_ERR_ARG, "NULL argument");
  CK(cudaMemcpyAsync(u_host, c->v.u, c->state_elems * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_get_primitive(exo_ctx* c, double* w_host) {
  if (!c || !w_host) return fail(EXO_ERR_ARG, "NULL argument");
  CK(cudaMemcpyAsync(w_host, c->v.w, c->state_elems * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_device_state(exo_ctx* c, double** u_dev, double** w_dev) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (u_dev) *u_dev = c->v.u;
  if (w_dev) *w_dev = c->v.w;
  return EXO_OK;
}

// One step: the captured CFL graph, or the launches of one_step when
// profiling or with a fixed dt.
static int step_once(exo_ctx* c, double dt_fixed) {
  if (!c->profiling && dt_fixed <= 0.) {
    int rc = capture_step(c);
    if (rc) return rc;
    CK(cudaGraphLaunch(c->step_graph, c->stream));
    c->launches += c->graph_launches;
    return EXO_OK;
  }
  return one_step(c, dt_fixed);
}

static int read_scalars(exo_ctx* c, const exo::DevScalars* src, exo::DevScalars* s) {
  CK(cudaMemcpyAsync(s, src, sizeof(*s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

// copy u, w, the FP32 primitive copy w32 (mixed builds: the flux kernels of
// the next stage read it) and the clock: to the redo copy (save) or back
// (!save)
static int redo_copy(exo_ctx* c, bool save) {
  const size_t b = c->state_elems * sizeof(double);
  double* keep_u = c->redo_state;
  double* keep_w = c->redo_state + c->state_elems;
  float* keep_w32 = reinterpret_cast<float*>(c->redo_state + 2 * c->state_elems);
  const size_t b32 = c->state_elems * sizeof(float);
  auto cp = [&](void* dst, const void* src, size_t n) {
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, c->stream);
  };
  if (save) {
    CK(cp(keep_u, c->v.u, b));
    CK(cp(keep_w, c->v.w, b));
    if (c->v.w32) CK(cp(keep_w32, c->v.w32, b32));
    CK(cp(c->redo_sc, c->v.sc, sizeof(exo::DevScalars)));
  } else {
    CK(cp(c->v.u, keep_u, b));
    CK(cp(c->v.w, keep_w, b));
    if (c->v.w32) CK(cp(c->v.w32, keep_w32, b32));
    CK(cp(c->v.sc, c->redo_sc, sizeof(exo::DevScalars)));
  }
  return EXO_OK;
}

// The main loop's redo (main.cpp.in:126-157, mesh_redo.cpp:12-46): keep the
// state, take the step, and while the state came out invalid put the kept
// state back and take the step again with half the time step.  The budget
// counts redos over the whole run, `attempts++ > max_redo` as there.
static int step_with_redo(exo_ctx* c, double dt_fixed) {
  exo::DevScalars s;
  int rc = read_scalars(c, c->v.sc, &s);
  if (rc) return rc;
  if (s.invalid) return fail(EXO_ERR_NONFINITE, "the state is invalid before the step");
  if ((rc = redo_copy(c, true))) return rc;
  // the step in use: the fixed one, or the CFL step the previous step chose
  double dt_step = dt_fixed > 0. ? dt_fixed : s.dt;
  if ((rc = step_once(c, dt_fixed))) return rc;
  if ((rc = read_scalars(c, c->v.sc, &s))) return rc;
  while (s.invalid) {
    exo::Range redo("exo redo");
    // LoadAllStates (the kept copy holds the pre-step clock), DecreaseTimeStep
    if ((rc = redo_copy(c, false))) return rc;
    dt_step *= 0.5;
    if (dt_fixed <= 0.) RK(STEP(launch_set_dt, c->v, dt_step, c->stream));
    if (c->redo_attempts++ > c->max_redo)
      return fail(EXO_ERR_NONFINITE, "too many attempts to redo the step");
    if ((rc = step_once(c, dt_fixed > 0. ? dt_step : 0.))) return rc;
    if ((rc = read_scalars(c, c->v.sc, &s))) return rc;
  }
  return EXO_OK;
}

int exo_set_max_redo(exo_ctx* c, int max_redo) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (max_redo < 0) return fail(EXO_ERR_ARG, "max_redo < 0");
  if (max_redo > 0 && !c->redo_state) {
    // u and w, then room for w32 (half a double array) when the build keeps one
    size_t words = 2 * c->state_elems + (c->v.w32 ? (c->state_elems + 1) / 2 : 0);
    CK(cudaMalloc((void**)&c->redo_state, words * sizeof(double)));
    c->owned.push_back(c->redo_state);
    CK(cudaMalloc((void**)&c->redo_sc, sizeof(exo::DevScalars)));
    c->owned.push_back(c->redo_sc);
  }
  c->max_redo = max_redo;
  return EXO_OK;
}

int exo_redo_count(exo_ctx* c, int64_t* redos) {
  if (!c || !redos) return fail(EXO_ERR_ARG, "NULL argument");
  *redos = c->redo_attempts;
  return EXO_OK;
}

int exo_step(exo_ctx* c, int nsteps, double dt_fixed) {
  exo::Range range("exo_step");
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (!c->has_state) return fail(EXO_ERR_ARG, "no state loaded (exo_set_primitive)");
  if (nsteps < 0) return fail(EXO_ERR_ARG, "nsteps < 0");
  if (c->max_redo > 0) {
    for (int n = 0; n < nsteps; ++n) {
      int rc = step_with_redo(c, dt_fixed);
      if (rc) return rc;
    }
    return EXO_OK;
  }
  if (!c->profiling && dt_fixed <= 0. && nsteps > 0) {
    // the CFL step is replayed from its graph: one launch per step on the host
    int rc = capture_step(c);
    if (rc) return rc;
    for (int n = 0; n < nsteps; ++n) CK(cudaGraphLaunch(c->step_graph, c->stream));
    c->launches += (int64_t)nsteps * c->graph_launches;
    return EXO_OK;
  }
  for (int n = 0; n < nsteps; ++n) {
    int rc = one_step(c, dt_fixed);
    if (rc) return rc;
  }
  return EXO_OK;
}

int exo_stage(exo_ctx* c, int stage) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (!c->has_state) return fail(EXO_ERR_ARG, "no state loaded (exo_set_primitive)");
  if (stage < 0 || stage > 2) return fail(EXO_ERR_ARG, "stage must be 0, 1 or 2");
  int rc = one_stage(c, stage, true);
  if (rc) return fail(rc, "stage launch failed");
  if (stage == 2) {
    rc = timed(c, EXO_K_OTHER, 1, [&] { return STEP(launch_dt_finalize, c->v, 0., true, c->stream); });
    if (rc) return fail(rc, "time-step launch failed");
  }
  return EXO_OK;
}

int exo_boundary(exo_ctx* c) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = boundary_and_prim(c, false);
  return rc ? fail(rc, "boundary launch failed") : EXO_OK;
}

int exo_change_to_perturbation(exo_ctx* c, double* w_host) {
  if (!c || !w_host) return fail(EXO_ERR_ARG, "NULL argument");
  if (c->v.eqn == EXO_EQN_SHALLOW_YZ)
    return fail(EXO_ERR_ARG, "the decomposition applies to the ideal gas (exo3)");
  if (c->v.grav == 0.) return EXO_OK;  // no gravity: nothing is decomposed
  if (!c->dec_refs) {
    CK(cudaMalloc((void**)&c->dec_refs, exo::decomposition_refs_doubles(c->v) * sizeof(double)));
  }
  size_t bytes = c->state_elems * sizeof(double);
  CK(cudaMemcpyAsync(c->v.w, w_host, bytes, cudaMemcpyHostToDevice, c->stream));
  int rc = exo::launch_change_to_perturbation(c->v, c->v.w, c->dec_refs, c->stream);
  if (rc) return fail(rc, "decomposition launch failed");
  CK(cudaMemcpyAsync(w_host, c->v.w, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->dec_done = true;
  return EXO_OK;
}

int exo_restore_from_perturbation(exo_ctx* c, double* w_host, double* wl_host, double* wr_host) {
  if (!c || !w_host || !wl_host || !wr_host) return fail(EXO_ERR_ARG, "NULL argument");
  if (c->v.eqn == EXO_EQN_SHALLOW_YZ)
    return fail(EXO_ERR_ARG, "the decomposition applies to the ideal gas (exo3)");
  if (c->v.grav == 0.) return EXO_OK;
  if (!c->dec_done) return fail(EXO_ERR_ARG, "no exo_change_to_perturbation before the restore");
  size_t bytes = c->state_elems * sizeof(double);
  double* wl = c->v.flux[1];  // staging: the context's x2/x3 flux arrays (same layout)
  double* wr = c->v.flux[2];
  CK(cudaMemcpyAsync(c->v.w, w_host, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(wl, wl_host, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(wr, wr_host, bytes, cudaMemcpyHostToDevice, c->stream));
  int rc = exo::launch_restore_from_perturbation(c->v, c->v.w, wl, wr, c->dec_refs, c->stream);
  if (rc) return fail(rc, "restore launch failed");
  CK(cudaMemcpyAsync(w_host, c->v.w, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(wl_host, wl, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(wr_host, wr, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_solve_implicit_3d(exo_ctx* c, double* du_host, const double* w_host, double dt) {
  if (!c || !du_host || !w_host) return fail(EXO_ERR_ARG, "NULL argument");
  if (c->v.eqn == EXO_EQN_SHALLOW_YZ || !(c->v.implicit_flag & 1))
    return fail(EXO_ERR_ARG, "the context has no implicit x1 solve (ideal gas, implicit_flag 1 or 9)");
  if (!(dt > 0.)) return fail(EXO_ERR_ARG, "dt must be positive");
  size_t bytes = c->state_elems * sizeof(double);
  CK(cudaMemcpyAsync(c->v.w, w_host, bytes, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->v.du, du_host, bytes, cudaMemcpyHostToDevice, c->stream));
  int rc = timed(c, EXO_K_IMPLICIT, exo::implicit_launches(c->v.implicit_flag, c->v.precision),
                 [&] { return STEP(launch_implicit_du, c->v, dt, c->stream); });
  if (rc) return fail(rc, "implicit launch failed");
  CK(cudaMemcpyAsync(du_host, c->v.du, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_checkpoint_bytes(const exo_ctx* c, size_t* bytes) {
  if (!c || !bytes) return fail(EXO_ERR_ARG, "NULL argument");
  *bytes = exo::checkpoint_bytes(c->v);
  return EXO_OK;
}

int exo_checkpoint_save(exo_ctx* c, void* image, size_t bytes) {
  exo::Range range("exo_checkpoint_save");
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (!c->has_state) return fail(EXO_ERR_ARG, "no state loaded (exo_set_primitive)");
  std::string err;
  int rc = exo::checkpoint_save(c->cfg, c->v, c->stream, image, bytes, &err);
  return rc ? fail(rc, err) : EXO_OK;
}

int exo_checkpoint_load(exo_ctx* c, const void* image, size_t bytes) {
  exo::Range range("exo_checkpoint_load");
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  exo_checkpoint_header h;
  std::string err;
  int rc = exo::checkpoint_parse(image, bytes, &h, &err);
  if (rc) return fail(rc, err);
  if (!exo::same_config_but_precision(h.cfg, c->cfg))
    return fail(EXO_ERR_ARG, "the checkpoint was written with another configuration");
  CK(cudaStreamSynchronize(c->stream));
  rc = exo::checkpoint_restore(c->v, c->stream, image, &err);
  if (rc) return fail(rc, err);
  // the primitives (and their FP32 copy in the mixed build) from u, as the
  // end of every step computes them
  rc = boundary_and_prim(c, false);
  if (rc) return fail(rc, "recomputing the primitives failed");
  CK(cudaStreamSynchronize(c->stream));
  c->has_state = true;
  return EXO_OK;
}

int exo_get_dt(exo_ctx* c, double* dt) {
  if (!c || !dt) return fail(EXO_ERR_ARG, "NULL argument");
  DevScalars s;
  CK(cudaMemcpyAsync(&s, c->v.sc, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *dt = s.dt;
  return EXO_OK;
}

int exo_get_time(exo_ctx* c, double* time, int64_t* ncycle) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  DevScalars s;
  CK(cudaMemcpyAsync(&s, c->v.sc, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (time) *time = s.time;
  if (ncycle) *ncycle = s.ncycle;
  return EXO_OK;
}

int exo_set_tiles(exo_ctx* c, const int* threads) {
  if (!c || !threads) return fail(EXO_ERR_ARG, "NULL argument");
  int t[exo::BK_COUNT];
  for (int k = 0; k < exo::BK_COUNT; ++k) t[k] = threads[k] > 0 ? threads[k] : c->v.tiles[k];
  std::string err;
  if (!exo::valid_tiles(t, &err)) return fail(EXO_ERR_ARG, err);
  CK(cudaStreamSynchronize(c->stream));  // launches already queued keep their tables
  drop_step_graph(c);                     // it holds the old launch shapes
  for (int k = 0; k < exo::BK_COUNT; ++k) c->v.tiles[k] = t[k];
  int rc = exo::view_refresh_self(c->v, c->stream, &err);
  return rc ? fail(rc, err) : EXO_OK;
}

int exo_get_tiles(exo_ctx* c, int* threads) {
  if (!c || !threads) return fail(EXO_ERR_ARG, "NULL argument");
  for (int k = 0; k < exo::BK_COUNT; ++k) threads[k] = c->v.tiles[k];
  return EXO_OK;
}

int exo_check_state(exo_ctx* c, int* invalid) {
  if (!c || !invalid) return fail(EXO_ERR_ARG, "NULL argument");
  DevScalars s;
  CK(cudaMemcpyAsync(&s, c->v.sc, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *invalid = s.invalid;
  int zero = 0;
  CK(cudaMemcpyAsync(&c->v.sc->invalid, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (s.timeout) return fail(EXO_ERR_TIMEOUT, "a kernel's bounded wait for its bulk copies gave up");
  return EXO_OK;
}

int exo_synchronize(exo_ctx* c) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_get_stream(exo_ctx* c, void** stream) {
  if (!c || !stream) return fail(EXO_ERR_ARG, "NULL argument");
  *stream = (void*)c->stream;
  return EXO_OK;
}

int exo_profile(exo_ctx* c, int enable) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  CK(cudaStreamSynchronize(c->stream));
  for (auto& e : c->prof_used) c->prof_pool.push_back(e);
  c->prof_used.clear();
  c->profiling = enable != 0;
  return EXO_OK;
}

int exo_profile_read(exo_ctx* c, int kernel, int64_t* launches, double* total_ms) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (kernel < 0 || kernel >= EXO_K_COUNT) return fail(EXO_ERR_ARG, "unknown kernel id");
  CK(cudaStreamSynchronize(c->stream));
  int64_t n = 0;
  double ms = 0.;
  for (auto& e : c->prof_used) {
    if (e.kernel != kernel) continue;
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e.a, e.b));
    ms += t;
    ++n;
  }
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return EXO_OK;
}

int exo_launch_count(exo_ctx* c, int64_t* launches) {
  if (!c || !launches) return fail(EXO_ERR_ARG, "NULL argument");
  *launches = c->launches;
  return EXO_OK;
}

int exo_calculate_fluxes(exo_ctx* c) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  if (!c->has_state) return fail(EXO_ERR_ARG, "no state loaded (exo_set_primitive)");
  RK(STEP(launch_flux_x1, c->v, c->stream));
  RK(STEP(launch_flux_x23, c->v, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_get_flux(exo_ctx* c, int dir, double* flux_host) {
  if (!c || !flux_host) return fail(EXO_ERR_ARG, "NULL argument");
  if (dir < 0 || dir > 2) return fail(EXO_ERR_ARG, "dir must be 0, 1 or 2");
  size_t bytes = c->state_elems * sizeof(double);
  if (!c->v.flux[dir]) {
    std::memset(flux_host, 0, bytes);
    return EXO_OK;
  }
  CK(cudaMemcpyAsync(flux_host, c->v.flux[dir], bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EXO_OK;
}

int exo_riemann(int rsolver, int eqn, int ivx, int n, double gamma, const double* wl,
                const double* wr, double* flx, const double* cos_face, const double* sin_face,
                const double* cth_proj, const double* cth_cell, void* stream) {
  if (n < 0 || !wl || !wr || !flx) return fail(EXO_ERR_ARG, "bad argument");
  if (ivx < exo::IVX || ivx > exo::IVZ) return fail(EXO_ERR_ARG, "ivx must be 1, 2 or 3");
  if (rsolver < EXO_RS_ROE_SHALLOW || rsolver > EXO_RS_LMARS_SHALLOW)
    return fail(EXO_ERR_ARG, "unknown Riemann solver");
  RK(exo::launch_riemann_rows(rsolver, eqn, ivx, n, gamma, wl, wr, flx, cos_face, sin_face,
                              cth_proj, cth_cell, stream));
  return EXO_OK;
}

int exo_implicit_columns(int ncol, int L, const double* w, double* du, const double* colgeo,
                         const double* x1f, const double* x1v, const double* dx1f, double dt,
                         double gamma, double grav, double* scratch, void* stream) {
  if (ncol < 0 || L < 1) return fail(EXO_ERR_ARG, "ncol must be >= 0 and L >= 1");
  if (ncol == 0) return EXO_OK;
  if (!w || !du || !colgeo || !x1f || !x1v || !dx1f || !scratch)
    return fail(EXO_ERR_ARG, "NULL array");
  if (!(dt > 0.) || !(gamma > 1.)) return fail(EXO_ERR_ARG, "dt must be > 0 and gamma > 1");
  RK(exo::launch_implicit_columns(ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav,
                                  scratch, stream, 1));
  return EXO_OK;
}

int exo_partial_correction_columns(int ncol, int L, const double* w, double* du,
                                   const double* colgeo, const double* x1f, const double* x1v,
                                   const double* dx1f, double dt, double gamma, double grav,
                                   double* scratch, void* stream) {
  if (ncol < 0 || L < 1) return fail(EXO_ERR_ARG, "ncol must be >= 0 and L >= 1");
  if (ncol == 0) return EXO_OK;
  if (!w || !du || !colgeo || !x1f || !x1v || !dx1f || !scratch)
    return fail(EXO_ERR_ARG, "NULL array");
  if (!(dt > 0.) || !(gamma > 1.)) return fail(EXO_ERR_ARG, "dt must be > 0 and gamma > 1");
  RK(exo::launch_implicit_columns(ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav,
                                  scratch, stream, 0));
  return EXO_OK;
}

int exo_implicit_columns_noalloc(int ncol, int L, const double* w, double* du,
                                 const double* colgeo, const double* x1f, const double* x1v,
                                 const double* dx1f, double dt, double gamma, double grav,
                                 void* stream) {
  if (ncol < 0 || L < 1) return fail(EXO_ERR_ARG, "ncol must be >= 0 and L >= 1");
  if (ncol > 0 && (!w || !du || !colgeo || !x1f || !x1v || !dx1f))
    return fail(EXO_ERR_ARG, "NULL array");
  if (!(dt > 0.) || !(gamma > 1.)) return fail(EXO_ERR_ARG, "dt must be > 0 and gamma > 1");
  std::string err;
  int rc = exo::launch_implicit_columns_noalloc(ncol, L, w, du, colgeo, x1f, x1v, dx1f, dt, gamma,
                                                grav, stream, &err);
  if (rc) return fail(rc, err);
  return EXO_OK;
}

int exo_check_bounded_wait(int* gave_up, double* waited_ms) {
  if (!gave_up || !waited_ms) return fail(EXO_ERR_ARG, "NULL argument");
  std::string err;
  int rc = exo::bounded_wait_selftest(gave_up, waited_ms, &err);
  if (rc) return fail(rc, err);
  return EXO_OK;
}

int exo_measure_fma_peak(int fp64, int repeats, double* flops_per_s) {
  if (!flops_per_s || repeats < 1) return fail(EXO_ERR_ARG, "flops_per_s NULL or repeats < 1");
  std::string err;
  int rc = exo::measure_fma_peak(fp64 != 0, repeats, flops_per_s, &err);
  if (rc) return fail(rc, err);
  return EXO_OK;
}

// ------------------------------------------------- panel-exchange hooks ----
static cudaStream_t hook_stream(exo_ctx* c, void* stream) {
  return stream ? (cudaStream_t)stream : c->stream;
}

int exo_panel_pack(exo_ctx* c, const double* src, double* buf, int sn, int en, int si, int ei,
                   int sj, int ej, int sk, int ek, int* offset, int ox1, int ox2, int ox3,
                   int panel, void* stream) {
  if (!c || !src || !buf || !offset) return fail(EXO_ERR_ARG, "NULL argument");
  const DevView& v = c->v;
  if (panel < 0 || panel > 5) return fail(EXO_ERR_ARG, "panel must be 0..5");
  if (sn < 0 || en >= v.nv || sn > en || si < 0 || ei >= v.nc1 || si > ei || sj < 0 ||
      ej >= v.nc2 || sj > ej || sk < 0 || ek >= v.nc3 || sk > ek)
    return fail(EXO_ERR_SHAPE, "index range outside the panel array");
  cudaStream_t st = hook_stream(c, stream);
  const bool face = ox1 == 0 && ((ox2 != 0) != (ox3 != 0));
  if (!face) {
    // corners and radial neighbours: PackDataR0, a plain copy of the range
    const int64_t ss[4] = {(int64_t)v.nc3 * v.nc2 * v.nc1, (int64_t)v.nc2 * v.nc1, v.nc1, 1};
    const int size[4] = {en - sn + 1, ek - sk + 1, ej - sj + 1, ei - si + 1};
    const int64_t ds[4] = {(int64_t)size[1] * size[2] * size[3], (int64_t)size[2] * size[3],
                           size[3], 1};
    const double* s0 = src + (((size_t)sn * v.nc3 + sk) * v.nc2 + sj) * v.nc1 + si;
    RK(exo::launch_view_copy(s0, ss, buf + *offset, ds, size, st));
    *offset += size[0] * size[1] * size[2] * size[3];
    return EXO_OK;
  }
  // a panel edge: the band LoadBoundaryBufferSameLevel hands to PackData
  const int G = exo::G;
  const int want_sj = ox2 > 0 ? v.je - G + 1 : v.js, want_ej = ox2 < 0 ? v.js + G - 1 : v.je;
  const int want_sk = ox3 > 0 ? v.ke - G + 1 : v.ks, want_ek = ox3 < 0 ? v.ks + G - 1 : v.ke;
  if (sn != 0 || en != v.nv - 1 || si != v.is || ei != v.ie || sj != want_sj || ej != want_ej ||
      sk != want_sk || ek != want_ek)
    return fail(EXO_ERR_SHAPE, "a panel-edge pack takes every variable and the G-wide edge band "
                               "of the interior (one block per panel)");
  const int side = ox2 < 0 ? 0 : ox2 > 0 ? 1 : ox3 < 0 ? 2 : 3;
  int tp, ts;
  exo::panel_neighbor(panel, side, &tp, &ts);
  const int tox2 = ts == 0 ? -1 : ts == 1 ? 1 : 0, tox3 = ts == 2 ? -1 : ts == 3 ? 1 : 0;
  const int rsj = tox2 < 0 ? v.js - G : tox2 > 0 ? v.je + 1 : v.js;
  const int rsk = tox3 < 0 ? v.ks - G : tox3 > 0 ? v.ke + 1 : v.ks;
  const int J = tox2 != 0 ? G : v.N, K = tox3 != 0 ? G : v.N;
  RK(exo::launch_panel_pack(v, src, buf + *offset, tp, rsk, rsj, K, J, st));
  *offset += v.nv * K * J * v.L;
  return EXO_OK;
}

static int lr3d_ensure(exo_ctx* c) {
  if (c->lr3d) return EXO_OK;
  CK(cudaMalloc((void**)&c->lr3d, 4 * c->state_elems * sizeof(double)));
  c->owned.push_back(c->lr3d);
  CK(cudaMemsetAsync(c->lr3d, 0, 4 * c->state_elems * sizeof(double), c->stream));
  return EXO_OK;
}
static double* lr3d_store(exo_ctx* c, int direction, bool right) {
  return c->lr3d + ((size_t)(direction - 2) * 2 + (right ? 1 : 0)) * c->state_elems;
}

int exo_save_lr3d(exo_ctx* c, const double* L_row, const double* R_row, int direction, int panel,
                  int k, int j, int il, int iu, void* stream) {
  if (!c || !L_row || !R_row) return fail(EXO_ERR_ARG, "NULL argument");
  const DevView& v = c->v;
  if (direction != 2 && direction != 3) return fail(EXO_ERR_ARG, "direction must be 2 or 3");
  if (panel < 0 || panel > 5 || k < 0 || k >= v.nc3 || j < 0 || j >= v.nc2 || il < 0 ||
      iu >= v.nc1 || il > iu)
    return fail(EXO_ERR_SHAPE, "row outside the arrays");
  int rc = lr3d_ensure(c);
  if (rc) return rc;
  cudaStream_t st = hook_stream(c, stream);
  const size_t w = (size_t)(iu - il + 1) * sizeof(double);
  for (int side = 0; side < 2; ++side) {
    double* dst = lr3d_store(c, direction, side == 1) + (((size_t)panel * v.nv * v.nc3 + k) * v.nc2 + j) * v.nc1 + il;
    const double* srow = (side ? R_row : L_row) + il;
    CK(cudaMemcpy2DAsync(dst, v.cells * sizeof(double), srow, v.nc1 * sizeof(double), w, v.nv,
                         cudaMemcpyDefault, st));
  }
  return EXO_OK;
}

int exo_load_lr3d(exo_ctx* c, double* L_row, double* R_row, int direction, int panel, int k,
                  int j, int il, int iu, void* stream) {
  if (!c || !L_row || !R_row) return fail(EXO_ERR_ARG, "NULL argument");
  const DevView& v = c->v;
  if (direction != 2 && direction != 3) return fail(EXO_ERR_ARG, "direction must be 2 or 3");
  if (panel < 0 || panel > 5 || k < 0 || k >= v.nc3 || j < 0 || j >= v.nc2 || il < 0 ||
      iu >= v.nc1 || il > iu)
    return fail(EXO_ERR_SHAPE, "row outside the arrays");
  int rc = lr3d_ensure(c);
  if (rc) return rc;
  cudaStream_t st = hook_stream(c, stream);
  const size_t w = (size_t)(iu - il + 1) * sizeof(double);
  for (int side = 0; side < 2; ++side) {
    const double* src = lr3d_store(c, direction, side == 1) + (((size_t)panel * v.nv * v.nc3 + k) * v.nc2 + j) * v.nc1 + il;
    double* drow = (side ? R_row : L_row) + il;
    CK(cudaMemcpy2DAsync(drow, v.nc1 * sizeof(double), src, v.cells * sizeof(double), w, v.nv,
                         cudaMemcpyDefault, st));
  }
  return EXO_OK;
}

int exo_lr3d_arrays(exo_ctx* c, double** L2, double** R2, double** L3, double** R3) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = lr3d_ensure(c);
  if (rc) return rc;
  if (L2) *L2 = lr3d_store(c, 2, false);
  if (R2) *R2 = lr3d_store(c, 2, true);
  if (L3) *L3 = lr3d_store(c, 3, false);
  if (R3) *R3 = lr3d_store(c, 3, true);
  return EXO_OK;
}

int exo_synchronize_faces(exo_ctx* c, void* stream) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = lr3d_ensure(c);
  if (rc) return rc;
  RK(exo::launch_face_sync(c->v, lr3d_store(c, 2, false), lr3d_store(c, 2, true),
                           lr3d_store(c, 3, false), lr3d_store(c, 3, true),
                           hook_stream(c, stream)));
  return EXO_OK;
}

// ------------------------------------------------- equation-of-state hooks --
static int eos_range(exo_ctx* c, int to_prim, const double* in, double* out, int il, int iu,
                     int jl, int ju, int kl, int ku, void* stream) {
  if (!c || !in || !out) return fail(EXO_ERR_ARG, "NULL argument");
  const DevView& v = c->v;
  if (il < 0 || iu >= v.nc1 || jl < 0 || ju >= v.nc2 || kl < 0 || ku >= v.nc3)
    return fail(EXO_ERR_SHAPE, "index range outside the arrays");
  RK(exo::launch_eos_range(v, to_prim, in, out, il, iu, jl, ju, kl, ku, hook_stream(c, stream)));
  return EXO_OK;
}

int exo_conserved_to_primitive(exo_ctx* c, const double* u, double* w, int il, int iu, int jl,
                               int ju, int kl, int ku, void* stream) {
  return eos_range(c, 1, u, w, il, iu, jl, ju, kl, ku, stream);
}

int exo_primitive_to_conserved(exo_ctx* c, const double* w, double* u, int il, int iu, int jl,
                               int ju, int kl, int ku, void* stream) {
  return eos_range(c, 0, w, u, il, iu, jl, ju, kl, ku, stream);
}

int exo_sound_speed(exo_ctx* c, int n, const double* prim, double* cs, void* stream) {
  if (!c || n < 0 || (n > 0 && (!prim || !cs))) return fail(EXO_ERR_ARG, "bad argument");
  RK(exo::launch_sound_speed(c->v, n, prim, cs, hook_stream(c, stream)));
  return EXO_OK;
}

// ----------------------------------------------------------- array views --
// Checks six panel views against the context's per-panel shape.
static int check_views(exo_ctx* c, const exo_array_view* views) {
  if (!views) return fail(EXO_ERR_ARG, "NULL views");
  const DevView& v = c->v;
  for (int p = 0; p < 6; ++p) {
    const exo_array_view& a = views[p];
    if (!a.data) return fail(EXO_ERR_ARG, "view without data");
    if (a.dtype != EXO_DTYPE_F64) return fail(EXO_ERR_ARG, "views hold FP64 values");
    if (a.nx4 != v.nv || a.nx3 != v.nc3 || a.nx2 != v.nc2 || a.nx1 != v.nc1)
      return fail(EXO_ERR_SHAPE, "a panel view is (nvar, N+6, N+6, L+6)");
    if (a.device >= 0 && a.device != c->device)
      return fail(EXO_ERR_ARG, "device view on another GPU than the context's");
  }
  return EXO_OK;
}

// six panel views <-> the contiguous host staging array (whole-atmosphere layout)
static int views_gather(exo_ctx* c, const exo_array_view* views, std::vector<double>& host) {
  const DevView& v = c->v;
  const size_t pan = (size_t)v.nv * v.cells;
  host.resize(6 * pan);
  const int size[4] = {v.nv, v.nc3, v.nc2, v.nc1};
  const int64_t cs[4] = {(int64_t)v.nc3 * v.nc2 * v.nc1, (int64_t)v.nc2 * v.nc1, v.nc1, 1};
  double* tmp = nullptr;
  for (int p = 0; p < 6; ++p) {
    const exo_array_view& a = views[p];
    const double* d = static_cast<const double*>(a.data);
    if (a.device < 0) {
      double* out = host.data() + p * pan;
      for (int n = 0; n < v.nv; ++n)
        for (int k = 0; k < v.nc3; ++k)
          for (int j = 0; j < v.nc2; ++j)
            for (int i = 0; i < v.nc1; ++i)
              *out++ = d[n * a.stride[0] + k * a.stride[1] + j * a.stride[2] + i * a.stride[3]];
    } else {
      if (!tmp) CK(cudaMalloc((void**)&tmp, pan * sizeof(double)));
      int rc = exo::launch_view_copy(d, a.stride, tmp, cs, size, c->stream);
      if (!rc && cudaMemcpyAsync(host.data() + p * pan, tmp, pan * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
        rc = EXO_ERR_CUDA;
      if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = EXO_ERR_CUDA;
      if (rc) {
        cudaFree(tmp);
        return fail(EXO_ERR_CUDA, "view gather failed");
      }
    }
  }
  if (tmp) cudaFree(tmp);
  return EXO_OK;
}

static int views_scatter(exo_ctx* c, const std::vector<double>& host, const exo_array_view* views) {
  const DevView& v = c->v;
  const size_t pan = (size_t)v.nv * v.cells;
  const int size[4] = {v.nv, v.nc3, v.nc2, v.nc1};
  const int64_t cs[4] = {(int64_t)v.nc3 * v.nc2 * v.nc1, (int64_t)v.nc2 * v.nc1, v.nc1, 1};
  double* tmp = nullptr;
  for (int p = 0; p < 6; ++p) {
    const exo_array_view& a = views[p];
    double* d = static_cast<double*>(a.data);
    if (a.device < 0) {
      const double* in = host.data() + p * pan;
      for (int n = 0; n < v.nv; ++n)
        for (int k = 0; k < v.nc3; ++k)
          for (int j = 0; j < v.nc2; ++j)
            for (int i = 0; i < v.nc1; ++i)
              d[n * a.stride[0] + k * a.stride[1] + j * a.stride[2] + i * a.stride[3]] = *in++;
    } else {
      if (!tmp) CK(cudaMalloc((void**)&tmp, pan * sizeof(double)));
      int rc = cudaMemcpyAsync(tmp, host.data() + p * pan, pan * sizeof(double),
                               cudaMemcpyHostToDevice, c->stream) == cudaSuccess ? 0 : EXO_ERR_CUDA;
      if (!rc) rc = exo::launch_view_copy(tmp, cs, d, a.stride, size, c->stream);
      if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = EXO_ERR_CUDA;
      if (rc) {
        cudaFree(tmp);
        return fail(EXO_ERR_CUDA, "view scatter failed");
      }
    }
  }
  if (tmp) cudaFree(tmp);
  return EXO_OK;
}

int exo_set_primitive_views(exo_ctx* c, const exo_array_view* w) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = check_views(c, w);
  std::vector<double> h;
  if (!rc) rc = views_gather(c, w, h);
  return rc ? rc : exo_set_primitive(c, h.data());
}

int exo_get_primitive_views(exo_ctx* c, const exo_array_view* w) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = check_views(c, w);
  if (rc) return rc;
  std::vector<double> h(c->state_elems);
  if ((rc = exo_get_primitive(c, h.data()))) return rc;
  return views_scatter(c, h, w);
}

int exo_get_conserved_views(exo_ctx* c, const exo_array_view* u) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = check_views(c, u);
  if (rc) return rc;
  std::vector<double> h(c->state_elems);
  if ((rc = exo_get_conserved(c, h.data()))) return rc;
  return views_scatter(c, h, u);
}

int exo_solve_implicit_3d_views(exo_ctx* c, const exo_array_view* du, const exo_array_view* w,
                                double dt) {
  if (!c) return fail(EXO_ERR_ARG, "ctx is NULL");
  int rc = check_views(c, du);
  if (!rc) rc = check_views(c, w);
  std::vector<double> hd, hw;
  if (!rc) rc = views_gather(c, du, hd);
  if (!rc) rc = views_gather(c, w, hw);
  if (!rc) rc = exo_solve_implicit_3d(c, hd.data(), hw.data(), dt);
  return rc ? rc : views_scatter(c, hd, du);
}

int exo_reciprocal(int precision, int n, const double* x, double* out, void* stream) {
  if (n < 0 || !x || !out) return fail(EXO_ERR_ARG, "bad argument");
  if (precision < EXO_PREC_FP64 || precision > EXO_PREC_MIXED_F32_SOLVE)
    return fail(EXO_ERR_ARG, "unknown precision");
  RK(exo::mixed_build(precision) ? exo::mixed::launch_reciprocal(n, x, out, stream)
                                 : exo::fp64::launch_reciprocal(n, x, out, stream));
  return EXO_OK;
}

int exo_weno5(int n, const double* a, const double* b, const double* c, const double* d,
              const double* e, double* out, void* stream) {
  if (n < 0 || !a || !b || !c || !d || !e || !out) return fail(EXO_ERR_ARG, "bad argument");
  RK(exo::launch_weno5(n, a, b, c, d, e, out, stream));
  return EXO_OK;
}

}  // extern "C"
