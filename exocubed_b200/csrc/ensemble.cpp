// ensemble.cpp -- many independent atmospheres of uneven size advanced by
// one batched launch per kernel, the whole SSPRK(3,3) step captured in one
// CUDA graph.
//
// Members are ensemble runs (the forward models of the reference's MCMC
// inversion, src/inversion/profile_inversion.cpp:112-120): each has its own
// cubed sphere (N, L), its own gas (gamma, g), its own CFL time step and its
// own device state; they share nothing but the launches.  Membership changes
// (exo_ensemble_add / exo_ensemble_remove) mark the batch tables dirty; the
// next exo_ensemble_step uploads the new tables and re-captures the graph.
// Device memory of members comes from the ensemble's own stream-ordered pool,
// and admission is checked against a byte budget (the resident-footprint
// ledger of the serving loop).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "exo_internal.h"

using exo::BatchPlan;
using exo::DevScalars;
using exo::DevView;

namespace {


struct Member {
  exo_config cfg;
  DevView v;
  std::vector<void*> owned;
  size_t bytes = 0;
};

}  // namespace

struct exo_ensemble {
  int precision = EXO_PREC_FP64;
  int capacity = 0;
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<Member*> slots;
  // batch tables (device) sized for the capacity
  DevView* d_views = nullptr;
  unsigned* d_start = nullptr;  // [BK_COUNT][capacity+1]
  bool dirty = true;
  cudaGraphExec_t exec = nullptr;
  int64_t launches_per_step = 0;
  int64_t launches = 0;
  int device = 0;
  exo::Tiles tiles = exo::default_tiles();
};

namespace {

int efail(int code, const std::string& msg) { return exo::set_error(code, msg); }

int cuda_efail(cudaError_t e, const char* what) {
  return exo::set_error(EXO_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define ECK(call)                                           \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_efail(e_, #call);    \
  } while (0)

int launch_single(int precision, int which, const DevView& v, void* st, double arg,
                  const double* src) {
  bool mixed = exo::mixed_build(precision);
  switch (which) {
    case 0: return mixed ? exo::mixed::launch_p2c_interior(v, src, st)
                         : exo::fp64::launch_p2c_interior(v, src, st);
    case 1: return mixed ? exo::mixed::launch_dt_reset(v, st) : exo::fp64::launch_dt_reset(v, st);
    case 2: return mixed ? exo::mixed::launch_prim_ghost(v, true, st)
                         : exo::fp64::launch_prim_ghost(v, true, st);
    case 4: return mixed ? exo::mixed::launch_prim_ghost(v, false, st)
                         : exo::fp64::launch_prim_ghost(v, false, st);
    default: return mixed ? exo::mixed::launch_dt_finalize(v, arg, false, st)
                          : exo::fp64::launch_dt_finalize(v, arg, false, st);
  }
}

// rebuild the batch tables and capture one batched step into a graph
int rebuild(exo_ensemble* e) {
  if (e->exec) {
    cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
  }
  std::vector<DevView> views;
  std::vector<unsigned> start((size_t)exo::BK_COUNT * (e->capacity + 1), 0);
  unsigned tot[exo::BK_COUNT] = {0, 0, 0, 0, 0, 0};
  bool any_full = false;  // some member takes the 5x5 correction
  int max_nc1 = 1;
  // the x1 blocks' threads: the ensemble's columns per block at the deepest
  // member; every member then takes as many columns as fill those threads
  int x1_threads = 32;
  for (Member* m : e->slots) {
    if (!m || m->v.eqn == EXO_EQN_SHALLOW_YZ) continue;
    DevView tv = m->v;  // with the ensemble's tiles
    for (int k = 0; k < exo::BK_COUNT; ++k) tv.tiles[k] = e->tiles.t[k];
    x1_threads = std::max(x1_threads, exo::x1_threads(tv));
  }
  size_t x1_smem = 8;
  // members in the batch deepest first: the blocks of a launch start in
  // index order, so the columns with the longest vertical walks start
  // first and the last wave holds short ones
  std::vector<Member*> order;
  for (Member* m : e->slots)
    if (m) order.push_back(m);
  std::stable_sort(order.begin(), order.end(),
                   [](const Member* a, const Member* b) { return a->v.L > b->v.L; });
  for (Member* m : order) {
    int idx = (int)views.size();
    views.push_back(m->v);
    DevView& mv = views.back();
    for (int k = 0; k < exo::BK_COUNT; ++k) mv.tiles[k] = e->tiles.t[k];
    if (mv.eqn != EXO_EQN_SHALLOW_YZ) {
      mv.tiles[exo::BK_X1] = exo::x1_member_columns(mv, x1_threads, exo::X1_SMEM_MAX);
      x1_smem = std::max(x1_smem, exo::x1_smem_bytes(mv));
    }
    max_nc1 = std::max(max_nc1, m->v.nc1);
    if (m->v.eqn != EXO_EQN_SHALLOW_YZ && (m->v.implicit_flag & 1) && (m->v.implicit_flag & 8))
      any_full = true;
    unsigned b[exo::BK_COUNT];
    exo::member_blocks(m->v, mv.tiles, b);
    for (int k = 0; k < exo::BK_COUNT; ++k) {
      start[(size_t)k * (e->capacity + 1) + idx] = tot[k];
      tot[k] += b[k];
    }
  }
  int n = (int)views.size();
  for (int k = 0; k < exo::BK_COUNT; ++k) start[(size_t)k * (e->capacity + 1) + n] = tot[k];
  e->dirty = false;
  e->launches_per_step = 0;
  if (n == 0) return 0;
  ECK(cudaMemcpyAsync(e->d_views, views.data(), n * sizeof(DevView), cudaMemcpyHostToDevice,
                      e->stream));
  ECK(cudaMemcpyAsync(e->d_start, start.data(), start.size() * sizeof(unsigned),
                      cudaMemcpyHostToDevice, e->stream));
  ECK(cudaStreamSynchronize(e->stream));  // host vectors go out of scope
  BatchPlan pl;
  pl.views = e->d_views;
  pl.n = n;
  for (int k = 0; k < exo::BK_COUNT; ++k) {
    pl.start[k] = e->d_start + (size_t)k * (e->capacity + 1);
    pl.total[k] = tot[k];
  }
  pl.x1_threads = x1_threads;
  pl.x1_smem = x1_smem;
  for (int k = 0; k < exo::BK_COUNT; ++k) pl.threads[k] = e->tiles.t[k];
  pl.max_nc1 = max_nc1;
  pl.precision = e->precision;
  pl.any_full_correction = any_full;
  // count the kernel nodes of one step
  int64_t per_stage = (tot[exo::BK_X1] ? 1 : 0) + 1 + 1 +
                      (tot[exo::BK_IMPLICIT] ? (any_full && exo::split_bwd(e->precision) ? 2 : 1) : 0) + 1;
  e->launches_per_step = 3 * per_stage + (tot[exo::BK_ROUNDTRIP] ? 1 : 0) + 1 + 1;
  cudaGraph_t graph;
  ECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  int rc = exo::mixed_build(e->precision) ? exo::mixed::launch_batched_step(pl, e->stream)
                                          : exo::fp64::launch_batched_step(pl, e->stream);
  cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
  if (rc) return efail(EXO_ERR_CUDA, "batched step capture failed");
  if (ce != cudaSuccess) return cuda_efail(ce, "cudaStreamEndCapture");
  ce = cudaGraphInstantiate(&e->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return cuda_efail(ce, "cudaGraphInstantiate");
  return 0;
}

Member* member_at(exo_ensemble* e, int slot) {
  if (!e || slot < 0 || slot >= e->capacity) return nullptr;
  return e->slots[slot];
}

}  // namespace

extern "C" {

int exo_ensemble_footprint(const exo_config* cfg, size_t* bytes) {
  if (!cfg || !bytes) return efail(EXO_ERR_ARG, "NULL argument");
  std::string err;
  if (!exo::validate_config(*cfg, &err)) return efail(EXO_ERR_ARG, err);
  *bytes = exo::view_footprint(*cfg);
  return EXO_OK;
}

int exo_ensemble_create(int precision, int capacity, size_t budget_bytes, exo_ensemble** out) {
  if (!out) return efail(EXO_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (precision != EXO_PREC_FP64 && !exo::mixed_build(precision))
    return efail(EXO_ERR_ARG,
                 "precision must be EXO_PREC_FP64, EXO_PREC_MIXED or EXO_PREC_MIXED_F32_SOLVE");
  if (capacity < 1 || capacity > 4096) return efail(EXO_ERR_ARG, "capacity must be in [1, 4096]");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return efail(EXO_ERR_NOGPU, "no CUDA device");
  exo_ensemble* e = new exo_ensemble();
  e->precision = precision;
  e->capacity = capacity;
  e->budget = budget_bytes;
  e->slots.assign(capacity, nullptr);
  cudaGetDevice(&e->device);
  if (exo::fp64::prepare_kernels() || exo::mixed::prepare_kernels()) {
    delete e;
    return efail(EXO_ERR_CUDA, "kernel attributes could not be set");
  }
  auto undo = [&](int rc) {
    if (e->d_views) cudaFree(e->d_views);
    if (e->d_start) cudaFree(e->d_start);
    if (e->pool) cudaMemPoolDestroy(e->pool);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return rc;
  };
  cudaError_t ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return undo(cuda_efail(ce, "cudaStreamCreate"));
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = e->device;
  ce = cudaMemPoolCreate(&e->pool, &props);
  if (ce != cudaSuccess) return undo(cuda_efail(ce, "cudaMemPoolCreate"));
  uint64_t keep = UINT64_MAX;  // retain freed member memory for the next admission
  cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  ce = cudaMalloc((void**)&e->d_views, (size_t)capacity * sizeof(DevView));
  if (ce != cudaSuccess) return undo(cuda_efail(ce, "cudaMalloc(views)"));
  ce = cudaMalloc((void**)&e->d_start, (size_t)exo::BK_COUNT * (capacity + 1) * sizeof(unsigned));
  if (ce != cudaSuccess) return undo(cuda_efail(ce, "cudaMalloc(starts)"));
  *out = e;
  return EXO_OK;
}

void exo_ensemble_destroy(exo_ensemble* e) {
  if (!e) return;
  cudaStreamSynchronize(e->stream);
  if (e->exec) cudaGraphExecDestroy(e->exec);
  for (Member*& m : e->slots) {
    if (!m) continue;
    for (void* p : m->owned) cudaFreeAsync(p, e->stream);
    delete m;
    m = nullptr;
  }
  cudaStreamSynchronize(e->stream);
  cudaFree(e->d_views);
  cudaFree(e->d_start);
  cudaMemPoolDestroy(e->pool);
  cudaStreamDestroy(e->stream);
  delete e;
}

namespace {

// Admission of a member: slot, budget, tables, device memory; then its
// state from the primitives w_host (PrimitiveToConserved, ghosts,
// primitives, first dt) or from a checkpoint image.
int admit(exo_ensemble* e, const exo_config* cfg, const double* w_host, const void* image,
          int* slot) {
  *slot = -1;
  std::string err;
  if (!exo::validate_config(*cfg, &err)) return efail(EXO_ERR_ARG, err);
  if (cfg->precision != e->precision)
    return efail(EXO_ERR_ARG, "member precision differs from the ensemble's");
  int free_slot = -1;
  for (int i = 0; i < e->capacity; ++i)
    if (!e->slots[i]) { free_slot = i; break; }
  if (free_slot < 0) return efail(EXO_ERR_CAPACITY, "no free member slot");
  size_t need = exo::view_footprint(*cfg);
  if (e->used + need > e->budget)
    return efail(EXO_ERR_CAPACITY, "member footprint exceeds the remaining memory budget");
  exo::HostTables tab;
  if (!exo::build_tables(*cfg, tab, &err)) return efail(EXO_ERR_ARG, err);
  Member* m = new Member();
  m->cfg = *cfg;
  m->bytes = need;
  // stream-ordered allocations from the ensemble's pool
  int rc = exo::view_allocate(*cfg, tab, m->v, m->owned, e->stream, e->pool, &err);
  if (rc) {
    for (void* p : m->owned) cudaFreeAsync(p, e->stream);
    delete m;
    return efail(rc, err);
  }
  if (image) {
    // u, w and the clock; the primitives (and their FP32 copy in the mixed
    // build) are recomputed from u as the end of every step computes them
    rc = exo::checkpoint_restore(m->v, e->stream, image, &err);
    if (!rc && launch_single(e->precision, 4, m->v, e->stream, 0., nullptr)) {
      rc = EXO_ERR_CUDA;
      err = "recomputing the member's primitives failed";
    }
    if (!rc) {
      cudaError_t ce = cudaStreamSynchronize(e->stream);
      if (ce != cudaSuccess) {
        rc = EXO_ERR_CUDA;
        err = std::string("exo_ensemble_add_checkpoint: ") + cudaGetErrorString(ce);
      }
    }
    if (rc) {
      for (void* p : m->owned) cudaFreeAsync(p, e->stream);
      delete m;
      return efail(rc, err);
    }
    e->launches += 1;
  } else {
    // the initial state: PrimitiveToConserved, ghosts, primitives, first dt
    size_t bytes = (size_t)6 * m->v.nv * m->v.cells * sizeof(double);
    cudaError_t ce = cudaMemcpyAsync(m->v.w, w_host, bytes, cudaMemcpyHostToDevice, e->stream);
    if (ce != cudaSuccess) {
      for (void* p : m->owned) cudaFreeAsync(p, e->stream);
      delete m;
      return cuda_efail(ce, "cudaMemcpyAsync(initial state)");
    }
    if (launch_single(e->precision, 0, m->v, e->stream, 0., m->v.w) ||
        launch_single(e->precision, 1, m->v, e->stream, 0., nullptr) ||
        launch_single(e->precision, 2, m->v, e->stream, 0., nullptr) ||
        launch_single(e->precision, 3, m->v, e->stream, 0., nullptr)) {
      for (void* p : m->owned) cudaFreeAsync(p, e->stream);
      delete m;
      return efail(EXO_ERR_CUDA, "initialising the member failed");
    }
    ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) {
      for (void* p : m->owned) cudaFreeAsync(p, e->stream);
      delete m;
      return cuda_efail(ce, "exo_ensemble_add");
    }
    e->launches += 4;
  }
  e->slots[free_slot] = m;
  e->used += need;
  e->dirty = true;
  *slot = free_slot;
  return EXO_OK;
}

}  // namespace

int exo_ensemble_add(exo_ensemble* e, const exo_config* cfg, const double* w_host, int* slot) {
  if (!e || !cfg || !w_host || !slot) return efail(EXO_ERR_ARG, "NULL argument");
  return admit(e, cfg, w_host, nullptr, slot);
}

int exo_ensemble_add_checkpoint(exo_ensemble* e, const void* image, size_t bytes, int* slot) {
  if (!e || !slot) return efail(EXO_ERR_ARG, "NULL argument");
  *slot = -1;
  exo_checkpoint_header h;
  std::string err;
  int rc = exo::checkpoint_parse(image, bytes, &h, &err);
  if (rc) return efail(rc, err);
  exo_config cfg = h.cfg;
  cfg.precision = e->precision;
  return admit(e, &cfg, nullptr, image, slot);
}

int exo_ensemble_checkpoint_bytes(exo_ensemble* e, int slot, size_t* bytes) {
  Member* m = member_at(e, slot);
  if (!m || !bytes) return efail(EXO_ERR_ARG, "bad slot or NULL argument");
  *bytes = exo::checkpoint_bytes(m->v);
  return EXO_OK;
}

int exo_ensemble_checkpoint_save(exo_ensemble* e, int slot, void* image, size_t bytes) {
  Member* m = member_at(e, slot);
  if (!m) return efail(EXO_ERR_ARG, "no member in that slot");
  std::string err;
  int rc = exo::checkpoint_save(m->cfg, m->v, e->stream, image, bytes, &err);
  return rc ? efail(rc, err) : EXO_OK;
}

int exo_ensemble_remove(exo_ensemble* e, int slot) {
  Member* m = member_at(e, slot);
  if (!m) return efail(EXO_ERR_ARG, "no member in that slot");
  for (void* p : m->owned) cudaFreeAsync(p, e->stream);
  e->used -= m->bytes;
  delete m;
  e->slots[slot] = nullptr;
  e->dirty = true;
  return EXO_OK;
}

int exo_ensemble_step(exo_ensemble* e, int nsteps) {
  exo::Range range("exo_ensemble_step");
  if (!e) return efail(EXO_ERR_ARG, "NULL ensemble");
  if (nsteps < 0) return efail(EXO_ERR_ARG, "nsteps < 0");
  if (e->dirty) {
    int rc = rebuild(e);
    if (rc) return rc;
  }
  if (!e->exec) return EXO_OK;  // no members
  for (int s = 0; s < nsteps; ++s) ECK(cudaGraphLaunch(e->exec, e->stream));
  e->launches += (int64_t)nsteps * e->launches_per_step;
  return EXO_OK;
}

int exo_ensemble_synchronize(exo_ensemble* e) {
  if (!e) return efail(EXO_ERR_ARG, "NULL ensemble");
  ECK(cudaStreamSynchronize(e->stream));
  return EXO_OK;
}

int exo_ensemble_get_conserved(exo_ensemble* e, int slot, double* u_host) {
  Member* m = member_at(e, slot);
  if (!m || !u_host) return efail(EXO_ERR_ARG, "bad slot or NULL buffer");
  size_t bytes = (size_t)6 * m->v.nv * m->v.cells * sizeof(double);
  ECK(cudaMemcpyAsync(u_host, m->v.u, bytes, cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return EXO_OK;
}

int exo_ensemble_get_primitive(exo_ensemble* e, int slot, double* w_host) {
  Member* m = member_at(e, slot);
  if (!m || !w_host) return efail(EXO_ERR_ARG, "bad slot or NULL buffer");
  size_t bytes = (size_t)6 * m->v.nv * m->v.cells * sizeof(double);
  ECK(cudaMemcpyAsync(w_host, m->v.w, bytes, cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  return EXO_OK;
}

int exo_ensemble_member_time(exo_ensemble* e, int slot, double* time, double* dt,
                             int64_t* ncycle) {
  Member* m = member_at(e, slot);
  if (!m) return efail(EXO_ERR_ARG, "no member in that slot");
  DevScalars s;
  ECK(cudaMemcpyAsync(&s, m->v.sc, sizeof(s), cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  if (time) *time = s.time;
  if (dt) *dt = s.dt;
  if (ncycle) *ncycle = s.ncycle;
  return EXO_OK;
}

int exo_ensemble_set_tiles(exo_ensemble* e, const int* threads) {
  if (!e || !threads) return efail(EXO_ERR_ARG, "NULL argument");
  exo::Tiles t = e->tiles;
  for (int k = 0; k < exo::BK_COUNT; ++k)
    if (threads[k] > 0) t.t[k] = threads[k];
  std::string err;
  if (!exo::valid_tiles(t.t, &err)) return efail(EXO_ERR_ARG, err);
  e->tiles = t;
  e->dirty = true;
  return EXO_OK;
}

int exo_ensemble_get_tiles(exo_ensemble* e, int* threads) {
  if (!e || !threads) return efail(EXO_ERR_ARG, "NULL argument");
  for (int k = 0; k < exo::BK_COUNT; ++k) threads[k] = e->tiles.t[k];
  return EXO_OK;
}

int exo_ensemble_check_state(exo_ensemble* e, int slot, int* invalid) {
  Member* m = member_at(e, slot);
  if (!m || !invalid) return efail(EXO_ERR_ARG, "bad slot or NULL argument");
  DevScalars s;
  ECK(cudaMemcpyAsync(&s, m->v.sc, sizeof(s), cudaMemcpyDeviceToHost, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  *invalid = s.invalid;
  int zero = 0;
  ECK(cudaMemcpyAsync(&m->v.sc->invalid, &zero, sizeof(int), cudaMemcpyHostToDevice, e->stream));
  ECK(cudaStreamSynchronize(e->stream));
  if (s.timeout)
    return efail(EXO_ERR_TIMEOUT, "a kernel's bounded wait for its bulk copies gave up");
  return EXO_OK;
}

int exo_ensemble_stats(exo_ensemble* e, int* members, size_t* bytes_in_use, int64_t* launches) {
  if (!e) return efail(EXO_ERR_ARG, "NULL ensemble");
  int n = 0;
  for (Member* m : e->slots) n += m ? 1 : 0;
  if (members) *members = n;
  if (bytes_in_use) *bytes_in_use = e->used;
  if (launches) *launches = e->launches;
  return EXO_OK;
}

int exo_ensemble_get_stream(exo_ensemble* e, void** stream) {
  if (!e || !stream) return efail(EXO_ERR_ARG, "NULL argument");
  *stream = (void*)e->stream;
  return EXO_OK;
}

}  // extern "C"
