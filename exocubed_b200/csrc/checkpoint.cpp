// checkpoint.cpp -- checkpoint images of one atmosphere: configuration,
// clock and the conserved and primitive arrays (ghosts included), the state
// an Athena++ restart file or MeshBlock::Impl::SaveAllStates keeps for the
// hydro (src/mesh_setup.cpp:25-97, src/impl.cpp:306-332).  Shared by the
// single-atmosphere context and the ensemble.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "exo_internal.h"

static_assert(sizeof(exo_checkpoint_header) == 512, "checkpoint header is 512 bytes");

namespace exo {
namespace {

constexpr char kMagic[8] = {'E', 'X', 'O', 'C', 'K', 'P', 'T', '1'};

size_t state_bytes(const DevView& v) { return (size_t)6 * v.nv * v.cells * sizeof(double); }

int cuda_err(cudaError_t e, const char* what, std::string* err) {
  *err = std::string(what) + ": " + cudaGetErrorString(e);
  return EXO_ERR_CUDA;
}

}  // namespace

size_t checkpoint_bytes(const DevView& v) {
  return sizeof(exo_checkpoint_header) + 2 * state_bytes(v);
}

bool same_config_but_precision(const exo_config& a, const exo_config& b) {
  exo_config x = a, y = b;
  x.precision = y.precision = 0;
  return std::memcmp(&x, &y, sizeof(exo_config)) == 0;
}

int checkpoint_save(const exo_config& cfg, const DevView& v, void* stream, void* image,
                    size_t bytes, std::string* err) {
  if (!image) {
    *err = "image is NULL";
    return EXO_ERR_ARG;
  }
  if (bytes < checkpoint_bytes(v)) {
    *err = "image buffer smaller than exo_checkpoint_bytes";
    return EXO_ERR_SHAPE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  char* out = static_cast<char*>(image);
  const size_t sb = state_bytes(v);
  DevScalars sc;
  cudaError_t e = cudaMemcpyAsync(&sc, v.sc, sizeof(sc), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out + sizeof(exo_checkpoint_header), v.u, sb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out + sizeof(exo_checkpoint_header) + sb, v.w, sb,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint copy", err);
  exo_checkpoint_header h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kMagic, sizeof(kMagic));
  h.version = EXO_CHECKPOINT_VERSION;
  h.header_bytes = sizeof(exo_checkpoint_header);
  h.values = (uint64_t)(sb / sizeof(double));
  h.time = sc.time;
  h.dt = sc.dt;
  h.ncycle = sc.ncycle;
  h.invalid = sc.invalid;
  h.cfg = cfg;
  std::memcpy(out, &h, sizeof(h));
  return EXO_OK;
}

int checkpoint_parse(const void* image, size_t bytes, exo_checkpoint_header* h,
                     std::string* err) {
  if (!image || bytes < sizeof(exo_checkpoint_header)) {
    *err = "checkpoint image missing or shorter than its header";
    return EXO_ERR_ARG;
  }
  std::memcpy(h, image, sizeof(*h));
  if (std::memcmp(h->magic, kMagic, sizeof(kMagic)) != 0 ||
      h->header_bytes != sizeof(exo_checkpoint_header)) {
    *err = "not a checkpoint image";
    return EXO_ERR_ARG;
  }
  if (h->version != EXO_CHECKPOINT_VERSION) {
    *err = "checkpoint version " + std::to_string(h->version) + " is not supported";
    return EXO_ERR_ARG;
  }
  if (!validate_config(h->cfg, err)) {
    *err = "checkpoint configuration: " + *err;
    return EXO_ERR_ARG;
  }
  const exo_config& c = h->cfg;
  const uint64_t nv = c.eqn == EXO_EQN_SHALLOW_YZ ? 4 : 5;
  const uint64_t want = 6 * nv * (uint64_t)(c.L + 2 * G) * (c.N + 2 * G) * (c.N + 2 * G);
  if (h->values != want ||
      bytes < sizeof(exo_checkpoint_header) + 2 * want * sizeof(double)) {
    *err = "checkpoint image size does not match its configuration";
    return EXO_ERR_ARG;
  }
  return EXO_OK;
}

int checkpoint_restore(const DevView& v, void* stream, const void* image, std::string* err) {
  exo_checkpoint_header h;
  std::memcpy(&h, image, sizeof(h));
  const char* in = static_cast<const char*>(image) + sizeof(exo_checkpoint_header);
  const size_t sb = state_bytes(v);
  if (h.values * sizeof(double) != sb) {
    *err = "checkpoint image size does not match the atmosphere";
    return EXO_ERR_SHAPE;
  }
  DevScalars sc;
  std::memset(&sc, 0, sizeof(sc));
  sc.dt = h.dt;
  sc.time = h.time;
  sc.dtmin_bits = 0x7FEFFFFFFFFFFFFFull;  // DBL_MAX: reset by every step anyway
  sc.invalid = h.invalid;
  sc.ncycle = h.ncycle;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(v.u, in, sb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(v.w, in + sb, sb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(v.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e, "checkpoint restore", err);
  return EXO_OK;
}

}  // namespace exo
