// peaks.cu -- the arithmetic ceiling the step's FP64-issue-bound kernels are
// measured against: a kernel of independent fused multiply-add chains on
// every SM, timed with CUDA events (exo_measure_fma_peak).
#include <cuda_runtime.h>

#include <string>

#include "exo_internal.h"
#include "exo_mbarrier.cuh"

namespace exo {
namespace {

constexpr int kChains = 8;        // independent FMA chains per thread
constexpr int kThreads = 256;
constexpr int kBlocksPerSm = 4;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fma_chains(T* sink, int iters, T a, T b) {
  T x[kChains];
#pragma unroll
  for (int r = 0; r < kChains; ++r) x[r] = (T)(threadIdx.x + r) * (T)1e-3;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int r = 0; r < kChains; ++r) x[r] = fma(x[r], a, b);
  }
  T s = 0;
#pragma unroll
  for (int r = 0; r < kChains; ++r) s += x[r];
  // a value the chains never reach: the store keeps the work alive
  if (s == (T)-12345.) sink[blockIdx.x] = s;
}

template <typename T>
int run(int repeats, double* out, std::string* err) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    *err = std::string("device query: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  const int blocks = sms * kBlocksPerSm;
  const int iters = sizeof(T) == 8 ? (1 << 16) : (1 << 17);
  T* sink = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  e = cudaMalloc((void**)&sink, blocks * sizeof(T));
  if (e == cudaSuccess) e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  double best = 0.;
  // a and b keep every chain bounded: x -> b / (1 - a)
  const T a = (T)0.999, b = (T)1e-4;
  for (int n = 0; n <= repeats && e == cudaSuccess; ++n) {
    e = cudaEventRecord(t0, 0);
    if (e != cudaSuccess) break;
    k_fma_chains<T><<<blocks, kThreads>>>(sink, iters, a, b);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(t1, 0);
    if (e == cudaSuccess) e = cudaEventSynchronize(t1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    if (e != cudaSuccess || n == 0) continue;  // launch 0 warms up
    double fma_count = (double)blocks * kThreads * kChains * 4. * iters;
    double rate = 2. * fma_count / (ms * 1e-3);
    if (rate > best) best = rate;
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (sink) cudaFree(sink);
  if (e != cudaSuccess) {
    *err = std::string("k_fma_chains: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  *out = best;
  return EXO_OK;
}

// A wait that must give up: one warp waits on an mbarrier phase that
// nothing completes (no arrival, no copy), through the same bounded wait
// the back-substitution kernel uses for its bulk copies.
__global__ void k_wait_selftest(int* gave_up, unsigned long long* waited_ns) {
  __shared__ unsigned long long mb;
  if (threadIdx.x == 0) {
    mbar_init(&mb, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncwarp();
  const unsigned long long t0 = global_ns();
  const bool done = mbar_wait(&mb, 0u);
  const unsigned long long t1 = global_ns();
  if (threadIdx.x == 0) {
    *gave_up = done ? 0 : 1;
    *waited_ns = t1 - t0;
  }
}

}  // namespace

int bounded_wait_selftest(int* gave_up, double* waited_ms, std::string* err) {
  int* g = nullptr;
  unsigned long long* w = nullptr;
  cudaError_t e = cudaMalloc((void**)&g, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&w, sizeof(unsigned long long));
  if (e == cudaSuccess) {
    k_wait_selftest<<<1, 32>>>(g, w);
    e = cudaGetLastError();
  }
  int hg = -1;
  unsigned long long hw = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&hg, g, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&hw, w, sizeof(hw), cudaMemcpyDeviceToHost);
  if (g) cudaFree(g);
  if (w) cudaFree(w);
  if (e != cudaSuccess) {
    *err = std::string("k_wait_selftest: ") + cudaGetErrorString(e);
    return EXO_ERR_CUDA;
  }
  *gave_up = hg;
  *waited_ms = hw * 1e-6;
  return EXO_OK;
}

int measure_fma_peak(bool fp64, int repeats, double* flops_per_s, std::string* err) {
  return fp64 ? run<double>(repeats, flops_per_s, err) : run<float>(repeats, flops_per_s, err);
}

}  // namespace exo
