// peaks.cu -- the arithmetic ceiling the step's FP64-issue-bound kernels are
// measured against: a kernel of independent fused multiply-add chains on
// every SM, timed with CUDA events (exo_measure_fma_peak).
#include <cuda_runtime.h>

#include <string>

#include "exo_internal.h"

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

}  // namespace

int measure_fma_peak(bool fp64, int repeats, double* flops_per_s, std::string* err) {
  return fp64 ? run<double>(repeats, flops_per_s, err) : run<float>(repeats, flops_per_s, err);
}

}  // namespace exo
