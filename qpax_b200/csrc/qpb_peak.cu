// qpb_peak.cu -- FMA throughput microbenchmark (qpb_peak.h), built as its own
// library (libqpb_peak.so) for the benchmark; not part of libqpb.so.
#include <cuda_runtime.h>

#include "qpb_peak.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;
constexpr int kThreads = 256;

template <class T>
__global__ void __launch_bounds__(kThreads) fma_chains(T* out, T a, T b) {
  T acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = (T)(threadIdx.x + c);
  for (int i = 0; i < kIters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = fma(acc[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class T>
double run(void* scratch, cudaStream_t s) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fma_chains<T>, kThreads, 0) != cudaSuccess) return -1;
  const int blocks = sms * per_sm;
  if ((size_t)blocks * kThreads * sizeof(T) > (size_t)4 << 20) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chains<T><<<blocks, kThreads, 0, s>>>((T*)scratch, (T)0.999, (T)1e-3);
  cudaEventRecord(e0, s);
  fma_chains<T><<<blocks, kThreads, 0, s>>>((T*)scratch, (T)0.999, (T)1e-3);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess || ms <= 0) return -1;
  const double flops = 2.0 * kChains * (double)kIters * blocks * kThreads;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

extern "C" double qpb_bench_fma_peak(int precision, void* scratch, void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return precision == 1 ? run<double>(scratch, s) : run<float>(scratch, s);
}
