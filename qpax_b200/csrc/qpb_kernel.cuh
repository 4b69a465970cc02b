// qpb_kernel.cuh -- the persistent interior-point kernel template and the
// per-translation-unit kernel tables.
#pragma once
#include "qpb_elastic.cuh"
#include "qpb_std.cuh"

namespace qpb {

// Register budget: blocks of up to 256 threads; 128-thread teams are held to
// the solver's kMinBlocks resident CTAs per SM (these kernels are
// latency-bound: resident instances hide each other's serial steps).
constexpr int kipm_max_threads(int NT) { return NT == 128 ? 128 : 256; }

// Persistent: each team pulls instance indices from P.counter until the
// batch is exhausted (a bounded loop: at most `batch` fetches in total).
template <class Solver, int NT>
__global__ void __launch_bounds__(kipm_max_threads(NT), Solver::kMinBlocks) ipm_kernel(const __grid_constant__ Params P) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int next_inst;
  const int teams = blockDim.x / NT;
  const int team = threadIdx.x / NT;
  const int rank = threadIdx.x - team * NT;
  unsigned char* arena = P.arena_in_smem
                             ? smem + (size_t)team * P.arena_bytes
                             : P.arena + ((size_t)blockIdx.x * teams + team) * P.arena_bytes;
  BlockedStage* stage = nullptr;
  if constexpr (NT > 32) {  // one team per CTA: the blocked FP64 path's staging
    __shared__ BlockedStage blocked_stage;
    stage = &blocked_stage;
  }
  Solver S;
  S.setup(P, arena, rank, stage);
  if constexpr (NT > 32) {
    // arena in global memory: dynamic shared memory holds the G chunk buffers
    if (!P.arena_in_smem && P.gstage_rows > 0) {
      S.k.gbuf = reinterpret_cast<double*>(smem);
      S.k.gstage_rows = P.gstage_rows;
    }
  }
  for (;;) {
    int inst;
    if constexpr (NT == 32) {
      int v = 0;
      if (rank == 0) v = atomicAdd(P.counter, 1);
      inst = __shfl_sync(kFull, v, 0);
    } else {
      if (rank == 0) next_inst = atomicAdd(P.counter, 1);
      __syncthreads();
      inst = next_inst;
      __syncthreads();
    }
    if (inst >= P.batch) break;
    S.run(inst);
  }
}

using KernelFn = void (*)(Params);

// Kernel for (team threads NT, register chunks KC); nullptr if not built.
KernelFn kernel_std_f64(int NT, int KC);
KernelFn kernel_std_mixed(int NT, int KC);
KernelFn kernel_elastic_f64(int NT, int KC);
KernelFn kernel_elastic_mixed(int NT, int KC);
// One warp per instance, n <= NP (8, 16, 32), m <= NP / 4; FP64.
KernelFn kernel_warp_f64(int NP);
// As kernel_warp_f64 in mixed precision (FP32 inverses, FP64 refinement);
// the instances it hands over are resumed by kernel_warp_f64 (resume launch).
KernelFn kernel_warp_mixed(int NP);
// 32 / NP instances per warp in lockstep (built for NP = 8); nullptr otherwise.
KernelFn kernel_group_f64(int NP);
constexpr int kWarpKernelThreads = 128;

// (NT, KC) variants compiled into the library.
#define QPB_FOR_EACH_VARIANT(X) X(32, 1) X(128, 1) X(128, 2) X(128, 4) X(128, 8) X(256, 4) X(256, 8)


}  // namespace qpb
