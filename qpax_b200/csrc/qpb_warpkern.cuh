// qpb_warpkern.cuh -- the persistent one-warp-per-instance kernel template
// (FP64, or mixed precision with kMixed), shared by the translation units
// that instantiate it.
#pragma once
#include "qpb_kernel.cuh"
#include "qpb_warpqp.cuh"

namespace qpb {

// kWarps instances per CTA; kMinBlocks bounds registers so that the register
// file does not cap residency below what shared memory allows.
template <int NP, int MP, int kMinBlocks, bool kMixed = false>
__global__ void __launch_bounds__(kWarpKernelThreads, kMinBlocks) warp_kernel(const __grid_constant__ Params P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int team = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  unsigned char* arena = P.arena_in_smem ? smem + (size_t)team * P.arena_bytes
                                         : P.arena + ((size_t)blockIdx.x * (blockDim.x >> 5) + team) * P.arena_bytes;
  WarpQP<NP, MP, kMixed> S;
  S.setup(P, arena, lane);
  // a resume launch covers the instances the mixed launch before it handed over
  const int batch = (!kMixed && P.resume) ? *P.hcount : P.batch;
  for (;;) {
    int v = 0;
    if (lane == 0) v = atomicAdd(P.counter, 1);
    const int inst = __shfl_sync(kFull, v, 0);
    if (inst >= batch) break;
    S.run(inst);
  }
}

}  // namespace qpb
