// Kernel instantiations: one warp per instance (n <= 32, m <= n_pad / 4), FP64.
#include "qpb_kernel.cuh"
#include "qpb_warpqp.cuh"

namespace qpb {

// kWarps instances per CTA; kMinBlocks bounds registers so that the register
// file does not cap residency below what shared memory allows.
template <int NP, int MP, int kMinBlocks>
__global__ void __launch_bounds__(kWarpKernelThreads, kMinBlocks) warp_kernel(const __grid_constant__ Params P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int team = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  unsigned char* arena = P.arena_in_smem ? smem + (size_t)team * P.arena_bytes
                                         : P.arena + ((size_t)blockIdx.x * (blockDim.x >> 5) + team) * P.arena_bytes;
  WarpQP<NP, MP> S;
  S.setup(P, arena, lane);
  for (;;) {
    int v = 0;
    if (lane == 0) v = atomicAdd(P.counter, 1);
    const int inst = __shfl_sync(kFull, v, 0);
    if (inst >= P.batch) break;
    S.run(inst);
  }
}

KernelFn kernel_warp_f64(int NP) {
  if (NP == 8) return warp_kernel<8, 2, 4>;
  if (NP == 16) return warp_kernel<16, 4, 4>;  // 128 registers, no spills: 24 % faster than 3 CTAs/SM
  if (NP == 32) return warp_kernel<32, 8, 2>;
  return nullptr;
}

}  // namespace qpb
