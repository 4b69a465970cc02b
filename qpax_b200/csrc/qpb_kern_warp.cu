// Kernel instantiations: one warp per instance (n <= 32, m <= n_pad / 4), and
// four instances per warp in lockstep for n_pad = 8; FP64.
#include "qpb_warpkern.cuh"
#include "qpb_groupqp.cuh"

namespace qpb {

// 32 / NP instances per warp (lane groups of NP), four warps per CTA; the
// instances of a warp are consecutive indices, fetched together.
template <int NP, int MP, int kMinBlocks>
__global__ void __launch_bounds__(kWarpKernelThreads, kMinBlocks) group_kernel(const __grid_constant__ Params P) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int kGroups = 32 / NP;
  const int team = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const size_t first =
      ((P.arena_in_smem ? (size_t)0 : (size_t)blockIdx.x * (blockDim.x >> 5)) + (size_t)team) * kGroups;
  unsigned char* arena0 = (P.arena_in_smem ? smem : P.arena) + first * P.arena_bytes;
  GroupQP<NP, MP> S;
  S.setup(P, arena0, P.arena_bytes, lane);
  for (;;) {
    int v = 0;
    if (lane == 0) v = atomicAdd(P.counter, kGroups);
    const int base = __shfl_sync(kFull, v, 0);
    if (base >= P.batch) break;
    const long inst = (long)base + lane / NP;
    S.run(inst, inst < P.batch);
  }
}

// n_pad = 8 only: four instances per warp ran the NNLS batch (n = 5) 1.4x
// faster than one per warp; at n_pad = 16 two per warp measured no faster.
KernelFn kernel_group_f64(int NP) {
  if (NP == 8) return group_kernel<8, 2, 3>;  // 168 registers: 8 % faster than 128 (which spills)
  return nullptr;
}

KernelFn kernel_warp_f64(int NP) {
  if (NP == 8) return warp_kernel<8, 2, 4>;
  if (NP == 16) return warp_kernel<16, 4, 4>;  // 128 registers, no spills: 24 % faster than 3 CTAs/SM
  if (NP == 32) return warp_kernel<32, 8, 2>;
  return nullptr;
}

}  // namespace qpb
