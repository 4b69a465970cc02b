// Kernel instantiations: one warp per instance (n <= 32, m <= n_pad / 4) in
// mixed precision -- FP32 factor in the FP64 factor's registers, FP64
// refinement, FP64 refactor once the FP32 factor is rejected -- with the
// FP64 kernel's register budgets where they hold without spills.
#include "qpb_warpkern.cuh"

namespace qpb {

KernelFn kernel_warp_mixed(int NP) {
  if (NP == 8) return warp_kernel<8, 2, 4, true>;
  if (NP == 16) return warp_kernel<16, 4, 3, true>;  // 168 registers: at 128 it spills
  if (NP == 32) return warp_kernel<32, 8, 2, true>;
  return nullptr;
}

}  // namespace qpb
