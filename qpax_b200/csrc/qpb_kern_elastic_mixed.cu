// Kernel instantiations: ElasticQP, FP32 factor + FP64 refinement.
#include "qpb_kernel.cuh"

namespace qpb {

KernelFn kernel_elastic_mixed(int NT, int KC) {
#define QPB_ENTRY(nt, kc) \
  if (NT == nt && KC == kc) return ipm_kernel<ElasticQP<nt, kc, true>, nt>;
  QPB_FOR_EACH_VARIANT(QPB_ENTRY)
#undef QPB_ENTRY
  return nullptr;
}

}  // namespace qpb
