// Kernel instantiations: ElasticQP, FP64 factor.
#include "qpb_kernel.cuh"

namespace qpb {

KernelFn kernel_elastic_f64(int NT, int KC) {
#define QPB_ENTRY(nt, kc) \
  if (NT == nt && KC == kc) return ipm_kernel<ElasticQP<nt, kc, false>, nt>;
  QPB_FOR_EACH_VARIANT(QPB_ENTRY)
#undef QPB_ENTRY
  return nullptr;
}

}  // namespace qpb
