// qpb_noalloc.cu -- qpb_solve_qp for callers that cannot allocate device
// memory (include/qpb.h: qpb_solve_qp_noalloc).
//
// Some hosts cannot call cudaMalloc at solve time: code running inside a
// CUDA-graph capture that forbids allocation, real-time control loops that
// allocate everything up front, or plugins whose host framework owns the
// device allocator and exposes no workspace hook.  For them this entry point
// takes its scratch -- the work counter of the persistent launch and, when an
// instance does not fit in shared memory, its global arena -- from a
// file-scope __device__ array that the library reserves once per device for
// the life of the process.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/qpb.h"

namespace {

// Every device that loads libqpb.so holds this array until the process exits.
constexpr size_t kStaticScratchBytes = size_t(1) << 20;  // 1 MiB
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices];

// Device address of g_static_scratch on the current device.  Host code may
// not use the symbol itself as a pointer (on the host it names a shadow
// variable, not device memory), so the address is looked up once per device.
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return QPB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_static_scratch) != cudaSuccess || !p) return QPB_ERR_CUDA;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return QPB_OK;
}

}  // namespace

extern "C" int qpb_solve_qp_noalloc(const qpb_dims* dims, const double* Q, const double* q, const double* A,
                                    const double* b, const double* G, const double* h, double solver_tol,
                                    double* x, double* s, double* z, double* y, int32_t* converged,
                                    int32_t* iters, const qpb_config* cfg, qpb_stream_t stream) {
  const size_t need = qpb_workspace_size(QPB_OP_SOLVE, dims, cfg);
  if (need == 0) {
    // invalid or unsupported dims/config: let the regular entry point name the error
    return qpb_solve_qp(dims, Q, q, A, b, G, h, solver_tol, x, s, z, y, converged, iters, cfg, nullptr, 0,
                        stream);
  }
  if (need > kStaticScratchBytes) return QPB_ERR_UNSUPPORTED;
  void* scratch = nullptr;
  const int st = scratch_address(&scratch);
  if (st != QPB_OK) return st;
  // qpb_solve_qp zeroes the work counter on `stream` before its launch and
  // allocates nothing; calls overlapping on the GPU would share the array.
  return qpb_solve_qp(dims, Q, q, A, b, G, h, solver_tol, x, s, z, y, converged, iters, cfg, scratch,
                      kStaticScratchBytes, stream);
}
