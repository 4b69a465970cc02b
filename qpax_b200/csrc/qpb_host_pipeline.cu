// qpb_host_pipeline.cu -- forward + backward of solve_qp_primal on a batch held
// in host memory: chunks of the batch flow through copy-in, the two solver
// launches and copy-out on internal streams, so that one chunk's copies
// overlap other chunks' kernels (the host <-> device link is full duplex).
//
// Streams by role: one copy-in stream (chunks arrive in order, each at the
// link's full rate), two compute streams taken in turn (a chunk's solve can
// start while the previous chunk's backward drains, filling the SMs its
// tail leaves idle), one copy-out stream.  Chunks cycle through kSlots device
// buffer sets; events order every reuse of a slot after the last reader of
// its previous chunk.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/qpb.h"
#include "qpb_host.h"

namespace qpb {
namespace {

constexpr int kSlots = 3;    // device buffer sets (chunks in flight)
constexpr int kStreams = 4;  // copy-in, compute (two), copy-out

// Internal streams of one device, created once (non-blocking: they never wait
// on the legacy default stream).
struct DeviceStreams {
  cudaStream_t s[kStreams];
  bool ok = false;
};

bool device_streams(cudaStream_t out[kStreams]) {
  static DeviceStreams cache[64];
  static std::mutex mu;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  std::lock_guard<std::mutex> lk(mu);
  DeviceStreams& d = cache[dev];
  if (!d.ok) {
    for (int i = 0; i < kStreams; ++i)
      if (cudaStreamCreateWithFlags(&d.s[i], cudaStreamNonBlocking) != cudaSuccess) return false;
    d.ok = true;
  }
  for (int i = 0; i < kStreams; ++i) out[i] = d.s[i];
  return true;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Device buffers of one slot (a chunk of up to `cap` instances), carved in
// 256-byte aligned pieces; the same walk sizes and places them.
struct Slot {
  double *Q, *q, *A, *b, *G, *h, *dl;
  double *x, *s, *z, *y;
  int32_t *conv, *iters;
  double *dQ, *dq, *dA, *db, *dG, *dh;
  void* ws;
  size_t ws_bytes;

  size_t carve(unsigned char* base, long cap, long n, long m, long p, size_t wsb) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
      unsigned char* ptr = base ? base + off : nullptr;
      off += align256(bytes);
      return ptr;
    };
    Q = (double*)take(cap * n * n * 8); q = (double*)take(cap * n * 8); A = (double*)take(cap * m * n * 8);
    b = (double*)take(cap * m * 8); G = (double*)take(cap * p * n * 8); h = (double*)take(cap * p * 8);
    dl = (double*)take(cap * n * 8);
    x = (double*)take(cap * n * 8); s = (double*)take(cap * p * 8); z = (double*)take(cap * p * 8);
    y = (double*)take(cap * m * 8);
    conv = (int32_t*)take(cap * 4); iters = (int32_t*)take(cap * 4);
    dQ = (double*)take(cap * n * n * 8); dq = (double*)take(cap * n * 8); dA = (double*)take(cap * m * n * 8);
    db = (double*)take(cap * m * 8); dG = (double*)take(cap * p * n * 8); dh = (double*)take(cap * p * 8);
    ws = take(wsb);
    ws_bytes = wsb;
    return off;
  }
};

long chunk_cap(long batch, int chunks) { return (batch + chunks - 1) / chunks; }

size_t solver_ws(const qpb_dims& d, const qpb_config* cfg) {
  const size_t a = qpb_workspace_size(QPB_OP_SOLVE, &d, cfg);
  const size_t b = qpb_workspace_size(QPB_OP_PRIMAL_BWD, &d, cfg);
  if (a == 0 || b == 0) return 0;
  return a > b ? a : b;
}

size_t slot_bytes(const qpb_dims& d, int chunks, const qpb_config* cfg) {
  const long cap = chunk_cap(d.batch, chunks);
  const qpb_dims dc{(int32_t)cap, d.n, d.m, d.p};
  const size_t wsb = solver_ws(dc, cfg);
  if (wsb == 0) return 0;
  Slot sl;
  return sl.carve(nullptr, cap, d.n, d.m, d.p, wsb);
}

int slots_for(int chunks) { return chunks < kSlots ? chunks : kSlots; }

cudaError_t copy_in(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
}
cudaError_t copy_out(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  return (bytes && dst) ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s) : cudaSuccess;
}

}  // namespace
}  // namespace qpb

using namespace qpb;

extern "C" {

size_t qpb_solve_qp_primal_vjp_host_workspace_size(const qpb_dims* dims, int32_t chunks, const qpb_config* cfg) {
  if (!dims || chunks < 1 || dims->batch < 0) return 0;
  if (check_common(kOpBwd, dims, cfg) != QPB_OK) return 0;
  if (dims->batch == 0) return 256;
  const size_t sb = slot_bytes(*dims, chunks, cfg);
  return sb ? (size_t)slots_for(chunks) * sb + 256 : 0;
}

int qpb_solve_qp_primal_vjp_host(const qpb_dims* dims, const double* Q, const double* q, const double* A,
                                 const double* b, const double* G, const double* h, const double* dl_dx,
                                 double solver_tol, double target_kappa, double* x, double* dQ, double* dq,
                                 double* dA, double* db, double* dG, double* dh, int32_t* converged, int32_t* iters,
                                 int32_t chunks, const qpb_config* cfg, void* workspace, size_t workspace_bytes,
                                 qpb_stream_t stream) {
  if (!dims || chunks < 1) return QPB_ERR_INVALID_ARGUMENT;
  int st = check_common(kOpBwd, dims, cfg);
  if (st) return st;
  const long B = dims->batch, n = dims->n, m = dims->m, p = dims->p;
  if (B == 0) return QPB_OK;
  if (!ok_ptr(Q, B * n * n) || !ok_ptr(q, B * n) || !ok_ptr(A, B * m * n) || !ok_ptr(b, B * m) ||
      !ok_ptr(G, B * p * n) || !ok_ptr(h, B * p) || !ok_ptr(dl_dx, B * n) || !ok_ptr(x, B * n) ||
      !ok_ptr(dQ, B * n * n) || !ok_ptr(dq, B * n) || !ok_ptr(dA, B * m * n) || !ok_ptr(db, B * m) ||
      !ok_ptr(dG, B * p * n) || !ok_ptr(dh, B * p))
    return QPB_ERR_INVALID_ARGUMENT;
  if (chunks > B) chunks = (int32_t)B;
  const size_t need = qpb_solve_qp_primal_vjp_host_workspace_size(dims, chunks, cfg);
  if (need == 0) return QPB_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255))
    return QPB_ERR_WORKSPACE;
  cudaStream_t ss[kStreams];
  if (!device_streams(ss)) return QPB_ERR_CUDA;
  cudaStream_t s_in = ss[0], s_out = ss[3];
  cudaStream_t s_comp[2] = {ss[1], ss[2]};
  const int S = slots_for(chunks);
  const long cap = chunk_cap(B, chunks);
  const size_t sb = slot_bytes(*dims, chunks, cfg);
  Slot slots[kSlots];
  for (int k = 0; k < S; ++k) {
    const qpb_dims dc{(int32_t)cap, dims->n, dims->m, dims->p};
    slots[k].carve(reinterpret_cast<unsigned char*>(workspace) + k * sb, cap, n, m, p, solver_ws(dc, cfg));
  }
  // per chunk: inputs on the device (in), x computed (x), backward done
  // (done), outputs copied (out); plus the fork and one join per stream
  enum { kIn, kX, kDone, kOut, kKinds };
  std::vector<cudaEvent_t> ev;
  const size_t n_ev = (size_t)chunks * kKinds + 1 + kStreams;
  ev.reserve(n_ev);
  st = QPB_OK;
  for (size_t i = 0; i < n_ev; ++i) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      st = QPB_ERR_CUDA;
      break;
    }
    ev.push_back(e);
  }
  auto E = [&](int c, int kind) { return ev[(size_t)c * kKinds + kind]; };
  cudaEvent_t fork = st == QPB_OK ? ev[(size_t)chunks * kKinds] : nullptr;
  // fork: the internal streams start after the work already queued on `stream`
  cudaStream_t s0 = reinterpret_cast<cudaStream_t>(stream);
  if (st == QPB_OK && cudaEventRecord(fork, s0) != cudaSuccess) st = QPB_ERR_CUDA;
  for (int k = 0; st == QPB_OK && k < kStreams; ++k)
    if (cudaStreamWaitEvent(ss[k], fork, 0) != cudaSuccess) st = QPB_ERR_CUDA;
  for (int c = 0; st == QPB_OK && c < chunks; ++c) {
    const long lo = B * c / chunks, hi = B * (c + 1) / chunks, cnt = hi - lo;
    const Slot& sl = slots[c % S];
    cudaStream_t sc = s_comp[c & 1];
    const qpb_dims dc{(int32_t)cnt, dims->n, dims->m, dims->p};
    cudaError_t e = cudaSuccess;
    // copy in (instances lo .. hi-1 are contiguous in every array), once the
    // slot's previous chunk no longer reads its inputs
    if (c >= S) e = cudaStreamWaitEvent(s_in, E(c - S, kDone), 0);
    e = e ? e : copy_in(sl.Q, Q + lo * n * n, cnt * n * n * 8, s_in);
    e = e ? e : copy_in(sl.q, q + lo * n, cnt * n * 8, s_in);
    e = e ? e : copy_in(sl.A, A + lo * m * n, cnt * m * n * 8, s_in);
    e = e ? e : copy_in(sl.b, b + lo * m, cnt * m * 8, s_in);
    e = e ? e : copy_in(sl.G, G + lo * p * n, cnt * p * n * 8, s_in);
    e = e ? e : copy_in(sl.h, h + lo * p, cnt * p * 8, s_in);
    e = e ? e : copy_in(sl.dl, dl_dx + lo * n, cnt * n * 8, s_in);
    e = e ? e : cudaEventRecord(E(c, kIn), s_in);
    // compute, once the inputs are in and the slot's previous outputs are out
    e = e ? e : cudaStreamWaitEvent(sc, E(c, kIn), 0);
    if (c >= S) e = e ? e : cudaStreamWaitEvent(sc, E(c - S, kOut), 0);
    if (e != cudaSuccess) {
      st = QPB_ERR_CUDA;
      break;
    }
    if (cnt > 0) {
      st = qpb_solve_qp(&dc, sl.Q, sl.q, sl.A, sl.b, sl.G, sl.h, solver_tol, sl.x, sl.s, sl.z, sl.y, sl.conv,
                        sl.iters, cfg, sl.ws, sl.ws_bytes, reinterpret_cast<qpb_stream_t>(sc));
      if (st) break;
    }
    e = cudaEventRecord(E(c, kX), sc);
    if (cnt > 0 && e == cudaSuccess) {
      st = qpb_solve_qp_primal_bwd(&dc, sl.Q, sl.q, sl.A, sl.b, sl.G, sl.h, sl.x, sl.s, sl.z, sl.y, sl.dl,
                                   solver_tol, target_kappa, sl.dQ, sl.dq, sl.dA, sl.db, sl.dG, sl.dh, nullptr,
                                   nullptr, nullptr, nullptr, nullptr, nullptr, cfg, sl.ws, sl.ws_bytes,
                                   reinterpret_cast<qpb_stream_t>(sc));
      if (st) break;
    }
    e = e ? e : cudaEventRecord(E(c, kDone), sc);
    // copy out: x as soon as the forward is done, the gradients after the backward
    e = e ? e : cudaStreamWaitEvent(s_out, E(c, kX), 0);
    if (converged) e = e ? e : copy_out(converged + lo, sl.conv, cnt * 4, s_out);
    if (iters) e = e ? e : copy_out(iters + lo, sl.iters, cnt * 4, s_out);
    e = e ? e : copy_out(x + lo * n, sl.x, cnt * n * 8, s_out);
    e = e ? e : cudaStreamWaitEvent(s_out, E(c, kDone), 0);
    e = e ? e : copy_out(dQ + lo * n * n, sl.dQ, cnt * n * n * 8, s_out);
    e = e ? e : copy_out(dq + lo * n, sl.dq, cnt * n * 8, s_out);
    e = e ? e : copy_out(dA + lo * m * n, sl.dA, cnt * m * n * 8, s_out);
    e = e ? e : copy_out(db + lo * m, sl.db, cnt * m * 8, s_out);
    e = e ? e : copy_out(dG + lo * p * n, sl.dG, cnt * p * n * 8, s_out);
    e = e ? e : copy_out(dh + lo * p, sl.dh, cnt * p * 8, s_out);
    e = e ? e : cudaEventRecord(E(c, kOut), s_out);
    if (e != cudaSuccess) st = QPB_ERR_CUDA;
  }
  // join: `stream` continues after everything queued on the internal streams
  // (also on error, so that nothing queued here outlives the caller's view of
  // the stream)
  if (ev.size() == n_ev) {
    for (int k = 0; k < kStreams; ++k) {
      cudaEvent_t j = ev[(size_t)chunks * kKinds + 1 + k];
      if (cudaEventRecord(j, ss[k]) != cudaSuccess || cudaStreamWaitEvent(s0, j, 0) != cudaSuccess)
        st = st ? st : QPB_ERR_CUDA;
    }
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  return st;
}

}  // extern "C"
