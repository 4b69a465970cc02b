// qpb_plan.cu -- uneven (packed) batches: instances of different (n, m, p)
// solved in one call.  A plan bins the instances by kernel variant once on
// the host; every call then runs one persistent launch per bin.  The bin
// launches are forked from the caller's stream onto the plan's own streams
// and joined back with events, so they run concurrently and a CUDA graph
// captures the whole call as one fork/join graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/qpb.h"
#include "qpb_kernel.cuh"
#include "qpb_host.h"

namespace qpb {

struct PlanBin {
  Plan launch;       // kernel, grid, shared memory, arena size, workspace bytes
  int count;         // instances in the bin
  long list_off;     // first entry of the bin in the device instance list
  size_t ws_off;     // bin's slice of the caller's workspace
  double work;       // estimated cost (for launch order)
  int n_max, m_max, p_max;
  int key;           // kernel-variant key (bin_key)
};

}  // namespace qpb

struct qpb_plan_st {
  int batch;
  int device;
  qpb_config cfg;
  std::vector<int32_t> shapes;  // host copy
  std::vector<int64_t> offs;    // host copy
  int64_t totals[6];            // packed lengths of Q, q, A, b, G, h
  int32_t *d_shapes = nullptr;
  int64_t *d_offs = nullptr;
  int32_t *d_list = nullptr;
  std::vector<qpb::PlanBin> bins;
  std::vector<cudaStream_t> streams;  // one per bin after the first
  std::vector<cudaEvent_t> events;    // fork + one per extra bin
  size_t ws_bytes = 0;
};

namespace qpb {

static void free_plan(qpb_plan* pl) {
  if (!pl) return;
  for (cudaStream_t s : pl->streams) cudaStreamDestroy(s);
  for (cudaEvent_t e : pl->events) cudaEventDestroy(e);
  cudaFree(pl->d_shapes);
  cudaFree(pl->d_offs);
  cudaFree(pl->d_list);
  delete pl;
}

// Bin key: the kernel variant an instance runs on.
static int bin_key(const qpb_dims& d, const qpb_config& c) {
  const int np = warp_np(d);
  if (np && (c.team_threads == 0 || c.team_threads == 32)) return np;  // 8, 16, 32 (FP64 or mixed)
  const int kc = chunks_for(d.n > d.m ? d.n : d.m);
  return 1000 + kc;  // team kernel, KC register chunks
}

// Workspace slices of the bins, in launch order.
static void layout_workspace(qpb_plan* pl) {
  size_t ws = 0;
  for (PlanBin& b : pl->bins) {
    b.ws_off = ws;
    ws += (b.launch.ws_bytes + 255) & ~size_t(255);
  }
  pl->ws_bytes = ws ? ws : 256;
}

}  // namespace qpb

using namespace qpb;

extern "C" {

int qpb_plan_create(qpb_plan** out, int32_t batch, const int32_t* shapes, const qpb_config* cfg) {
  if (!out) return QPB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (batch < 0 || (batch > 0 && !shapes)) return QPB_ERR_INVALID_ARGUMENT;
  const qpb_config c = resolve_config(cfg);
  if (cfg) {
    const qpb_dims probe{1, 1, 0, 1};
    const int st = check_common(kOpSolve, &probe, cfg);
    if (st) return st;
  }
  for (int i = 0; i < batch; ++i) {
    const qpb_dims d{1, shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2]};
    int st = check_common(kOpSolve, &d, nullptr);
    if (st) return st;
    if (d.p < 1) return QPB_ERR_UNSUPPORTED;  // packed batches carry inequalities (relax/VJP need them)
  }
  qpb_plan* pl = new (std::nothrow) qpb_plan_st();
  if (!pl) return QPB_ERR_CUDA;
  pl->batch = batch;
  pl->cfg = c;
  if (cudaGetDevice(&pl->device) != cudaSuccess) {
    delete pl;
    return QPB_ERR_CUDA;
  }
  pl->shapes.assign(shapes, shapes + 3 * (size_t)batch);
  pl->offs.resize(6 * (size_t)batch);
  int64_t cur[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < batch; ++i) {
    const int64_t n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    for (int k = 0; k < 6; ++k) pl->offs[6 * (size_t)i + k] = cur[k];
    cur[0] += n * n; cur[1] += n; cur[2] += m * n; cur[3] += m; cur[4] += p * n; cur[5] += p;
  }
  std::memcpy(pl->totals, cur, sizeof(cur));
  // group instances by kernel variant
  std::vector<int> keys(batch);
  std::vector<int> uniq;
  for (int i = 0; i < batch; ++i) {
    const qpb_dims d{1, shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2]};
    keys[i] = bin_key(d, c);
    if (std::find(uniq.begin(), uniq.end(), keys[i]) == uniq.end()) uniq.push_back(keys[i]);
  }
  std::vector<int32_t> list;
  list.reserve(batch);
  size_t ws = 0;
  for (int key : uniq) {
    PlanBin b{};
    b.list_off = (long)list.size();
    double work = 0.0;
    for (int i = 0; i < batch; ++i) {
      if (keys[i] != key) continue;
      list.push_back(i);
      const double n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
      b.n_max = std::max(b.n_max, (int)n);
      b.m_max = std::max(b.m_max, (int)m);
      b.p_max = std::max(b.p_max, (int)p);
      work += p * n * n + n * n * n / 3.0 + 2.0 * m * n * n;
    }
    b.count = (int)(list.size() - b.list_off);
    b.work = work;
    // heaviest instances first: the persistent teams pull them in list
    // order, so the launch ends on light instances instead of a long tail
    auto inst_work = [&](int32_t i) {
      const double n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
      return p * n * n + n * n * n / 3.0 + 2.0 * m * n * n;
    };
    std::stable_sort(list.begin() + b.list_off, list.end(),
                     [&](int32_t x, int32_t y) { return inst_work(x) > inst_work(y); });
    const qpb_dims dm{b.count, b.n_max, b.m_max, b.p_max};
    b.key = key;
    // size the launch for the largest member; the backward op needs the same
    // arena.  A launch shape tuned earlier on this device for a bin with the
    // same largest (n, m, p) is reused (make_plan looks it up).
    int st = make_plan(kOpSolve, dm, c, &b.launch);
    if (st) {
      free_plan(pl);
      return st;
    }
    b.ws_off = ws;
    ws += (b.launch.ws_bytes + 255) & ~size_t(255);
    pl->bins.push_back(b);
  }
  std::sort(pl->bins.begin(), pl->bins.end(), [](const PlanBin& x, const PlanBin& y) { return x.work > y.work; });
  layout_workspace(pl);
  if (batch > 0) {
    if (cudaMalloc(&pl->d_shapes, sizeof(int32_t) * pl->shapes.size()) != cudaSuccess ||
        cudaMalloc(&pl->d_offs, sizeof(int64_t) * pl->offs.size()) != cudaSuccess ||
        cudaMalloc(&pl->d_list, sizeof(int32_t) * list.size()) != cudaSuccess ||
        cudaMemcpy(pl->d_shapes, pl->shapes.data(), sizeof(int32_t) * pl->shapes.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(pl->d_offs, pl->offs.data(), sizeof(int64_t) * pl->offs.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(pl->d_list, list.data(), sizeof(int32_t) * list.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      free_plan(pl);
      return QPB_ERR_CUDA;
    }
  }
  cudaEvent_t fork;
  if (cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess) {
    free_plan(pl);
    return QPB_ERR_CUDA;
  }
  pl->events.push_back(fork);
  for (size_t b = 1; b < pl->bins.size(); ++b) {
    cudaStream_t s;
    cudaEvent_t e;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      free_plan(pl);
      return QPB_ERR_CUDA;
    }
    pl->streams.push_back(s);
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      free_plan(pl);
      return QPB_ERR_CUDA;
    }
    pl->events.push_back(e);
  }
  *out = pl;
  return QPB_OK;
}

int qpb_plan_destroy(qpb_plan* plan) {
  free_plan(plan);
  return QPB_OK;
}

size_t qpb_plan_workspace_size(const qpb_plan* plan) { return plan ? plan->ws_bytes : 0; }

int32_t qpb_plan_num_bins(const qpb_plan* plan) { return plan ? (int32_t)plan->bins.size() : 0; }

}  // extern "C"

namespace qpb {

// Launch every bin of the plan for op (fields of P other than the packing
// fields, batch and workspace are set by the caller).
static int launch_packed(const qpb_plan* pl, Params P, void* ws, size_t ws_bytes, qpb_stream_t stream) {
  if (!pl) return QPB_ERR_INVALID_ARGUMENT;
  if (pl->batch == 0) return QPB_OK;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != pl->device) return QPB_ERR_INVALID_ARGUMENT;
  if (!ws || ws_bytes < pl->ws_bytes || (reinterpret_cast<uintptr_t>(ws) & 255)) return QPB_ERR_WORKSPACE;
  cudaStream_t s0 = reinterpret_cast<cudaStream_t>(stream);
  P.shapes = pl->d_shapes;
  P.offs = pl->d_offs;
  P.mixed = pl->cfg.precision == QPB_PRECISION_MIXED;
  P.pivot_max = pl->cfg.pivot_max;
  P.max_sweeps = pl->cfg.max_sweeps;
  P.stats = pl->cfg.stats;
  if (pl->bins.size() > 1 && cudaEventRecord(pl->events[0], s0) != cudaSuccess) return QPB_ERR_CUDA;
  for (size_t k = 0; k < pl->bins.size(); ++k) {
    const PlanBin& b = pl->bins[k];
    cudaStream_t s = k == 0 ? s0 : pl->streams[k - 1];
    if (k > 0 && cudaStreamWaitEvent(s, pl->events[0], 0) != cudaSuccess) return QPB_ERR_CUDA;
    unsigned char* wsb = reinterpret_cast<unsigned char*>(ws) + b.ws_off;
    Params Q = P;
    Q.batch = b.count;
    Q.n = b.n_max;
    Q.m = b.m_max;
    Q.p = b.p_max;
    Q.list = pl->d_list + b.list_off;
    const int st = enqueue(b.launch, Q, wsb, b.launch.grid, s);
    if (st != QPB_OK) return st;
    if (k > 0) {
      if (cudaEventRecord(pl->events[k], s) != cudaSuccess) return QPB_ERR_CUDA;
      if (cudaStreamWaitEvent(s0, pl->events[k], 0) != cudaSuccess) return QPB_ERR_CUDA;
    }
  }
  return QPB_OK;
}

}  // namespace qpb

extern "C" {

int qpb_plan_totals(const qpb_plan* plan, int64_t totals[6]) {
  if (!plan || !totals) return QPB_ERR_INVALID_ARGUMENT;
  std::memcpy(totals, plan->totals, sizeof(plan->totals));
  return QPB_OK;
}

int qpb_solve_qp_packed(const qpb_plan* plan, const double* Q, const double* q, const double* A, const double* b,
                        const double* G, const double* h, double solver_tol, double* x, double* s, double* z,
                        double* y, int32_t* converged, int32_t* iters, void* workspace, size_t workspace_bytes,
                        qpb_stream_t stream) {
  if (!plan) return QPB_ERR_INVALID_ARGUMENT;
  const int64_t* t = plan->totals;
  if (!ok_ptr(Q, t[0]) || !ok_ptr(q, t[1]) || !ok_ptr(A, t[2]) || !ok_ptr(b, t[3]) || !ok_ptr(G, t[4]) ||
      !ok_ptr(h, t[5]) || !ok_ptr(x, t[1]) || !ok_ptr(s, t[5]) || !ok_ptr(z, t[5]) || !ok_ptr(y, t[3]) ||
      (plan->batch && (!converged || !iters)))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpSolve;
  P.tol = solver_tol;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.out[0] = x; P.out[1] = s; P.out[2] = z; P.out[3] = y;
  P.conv = converged;
  P.iters = iters;
  return launch_packed(plan, P, workspace, workspace_bytes, stream);
}

int qpb_solve_qp_primal_bwd_packed(const qpb_plan* plan, const double* Q, const double* q, const double* A,
                                   const double* b, const double* G, const double* h, const double* x,
                                   const double* s, const double* z, const double* y, const double* dl_dx,
                                   double solver_tol, double target_kappa, double* dQ, double* dq, double* dA,
                                   double* db, double* dG, double* dh, int32_t* converged, int32_t* iters,
                                   void* workspace, size_t workspace_bytes, qpb_stream_t stream) {
  if (!plan) return QPB_ERR_INVALID_ARGUMENT;
  const int64_t* t = plan->totals;
  if (!ok_ptr(Q, t[0]) || !ok_ptr(q, t[1]) || !ok_ptr(A, t[2]) || !ok_ptr(b, t[3]) || !ok_ptr(G, t[4]) ||
      !ok_ptr(h, t[5]) || !ok_ptr(x, t[1]) || !ok_ptr(s, t[5]) || !ok_ptr(z, t[5]) || !ok_ptr(y, t[3]) ||
      !ok_ptr(dl_dx, t[1]) || !ok_ptr(dQ, t[0]) || !ok_ptr(dq, t[1]) || !ok_ptr(dA, t[2]) || !ok_ptr(db, t[3]) ||
      !ok_ptr(dG, t[4]) || !ok_ptr(dh, t[5]))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpBwd;
  P.tol = solver_tol;
  P.kappa = target_kappa;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.in[0] = x; P.in[1] = s; P.in[2] = z; P.in[3] = y;
  P.gx = dl_dx;
  P.dQ = dQ; P.dq = dq; P.dA = dA; P.db = db; P.dG = dG; P.dh = dh;
  P.conv = converged;
  P.iters = iters;
  return launch_packed(plan, P, workspace, workspace_bytes, stream);
}

}  // extern "C"

extern "C" {

// Tuning times one bin at a time from the start of the workspace (the
// largest candidate of any bin), and afterwards every bin keeps its tuned
// shape, laid out one after another: the bound is the sum over bins of each
// bin's largest candidate (a tuned shape may need more than the heuristic's,
// e.g. a global arena instead of shared memory).
size_t qpb_plan_tune_workspace_size(const qpb_plan* plan) {
  if (!plan) return 0;
  size_t total = 0;
  for (const PlanBin& b : plan->bins) {
    const qpb_dims d{b.count, b.n_max, b.m_max, b.p_max};
    total += (tune_workspace(kOpSolve, d, plan->cfg) + 255) & ~size_t(255);
  }
  return total > plan->ws_bytes ? total : plan->ws_bytes;
}

int qpb_plan_tune(qpb_plan* plan, const double* Q, const double* q, const double* A, const double* b,
                  const double* G, const double* h, double solver_tol, double* x, double* s, double* z, double* y,
                  int32_t* converged, int32_t* iters, void* workspace, size_t workspace_bytes,
                  qpb_stream_t stream) {
  if (!plan) return QPB_ERR_INVALID_ARGUMENT;
  const int64_t* t = plan->totals;
  if (!ok_ptr(Q, t[0]) || !ok_ptr(q, t[1]) || !ok_ptr(A, t[2]) || !ok_ptr(b, t[3]) || !ok_ptr(G, t[4]) ||
      !ok_ptr(h, t[5]) || !ok_ptr(x, t[1]) || !ok_ptr(s, t[5]) || !ok_ptr(z, t[5]) || !ok_ptr(y, t[3]) ||
      (plan->batch && (!converged || !iters)))
    return QPB_ERR_INVALID_ARGUMENT;
  if (plan->batch == 0) return QPB_OK;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != plan->device) return QPB_ERR_INVALID_ARGUMENT;
  if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255)) return QPB_ERR_WORKSPACE;
  if (plan->cfg.team_threads != 0) {  // the caller fixed the launch shape
    if (workspace_bytes < plan->ws_bytes) return QPB_ERR_WORKSPACE;
    return qpb_solve_qp_packed(plan, Q, q, A, b, G, h, solver_tol, x, s, z, y, converged, iters, workspace,
                               workspace_bytes, stream);
  }
  Params P{};
  P.op = kOpSolve;
  P.tol = solver_tol;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.out[0] = x; P.out[1] = s; P.out[2] = z; P.out[3] = y;
  P.conv = converged;
  P.iters = iters;
  P.shapes = plan->d_shapes;
  P.offs = plan->d_offs;
  P.mixed = plan->cfg.precision == QPB_PRECISION_MIXED;
  P.pivot_max = plan->cfg.pivot_max;
  P.max_sweeps = plan->cfg.max_sweeps;
  for (PlanBin& bn : plan->bins) {
    const qpb_dims d{bn.count, bn.n_max, bn.m_max, bn.p_max};
    P.list = plan->d_list + bn.list_off;  // the bin's instances, heaviest first
    LaunchChoice best{};
    const int status = tune_pick(P, kOpSolve, d, plan->cfg, workspace, workspace_bytes, stream, &best);
    if (status != QPB_OK) return status;
    Plan full;  // the chosen shape, sized for the whole bin
    if (make_plan(kOpSolve, d, plan->cfg, &full, &best) == QPB_OK) {
      bn.launch = full;
      tune_record(kOpSolve, d, plan->cfg, best);
    }
  }
  layout_workspace(plan);
  if (workspace_bytes < plan->ws_bytes) return QPB_ERR_WORKSPACE;
  // outputs for the whole batch with the tuned plan
  return qpb_solve_qp_packed(plan, Q, q, A, b, G, h, solver_tol, x, s, z, y, converged, iters, workspace,
                             workspace_bytes, stream);
}

int32_t qpb_plan_bin_info(const qpb_plan* plan, int32_t bin, int32_t info[8]) {
  if (!plan || !info || bin < 0 || bin >= (int32_t)plan->bins.size()) return QPB_ERR_INVALID_ARGUMENT;
  const PlanBin& b = plan->bins[bin];
  const int sms = device_sms();
  info[0] = b.count;
  info[1] = b.n_max;
  info[2] = b.m_max;
  info[3] = b.p_max;
  info[4] = b.launch.threads / b.launch.teams;  // threads per instance team
  info[5] = b.launch.in_smem ? 1 : 2;
  info[6] = b.launch.gstage_rows;
  info[7] = sms > 0 ? (b.launch.grid + sms - 1) / sms : 0;  // resident CTAs per SM
  return QPB_OK;
}

}  // extern "C"
