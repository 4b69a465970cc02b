// qpb_host.h -- launch planning shared by the uniform entry points
// (qpb_capi.cu) and the packed-batch plans (qpb_plan.cu).
#pragma once
#include <stddef.h>

#include "../../include/qpb.h"
#include <cuda_runtime_api.h>

#include "qpb_params.h"

namespace qpb {

constexpr size_t kCounterBytes = 256;  // work counter slot at the head of every workspace
constexpr int kMaxN = 256;

// One persistent launch: kernel, shape, shared memory, arena and workspace.
struct Plan {
  const void* fn;
  int NT, threads, teams, grid;
  size_t arena_bytes, smem_bytes, ws_bytes;
  int in_smem;
  int gstage_rows;  // rows of G per shared-memory chunk (arena in global memory), 0: none
  // mixed precision on the one-warp kernels: the FP64 kernel that resumes
  // the instances the mixed launch hands over (nullptr: one launch), and
  // the hand-over region of the workspace (list, states, iterate blocks)
  const void* fn_resume;
  size_t hlist_off, hstate_off, hiter_off;
  int hstride;
};

// Enqueues the plan's launch(es) on `s`: zeroes the work counters, runs the
// persistent kernel over P.batch instances with `grid` CTAs and, for
// mixed-precision warp plans, the FP64 resume launch after it.  Sets P's
// counter, arena and hand-over fields from `ws`.
int enqueue(const Plan& pl, Params P, void* ws, int grid, cudaStream_t s);

// A launch shape chosen by the autotuner (zero fields: the heuristic's choice).
struct LaunchChoice {
  int team_threads;  // 32 (one warp per instance; warp kernels), 128, 256
  int placement;     // 1: arena in shared memory, 2: arena in global memory
  int gstage_rows;   // global arena: rows of G per shared-memory chunk (8, 16, 32)
  int per_sm_cap;    // resident CTAs per SM at most (grid = cap x SMs)
};

int warp_np(const qpb_dims& d);
int device_sms();  // SMs of the current device (0 on error)
int chunks_for(int k);
// Launch shape for `op` on dims `d`: `ch` (when given) overrides the
// heuristic; otherwise a tuned choice recorded for these dims on this device
// (tune_record) is used when cfg leaves team_threads automatic.
int make_plan(int op, const qpb_dims& d, const qpb_config& cfg, Plan* pl, const LaunchChoice* ch = nullptr);
// Per-device cache of tuned launch shapes, keyed by (op family, precision,
// n, m, p); batch sizes share an entry.
void tune_record(int op, const qpb_dims& d, const qpb_config& cfg, const LaunchChoice& ch);
bool tune_lookup(int op, const qpb_dims& d, const qpb_config& cfg, LaunchChoice* ch);
// Autotuner: times `P` (every field set but batch and the workspace fields;
// with P.list set, a packed bin whose list is ordered heaviest first) on its
// first instances under each candidate launch shape for dims `d` and returns
// the fastest per instance in `best`.  The host waits on `stream`.
int tune_pick(Params P, int op, const qpb_dims& d, const qpb_config& cfg, void* ws, size_t ws_bytes,
              qpb_stream_t stream, LaunchChoice* best);
// Workspace bytes the autotuner's largest candidate for `d` needs.
size_t tune_workspace(int op, const qpb_dims& d, const qpb_config& cfg);
qpb_config resolve_config(const qpb_config* c);
int check_common(int op, const qpb_dims* d, const qpb_config* cfg);
bool ok_ptr(const void* p, long count);

}  // namespace qpb
