// qpb_capi.cu -- persistent kernels, launch planning and the extern "C"
// entry points declared in include/qpb.h.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/qpb.h"
#include "qpb_host.h"
#include "qpb_kernel.cuh"
#include "qpb_warpqp.cuh"

namespace qpb {

// ------------------------------------------------------------- planning

static KernelFn pick_kernel(bool elastic, bool mixed, int NT, int KC) {
  if (elastic) return mixed ? kernel_elastic_mixed(NT, KC) : kernel_elastic_f64(NT, KC);
  return mixed ? kernel_std_mixed(NT, KC) : kernel_std_f64(NT, KC);
}

int chunks_for(int k) {
  const int c = (k + 31) / 32;
  return c <= 1 ? 1 : c <= 2 ? 2 : c <= 4 ? 4 : 8;
}

// Threads per instance.  FP64: 128 (four warps saturate the FP64 tensor
// pipe; several instances share an SM and hide each other's serial steps).
// Mixed keeps the per-column FP32 factorisation, which wants more threads
// for large n.
static int auto_team(int n, int KC, bool mixed) {
  if (n <= 16 && KC == 1) return 32;
  if (mixed && KC >= 8) return 256;
  if (mixed && KC >= 4) return n > 96 ? 256 : 128;
  return 128;
}

struct DevInfo {
  int sms = 0, smem_optin = 0;
  bool ok = false;
};

static DevInfo dev_info() {
  static DevInfo cache[64];
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DevInfo{};
  std::lock_guard<std::mutex> lk(mu);
  if (!cache[dev].ok) {
    DevInfo d;
    if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return DevInfo{};
    if (cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      return DevInfo{};
    d.ok = true;
    cache[dev] = d;
  }
  return cache[dev];
}

int device_sms() {
  const DevInfo d = dev_info();
  return d.ok ? d.sms : 0;
}

// Per (device, kernel, block, shared memory): raises the kernel's dynamic
// shared-memory limit once and caches its occupancy, so planning a launch
// makes no CUDA call after the first time (those calls can serialize work
// in flight on other streams).
struct OccKey {
  int dev;
  const void* fn;
  int threads;
  size_t smem;
};
static int occupancy(const void* fn, int threads, size_t smem, int* per_sm) {
  static std::mutex mu;
  static OccKey keys[256];
  static int vals[256];
  static int count = 0;
  // per (device, kernel): the dynamic shared-memory limit set so far.  The
  // limit only ever grows, so every earlier plan of the kernel stays valid.
  static OccKey limits[128];
  static int nlimits = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return QPB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(mu);
  for (int i = 0; i < count; ++i)
    if (keys[i].dev == dev && keys[i].fn == fn && keys[i].threads == threads && keys[i].smem == smem) {
      *per_sm = vals[i];
      return QPB_OK;
    }
  // the default dynamic limit is 48 KB minus the kernel's static shared
  // memory, so raise it for any request
  if (smem > 0) {
    int li = -1;
    for (int i = 0; i < nlimits; ++i)
      if (limits[i].dev == dev && limits[i].fn == fn) li = i;
    if (li < 0 || limits[li].smem < smem) {
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return QPB_ERR_CUDA;
      if (li >= 0) {
        limits[li].smem = smem;
      } else if (nlimits < 128) {
        limits[nlimits++] = OccKey{dev, fn, 0, smem};
      } else {
        return QPB_ERR_CUDA;
      }
    }
  }
  int v = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, fn, threads, smem) != cudaSuccess) return QPB_ERR_CUDA;
  if (count < 256) {
    keys[count] = OccKey{dev, fn, threads, smem};
    vals[count] = v;
    ++count;
  }
  *per_sm = v;
  return QPB_OK;
}

// Padded column count of the one-warp-per-instance kernel, or 0 when the
// instance does not fit it (n <= 32, m <= NP / 4).
int warp_np(const qpb_dims& d) {
  const int np = d.n <= 8 ? 8 : d.n <= 16 ? 16 : d.n <= 32 ? 32 : 0;
  return (np && d.m <= np / 4) ? np : 0;
}

// ------------------------------------------------------- tuned choices

struct TuneEntry {
  int dev, elastic, precision, n, m, p;
  LaunchChoice ch;
};
static std::mutex g_tune_mu;
static TuneEntry g_tune[512];
static int g_tune_count = 0;

void tune_record(int op, const qpb_dims& d, const qpb_config& cfg, const LaunchChoice& ch) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const TuneEntry e{dev, op_is_elastic(op) ? 1 : 0, cfg.precision, d.n, d.m, d.p, ch};
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (int i = 0; i < g_tune_count; ++i) {
    TuneEntry& t = g_tune[i];
    if (t.dev == e.dev && t.elastic == e.elastic && t.precision == e.precision && t.n == e.n && t.m == e.m &&
        t.p == e.p) {
      t.ch = ch;
      return;
    }
  }
  if (g_tune_count < 512) g_tune[g_tune_count++] = e;
}

bool tune_lookup(int op, const qpb_dims& d, const qpb_config& cfg, LaunchChoice* ch) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  const int el = op_is_elastic(op) ? 1 : 0;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (int i = 0; i < g_tune_count; ++i) {
    const TuneEntry& t = g_tune[i];
    if (t.dev == dev && t.elastic == el && t.precision == cfg.precision && t.n == d.n && t.m == d.m &&
        t.p == d.p) {
      *ch = t.ch;
      return true;
    }
  }
  return false;
}

int make_plan(int op, const qpb_dims& d, const qpb_config& cfg, Plan* pl, const LaunchChoice* ch) {
  LaunchChoice tuned{};
  if (!ch && cfg.team_threads == 0 && tune_lookup(op, d, cfg, &tuned)) ch = &tuned;
  const bool elastic = op_is_elastic(op);
  const bool mixed = cfg.precision == QPB_PRECISION_MIXED;
  const DevInfo di = dev_info();
  if (!di.ok) return QPB_ERR_CUDA;
  pl->gstage_rows = 0;
  pl->fn_resume = nullptr;
  pl->hlist_off = pl->hstate_off = pl->hiter_off = 0;
  pl->hstride = 0;
  const size_t smem_budget = (size_t)di.smem_optin - 1024;  // room for static shared + reserve
  const int np = warp_np(d);
  const int want_threads = ch && ch->team_threads ? ch->team_threads : cfg.team_threads;
  const int cap = ch ? ch->per_sm_cap : 0;
  if (!elastic && np && (want_threads == 0 || want_threads == 32)) {
    // one warp per instance (n_pad = 16, 32; mixed precision at every
    // n_pad) or four instances per warp in lockstep (n_pad = 8, FP64), four
    // warps per CTA; `teams` counts instances per CTA
    KernelFn gfn = mixed ? nullptr : kernel_group_f64(np);
    const int per_warp = gfn ? 32 / np : 1;
    KernelFn fn = gfn ? gfn : (mixed ? kernel_warp_mixed(np) : kernel_warp_f64(np));
    if (!fn) return QPB_ERR_UNSUPPORTED;
    size_t arena = (WarpArena::bytes(np, np / 4, d.p) + 255) & ~size_t(255);
    pl->fn = (const void*)fn;
    pl->NT = 32;
    pl->arena_bytes = arena;
    pl->teams = (kWarpKernelThreads / 32) * per_warp;
    pl->threads = kWarpKernelThreads;
    const bool fits = arena * pl->teams <= smem_budget;
    if (ch && ch->placement == 1 && !fits) return QPB_ERR_UNSUPPORTED;
    if (fits && !(ch && ch->placement == 2)) {
      pl->in_smem = 1;
      pl->smem_bytes = arena * pl->teams;
    } else {
      pl->in_smem = 0;
      pl->smem_bytes = 0;
    }
    int per_sm = 0;
    if (occupancy(pl->fn, pl->threads, pl->smem_bytes, &per_sm) != QPB_OK) return QPB_ERR_CUDA;
    if (per_sm < 1) return QPB_ERR_UNSUPPORTED;
    if (!pl->in_smem && per_sm > 4) per_sm = 4;
    if (cap > 0 && per_sm > cap) per_sm = cap;
    const long need = ((long)d.batch + pl->teams - 1) / pl->teams;
    long grid = (long)per_sm * di.sms;
    grid = grid > need ? need : grid;
    pl->grid = (int)(grid < 1 ? 1 : grid);
    pl->ws_bytes = kCounterBytes + (pl->in_smem ? 0 : (size_t)pl->grid * pl->teams * arena);
    if (mixed) {
      // instances whose FP32 factor is rejected continue on the FP64 kernel
      // (same arena layout), from their iterate in the hand-over region
      pl->fn_resume = (const void*)kernel_warp_f64(np);
      if (!pl->fn_resume) return QPB_ERR_UNSUPPORTED;
      int v = 0;  // (also raises the resume kernel's dynamic shared-memory limit)
      if (occupancy(pl->fn_resume, pl->threads, pl->smem_bytes, &v) != QPB_OK) return QPB_ERR_CUDA;
      if (v < 1) return QPB_ERR_UNSUPPORTED;
      const size_t B = (size_t)d.batch;
      pl->hstride = d.n + 2 * d.p + d.m;
      pl->hlist_off = (pl->ws_bytes + 255) & ~size_t(255);
      pl->hstate_off = pl->hlist_off + ((4 * B + 255) & ~size_t(255));
      pl->hiter_off = pl->hstate_off + ((12 * B + 255) & ~size_t(255));
      pl->ws_bytes = pl->hiter_off + 8 * B * (size_t)pl->hstride;
    }
    return QPB_OK;
  }
  const int KC = chunks_for(d.n > d.m ? d.n : d.m);
  int NT = want_threads ? want_threads : auto_team(d.n, KC, mixed);
  if (NT == 32 && KC > 1) NT = 128;
  if (NT == 256 && KC < 4) NT = 128;
  KernelFn fn = pick_kernel(elastic, mixed, NT, KC);
  if (!fn) return QPB_ERR_UNSUPPORTED;
  // dynamic shared memory left beside the kernel's static staging
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, (const void*)fn) != cudaSuccess) return QPB_ERR_CUDA;
  const size_t team_budget = smem_budget > fa.sharedSizeBytes ? smem_budget - fa.sharedSizeBytes : 0;
  size_t arena = elastic ? ElasticArena::bytes(d.n, d.p, mixed) : StdArena::bytes(d.n, d.m, d.p, mixed);
  arena = (arena + 255) & ~size_t(255);
  pl->fn = (const void*)fn;
  pl->NT = NT;
  pl->arena_bytes = arena;
  int teams = 1;
  if (NT == 32) {
    // several warp teams per CTA, as many as fit (up to 8)
    teams = (int)(team_budget / arena);
    teams = teams > 8 ? 8 : teams;
  }
  // The arena in shared memory, when it fits, unless (blocked FP64 path) an
  // arena in global memory with G streamed through shared memory keeps more
  // instances resident per SM: these kernels are latency-bound.
  int per_sm_smem = 0;
  if (teams >= 1 && arena * teams <= team_budget &&
      occupancy(pl->fn, NT * teams, arena * teams, &per_sm_smem) != QPB_OK)
    return QPB_ERR_CUDA;
  int gstage = 0, per_sm_global = 0;
  size_t gbytes = 0;
  if (NT > 32 && d.n > 32 && d.p > 0 && !mixed) {
    // stream G through shared memory in chunks of 32, 16 or 8 rows: the
    // largest chunk among those that keep the most instances per SM (or the
    // tuned chunk)
    const int ldg = (d.n + 3) & ~3;
    for (int rows = 32; rows >= 8; rows >>= 1) {
      if (ch && ch->gstage_rows && ch->gstage_rows != rows) continue;
      const size_t b = gstage_bytes(ldg, rows);
      if (b > team_budget) continue;
      int v = 0;
      if (occupancy(pl->fn, NT, b, &v) != QPB_OK) return QPB_ERR_CUDA;
      if (v > 4) v = 4;
      if (v > per_sm_global) {
        per_sm_global = v;
        gstage = rows;
        gbytes = b;
      }
    }
  }
  bool use_smem = per_sm_smem >= 1 && per_sm_smem >= per_sm_global;
  if (ch && ch->placement == 1) {
    if (per_sm_smem < 1) return QPB_ERR_UNSUPPORTED;
    use_smem = true;
  } else if (ch && ch->placement == 2) {
    use_smem = false;
  }
  if (use_smem) {
    pl->in_smem = 1;
    pl->teams = teams;
    pl->smem_bytes = arena * teams;
  } else {
    pl->in_smem = 0;
    pl->teams = NT == 32 ? 4 : 1;
    pl->smem_bytes = gbytes;
    pl->gstage_rows = gstage;
  }
  pl->threads = NT * pl->teams;
  int per_sm = 0;
  if (occupancy(pl->fn, pl->threads, pl->smem_bytes, &per_sm) != QPB_OK) return QPB_ERR_CUDA;
  if (per_sm < 1) return QPB_ERR_UNSUPPORTED;
  if (!pl->in_smem && per_sm > 4) per_sm = 4;
  if (cap > 0 && per_sm > cap) per_sm = cap;
  const long need = ((long)d.batch + pl->teams - 1) / pl->teams;
  long grid = (long)per_sm * di.sms;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  pl->grid = (int)grid;
  pl->ws_bytes = kCounterBytes + (pl->in_smem ? 0 : (size_t)grid * pl->teams * arena);
  return QPB_OK;
}

// Candidate launch shapes for the autotuner: the heuristic's own choice
// first, then the team sizes, arena placements, G chunk rows and resident-CTA
// caps (the occupancy limit and one below it) the kernels support for `d`.
static std::vector<LaunchChoice> tune_candidates(int op, const qpb_dims& d, const qpb_config& c) {
  std::vector<LaunchChoice> out;
  out.push_back(LaunchChoice{});
  const bool elastic = op_is_elastic(op);
  const bool mixed = c.precision == QPB_PRECISION_MIXED;
  const int KC = chunks_for(d.n > d.m ? d.n : d.m);
  std::vector<int> teams;
  if ((!elastic && warp_np(d)) || KC == 1) teams.push_back(32);
  teams.push_back(128);
  if (KC >= 4) teams.push_back(256);
  const int sms = device_sms();
  for (int nt : teams) {
    std::vector<LaunchChoice> shapes;
    shapes.push_back(LaunchChoice{nt, 1, 0, 0});
    if (nt > 32 && d.n > 32 && !mixed) {
      for (int rows : {32, 16, 8}) shapes.push_back(LaunchChoice{nt, 2, rows, 0});
    } else {
      shapes.push_back(LaunchChoice{nt, 2, 0, 0});
    }
    for (const LaunchChoice& sh : shapes) {
      Plan pl;
      if (make_plan(op, d, c, &pl, &sh) != QPB_OK) continue;
      const int per_sm = sms > 0 ? (pl.grid + sms - 1) / sms : 1;
      for (int cap = per_sm; cap >= 1 && cap >= per_sm - 1; --cap) {
        LaunchChoice ch = sh;
        ch.per_sm_cap = cap;
        out.push_back(ch);
      }
    }
  }
  return out;
}

size_t tune_workspace(int op, const qpb_dims& d, const qpb_config& cfg) {
  size_t need = kCounterBytes;
  for (const LaunchChoice& ch : tune_candidates(op, d, cfg)) {
    Plan pl;
    if (make_plan(op, d, cfg, &pl, &ch) == QPB_OK && pl.ws_bytes > need) need = pl.ws_bytes;
  }
  return need;
}

int tune_pick(Params P, int op, const qpb_dims& d, const qpb_config& cfg, void* ws, size_t ws_bytes,
              qpb_stream_t stream, LaunchChoice* best) {
  *best = LaunchChoice{};
  if (d.batch == 0) return QPB_OK;
  if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255)) return QPB_ERR_WORKSPACE;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return QPB_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return QPB_ERR_CUDA;
  }
  int status = QPB_OK;
  float best_per = 0.0f;
  bool have = false;
  P.n = d.n;
  P.m = d.m;
  P.p = d.p;
  for (const LaunchChoice& ch : tune_candidates(op, d, cfg)) {
    Plan pl;
    if (make_plan(op, d, cfg, &pl, &ch) != QPB_OK || pl.ws_bytes > ws_bytes) continue;
    // about two waves of the candidate's resident teams
    long sample = 2L * pl.grid * pl.teams;
    if (sample < 64) sample = 64;
    if (sample > d.batch) sample = d.batch;
    Params R = P;
    R.batch = (int)sample;
    const long need_teams = (sample + pl.teams - 1) / pl.teams;
    const int grid = (int)(need_teams < pl.grid ? need_teams : pl.grid);
    float ms = 0.0f;
    for (int rep = 0; rep < 2 && status == QPB_OK; ++rep) {  // the first run warms the caches
      if (cudaEventRecord(e0, st) != cudaSuccess || enqueue(pl, R, ws, grid, st) != QPB_OK ||
          cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
          cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
        status = QPB_ERR_CUDA;
    }
    if (status != QPB_OK) break;
    const float per = ms / (float)sample;  // the candidates' samples differ in size
    if (!have || per < best_per) {
      have = true;
      best_per = per;
      *best = ch;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return status;
}

qpb_config resolve_config(const qpb_config* c) {
  qpb_config r{};
  if (c) r = *c;
  if (r.pivot_max <= 0) r.pivot_max = 1e7;  // FP64 refactor above a pivot ratio of 1e7
  if (r.max_sweeps <= 0) r.max_sweeps = 8;
  return r;
}

static bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

// Pointer check: required when count > 0.
bool ok_ptr(const void* p, long count) { return count == 0 || (p != nullptr && aligned8(p)); }

int check_common(int op, const qpb_dims* d, const qpb_config* cfg) {
  if (!d) return QPB_ERR_INVALID_ARGUMENT;
  if (d->batch < 0 || d->n < 1 || d->m < 0 || d->p < 0) return QPB_ERR_INVALID_ARGUMENT;
  if (d->n > kMaxN || d->m > kMaxN) return QPB_ERR_UNSUPPORTED;
  if (cfg) {
    if (cfg->precision != QPB_PRECISION_AUTO && cfg->precision != QPB_PRECISION_MIXED &&
        cfg->precision != QPB_PRECISION_FP64)
      return QPB_ERR_INVALID_ARGUMENT;
    if (cfg->team_threads != 0 && cfg->team_threads != 32 && cfg->team_threads != 128 && cfg->team_threads != 256)
      return QPB_ERR_INVALID_ARGUMENT;
    if (cfg->max_sweeps < 0 || cfg->max_sweeps > 64) return QPB_ERR_INVALID_ARGUMENT;
    if (cfg->stats && !aligned8(cfg->stats) && (reinterpret_cast<uintptr_t>(cfg->stats) & 3))
      return QPB_ERR_INVALID_ARGUMENT;
  }
  if (op_is_elastic(op)) {
    if (d->m != 0) return QPB_ERR_INVALID_ARGUMENT;
    if (d->p < 1) return QPB_ERR_UNSUPPORTED;
  } else if (op != kOpSolve && op != kOpInit && d->p < 1) {
    return QPB_ERR_UNSUPPORTED;  // qpax's relax/VJP cannot run without inequalities
  }
  return QPB_OK;
}

// With `tune`, the launch shape is first chosen by timing the candidates
// (tune_pick) and recorded for these dims on this device.
static int launch(Params P, const qpb_dims* d, const qpb_config* cfg, void* ws, size_t ws_bytes,
                  qpb_stream_t stream, bool tune = false) {
  const qpb_config c = resolve_config(cfg);
  if (d->batch == 0) return QPB_OK;
  if (tune && c.team_threads == 0) {
    Params T = P;
    T.mixed = c.precision == QPB_PRECISION_MIXED;
    T.pivot_max = c.pivot_max;
    T.max_sweeps = c.max_sweeps;
    T.stats = c.stats;
    LaunchChoice best{};
    const int st = tune_pick(T, P.op, *d, c, ws, ws_bytes, stream, &best);
    if (st != QPB_OK) return st;
    tune_record(P.op, *d, c, best);
  }
  Plan pl;
  int st = make_plan(P.op, *d, c, &pl);
  if (st != QPB_OK) return st;
  if (!ws || ws_bytes < pl.ws_bytes || (reinterpret_cast<uintptr_t>(ws) & 255)) return QPB_ERR_WORKSPACE;
  P.batch = d->batch;
  P.n = d->n;
  P.m = d->m;
  P.p = d->p;
  P.mixed = c.precision == QPB_PRECISION_MIXED;
  P.pivot_max = c.pivot_max;
  P.max_sweeps = c.max_sweeps;
  P.stats = c.stats;
  return enqueue(pl, P, ws, pl.grid, reinterpret_cast<cudaStream_t>(stream));
}

int enqueue(const Plan& pl, Params P, void* ws, int grid, cudaStream_t s) {
  unsigned char* w = reinterpret_cast<unsigned char*>(ws);
  int* ctr = reinterpret_cast<int*>(ws);  // [0] work counter, [2] resume counter, [4] hand-overs
  P.counter = ctr;
  P.arena = w + kCounterBytes;
  P.arena_bytes = pl.arena_bytes;
  P.arena_in_smem = pl.in_smem;
  P.gstage_rows = pl.gstage_rows;
  P.resume = 0;
  if (pl.fn_resume) {
    P.hcount = ctr + 4;
    P.hlist = reinterpret_cast<int32_t*>(w + pl.hlist_off);
    P.hstate = reinterpret_cast<int32_t*>(w + pl.hstate_off);
    P.hiter = reinterpret_cast<double*>(w + pl.hiter_off);
    P.hstride = pl.hstride;
  }
  if (cudaMemsetAsync(ws, 0, 64, s) != cudaSuccess) return QPB_ERR_CUDA;
  void* args[] = {&P};
  if (cudaLaunchKernel(pl.fn, dim3(grid), dim3(pl.threads), args, pl.smem_bytes, s) != cudaSuccess)
    return QPB_ERR_CUDA;
  if (pl.fn_resume) {
    Params R = P;
    R.resume = 1;
    R.mixed = 0;
    R.counter = ctr + 2;
    void* rargs[] = {&R};
    if (cudaLaunchKernel(pl.fn_resume, dim3(grid), dim3(pl.threads), rargs, pl.smem_bytes, s) != cudaSuccess)
      return QPB_ERR_CUDA;
  }
  return QPB_OK;
}

}  // namespace qpb

using namespace qpb;

extern "C" {

int32_t qpb_version(void) { return 100; }

const char* qpb_status_string(int status) {
  switch (status) {
    case QPB_OK: return "ok";
    case QPB_ERR_INVALID_ARGUMENT: return "invalid argument";
    case QPB_ERR_UNSUPPORTED: return "unsupported shape or entry point";
    case QPB_ERR_WORKSPACE: return "workspace too small or misaligned";
    case QPB_ERR_CUDA: return "CUDA runtime error";
    default: return "unknown status";
  }
}

size_t qpb_workspace_size(int32_t op, const qpb_dims* dims, const qpb_config* cfg) {
  if (check_common(op, dims, cfg) != QPB_OK) return 0;
  const qpb_config c = resolve_config(cfg);
  qpb_dims d = *dims;
  if (d.batch == 0) return kCounterBytes;
  Plan pl;
  if (make_plan(op, d, c, &pl) != QPB_OK) return 0;
  return pl.ws_bytes;
}

}  // extern "C"

namespace qpb {

static int solve_qp_impl(const qpb_dims* d, const double* Q, const double* q, const double* A, const double* b,
                         const double* G, const double* h, double solver_tol, double* x, double* s, double* z,
                         double* y, int32_t* converged, int32_t* iters, const qpb_config* cfg, void* ws,
                         size_t ws_bytes, qpb_stream_t stream, bool tune) {
  int st = check_common(kOpSolve, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, m = d->m, p = d->p;
  if (!ok_ptr(Q, B * n * n) || !ok_ptr(q, B * n) || !ok_ptr(A, B * m * n) || !ok_ptr(b, B * m) ||
      !ok_ptr(G, B * p * n) || !ok_ptr(h, B * p) || !ok_ptr(x, B * n) || !ok_ptr(s, B * p) || !ok_ptr(z, B * p) ||
      !ok_ptr(y, B * m) || (B && (!converged || !iters)))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpSolve;
  P.tol = solver_tol;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.out[0] = x; P.out[1] = s; P.out[2] = z; P.out[3] = y;
  P.conv = converged;
  P.iters = iters;
  return launch(P, d, cfg, ws, ws_bytes, stream, tune);
}

}  // namespace qpb

extern "C" {

int qpb_solve_qp(const qpb_dims* d, const double* Q, const double* q, const double* A, const double* b,
                 const double* G, const double* h, double solver_tol, double* x, double* s, double* z, double* y,
                 int32_t* converged, int32_t* iters, const qpb_config* cfg, void* ws, size_t ws_bytes,
                 qpb_stream_t stream) {
  return solve_qp_impl(d, Q, q, A, b, G, h, solver_tol, x, s, z, y, converged, iters, cfg, ws, ws_bytes, stream,
                       false);
}

int qpb_tune_solve_qp(const qpb_dims* d, const double* Q, const double* q, const double* A, const double* b,
                      const double* G, const double* h, double solver_tol, double* x, double* s, double* z,
                      double* y, int32_t* converged, int32_t* iters, const qpb_config* cfg, void* ws,
                      size_t ws_bytes, qpb_stream_t stream) {
  return solve_qp_impl(d, Q, q, A, b, G, h, solver_tol, x, s, z, y, converged, iters, cfg, ws, ws_bytes, stream,
                       true);
}

size_t qpb_tune_workspace_size(int32_t op, const qpb_dims* dims, const qpb_config* cfg) {
  if (check_common(op, dims, cfg) != QPB_OK) return 0;
  const qpb_config c = resolve_config(cfg);
  return tune_workspace(op, *dims, c);
}

int qpb_initialize(const qpb_dims* d, const double* Q, const double* q, const double* A, const double* b,
                   const double* G, const double* h, double* x, double* s, double* z, double* y,
                   const qpb_config* cfg, void* ws, size_t ws_bytes, qpb_stream_t stream) {
  int st = check_common(kOpInit, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, m = d->m, p = d->p;
  if (!ok_ptr(Q, B * n * n) || !ok_ptr(q, B * n) || !ok_ptr(A, B * m * n) || !ok_ptr(b, B * m) ||
      !ok_ptr(G, B * p * n) || !ok_ptr(h, B * p) || !ok_ptr(x, B * n) || !ok_ptr(s, B * p) || !ok_ptr(z, B * p) ||
      !ok_ptr(y, B * m))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpInit;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.out[0] = x; P.out[1] = s; P.out[2] = z; P.out[3] = y;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

int qpb_relax_qp(const qpb_dims* d, const double* Q, const double* q, const double* A, const double* b,
                 const double* G, const double* h, const double* x_in, const double* s_in, const double* z_in,
                 const double* y_in, double solver_tol, double target_kappa, double* x, double* s, double* z,
                 double* y, int32_t* converged, int32_t* iters, const qpb_config* cfg, void* ws, size_t ws_bytes,
                 qpb_stream_t stream) {
  int st = check_common(kOpRelax, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, m = d->m, p = d->p;
  if (!ok_ptr(Q, B * n * n) || !ok_ptr(q, B * n) || !ok_ptr(A, B * m * n) || !ok_ptr(b, B * m) ||
      !ok_ptr(G, B * p * n) || !ok_ptr(h, B * p) || !ok_ptr(x_in, B * n) || !ok_ptr(s_in, B * p) ||
      !ok_ptr(z_in, B * p) || !ok_ptr(y_in, B * m) || !ok_ptr(x, B * n) || !ok_ptr(s, B * p) ||
      !ok_ptr(z, B * p) || !ok_ptr(y, B * m) || (B && (!converged || !iters)))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpRelax;
  P.tol = solver_tol;
  P.kappa = target_kappa;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.in[0] = x_in; P.in[1] = s_in; P.in[2] = z_in; P.in[3] = y_in;
  P.out[0] = x; P.out[1] = s; P.out[2] = z; P.out[3] = y;
  P.conv = converged;
  P.iters = iters;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

int qpb_diff_qp(const qpb_dims* d, const double* Q, const double* q, const double* A, const double* b,
                const double* G, const double* h, const double* x, const double* s, const double* lam,
                const double* nu, const double* dl_dx, double* dQ, double* dq, double* dA, double* db, double* dG,
                double* dh, const qpb_config* cfg, void* ws, size_t ws_bytes, qpb_stream_t stream) {
  int st = check_common(kOpAdjoint, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, m = d->m, p = d->p;
  if (!ok_ptr(Q, B * n * n) || !ok_ptr(q, B * n) || !ok_ptr(A, B * m * n) || !ok_ptr(b, B * m) ||
      !ok_ptr(G, B * p * n) || !ok_ptr(h, B * p) || !ok_ptr(x, B * n) || !ok_ptr(s, B * p) || !ok_ptr(lam, B * p) ||
      !ok_ptr(nu, B * m) || !ok_ptr(dl_dx, B * n) || !ok_ptr(dQ, B * n * n) || !ok_ptr(dq, B * n) ||
      !ok_ptr(dA, B * m * n) || !ok_ptr(db, B * m) || !ok_ptr(dG, B * p * n) || !ok_ptr(dh, B * p))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpAdjoint;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.in[0] = x; P.in[1] = s; P.in[2] = lam; P.in[3] = nu;
  P.gx = dl_dx;
  P.dQ = dQ; P.dq = dq; P.dA = dA; P.db = db; P.dG = dG; P.dh = dh;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

int qpb_solve_qp_primal_bwd(const qpb_dims* d, const double* Q, const double* q, const double* A,
                            const double* b, const double* G, const double* h, const double* x, const double* s,
                            const double* z, const double* y, const double* dl_dx, double solver_tol,
                            double target_kappa, double* dQ, double* dq, double* dA, double* db, double* dG,
                            double* dh, double* xr, double* sr, double* zr, double* yr, int32_t* converged,
                            int32_t* iters, const qpb_config* cfg, void* ws, size_t ws_bytes,
                            qpb_stream_t stream) {
  int st = check_common(kOpBwd, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, m = d->m, p = d->p;
  const bool want_iter = xr != nullptr;
  if (!ok_ptr(Q, B * n * n) || !ok_ptr(q, B * n) || !ok_ptr(A, B * m * n) || !ok_ptr(b, B * m) ||
      !ok_ptr(G, B * p * n) || !ok_ptr(h, B * p) || !ok_ptr(x, B * n) || !ok_ptr(s, B * p) || !ok_ptr(z, B * p) ||
      !ok_ptr(y, B * m) || !ok_ptr(dl_dx, B * n) || !ok_ptr(dQ, B * n * n) || !ok_ptr(dq, B * n) ||
      !ok_ptr(dA, B * m * n) || !ok_ptr(db, B * m) || !ok_ptr(dG, B * p * n) || !ok_ptr(dh, B * p))
    return QPB_ERR_INVALID_ARGUMENT;
  if (want_iter && (!ok_ptr(xr, B * n) || !ok_ptr(sr, B * p) || !ok_ptr(zr, B * p) || !ok_ptr(yr, B * m)))
    return QPB_ERR_INVALID_ARGUMENT;
  if (!ok_ptr(converged, 0) || !ok_ptr(iters, 0)) return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpBwd;
  P.tol = solver_tol;
  P.kappa = target_kappa;
  P.Q = Q; P.q = q; P.A = A; P.b = b; P.G = G; P.h = h;
  P.in[0] = x; P.in[1] = s; P.in[2] = z; P.in[3] = y;
  P.gx = dl_dx;
  if (want_iter) {
    P.out[0] = xr; P.out[1] = sr; P.out[2] = zr; P.out[3] = yr;
  }
  P.conv = converged;
  P.iters = iters;
  P.dQ = dQ; P.dq = dq; P.dA = dA; P.db = db; P.dG = dG; P.dh = dh;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

static bool ok_elastic_inputs(const qpb_dims* d, const double* Q, const double* q, const double* G,
                              const double* h, const double* pen) {
  const long B = d->batch, n = d->n, p = d->p;
  return ok_ptr(Q, B * n * n) && ok_ptr(q, B * n) && ok_ptr(G, B * p * n) && ok_ptr(h, B * p) && ok_ptr(pen, B);
}

static bool ok_iterate6(const qpb_dims* d, const double* const it[6]) {
  if (!it) return d->batch == 0;
  const long B = d->batch, n = d->n, p = d->p;
  if (!ok_ptr(it[0], B * n)) return false;
  for (int k = 1; k < 6; ++k)
    if (!ok_ptr(it[k], B * p)) return false;
  return true;
}

}  // extern "C"

namespace qpb {

static int solve_qp_elastic_impl(const qpb_dims* d, const double* Q, const double* q, const double* G,
                                 const double* h, const double* penalty, double solver_tol, double* x, double* t,
                                 double* s1, double* s2, double* z1, double* z2, int32_t* converged,
                                 int32_t* iters, const qpb_config* cfg, void* ws, size_t ws_bytes,
                                 qpb_stream_t stream, bool tune) {
  int st = check_common(kOpESolve, d, cfg);
  if (st) return st;
  double* out[6] = {x, t, s1, s2, z1, z2};
  if (!ok_elastic_inputs(d, Q, q, G, h, penalty) || !ok_iterate6(d, out) ||
      (d->batch && (!converged || !iters)))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpESolve;
  P.tol = solver_tol;
  P.Q = Q; P.q = q; P.G = G; P.h = h; P.penalty = penalty;
  for (int k = 0; k < 6; ++k) P.out[k] = out[k];
  P.conv = converged;
  P.iters = iters;
  return launch(P, d, cfg, ws, ws_bytes, stream, tune);
}

}  // namespace qpb

extern "C" {

int qpb_solve_qp_elastic(const qpb_dims* d, const double* Q, const double* q, const double* G, const double* h,
                         const double* penalty, double solver_tol, double* x, double* t, double* s1, double* s2,
                         double* z1, double* z2, int32_t* converged, int32_t* iters, const qpb_config* cfg,
                         void* ws, size_t ws_bytes, qpb_stream_t stream) {
  return solve_qp_elastic_impl(d, Q, q, G, h, penalty, solver_tol, x, t, s1, s2, z1, z2, converged, iters, cfg, ws,
                               ws_bytes, stream, false);
}

int qpb_tune_solve_qp_elastic(const qpb_dims* d, const double* Q, const double* q, const double* G,
                              const double* h, const double* penalty, double solver_tol, double* x, double* t,
                              double* s1, double* s2, double* z1, double* z2, int32_t* converged, int32_t* iters,
                              const qpb_config* cfg, void* ws, size_t ws_bytes, qpb_stream_t stream) {
  return solve_qp_elastic_impl(d, Q, q, G, h, penalty, solver_tol, x, t, s1, s2, z1, z2, converged, iters, cfg, ws,
                               ws_bytes, stream, true);
}

int qpb_initialize_elastic(const qpb_dims* d, const double* Q, const double* q, const double* G, const double* h,
                           const double* penalty, double* x, double* t, double* s1, double* s2, double* z1,
                           double* z2, const qpb_config* cfg, void* ws, size_t ws_bytes, qpb_stream_t stream) {
  int st = check_common(kOpEInit, d, cfg);
  if (st) return st;
  double* out[6] = {x, t, s1, s2, z1, z2};
  if (!ok_elastic_inputs(d, Q, q, G, h, penalty) || !ok_iterate6(d, out)) return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpEInit;
  P.Q = Q; P.q = q; P.G = G; P.h = h; P.penalty = penalty;
  for (int k = 0; k < 6; ++k) P.out[k] = out[k];
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

int qpb_relax_qp_elastic(const qpb_dims* d, const double* Q, const double* q, const double* G, const double* h,
                         const double* penalty, const double* const iterate_in[6], double solver_tol,
                         double target_kappa, double* const iterate_out[6], int32_t* converged, int32_t* iters,
                         const qpb_config* cfg, void* ws, size_t ws_bytes, qpb_stream_t stream) {
  int st = check_common(kOpERelax, d, cfg);
  if (st) return st;
  if (!ok_elastic_inputs(d, Q, q, G, h, penalty) || !ok_iterate6(d, iterate_in) ||
      !ok_iterate6(d, (const double* const*)iterate_out) || (d->batch && (!converged || !iters)))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpERelax;
  P.tol = solver_tol;
  P.kappa = target_kappa;
  P.Q = Q; P.q = q; P.G = G; P.h = h; P.penalty = penalty;
  for (int k = 0; k < 6 && d->batch; ++k) {
    P.in[k] = iterate_in[k];
    P.out[k] = iterate_out[k];
  }
  P.conv = converged;
  P.iters = iters;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

int qpb_diff_qp_elastic(const qpb_dims* d, const double* Q, const double* q, const double* G, const double* h,
                        const double* penalty, const double* const iterate[6], const double* dl_dx, double* dQ,
                        double* dq, double* dG, double* dh, const qpb_config* cfg, void* ws, size_t ws_bytes,
                        qpb_stream_t stream) {
  int st = check_common(kOpEAdjoint, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, p = d->p;
  if (!ok_elastic_inputs(d, Q, q, G, h, penalty) || !ok_iterate6(d, iterate) || !ok_ptr(dl_dx, B * n) ||
      !ok_ptr(dQ, B * n * n) || !ok_ptr(dq, B * n) || !ok_ptr(dG, B * p * n) || !ok_ptr(dh, B * p))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpEAdjoint;
  P.Q = Q; P.q = q; P.G = G; P.h = h; P.penalty = penalty;
  for (int k = 0; k < 6 && B; ++k) P.in[k] = iterate[k];
  P.gx = dl_dx;
  P.dQ = dQ; P.dq = dq; P.dG = dG; P.dh = dh;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

int qpb_solve_qp_elastic_primal_bwd(const qpb_dims* d, const double* Q, const double* q, const double* G,
                                    const double* h, const double* penalty, const double* const iterate[6],
                                    const double* dl_dx, double solver_tol, double target_kappa, double* dQ,
                                    double* dq, double* dG, double* dh, const qpb_config* cfg, void* ws,
                                    size_t ws_bytes, qpb_stream_t stream) {
  int st = check_common(kOpEBwd, d, cfg);
  if (st) return st;
  const long B = d->batch, n = d->n, p = d->p;
  if (!ok_elastic_inputs(d, Q, q, G, h, penalty) || !ok_iterate6(d, iterate) || !ok_ptr(dl_dx, B * n) ||
      !ok_ptr(dQ, B * n * n) || !ok_ptr(dq, B * n) || !ok_ptr(dG, B * p * n) || !ok_ptr(dh, B * p))
    return QPB_ERR_INVALID_ARGUMENT;
  Params P{};
  P.op = kOpEBwd;
  P.tol = solver_tol;
  P.kappa = target_kappa;
  P.Q = Q; P.q = q; P.G = G; P.h = h; P.penalty = penalty;
  for (int k = 0; k < 6 && B; ++k) P.in[k] = iterate[k];
  P.gx = dl_dx;
  P.dQ = dQ; P.dq = dq; P.dG = dG; P.dh = dh;
  return launch(P, d, cfg, ws, ws_bytes, stream);
}

}  // extern "C"
