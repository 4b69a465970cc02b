/*
 * qpb.h -- C ABI of libqpb, the batched interior-point QP solver for B200.
 *
 * Every entry point solves a batch of independent QPs of one shape
 *   min 1/2 x'Qx + q'x   s.t.  A x = b,  G x <= h
 * on the GPU, one persistent launch per call, stream-ordered, without host
 * synchronisation.  All array arguments are DEVICE pointers to FP64 row-major
 * data with a leading instance axis (the axis qpax users vmap over):
 *   Q[batch][n][n], q[batch][n], A[batch][m][n], b[batch][m],
 *   G[batch][p][n], h[batch][p]; outputs likewise.
 * Outputs must not alias inputs.  The caller owns every buffer; scratch
 * comes from `workspace` (size from qpb_workspace_size, 256-byte aligned).
 * Functions return QPB_OK or a qpb_status code and never abort; a rejected
 * call launches nothing.  Per-instance convergence is reported in
 * `converged` / `iters` exactly as qpax returns them.
 *
 * Each entry point replaces one function of qpax (kevin-tracy/qpax, v0.0.9);
 * the citation is on the declaration.  Defaults of the qpax Python API
 * (solver_tol, target_kappa) live in the Python layer, as in qpax.
 */
#ifndef QPB_H_
#define QPB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct CUstream_st;
typedef struct CUstream_st* qpb_stream_t; /* a cudaStream_t; NULL = legacy default stream */

typedef enum {
  QPB_OK = 0,
  QPB_ERR_INVALID_ARGUMENT = 1, /* null / misaligned pointer, negative size, bad option */
  QPB_ERR_UNSUPPORTED = 2,      /* shape outside the supported range (n, m <= 256), or an
                                   entry point qpax itself cannot evaluate (p == 0 relax) */
  QPB_ERR_WORKSPACE = 3,        /* workspace smaller than qpb_workspace_size() */
  QPB_ERR_CUDA = 4              /* a CUDA runtime call failed (launch, attributes) */
} qpb_status;

/* AUTO picks, per problem size, the fastest path that meets FP64 accuracy:
 * today the FP64 kernels (four instances per warp for n <= 8, m <= 2; one
 * warp per instance for n <= 32, m <= n_pad/4; one CTA per instance above).
 * MIXED factors in FP32 and refines every reduced KKT solve in FP64 (to
 * 1e-12 of the solution) against the FP64 operator; an instance whose FP32
 * factor has a pivot ratio max(d)/min(d) above pivot_max, or whose
 * refinement stalls, continues with FP64 factors.  For n <= 32, m <= n_pad/4
 * this is two launches on `stream`: the mixed one-warp kernel, then the
 * FP64 one-warp kernel resuming the instances handed over to it (the
 * workspace holds their iterates); above, one CTA per instance.  FP64 forces
 * FP64 factorisation. */
typedef enum { QPB_PRECISION_AUTO = 0, QPB_PRECISION_MIXED = 1, QPB_PRECISION_FP64 = 2 } qpb_precision;

typedef enum {
  QPB_OP_SOLVE = 0,
  QPB_OP_INITIALIZE = 1,
  QPB_OP_RELAX = 2,
  QPB_OP_PRIMAL_BWD = 3,
  QPB_OP_DIFF = 4,
  QPB_OP_ELASTIC_SOLVE = 5,
  QPB_OP_ELASTIC_INITIALIZE = 6,
  QPB_OP_ELASTIC_RELAX = 7,
  QPB_OP_ELASTIC_PRIMAL_BWD = 8,
  QPB_OP_ELASTIC_DIFF = 9
} qpb_op;

typedef struct {
  int32_t batch; /* number of instances (>= 0) */
  int32_t n;     /* variables (1..256) */
  int32_t m;     /* equality rows (0..256); 0 for the elastic entry points */
  int32_t p;     /* inequality rows (>= 0; >= 1 where noted) */
} qpb_dims;

/* Optional tuning; pass NULL for defaults. */
typedef struct {
  int32_t precision;    /* qpb_precision; default QPB_PRECISION_AUTO */
  int32_t team_threads; /* threads per instance: 0 = automatic, 32, 128 or 256
                           (128/256 force the one-CTA-per-instance kernel) */
  double pivot_max;     /* mixed: FP32 factor used while max(d)/min(d) <= pivot_max (0 = 1e7) */
  int32_t max_sweeps;   /* mixed: FP64 refinement sweeps per solve before FP64 refactor (0 = 8);
                           refinement also gives up early when the observed contraction
                           cannot reach 1e-12 within this many sweeps */
  int32_t* stats;       /* optional device int32[batch][4]: FP32 factorisations, FP64
                           factorisations, refinement sweeps, flag bits (1 FP32 factor
                           rejected, 2 refinement stalled, 4 FP64 pivot breakdown) */
} qpb_config;

/* Bytes of device workspace an entry point needs for these dims/config. */
size_t qpb_workspace_size(int32_t op, const qpb_dims* dims, const qpb_config* cfg);

/* qpax/pdip.py:181-251 solve_qp(Q, q, A, b, G, h, solver_tol) ->
 * (x, s, z, y, converged, iters).  Q is symmetrized, h = +-inf rows are
 * dropped (s = inf, z = 0 on return), p == 0 takes qpax's direct exits
 * (converged = 1, iters = 0). s, z may be NULL when p == 0, y when m == 0. */
int qpb_solve_qp(const qpb_dims* dims, const double* Q, const double* q, const double* A, const double* b,
                 const double* G, const double* h, double solver_tol, double* x, double* s, double* z, double* y,
                 int32_t* converged, int32_t* iters, const qpb_config* cfg, void* workspace,
                 size_t workspace_bytes, qpb_stream_t stream);

/* Autotuned solve_qp (no qpax counterpart; it stands where qpax compiles one
 * jit(vmap) per shape, qpax/pdip.py:208-217): times the launch shapes the
 * kernels support for `dims` -- threads per instance, arena placement, G
 * chunk rows, resident CTAs per SM -- on the first instances of this batch
 * (about two waves each; the host waits on `stream`), records the fastest
 * per instance for these (n, m, p) on this device, then solves the whole
 * batch with it; later qpb_solve_qp / qpb_workspace_size calls with these
 * (n, m, p) and automatic team_threads use the recorded shape.  Arguments
 * and outputs as qpb_solve_qp; `workspace` must hold
 * qpb_tune_workspace_size(QPB_OP_SOLVE, dims, cfg) bytes. */
int qpb_tune_solve_qp(const qpb_dims* dims, const double* Q, const double* q, const double* A, const double* b,
                      const double* G, const double* h, double solver_tol, double* x, double* s, double* z,
                      double* y, int32_t* converged, int32_t* iters, const qpb_config* cfg, void* workspace,
                      size_t workspace_bytes, qpb_stream_t stream);
/* Workspace bytes of the autotuned calls (the largest candidate's). */
size_t qpb_tune_workspace_size(int32_t op, const qpb_dims* dims, const qpb_config* cfg);

/* qpax/pdip.py:15-35 initialize(Q, q, A, b, G, h) -> (x, s, z, y), on the data as given. */
int qpb_initialize(const qpb_dims* dims, const double* Q, const double* q, const double* A, const double* b,
                   const double* G, const double* h, double* x, double* s, double* z, double* y,
                   const qpb_config* cfg, void* workspace, size_t workspace_bytes, qpb_stream_t stream);

/* qpax/pdip_relaxed.py:70-103 relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol, target_kappa)
 * -> (xr, sr, zr, yr, converged, iters).  Requires p >= 1. */
int qpb_relax_qp(const qpb_dims* dims, const double* Q, const double* q, const double* A, const double* b,
                 const double* G, const double* h, const double* x_in, const double* s_in, const double* z_in,
                 const double* y_in, double solver_tol, double target_kappa, double* x, double* s, double* z,
                 double* y, int32_t* converged, int32_t* iters, const qpb_config* cfg, void* workspace,
                 size_t workspace_bytes, qpb_stream_t stream);

/* qpax/diff_qp.py:20-46 diff_qp(Q, q, A, b, G, h, x, s, lam, nu, dl_dx)
 * -> (dQ, dq, dA, db, dG, dh) at a given (relaxed) iterate.  Requires p >= 1. */
int qpb_diff_qp(const qpb_dims* dims, const double* Q, const double* q, const double* A, const double* b,
                const double* G, const double* h, const double* x, const double* s, const double* lam,
                const double* nu, const double* dl_dx, double* dQ, double* dq, double* dA, double* db, double* dG,
                double* dh, const qpb_config* cfg, void* workspace, size_t workspace_bytes, qpb_stream_t stream);

/* Backward pass of qpax/diff_qp.py:49-82 solve_qp_primal (the custom_vjp):
 * relax_qp from the forward iterate (x, s, z, y) returned by qpb_solve_qp,
 * then diff_qp at the relaxed iterate, in one launch.  Only (x, s, z, y) is
 * kept between forward and backward; the factor is recomputed here.
 * xr..yr, converged, iters (of the relaxation) may be NULL.  Requires p >= 1. */
int qpb_solve_qp_primal_bwd(const qpb_dims* dims, const double* Q, const double* q, const double* A,
                            const double* b, const double* G, const double* h, const double* x, const double* s,
                            const double* z, const double* y, const double* dl_dx, double solver_tol,
                            double target_kappa, double* dQ, double* dq, double* dA, double* db, double* dG,
                            double* dh, double* xr, double* sr, double* zr, double* yr, int32_t* converged,
                            int32_t* iters, const qpb_config* cfg, void* workspace, size_t workspace_bytes,
                            qpb_stream_t stream);

/* qpax/elastic_qp.py:184-228 solve_qp_elastic(Q, q, G, h, penalty, solver_tol)
 * -> (x, t, s1, s2, z1, z2, converged, iters).  dims->m must be 0, p >= 1;
 * penalty holds one value per instance. */
int qpb_solve_qp_elastic(const qpb_dims* dims, const double* Q, const double* q, const double* G,
                         const double* h, const double* penalty, double solver_tol, double* x, double* t,
                         double* s1, double* s2, double* z1, double* z2, int32_t* converged, int32_t* iters,
                         const qpb_config* cfg, void* workspace, size_t workspace_bytes, qpb_stream_t stream);

/* Autotuned solve_qp_elastic: as qpb_tune_solve_qp, for the elastic entry
 * points (the recorded shape serves every elastic op with these dims);
 * workspace: qpb_tune_workspace_size(QPB_OP_ELASTIC_SOLVE, dims, cfg). */
int qpb_tune_solve_qp_elastic(const qpb_dims* dims, const double* Q, const double* q, const double* G,
                              const double* h, const double* penalty, double solver_tol, double* x, double* t,
                              double* s1, double* s2, double* z1, double* z2, int32_t* converged, int32_t* iters,
                              const qpb_config* cfg, void* workspace, size_t workspace_bytes,
                              qpb_stream_t stream);

/* qpax/elastic_qp.py:27-47 initialize_elastic -> (x, t, s1, s2, z1, z2). */
int qpb_initialize_elastic(const qpb_dims* dims, const double* Q, const double* q, const double* G,
                           const double* h, const double* penalty, double* x, double* t, double* s1, double* s2,
                           double* z1, double* z2, const qpb_config* cfg, void* workspace, size_t workspace_bytes,
                           qpb_stream_t stream);

/* qpax/elastic_qp.py:319-359 relax_qp_elastic from (x_in, t_in, s1_in, s2_in, z1_in, z2_in). */
int qpb_relax_qp_elastic(const qpb_dims* dims, const double* Q, const double* q, const double* G,
                         const double* h, const double* penalty, const double* const iterate_in[6],
                         double solver_tol, double target_kappa, double* const iterate_out[6],
                         int32_t* converged, int32_t* iters, const qpb_config* cfg, void* workspace,
                         size_t workspace_bytes, qpb_stream_t stream);

/* qpax/elastic_qp.py:381-417 diff_qp_elastic at iterate (x, t, s1, s2, lam1, lam2)
 * -> (dQ, dq, dG, dh) cropped to the caller's blocks. */
int qpb_diff_qp_elastic(const qpb_dims* dims, const double* Q, const double* q, const double* G,
                        const double* h, const double* penalty, const double* const iterate[6],
                        const double* dl_dx, double* dQ, double* dq, double* dG, double* dh,
                        const qpb_config* cfg, void* workspace, size_t workspace_bytes, qpb_stream_t stream);

/* Backward pass of qpax/elastic_qp.py:420-469 solve_qp_elastic_primal:
 * relax_qp_elastic from the forward iterate, then diff_qp_elastic. */
int qpb_solve_qp_elastic_primal_bwd(const qpb_dims* dims, const double* Q, const double* q, const double* G,
                                    const double* h, const double* penalty, const double* const iterate[6],
                                    const double* dl_dx, double solver_tol, double target_kappa, double* dQ,
                                    double* dq, double* dG, double* dh, const qpb_config* cfg, void* workspace,
                                    size_t workspace_bytes, qpb_stream_t stream);

/* ---- Uneven batches ----------------------------------------------------
 * A qpax user with instances of different shapes runs one jit(vmap(solve_qp))
 * per shape (qpax/pdip.py:208-217 branch on Python shapes).  Here one call
 * serves them all: instance i has its own (n_i, m_i, p_i), p_i >= 1, and each
 * array is the concatenation of the per-instance row-major arrays in instance
 * order (Q_0 Q_1 ... ; q_0 q_1 ... ; likewise A, b, G, h and the outputs).
 * A plan groups the instances by kernel variant once (host side, allocating
 * its small index tables and streams); each call then runs one persistent
 * launch per size bin, forked from `stream` onto the plan's streams and
 * joined back, so a CUDA graph captures the call whole.  A plan belongs to
 * the device current at its creation; calls sharing a plan must not overlap. */
typedef struct qpb_plan_st qpb_plan;

/* shapes: host int32[batch][3] = (n, m, p).  cfg as for the uniform calls. */
int qpb_plan_create(qpb_plan** plan, int32_t batch, const int32_t* shapes, const qpb_config* cfg);
/* Frees the plan's index tables, streams and events.  Calls already enqueued
 * finish first (the tables are freed with cudaFree, which waits for the
 * device), but a CUDA graph that captured a call with this plan reads those
 * tables at every launch: destroy the plan only after its last launch. */
int qpb_plan_destroy(qpb_plan* plan);
/* Workspace bytes a call with this plan needs (every op). */
size_t qpb_plan_workspace_size(const qpb_plan* plan);
/* Number of size bins (persistent launches per call). */
int32_t qpb_plan_num_bins(const qpb_plan* plan);
/* Packed lengths (elements) of Q, q, A, b, G, h. */
int qpb_plan_totals(const qpb_plan* plan, int64_t totals[6]);

/* Size-bin autotuner.  Replaces qpax's per-shape compilation
 * (qpax/pdip.py:208-217: one jit(vmap) per shape, each traced and compiled
 * by XLA) with a per-bin search of launch shapes: threads per instance (one
 * warp, 128 or 256), arena placement (shared or global memory), rows of G
 * per shared-memory chunk and resident CTAs per SM.  Each candidate the
 * kernels support for the bin's dims runs the forward solve on the bin's
 * heaviest instances (about two waves) on `stream`, timed with events (the
 * host waits); the fastest per instance becomes the bin's launch shape and
 * is recorded for this device, so later plans -- and uniform calls -- whose
 * bin has the same largest (n, m, p) start from it.  The whole batch is then
 * solved with the tuned plan: outputs as qpb_solve_qp_packed.  Plans created
 * with cfg->team_threads != 0 keep their launch shape (the call only
 * solves).  The plan's workspace size may change: query
 * qpb_plan_workspace_size again afterwards.  `workspace` must hold
 * qpb_plan_tune_workspace_size(plan) bytes. */
size_t qpb_plan_tune_workspace_size(const qpb_plan* plan);
int qpb_plan_tune(qpb_plan* plan, const double* Q, const double* q, const double* A, const double* b,
                  const double* G, const double* h, double solver_tol, double* x, double* s, double* z, double* y,
                  int32_t* converged, int32_t* iters, void* workspace, size_t workspace_bytes,
                  qpb_stream_t stream);
/* Launch shape of bin `bin` (0 .. num_bins - 1, launch order): info =
 * {instances, n_max, m_max, p_max, threads per instance, arena placement
 * (1 shared, 2 global memory), G chunk rows, resident CTAs per SM}. */
int32_t qpb_plan_bin_info(const qpb_plan* plan, int32_t bin, int32_t info[8]);

/* qpax/pdip.py:181-251 solve_qp over a packed batch (outputs packed like q, h, h, b). */
int qpb_solve_qp_packed(const qpb_plan* plan, const double* Q, const double* q, const double* A, const double* b,
                        const double* G, const double* h, double solver_tol, double* x, double* s, double* z,
                        double* y, int32_t* converged, int32_t* iters, void* workspace, size_t workspace_bytes,
                        qpb_stream_t stream);

/* qpax/diff_qp.py:74-79 backward of solve_qp_primal over a packed batch
 * (gradients packed like Q, q, A, b, G, h).  converged / iters (batch int32
 * each, may be NULL) receive the relaxation's outcome per instance
 * (qpax/pdip_relaxed.py:70-103). */
int qpb_solve_qp_primal_bwd_packed(const qpb_plan* plan, const double* Q, const double* q, const double* A,
                                   const double* b, const double* G, const double* h, const double* x,
                                   const double* s, const double* z, const double* y, const double* dl_dx,
                                   double solver_tol, double target_kappa, double* dQ, double* dq, double* dA,
                                   double* db, double* dG, double* dh, int32_t* converged, int32_t* iters,
                                   void* workspace, size_t workspace_bytes, qpb_stream_t stream);

/* qpb_solve_qp for callers that cannot allocate device memory.  No
 * counterpart in qpax: it exists for hosts where a solve must not call
 * cudaMalloc -- code recorded into a CUDA graph whose capture forbids
 * allocation, real-time loops that allocate everything at start-up, plugins
 * whose framework owns the device allocator and offers no workspace hook.
 * Same arguments and results as qpb_solve_qp, minus the workspace: the
 * scratch (the persistent launch's work counter, and the global arena of
 * instances too large for shared memory) comes from a 1 MiB array that the
 * library keeps in device memory on every GPU that loads it, until the
 * process exits.  Problems whose qpb_workspace_size exceeds 1 MiB are
 * rejected with QPB_ERR_UNSUPPORTED.  Problems planned with their instances
 * in shared memory need only 256 bytes of it, for any batch size: all
 * FP64 n <= 32, and mixed precision with n > 32 up to about n = 64 when
 * p = 2n.  Mixed precision with n <= 32 also keeps a hand-over record per
 * instance ((n + 2p + m) * 8 + 16 bytes: about 770 instances at n = 32,
 * m = 8, p = 64); FP64 instances with n > 32 run from global arenas (more
 * of them stay resident per SM that way) and fit only in small batches.
 * Nothing is allocated, by this call or by the library on its behalf.  The
 * first call on a device looks up the array's device address (one-time
 * set-up), so make that first call before any stream capture.  All calls
 * share the one array: calls that may overlap on the GPU (different streams
 * without ordering between them) race on it and must be serialised by the
 * caller; calls on one stream are safe. */
int qpb_solve_qp_noalloc(const qpb_dims* dims, const double* Q, const double* q, const double* A,
                         const double* b, const double* G, const double* h, double solver_tol, double* x,
                         double* s, double* z, double* y, int32_t* converged, int32_t* iters,
                         const qpb_config* cfg, qpb_stream_t stream);

/* Forward and backward of qpax/diff_qp.py:49-82 solve_qp_primal (qpb_solve_qp,
 * then qpb_solve_qp_primal_bwd) on a batch held in HOST memory -- the call a
 * qpax user with NumPy / CPU arrays makes.  The batch is cut into `chunks`
 * slices; each slice is copied in, solved forward and backward, and its x,
 * six gradients and (optional) converged / iters are copied out, on three
 * internal streams so that copies of one slice overlap the kernels of
 * another.  Q..h, dl_dx, x, dQ..dh, converged, iters are HOST pointers (pin
 * them -- cudaHostAlloc / cudaHostRegister -- for the copies to overlap);
 * converged and iters may be NULL.  `workspace` is DEVICE memory of
 * qpb_solve_qp_primal_vjp_host_workspace_size bytes (256-byte aligned).
 * Everything is enqueued after the work already on `stream`, and `stream`
 * waits for all of it: synchronize `stream` before reading the outputs.
 * The internal streams are created once per device and shared by every call
 * on that device: calls from several host threads are safe when each has
 * its own workspace, but their chunks are queued on the same streams and
 * interleave in enqueue order -- concurrent calls share the streams rather
 * than running side by side.
 * Requires p >= 1. */
size_t qpb_solve_qp_primal_vjp_host_workspace_size(const qpb_dims* dims, int32_t chunks, const qpb_config* cfg);
int qpb_solve_qp_primal_vjp_host(const qpb_dims* dims, const double* Q, const double* q, const double* A,
                                 const double* b, const double* G, const double* h, const double* dl_dx,
                                 double solver_tol, double target_kappa, double* x, double* dQ, double* dq,
                                 double* dA, double* db, double* dG, double* dh, int32_t* converged, int32_t* iters,
                                 int32_t chunks, const qpb_config* cfg, void* workspace, size_t workspace_bytes,
                                 qpb_stream_t stream);

/* Human-readable name of a qpb_status code. */
const char* qpb_status_string(int status);

/* Library ABI version (major * 10000 + minor * 100 + patch). */
int32_t qpb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* QPB_H_ */
