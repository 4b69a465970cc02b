// qpb_params.h -- launch parameters shared by the host launcher and kernels.
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace qpb {

enum Op : int {
  kOpSolve = 0,    // solve_qp                     qpax/pdip.py:181-251
  kOpInit = 1,     // initialize                   qpax/pdip.py:15-35
  kOpRelax = 2,    // relax_qp                     qpax/pdip_relaxed.py:70-103
  kOpBwd = 3,      // relax_qp + diff_qp           qpax/diff_qp.py:61-79
  kOpAdjoint = 4,  // diff_qp                      qpax/diff_qp.py:20-46
  kOpESolve = 5,   // solve_qp_elastic             qpax/elastic_qp.py:184-228
  kOpEInit = 6,    // initialize_elastic           qpax/elastic_qp.py:27-47
  kOpERelax = 7,   // relax_qp_elastic             qpax/elastic_qp.py:319-359
  kOpEBwd = 8,     // relax_qp_elastic + diff_qp_elastic  qpax/elastic_qp.py:433-466
  kOpEAdjoint = 9  // diff_qp_elastic              qpax/elastic_qp.py:381-417
};

inline bool op_is_elastic(int op) { return op >= kOpESolve; }

// Per-instance statistics (optional output, 4 int32 per instance).
enum Stat : int { kStatFact32 = 0, kStatFact64 = 1, kStatSweeps = 2, kStatFlags = 3 };
enum Flag : int {
  kFlagFallback = 1,      // FP32 factor rejected at least once -> FP64 refactor
  kFlagRefineStall = 2,   // refinement did not reach FP64 accuracy in the sweep limit
  kFlagBreakdown64 = 4,   // FP64 factor had a non-positive pivot (outputs follow IEEE arithmetic)
  kFlagNonFinite = 8      // a non-finite value reached the iterate
};

struct Params {
  int op, batch, n, m, p;
  int mixed;            // 0: FP64 factor; 1: FP32 factor + FP64 refinement
  double tol, kappa;
  double pivot_max;     // mixed: FP32 factor rejected when max(d)/min(d) exceeds this
  int max_sweeps;       // mixed: refinement sweeps before falling back to FP64
  const double *Q, *q, *A, *b, *G, *h, *penalty;
  const double *in[6];  // starting iterate: (x,s,z,y) or elastic (x,t,s1,s2,z1,z2)
  const double *gx;     // incoming gradient dl/dx
  double *out[6];       // iterate out (same order)
  int32_t *conv, *iters;
  double *dQ, *dq, *dA, *db, *dG, *dh;
  int32_t *stats;       // optional
  unsigned char *arena; // global arenas when they do not fit in shared memory
  size_t arena_bytes;   // bytes per team arena
  int arena_in_smem;
  int gstage_rows;      // global arenas: rows of G per chunk staged in dynamic shared memory (0: none)
  int *counter;         // work counter (zeroed before launch)
  // Packed (uneven) batches: when `shapes` is set, instance i has its own
  // (n, m, p) = shapes[3i..3i+2] and element offsets offs[6i..6i+5] into the
  // packed Q, q, A, b, G, h arrays (x, dq, gx follow q; y, db follow b; s, z,
  // dh follow h; dQ, dA, dG follow Q, A, G).  `list` names the instances of
  // this launch (one size bin); the launch covers list[0 .. batch).
  const int32_t *shapes;
  const int64_t *offs;
  const int32_t *list;
  // Mixed precision on the one-warp kernels runs in two launches: the mixed
  // kernel hands an instance whose FP32 factor is rejected (pivot ratio,
  // refinement stall) over to the FP64 kernel, which resumes it where it
  // stopped.  Per launch-local instance index li: iterate block
  // hiter[li * hstride ...] = x (n) | s (p) | z (p) | y (m), with the
  // launch's (largest) n, m, p; hstate[3 li ...] = stage, iteration,
  // converged; hlist[0 .. *hcount) = the handed-over indices.
  int resume;           // 1: this launch resumes the instances in hlist (FP64 kernel)
  int *hcount;
  int32_t *hlist, *hstate;
  double *hiter;
  int hstride;
};

// Where instance `inst` (a launch-local index) lives.
struct InstRef {
  long id;                       // instance index in the whole batch
  long oQ, oq, oA, ob, oG, oh;   // element offsets
  int n, m, p;
};

#ifdef __CUDACC__
__device__ __forceinline__ InstRef inst_ref(const Params& P, long i) {
  InstRef r;
  if (P.shapes) {
    const long id = P.list ? P.list[i] : i;
    r.id = id;
    r.n = P.shapes[3 * id];
    r.m = P.shapes[3 * id + 1];
    r.p = P.shapes[3 * id + 2];
    const int64_t* o = P.offs + 6 * id;
    r.oQ = o[0]; r.oq = o[1]; r.oA = o[2]; r.ob = o[3]; r.oG = o[4]; r.oh = o[5];
  } else {
    r.id = i;
    r.n = P.n; r.m = P.m; r.p = P.p;
    r.oQ = i * (long)P.n * P.n; r.oq = i * (long)P.n; r.oA = i * (long)P.m * P.n;
    r.ob = i * (long)P.m; r.oG = i * (long)P.p * P.n; r.oh = i * (long)P.p;
  }
  return r;
}
#endif

}  // namespace qpb
