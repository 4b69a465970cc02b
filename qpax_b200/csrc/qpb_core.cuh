// qpb_core.cuh -- the reduced KKT core shared by the standard and elastic
// solvers: factor [H A'; A 0] for the weights in `w`, and solve with it.
//
// Precision modes:
//   FP64  (kMixed == false): H, LDL^T, Y, F and the solves in double.
//   mixed (kMixed == true):  H formed from float(sqrt(w) G), LDL^T, Y, F in
//         float; every reduced solve is refined in double against the FP64
//         operator Q + G' diag(w) G (and A) until the correction stops
//         mattering.  A float factor whose pivot ratio exceeds pivot_max, or
//         whose refinement stalls, is replaced by an FP64 factor for the rest
//         of the loop (the conditioning of H only grows as the IPM converges).
#pragma once
#include "qpb_linalg.cuh"
#include "qpb_params.h"

namespace qpb {

// Iteration cap of every IPM loop: qpax/pdip.py:232, pdip_relaxed.py:76,
// elastic_qp.py:195,325.
constexpr int kMaxIters = 30;

struct CoreArena {
  int ld;
  double *Q, *G, *A;  // n4-padded FP64 operands
  double* w;          // weights of G' diag(w) G
  double *p1, *tp, *rx, *ry, *ex, *ey;
  double* red;
  float* GS;
  FactorRegion fr;

  __host__ __device__ void carve_core(Carver& c, int n, int m, int p, bool mixed) {
    ld = pad4(n);
    Q = c.take<double>((size_t)n * ld);
    G = c.take<double>((size_t)p * ld);
    A = c.take<double>((size_t)m * ld);
    w = c.take<double>(p);
    p1 = c.take<double>(n); tp = c.take<double>(p); rx = c.take<double>(n); ry = c.take<double>(m);
    ex = c.take<double>(n); ey = c.take<double>(m);
    red = c.take<double>(16);
    GS = mixed ? c.take<float>((size_t)p * ld) : nullptr;
    fr.n = n;
    fr.m = m;
    fr.base = c.take<unsigned char>(FactorRegion::bytes(n, m));
  }
};

template <int NT, int KC, bool kMixed>
struct Core {
  Team<NT> t;
  int n, m, p, ld;
  CoreArena c;
  double pivot_max;
  int max_sweeps;
  int use64;
  int st_f32, st_f64, st_sweeps, st_flags;
  BlockedStage* st;  // shared staging of the blocked FP64 path (teams of >= 2 warps)
  double* gbuf = nullptr;  // G chunk buffers in shared memory (arena in global memory), or none
  int gstage_rows = 0;

  // FP64 factors: teams of one warp, and instances with n <= 32, keep the
  // split layout (L, Y, F) and per-column elimination (one panel's worth of
  // work: the blocked pass's serial diagonal step would dominate); larger
  // instances on larger teams factor the whole KKT matrix blocked on the
  // FP64 tensor cores (qpb_blocked.cuh).
  static constexpr bool kBlocked = NT > 32;
  QPB_DEV bool blocked() const { return kBlocked && n > kPanel; }

  QPB_DEV void reset_stats() { st_f32 = st_f64 = st_sweeps = st_flags = 0; use64 = 0; }

  QPB_NOINLINE void factor64() {
    double r = 0.0;
    bool done = false;
    if constexpr (kBlocked) {
      if (blocked()) {
        const KKTView f = KKTRegion::view(c.fr.base, n, m);
        form_kkt<NT, KC>(t, f, p, c.Q, ld, c.G, ld, c.A, ld, c.w, gbuf, gstage_rows);
        t.sync();
        // the G chunk buffers are free again: they hold the factor's panels
        const size_t pcap = gbuf ? (gstage_bytes(ld, gstage_rows) - 64) / sizeof(double) : 0;
        r = kkt_factor<NT, KC>(t, f, st, gbuf, pcap);
        done = true;
      }
    }
    if (!done) r = factor_kkt<NT, KC, double>(t, n, m, p, c.Q, c.G, c.A, ld, c.w, nullptr, c.fr.view<double>());
    st_f64++;
    if (!(r < INFINITY)) st_flags |= kFlagBreakdown64;
  }

  // [H A'; A 0][dx; dy] = [rhs; v4] with the blocked FP64 factor.
  QPB_NOINLINE void reduced_blocked(const double* rhs, const double* v4, double* dx, double* dy) {
    const KKTView f = KKTRegion::view(c.fr.base, n, m);
    double* v = st->v;
    for (int i = t.r; i < f.N; i += NT) {
      double x = 0.0;
      if (i < n)
        x = rhs[i];
      else if (i >= f.n8 && i - f.n8 < m)
        x = v4[i - f.n8];
      v[i] = x;
    }
    t.sync();
    kkt_solve<NT, KC>(t, f, v, st);
    for (int i = t.r; i < n; i += NT) dx[i] = v[i];
    for (int i = t.r; i < m; i += NT) dy[i] = v[f.n8 + i];
    t.sync();
  }

  // Factor for the weights currently in c.w.
  QPB_NOINLINE void factor() {
    if constexpr (kMixed) {
      if (!use64) {
        const double r = factor_kkt<NT, KC, float>(t, n, m, p, c.Q, c.G, c.A, ld, c.w, c.GS, c.fr.view<float>());
        if (r <= pivot_max) {
          st_f32++;
          return;
        }
        use64 = 1;
        st_flags |= kFlagFallback;
      }
    }
    factor64();
  }

  // FP64 iterative refinement of [H A'; A 0][dx; dy] = [rhs; v4] against the
  // float factor.  Returns false when the corrections stop shrinking.
  QPB_NOINLINE bool refine(const double* rhs, const double* v4, double* dx, double* dy) {
    const Factor<float> f = c.fr.view<float>();
    double prev = INFINITY;
    for (int sw = 0; sw < max_sweeps; ++sw) {
      rows_dot(t, p, n, c.G, ld, dx, [&](int k, double g) { c.tp[k] = c.w[k] * g; });
      rows_dot(t, m, n, c.A, ld, dx, [&](int i, double g) { c.ry[i] = v4[i] - g; });
      t.sync();
      for (int j = t.r; j < n; j += NT) {
        double qd = 0.0, gt = 0.0, ad = 0.0;
        for (int i = 0; i < n; ++i) qd = fma(c.Q[i * ld + j], dx[i], qd);
        for (int k = 0; k < p; ++k) gt = fma(c.G[k * ld + j], c.tp[k], gt);
        for (int i = 0; i < m; ++i) ad = fma(c.A[i * ld + j], dy[i], ad);
        c.rx[j] = rhs[j] - ((qd + gt) + ad);
      }
      t.sync();
      if (t.warp() == 0) {
        const int lane = t.lane();
        reduced_solve_warp<KC, float>(f, n, m, c.rx, c.ry, c.ex, c.ey, lane);
        __syncwarp();
        double exn = 0.0, dxn = 0.0, eyn = 0.0, dyn = 0.0;
        for (int i = lane; i < n; i += 32) {
          const double d = dx[i] + c.ex[i];
          dx[i] = d;
          exn = nmax(exn, fabs(c.ex[i]));
          dxn = nmax(dxn, fabs(d));
        }
        for (int i = lane; i < m; i += 32) {
          const double d = dy[i] + c.ey[i];
          dy[i] = d;
          eyn = nmax(eyn, fabs(c.ey[i]));
          dyn = nmax(dyn, fabs(d));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          exn = nmax(exn, __shfl_xor_sync(kFull, exn, o));
          dxn = nmax(dxn, __shfl_xor_sync(kFull, dxn, o));
          eyn = nmax(eyn, __shfl_xor_sync(kFull, eyn, o));
          dyn = nmax(dyn, __shfl_xor_sync(kFull, dyn, o));
        }
        if (lane == 0) c.red[8] = nmax(exn / (dxn > 0 ? dxn : 1.0), eyn / (dyn > 0 ? dyn : 1.0));
      }
      t.sync();
      const double rel = c.red[8];
      st_sweeps++;
      // done when this correction, or the next one predicted from the
      // observed contraction, is below 1e-12 of the solution
      if (rel <= 1e-12 || (sw > 0 && rel * (rel / prev) <= 1e-12)) return true;
      if (!(rel < 0.5 * prev)) return false;
      prev = rel;
    }
    return false;
  }

  // [H A'; A 0][dx; dy] = [rhs; v4]; rhs, v4 in shared memory.
  QPB_NOINLINE void reduced(const double* rhs, const double* v4, double* dx, double* dy) {
    if constexpr (kMixed) {
      if (!use64) {
        if (t.warp() == 0) reduced_solve_warp<KC, float>(c.fr.view<float>(), n, m, rhs, v4, dx, dy, t.lane());
        t.sync();
        if (refine(rhs, v4, dx, dy)) return;
        st_flags |= kFlagRefineStall | kFlagFallback;
        use64 = 1;
        factor64();
      }
    }
    if constexpr (kBlocked) {
      if (blocked()) {
        reduced_blocked(rhs, v4, dx, dy);
        return;
      }
    }
    if (t.warp() == 0) reduced_solve_warp<KC, double>(c.fr.view<double>(), n, m, rhs, v4, dx, dy, t.lane());
    t.sync();
  }

  // min over the team's entries of -v/d for d < 0 (qpax/pdip.py:66-73 before the cap at 1).
  QPB_DEV double ls_local(const double* v, const double* d, int len) const {
    double mn = INFINITY;
    for (int i = t.r; i < len; i += NT) {
      const double di = d[i];
      if (di < 0) mn = nmin(mn, -v[i] / di);
    }
    return mn;
  }
};

}  // namespace qpb
