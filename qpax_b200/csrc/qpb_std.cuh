// qpb_std.cuh -- the standard QP  min 1/2 x'Qx + q'x  s.t. Ax = b, Gx <= h
// solved by one team per instance, the instance resident in its arena for the
// whole interior-point loop.
//
// Follows qpax (kevin-tracy/qpax):
//   solve_qp            qpax/pdip.py:181-251  (early exits :208-217, inf rows
//                       :166-178 and :243-246, symmetrize :223)
//   initialize          qpax/pdip.py:15-35
//   pdip_pc_step        qpax/pdip.py:87-119   (test before step, step always taken)
//   solve_kkt_rhs       qpax/pdip.py:49-63    (cvxopt-style reduced solve)
//   centering_params    qpax/pdip.py:76-84, ort_linesearch :66-73
//   solve_eq_only       qpax/pdip.py:137-150  (same reduced solve with p = 0)
//   pdip_newton_step    qpax/pdip_relaxed.py:7-52, relax_qp :70-103
//   diff_qp             qpax/diff_qp.py:20-46, optnet_derivatives :8-17
// The factorisation is LDL^T of H where qpax uses QR; both solve the same
// reduced system to rounding.
#pragma once
#include "qpb_core.cuh"

namespace qpb {

struct StdArena : CoreArena {
  double *q, *b, *h;
  double *x, *s, *z, *y;
  double *v1, *v2, *v3, *v4;  // negated residuals (right-hand sides)
  double *dx, *ds, *dz, *dy, *dsa, *dza;
  double *zp, *zm;            // zero vectors

  __host__ __device__ uintptr_t carve(uintptr_t base, int n, int m, int p, bool mixed) {
    Carver c(base);
    carve_core(c, n, m, p, mixed);
    q = c.take<double>(n); b = c.take<double>(m); h = c.take<double>(p);
    x = c.take<double>(n); s = c.take<double>(p); z = c.take<double>(p); y = c.take<double>(m);
    v1 = c.take<double>(n); v2 = c.take<double>(p); v3 = c.take<double>(p); v4 = c.take<double>(m);
    dx = c.take<double>(n); ds = c.take<double>(p); dz = c.take<double>(p); dy = c.take<double>(m);
    dsa = c.take<double>(p); dza = c.take<double>(p);
    zp = c.take<double>(p); zm = c.take<double>(m);
    return c.cur;
  }
  static size_t bytes(int n, int m, int p, bool mixed) {
    StdArena a;
    return (size_t)a.carve(0, n, m, p, mixed) + 16;
  }
};

template <int NT, int KC, bool kMixed>
struct StdQP {
  // CTAs per SM the register budget is cut for (128-thread teams): four up
  // to n = 128 (168 -> 128 registers measured 20 % faster per iteration at
  // n = 48..96), three above (the blocked factorisation's tiles spill at 128).
  static constexpr int kMinBlocks = NT == 128 ? (KC <= 4 ? 4 : 3) : 1;
  Core<NT, KC, kMixed> k;
  StdArena a;
  const Params* P;
  int n, m, p, ld;
  InstRef R;                 // the instance being solved
  unsigned char* arena_base;

  QPB_DEV const Team<NT>& t() const { return k.t; }

  QPB_DEV void setup(const Params& prm, unsigned char* arena, int rank, BlockedStage* stage) {
    P = &prm;
    arena_base = arena;
    n = prm.n; m = prm.m; p = prm.p;
    a.carve(reinterpret_cast<uintptr_t>(arena), n, m, p, kMixed);
    ld = a.ld;
    k.n = n; k.m = m; k.p = p; k.ld = ld;
    k.c = a;  // slices CoreArena
    k.t.r = rank;
    k.t.red = a.red;
    k.st = stage;
    k.pivot_max = prm.pivot_max;
    k.max_sweeps = prm.max_sweeps;
  }

  // Copies instance `inst` into the arena; Q is symmetrized (every device
  // entry point treats Q as (Q+Q')/2).  With remove_inf, rows whose h is
  // +-inf get h = 0 and a zero row of G (qpax/pdip.py:166-178).
  QPB_NOINLINE void load(long inst, bool remove_inf) {
    const Team<NT>& T = t();
    (void)inst;
    const double* gQ = P->Q + R.oQ;
    const double* gG = P->G + R.oG;
    const double* gA = P->A + R.oA;
    const double* gh = P->h + R.oh;
    team_copy_rows(T, a.Q, ld, gQ, n, n, true);
    team_copy_rows(T, a.G, ld, gG, p, n, false, [&](int i) { return remove_inf && isinf(__ldg(gh + i)); });
    team_copy_rows(T, a.A, ld, gA, m, n, false);
    for (int i = T.r; i < n; i += NT) a.q[i] = P->q[R.oq + i];
    for (int i = T.r; i < m; i += NT) {
      a.b[i] = P->b[R.ob + i];
      a.zm[i] = 0.0;
    }
    for (int i = T.r; i < p; i += NT) {
      const double hv = gh[i];
      a.h[i] = (remove_inf && isinf(hv)) ? 0.0 : hv;
      a.zp[i] = 0.0;
    }
    T.sync();
  }

  QPB_NOINLINE void load_iterate(long inst) {
    const Team<NT>& T = t();
    (void)inst;
    for (int i = T.r; i < n; i += NT) a.x[i] = P->in[0][R.oq + i];
    for (int i = T.r; i < p; i += NT) {
      a.s[i] = P->in[1][R.oh + i];
      a.z[i] = P->in[2][R.oh + i];
    }
    for (int i = T.r; i < m; i += NT) a.y[i] = P->in[3][R.ob + i];
    T.sync();
  }

  QPB_NOINLINE void store_iterate(long inst, bool inf_rows) {
    const Team<NT>& T = t();
    (void)inst;
    for (int i = T.r; i < n; i += NT) P->out[0][R.oq + i] = a.x[i];
    for (int i = T.r; i < p; i += NT) {
      double sv = a.s[i], zv = a.z[i];
      if (inf_rows && isinf(P->h[R.oh + i])) {  // qpax/pdip.py:243-246
        zv = 0.0;
        sv = INFINITY;
      }
      P->out[1][R.oh + i] = sv;
      P->out[2][R.oh + i] = zv;
    }
    for (int i = T.r; i < m; i += NT) P->out[3][R.ob + i] = a.y[i];
  }

  // qpax/pdip.py:49-63 solve_kkt_rhs for right-hand sides (c1, c2, c3, c4).
  QPB_NOINLINE void solve(const double* c1, const double* c2, const double* c3, const double* c4, double* odx,
                     double* ods, double* odz, double* ody) {
    const Team<NT>& T = t();
    for (int i = T.r; i < p; i += NT) a.tp[i] = a.w[i] * (c3[i] - c2[i] / a.z[i]);
    T.sync();
    cols_dot(T, p, n, a.G, ld, a.tp, [&](int j, double g) { a.p1[j] = c1[j] + g; });
    T.sync();
    k.reduced(a.p1, c4, odx, ody);
    rows_dot(T, p, n, a.G, ld, odx, [&](int i, double g) {
      const double dsi = c3[i] - g;
      ods[i] = dsi;
      odz[i] = (c2[i] - a.z[i] * dsi) / a.s[i];
    });
    T.sync();
  }

  // v = -(relaxed KKT residuals), w = z/s; returns the inf-norm of the
  // residuals (qpax/pdip.py:93-100, pdip_relaxed.py:16-23).
  QPB_NOINLINE double residuals(double kappa) {
    const Team<NT>& T = t();
    double loc = 0.0;
    for (int j = T.r; j < n; j += NT) {
      double qx = 0.0, ay = 0.0, gz = 0.0;
      for (int i = 0; i < n; ++i) qx = fma(a.Q[i * ld + j], a.x[i], qx);
      for (int i = 0; i < m; ++i) ay = fma(a.A[i * ld + j], a.y[i], ay);
      for (int i = 0; i < p; ++i) gz = fma(a.G[i * ld + j], a.z[i], gz);
      const double r = ((qx + a.q[j]) + ay) + gz;
      a.v1[j] = -r;
      loc = nmax(loc, fabs(r));
    }
    rows_dot(T, p, n, a.G, ld, a.x, [&](int i, double g) {
      const double r3 = (g + a.s[i]) - a.h[i];
      const double r2 = a.s[i] * a.z[i] - kappa;
      a.v3[i] = -r3;
      a.v2[i] = -r2;
      loc = nmax(loc, nmax(fabs(r3), fabs(r2)));
    });
    rows_dot(T, m, n, a.A, ld, a.x, [&](int i, double g) {
      const double r4 = g - a.b[i];
      a.v4[i] = -r4;
      loc = nmax(loc, fabs(r4));
    });
    for (int i = T.r; i < p; i += NT) a.w[i] = a.z[i] / a.s[i];
    const double nrm = T.max(loc);
    T.sync();
    return nrm;
  }

  QPB_NOINLINE void step_update(double alpha) {
    const Team<NT>& T = t();
    for (int i = T.r; i < n; i += NT) a.x[i] += alpha * a.dx[i];
    for (int i = T.r; i < p; i += NT) {
      a.s[i] += alpha * a.ds[i];
      a.z[i] += alpha * a.dz[i];
    }
    for (int i = T.r; i < m; i += NT) a.y[i] += alpha * a.dy[i];
    T.sync();
  }

  // qpax/pdip.py:87-119
  QPB_NOINLINE int pc_step() {
    const Team<NT>& T = t();
    const double nrm = residuals(0.0);
    const int converged = (nrm < P->tol) ? 1 : 0;
    k.factor();
    solve(a.v1, a.v2, a.v3, a.v4, a.dx, a.dsa, a.dza, a.dy);
    // centering_params (qpax/pdip.py:76-84)
    double sz = 0.0;
    for (int i = T.r; i < p; i += NT) sz = fma(a.s[i], a.z[i], sz);
    sz = T.sum(sz);
    const double mu = sz / p;
    const double alpha_a = nmin(1.0, T.min(nmin(k.ls_local(a.s, a.dsa, p), k.ls_local(a.z, a.dza, p))));
    double num = 0.0;
    for (int i = T.r; i < p; i += NT) num = fma(a.s[i] + alpha_a * a.dsa[i], a.z[i] + alpha_a * a.dza[i], num);
    num = T.sum(num);
    const double ratio = num / sz;
    const double sigma = ratio * ratio * ratio;
    // r2 <- r2 - (sigma mu - ds_a dz_a), kept negated in v2
    for (int i = T.r; i < p; i += NT) a.v2[i] = -(-a.v2[i] - (sigma * mu - a.dsa[i] * a.dza[i]));
    T.sync();
    solve(a.v1, a.v2, a.v3, a.v4, a.dx, a.ds, a.dz, a.dy);
    const double alpha = 0.99 * nmin(1.0, T.min(nmin(k.ls_local(a.s, a.ds, p), k.ls_local(a.z, a.dz, p))));
    step_update(alpha);
    return converged;
  }

  // qpax/pdip_relaxed.py:7-52
  QPB_NOINLINE int newton_step() {
    const Team<NT>& T = t();
    const double nrm = residuals(P->kappa);
    const int converged = (nrm < P->tol) ? 1 : 0;
    k.factor();
    solve(a.v1, a.v2, a.v3, a.v4, a.dx, a.ds, a.dz, a.dy);
    const double ls = T.min(nmin(k.ls_local(a.s, a.ds, p), k.ls_local(a.z, a.dz, p)));
    // 0.99 min(1, 0.99 ls_s, 0.99 ls_z) with ls_s, ls_z already capped at 1
    const double alpha = 0.99 * nmin(1.0, 0.99 * nmin(1.0, ls));
    step_update(alpha);
    return converged;
  }

  // qpax/pdip.py:15-35 on the arena data (and the p == 0 exits :208-217).
  QPB_NOINLINE void initialize() {
    const Team<NT>& T = t();
    for (int i = T.r; i < p; i += NT) a.w[i] = 1.0;
    T.sync();
    k.factor();
    // r1 = -q + G' h ; [H A'; A 0][x; y] = [r1; b]
    cols_dot(T, p, n, a.G, ld, a.h, [&](int j, double g) { a.v1[j] = -a.q[j] + g; });
    T.sync();
    k.reduced(a.v1, a.b, a.x, a.y);
    if (p == 0) return;
    double zmax = -INFINITY, zmin = INFINITY;
    rows_dot(T, p, n, a.G, ld, a.x, [&](int i, double g) {
      const double zi = g - a.h[i];
      a.z[i] = zi;
      zmax = nmax(zmax, zi);
      zmin = nmin(zmin, zi);
    });
    const double alpha_p = T.max(zmax);
    const double alpha_d = -T.min(zmin);
    for (int i = T.r; i < p; i += NT) {
      const double zi = a.z[i];
      a.s[i] = (alpha_p < 0) ? -zi : -zi + (1.0 + alpha_p);
      if (alpha_d >= 0) a.z[i] = zi + (1.0 + alpha_d);
    }
    T.sync();
  }

  QPB_DEV void loop(bool relaxed, int* conv_out, int* iters_out) {
    int converged = 0, it = 0;
    k.use64 = 0;
    while (it < kMaxIters && converged == 0) {
      converged = relaxed ? newton_step() : pc_step();
      ++it;
    }
    *conv_out = converged;
    *iters_out = it;
  }

  // qpax/diff_qp.py:20-46 + optnet_derivatives :8-17 at the arena iterate
  // (x, s, lambda = z, nu = y); writes the six gradients of instance inst.
  QPB_NOINLINE void adjoint(long inst) {
    const Team<NT>& T = t();
    for (int i = T.r; i < p; i += NT) a.w[i] = a.z[i] / a.s[i];
    (void)inst;
    for (int j = T.r; j < n; j += NT) a.v1[j] = -P->gx[R.oq + j];
    T.sync();
    k.use64 = 0;
    k.factor();
    solve(a.v1, a.zp, a.zp, a.zm, a.dx, a.ds, a.dz, a.dy);
    for (int i = T.r; i < p; i += NT) a.dz[i] = a.dz[i] / a.z[i];  // dlam = dlam_tilde / lam
    T.sync();
    double* dQ = P->dQ + R.oQ;
    for (int e = T.r; e < n * n; e += NT) {
      const int i = e / n, j = e - i * n;
      dQ[e] = 0.5 * (a.dx[i] * a.x[j] + a.x[i] * a.dx[j]);
    }
    double* dA = P->dA + R.oA;
    for (int e = T.r; e < m * n; e += NT) {
      const int i = e / n, j = e - i * n;
      dA[e] = a.dy[i] * a.x[j] + a.y[i] * a.dx[j];
    }
    double* dG = P->dG + R.oG;
    for (int e = T.r; e < p * n; e += NT) {
      const int i = e / n, j = e - i * n;
      dG[e] = a.z[i] * (a.dz[i] * a.x[j] + a.z[i] * a.dx[j]);
    }
    for (int j = T.r; j < n; j += NT) P->dq[R.oq + j] = a.dx[j];
    for (int i = T.r; i < m; i += NT) P->db[R.ob + i] = -a.dy[i];
    for (int i = T.r; i < p; i += NT) P->dh[R.oh + i] = -a.z[i] * a.dz[i];
  }

  QPB_NOINLINE void run(long i) {
    const Team<NT>& T = t();
    R = inst_ref(*P, i);
    const long inst = R.id;
    if (P->shapes) {  // packed batch: this instance's shapes and arena layout
      n = R.n; m = R.m; p = R.p;
      a.carve(reinterpret_cast<uintptr_t>(arena_base), n, m, p, kMixed);
      ld = a.ld;
      k.n = n; k.m = m; k.p = p; k.ld = ld;
      k.c = a;
      k.t.red = a.red;
    }
    k.reset_stats();
    const int op = P->op;
    int conv = 0, iters = 0;
    if (op == kOpSolve) {
      load(inst, true);
      initialize();
      if (p == 0) {
        conv = 1;  // qpax/pdip.py:208-217: direct solve, converged = 1, iters = 0
      } else {
        loop(false, &conv, &iters);
      }
      store_iterate(inst, true);
    } else if (op == kOpInit) {
      load(inst, false);
      initialize();
      store_iterate(inst, false);
    } else if (op == kOpRelax || op == kOpBwd) {
      load(inst, false);
      load_iterate(inst);
      loop(true, &conv, &iters);
      if (P->out[0]) store_iterate(inst, false);
      if (op == kOpBwd) adjoint(inst);
    } else if (op == kOpAdjoint) {
      load(inst, false);
      load_iterate(inst);
      adjoint(inst);
    }
    if (T.r == 0) {
      if (P->conv) P->conv[inst] = conv;
      if (P->iters) P->iters[inst] = iters;
      if (P->stats) {
        P->stats[inst * 4 + kStatFact32] = k.st_f32;
        P->stats[inst * 4 + kStatFact64] = k.st_f64;
        P->stats[inst * 4 + kStatSweeps] = k.st_sweeps;
        P->stats[inst * 4 + kStatFlags] = k.st_flags;
      }
    }
    T.sync();
  }
};

}  // namespace qpb
