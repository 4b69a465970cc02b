// qpb_elastic.cuh -- the elastic QP of qpax: Gx <= h relaxed with slacks t
// penalised by `penalty`, one team per instance.
//
// Follows qpax/elastic_qp.py (kevin-tracy/qpax):
//   solve_init_elastic_ls :9-24, initialize_elastic :27-47
//   solve_elastic_kkt_affine :50-72 / _cc :75-96 (Algorithm 5: one n x n
//                          factor of H = Q + G' diag(1/(s1/z1 + s2/z2)) G)
//   pdip_pc_step_elastic :99-174, solve_qp_elastic :184-228
//   pdip_newton_step_elastic :235-316, relax_qp_elastic :319-359
//     (its residual signs differ from the PC step's -- r2 = z1+z2-p,
//      r5 = t+s1, r6 = Gx+t+s2-h -- and are reproduced as written)
//   diff_qp_elastic :381-417 with optnet_derivatives_elastic :366-373,
//     cropped to the (Q, q, G, h) blocks as :412-415 do.
#pragma once
#include "qpb_core.cuh"

namespace qpb {

struct ElasticArena : CoreArena {
  double *q, *h;
  double *x, *t, *s1, *s2, *z1, *z2;
  double *v1, *v2, *v3, *v4, *v5, *v6;
  double *dx, *dt, *ds1, *ds2, *dz1, *dz2;
  double *dsa1, *dsa2, *dza1, *dza2;
  double *pe, *a3, *zp;

  __host__ __device__ uintptr_t carve(uintptr_t base, int n, int p, bool mixed) {
    Carver c(base);
    carve_core(c, n, 0, p, mixed);
    q = c.take<double>(n); h = c.take<double>(p);
    x = c.take<double>(n);
    t = c.take<double>(p); s1 = c.take<double>(p); s2 = c.take<double>(p);
    z1 = c.take<double>(p); z2 = c.take<double>(p);
    v1 = c.take<double>(n);
    v2 = c.take<double>(p); v3 = c.take<double>(p); v4 = c.take<double>(p);
    v5 = c.take<double>(p); v6 = c.take<double>(p);
    dx = c.take<double>(n);
    dt = c.take<double>(p); ds1 = c.take<double>(p); ds2 = c.take<double>(p);
    dz1 = c.take<double>(p); dz2 = c.take<double>(p);
    dsa1 = c.take<double>(p); dsa2 = c.take<double>(p); dza1 = c.take<double>(p); dza2 = c.take<double>(p);
    pe = c.take<double>(p); a3 = c.take<double>(p); zp = c.take<double>(p);
    return c.cur;
  }
  static size_t bytes(int n, int p, bool mixed) {
    ElasticArena a;
    return (size_t)a.carve(0, n, p, mixed) + 16;
  }
};

template <int NT, int KC, bool kMixed>
struct ElasticQP {
  // CTAs per SM the register budget is cut for (128-thread teams): three
  // (at four, 128 registers, the elastic steps spill and run slower).
  static constexpr int kMinBlocks = NT == 128 ? 3 : 1;
  Core<NT, KC, kMixed> k;
  ElasticArena a;
  const Params* P;
  int n, p, ld;
  double pen;

  QPB_DEV const Team<NT>& T() const { return k.t; }

  QPB_DEV void setup(const Params& prm, unsigned char* arena, int rank, BlockedStage* stage) {
    P = &prm;
    n = prm.n; p = prm.p;
    a.carve(reinterpret_cast<uintptr_t>(arena), n, p, kMixed);
    ld = a.ld;
    k.n = n; k.m = 0; k.p = p; k.ld = ld;
    k.c = a;
    k.t.r = rank;
    k.t.red = a.red;
    k.st = stage;
    k.pivot_max = prm.pivot_max;
    k.max_sweeps = prm.max_sweeps;
  }

  QPB_NOINLINE void load(long inst) {
    const Team<NT>& tm = T();
    const double* gQ = P->Q + inst * (long)n * n;
    const double* gG = P->G + inst * (long)p * n;
    team_copy_rows(tm, a.Q, ld, gQ, n, n, true);
    team_copy_rows(tm, a.G, ld, gG, p, n, false);
    for (int i = tm.r; i < n; i += NT) a.q[i] = P->q[inst * n + i];
    for (int i = tm.r; i < p; i += NT) {
      a.h[i] = P->h[inst * p + i];
      a.zp[i] = 0.0;
    }
    pen = P->penalty[inst];
    tm.sync();
  }

  QPB_NOINLINE void load_iterate(long inst) {
    const Team<NT>& tm = T();
    for (int i = tm.r; i < n; i += NT) a.x[i] = P->in[0][inst * n + i];
    double* dst[5] = {a.t, a.s1, a.s2, a.z1, a.z2};
    for (int v = 0; v < 5; ++v)
      for (int i = tm.r; i < p; i += NT) dst[v][i] = P->in[v + 1][inst * p + i];
    tm.sync();
  }

  QPB_NOINLINE void store_iterate(long inst) {
    const Team<NT>& tm = T();
    for (int i = tm.r; i < n; i += NT) P->out[0][inst * n + i] = a.x[i];
    const double* src[5] = {a.t, a.s1, a.s2, a.z1, a.z2};
    for (int v = 0; v < 5; ++v)
      for (int i = tm.r; i < p; i += NT) P->out[v + 1][inst * p + i] = src[v][i];
  }

  // Algorithm 5 (qpax/elastic_qp.py:50-96); refactor selects _affine (new
  // factor of H) or _cc (reuse).
  QPB_NOINLINE void solve(const double* c1, const double* c2, const double* c3, const double* c4, const double* c5,
                     const double* c6, bool refactor, double* odx, double* odt, double* ods1, double* ods2,
                     double* odz1, double* odz2) {
    const Team<NT>& tm = T();
    for (int i = tm.r; i < p; i += NT) {
      const double a1 = a.s1[i] / a.z1[i];
      const double a2 = a.s2[i] / a.z2[i];
      const double w1 = c3[i] / a.z1[i];
      const double w2 = c4[i] / a.z2[i];
      const double pi = c5[i] - c6[i] + w2 - w1 - a1 * c2[i];
      const double a3i = a1 + a2;
      a.pe[i] = pi;
      a.a3[i] = a3i;
      a.tp[i] = pi / a3i;
      if (refactor) a.w[i] = 1.0 / a3i;
    }
    tm.sync();
    if (refactor) k.factor();
    cols_dot(tm, p, n, a.G, ld, a.tp, [&](int j, double g) { a.p1[j] = c1[j] - g; });
    tm.sync();
    k.reduced(a.p1, nullptr, odx, nullptr);
    rows_dot(tm, p, n, a.G, ld, odx, [&](int i, double g) {
      const double dz2 = (a.pe[i] + g) / a.a3[i];
      const double dz1 = -c2[i] - dz2;
      const double ds1 = (c3[i] - a.s1[i] * dz1) / a.z1[i];
      odz2[i] = dz2;
      odz1[i] = dz1;
      ods1[i] = ds1;
      ods2[i] = (c4[i] - a.s2[i] * dz2) / a.z2[i];
      odt[i] = ds1 - c5[i];
    });
    tm.sync();
  }

  // Negated residuals into v1..v6; returns their inf-norm.
  // relaxed == false: qpax/elastic_qp.py:105-110; true: :256-261.
  QPB_NOINLINE double residuals(bool relaxed, double kappa) {
    const Team<NT>& tm = T();
    double loc = 0.0;
    for (int j = tm.r; j < n; j += NT) {
      double qx = 0.0, gz = 0.0;
      for (int i = 0; i < n; ++i) qx = fma(a.Q[i * ld + j], a.x[i], qx);
      for (int i = 0; i < p; ++i) gz = fma(a.G[i * ld + j], a.z2[i], gz);
      const double r = (qx + a.q[j]) + gz;
      a.v1[j] = -r;
      loc = nmax(loc, fabs(r));
    }
    rows_dot(tm, p, n, a.G, ld, a.x, [&](int i, double g) {
      double r2, r3, r4, r5, r6;
      if (!relaxed) {
        r2 = (-a.z1[i] - a.z2[i]) + pen;
        r3 = a.s1[i] * a.z1[i];
        r4 = a.s2[i] * a.z2[i];
        r5 = -a.t[i] + a.s1[i];
        r6 = ((g - a.t[i]) + a.s2[i]) - a.h[i];
      } else {
        r2 = (a.z1[i] + a.z2[i]) - pen;
        r3 = a.s1[i] * a.z1[i] - kappa;
        r4 = a.s2[i] * a.z2[i] - kappa;
        r5 = a.t[i] + a.s1[i];
        r6 = ((g + a.t[i]) + a.s2[i]) - a.h[i];
      }
      a.v2[i] = -r2; a.v3[i] = -r3; a.v4[i] = -r4; a.v5[i] = -r5; a.v6[i] = -r6;
      loc = nmax(loc, nmax(nmax(nmax(fabs(r2), fabs(r3)), nmax(fabs(r4), fabs(r5))), fabs(r6)));
    });
    const double nrm = tm.max(loc);
    tm.sync();
    return nrm;
  }

  QPB_DEV double ls_all(const double* d1, const double* d2, const double* e1, const double* e2) const {
    return nmin(nmin(k.ls_local(a.s1, d1, p), k.ls_local(a.s2, d2, p)),
                nmin(k.ls_local(a.z1, e1, p), k.ls_local(a.z2, e2, p)));
  }

  QPB_NOINLINE void step_update(double alpha) {
    const Team<NT>& tm = T();
    for (int i = tm.r; i < n; i += NT) a.x[i] += alpha * a.dx[i];
    for (int i = tm.r; i < p; i += NT) {
      a.t[i] += alpha * a.dt[i];
      a.s1[i] += alpha * a.ds1[i];
      a.s2[i] += alpha * a.ds2[i];
      a.z1[i] += alpha * a.dz1[i];
      a.z2[i] += alpha * a.dz2[i];
    }
    tm.sync();
  }

  // qpax/elastic_qp.py:99-174
  QPB_NOINLINE int pc_step() {
    const Team<NT>& tm = T();
    const double nrm = residuals(false, 0.0);
    const int converged = (nrm < P->tol) ? 1 : 0;
    solve(a.v1, a.v2, a.v3, a.v4, a.v5, a.v6, true, a.dx, a.dt, a.dsa1, a.dsa2, a.dza1, a.dza2);
    double sz = 0.0;
    for (int i = tm.r; i < p; i += NT) sz = fma(a.s2[i], a.z2[i], fma(a.s1[i], a.z1[i], sz));
    sz = tm.sum(sz);
    const double mu = sz / (2 * p);
    const double alpha_a = nmin(1.0, tm.min(ls_all(a.dsa1, a.dsa2, a.dza1, a.dza2)));
    double num = 0.0;
    for (int i = tm.r; i < p; i += NT) {
      num = fma(a.s1[i] + alpha_a * a.dsa1[i], a.z1[i] + alpha_a * a.dza1[i], num);
      num = fma(a.s2[i] + alpha_a * a.dsa2[i], a.z2[i] + alpha_a * a.dza2[i], num);
    }
    num = tm.sum(num);
    const double ratio = num / sz;
    const double sigma = ratio * ratio * ratio;
    for (int i = tm.r; i < p; i += NT) {
      a.v3[i] = -(-a.v3[i] - (sigma * mu - a.dsa1[i] * a.dza1[i]));
      a.v4[i] = -(-a.v4[i] - (sigma * mu - a.dsa2[i] * a.dza2[i]));
    }
    tm.sync();
    solve(a.v1, a.v2, a.v3, a.v4, a.v5, a.v6, false, a.dx, a.dt, a.ds1, a.ds2, a.dz1, a.dz2);
    const double ls = tm.min(ls_all(a.ds1, a.ds2, a.dz1, a.dz2));
    const double alpha = 0.99 * nmin(1.0, 0.99 * nmin(1.0, ls));
    step_update(alpha);
    return converged;
  }

  // qpax/elastic_qp.py:235-316
  QPB_NOINLINE int newton_step() {
    const Team<NT>& tm = T();
    const double nrm = residuals(true, P->kappa);
    const int converged = (nrm < P->tol) ? 1 : 0;
    solve(a.v1, a.v2, a.v3, a.v4, a.v5, a.v6, true, a.dx, a.dt, a.ds1, a.ds2, a.dz1, a.dz2);
    const double ls = tm.min(ls_all(a.ds1, a.ds2, a.dz1, a.dz2));
    const double alpha = 0.99 * nmin(1.0, 0.99 * nmin(1.0, ls));
    step_update(alpha);
    return converged;
  }

  // qpax/elastic_qp.py:9-47
  QPB_NOINLINE void initialize() {
    const Team<NT>& tm = T();
    for (int i = tm.r; i < p; i += NT) {
      a.w[i] = 0.5;
      a.tp[i] = 0.5 * (pen - a.h[i]);
    }
    tm.sync();
    k.factor();
    cols_dot(tm, p, n, a.G, ld, a.tp, [&](int j, double g) { a.v1[j] = -a.q[j] - g; });
    tm.sync();
    k.reduced(a.v1, nullptr, a.x, nullptr);
    double zmax = -INFINITY, zmin = INFINITY;
    rows_dot(tm, p, n, a.G, ld, a.x, [&](int i, double g) {
      const double z2 = 0.5 * ((g + pen) - a.h[i]);
      const double z1 = pen - z2;
      a.z2[i] = z2;
      a.z1[i] = z1;
      a.t[i] = -z1;
      zmax = nmax(zmax, nmax(z1, z2));
      zmin = nmin(zmin, nmin(z1, z2));
    });
    const double alpha_p = tm.max(zmax);
    const double alpha_d = -tm.min(zmin);
    for (int i = tm.r; i < p; i += NT) {
      const double z1 = a.z1[i], z2 = a.z2[i];
      a.s1[i] = (alpha_p < 0) ? -z1 : -z1 + (1.0 + alpha_p);
      a.s2[i] = (alpha_p < 0) ? -z2 : -z2 + (1.0 + alpha_p);
      if (alpha_d >= 0) {
        a.z1[i] = z1 + (1.0 + alpha_d);
        a.z2[i] = z2 + (1.0 + alpha_d);
      }
    }
    tm.sync();
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

  // qpax/elastic_qp.py:381-417 at the arena iterate (lam1 = z1, lam2 = z2).
  QPB_NOINLINE void adjoint(long inst) {
    const Team<NT>& tm = T();
    for (int j = tm.r; j < n; j += NT) a.v1[j] = -P->gx[inst * n + j];
    tm.sync();
    k.use64 = 0;
    solve(a.v1, a.zp, a.zp, a.zp, a.zp, a.zp, true, a.dx, a.dt, a.ds1, a.ds2, a.dz1, a.dz2);
    double* dQ = P->dQ + inst * (long)n * n;
    for (int e = tm.r; e < n * n; e += NT) {
      const int i = e / n, j = e - i * n;
      dQ[e] = 0.5 * (a.dx[i] * a.x[j] + a.x[i] * a.dx[j]);
    }
    double* dG = P->dG + inst * (long)p * n;
    for (int e = tm.r; e < p * n; e += NT) {
      const int i = e / n, j = e - i * n;
      const double lam = a.z2[i];
      const double dlam = a.dz2[i] / lam;
      dG[e] = lam * (dlam * a.x[j] + lam * a.dx[j]);
    }
    for (int j = tm.r; j < n; j += NT) P->dq[inst * n + j] = a.dx[j];
    for (int i = tm.r; i < p; i += NT) {
      const double lam = a.z2[i];
      P->dh[inst * p + i] = -lam * (a.dz2[i] / lam);
    }
  }

  QPB_NOINLINE void run(long inst) {
    const Team<NT>& tm = T();
    k.reset_stats();
    const int op = P->op;
    int conv = 0, iters = 0;
    load(inst);
    if (op == kOpESolve) {
      initialize();
      loop(false, &conv, &iters);
      store_iterate(inst);
    } else if (op == kOpEInit) {
      initialize();
      store_iterate(inst);
    } else if (op == kOpERelax || op == kOpEBwd) {
      load_iterate(inst);
      loop(true, &conv, &iters);
      if (P->out[0]) store_iterate(inst);
      if (op == kOpEBwd) adjoint(inst);
    } else if (op == kOpEAdjoint) {
      load_iterate(inst);
      adjoint(inst);
    }
    if (tm.r == 0) {
      if (P->conv) P->conv[inst] = conv;
      if (P->iters) P->iters[inst] = iters;
      if (P->stats) {
        P->stats[inst * 4 + kStatFact32] = k.st_f32;
        P->stats[inst * 4 + kStatFact64] = k.st_f64;
        P->stats[inst * 4 + kStatSweeps] = k.st_sweeps;
        P->stats[inst * 4 + kStatFlags] = k.st_flags;
      }
    }
    tm.sync();
  }
};

}  // namespace qpb
