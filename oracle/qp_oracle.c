/*
 * qp_oracle.c -- FP64 CPU restatement of qpax's interior-point QP method.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed
 * CPU baseline for the CUDA library in qpax_b200/.  It is never linked into,
 * called by, or used as a fallback for the product path.
 *
 * Every routine restates one function of qpax (kevin-tracy/qpax, v0.0.9)
 * formula by formula, in the same order, in double precision:
 *   qpax/pdip.py          qr_solve :10-12, initialize :15-35,
 *                         factorize_kkt :38-46, solve_kkt_rhs :49-63,
 *                         ort_linesearch :66-73, centering_params :76-84,
 *                         pdip_pc_step :87-119, solve_eq_only :137-150,
 *                         remove_inf_constraints :166-178, solve_qp :181-251
 *   qpax/pdip_relaxed.py  pdip_newton_step :7-52, relax_qp :70-103
 *   qpax/diff_qp.py       optnet_derivatives :8-17, diff_qp :20-46
 *   qpax/elastic_qp.py    solve_init_elastic_ls :9-24, initialize_elastic :27-47,
 *                         solve_elastic_kkt_affine :50-72, solve_elastic_kkt_cc :75-96,
 *                         pdip_pc_step_elastic :99-174, solve_qp_elastic :184-228,
 *                         pdip_newton_step_elastic :235-316, relax_qp_elastic :319-359,
 *                         optnet_derivatives_elastic :366-373, diff_qp_elastic :381-417
 *
 * qpax delegates QR and triangular solves to jax/jaxlib (jnp.linalg.qr,
 * jax.scipy.linalg.solve_triangular; pyproject.toml pins jax>=0.4.0 only).
 * Both are LAPACK-style Householder QR (geqrf) and an upper-triangular
 * back substitution; they are restated here (qr_factor / qr_solve) after the
 * published LAPACK dgeqrf/dlarfg algorithm.  jnp.linalg.solve (LU with
 * partial pivoting, LAPACK dgesv) is restated in lu_solve.
 *
 * Batched entry points take a ragged batch: shapes[3*i] = (n, m, p) of
 * instance i, and every array is the concatenation of the per-instance
 * row-major arrays in instance order.  Instances run in parallel with OpenMP.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAX_ITERS 30 /* qpax/pdip.py:232, pdip_relaxed.py:76, elastic_qp.py:195,325 */

/* Optional per-iteration record of the KKT residual inf-norm (debug aid). */
static __thread double *g_trace = NULL;

/* ---------------------------------------------------------------- helpers */

/* NaN-propagating min/max, as jnp.min / jnp.max behave. */
static double nmin(double a, double b) { return (isnan(a) || isnan(b)) ? NAN : (a < b ? a : b); }
static double nmax(double a, double b) { return (isnan(a) || isnan(b)) ? NAN : (a > b ? a : b); }

/* jnp.linalg.norm(v, ord=inf) accumulated over several vectors. */
static double inf_norm_acc(double acc, const double *v, int k) {
  for (int i = 0; i < k; i++) acc = nmax(acc, fabs(v[i]));
  return acc;
}

/* y = M x, M is r x c row-major */
static void mv(int r, int c, const double *M, const double *x, double *y) {
  for (int i = 0; i < r; i++) {
    double a = 0.0;
    for (int j = 0; j < c; j++) a += M[(size_t)i * c + j] * x[j];
    y[i] = a;
  }
}

/* y = M^T x, M is r x c row-major */
static void mtv(int r, int c, const double *M, const double *x, double *y) {
  for (int j = 0; j < c; j++) y[j] = 0.0;
  for (int i = 0; i < r; i++) {
    const double xi = x[i];
    for (int j = 0; j < c; j++) y[j] += M[(size_t)i * c + j] * xi;
  }
}

static double dot(int k, const double *a, const double *b) {
  double s = 0.0;
  for (int i = 0; i < k; i++) s += a[i] * b[i];
  return s;
}

/* ------------------------------------------------- Householder QR (geqrf) */

/* In-place QR of the k x k row-major matrix R: R keeps the triangular
 * factor on and above the diagonal and the Householder vectors (unit
 * leading entry implied) below it; tau holds the reflector scales.
 * Follows LAPACK dgeqrf / dlarfg. */
static void qr_factor(int k, double *R, double *tau) {
  for (int j = 0; j < k; j++) {
    const double alpha = R[(size_t)j * k + j];
    double xn = 0.0;
    for (int i = j + 1; i < k; i++) xn += R[(size_t)i * k + j] * R[(size_t)i * k + j];
    xn = sqrt(xn);
    if (xn == 0.0) {
      tau[j] = 0.0;
      continue;
    }
    const double beta = -copysign(hypot(alpha, xn), alpha);
    tau[j] = (beta - alpha) / beta;
    const double scal = 1.0 / (alpha - beta);
    for (int i = j + 1; i < k; i++) R[(size_t)i * k + j] *= scal;
    R[(size_t)j * k + j] = beta;
    for (int c = j + 1; c < k; c++) {
      double d = R[(size_t)j * k + c];
      for (int i = j + 1; i < k; i++) d += R[(size_t)i * k + j] * R[(size_t)i * k + c];
      d *= tau[j];
      R[(size_t)j * k + c] -= d;
      for (int i = j + 1; i < k; i++) R[(size_t)i * k + c] -= d * R[(size_t)i * k + j];
    }
  }
}

/* qpax/pdip.py:10-12  qr_solve(qr, rhs) = solve_triangular(R, Q^T rhs). In place on b. */
static void qr_solve(int k, const double *R, const double *tau, double *b) {
  for (int j = 0; j < k; j++) {
    if (tau[j] == 0.0) continue;
    double d = b[j];
    for (int i = j + 1; i < k; i++) d += R[(size_t)i * k + j] * b[i];
    d *= tau[j];
    b[j] -= d;
    for (int i = j + 1; i < k; i++) b[i] -= d * R[(size_t)i * k + j];
  }
  for (int i = k - 1; i >= 0; i--) {
    double v = b[i];
    for (int c = i + 1; c < k; c++) v -= R[(size_t)i * k + c] * b[c];
    b[i] = v / R[(size_t)i * k + i];
  }
}

/* jnp.linalg.solve(M, b): LU with partial pivoting (LAPACK dgesv). M is destroyed. */
static void lu_solve(int k, double *M, double *b) {
  for (int j = 0; j < k; j++) {
    int piv = j;
    double best = fabs(M[(size_t)j * k + j]);
    for (int i = j + 1; i < k; i++) {
      double a = fabs(M[(size_t)i * k + j]);
      if (a > best) { best = a; piv = i; }
    }
    if (piv != j) {
      for (int c = 0; c < k; c++) {
        double t = M[(size_t)j * k + c];
        M[(size_t)j * k + c] = M[(size_t)piv * k + c];
        M[(size_t)piv * k + c] = t;
      }
      double t = b[j]; b[j] = b[piv]; b[piv] = t;
    }
    const double d = M[(size_t)j * k + j];
    for (int i = j + 1; i < k; i++) {
      const double l = M[(size_t)i * k + j] / d;
      M[(size_t)i * k + j] = l;
      for (int c = j + 1; c < k; c++) M[(size_t)i * k + c] -= l * M[(size_t)j * k + c];
      b[i] -= l * b[j];
    }
  }
  for (int i = k - 1; i >= 0; i--) {
    double v = b[i];
    for (int c = i + 1; c < k; c++) v -= M[(size_t)i * k + c] * b[c];
    b[i] = v / M[(size_t)i * k + i];
  }
}

/* ------------------------------------------------------------ KKT system */

typedef struct {
  int n, m, p;
  double *w;      /* P_inv_vec = z/s               (p)   */
  double *RH;     /* QR of H = Q + G^T diag(w) G    (n*n) */
  double *tH;     /*                                (n)   */
  double *RF;     /* QR of F = A H^-1 A^T           (m*m) */
  double *tF;     /*                                (m)   */
  double *tmp_n;  /* scratch                        (n)   */
  double *tmp_n2; /*                                (n)   */
  double *tmp_m;  /*                                (m)   */
  double *tmp_p;  /*                                (p)   */
} kkt_t;

static void kkt_alloc(kkt_t *K, int n, int m, int p) {
  K->n = n; K->m = m; K->p = p;
  size_t tot = (size_t)p + (size_t)n * n + n + (size_t)m * m + m + n + n + m + p + 8;
  double *buf = (double *)calloc(tot, sizeof(double));
  K->w = buf; buf += p;
  K->RH = buf; buf += (size_t)n * n;
  K->tH = buf; buf += n;
  K->RF = buf; buf += (size_t)m * m;
  K->tF = buf; buf += m;
  K->tmp_n = buf; buf += n;
  K->tmp_n2 = buf; buf += n;
  K->tmp_m = buf; buf += m;
  K->tmp_p = buf;
}
static void kkt_free(kkt_t *K) { free(K->w); }

/* H = Q + G^T diag(w) G, then QR(H), F = A qr_solve(H, A^T), QR(F). */
static void factor_H_F(kkt_t *K, const double *Q, const double *G, const double *A) {
  const int n = K->n, m = K->m, p = K->p;
  double *H = K->RH;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double a = 0.0;
      for (int k = 0; k < p; k++) a += G[(size_t)k * n + i] * (K->w[k] * G[(size_t)k * n + j]);
      H[(size_t)i * n + j] = Q[(size_t)i * n + j] + a;
    }
  qr_factor(n, H, K->tH);
  /* F[:, c] = A (H^-1 A[c, :]^T) */
  for (int c = 0; c < m; c++) {
    memcpy(K->tmp_n, A + (size_t)c * n, sizeof(double) * n);
    qr_solve(n, K->RH, K->tH, K->tmp_n);
    for (int r = 0; r < m; r++) K->RF[(size_t)r * m + c] = dot(n, A + (size_t)r * n, K->tmp_n);
  }
  qr_factor(m, K->RF, K->tF);
}

/* qpax/pdip.py:38-46 factorize_kkt */
static void factorize_kkt(kkt_t *K, const double *Q, const double *G, const double *A, const double *s,
                          const double *z) {
  for (int i = 0; i < K->p; i++) K->w[i] = z[i] / s[i];
  factor_H_F(K, Q, G, A);
}

/* qpax/pdip.py:49-63 solve_kkt_rhs (Algorithm 1). Outputs dx(n) ds(p) dz(p) dy(m). */
static void solve_kkt_rhs(kkt_t *K, const double *G, const double *A, const double *s, const double *z,
                          const double *v1, const double *v2, const double *v3, const double *v4, double *dx,
                          double *ds, double *dz, double *dy) {
  const int n = K->n, m = K->m, p = K->p;
  double *r2 = K->tmp_p;
  double *p1 = K->tmp_n2;
  for (int i = 0; i < p; i++) r2[i] = v3[i] - v2[i] / z[i];
  for (int i = 0; i < p; i++) r2[i] = K->w[i] * r2[i];
  mtv(p, n, G, r2, p1);
  for (int j = 0; j < n; j++) p1[j] = v1[j] + p1[j];
  /* dy = qr_solve(L_F, A @ qr_solve(L_H, p1) - v4) */
  memcpy(K->tmp_n, p1, sizeof(double) * n);
  qr_solve(n, K->RH, K->tH, K->tmp_n);
  mv(m, n, A, K->tmp_n, dy);
  for (int i = 0; i < m; i++) dy[i] = dy[i] - v4[i];
  qr_solve(m, K->RF, K->tF, dy);
  /* dx = qr_solve(L_H, p1 - A^T dy) */
  mtv(m, n, A, dy, dx);
  for (int j = 0; j < n; j++) dx[j] = p1[j] - dx[j];
  qr_solve(n, K->RH, K->tH, dx);
  /* ds = v3 - G dx ; dz = (v2 - z*ds)/s */
  mv(p, n, G, dx, ds);
  for (int i = 0; i < p; i++) ds[i] = v3[i] - ds[i];
  for (int i = 0; i < p; i++) dz[i] = (v2[i] - z[i] * ds[i]) / s[i];
}

/* qpax/pdip.py:66-73 ort_linesearch: min(1, min_{dx<0} -x/dx) */
static double ort_linesearch(int k, const double *x, const double *dx) {
  double mn = INFINITY;
  for (int i = 0; i < k; i++) {
    double v = (dx[i] < 0) ? -x[i] / dx[i] : INFINITY;
    mn = nmin(mn, v);
  }
  return nmin(1.0, mn);
}

/* qpax/pdip.py:76-84 centering_params */
static void centering_params(int k, const double *s, const double *z, const double *ds_a, const double *dz_a,
                             double *sigma, double *mu) {
  const double sz = dot(k, s, z);
  *mu = sz / k;
  const double alpha = nmin(ort_linesearch(k, s, ds_a), ort_linesearch(k, z, dz_a));
  double num = 0.0;
  for (int i = 0; i < k; i++) num += (s[i] + alpha * ds_a[i]) * (z[i] + alpha * dz_a[i]);
  const double ratio = num / sz;
  *sigma = ratio * ratio * ratio;
}

/* -------------------------------------------------------------- solve_qp */

/* qpax/pdip.py:15-35 initialize (CVXGEN/CVXOPT starting point). */
static void initialize(int n, int m, int p, const double *Q, const double *q, const double *A, const double *b,
                       const double *G, const double *h, double *x, double *s, double *z, double *y) {
  kkt_t K;
  kkt_alloc(&K, n, m, p);
  for (int i = 0; i < p; i++) K.w[i] = 1.0; /* H = Q + G^T G */
  factor_H_F(&K, Q, G, A);
  double *r1 = K.tmp_n2;
  mtv(p, n, G, h, r1);
  for (int j = 0; j < n; j++) r1[j] = -q[j] + r1[j];
  memcpy(K.tmp_n, r1, sizeof(double) * n);
  qr_solve(n, K.RH, K.tH, K.tmp_n);
  mv(m, n, A, K.tmp_n, y);
  for (int i = 0; i < m; i++) y[i] = y[i] - b[i];
  qr_solve(m, K.RF, K.tF, y);
  mtv(m, n, A, y, x);
  for (int j = 0; j < n; j++) x[j] = r1[j] - x[j];
  qr_solve(n, K.RH, K.tH, x);
  mv(p, n, G, x, z);
  for (int i = 0; i < p; i++) z[i] = z[i] - h[i];
  double alpha_p = -INFINITY, minz = INFINITY;
  for (int i = 0; i < p; i++) {
    alpha_p = nmax(alpha_p, z[i]); /* -min(-z) */
    minz = nmin(minz, z[i]);
  }
  for (int i = 0; i < p; i++) s[i] = (alpha_p < 0) ? -z[i] : -z[i] + (1.0 + alpha_p);
  const double alpha_d = -minz;
  if (alpha_d >= 0)
    for (int i = 0; i < p; i++) z[i] = z[i] + (1.0 + alpha_d);
  kkt_free(&K);
}

/* Residuals of the (relaxed) KKT conditions; returns the inf-norm.
 * qpax/pdip.py:93-100 (kappa = 0) and pdip_relaxed.py:16-23. */
static double kkt_residuals(int n, int m, int p, const double *Q, const double *q, const double *A, const double *b,
                            const double *G, const double *h, const double *x, const double *s, const double *z,
                            const double *y, double kappa, double *r1, double *r2, double *r3, double *r4,
                            double *tmp_n) {
  mv(n, n, Q, x, r1);
  for (int j = 0; j < n; j++) r1[j] += q[j];
  mtv(m, n, A, y, tmp_n);
  for (int j = 0; j < n; j++) r1[j] += tmp_n[j];
  mtv(p, n, G, z, tmp_n);
  for (int j = 0; j < n; j++) r1[j] += tmp_n[j];
  for (int i = 0; i < p; i++) r2[i] = s[i] * z[i] - kappa;
  mv(p, n, G, x, r3);
  for (int i = 0; i < p; i++) r3[i] = r3[i] + s[i] - h[i];
  mv(m, n, A, x, r4);
  for (int i = 0; i < m; i++) r4[i] = r4[i] - b[i];
  double nrm = -INFINITY;
  nrm = inf_norm_acc(nrm, r1, n);
  nrm = inf_norm_acc(nrm, r2, p);
  nrm = inf_norm_acc(nrm, r3, p);
  nrm = inf_norm_acc(nrm, r4, m);
  return nrm;
}

typedef struct {
  double *r1, *r2, *r3, *r4, *dx, *ds, *dz, *dy, *dsa, *dza, *tmp_n, *v1, *v2, *v3, *v4;
  double *buf;
} step_ws_t;

static void step_ws_alloc(step_ws_t *W, int n, int m, int p) {
  size_t tot = (size_t)4 * n + 7 * (size_t)p + 3 * (size_t)m + 8 + (size_t)p;
  double *b = (double *)calloc(tot, sizeof(double));
  W->buf = b;
  W->r1 = b; b += n;
  W->r2 = b; b += p;
  W->r3 = b; b += p;
  W->r4 = b; b += m;
  W->dx = b; b += n;
  W->ds = b; b += p;
  W->dz = b; b += p;
  W->dy = b; b += m;
  W->dsa = b; b += p;
  W->dza = b; b += p;
  W->tmp_n = b; b += n;
  W->v1 = b; b += n;
  W->v2 = b; b += p;
  W->v3 = b; b += p;
  W->v4 = b;
}

/* qpax/pdip.py:87-119 pdip_pc_step. Tests convergence on the incoming
 * iterate, then always takes the step. Returns the converged flag. */
static int pdip_pc_step(kkt_t *K, step_ws_t *W, const double *Q, const double *q, const double *A, const double *b,
                        const double *G, const double *h, double *x, double *s, double *z, double *y, double tol) {
  const int n = K->n, m = K->m, p = K->p;
  const double nrm = kkt_residuals(n, m, p, Q, q, A, b, G, h, x, s, z, y, 0.0, W->r1, W->r2, W->r3, W->r4, W->tmp_n);
  const int converged = (nrm < tol) ? 1 : 0;
  if (g_trace) *g_trace++ = nrm;
  factorize_kkt(K, Q, G, A, s, z);
  for (int j = 0; j < n; j++) W->v1[j] = -W->r1[j];
  for (int i = 0; i < p; i++) W->v2[i] = -W->r2[i];
  for (int i = 0; i < p; i++) W->v3[i] = -W->r3[i];
  for (int i = 0; i < m; i++) W->v4[i] = -W->r4[i];
  solve_kkt_rhs(K, G, A, s, z, W->v1, W->v2, W->v3, W->v4, W->dx, W->dsa, W->dza, W->dy);
  double sigma, mu;
  centering_params(p, s, z, W->dsa, W->dza, &sigma, &mu);
  for (int i = 0; i < p; i++) W->r2[i] = W->r2[i] - (sigma * mu - (W->dsa[i] * W->dza[i]));
  for (int i = 0; i < p; i++) W->v2[i] = -W->r2[i];
  solve_kkt_rhs(K, G, A, s, z, W->v1, W->v2, W->v3, W->v4, W->dx, W->ds, W->dz, W->dy);
  const double alpha = 0.99 * nmin(ort_linesearch(p, s, W->ds), ort_linesearch(p, z, W->dz));
  for (int j = 0; j < n; j++) x[j] = x[j] + alpha * W->dx[j];
  for (int i = 0; i < p; i++) s[i] = s[i] + alpha * W->ds[i];
  for (int i = 0; i < p; i++) z[i] = z[i] + alpha * W->dz[i];
  for (int i = 0; i < m; i++) y[i] = y[i] + alpha * W->dy[i];
  return converged;
}

/* qpax/pdip.py:137-150 solve_eq_only (Schur complement on A, QR of raw Q). */
static void solve_eq_only(int n, int m, const double *Q, const double *q, const double *A, const double *b, double *x,
                          double *y) {
  double *RQ = (double *)malloc(sizeof(double) * ((size_t)n * n + n + (size_t)m * m + m + 2 * (size_t)n + 2));
  double *tQ = RQ + (size_t)n * n;
  double *RS = tQ + n;
  double *tS = RS + (size_t)m * m;
  double *tn = tS + m;
  double *tn2 = tn + n;
  memcpy(RQ, Q, sizeof(double) * n * n);
  qr_factor(n, RQ, tQ);
  /* S = -A Q^-1 A^T */
  for (int c = 0; c < m; c++) {
    memcpy(tn, A + (size_t)c * n, sizeof(double) * n);
    qr_solve(n, RQ, tQ, tn);
    for (int r = 0; r < m; r++) RS[(size_t)r * m + c] = -dot(n, A + (size_t)r * n, tn);
  }
  qr_factor(m, RS, tS);
  memcpy(tn, q, sizeof(double) * n);
  qr_solve(n, RQ, tQ, tn); /* Qinv_g */
  mv(m, n, A, tn, y);
  for (int i = 0; i < m; i++) y[i] = y[i] + b[i];
  qr_solve(m, RS, tS, y);
  mtv(m, n, A, y, tn2);
  for (int j = 0; j < n; j++) x[j] = -tn2[j] - q[j];
  qr_solve(n, RQ, tQ, x);
  free(RQ);
}

/* qpax/pdip.py:181-251 solve_qp for one instance. */
static void solve_qp_one(int n, int m, int p, const double *Qin, const double *q, const double *A, const double *b,
                         const double *Gin, const double *hin, double tol, double *x, double *s, double *z, double *y,
                         int32_t *conv, int32_t *iters) {
  if (m == 0 && p == 0) { /* :208-211 */
    double *M = (double *)malloc(sizeof(double) * ((size_t)n * n + 1));
    memcpy(M, Qin, sizeof(double) * n * n);
    for (int j = 0; j < n; j++) x[j] = -q[j];
    lu_solve(n, M, x);
    free(M);
    *conv = 1;
    *iters = 0;
    return;
  }
  if (p == 0) { /* :213-217 */
    solve_eq_only(n, m, Qin, q, A, b, x, y);
    *conv = 1;
    *iters = 0;
    return;
  }
  double *Q = (double *)malloc(sizeof(double) * ((size_t)n * n + (size_t)p * n + p + 1));
  double *G = Q + (size_t)n * n;
  double *h = G + (size_t)p * n;
  unsigned char *mask = (unsigned char *)malloc((size_t)p + 1);
  /* :166-178 remove_inf_constraints */
  for (int i = 0; i < p; i++) {
    mask[i] = isinf(hin[i]) ? 1 : 0;
    h[i] = mask[i] ? 0.0 : hin[i];
    for (int j = 0; j < n; j++) G[(size_t)i * n + j] = mask[i] ? 0.0 : Gin[(size_t)i * n + j];
  }
  /* :223 symmetrize */
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) Q[(size_t)i * n + j] = 0.5 * (Qin[(size_t)i * n + j] + Qin[(size_t)j * n + i]);
  initialize(n, m, p, Q, q, A, b, G, h, x, s, z, y);
  kkt_t K;
  kkt_alloc(&K, n, m, p);
  step_ws_t W;
  step_ws_alloc(&W, n, m, p);
  int converged = 0, it = 0;
  while (it < MAX_ITERS && converged == 0) {
    converged = pdip_pc_step(&K, &W, Q, q, A, b, G, h, x, s, z, y, tol);
    it++;
  }
  for (int i = 0; i < p; i++)
    if (mask[i]) {
      z[i] = 0.0;
      s[i] = INFINITY;
    }
  *conv = converged;
  *iters = it;
  free(W.buf);
  kkt_free(&K);
  free(mask);
  free(Q);
}

/* ------------------------------------------------------------ relax_qp */

/* qpax/pdip_relaxed.py:7-52 pdip_newton_step */
static int pdip_newton_step(kkt_t *K, step_ws_t *W, const double *Q, const double *q, const double *A,
                            const double *b, const double *G, const double *h, double *x, double *s, double *z,
                            double *y, double tol, double kappa) {
  const int n = K->n, m = K->m, p = K->p;
  const double nrm =
      kkt_residuals(n, m, p, Q, q, A, b, G, h, x, s, z, y, kappa, W->r1, W->r2, W->r3, W->r4, W->tmp_n);
  const int converged = (nrm < tol) ? 1 : 0;
  factorize_kkt(K, Q, G, A, s, z);
  for (int j = 0; j < n; j++) W->v1[j] = -W->r1[j];
  for (int i = 0; i < p; i++) W->v2[i] = -W->r2[i];
  for (int i = 0; i < p; i++) W->v3[i] = -W->r3[i];
  for (int i = 0; i < m; i++) W->v4[i] = -W->r4[i];
  solve_kkt_rhs(K, G, A, s, z, W->v1, W->v2, W->v3, W->v4, W->dx, W->ds, W->dz, W->dy);
  const double alpha =
      0.99 * nmin(1.0, nmin(0.99 * ort_linesearch(p, s, W->ds), 0.99 * ort_linesearch(p, z, W->dz)));
  for (int j = 0; j < n; j++) x[j] = x[j] + alpha * W->dx[j];
  for (int i = 0; i < p; i++) s[i] = s[i] + alpha * W->ds[i];
  for (int i = 0; i < p; i++) z[i] = z[i] + alpha * W->dz[i];
  for (int i = 0; i < m; i++) y[i] = y[i] + alpha * W->dy[i];
  return converged;
}

/* qpax/pdip_relaxed.py:70-103 relax_qp (raw Q, G, h: no symmetrization or inf removal). */
static void relax_qp_one(int n, int m, int p, const double *Q, const double *q, const double *A, const double *b,
                         const double *G, const double *h, double *x, double *s, double *z, double *y, double tol,
                         double kappa, int32_t *conv, int32_t *iters) {
  kkt_t K;
  kkt_alloc(&K, n, m, p);
  step_ws_t W;
  step_ws_alloc(&W, n, m, p);
  int converged = 0, it = 0;
  while (it < MAX_ITERS && converged == 0) {
    converged = pdip_newton_step(&K, &W, Q, q, A, b, G, h, x, s, z, y, tol, kappa);
    it++;
  }
  *conv = converged;
  *iters = it;
  free(W.buf);
  kkt_free(&K);
}

/* qpax/diff_qp.py:20-46 diff_qp + :8-17 optnet_derivatives.
 * (x, s, lam, nu) is the relaxed iterate (xr, sr, zr, yr). */
static void diff_qp_one(int n, int m, int p, const double *Q, const double *A, const double *G, const double *x,
                        const double *s, const double *lam, const double *nu, const double *dl_dx, double *dQ,
                        double *dq, double *dA, double *db, double *dG, double *dh) {
  kkt_t K;
  kkt_alloc(&K, n, m, p);
  double *buf = (double *)calloc((size_t)4 * n + 6 * (size_t)p + 2 * (size_t)m + 8, sizeof(double));
  double *v1 = buf, *zp = v1 + n, *zm = zp + p, *dz = zm + m, *ds = dz + n, *dlt = ds + p, *dnu = dlt + p,
         *dlam = dnu + m;
  factorize_kkt(&K, Q, G, A, s, lam);
  for (int j = 0; j < n; j++) v1[j] = -dl_dx[j];
  solve_kkt_rhs(&K, G, A, s, lam, v1, zp, zp, zm, dz, ds, dlt, dnu);
  for (int i = 0; i < p; i++) dlam[i] = dlt[i] / lam[i];
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) dQ[(size_t)i * n + j] = 0.5 * (dz[i] * x[j] + x[i] * dz[j]);
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) dA[(size_t)i * n + j] = dnu[i] * x[j] + nu[i] * dz[j];
  for (int i = 0; i < p; i++)
    for (int j = 0; j < n; j++) dG[(size_t)i * n + j] = lam[i] * (dlam[i] * x[j] + lam[i] * dz[j]);
  for (int j = 0; j < n; j++) dq[j] = dz[j];
  for (int i = 0; i < m; i++) db[i] = -dnu[i];
  for (int i = 0; i < p; i++) dh[i] = -lam[i] * dlam[i];
  free(buf);
  kkt_free(&K);
}

/* ----------------------------------------------------------- elastic QP */

/* qpax/elastic_qp.py:50-72 / :75-96 Algorithm 5.  When `refactor` is set, H
 * is formed and factored (solve_elastic_kkt_affine); otherwise the QR held
 * in K from the previous call is reused (solve_elastic_kkt_cc). */
static void solve_elastic_kkt(kkt_t *K, int refactor, const double *s1, const double *z1, const double *s2,
                              const double *z2, const double *Q, const double *G, const double *r1, const double *r2,
                              const double *r3, const double *r4, const double *r5, const double *r6, double *dx,
                              double *dt, double *ds1, double *ds2, double *dz1, double *dz2, double *p1,
                              double *a3) {
  const int n = K->n, p = K->p;
  for (int i = 0; i < p; i++) {
    const double a1 = s1[i] / z1[i];
    const double a2 = s2[i] / z2[i];
    const double w1 = r3[i] / z1[i];
    const double w2 = r4[i] / z2[i];
    p1[i] = r5[i] - r6[i] + w2 - w1 - a1 * r2[i];
    a3[i] = a1 + a2;
  }
  if (refactor) {
    for (int i = 0; i < p; i++) K->w[i] = 1.0 / a3[i];
    factor_H_F(K, Q, G, NULL);
  }
  double *t = K->tmp_p;
  for (int i = 0; i < p; i++) t[i] = p1[i] / a3[i];
  mtv(p, n, G, t, dx);
  for (int j = 0; j < n; j++) dx[j] = r1[j] - dx[j];
  qr_solve(n, K->RH, K->tH, dx);
  mv(p, n, G, dx, dz2);
  for (int i = 0; i < p; i++) dz2[i] = (p1[i] + dz2[i]) / a3[i];
  for (int i = 0; i < p; i++) dz1[i] = -r2[i] - dz2[i];
  for (int i = 0; i < p; i++) ds1[i] = (r3[i] - s1[i] * dz1[i]) / z1[i];
  for (int i = 0; i < p; i++) ds2[i] = (r4[i] - s2[i] * dz2[i]) / z2[i];
  for (int i = 0; i < p; i++) dt[i] = ds1[i] - r5[i];
}

/* qpax/elastic_qp.py:9-47 solve_init_elastic_ls + initialize_elastic */
static void initialize_elastic(int n, int p, const double *Q, const double *q, const double *G, const double *h,
                               double penalty, double *x, double *t, double *s1, double *s2, double *z1,
                               double *z2) {
  kkt_t K;
  kkt_alloc(&K, n, 0, p);
  for (int i = 0; i < p; i++) K.w[i] = 0.5; /* Q + 0.5 G^T G */
  factor_H_F(&K, Q, G, NULL);
  double *d = K.tmp_p;
  for (int i = 0; i < p; i++) d[i] = 0.5 * (penalty - h[i]);
  mtv(p, n, G, d, x);
  for (int j = 0; j < n; j++) x[j] = -q[j] - x[j];
  qr_solve(n, K.RH, K.tH, x);
  mv(p, n, G, x, z2);
  for (int i = 0; i < p; i++) z2[i] = 0.5 * (z2[i] + penalty - h[i]);
  for (int i = 0; i < p; i++) z1[i] = penalty - z2[i];
  for (int i = 0; i < p; i++) t[i] = -z1[i];
  double alpha_p = -INFINITY, minz = INFINITY;
  for (int i = 0; i < p; i++) {
    alpha_p = nmax(alpha_p, nmax(z1[i], z2[i]));
    minz = nmin(minz, nmin(z1[i], z2[i]));
  }
  for (int i = 0; i < p; i++) {
    s1[i] = (alpha_p < 0) ? -z1[i] : -z1[i] + (1.0 + alpha_p);
    s2[i] = (alpha_p < 0) ? -z2[i] : -z2[i] + (1.0 + alpha_p);
  }
  const double alpha_d = -minz;
  if (alpha_d >= 0)
    for (int i = 0; i < p; i++) {
      z1[i] = z1[i] + (1.0 + alpha_d);
      z2[i] = z2[i] + (1.0 + alpha_d);
    }
  kkt_free(&K);
}

typedef struct {
  double *r1, *r2, *r3, *r4, *r5, *r6, *v1, *v2, *v3, *v4, *v5, *v6;
  double *dx, *dt, *ds1, *ds2, *dz1, *dz2, *p1, *a3, *tmp_n, *tmp_p;
  double *buf;
} ews_t;

static void ews_alloc(ews_t *W, int n, int p) {
  double *b = (double *)calloc((size_t)5 * n + 19 * (size_t)p + 8, sizeof(double));
  W->buf = b;
  W->r1 = b; b += n;
  W->v1 = b; b += n;
  W->dx = b; b += n;
  W->tmp_n = b; b += n;
  double **ps[] = {&W->r2, &W->r3, &W->r4, &W->r5, &W->r6, &W->v2, &W->v3, &W->v4, &W->v5,
                   &W->v6, &W->dt, &W->ds1, &W->ds2, &W->dz1, &W->dz2, &W->p1, &W->a3, &W->tmp_p};
  for (size_t k = 0; k < sizeof(ps) / sizeof(ps[0]); k++) {
    *ps[k] = b;
    b += p;
  }
}

/* Elastic residuals. `relaxed` selects the sign convention of
 * pdip_newton_step_elastic (:255-261) instead of pdip_pc_step_elastic
 * (:105-110); both are reproduced as written in qpax. */
static double elastic_residuals(ews_t *W, int n, int p, const double *Q, const double *q, const double *G,
                                const double *h, double pen, const double *x, const double *t, const double *s1,
                                const double *s2, const double *z1, const double *z2, int relaxed, double kappa) {
  mv(n, n, Q, x, W->r1);
  mtv(p, n, G, z2, W->tmp_n);
  for (int j = 0; j < n; j++) W->r1[j] = W->r1[j] + q[j] + W->tmp_n[j];
  mv(p, n, G, x, W->tmp_p);
  for (int i = 0; i < p; i++) {
    if (!relaxed) {
      W->r2[i] = -z1[i] - z2[i] + pen;
      W->r3[i] = s1[i] * z1[i];
      W->r4[i] = s2[i] * z2[i];
      W->r5[i] = -t[i] + s1[i];
      W->r6[i] = W->tmp_p[i] - t[i] + s2[i] - h[i];
    } else {
      W->r2[i] = z1[i] + z2[i] - pen;
      W->r3[i] = s1[i] * z1[i] - kappa;
      W->r4[i] = s2[i] * z2[i] - kappa;
      W->r5[i] = t[i] + s1[i];
      W->r6[i] = W->tmp_p[i] + t[i] + s2[i] - h[i];
    }
  }
  double nrm = -INFINITY;
  nrm = inf_norm_acc(nrm, W->r1, n);
  nrm = inf_norm_acc(nrm, W->r2, p);
  nrm = inf_norm_acc(nrm, W->r3, p);
  nrm = inf_norm_acc(nrm, W->r4, p);
  nrm = inf_norm_acc(nrm, W->r5, p);
  nrm = inf_norm_acc(nrm, W->r6, p);
  for (int j = 0; j < n; j++) W->v1[j] = -W->r1[j];
  for (int i = 0; i < p; i++) {
    W->v2[i] = -W->r2[i];
    W->v3[i] = -W->r3[i];
    W->v4[i] = -W->r4[i];
    W->v5[i] = -W->r5[i];
    W->v6[i] = -W->r6[i];
  }
  return nrm;
}

/* ort_linesearch on the stacked vectors (a1;a2) with directions (d1;d2). */
static double ls_stacked(int p, const double *a1, const double *a2, const double *d1, const double *d2) {
  return nmin(ort_linesearch(p, a1, d1), ort_linesearch(p, a2, d2));
}

/* qpax/elastic_qp.py:99-174 pdip_pc_step_elastic */
static int pdip_pc_step_elastic(kkt_t *K, ews_t *W, const double *Q, const double *q, const double *G,
                                const double *h, double pen, double *x, double *t, double *s1, double *s2, double *z1,
                                double *z2, double tol) {
  const int n = K->n, p = K->p;
  const double nrm = elastic_residuals(W, n, p, Q, q, G, h, pen, x, t, s1, s2, z1, z2, 0, 0.0);
  const int converged = (nrm < tol) ? 1 : 0;
  solve_elastic_kkt(K, 1, s1, z1, s2, z2, Q, G, W->v1, W->v2, W->v3, W->v4, W->v5, W->v6, W->dx, W->dt, W->ds1,
                    W->ds2, W->dz1, W->dz2, W->p1, W->a3);
  /* centering on s = [s1; s2], z = [z1; z2] (qpax/pdip.py:76-84) */
  const double sz = dot(p, s1, z1) + dot(p, s2, z2);
  const double mu = sz / (2 * p);
  const double alpha_a = nmin(ls_stacked(p, s1, s2, W->ds1, W->ds2), ls_stacked(p, z1, z2, W->dz1, W->dz2));
  double num = 0.0;
  for (int i = 0; i < p; i++) num += (s1[i] + alpha_a * W->ds1[i]) * (z1[i] + alpha_a * W->dz1[i]);
  for (int i = 0; i < p; i++) num += (s2[i] + alpha_a * W->ds2[i]) * (z2[i] + alpha_a * W->dz2[i]);
  const double ratio = num / sz;
  const double sigma = ratio * ratio * ratio;
  for (int i = 0; i < p; i++) {
    W->r3[i] = W->r3[i] - (sigma * mu - (W->ds1[i] * W->dz1[i]));
    W->r4[i] = W->r4[i] - (sigma * mu - (W->ds2[i] * W->dz2[i]));
    W->v3[i] = -W->r3[i];
    W->v4[i] = -W->r4[i];
  }
  solve_elastic_kkt(K, 0, s1, z1, s2, z2, Q, G, W->v1, W->v2, W->v3, W->v4, W->v5, W->v6, W->dx, W->dt, W->ds1,
                    W->ds2, W->dz1, W->dz2, W->p1, W->a3);
  const double alpha = 0.99 * nmin(1.0, nmin(0.99 * ls_stacked(p, s1, s2, W->ds1, W->ds2),
                                             0.99 * ls_stacked(p, z1, z2, W->dz1, W->dz2)));
  for (int j = 0; j < n; j++) x[j] = x[j] + alpha * W->dx[j];
  for (int i = 0; i < p; i++) {
    t[i] = t[i] + alpha * W->dt[i];
    s1[i] = s1[i] + alpha * W->ds1[i];
    s2[i] = s2[i] + alpha * W->ds2[i];
    z1[i] = z1[i] + alpha * W->dz1[i];
    z2[i] = z2[i] + alpha * W->dz2[i];
  }
  return converged;
}

/* qpax/elastic_qp.py:235-316 pdip_newton_step_elastic */
static int pdip_newton_step_elastic(kkt_t *K, ews_t *W, const double *Q, const double *q, const double *G,
                                    const double *h, double pen, double *x, double *t, double *s1, double *s2,
                                    double *z1, double *z2, double tol, double kappa) {
  const int n = K->n, p = K->p;
  const double nrm = elastic_residuals(W, n, p, Q, q, G, h, pen, x, t, s1, s2, z1, z2, 1, kappa);
  const int converged = (nrm < tol) ? 1 : 0;
  solve_elastic_kkt(K, 1, s1, z1, s2, z2, Q, G, W->v1, W->v2, W->v3, W->v4, W->v5, W->v6, W->dx, W->dt, W->ds1,
                    W->ds2, W->dz1, W->dz2, W->p1, W->a3);
  const double alpha = 0.99 * nmin(1.0, nmin(0.99 * ls_stacked(p, s1, s2, W->ds1, W->ds2),
                                             0.99 * ls_stacked(p, z1, z2, W->dz1, W->dz2)));
  for (int j = 0; j < n; j++) x[j] = x[j] + alpha * W->dx[j];
  for (int i = 0; i < p; i++) {
    t[i] = t[i] + alpha * W->dt[i];
    s1[i] = s1[i] + alpha * W->ds1[i];
    s2[i] = s2[i] + alpha * W->ds2[i];
    z1[i] = z1[i] + alpha * W->dz1[i];
    z2[i] = z2[i] + alpha * W->dz2[i];
  }
  return converged;
}

/* qpax/elastic_qp.py:184-228 solve_qp_elastic (symmetrizes Q) and
 * :319-359 relax_qp_elastic (raw Q).  `relax` selects the loop. */
static void elastic_loop_one(int relax, int n, int p, const double *Qin, const double *q, const double *G,
                             const double *h, double pen, double tol, double kappa, double *x, double *t, double *s1,
                             double *s2, double *z1, double *z2, int32_t *conv, int32_t *iters) {
  double *Q = (double *)malloc(sizeof(double) * ((size_t)n * n + 1));
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      Q[(size_t)i * n + j] =
          relax ? Qin[(size_t)i * n + j] : 0.5 * (Qin[(size_t)i * n + j] + Qin[(size_t)j * n + i]);
  if (!relax) initialize_elastic(n, p, Q, q, G, h, pen, x, t, s1, s2, z1, z2);
  kkt_t K;
  kkt_alloc(&K, n, 0, p);
  ews_t W;
  ews_alloc(&W, n, p);
  int converged = 0, it = 0;
  while (it < MAX_ITERS && converged == 0) {
    converged = relax ? pdip_newton_step_elastic(&K, &W, Q, q, G, h, pen, x, t, s1, s2, z1, z2, tol, kappa)
                      : pdip_pc_step_elastic(&K, &W, Q, q, G, h, pen, x, t, s1, s2, z1, z2, tol);
    it++;
  }
  *conv = converged;
  *iters = it;
  free(W.buf);
  kkt_free(&K);
  free(Q);
}

/* qpax/elastic_qp.py:381-417 diff_qp_elastic + :366-373 optnet_derivatives_elastic,
 * already cropped to the (Q, q, G, h) blocks as :412-415 do. */
static void diff_qp_elastic_one(int n, int p, const double *Q, const double *G, const double *x, const double *t,
                                const double *s1, const double *s2, const double *lam1, const double *lam2,
                                const double *dl_dx, double *dQ, double *dq, double *dG, double *dh) {
  (void)t;
  kkt_t K;
  kkt_alloc(&K, n, 0, p);
  double *buf = (double *)calloc((size_t)2 * n + 10 * (size_t)p + 8, sizeof(double));
  double *v1 = buf, *dx = v1 + n, *zp = dx + n, *dt = zp + p, *ds1 = dt + p, *ds2 = ds1 + p, *dl1 = ds2 + p,
         *dl2 = dl1 + p, *p1 = dl2 + p, *a3 = p1 + p;
  for (int j = 0; j < n; j++) v1[j] = -dl_dx[j];
  solve_elastic_kkt(&K, 1, s1, lam1, s2, lam2, Q, G, v1, zp, zp, zp, zp, zp, dx, dt, ds1, ds2, dl1, dl2, p1, a3);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) dQ[(size_t)i * n + j] = 0.5 * (dx[i] * x[j] + x[i] * dx[j]);
  for (int j = 0; j < n; j++) dq[j] = dx[j];
  for (int i = 0; i < p; i++) {
    const double dlam = dl2[i] / lam2[i];
    for (int j = 0; j < n; j++) dG[(size_t)i * n + j] = lam2[i] * (dlam * x[j] + lam2[i] * dx[j]);
    dh[i] = -lam2[i] * dlam;
  }
  free(buf);
  kkt_free(&K);
}

/* ------------------------------------------------------- batched C ABI */

typedef struct {
  int64_t Q, q, A, b, G, h, n, m, p;
} offs_t;

/* Exclusive prefix sums of the per-instance array sizes. */
static offs_t *make_offsets(int B, const int32_t *shapes) {
  offs_t *o = (offs_t *)malloc(sizeof(offs_t) * ((size_t)B + 1));
  offs_t c = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < B; i++) {
    o[i] = c;
    const int64_t n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    c.Q += n * n; c.q += n; c.A += m * n; c.b += m; c.G += p * n; c.h += p;
    c.n += n; c.m += m; c.p += p;
  }
  o[B] = c;
  return o;
}

static int set_threads(int nthreads) {
#ifdef _OPENMP
  return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

int oracle_num_threads(void) { return set_threads(0); }

/* Batched solve_qp: x,s,z,y are packed like q,h,h,b. */
int oracle_solve_qp(int B, const int32_t *shapes, const double *Q, const double *q, const double *A, const double *b,
                    const double *G, const double *h, double tol, double *x, double *s, double *z, double *y,
                    int32_t *conv, int32_t *iters, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    solve_qp_one(n, m, p, Q + o[i].Q, q + o[i].q, A + o[i].A, b + o[i].b, G + o[i].G, h + o[i].h, tol, x + o[i].n,
                 s + o[i].p, z + o[i].p, y + o[i].m, conv + i, iters + i);
  }
  free(o);
  return 0;
}

/* Batched initialize (qpax/pdip.py:15-35), applied to the data as given. */
int oracle_initialize(int B, const int32_t *shapes, const double *Q, const double *q, const double *A,
                      const double *b, const double *G, const double *h, double *x, double *s, double *z, double *y,
                      int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    initialize(n, m, p, Q + o[i].Q, q + o[i].q, A + o[i].A, b + o[i].b, G + o[i].G, h + o[i].h, x + o[i].n,
               s + o[i].p, z + o[i].p, y + o[i].m);
  }
  free(o);
  return 0;
}

/* Batched relax_qp: (x,s,z,y) are read as the starting iterate and
 * overwritten with the relaxed iterate. */
int oracle_relax_qp(int B, const int32_t *shapes, const double *Q, const double *q, const double *A, const double *b,
                    const double *G, const double *h, double tol, double kappa, double *x, double *s, double *z,
                    double *y, int32_t *conv, int32_t *iters, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    relax_qp_one(n, m, p, Q + o[i].Q, q + o[i].q, A + o[i].A, b + o[i].b, G + o[i].G, h + o[i].h, x + o[i].n,
                 s + o[i].p, z + o[i].p, y + o[i].m, tol, kappa, conv + i, iters + i);
  }
  free(o);
  return 0;
}

/* Batched diff_qp at the relaxed iterate; gradients packed like the inputs. */
int oracle_diff_qp(int B, const int32_t *shapes, const double *Q, const double *A, const double *G, const double *x,
                   const double *s, const double *z, const double *y, const double *dl_dx, double *dQ, double *dq,
                   double *dA, double *db, double *dG, double *dh, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    diff_qp_one(n, m, p, Q + o[i].Q, A + o[i].A, G + o[i].G, x + o[i].n, s + o[i].p, z + o[i].p, y + o[i].m,
                dl_dx + o[i].n, dQ + o[i].Q, dq + o[i].q, dA + o[i].A, db + o[i].b, dG + o[i].G, dh + o[i].h);
  }
  free(o);
  return 0;
}

/* Forward + backward of solve_qp_primal in one call (qpax/diff_qp.py:61-79):
 * solve_qp, relax_qp from its output, then diff_qp with the incoming
 * gradient dl_dx.  Returns the unrelaxed x and the six gradients. */
int oracle_solve_qp_primal_fwd_bwd(int B, const int32_t *shapes, const double *Q, const double *q, const double *A,
                                   const double *b, const double *G, const double *h, double tol, double kappa,
                                   const double *dl_dx, double *x, double *dQ, double *dq, double *dA, double *db,
                                   double *dG, double *dh, int32_t *conv, int32_t *iters, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], m = shapes[3 * i + 1], p = shapes[3 * i + 2];
    double *buf = (double *)malloc(sizeof(double) * ((size_t)n + 2 * (size_t)p + m + 4));
    double *xr = buf, *sr = xr + n, *zr = sr + p, *yr = zr + p;
    int32_t c2, it2;
    solve_qp_one(n, m, p, Q + o[i].Q, q + o[i].q, A + o[i].A, b + o[i].b, G + o[i].G, h + o[i].h, tol, xr, sr, zr,
                 yr, conv + i, iters + i);
    memcpy(x + o[i].n, xr, sizeof(double) * n);
    relax_qp_one(n, m, p, Q + o[i].Q, q + o[i].q, A + o[i].A, b + o[i].b, G + o[i].G, h + o[i].h, xr, sr, zr, yr,
                 tol, kappa, &c2, &it2);
    diff_qp_one(n, m, p, Q + o[i].Q, A + o[i].A, G + o[i].G, xr, sr, zr, yr, dl_dx + o[i].n, dQ + o[i].Q,
                dq + o[i].q, dA + o[i].A, db + o[i].b, dG + o[i].G, dh + o[i].h);
    free(buf);
  }
  free(o);
  return 0;
}

/* Elastic batches use shapes (n, 0, p); x is packed like q, and
 * t, s1, s2, z1, z2 like h.  penalty holds one value per instance. */
int oracle_solve_qp_elastic(int B, const int32_t *shapes, const double *Q, const double *q, const double *G,
                            const double *h, const double *penalty, double tol, double *x, double *t, double *s1,
                            double *s2, double *z1, double *z2, int32_t *conv, int32_t *iters, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], p = shapes[3 * i + 2];
    elastic_loop_one(0, n, p, Q + o[i].Q, q + o[i].q, G + o[i].G, h + o[i].h, penalty[i], tol, 0.0, x + o[i].n,
                     t + o[i].p, s1 + o[i].p, s2 + o[i].p, z1 + o[i].p, z2 + o[i].p, conv + i, iters + i);
  }
  free(o);
  return 0;
}

int oracle_initialize_elastic(int B, const int32_t *shapes, const double *Q, const double *q, const double *G,
                              const double *h, const double *penalty, double *x, double *t, double *s1, double *s2,
                              double *z1, double *z2, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], p = shapes[3 * i + 2];
    initialize_elastic(n, p, Q + o[i].Q, q + o[i].q, G + o[i].G, h + o[i].h, penalty[i], x + o[i].n, t + o[i].p,
                       s1 + o[i].p, s2 + o[i].p, z1 + o[i].p, z2 + o[i].p);
  }
  free(o);
  return 0;
}

/* Batched relax_qp_elastic: the iterate is read and overwritten. */
int oracle_relax_qp_elastic(int B, const int32_t *shapes, const double *Q, const double *q, const double *G,
                            const double *h, const double *penalty, double tol, double kappa, double *x, double *t,
                            double *s1, double *s2, double *z1, double *z2, int32_t *conv, int32_t *iters,
                            int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], p = shapes[3 * i + 2];
    elastic_loop_one(1, n, p, Q + o[i].Q, q + o[i].q, G + o[i].G, h + o[i].h, penalty[i], tol, kappa, x + o[i].n,
                     t + o[i].p, s1 + o[i].p, s2 + o[i].p, z1 + o[i].p, z2 + o[i].p, conv + i, iters + i);
  }
  free(o);
  return 0;
}

int oracle_diff_qp_elastic(int B, const int32_t *shapes, const double *Q, const double *G, const double *x,
                           const double *t, const double *s1, const double *s2, const double *z1, const double *z2,
                           const double *dl_dx, double *dQ, double *dq, double *dG, double *dh, int nthreads) {
  offs_t *o = make_offsets(B, shapes);
  const int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int i = 0; i < B; i++) {
    const int n = shapes[3 * i], p = shapes[3 * i + 2];
    diff_qp_elastic_one(n, p, Q + o[i].Q, G + o[i].G, x + o[i].n, t + o[i].p, s1 + o[i].p, s2 + o[i].p, z1 + o[i].p,
                        z2 + o[i].p, dl_dx + o[i].n, dQ + o[i].Q, dq + o[i].q, dG + o[i].G, dh + o[i].h);
  }
  free(o);
  return 0;
}

/* solve_qp on one instance, recording the residual inf-norm tested at each
 * predictor-corrector iteration into trace[0..iters) (debug aid). */
int oracle_solve_qp_trace(int n, int m, int p, const double *Q, const double *q, const double *A, const double *b,
                          const double *G, const double *h, double tol, double *x, double *s, double *z, double *y,
                          int32_t *conv, int32_t *iters, double *trace) {
  g_trace = trace;
  solve_qp_one(n, m, p, Q, q, A, b, G, h, tol, x, s, z, y, conv, iters);
  g_trace = NULL;
  return 0;
}
