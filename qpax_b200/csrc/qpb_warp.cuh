// qpb_warp.cuh -- one warp per QP instance for n <= NP (NP = 8, 16, 32),
// m <= MP = NP / 4, any p; FP64 throughout.
//
// Same method and formula order as qpb_std.cuh (qpax/pdip.py, pdip_relaxed.py,
// diff_qp.py; citations there), laid out for a single warp so that no phase
// needs a block-wide barrier:
//   * lane j owns column j of H = Q + G' diag(w) G in registers (hc[NP]) and
//     factors it in place (LDL^T, right-looking, one shared-memory broadcast
//     of the pivot row per step).  Afterwards lane j holds column j of L
//     (scaled by d_j) below the diagonal and row j of L (scaled by d_i) above
//     it, which is exactly what column-oriented forward and backward
//     substitution need from that lane;
//   * Y = L^-1 A' (lane j holds Y[:, j]) and the Schur complement
//     F = Y' D^-1 Y (lane j < m holds column j of its LDL^T factor) stay in
//     registers too;
//   * n-vectors and m-vectors are lane-distributed registers; p-vectors and
//     the G, A operands live in shared memory; Q is read through L1/L2.
#pragma once
#include "qpb_params.h"
#include "qpb_team.cuh"

namespace qpb {

QPB_DEV double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
QPB_DEV double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
QPB_DEV double wmin(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Shared-memory layout of one warp instance (doubles, in this order):
//   G (p x NP) | A (MP x NP) | 9 p-vectors | xs, cb, dvi (NP each) |
//   Y (MP x NP, Y[i][j] = (L^-1 A')[j][i]) | F (MP x MP, column-held factor)
// Addresses are recomputed from the base and p where used (no pointer table).
struct WarpArena {
  static __host__ __device__ size_t doubles(int NP, int MP, int p) {
    return (size_t)p * NP + (size_t)MP * NP + 9 * (size_t)p + 3 * (size_t)NP + (size_t)MP * NP +
           (size_t)MP * MP;
  }
  static size_t bytes(int NP, int MP, int p) { return doubles(NP, MP, p) * sizeof(double) + 16; }
};

enum WarpSlot : int { kVh = 0, kVs, kVz, kVw, kVv2, kVv3, kVds, kVdz, kVtp };

// Arena addresses of one warp instance, recomputed from the base and p.
template <int NP, int MP>
struct WarpAddr {
  double* base;
  int p;
  QPB_DEV double* G() const { return base; }
  QPB_DEV double* A() const { return base + p * NP; }
  QPB_DEV double* v(int k) const { return base + p * NP + MP * NP + k * p; }
  QPB_DEV double* h() const { return v(kVh); }
  QPB_DEV double* s() const { return v(kVs); }
  QPB_DEV double* z() const { return v(kVz); }
  QPB_DEV double* w() const { return v(kVw); }
  QPB_DEV double* v2() const { return v(kVv2); }
  QPB_DEV double* v3() const { return v(kVv3); }
  QPB_DEV double* ds() const { return v(kVds); }
  QPB_DEV double* dz() const { return v(kVdz); }
  QPB_DEV double* tp() const { return v(kVtp); }
  QPB_DEV double* xs() const { return base + p * NP + MP * NP + 9 * p; }
  QPB_DEV double* cb() const { return xs() + NP; }
  QPB_DEV double* dvi() const { return xs() + 2 * NP; }
  QPB_DEV double* Y() const { return xs() + 3 * NP; }
  QPB_DEV double* F() const { return Y() + MP * NP; }
};

template <int NP, int MP>
struct WarpQP {
  static_assert(NP == 8 || NP == 16 || NP == 32, "NP");
  const Params* P;
  WarpAddr<NP, MP> a;
  int n, m, p, lane;
  const double* gQ;  // this instance's Q (row-major n x n, global)
  // lane-distributed registers
  double hc[NP];  // H column -> L, D
  double dinv;    // 1 / d_lane
  double fdinv;   // 1 / df_lane
  double x, q, v1, dx;  // n-vectors (lane j)
  double y, b, v4, dy;  // m-vectors (lane i)
  int st_f64, st_flags;

  QPB_DEV void setup(const Params& prm, unsigned char* arena, int ln) {
    P = &prm;
    n = prm.n; m = prm.m; p = prm.p;
    lane = ln;
    a.base = reinterpret_cast<double*>(arena);
    a.p = p;
  }

  // sym(Q)[i][lane] through L1 (Q is symmetrized on the fly: (Q + Q')/2).
  QPB_DEV double qsym(int i) const {
    return (i < n && lane < n) ? 0.5 * (gQ[i * n + lane] + gQ[lane * n + i]) : 0.0;
  }

  QPB_DEV void load(long inst, bool remove_inf) {
    gQ = P->Q + inst * (long)n * n;
    const double* gG = P->G + inst * (long)p * n;
    const double* gA = P->A + inst * (long)m * n;
    const double* gh = P->h + inst * (long)p;
    for (int r = 0; r < p; ++r) {
      double v = (lane < n) ? gG[r * n + lane] : 0.0;
      if (remove_inf && isinf(gh[r])) v = 0.0;
      if (lane < NP) a.G()[r * NP + lane] = v;
    }
#pragma unroll
    for (int i = 0; i < MP; ++i)
      if (lane < NP) a.A()[i * NP + lane] = (i < m && lane < n) ? gA[i * n + lane] : 0.0;
    for (int r = lane; r < p; r += 32) {
      const double hv = gh[r];
      a.h()[r] = (remove_inf && isinf(hv)) ? 0.0 : hv;
    }
    q = (lane < n) ? P->q[inst * n + lane] : 0.0;
    b = (lane < m) ? P->b[inst * m + lane] : 0.0;
    __syncwarp();
  }

  QPB_DEV void load_iterate(long inst) {
    x = (lane < n) ? P->in[0][inst * n + lane] : 0.0;
    y = (lane < m) ? P->in[3][inst * m + lane] : 0.0;
    for (int r = lane; r < p; r += 32) {
      a.s()[r] = P->in[1][inst * p + r];
      a.z()[r] = P->in[2][inst * p + r];
    }
    __syncwarp();
  }

  QPB_DEV void store_iterate(long inst, bool inf_rows) {
    if (lane < n) P->out[0][inst * n + lane] = x;
    if (lane < m) P->out[3][inst * m + lane] = y;
    for (int r = lane; r < p; r += 32) {
      double sv = a.s()[r], zv = a.z()[r];
      if (inf_rows && isinf(P->h[inst * p + r])) {  // qpax/pdip.py:243-246
        zv = 0.0;
        sv = INFINITY;
      }
      P->out[1][inst * p + r] = sv;
      P->out[2][inst * p + r] = zv;
    }
  }

  // ---------------------------------------------------------------- factor
  // H = sym(Q) + G' diag(w) G, LDL^T in registers, then Y and F.
  QPB_DEV void factor() {
    st_f64++;
    dinv = 0.0;
    fdinv = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) hc[i] = (lane >= n && i == lane) ? 1.0 : qsym(i);
    const double* Gc = a.G() + lane;
    for (int r = 0; r < p; ++r) {
      const double* row = a.G() + r * NP;
      const double ar = a.w()[r] * (lane < NP ? Gc[r * NP] : 0.0);
#pragma unroll
      for (int i = 0; i < NP; i += 2) {
        const double2 g2 = *reinterpret_cast<const double2*>(row + i);
        hc[i] = fma(g2.x, ar, hc[i]);
        hc[i + 1] = fma(g2.y, ar, hc[i + 1]);
      }
    }
    // LDL^T: step k broadcasts row k of the Schur complement (= column k)
    double dmin = INFINITY, dmax = 0.0;
    int bad = 0;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      if (lane < NP) a.cb()[lane] = hc[k];
      __syncwarp();
      const double dk = a.cb()[k];
      const double rk = 1.0 / dk;
      if (k < n) {
        bad |= !(dk > 0.0) || !isfinite(dk);
        dmin = fmin(dmin, dk);
        dmax = fmax(dmax, dk);
      }
      if (lane == k) dinv = rk;
      const double f = hc[k] * rk;
      if (lane > k) {
#pragma unroll
        for (int i = k + 1; i < NP; ++i) hc[i] = fma(-a.cb()[i], f, hc[i]);
      }
      __syncwarp();
    }
    if (lane < NP) a.dvi()[lane] = dinv;
    if (bad) st_flags |= kFlagBreakdown64;
    __syncwarp();
    // Y = L^-1 A'   (unit L; L[j][k] = hc[k] * dinv_k for lane j > k)
    double yc[MP];
#pragma unroll
    for (int i = 0; i < MP; ++i) yc[i] = (lane < NP) ? a.A()[i * NP + lane] : 0.0;
#pragma unroll
    for (int k = 0; k < NP - 1; ++k) {
      const double l = (lane > k && lane < NP) ? hc[k] * a.dvi()[k] : 0.0;
#pragma unroll
      for (int i = 0; i < MP; ++i) yc[i] = fma(-l, __shfl_sync(kFull, yc[i], k), yc[i]);
    }
    if (lane < NP) {
#pragma unroll
      for (int i = 0; i < MP; ++i) a.Y()[i * NP + lane] = yc[i];
    }
    __syncwarp();
    // F = Y D^-1 Y' (MP x MP, full storage, identity beyond m), one entry per lane
    double* Fm = a.F();
    const double* Ys = a.Y();
    const double* dv = a.dvi();
    for (int e = lane; e < MP * MP; e += 32) {
      const int r = e / MP, c = e - r * MP;
      double v = (r == c) ? 1.0 : 0.0;
      if (r < m && c < m) {
        double acc = 0.0;
#pragma unroll 8
        for (int j = 0; j < NP; ++j) acc = fma(Ys[r * NP + j] * dv[j], Ys[c * NP + j], acc);
        v = acc;
      }
      Fm[e] = v;
    }
    __syncwarp();
    // LDL^T of F in the same in-place layout as H: lane c owns column c
    for (int k = 0; k < MP; ++k) {
      const double dk = Fm[k * MP + k];
      const double rk = 1.0 / dk;
      if (k < m) bad |= !(dk > 0.0) || !isfinite(dk);
      if (lane == k) fdinv = rk;
      if (lane > k && lane < MP) {
        const double f = Fm[k * MP + lane] * rk;
        for (int i = k + 1; i < MP; ++i) Fm[i * MP + lane] = fma(-Fm[i * MP + k], f, Fm[i * MP + lane]);
      }
      __syncwarp();
    }
    if (bad) st_flags |= kFlagBreakdown64;
  }

  // Y[i][lane] and the lane's column of the F factor, from shared memory.
  QPB_DEV double ycol(int i) const { return lane < NP ? a.Y()[i * NP + lane] : 0.0; }
  QPB_DEV double fcol(int k) const { return lane < MP ? a.F()[k * MP + lane] : 0.0; }

  // --------------------------------------------------------- reduced solve
  // [H A'; A 0][dx; dy] = [r; v]  (r lane j < n, v lane i < m)
  QPB_DEV void reduced(double r, double v, double& odx, double& ody) {
    // u = L^-1 r
    double u = (lane < n) ? r : 0.0;
#pragma unroll
    for (int k = 0; k < NP - 1; ++k) {
      const double uk = __shfl_sync(kFull, u, k) * a.dvi()[k];
      if (lane > k) u = fma(-hc[k], uk, u);
    }
    const double ud = (lane < NP) ? u * dinv : 0.0;
    double g = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const double gi = wsum(ycol(i) * ud);
      if (lane == i) g = gi - v;
    }
    if (lane >= m) g = 0.0;
    // dy = F^-1 g with F = Lf diag(df) Lf' (same register layout as H):
    // forward: lane i > k holds Lf[i][k] * df_k in fc[k]
#pragma unroll
    for (int k = 0; k < MP - 1; ++k) {
      const double gk = __shfl_sync(kFull, g, k) * __shfl_sync(kFull, fdinv, k);
      if (lane > k && lane < MP) g = fma(-fcol(k), gk, g);
    }
    g = (lane < MP) ? g * fdinv : 0.0;
    // backward: lane i < k holds Lf[k][i] * df_i in fc[k]
#pragma unroll
    for (int k = MP - 1; k > 0; --k) {
      const double gk = __shfl_sync(kFull, g, k);
      if (lane < k) g = fma(-fcol(k) * fdinv, gk, g);
    }
    ody = (lane < m) ? g : 0.0;
    // w = u - Y dy ; dx = L^-T D^-1 w
    double wv = u;
#pragma unroll
    for (int i = 0; i < MP; ++i) wv = fma(-ycol(i), __shfl_sync(kFull, g, i), wv);
    double xv = (lane < NP) ? wv * dinv : 0.0;
#pragma unroll
    for (int k = NP - 1; k >= 0; --k) {
      const double xk = __shfl_sync(kFull, xv, k);
      // L[k][i] (k > i) = hc[k] * dinv_i in lane i
      if (lane < k) xv = fma(-hc[k] * dinv, xk, xv);
    }
    odx = (lane < n) ? xv : 0.0;
  }

  // ------------------------------------------------------------ KKT solve
  // qpax/pdip.py:49-63 with c1, c4 in registers, c2, c3 in shared memory;
  // writes ds, dz (shared) and returns dx, dy in registers.
  QPB_DEV void solve(double c1, const double* c2, const double* c3, double c4, double& odx, double* ods,
                     double* odz, double& ody) {
    for (int r = lane; r < p; r += 32) a.tp()[r] = a.w()[r] * (c3[r] - c2[r] / a.z()[r]);
    __syncwarp();
    double acc0 = 0.0, acc1 = 0.0;
    const double* Gc = a.G() + (lane < NP ? lane : 0);
    int r = 0;
    for (; r + 2 <= p; r += 2) {
      acc0 = fma(Gc[r * NP], a.tp()[r], acc0);
      acc1 = fma(Gc[(r + 1) * NP], a.tp()[r + 1], acc1);
    }
    if (r < p) acc0 = fma(Gc[r * NP], a.tp()[r], acc0);
    const double p1 = (lane < n) ? c1 + (acc0 + acc1) : 0.0;
    reduced(p1, c4, odx, ody);
    if (lane < NP) a.xs()[lane] = odx;
    __syncwarp();
    for (int rr = lane; rr < p; rr += 32) {
      const double* row = a.G() + rr * NP;
      double g0 = 0.0, g1 = 0.0;
#pragma unroll
      for (int t = 0; t < NP; t += 2) {
        const int c0 = (t + rr) & (NP - 1), c1_ = (t + 1 + rr) & (NP - 1);
        g0 = fma(row[c0], a.xs()[c0], g0);
        g1 = fma(row[c1_], a.xs()[c1_], g1);
      }
      const double dsr = c3[rr] - (g0 + g1);
      ods[rr] = dsr;
      odz[rr] = (c2[rr] - a.z()[rr] * dsr) / a.s()[rr];
    }
    __syncwarp();
  }

  // v1, v2, v3, v4 = -(relaxed residuals), w = z/s; returns the inf-norm.
  QPB_DEV double residuals(double kappa) {
    // r1 = ((sym(Q) x + q) + A' y) + G' z
    double qx = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) qx = fma(qsym(i), __shfl_sync(kFull, x, i), qx);
    double ay = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) ay = fma((lane < NP ? a.A()[i * NP + lane] : 0.0), __shfl_sync(kFull, y, i), ay);
    double gz0 = 0.0, gz1 = 0.0;
    const double* Gc = a.G() + (lane < NP ? lane : 0);
    int r = 0;
    for (; r + 2 <= p; r += 2) {
      gz0 = fma(Gc[r * NP], a.z()[r], gz0);
      gz1 = fma(Gc[(r + 1) * NP], a.z()[r + 1], gz1);
    }
    if (r < p) gz0 = fma(Gc[r * NP], a.z()[r], gz0);
    const double r1 = ((qx + q) + ay) + (gz0 + gz1);
    double loc = (lane < n) ? fabs(r1) : 0.0;
    v1 = (lane < n) ? -r1 : 0.0;
    // r4 = A x - b
    if (lane < NP) a.xs()[lane] = x;
    __syncwarp();
    double r4 = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const double ax = wsum((lane < NP ? a.A()[i * NP + lane] : 0.0) * x);
      if (lane == i) r4 = ax - b;
    }
    v4 = (lane < m) ? -r4 : 0.0;
    if (lane < m) loc = nmax(loc, fabs(r4));
    // r3 = (G x + s) - h ; r2 = s z - kappa ; w = z / s
    for (int rr = lane; rr < p; rr += 32) {
      const double* row = a.G() + rr * NP;
      double g0 = 0.0, g1 = 0.0;
#pragma unroll
      for (int t = 0; t < NP; t += 2) {
        const int c0 = (t + rr) & (NP - 1), c1 = (t + 1 + rr) & (NP - 1);
        g0 = fma(row[c0], a.xs()[c0], g0);
        g1 = fma(row[c1], a.xs()[c1], g1);
      }
      const double sr = a.s()[rr], zr = a.z()[rr];
      const double r3 = ((g0 + g1) + sr) - a.h()[rr];
      const double r2 = sr * zr - kappa;
      a.v3()[rr] = -r3;
      a.v2()[rr] = -r2;
      a.w()[rr] = zr / sr;
      loc = nmax(loc, nmax(fabs(r3), fabs(r2)));
    }
    __syncwarp();
    return wmax(loc);
  }

  QPB_DEV double ls_local(const double* v, const double* d) const {
    double mn = INFINITY;
    for (int r = lane; r < p; r += 32) {
      const double dr = d[r];
      if (dr < 0) mn = nmin(mn, -v[r] / dr);
    }
    return mn;
  }

  QPB_DEV void step_update(double alpha, double ddx, double ddy) {
    x += alpha * ddx;
    y += alpha * ddy;
    for (int r = lane; r < p; r += 32) {
      a.s()[r] += alpha * a.ds()[r];
      a.z()[r] += alpha * a.dz()[r];
    }
    __syncwarp();
  }

  // qpax/pdip.py:87-119
  QPB_DEV int pc_step() {
    const double nrm = residuals(0.0);
    const int converged = (nrm < P->tol) ? 1 : 0;
    factor();
    double ddx, ddy;
    solve(v1, a.v2(), a.v3(), v4, ddx, a.ds(), a.dz(), ddy);  // affine: ds_a, dz_a
    double sz = 0.0;
    for (int r = lane; r < p; r += 32) sz = fma(a.s()[r], a.z()[r], sz);
    sz = wsum(sz);
    const double mu = sz / p;
    const double alpha_a = nmin(1.0, wmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz()))));
    double num = 0.0;
    for (int r = lane; r < p; r += 32) num = fma(a.s()[r] + alpha_a * a.ds()[r], a.z()[r] + alpha_a * a.dz()[r], num);
    num = wsum(num);
    const double ratio = num / sz;
    const double sigma = ratio * ratio * ratio;
    for (int r = lane; r < p; r += 32) a.v2()[r] = -(-a.v2()[r] - (sigma * mu - a.ds()[r] * a.dz()[r]));
    __syncwarp();
    solve(v1, a.v2(), a.v3(), v4, ddx, a.ds(), a.dz(), ddy);
    const double alpha = 0.99 * nmin(1.0, wmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz()))));
    step_update(alpha, ddx, ddy);
    return converged;
  }

  // qpax/pdip_relaxed.py:7-52
  QPB_DEV int newton_step() {
    const double nrm = residuals(P->kappa);
    const int converged = (nrm < P->tol) ? 1 : 0;
    factor();
    double ddx, ddy;
    solve(v1, a.v2(), a.v3(), v4, ddx, a.ds(), a.dz(), ddy);
    const double ls = wmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz())));
    const double alpha = 0.99 * nmin(1.0, 0.99 * nmin(1.0, ls));
    step_update(alpha, ddx, ddy);
    return converged;
  }

  // qpax/pdip.py:15-35 (and the p == 0 exits :208-217)
  QPB_DEV void initialize() {
    for (int r = lane; r < p; r += 32) a.w()[r] = 1.0;
    __syncwarp();
    factor();
    // r1 = -q + G' h
    double acc = 0.0;
    const double* Gc = a.G() + (lane < NP ? lane : 0);
    for (int r = 0; r < p; ++r) acc = fma(Gc[r * NP], a.h()[r], acc);
    const double r1 = (lane < n) ? -q + acc : 0.0;
    double yy;
    reduced(r1, b, x, yy);
    y = yy;
    if (p == 0) return;
    if (lane < NP) a.xs()[lane] = x;
    __syncwarp();
    double zmax = -INFINITY, zmin = INFINITY;
    for (int rr = lane; rr < p; rr += 32) {
      const double* row = a.G() + rr * NP;
      double g = 0.0;
#pragma unroll
      for (int t = 0; t < NP; ++t) {
        const int c = (t + rr) & (NP - 1);
        g = fma(row[c], a.xs()[c], g);
      }
      const double zr = g - a.h()[rr];
      a.z()[rr] = zr;
      zmax = nmax(zmax, zr);
      zmin = nmin(zmin, zr);
    }
    const double alpha_p = wmax(zmax);
    const double alpha_d = -wmin(zmin);
    for (int rr = lane; rr < p; rr += 32) {
      const double zr = a.z()[rr];
      a.s()[rr] = (alpha_p < 0) ? -zr : -zr + (1.0 + alpha_p);
      if (alpha_d >= 0) a.z()[rr] = zr + (1.0 + alpha_d);
    }
    __syncwarp();
  }

  QPB_DEV void loop(bool relaxed, int* conv_out, int* iters_out) {
    int converged = 0, it = 0;
    while (it < kMaxIters && converged == 0) {
      converged = relaxed ? newton_step() : pc_step();
      ++it;
    }
    *conv_out = converged;
    *iters_out = it;
  }

  // qpax/diff_qp.py:20-46 + optnet_derivatives :8-17
  QPB_DEV void adjoint(long inst) {
    for (int r = lane; r < p; r += 32) {
      a.w()[r] = a.z()[r] / a.s()[r];
      a.v2()[r] = 0.0;
    }
    __syncwarp();
    factor();
    const double g1 = (lane < n) ? -P->gx[inst * n + lane] : 0.0;
    double ddx, ddy;
    solve(g1, a.v2(), a.v2(), 0.0, ddx, a.ds(), a.dz(), ddy);
    for (int r = lane; r < p; r += 32) a.dz()[r] = a.dz()[r] / a.z()[r];  // dlam = dlam_tilde / lam
    __syncwarp();
    double* dQ = P->dQ + inst * (long)n * n;
    for (int i = 0; i < n; ++i) {
      const double dxi = __shfl_sync(kFull, ddx, i), xi = __shfl_sync(kFull, x, i);
      if (lane < n) dQ[i * n + lane] = 0.5 * (dxi * x + xi * ddx);
    }
    double* dA = P->dA + inst * (long)m * n;
    for (int i = 0; i < m; ++i) {
      const double dyi = __shfl_sync(kFull, ddy, i), yi = __shfl_sync(kFull, y, i);
      if (lane < n) dA[i * n + lane] = dyi * x + yi * ddx;
    }
    double* dG = P->dG + inst * (long)p * n;
    for (int r = 0; r < p; ++r) {
      const double lam = a.z()[r], dl = a.dz()[r];
      if (lane < n) dG[r * n + lane] = lam * (dl * x + lam * ddx);
    }
    if (lane < n) P->dq[inst * n + lane] = ddx;
    if (lane < m) P->db[inst * m + lane] = -ddy;
    for (int r = lane; r < p; r += 32) P->dh[inst * p + r] = -a.z()[r] * a.dz()[r];
  }

  QPB_DEV void run(long inst) {
    st_f64 = st_flags = 0;
    const int op = P->op;
    int conv = 0, iters = 0;
    if (op == kOpSolve) {
      load(inst, true);
      initialize();
      if (p == 0) {
        conv = 1;
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
    if (lane == 0) {
      if (P->conv) P->conv[inst] = conv;
      if (P->iters) P->iters[inst] = iters;
      if (P->stats) {
        P->stats[inst * 4 + kStatFact32] = 0;
        P->stats[inst * 4 + kStatFact64] = st_f64;
        P->stats[inst * 4 + kStatSweeps] = 0;
        P->stats[inst * 4 + kStatFlags] = st_flags;
      }
    }
    __syncwarp();
  }
};

}  // namespace qpb
