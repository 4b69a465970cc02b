// qpb_groupqp.cuh -- several QP instances per warp, in lockstep, for n <= NP
// (32 / NP instances per warp; built for NP = 8: four), m <= MP = NP / 4,
// any p; FP64 throughout.
//
// Per instance the layout and arithmetic are those of the one-warp kernel
// (qpb_warpqp.cuh; qpax/pdip.py, pdip_relaxed.py, diff_qp.py): lane group g
// (lanes g*NP .. g*NP + NP - 1) owns its instance's H columns, n- and
// m-vectors in registers and has its own shared-memory arena.  With NP < 32 a
// single instance leaves most of a warp's lanes idle in every column step;
// here one instruction stream serves 32 / NP instances.
//
// Lockstep: every shuffle, FP64 MMA and __syncwarp runs in warp-uniform
// control flow.  The groups take the same stage sequence (initial point, IPM
// iterations, adjoint); a group whose instance has left qpax's loop
// (converged or at the iteration cap) keeps its iterate fixed while the
// others finish, its lanes still taking part in the collective steps.  Loops
// whose bounds differ between groups (p, n, m of a packed bin) contain no
// collective operation.
#pragma once
#include "qpb_warpqp.cuh"

namespace qpb {

template <int NP, int MP>
struct GroupQP {
  static_assert(NP == 8 || NP == 16, "NP");
  using W = WarpQP<NP, MP>;
  static constexpr int kGroups = 32 / NP;
  static constexpr unsigned kGroupMask = (1u << NP) - 1u;
  static constexpr int kYld = W::kYld;

  const Params* P;
  WarpAddr<NP, MP> a;      // this group's arena
  unsigned char* arena0;   // group 0's arena; group g's at arena0 + g * astride
  size_t astride;
  int n, m, p;             // this group's instance shape (0 for an empty group)
  int lane, sl, grp, gb;   // lane, lane within the group (= owned column), group, group's first lane
  const double* gQ;
  bool q_symmetric;
  double hc[NP];
  double dinv, fdinv;
  double x, q, y, b;
  int st_f64, st_flags;

  // ---------------------------------------------------- group collectives
  QPB_DEV double gsum(double v) const {
#pragma unroll
    for (int o = NP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
  }
  QPB_DEV double gmax(double v) const {
#pragma unroll
    for (int o = NP / 2; o > 0; o >>= 1) v = nmax(v, __shfl_xor_sync(kFull, v, o));
    return v;
  }
  QPB_DEV double gmin(double v) const {
#pragma unroll
    for (int o = NP / 2; o > 0; o >>= 1) v = nmin(v, __shfl_xor_sync(kFull, v, o));
    return v;
  }
  // value of column k's lane in this group
  QPB_DEV double bc(double v, int k) const { return __shfl_sync(kFull, v, gb + k); }
  QPB_DEV bool gany(bool pred) const { return ((__ballot_sync(kFull, pred) >> gb) & kGroupMask) != 0u; }

  QPB_DEV void setup(const Params& prm, unsigned char* arena_group0, size_t stride, int ln) {
    P = &prm;
    lane = ln;
    grp = ln / NP;
    sl = ln - grp * NP;
    gb = grp * NP;
    arena0 = arena_group0;
    astride = stride;
    a.base = reinterpret_cast<double*>(arena0 + (size_t)grp * stride);
    a.p = 0;
  }

  QPB_DEV void load_q(double (&qv)[NP]) const {
    const bool in = sl < n;
#pragma unroll
    for (int i = 0; i < NP; ++i) qv[i] = (in && i < n) ? __ldg(gQ + i * n + sl) : 0.0;
    if (!q_symmetric) {
#pragma unroll
      for (int i = 0; i < NP; ++i)
        if (in && i < n) qv[i] = 0.5 * (qv[i] + __ldg(gQ + sl * n + i));
    }
  }

  // Operands (and the starting iterate) into the group's arena, as in the
  // one-warp kernel; pmax = the largest p of the warp's groups.
  QPB_DEV void load(const InstRef& R, bool remove_inf, bool iterate, int pmax) {
    gQ = P->Q + R.oQ;
    const double* gG = P->G + R.oG;
    const double* gA = P->A + R.oA;
    const double* gh = P->h + R.oh;
    if (P->arena_in_smem) {
      for (int r = 0; r < p; ++r) {
        if (sl < n)
          W::cp_async8(a.G() + r * NP + (sl ^ W::gswz(r)), gG + r * n + sl);
        else
          a.G()[r * NP + (sl ^ W::gswz(r))] = 0.0;
      }
#pragma unroll
      for (int i = 0; i < MP; ++i) {
        if (i < m && sl < n)
          W::cp_async8(a.A() + i * NP + sl, gA + i * n + sl);
        else
          a.A()[i * NP + sl] = 0.0;
      }
      for (int r = sl; r < p; r += NP) W::cp_async8(a.h() + r, gh + r);
      if (iterate) {
        for (int r = sl; r < p; r += NP) {
          W::cp_async8(a.s() + r, P->in[1] + R.oh + r);
          W::cp_async8(a.z() + r, P->in[2] + R.oh + r);
        }
      }
      W::cp_async_wait_all();
      // each lane copied G's column sl and h's rows sl, sl + NP, ...: the
      // fix-up touches only this lane's own copies
      if (remove_inf) {
        for (int r0 = 0; r0 < pmax; r0 += NP) {
          const int r = r0 + sl;
          const bool inf = r < p && isinf(a.h()[r]);
          unsigned mask = (__ballot_sync(kFull, inf) >> gb) & kGroupMask;
          while (mask) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1;
            a.G()[(r0 + bit) * NP + (sl ^ W::gswz(r0 + bit))] = 0.0;
          }
          if (inf) a.h()[r] = 0.0;
        }
      }
    } else {
      for (int r0 = 0; r0 < p; r0 += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int r = r0 + u;
          v[u] = (r < p && sl < n) ? __ldg(gG + r * n + sl) : 0.0;
          if (remove_inf && r < p && isinf(__ldg(gh + r))) v[u] = 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (r0 + u < p) a.G()[(r0 + u) * NP + (sl ^ W::gswz(r0 + u))] = v[u];
      }
#pragma unroll
      for (int i = 0; i < MP; ++i) a.A()[i * NP + sl] = (i < m && sl < n) ? gA[i * n + sl] : 0.0;
      for (int r = sl; r < p; r += NP) {
        const double hv = gh[r];
        a.h()[r] = (remove_inf && isinf(hv)) ? 0.0 : hv;
      }
      if (iterate) {
        for (int r = sl; r < p; r += NP) {
          a.s()[r] = P->in[1][R.oh + r];
          a.z()[r] = P->in[2][R.oh + r];
        }
      }
    }
    q = (sl < n) ? P->q[R.oq + sl] : 0.0;
    b = (sl < m) ? P->b[R.ob + sl] : 0.0;
    if (iterate) {
      x = (sl < n) ? P->in[0][R.oq + sl] : 0.0;
      y = (sl < m) ? P->in[3][R.ob + sl] : 0.0;
    }
    int asym = 0;
#pragma unroll
    for (int i = 0; i < NP; ++i)
      if (sl < n && i < n) asym |= (__ldg(gQ + i * n + sl) != __ldg(gQ + sl * n + i));
    q_symmetric = !gany(asym != 0);
    __syncwarp();
  }

  QPB_DEV void store_iterate(const InstRef& R, bool inf_rows) {
    if (sl < n) P->out[0][R.oq + sl] = x;
    if (sl < m) P->out[3][R.ob + sl] = y;
    for (int r = sl; r < p; r += NP) {
      double sv = a.s()[r], zv = a.z()[r];
      if (inf_rows && isinf(P->h[R.oh + r])) {  // qpax/pdip.py:243-246
        zv = 0.0;
        sv = INFINITY;
      }
      P->out[1][R.oh + r] = sv;
      P->out[2][R.oh + r] = zv;
    }
  }

  // ------------------------------------------- G' diag(w) G on FP64 MMA
  // Tile row TI of group g's instance: every lane supplies fragments of that
  // instance (the MMA is warp-wide), the finished tile row goes through the
  // instance's scratch into its group's lane-owned columns.  As in the
  // one-warp kernel, every element comes from the lower triangle.
  template <int TI>
  QPB_DEV void h_tile_row(int g) {
    const int fg = lane >> 2, t = lane & 3;
    const int pg = __shfl_sync(kFull, p, g * NP);
    WarpAddr<NP, MP> ag;
    ag.base = reinterpret_cast<double*>(arena0 + (size_t)g * astride);
    ag.p = pg;
    const double* Gs = ag.G();
    const double* wv = ag.w();
    double* S = ag.Y();
    const int kblocks = (pg + 3) >> 2;
    double acc[TI + 1][2];
#pragma unroll
    for (int tj = 0; tj <= TI; ++tj) acc[tj][0] = acc[tj][1] = 0.0;
    const int sw = W::gswz(t);
    for (int kb = 0; kb < kblocks; ++kb) {
      const int k = 4 * kb + t;
      const bool in = k < pg;
      const double* row = Gs + (in ? k : 0) * NP;
      const double a0 = in ? wv[k] * row[(8 * TI + fg) ^ sw] : 0.0;
#pragma unroll
      for (int tj = 0; tj <= TI; ++tj) {
        const double b0 = in ? row[(8 * tj + fg) ^ sw] : 0.0;
        W::dmma884(acc[tj][0], acc[tj][1], a0, b0);
      }
    }
    const int gs = W::sswz(fg);
#pragma unroll
    for (int tj = 0; tj <= TI; ++tj) {
      S[fg * NP + ((8 * tj + 2 * t) ^ gs)] = acc[tj][0];
      S[fg * NP + ((8 * tj + 2 * t + 1) ^ gs)] = acc[tj][1];
    }
    __syncwarp();
    if (grp == g) {
      const int tl = sl >> 3;
      if (tl < TI) {
#pragma unroll
        for (int r = 0; r < 8; ++r) hc[8 * TI + r] += S[r * NP + (sl ^ W::sswz(r))];
      }
      if (tl == TI) {
        const int c = sl - 8 * TI;
        const int cs = W::sswz(c);
#pragma unroll
        for (int r = 0; r < 8; ++r)
          hc[8 * TI + r] += (r >= c) ? S[r * NP + (sl ^ W::sswz(r))] : S[c * NP + ((8 * TI + r) ^ cs)];
#pragma unroll
        for (int i = 0; i < 8 * TI; ++i) hc[i] += S[c * NP + (i ^ cs)];
      }
    }
    __syncwarp();
  }

  QPB_DEV void form_h_tensor() {
#pragma unroll
    for (int g = 0; g < kGroups; ++g) {
      h_tile_row<0>(g);
      if constexpr (NP > 8) h_tile_row<1>(g);
    }
  }

  // ---------------------------------------------------------------- factor
  // As WarpQP::factor, per group.  `count` = this group's instance is live
  // (statistics count only its own factorisations).
  QPB_DEV void factor(bool count) {
    if (count) st_f64++;
    dinv = 0.0;
    fdinv = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) hc[i] = 0.0;
    form_h_tensor();
    {
      double qv[NP];
      load_q(qv);
#pragma unroll
      for (int i = 0; i < NP; ++i) hc[i] = (sl >= n && i == sl) ? 1.0 : qv[i] + hc[i];
    }
    int bad = 0;
    double* cb = a.cb();
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      cb[sl] = hc[k];
      __syncwarp();
      const double dk = cb[k];
      const double rk = 1.0 / dk;
      if (k < n) bad |= !(dk > 0.0) || !isfinite(dk);
      if (sl == k) dinv = rk;
      const double hk = hc[k];
      if (sl > k) {
#pragma unroll
        for (int i = k + 1; i < NP; ++i) hc[i] = fma(-(cb[i] * hk), rk, hc[i]);
      }
      __syncwarp();
    }
    a.dvi()[sl] = dinv;
    __syncwarp();
    double yc[MP];
#pragma unroll
    for (int i = 0; i < MP; ++i) yc[i] = a.A()[i * NP + sl];
#pragma unroll
    for (int k = 0; k < NP - 1; ++k) {
      const double l = (sl > k) ? hc[k] * a.dvi()[k] : 0.0;
#pragma unroll
      for (int i = 0; i < MP; ++i) yc[i] = fma(-l, bc(yc[i], k), yc[i]);
    }
#pragma unroll
    for (int i = 0; i < MP; ++i) a.Y()[i * kYld + sl] = yc[i];
    __syncwarp();
    double* Fm = a.F();
    const double* Ys = a.Y();
    const double* dv = a.dvi();
    for (int e = sl; e < MP * MP; e += NP) {
      const int r = e / MP, c = e - r * MP;
      double v = (r == c) ? 1.0 : 0.0;
      if (r < m && c < m) {
        double acc = 0.0;
#pragma unroll 8
        for (int j = 0; j < NP; ++j) acc = fma(Ys[r * kYld + j] * dv[j], Ys[c * kYld + j], acc);
        v = acc;
      }
      Fm[e] = v;
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < MP; ++k) {
      const double dk = Fm[k * MP + k];
      const double rk = 1.0 / dk;
      if (k < m) bad |= !(dk > 0.0) || !isfinite(dk);
      if (sl == k) fdinv = rk;
      if (sl > k && sl < MP) {
        const double f = Fm[k * MP + sl] * rk;
        for (int i = k + 1; i < MP; ++i) Fm[i * MP + sl] = fma(-Fm[i * MP + k], f, Fm[i * MP + sl]);
      }
      __syncwarp();
    }
    if (bad && count) st_flags |= kFlagBreakdown64;
  }

  QPB_DEV double ycol(int i) const { return a.Y()[i * kYld + sl]; }
  QPB_DEV double fcol(int k) const { return sl < MP ? a.F()[k * MP + sl] : 0.0; }
  QPB_DEV double acol(int i) const { return a.A()[i * NP + sl]; }

  // --------------------------------------------------------- reduced solve
  QPB_DEV void reduced(double r, double v, double& odx, double& ody) {
    double u = (sl < n) ? r : 0.0;
#pragma unroll
    for (int k = 0; k < NP - 1; ++k) {
      const double uk = bc(u, k) * a.dvi()[k];
      if (sl > k) u = fma(-hc[k], uk, u);
    }
    const double ud = u * dinv;
    double g = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const double gi = gsum(ycol(i) * ud);
      if (sl == i) g = gi - v;
    }
    if (sl >= m) g = 0.0;
#pragma unroll
    for (int k = 0; k < MP - 1; ++k) {
      const double gk = bc(g, k) * bc(fdinv, k);
      if (sl > k && sl < MP) g = fma(-fcol(k), gk, g);
    }
    g = (sl < MP) ? g * fdinv : 0.0;
#pragma unroll
    for (int k = MP - 1; k > 0; --k) {
      const double gk = bc(g, k);
      if (sl < k) g = fma(-fcol(k) * fdinv, gk, g);
    }
    ody = (sl < m) ? g : 0.0;
    double wv = u;
#pragma unroll
    for (int i = 0; i < MP; ++i) wv = fma(-ycol(i), bc(g, i), wv);
    double xv = wv * dinv;
#pragma unroll
    for (int k = NP - 1; k > 0; --k) {
      const double xk = bc(xv, k);
      if (sl < k) xv = fma(-hc[k] * dinv, xk, xv);
    }
    odx = (sl < n) ? xv : 0.0;
  }

  QPB_DEV double grow_dot(int r, const double* xsv) const {
    const double* row = a.G() + r * NP;
    const int sw = W::gswz(r);
    double g0 = 0.0, g1 = 0.0;
#pragma unroll
    for (int t = 0; t < NP; t += 2) {
      const int c0 = (t + r) & (NP - 1), c1 = (t + 1 + r) & (NP - 1);
      g0 = fma(row[c0 ^ sw], xsv[c0], g0);
      g1 = fma(row[c1 ^ sw], xsv[c1], g1);
    }
    return g0 + g1;
  }

  QPB_DEV double gcol_dot(const double* vv) const {
    const double* G = a.G();
    const int c0 = sl ^ W::gswz(0), c1 = sl ^ W::gswz(1), c2 = sl ^ W::gswz(2), c3 = sl ^ W::gswz(3);
    double acc0 = 0.0, acc1 = 0.0;
    int r = 0;
    for (; r + 4 <= p; r += 4) {
      acc0 = fma(G[r * NP + c0], vv[r], acc0);
      acc1 = fma(G[(r + 1) * NP + c1], vv[r + 1], acc1);
      acc0 = fma(G[(r + 2) * NP + c2], vv[r + 2], acc0);
      acc1 = fma(G[(r + 3) * NP + c3], vv[r + 3], acc1);
    }
    for (; r < p; ++r) {
      const double gv = G[r * NP + (sl ^ W::gswz(r))];
      if (r & 1)
        acc1 = fma(gv, vv[r], acc1);
      else
        acc0 = fma(gv, vv[r], acc0);
    }
    return acc0 + acc1;
  }

  // qpax/pdip.py:49-63 (slack == false: the reduced system directly).
  QPB_DEV void solve(bool slack, double c1, const double* c2, const double* c3, double c4, double& odx,
                     double& ody) {
    double p1 = c1;
    if (slack) {
      double* tp = a.tp();
      for (int r = sl; r < p; r += NP) tp[r] = a.w()[r] * (c3[r] - c2[r] / a.z()[r]);
      __syncwarp();
      p1 = (sl < n) ? c1 + gcol_dot(tp) : 0.0;
    }
    reduced(p1, c4, odx, ody);
    if (slack) {
      a.xs()[sl] = odx;
      __syncwarp();
      double* ds = a.ds();
      double* dz = a.dz();
      for (int r = sl; r < p; r += NP) {
        const double dsr = c3[r] - grow_dot(r, a.xs());
        ds[r] = dsr;
        dz[r] = (c2[r] - a.z()[r] * dsr) / a.s()[r];
      }
      __syncwarp();
    }
  }

  // qpax/pdip.py:93-100, pdip_relaxed.py:16-23 (as WarpQP::residuals).
  QPB_DEV double residuals(double kappa, double& v1, double& v4) {
    double qx = 0.0;
    {
      double qv[NP];
      load_q(qv);
#pragma unroll
      for (int i = 0; i < NP; ++i) qx = fma(qv[i], bc(x, i), qx);
    }
    double ay = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) ay = fma(acol(i), bc(y, i), ay);
    const double r1 = ((qx + q) + ay) + gcol_dot(a.z());
    double loc = (sl < n) ? fabs(r1) : 0.0;
    v1 = (sl < n) ? -r1 : 0.0;
    a.xs()[sl] = x;
    __syncwarp();
    double r4 = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const double ax = gsum(acol(i) * x);
      if (sl == i) r4 = ax - b;
    }
    v4 = (sl < m) ? -r4 : 0.0;
    if (sl < m) loc = nmax(loc, fabs(r4));
    for (int r = sl; r < p; r += NP) {
      const double sr = a.s()[r], zr = a.z()[r];
      const double r3 = (grow_dot(r, a.xs()) + sr) - a.h()[r];
      const double r2 = sr * zr - kappa;
      a.v3()[r] = -r3;
      a.v2()[r] = -r2;
      a.w()[r] = zr / sr;
      loc = nmax(loc, nmax(fabs(r3), fabs(r2)));
    }
    __syncwarp();
    return gmax(loc);
  }

  QPB_DEV double ls_local(const double* v, const double* d) const {
    double mn = INFINITY;
    for (int r = sl; r < p; r += NP) {
      const double dr = d[r];
      if (dr < 0) mn = nmin(mn, -v[r] / dr);
    }
    return mn;
  }

  // qpax/diff_qp.py:20-46 optnet_derivatives :8-17; `live` = write them.
  QPB_DEV void write_grads(const InstRef& R, double ddx, double ddy, bool live) {
    for (int r = sl; r < p; r += NP) a.dz()[r] = a.dz()[r] / a.z()[r];
    __syncwarp();
    double* dQ = P->dQ + R.oQ;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double dxi = bc(ddx, i), xi = bc(x, i);
      if (live && i < n && sl < n) dQ[i * n + sl] = 0.5 * (dxi * x + xi * ddx);
    }
    double* dA = P->dA + R.oA;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const double dyi = bc(ddy, i), yi = bc(y, i);
      if (live && i < m && sl < n) dA[i * n + sl] = dyi * x + yi * ddx;
    }
    if (!live) return;
    double* dG = P->dG + R.oG;
    for (int r = 0; r < p; ++r) {
      const double lam = a.z()[r], dl = a.dz()[r];
      if (sl < n) dG[r * n + sl] = lam * (dl * x + lam * ddx);
    }
    if (sl < n) P->dq[R.oq + sl] = ddx;
    if (sl < m) P->db[R.ob + sl] = -ddy;
    for (int r = sl; r < p; r += NP) P->dh[R.oh + r] = -a.z()[r] * a.dz()[r];
  }

  // --------------------------------------------------------------- driver
  enum Stage : int { kInit, kStep, kCorrector, kAdjoint, kDone };

  // Instance `inst` for this group (live = inst < batch; an empty group
  // takes shape 0 x 0 x 0 and only joins the collective steps).  A
  // warp-uniform state machine with one factor() and one solve() call site,
  // as in the one-warp kernel; `active` marks the groups still inside qpax's
  // loop.
  QPB_DEV void run(long inst, bool live) {
    st_f64 = st_flags = 0;
    const InstRef R = inst_ref(*P, live ? inst : 0);
    n = live ? R.n : 0;
    m = live ? R.m : 0;
    p = live ? R.p : 0;
    a.p = p;
    const int pmax = (int)__reduce_max_sync(kFull, (unsigned)p);
    const int op = P->op;
    const bool relaxed = (op == kOpRelax || op == kOpBwd);
    const bool fresh = (op == kOpSolve || op == kOpInit);
    load(R, op == kOpSolve, !fresh, pmax);
    int stage = fresh ? kInit : (op == kOpAdjoint ? kAdjoint : kStep);
    int it = 0, converged = 0, conv_now = 0;
    bool active = live;
    double v1 = 0.0, v4 = 0.0, dxr = 0.0, dyr = 0.0;
    // bounded: initial point + 2 solves per iteration + the final test + adjoint
    for (int guard = 0; guard < 2 * kMaxIters + 4 && stage != kDone; ++guard) {
      bool slack = true, refactor = true;
      double c1 = 0.0, c4 = 0.0;
      const double *c2 = a.v2(), *c3 = a.v3();
      if (stage == kInit) {
        for (int r = sl; r < p; r += NP) a.w()[r] = 1.0;
        __syncwarp();
        slack = false;
        c1 = (sl < n) ? -q + gcol_dot(a.h()) : 0.0;  // r1 = -q + G' h (qpax/pdip.py:15-35)
        c4 = b;
      } else if (stage == kStep) {
        if (it >= kMaxIters || converged) active = false;  // the while-loop condition of qpax
        if (!__any_sync(kFull, active)) {
          if (op == kOpBwd) {
            if (live && P->out[0]) store_iterate(R, false);
            stage = kAdjoint;
            continue;
          }
          stage = kDone;
          continue;
        }
        const double nrm = residuals(relaxed ? P->kappa : 0.0, v1, v4);
        conv_now = (nrm < P->tol) ? 1 : 0;
        c1 = v1;
        c4 = v4;
      } else if (stage == kCorrector) {
        refactor = false;
        c1 = v1;
        c4 = v4;
      } else {  // kAdjoint: qpax/diff_qp.py:20-46 at (s, z), rhs (-dl/dx, 0, 0, 0)
        for (int r = sl; r < p; r += NP) {
          a.w()[r] = a.z()[r] / a.s()[r];
          a.v2()[r] = 0.0;
        }
        __syncwarp();
        c1 = (sl < n) ? -P->gx[R.oq + sl] : 0.0;
        c3 = a.v2();
      }
      if (refactor) factor(stage == kStep ? active : live);
      solve(slack, c1, c2, c3, c4, dxr, dyr);
      if (stage == kInit) {
        x = dxr;
        y = dyr;
        // z = G x - h, then the positivity shifts (qpax/pdip.py:25-33; no-ops when p == 0)
        a.xs()[sl] = x;
        __syncwarp();
        double zmax = -INFINITY, zmin = INFINITY;
        for (int r = sl; r < p; r += NP) {
          const double zr = grow_dot(r, a.xs()) - a.h()[r];
          a.z()[r] = zr;
          zmax = nmax(zmax, zr);
          zmin = nmin(zmin, zr);
        }
        const double alpha_p = gmax(zmax);
        const double alpha_d = -gmin(zmin);
        for (int r = sl; r < p; r += NP) {
          const double zr = a.z()[r];
          a.s()[r] = (alpha_p < 0) ? -zr : -zr + (1.0 + alpha_p);
          if (alpha_d >= 0) a.z()[r] = zr + (1.0 + alpha_d);
        }
        __syncwarp();
        if (op == kOpSolve && p == 0) converged = 1;  // qpax/pdip.py:208-217
        if (op == kOpInit || p == 0) active = false;
        stage = (op == kOpSolve) ? kStep : kDone;
      } else if (stage == kStep && !relaxed) {
        // predictor done: centering_params, qpax/pdip.py:76-84
        double sz = 0.0;
        for (int r = sl; r < p; r += NP) sz = fma(a.s()[r], a.z()[r], sz);
        sz = gsum(sz);
        const double mu = sz / p;
        const double alpha_a = nmin(1.0, gmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz()))));
        double num = 0.0;
        for (int r = sl; r < p; r += NP)
          num = fma(a.s()[r] + alpha_a * a.ds()[r], a.z()[r] + alpha_a * a.dz()[r], num);
        num = gsum(num);
        const double ratio = num / sz;
        const double sigma_mu = ratio * ratio * ratio * mu;
        for (int r = sl; r < p; r += NP) a.v2()[r] = -(-a.v2()[r] - (sigma_mu - a.ds()[r] * a.dz()[r]));
        __syncwarp();
        stage = kCorrector;
      } else if (stage == kStep || stage == kCorrector) {
        // step length and update (qpax/pdip.py:112-117, pdip_relaxed.py:30-35)
        const double ls = gmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz())));
        const double alpha = relaxed ? 0.99 * nmin(1.0, 0.99 * nmin(1.0, ls)) : 0.99 * nmin(1.0, ls);
        if (active) {
          x += alpha * dxr;
          y += alpha * dyr;
          for (int r = sl; r < p; r += NP) {
            a.s()[r] += alpha * a.ds()[r];
            a.z()[r] += alpha * a.dz()[r];
          }
          ++it;
          converged = conv_now;
        }
        __syncwarp();
        stage = kStep;
      } else {  // kAdjoint
        write_grads(R, dxr, dyr, live);
        stage = kDone;
      }
    }
    if (live && (op == kOpSolve || op == kOpInit || op == kOpRelax)) store_iterate(R, op == kOpSolve);
    if (live && sl == 0) {
      const long id = R.id;
      if (P->conv) P->conv[id] = (op == kOpInit || op == kOpAdjoint) ? 0 : converged;
      if (P->iters) P->iters[id] = it;
      if (P->stats) {
        P->stats[id * 4 + kStatFact32] = 0;
        P->stats[id * 4 + kStatFact64] = st_f64;
        P->stats[id * 4 + kStatSweeps] = 0;
        P->stats[id * 4 + kStatFlags] = st_flags;
      }
    }
    __syncwarp();
  }
};

}  // namespace qpb
