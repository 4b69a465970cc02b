// qpb_warpqp.cuh -- one warp per QP instance for n <= NP (NP = 8, 16, 32),
// m <= MP = NP / 4, any p; FP64 (WarpQP<NP, MP>), or mixed precision
// (WarpQP<NP, MP, true>: FP32 inverses with FP64 refinement, handing an
// instance over to the FP64 kernel once its FP32 factor is rejected).
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
//   * Y = L^-1 A' is formed inside the same elimination loop (lane j holds
//     row j of Y) and kept in shared memory with the m x m Schur complement
//     F = Y' D^-1 Y (one FP64 tensor-core tile) and its register-factored LDL^T;
//   * n- and m-vectors are lane-distributed registers; p-vectors and the G,
//     A operands live in shared memory; Q is read through L1/L2.
// Every solve of the instance -- initial point, predictor, corrector, Newton
// step of the relaxation, adjoint -- runs through one factor() and one
// solve() call site (run() is a bounded state machine), which keeps the
// unrolled code small enough for the instruction cache.
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
//   G (p x NP, columns swizzled: element (r, c) at r * NP + (c ^ gswz(r))) |
//   A (MP x NP) | 9 p-vectors | a pad double when p is odd | xs, cb, dvi (NP each) |
//   Y (MP x (NP + 1), Y[i][j] = (L^-1 A')[j][i]; the padded row stride keeps
//   the F = Y D^-1 Y' reads in distinct banks) | F (MP x MP, column-held factor)
// Addresses are recomputed from the base and p where used (no pointer table).
struct WarpArena {
  static __host__ __device__ size_t doubles(int NP, int MP, int p) {
    // the Y region doubles as the 8 x NP tile-row scratch of the H formation;
    // one pad double after the p-vectors when p is odd (16-byte aligned xs, cb, ...)
    return (size_t)p * NP + (size_t)MP * NP + 9 * (size_t)p + (size_t)(p & 1) + 3 * (size_t)NP +
           (size_t)(MP > 8 ? MP : 8) * (NP + 1) + (size_t)MP * MP;
  }
  static size_t bytes(int NP, int MP, int p) { return doubles(NP, MP, p) * sizeof(double) + 16; }
};

// Starting iterate of one instance: the caller's arrays, or the block a
// mixed-kernel hand-over left in the workspace.
struct IterSrc {
  const double *x, *s, *z, *y;
};

enum WarpSlot : int { kVh = 0, kVs, kVz, kVw, kVv2, kVv3, kVds, kVdz, kVtp };

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
  QPB_DEV double* xs() const { return base + p * NP + MP * NP + 9 * p + (p & 1); }
  QPB_DEV double* cb() const { return xs() + NP; }
  QPB_DEV double* dvi() const { return xs() + 2 * NP; }
  QPB_DEV double* Y() const { return xs() + 3 * NP; }
  QPB_DEV double* F() const { return Y() + (MP > 8 ? MP : 8) * (NP + 1); }
};

// kMixed: FP32 factorisation with FP64 iterative refinement (the mixed
// precision mode); the FP64 instantiation is unaffected by it.
template <int NP, int MP, bool kMixed = false>
struct WarpQP {
  static_assert(NP == 8 || NP == 16 || NP == 32, "NP");
  static constexpr int kYld = NP + 1;  // row stride of Y (doubles, or floats in the FP32 factor)
  // Column swizzle of G's row r (period 4 in r): the four rows of one DMMA
  // k-step fall in distinct shared-memory banks.
  static QPB_DEV int gswz(int r) { return NP == 8 ? (r & 2) << 1 : (4 * r) & 12; }
  // Column swizzle of row g of the H-formation scratch (fragment stores in
  // distinct banks).
  static QPB_DEV int sswz(int g) { return NP == 8 ? (g >> 1) & 1 : (g & 1) | ((g & 2) << 2); }
  const Params* P;
  WarpAddr<NP, MP> a;
  int n, m, p, lane;
  const double* gQ;  // this instance's Q (row-major n x n, global)
  double hc[NP];     // H column -> L, D (lane-owned column)
  double dinv;       // 1 / d_lane
  double fdinv;      // 1 / df_lane (lanes < MP)
  double x, q;       // n-vectors (lane j)
  double y, b;       // m-vectors (lane i)
  int st_f64, st_flags;
  // mixed precision: hc[] keeps H in FP64 (the refinement's operator) and
  // lf2[] holds column `lane` of the FP32 inverse of H; Y' = H^-1 A' and
  // F^-1 live in the FP64 factor's shared regions.
  float2 lf2[NP / 2];  // (lf[2t], lf[2t + 1]): pairs for the packed FP32x2 updates
  int st_f32, st_sweeps;
  double pivot_max;
  int max_sweeps;

  QPB_DEV void setup(const Params& prm, unsigned char* arena, int ln) {
    P = &prm;
    n = prm.n; m = prm.m; p = prm.p;
    lane = ln;
    a.base = reinterpret_cast<double*>(arena);
    a.p = p;
    if constexpr (kMixed) {
      pivot_max = prm.pivot_max;
      max_sweeps = prm.max_sweeps;
    }
  }

  // qv[i] = sym(Q)[i][lane]: (Q + Q')/2, or the coalesced Q[i][lane] alone
  // when Q is exactly symmetric (checked once per instance).  All loads are
  // issued before the first use: the column costs one L2 round trip.
  QPB_DEV void load_q(double (&qv)[NP]) const {
    const bool in = lane < n;
#pragma unroll
    for (int i = 0; i < NP; ++i) qv[i] = (in && i < n) ? __ldg(gQ + i * n + lane) : 0.0;
    if (!q_symmetric) {
#pragma unroll
      for (int i = 0; i < NP; ++i)
        if (in && i < n) qv[i] = 0.5 * (qv[i] + __ldg(gQ + lane * n + i));
    }
  }
  bool q_symmetric;

  // 8-byte asynchronous copy global -> shared (dst must be shared memory).
  static QPB_DEV void cp_async8(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
  }
  static QPB_DEV void cp_async_wait_all() { asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory"); }

  // Instance operands (and, with `iterate`, the starting iterate) into the
  // arena.  A shared-memory arena is filled with asynchronous copies, every
  // row in flight at once (one memory round trip per instance); a global
  // arena (large p) with grouped loads.  Rows with h = inf are zeroed in G and
  // h when remove_inf (qpax/pdip.py:166-178).  `it` points at the starting
  // iterate (x, s, z, y) of this instance.
  QPB_DEV void load(const InstRef& R, bool remove_inf, bool iterate, const IterSrc& it) {
    gQ = P->Q + R.oQ;
    const double* gG = P->G + R.oG;
    const double* gA = P->A + R.oA;
    const double* gh = P->h + R.oh;
    if (P->arena_in_smem) {
      for (int r = 0; r < p; ++r) {
        if (lane < n)
          cp_async8(a.G() + r * NP + (lane ^ gswz(r)), gG + r * n + lane);
        else if (lane < NP)
          a.G()[r * NP + (lane ^ gswz(r))] = 0.0;
      }
#pragma unroll
      for (int i = 0; i < MP; ++i) {
        if (i < m && lane < n)
          cp_async8(a.A() + i * NP + lane, gA + i * n + lane);
        else if (lane < NP)
          a.A()[i * NP + lane] = 0.0;
      }
      for (int r = lane; r < p; r += 32) cp_async8(a.h() + r, gh + r);
      if (iterate) {
        for (int r = lane; r < p; r += 32) {
          cp_async8(a.s() + r, it.s + r);
          cp_async8(a.z() + r, it.z + r);
        }
      }
      cp_async_wait_all();
      // each lane copied G's column `lane` and h's rows lane, lane + 32, ...:
      // the fix-up below touches only this lane's own copies
      if (remove_inf) {
        for (int r0 = 0; r0 < p; r0 += 32) {
          const int r = r0 + lane;
          const bool inf = r < p && isinf(a.h()[r]);
          unsigned mask = __ballot_sync(kFull, inf);
          while (mask) {
            const int bit = __ffs(mask) - 1;
            mask &= mask - 1;
            if (lane < NP) a.G()[(r0 + bit) * NP + (lane ^ gswz(r0 + bit))] = 0.0;
          }
          if (inf) a.h()[r] = 0.0;
        }
      }
    } else {
      // G rows in groups of 8: the group's loads are issued before its stores
      for (int r0 = 0; r0 < p; r0 += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int r = r0 + u;
          v[u] = (r < p && lane < n) ? __ldg(gG + r * n + lane) : 0.0;
          if (remove_inf && r < p && isinf(__ldg(gh + r))) v[u] = 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (r0 + u < p && lane < NP) a.G()[(r0 + u) * NP + (lane ^ gswz(r0 + u))] = v[u];
      }
#pragma unroll
      for (int i = 0; i < MP; ++i)
        if (lane < NP) a.A()[i * NP + lane] = (i < m && lane < n) ? gA[i * n + lane] : 0.0;
      for (int r = lane; r < p; r += 32) {
        const double hv = gh[r];
        a.h()[r] = (remove_inf && isinf(hv)) ? 0.0 : hv;
      }
      if (iterate) {
        for (int r = lane; r < p; r += 32) {
          a.s()[r] = it.s[r];
          a.z()[r] = it.z[r];
        }
      }
    }
    q = (lane < n) ? P->q[R.oq + lane] : 0.0;
    b = (lane < m) ? P->b[R.ob + lane] : 0.0;
    if (iterate) {
      x = (lane < n) ? it.x[lane] : 0.0;
      y = (lane < m) ? it.y[lane] : 0.0;
    }
    int asym = 0;
#pragma unroll
    for (int i = 0; i < NP; ++i)
      if (lane < n && i < n) asym |= (__ldg(gQ + i * n + lane) != __ldg(gQ + lane * n + i));
    q_symmetric = !__any_sync(kFull, asym);
    __syncwarp();
  }

  QPB_DEV void store_iterate(const InstRef& R, bool inf_rows) {
    if (lane < n) P->out[0][R.oq + lane] = x;
    if (lane < m) P->out[3][R.ob + lane] = y;
    for (int r = lane; r < p; r += 32) {
      double sv = a.s()[r], zv = a.z()[r];
      if (inf_rows && isinf(P->h[R.oh + r])) {  // qpax/pdip.py:243-246
        zv = 0.0;
        sv = INFINITY;
      }
      P->out[1][R.oh + r] = sv;
      P->out[2][R.oh + r] = zv;
    }
  }

  // -------------------------------------------------- G' diag(w) G on DMMA
  // D (8x8) += A (8x4, row) * B (4x8, col) in FP64 on the tensor cores.
  // Fragments (PTX mma.m8n8k4 .f64): a0 = A[lane/4][lane%4],
  // b0 = B[lane%4][lane/4], (d0, d1) = D[lane/4][2*(lane%4) + {0, 1}].
  static QPB_DEV void dmma884(double& d0, double& d1, double a0, double b0) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a0), "d"(b0));
  }

  // Adds tile row TI of G' diag(w) G (tiles (TI, 0..TI), accumulators
  // acc[tj][0..1] in the fragment layout) to the lane-owned columns: the
  // tiles go through the 8 x NP scratch (the Y region, rebuilt later in
  // factor()), the upper triangle coming from the symmetric element of a
  // later tile row.
  template <int TI>
  QPB_DEV void scatter_tile_row(const double (&acc)[TI + 1][2]) {
    const int g = lane >> 2, t = lane & 3;
    double* S = a.Y();
    const int gs = sswz(g);
#pragma unroll
    for (int tj = 0; tj <= TI; ++tj) {
      S[g * NP + ((8 * tj + 2 * t) ^ gs)] = acc[tj][0];
      S[g * NP + ((8 * tj + 2 * t + 1) ^ gs)] = acc[tj][1];
    }
    __syncwarp();
    // Every element is taken from the lower triangle (row >= column) so that
    // H is exactly symmetric; the factorization relies on that.
    const int tl = lane >> 3;  // this lane's tile column
    if (lane < NP && tl < TI) {
#pragma unroll
      for (int r = 0; r < 8; ++r) hc[8 * TI + r] += S[r * NP + (lane ^ sswz(r))];  // rows of tile row TI
    }
    if (lane < NP && tl == TI) {
      const int c = lane - 8 * TI;  // column within the diagonal tile
      const int cs = sswz(c);
#pragma unroll
      for (int r = 0; r < 8; ++r)
        hc[8 * TI + r] += (r >= c) ? S[r * NP + (lane ^ sswz(r))] : S[c * NP + ((8 * TI + r) ^ cs)];
#pragma unroll
      for (int i = 0; i < 8 * TI; ++i) hc[i] += S[c * NP + (i ^ cs)];  // H[i][j] = H[j][i], i < 8TI
    }
    __syncwarp();
  }

  // hc[i] += (G' diag(w) G)[i][lane]: the lower-triangle 8x8 tiles
  // H_tile(ti, tj) = sum_k (w_k G[k][8ti..]) (x) G[k][8tj..] on the FP64
  // tensor cores, all in one pass over G (each k-step loads the NP/8
  // fragments once and feeds every tile), then scattered one tile row at a
  // time.
  QPB_DEV void form_h_onepass() {
    constexpr int T = NP / 8;
    const int g = lane >> 2, t = lane & 3;
    const double* Gs = a.G();
    const double* wv = a.w();
    const int kblocks = (p + 3) >> 2;
    // accumulators of tile rows 0..3 (tiles (ti, 0..ti)); rows beyond T unused
    double a0c[1][2] = {{0.0, 0.0}};
    double a1c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    double a2c[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    double a3c[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    const int sw = gswz(t);
    for (int kb = 0; kb < kblocks; ++kb) {
      const int k = 4 * kb + t;
      const bool in = k < p;
      const double* row = Gs + (in ? k : 0) * NP;
      const double wk = in ? wv[k] : 0.0;
      double gv[T];
#pragma unroll
      for (int tj = 0; tj < T; ++tj) gv[tj] = in ? row[(8 * tj + g) ^ sw] : 0.0;
      dmma884(a0c[0][0], a0c[0][1], wk * gv[0], gv[0]);
      if constexpr (T > 1) {
        const double w1 = wk * gv[1];
#pragma unroll
        for (int tj = 0; tj < 2; ++tj) dmma884(a1c[tj][0], a1c[tj][1], w1, gv[tj]);
      }
      if constexpr (T > 2) {
        const double w2 = wk * gv[2], w3 = wk * gv[3];
#pragma unroll
        for (int tj = 0; tj < 3; ++tj) dmma884(a2c[tj][0], a2c[tj][1], w2, gv[tj]);
#pragma unroll
        for (int tj = 0; tj < 4; ++tj) dmma884(a3c[tj][0], a3c[tj][1], w3, gv[tj]);
      }
    }
    scatter_tile_row<0>(a0c);
    if constexpr (T > 1) scatter_tile_row<1>(a1c);
    if constexpr (T > 2) {
      scatter_tile_row<2>(a2c);
      scatter_tile_row<3>(a3c);
    }
  }

  // Adds G' diag(w) G to hc (each element of the column exactly once).
  QPB_DEV void form_h_tensor() { form_h_onepass(); }

  // ---------------------------------------------------------------- factor
  // Factor for the weights in shared memory: FP64, or (mixed) FP32.
  // Returns false when the mixed kernel's FP32 factor is rejected: the
  // instance is then handed over to the FP64 kernel (the mixed kernel holds
  // no FP64 factorisation, which keeps its code within the instruction
  // cache: both fully unrolled eliminations in one kernel thrash it).
  QPB_DEV bool factor() {
    if constexpr (kMixed) {
      form_hfull();
      if (inv32()) {
        st_f32++;
        return true;
      }
      st_flags |= kFlagFallback;
      return false;
    } else {
      factor64();
      return true;
    }
  }

  // hc = column `lane` of H = sym(Q) + G' diag(w) G in FP64 (identity
  // columns beyond n)
  QPB_DEV void form_hfull() {
    // (starting from zeros rather than from Q keeps hc in registers)
#pragma unroll
    for (int i = 0; i < NP; ++i) hc[i] = 0.0;
    form_h_tensor();
    double qv[NP];
    load_q(qv);
#pragma unroll
    for (int i = 0; i < NP; ++i) hc[i] = (lane >= n && i == lane) ? 1.0 : qv[i] + hc[i];
  }

  // Shared float regions of the inverse (inside the FP64 factor's regions):
  // Y'[j][i] at Yf[i * kYld + j], float(A) at Af[i * NP + j] (during the
  // factorisation only), F^-1 column-held at Ff[c * MP + i] = F^-1[i][c].
  QPB_DEV float* Yf() const { return reinterpret_cast<float*>(a.Y()); }
  QPB_DEV float* Af() const { return reinterpret_cast<float*>(a.Y()) + MP * kYld; }
  QPB_DEV float* Ff() const { return reinterpret_cast<float*>(a.F()); }

  // Mixed: H (FP64 in hc, from form_hfull, kept there) rounded to FP32 and
  // inverted in FP32 in lf2[] (column `lane` of H^-1), then Y' = H^-1 A'
  // (smem, FP32), F = A Y' (one FP64 tensor-core tile) and F^-1 (smem,
  // FP32).  With explicit inverses every FP32 solve is a few independent
  // dot products instead of two serial triangular sweeps.  Returns false
  // when a pivot is not positive and finite or the pivot ratio
  // max(d)/min(d) of H exceeds pivot_max.
  //
  // Symmetric sweep operator (Gauss-Jordan elimination of a symmetric
  // positive definite matrix, in place): step k maps a_kk -> -1/a_kk,
  // a_ik, a_kj -> a_ik / a_kk, a_kj / a_kk and a_ij -> a_ij - a_ik a_kj / a_kk;
  // after all steps the matrix is -H^-1.  Its step-k pivot a_kk is the LDL^T
  // pivot d_k.  Lane j holds column j; row k is column k (symmetry), so one
  // broadcast per step serves every lane.  The step is branch-free: lane
  // k's own column (its entries are the broadcast ones) is first scaled by
  // 0 and then takes a_ik * (1/a_kk) from the same packed FMA.  (Folding it
  // into one FMA with the multiplier 1/a_kk - 1 loses the relative accuracy
  // of 1/a_kk for large pivots: measured 400x worse inverses.)
  QPB_DEV bool inv32() {
#pragma unroll
    for (int t = 0; t < NP / 2; ++t) lf2[t] = make_float2(__double2float_rn(hc[2 * t]), __double2float_rn(hc[2 * t + 1]));
    int bad = 0;
    float dmax = 0.0f, dmin = INFINITY;
    float* cb = reinterpret_cast<float*>(a.cb());
    const float2* cb2 = reinterpret_cast<const float2*>(cb);
    // The step loop is rolled (one copy of two steps in the instruction
    // cache): at the start of pass k (even) slot s of lf2[] holds entry
    // (k + s) mod NP, so steps k and k + 1 find their pivot entry in slots 0
    // and 1; each pass ends by rotating the slots by one pair.  After NP
    // steps the slots are back in natural order.
#pragma unroll 1
    for (int k = 0; k < NP; k += 2) {
#pragma unroll
      for (int sg = 0; sg < 2; ++sg) {
        const int kk = k + sg;
        const float akj = sg ? lf2[0].y : lf2[0].x;  // this lane's entry kk
        if (lane < NP) cb[lane] = akj;              // = column kk, natural order (symmetry)
        __syncwarp();
        const float pk = cb[kk];
        const float rp = __frcp_rn(pk);
        if (kk < n) {
          bad |= !(pk > 0.0f) || !isfinite(pk);
          dmax = fmaxf(dmax, pk);
          dmin = fminf(dmin, pk);
        }
        const bool own = (lane == kk);
        const float c1 = own ? rp : -(akj * rp);
        const float mu = own ? 0.0f : 1.0f;
        const float2 c12 = make_float2(c1, c1), mu2 = make_float2(mu, mu);
#pragma unroll
        for (int t = 0; t < NP / 2; ++t)  // slot pair t = entries k + 2t, k + 2t + 1
          lf2[t] = __ffma2_rn(cb2[(k / 2 + t) & (NP / 2 - 1)], c12, __fmul2_rn(lf2[t], mu2));
        const float nv = own ? -rp : akj * rp;
        if (sg)
          lf2[0].y = nv;
        else
          lf2[0].x = nv;
        __syncwarp();
      }
      const float2 first = lf2[0];
#pragma unroll
      for (int t = 0; t < NP / 2 - 1; ++t) lf2[t] = lf2[t + 1];
      lf2[NP / 2 - 1] = first;
    }
#pragma unroll
    for (int t = 0; t < NP / 2; ++t) lf2[t] = make_float2(-lf2[t].x, -lf2[t].y);  // H^-1
    // Y'[lane][i] = sum_l H^-1[lane][l] A[i][l] (column `lane` of H^-1 is row `lane`)
    float* Yf = this->Yf();
    float* Af = this->Af();
    if (lane < NP) {
#pragma unroll
      for (int i = 0; i < MP; ++i) Af[i * NP + lane] = __double2float_rn(a.A()[i * NP + lane]);
    }
    __syncwarp();
#pragma unroll 1
    for (int i = 0; i < MP; ++i) {
      float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int t = 0; t < NP / 2; ++t) acc = __ffma2_rn(lf2[t], *reinterpret_cast<const float2*>(Af + i * NP + 2 * t), acc);
      if (lane < NP) Yf[i * kYld + lane] = acc.x + acc.y;
    }
    __syncwarp();
    // F = A Y' (MP x MP, identity beyond m) on the FP64 tensor cores:
    // F[g][c] = sum_k A[g][k] Y'[k][c], four k per step
    float* Ff = this->Ff();
    float fc[MP];
    {
      const int g = lane >> 2, t = lane & 3;
      double f0 = 0.0, f1 = 0.0;
#pragma unroll
      for (int kb = 0; kb < NP / 4; ++kb) {
        const int k = 4 * kb + t;
        const double a0 = (g < MP) ? a.A()[g * NP + k] : 0.0;
        const double b0 = (g < MP) ? (double)Yf[g * kYld + k] : 0.0;
        dmma884(f0, f1, a0, b0);
      }
      if (g < MP) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int c = 2 * t + u;
          if (c < MP) Ff[g * MP + c] = (g < m && c < m) ? __double2float_rn(u ? f1 : f0) : (g == c ? 1.0f : 0.0f);
        }
      }
      __syncwarp();
#pragma unroll
      for (int i = 0; i < MP; ++i) fc[i] = (lane < MP) ? Ff[i * MP + lane] : 0.0f;  // column `lane` of F
      __syncwarp();
    }
    // F^-1 by the same sweep, lanes 0..MP-1 (column-held), back to shared memory
#pragma unroll
    for (int k = 0; k < MP; ++k) {
      if (lane == k) {
#pragma unroll
        for (int i = 0; i < MP; ++i) cb[i] = fc[i];
      }
      __syncwarp();
      const float pk = cb[k];
      const float rp = __frcp_rn(pk);
      if (k < m) bad |= !(pk > 0.0f) || !isfinite(pk);
      const bool own = (lane == k);
      const float akc = fc[k];
      const float c1 = own ? rp : -(akc * rp);
#pragma unroll
      for (int i = 0; i < MP; ++i) fc[i] = fmaf(cb[i], c1, own ? 0.0f : fc[i]);
      fc[k] = own ? -rp : akc * rp;
      __syncwarp();
    }
    if (lane < MP) {
#pragma unroll
      for (int i = 0; i < MP; ++i) Ff[lane * MP + i] = -fc[i];  // F^-1[i][lane]
    }
    __syncwarp();
    return !bad && (double)dmax <= pivot_max * (double)dmin;
  }

  // H = sym(Q) + G' diag(w) G (w in shared memory), LDL^T in registers,
  // then Y = L^-1 A' and F = Y D^-1 Y' with its LDL^T in shared memory.
  QPB_DEV void factor64() {
    form_hfull();
    ldlt64();
  }

  // LDL^T of H (in hc) in FP64, then Y, F and F's factor.
  QPB_DEV void ldlt64() {
    st_f64++;
    dinv = 0.0;
    fdinv = 0.0;
    // LDL^T: step k broadcasts row k of the Schur complement (= column k);
    // Y = L^-1 A' is formed in the same loop: lane j holds Y[j][0..MP), and
    // step k broadcasts lane k's (final) row of Y beside the pivot row.
    int bad = 0;
    double* cb = a.cb();  // 16-byte aligned (WarpArena pads it)
    double* yb = a.Y();   // free until Y is stored below
    double yc[MP];
#pragma unroll
    for (int i = 0; i < MP; ++i) yc[i] = (lane < NP) ? a.A()[i * NP + lane] : 0.0;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      if (lane < NP) cb[lane] = hc[k];
      if (lane == k) {
#pragma unroll
        for (int i = 0; i < MP; ++i) yb[i] = yc[i];
      }
      __syncwarp();
      const double dk = cb[k];
      const double rk = 1.0 / dk;
      if (k < n) bad |= !(dk > 0.0) || !isfinite(dk);
      if (lane == k) dinv = rk;
      // S[i][j] -= (S[k][i] * S[k][j]) / d_k: the product is formed the same
      // way for (i, j) and (j, i), so both triangles stay bit-identical and the
      // row-held and column-held copies of L agree exactly.  The pivot row is
      // read in 16-byte pairs.
      const double hk = hc[k];
      if (lane > k) {
        if ((k + 1) & 1) hc[k + 1] = fma(-(cb[k + 1] * hk), rk, hc[k + 1]);
#pragma unroll
        for (int i2 = ((k + 2) & ~1); i2 < NP; i2 += 2) {
          const double2 c2 = *reinterpret_cast<const double2*>(cb + i2);
          hc[i2] = fma(-(c2.x * hk), rk, hc[i2]);
          hc[i2 + 1] = fma(-(c2.y * hk), rk, hc[i2 + 1]);
        }
        const double l = hk * rk;  // L[lane][k]
#pragma unroll
        for (int i = 0; i < MP; ++i) yc[i] = fma(-l, yb[i], yc[i]);
      }
      __syncwarp();
    }
    if (lane < NP) a.dvi()[lane] = dinv;
    if (lane < NP) {
#pragma unroll
      for (int i = 0; i < MP; ++i) a.Y()[i * kYld + lane] = yc[i];
    }
    __syncwarp();
    // F = Y' D^-1 Y (MP x MP, identity beyond m) on the FP64 tensor cores: one
    // 8 x 8 tile, F[g][c] = sum_j (Y[j][g] dinv_j) Y[j][c], four j per step
    double* Fm = a.F();
    {
      const double* Ys = a.Y();
      const double* dv = a.dvi();
      const int g = lane >> 2, t = lane & 3;
      double f0 = 0.0, f1 = 0.0;
#pragma unroll
      for (int kb = 0; kb < NP / 4; ++kb) {
        const int j = 4 * kb + t;
        const double b0 = (g < MP) ? Ys[g * kYld + j] : 0.0;
        dmma884(f0, f1, b0 * dv[j], b0);
      }
      if (g < MP) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int c = 2 * t + u;
          if (c < MP) Fm[g * MP + c] = (g < m && c < m) ? (u ? f1 : f0) : (g == c ? 1.0 : 0.0);
        }
      }
    }
    __syncwarp();
    // LDL^T of F in registers, lane c owning column c; step k broadcasts
    // column k; the factor goes back to shared memory (the solves read it)
    {
      double fc[MP];
#pragma unroll
      for (int i = 0; i < MP; ++i) fc[i] = (lane < MP) ? Fm[i * MP + lane] : 0.0;
      __syncwarp();
#pragma unroll
      for (int k = 0; k < MP; ++k) {
        if (lane == k) {
#pragma unroll
          for (int i = 0; i < MP; ++i) cb[i] = fc[i];
        }
        __syncwarp();
        const double dk = cb[k];
        const double rk = 1.0 / dk;
        if (k < m) bad |= !(dk > 0.0) || !isfinite(dk);
        if (lane == k) fdinv = rk;
        if (lane > k && lane < MP) {
          const double f = fc[k] * rk;
#pragma unroll
          for (int i = k + 1; i < MP; ++i) fc[i] = fma(-cb[i], f, fc[i]);
        }
        __syncwarp();
      }
      if (lane < MP) {
#pragma unroll
        for (int i = 0; i < MP; ++i) Fm[i * MP + lane] = fc[i];
      }
      __syncwarp();
    }
    if (bad) st_flags |= kFlagBreakdown64;
  }

  QPB_DEV double ycol(int i) const { return lane < NP ? a.Y()[i * kYld + lane] : 0.0; }
  QPB_DEV double fcol(int k) const { return lane < MP ? a.F()[k * MP + lane] : 0.0; }

  // --------------------------------------------------------- reduced solve
  // [H A'; A 0][dx; dy] = [r; v]  (r lane j < n, v lane i < m).  Returns
  // false only in the mixed kernel, when FP64 refinement against the FP32
  // factor stalls (the instance is handed over to the FP64 kernel).
  QPB_DEV bool reduced(double r, double v, double& odx, double& ody) {
    if constexpr (kMixed) {
      if (reduced_refined(r, v, odx, ody)) return true;
      st_flags |= kFlagRefineStall | kFlagFallback;
      return false;
    } else {
      reduced64(r, v, odx, ody);
      return true;
    }
  }

  static QPB_DEV float wmaxf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
  }
  static QPB_DEV float wsumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
  }

  // [H A'; A 0][dx; dy] = [r; v] in FP32 with the explicit inverses:
  // t = H^-1 r, dy = F^-1 (Y'^T r - v), dx = t - Y' dy (F = A H^-1 A').
  QPB_DEV void reduced32(float r, float v, float& odx, float& ody) const {
    float* rb = reinterpret_cast<float*>(a.cb());
    const float* Yf = this->Yf();
    const float* Ff = this->Ff();
    if (lane < NP) rb[lane] = (lane < n) ? r : 0.0f;
    __syncwarp();
    float2 a0 = make_float2(0.0f, 0.0f), a1 = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int t = 0; t < NP / 2; t += 2) {
      a0 = __ffma2_rn(lf2[t], *reinterpret_cast<const float2*>(rb + 2 * t), a0);
      if (t + 1 < NP / 2) a1 = __ffma2_rn(lf2[t + 1], *reinterpret_cast<const float2*>(rb + 2 * t + 2), a1);
    }
    const float tj = (a0.x + a0.y) + (a1.x + a1.y);
    // g_i = (Y'^T r)_i - v_i on lanes i < m (row i of the stored Y'^T)
    float g = 0.0f;
    if (lane < MP) {
      float g0 = 0.0f, g1 = 0.0f;
#pragma unroll
      for (int j = 0; j < NP; j += 2) {
        g0 = fmaf(Yf[lane * kYld + j], rb[j], g0);
        g1 = fmaf(Yf[lane * kYld + j + 1], rb[j + 1], g1);
      }
      g = (lane < m) ? (g0 + g1) - v : 0.0f;
    }
    // dy_i = sum_c F^-1[i][c] g_c on lanes i < m
    float dy = 0.0f;
#pragma unroll
    for (int c = 0; c < MP; ++c) {
      const float gc = __shfl_sync(kFull, g, c);
      if (lane < MP) dy = fmaf(Ff[c * MP + lane], gc, dy);
    }
    dy = (lane < m) ? dy : 0.0f;
    // dx_j = t_j - sum_i Y'[j][i] dy_i
    float xv = tj;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const float di = __shfl_sync(kFull, dy, i);
      if (lane < NP) xv = fmaf(-Yf[i * kYld + lane], di, xv);
    }
    __syncwarp();  // rb read by every lane before the next broadcast
    odx = (lane < n) ? xv : 0.0f;
    ody = dy;
  }

  // Mixed: FP32 solves with FP64 iterative refinement against the FP64
  // operator [H, A'; A, 0], H = sym(Q) + G' diag(w) G as formed in FP64 for
  // this factor (hc: lane j holds column j, so (H dx)_j is one 32-term dot
  // product per lane).  Sweep 0 solves for the right-hand side itself; each
  // later sweep solves for the residual of the current solution and adds
  // the correction.  Stops when the correction, or the next one predicted
  // from the observed contraction, is below 1e-12 of the solution; returns
  // false when the corrections stop shrinking or max_sweeps refinement
  // sweeps do not get there.
  QPB_DEV bool reduced_refined(double r, double v, double& odx, double& ody) {
    double dx = 0.0, dy = 0.0, prev = INFINITY;
    double rx = (lane < n) ? r : 0.0, ry = (lane < m) ? v : 0.0;
#pragma unroll 1
    for (int sw = 0; sw <= max_sweeps; ++sw) {
      if (sw > 0) {
        if (lane < NP) a.xs()[lane] = dx;
        __syncwarp();
        const double* xsv = a.xs();
        double h0 = 0.0, h1 = 0.0;
#pragma unroll
        for (int i = 0; i < NP; i += 2) {
          const double2 x2 = *reinterpret_cast<const double2*>(xsv + i);
          h0 = fma(hc[i], x2.x, h0);
          h1 = fma(hc[i + 1], x2.y, h1);
        }
        double ad = 0.0, adx = 0.0;
#pragma unroll
        for (int i = 0; i < MP; ++i) ad = fma(ycol_a(i), __shfl_sync(kFull, dy, i), ad);
        if constexpr (NP < 32) {  // (warp sums here: the row walk below spills at these budgets)
#pragma unroll
          for (int i = 0; i < MP; ++i) {
            const double s = wsum(ycol_a(i) * dx);
            if (lane == i) adx = s;
          }
        } else if (lane < MP) {
          // (A dx)_lane from row `lane` of A and the broadcast dx; the
          // rotated walk puts the MP lanes' 16-byte reads in distinct banks
          const double* Ar = a.A() + lane * NP;
          double s0 = 0.0, s1 = 0.0;
#pragma unroll
          for (int t = 0; t < NP / 2; ++t) {
            const int j = (2 * (t + lane)) & (NP - 1);
            const double2 A2 = *reinterpret_cast<const double2*>(Ar + j);
            const double2 x2 = *reinterpret_cast<const double2*>(xsv + j);
            s0 = fma(A2.x, x2.x, s0);
            s1 = fma(A2.y, x2.y, s1);
          }
          adx = s0 + s1;
        }
        rx = (lane < n) ? r - ((h0 + h1) + ad) : 0.0;
        ry = (lane < m) ? v - adx : 0.0;
        __syncwarp();  // xs read before it is written again
      }
      float ex, ey;
      reduced32(__double2float_rn(rx), __double2float_rn(ry), ex, ey);
      dx += (double)ex;
      dy += (double)ey;
      if (sw > 0) {
        st_sweeps++;
        // |correction| / |solution| over (dx, dy) jointly; a ratio test
        // needs no more than FP32
        const float en = wmaxf(fmaxf(fabsf(ex), fabsf(ey)));
        const float dn = wmaxf(fmaxf(__double2float_rn(fabs(dx)), __double2float_rn(fabs(dy))));
        const double rel = (double)en / (dn > 0.0f ? (double)dn : 1.0);
        if (rel <= 1e-12 || (sw > 1 && rel * (rel / prev) <= 1e-12)) {
          odx = dx;
          ody = dy;
          return true;
        }
        if (!(rel < 0.5 * prev)) return false;
        if (sw > 1) {
          // at the observed contraction c the last allowed sweep would stop
          // only if rel * c^(max_sweeps - sw + 1) <= 1e-12: give up now
          // otherwise (a stall restarts the iteration in FP64 from the same
          // iterate, so the outcome is the same, without the futile sweeps)
          const double c = rel / prev;
          double pred = rel;
          for (int j = sw; j <= max_sweeps; ++j) pred *= c;
          if (pred > 1e-12) return false;
        }
        prev = rel;
      }
    }
    return false;
  }

  // FP64 factor: [H A'; A 0][dx; dy] = [r; v]  (r lane j < n, v lane i < m)
  QPB_DEV void reduced64(double r, double v, double& odx, double& ody) {
    double u = (lane < n) ? r : 0.0;  // u = L^-1 r
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
    // dy = F^-1 g: forward (lane i > k holds Lf[i][k] df_k in column slot k)
#pragma unroll
    for (int k = 0; k < MP - 1; ++k) {
      const double gk = __shfl_sync(kFull, g, k) * __shfl_sync(kFull, fdinv, k);
      if (lane > k && lane < MP) g = fma(-fcol(k), gk, g);
    }
    g = (lane < MP) ? g * fdinv : 0.0;
    // backward (lane i < k holds Lf[k][i] df_i in slot k)
#pragma unroll
    for (int k = MP - 1; k > 0; --k) {
      const double gk = __shfl_sync(kFull, g, k);
      if (lane < k) g = fma(-fcol(k) * fdinv, gk, g);
    }
    ody = (lane < m) ? g : 0.0;
    // dx = L^-T D^-1 (u - Y dy)
    double wv = u;
#pragma unroll
    for (int i = 0; i < MP; ++i) wv = fma(-ycol(i), __shfl_sync(kFull, g, i), wv);
    double xv = (lane < NP) ? wv * dinv : 0.0;
#pragma unroll
    for (int k = NP - 1; k > 0; --k) {
      const double xk = __shfl_sync(kFull, xv, k);
      if (lane < k) xv = fma(-hc[k] * dinv, xk, xv);  // L[k][i] = hc[k] dinv_i in lane i
    }
    odx = (lane < n) ? xv : 0.0;
  }

  // Row dots G x with x in xs (rotated walk: conflict-free shared reads).
  QPB_DEV double grow_dot(int r, const double* xsv) const {
    const double* row = a.G() + r * NP;
    const int sw = gswz(r);
    double g0 = 0.0, g1 = 0.0;
#pragma unroll
    for (int t = 0; t < NP; t += 2) {
      const int c0 = (t + r) & (NP - 1), c1 = (t + 1 + r) & (NP - 1);
      g0 = fma(row[c0 ^ sw], xsv[c0], g0);
      g1 = fma(row[c1 ^ sw], xsv[c1], g1);
    }
    return g0 + g1;
  }

  // Column dots G' v (v in shared memory, length p), lane j.
  QPB_DEV double gcol_dot(const double* vv) const {
    const int c = lane < NP ? lane : 0;
    const double* G = a.G();
    // the column's position in row r repeats with period 4 (gswz)
    const int c0 = c ^ gswz(0), c1 = c ^ gswz(1), c2 = c ^ gswz(2), c3 = c ^ gswz(3);
    double acc0 = 0.0, acc1 = 0.0;  // even rows, odd rows
    int r = 0;
    for (; r + 4 <= p; r += 4) {
      acc0 = fma(G[r * NP + c0], vv[r], acc0);
      acc1 = fma(G[(r + 1) * NP + c1], vv[r + 1], acc1);
      acc0 = fma(G[(r + 2) * NP + c2], vv[r + 2], acc0);
      acc1 = fma(G[(r + 3) * NP + c3], vv[r + 3], acc1);
    }
    for (; r < p; ++r) {
      const double g = G[r * NP + (c ^ gswz(r))];
      if (r & 1)
        acc1 = fma(g, vv[r], acc1);
      else
        acc0 = fma(g, vv[r], acc0);
    }
    return acc0 + acc1;
  }

  // ------------------------------------------------------------ KKT solve
  // qpax/pdip.py:49-63.  With slack == false the right-hand side is the
  // reduced one directly ([H A'; A 0][dx; dy] = [c1; c4], qpax/pdip.py:22-24).
  // Returns false when the mixed mode's refinement stalled (nothing written).
  QPB_DEV bool solve(bool slack, double c1, const double* c2, const double* c3, double c4, double& odx,
                     double& ody) {
    double p1 = c1;
    if (slack) {
      double* tp = a.tp();
      for (int r = lane; r < p; r += 32) tp[r] = a.w()[r] * (c3[r] - c2[r] / a.z()[r]);
      __syncwarp();
      p1 = (lane < n) ? c1 + gcol_dot(tp) : 0.0;
    }
    if (!reduced(p1, c4, odx, ody)) return false;
    if (slack) {
      if (lane < NP) a.xs()[lane] = odx;
      __syncwarp();
      double* ds = a.ds();
      double* dz = a.dz();
      for (int r = lane; r < p; r += 32) {
        const double dsr = c3[r] - grow_dot(r, a.xs());
        ds[r] = dsr;
        dz[r] = (c2[r] - a.z()[r] * dsr) / a.s()[r];
      }
      __syncwarp();
    }
    return true;
  }

  // -(relaxed KKT residuals): v1, v4 returned in registers, v2, v3 and
  // w = z/s in shared memory; returns the inf-norm.
  // qpax/pdip.py:93-100, pdip_relaxed.py:16-23.
  QPB_DEV double residuals(double kappa, double& v1, double& v4) {
    double qx = 0.0;
    if (lane < NP) a.xs()[lane] = x;  // x broadcast for Q x (and G x below)
    __syncwarp();
    {
      double qv[NP];
      load_q(qv);
      const double* xsv = a.xs();
#pragma unroll
      for (int i = 0; i < NP; ++i) qx = fma(qv[i], xsv[i], qx);
    }
    double ay = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) ay = fma(ycol_a(i), __shfl_sync(kFull, y, i), ay);
    const double r1 = ((qx + q) + ay) + gcol_dot(a.z());
    double loc = (lane < n) ? fabs(r1) : 0.0;
    v1 = (lane < n) ? -r1 : 0.0;
    double r4 = 0.0;
#pragma unroll
    for (int i = 0; i < MP; ++i) {
      const double ax = wsum(ycol_a(i) * x);
      if (lane == i) r4 = ax - b;
    }
    v4 = (lane < m) ? -r4 : 0.0;
    if (lane < m) loc = nmax(loc, fabs(r4));
    for (int r = lane; r < p; r += 32) {
      const double sr = a.s()[r], zr = a.z()[r];
      const double r3 = (grow_dot(r, a.xs()) + sr) - a.h()[r];
      const double r2 = sr * zr - kappa;
      a.v3()[r] = -r3;
      a.v2()[r] = -r2;
      a.w()[r] = zr / sr;
      loc = nmax(loc, nmax(fabs(r3), fabs(r2)));
    }
    __syncwarp();
    return wmax(loc);
  }

  QPB_DEV double ycol_a(int i) const { return lane < NP ? a.A()[i * NP + lane] : 0.0; }

  // min over the lane's entries of -v/d for d < 0 (qpax/pdip.py:66-73 before the cap).
  QPB_DEV double ls_local(const double* v, const double* d) const {
    double mn = INFINITY;
    for (int r = lane; r < p; r += 32) {
      const double dr = d[r];
      if (dr < 0) mn = nmin(mn, -v[r] / dr);
    }
    return mn;
  }

  // qpax/diff_qp.py:20-46 optnet_derivatives :8-17, from the adjoint solution.
  QPB_DEV void write_grads(const InstRef& R, double ddx, double ddy) {
    for (int r = lane; r < p; r += 32) a.dz()[r] = a.dz()[r] / a.z()[r];  // dlam = dlam_tilde / lam
    __syncwarp();
    double* dQ = P->dQ + R.oQ;
    for (int i = 0; i < n; ++i) {
      const double dxi = __shfl_sync(kFull, ddx, i), xi = __shfl_sync(kFull, x, i);
      if (lane < n) dQ[i * n + lane] = 0.5 * (dxi * x + xi * ddx);
    }
    double* dA = P->dA + R.oA;
    for (int i = 0; i < m; ++i) {
      const double dyi = __shfl_sync(kFull, ddy, i), yi = __shfl_sync(kFull, y, i);
      if (lane < n) dA[i * n + lane] = dyi * x + yi * ddx;
    }
    double* dG = P->dG + R.oG;
    for (int r = 0; r < p; ++r) {
      const double lam = a.z()[r], dl = a.dz()[r];
      if (lane < n) dG[r * n + lane] = lam * (dl * x + lam * ddx);
    }
    if (lane < n) P->dq[R.oq + lane] = ddx;
    if (lane < m) P->db[R.ob + lane] = -ddy;
    for (int r = lane; r < p; r += 32) P->dh[R.oh + r] = -a.z()[r] * a.dz()[r];
  }

  // --------------------------------------------------------------- driver
  enum Stage : int { kInit, kStep, kCorrector, kAdjoint, kDone };

  // Mixed kernel: hands this instance over to the FP64 kernel, to resume
  // at `stage` from the current iterate with `it` iterations done and the
  // converged flag so far; records what the mixed kernel did in `stats`.
  QPB_DEV void hand_over(const InstRef& R, long li, int stage, int it, int converged) {
    double* hb = P->hiter + li * (long)P->hstride;
    if (lane < n) hb[lane] = x;
    for (int r = lane; r < p; r += 32) {
      hb[P->n + r] = a.s()[r];
      hb[P->n + P->p + r] = a.z()[r];
    }
    if (lane < m) hb[P->n + 2 * P->p + lane] = y;
    if (lane == 0) {
      P->hstate[3 * li] = stage;
      P->hstate[3 * li + 1] = it;
      P->hstate[3 * li + 2] = converged;
      P->hlist[atomicAdd(P->hcount, 1)] = (int32_t)li;
      if (P->stats) {
        P->stats[R.id * 4 + kStatFact32] = st_f32;
        P->stats[R.id * 4 + kStatFact64] = 0;
        P->stats[R.id * 4 + kStatSweeps] = st_sweeps;
        P->stats[R.id * 4 + kStatFlags] = st_flags;
      }
    }
    __syncwarp();
  }

  // Instance i of this launch; a resume launch (FP64 kernel after the
  // mixed one) takes the i-th handed-over instance.
  QPB_DEV void run(long i) {
    st_f64 = st_flags = 0;
    if constexpr (kMixed) st_f32 = st_sweeps = 0;
    const bool resume = !kMixed && P->resume;
    const long li = resume ? (long)P->hlist[i] : i;  // launch-local index
    const InstRef R = inst_ref(*P, li);
    n = R.n;
    m = R.m;
    p = R.p;
    a.p = p;
    const long inst = R.id;
    const int op = P->op;
    const bool relaxed = (op == kOpRelax || op == kOpBwd);
    const bool fresh = (op == kOpSolve || op == kOpInit);
    int stage;
    if (fresh)
      stage = kInit;
    else
      stage = (op == kOpAdjoint) ? kAdjoint : kStep;
    if (op == kOpSolve && p == 0) stage = kInit;
    int it = 0, converged = 0, conv_now = 0;
    IterSrc src{nullptr, nullptr, nullptr, nullptr};
    if (!fresh) src = IterSrc{P->in[0] + R.oq, P->in[1] + R.oh, P->in[2] + R.oh, P->in[3] + R.ob};
    bool from_iterate = !fresh;
    if (resume) {
      stage = P->hstate[3 * li];
      it = P->hstate[3 * li + 1];
      converged = P->hstate[3 * li + 2];
      const double* hb = P->hiter + li * (long)P->hstride;
      src = IterSrc{hb, hb + P->n, hb + P->n + P->p, hb + P->n + 2 * P->p};
      from_iterate = stage != kInit;
    }
    load(R, op == kOpSolve, from_iterate, src);
    double v1 = 0.0, v4 = 0.0, dxr = 0.0, dyr = 0.0;
    double sigma_mu = 0.0;
    // bounded: initial point + 2 solves per iteration + adjoint; kept
    // rolled (one copy of the stage code in the instruction cache)
#pragma unroll 1
    for (int guard = 0; guard < 2 * kMaxIters + 4 && stage != kDone; ++guard) {
      // ---- prepare the system: weights, right-hand side, factor or not
      bool slack = true, refactor = true;
      double c1 = 0.0, c4 = 0.0;
      const double *c2 = a.v2(), *c3 = a.v3();
      if (stage == kInit) {
        for (int r = lane; r < p; r += 32) a.w()[r] = 1.0;
        __syncwarp();
        slack = false;
        c1 = (lane < n) ? -q + gcol_dot(a.h()) : 0.0;  // r1 = -q + G' h
        c4 = b;
      } else if (stage == kStep) {
        if (it >= kMaxIters || converged) {  // the while-loop condition of qpax
          if (op == kOpBwd) {
            if (P->out[0]) store_iterate(R, false);
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
      } else {  // kAdjoint
        for (int r = lane; r < p; r += 32) {
          a.w()[r] = a.z()[r] / a.s()[r];
          a.v2()[r] = 0.0;
        }
        __syncwarp();
        c1 = (lane < n) ? -P->gx[R.oq + lane] : 0.0;
        c3 = a.v2();
      }
      if constexpr (kMixed) {
        // FP32 factor rejected or refinement stalled: the FP64 kernel takes
        // over (a corrector restarts its iteration from the residuals)
        if ((refactor && !factor()) || !solve(slack, c1, c2, c3, c4, dxr, dyr)) {
          hand_over(R, li, stage == kCorrector ? (int)kStep : stage, it, converged);
          return;
        }
      } else {
        if (refactor) factor();
        solve(slack, c1, c2, c3, c4, dxr, dyr);
      }
      // ---- consume the solution
      if (stage == kInit) {
        x = dxr;
        y = dyr;
        if (p > 0) {  // z = G x - h, then the positivity shifts (qpax/pdip.py:25-33)
          if (lane < NP) a.xs()[lane] = x;
          __syncwarp();
          double zmax = -INFINITY, zmin = INFINITY;
          for (int r = lane; r < p; r += 32) {
            const double zr = grow_dot(r, a.xs()) - a.h()[r];
            a.z()[r] = zr;
            zmax = nmax(zmax, zr);
            zmin = nmin(zmin, zr);
          }
          const double alpha_p = wmax(zmax);
          const double alpha_d = -wmin(zmin);
          for (int r = lane; r < p; r += 32) {
            const double zr = a.z()[r];
            a.s()[r] = (alpha_p < 0) ? -zr : -zr + (1.0 + alpha_p);
            if (alpha_d >= 0) a.z()[r] = zr + (1.0 + alpha_d);
          }
          __syncwarp();
        }
        stage = (op == kOpSolve && p > 0) ? kStep : kDone;
        if (op == kOpSolve && p == 0) converged = 1;  // qpax/pdip.py:208-217
      } else if (stage == kStep && !relaxed) {
        // predictor done (ds, dz hold ds_a, dz_a): centering_params, qpax/pdip.py:76-84
        double sz = 0.0;
        for (int r = lane; r < p; r += 32) sz = fma(a.s()[r], a.z()[r], sz);
        sz = wsum(sz);
        const double mu = sz / p;
        const double alpha_a = nmin(1.0, wmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz()))));
        double num = 0.0;
        for (int r = lane; r < p; r += 32)
          num = fma(a.s()[r] + alpha_a * a.ds()[r], a.z()[r] + alpha_a * a.dz()[r], num);
        num = wsum(num);
        const double ratio = num / sz;
        sigma_mu = ratio * ratio * ratio * mu;
        for (int r = lane; r < p; r += 32) a.v2()[r] = -(-a.v2()[r] - (sigma_mu - a.ds()[r] * a.dz()[r]));
        __syncwarp();
        stage = kCorrector;
      } else if (stage == kStep || stage == kCorrector) {
        // step length and update (qpax/pdip.py:112-117, pdip_relaxed.py:30-35)
        const double ls = wmin(nmin(ls_local(a.s(), a.ds()), ls_local(a.z(), a.dz())));
        const double alpha = relaxed ? 0.99 * nmin(1.0, 0.99 * nmin(1.0, ls)) : 0.99 * nmin(1.0, ls);
        x += alpha * dxr;
        y += alpha * dyr;
        for (int r = lane; r < p; r += 32) {
          a.s()[r] += alpha * a.ds()[r];
          a.z()[r] += alpha * a.dz()[r];
        }
        __syncwarp();
        ++it;
        converged = conv_now;
        stage = kStep;
      } else {  // kAdjoint
        write_grads(R, dxr, dyr);
        stage = kDone;
      }
    }
    if (op == kOpSolve || op == kOpInit || op == kOpRelax) store_iterate(R, op == kOpSolve);
    if (lane == 0) {
      if (P->conv) P->conv[inst] = (op == kOpInit || op == kOpAdjoint) ? 0 : converged;
      if (P->iters) P->iters[inst] = it;
      if (P->stats && resume) {  // added to the mixed kernel's record
        P->stats[inst * 4 + kStatFact64] += st_f64;
        P->stats[inst * 4 + kStatFlags] |= st_flags;
      } else if (P->stats) {
        P->stats[inst * 4 + kStatFact32] = kMixed ? st_f32 : 0;
        P->stats[inst * 4 + kStatFact64] = st_f64;
        P->stats[inst * 4 + kStatSweeps] = kMixed ? st_sweeps : 0;
        P->stats[inst * 4 + kStatFlags] = st_flags;
      }
    }
    __syncwarp();
  }
};

}  // namespace qpb
