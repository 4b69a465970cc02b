// qpb_linalg.cuh -- per-instance dense kernels of the reduced KKT system:
// H = Q + G^T diag(w) G, its LDL^T factor, the Schur complement on A, and
// the reduced solve used by every Newton / predictor-corrector step.
#pragma once
#include "qpb_blocked.cuh"
#include "qpb_team.cuh"

namespace qpb {

// Bytes carved in 16-byte aligned slices out of one instance's arena.  The
// same walk runs on the host (sizing) and on the device (pointers).
struct Carver {
  uintptr_t cur;
  __host__ __device__ explicit Carver(uintptr_t base) : cur(base) {}
  template <class T>
  __host__ __device__ T* take(size_t count) {
    cur = (cur + 15) & ~uintptr_t(15);
    T* p = reinterpret_cast<T*>(cur);
    cur += count * sizeof(T);
    return p;
  }
};

__host__ __device__ inline int pad4(int n) { return (n + 3) & ~3; }
__host__ __device__ inline int odd_ld(int n) { return n | 1; }

// Factor of the reduced KKT matrix [H A^T; A 0] stored in element type R:
//   H = L diag(d) L^T (unit L, n x n, ld = ldl)   dinv = 1/d
//   Y = L^-1 A^T stored by rows (m x ldy)
//   F = A H^-1 A^T = Y^T diag(dinv) Y = Lf diag(df) Lf^T (m x m, ld = ldf)
template <class R>
struct Factor {
  R *L, *dinv, *Y, *F, *dfinv;
  int ldl, ldy, ldf;
};

// A factor region sized for doubles; a float view reuses the same bytes, and
// so does the blocked FP64 view of the whole KKT matrix (KKTRegion).
struct FactorRegion {
  unsigned char* base;
  int n, m;
  __host__ __device__ static size_t bytes(int n, int m) {
    Carver c(0);
    c.take<double>((size_t)n * odd_ld(n));
    c.take<double>(n);
    c.take<double>((size_t)m * pad4(n));
    c.take<double>((size_t)m * odd_ld(m));
    c.take<double>(m);
    const size_t split = c.cur + 16, whole = KKTRegion::bytes(n, m);
    return split > whole ? split : whole;
  }
  template <class R>
  __device__ Factor<R> view() const {
    Carver c(reinterpret_cast<uintptr_t>(base));
    Factor<R> f;
    f.ldl = odd_ld(n);
    f.ldy = pad4(n);
    f.ldf = odd_ld(m);
    f.L = c.take<R>((size_t)n * f.ldl);
    f.dinv = c.take<R>(n);
    f.Y = c.take<R>((size_t)m * f.ldy);
    f.F = c.take<R>((size_t)m * f.ldf);
    f.dfinv = c.take<R>(m);
    return f;
  }
};

// Lower triangle (with diagonal) of H = sym(Q) + sum_k wk * G[k,:]^T G[k,:]
// in 4x4 register tiles, one tile per thread.  E is the element type of the
// G operand; when kScaleW is false the operand is pre-scaled by sqrt(w) and
// wv is ignored.  Q, G are n4-padded (zero pad columns), ld = ldg.
template <int NT, class R, class E, bool kScaleW>
QPB_NOINLINE void form_H(const Team<NT>& t, int n, int p, const double* Q, int ldq, const E* G, int ldg,
                    const double* wv, R* H, int ldh) {
  const int nb = (n + 3) >> 2;
  const int ntiles = nb * (nb + 1) / 2;
  for (int tau = t.r; tau < ntiles; tau += NT) {
    int bi = (int)((sqrtf(8.0f * tau + 1.0f) - 1.0f) * 0.5f);
    while (bi * (bi + 1) / 2 > tau) --bi;
    while ((bi + 1) * (bi + 2) / 2 <= tau) ++bi;
    const int bj = tau - bi * (bi + 1) / 2;
    R acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] = R(0);
    const E* gi = G + 4 * bi;
    const E* gj = G + 4 * bj;
    for (int k = 0; k < p; ++k) {
      R av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        av[a] = (R)gi[(size_t)k * ldg + a];
        bv[a] = (R)gj[(size_t)k * ldg + a];
      }
      if constexpr (kScaleW) {
        const R wk = (R)wv[k];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] *= wk;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = fma(av[a], bv[c], acc[a][c]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = 4 * bi + a;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int j = 4 * bj + c;
        if (i < n && j <= i) {
          const double qs = 0.5 * (Q[(size_t)i * ldq + j] + Q[(size_t)j * ldq + i]);
          H[(size_t)i * ldh + j] = (R)qs + acc[a][c];
        }
      }
    }
  }
}

// Lower triangle of H = sym(Q) + G' diag(w) G in FP64 on the tensor cores:
// 8x8 tiles of H, one warp per tile, accumulated over p in steps of 4 with
// mma.m8n8k4.f64 (fragments: a0 = A[lane/4][lane%4], b0 = B[lane%4][lane/4],
// (d0, d1) = D[lane/4][2*(lane%4) + {0,1}]).  Columns beyond n read as zero.
template <int NT>
QPB_NOINLINE void form_H_dmma(const Team<NT>& t, int n, int p, const double* Q, int ldq, const double* G, int ldg,
                              const double* wv, double* H, int ldh) {
  const int nb = (n + 7) >> 3;
  const int ntiles = nb * (nb + 1) / 2;
  const int lane = t.lane(), g = lane >> 2, tg = lane & 3;
  for (int tau = t.warp(); tau < ntiles; tau += NT / 32) {
    int bi = (int)((sqrtf(8.0f * tau + 1.0f) - 1.0f) * 0.5f);
    while (bi * (bi + 1) / 2 > tau) --bi;
    while ((bi + 1) * (bi + 2) / 2 <= tau) ++bi;
    const int bj = tau - bi * (bi + 1) / 2;
    const int ci = 8 * bi + g, cj = 8 * bj + g;  // A row / B column this lane feeds
    double d0 = 0.0, d1 = 0.0;
    for (int k0 = 0; k0 < p; k0 += 4) {
      const int k = k0 + tg;
      const bool in = k < p;
      const double* row = G + (size_t)(in ? k : 0) * ldg;
      const double a0 = (in && ci < n) ? wv[k] * row[ci] : 0.0;
      const double b0 = (in && cj < n) ? row[cj] : 0.0;
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                   : "+d"(d0), "+d"(d1)
                   : "d"(a0), "d"(b0));
    }
    const int i = 8 * bi + g;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int j = 8 * bj + 2 * tg + e;
      if (i < n && j <= i) {
        const double qs = 0.5 * (Q[(size_t)i * ldq + j] + Q[(size_t)j * ldq + i]);
        H[(size_t)i * ldh + j] = qs + (e ? d1 : d0);
      }
    }
  }
}

// FP32 H = sym(Q) + GS' GS on the tensor cores for the mixed path (n >= 64),
// GS = float(sqrt(w) G): 16 x 8 tiles of the lower triangle, one warp per
// tile, mma.m16n8k8 over TF32 operands in the 3xTF32 split (x = big + small,
// both TF32; big*big + big*small + small*big accumulated in FP32, small
// products first), which keeps about FP32 accuracy.  Fragments (PTX
// m16n8k8 .tf32): a = A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4];
// b = B[t][g], B[t+4][g]; d = D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]
// with g = lane / 4, t = lane % 4.  A = GS' (row r, column k = GS[k][r]).
QPB_DEV unsigned tf32_big(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
QPB_DEV void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int NT>
QPB_NOINLINE void form_H_tf32(const Team<NT>& t, int n, int p, const double* Q, int ldq, const float* GS, int ldg,
                              float* H, int ldh) {
  const int rb = (n + 15) >> 4, cb = (n + 7) >> 3;
  // tiles (bi, bj) with 8 bj < 16 (bi + 1): the 16-row blocks of the lower triangle
  int ntiles = 0;
  for (int bi = 0; bi < rb; ++bi) ntiles += min(2 * bi + 2, cb);
  const int lane = t.lane(), g = lane >> 2, tg = lane & 3;
  for (int tau = t.warp(); tau < ntiles; tau += NT / 32) {
    int bi = 0, rem = tau;
    while (rem >= min(2 * bi + 2, cb)) {
      rem -= min(2 * bi + 2, cb);
      ++bi;
    }
    const int bj = rem;
    const int r0 = 16 * bi + g, r1 = r0 + 8, cj = 8 * bj + g;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k0 = 0; k0 < p; k0 += 8) {
      const int ka = k0 + tg, kb = ka + 4;
      const float* ra = GS + (size_t)(ka < p ? ka : 0) * ldg;
      const float* rbp = GS + (size_t)(kb < p ? kb : 0) * ldg;
      const float av[4] = {(ka < p && r0 < n) ? ra[r0] : 0.f, (ka < p && r1 < n) ? ra[r1] : 0.f,
                           (kb < p && r0 < n) ? rbp[r0] : 0.f, (kb < p && r1 < n) ? rbp[r1] : 0.f};
      const float bv[2] = {(ka < p && cj < n) ? ra[cj] : 0.f, (kb < p && cj < n) ? rbp[cj] : 0.f};
      unsigned abig[4], asml[4], bbig[2], bsml[2];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        abig[e] = tf32_big(av[e]);
        asml[e] = tf32_big(av[e] - __uint_as_float(abig[e]));
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        bbig[e] = tf32_big(bv[e]);
        bsml[e] = tf32_big(bv[e] - __uint_as_float(bbig[e]));
      }
      mma_tf32(d, abig, bsml);
      mma_tf32(d, asml, bbig);
      mma_tf32(d, abig, bbig);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = (e < 2) ? r0 : r1;
      const int j = 8 * bj + 2 * tg + (e & 1);
      if (i < n && j <= i) {
        const double qs = 0.5 * (Q[(size_t)i * ldq + j] + Q[(size_t)j * ldq + i]);
        H[(size_t)i * ldh + j] = (float)qs + d[e];
      }
    }
  }
}

// Factor the reduced KKT matrix for weights wv.  G, A are n4-padded FP64.
// For R == float, GS (p x ldg floats) is scratch for sqrt(w)-scaled G.
// Returns the H pivot ratio (+inf when the factor is unusable) to all threads.
template <int NT, int KC, class R>
QPB_NOINLINE double factor_kkt(const Team<NT>& t, int n, int m, int p, const double* Q, const double* G, const double* A,
                          int ld, const double* wv, float* GS, const Factor<R>& f) {
  if constexpr (sizeof(R) == 4) {
    for (int e = t.r; e < p * ld; e += NT) {
      const int k = e / ld;
      GS[e] = (float)(sqrt(wv[k]) * G[e]);
    }
    t.sync();
    if (n >= 64)  // GS' GS on the tensor cores (3xTF32) for the larger size bins
      form_H_tf32<NT>(t, n, p, Q, ld, GS, ld, f.L, f.ldl);
    else
      form_H<NT, float, float, false>(t, n, p, Q, ld, GS, ld, wv, f.L, f.ldl);
  } else {
    form_H_dmma<NT>(t, n, p, Q, ld, G, ld, wv, f.L, f.ldl);
  }
  t.sync();
  const double ratio = ldlt<NT, R>(t, n, f.L, f.ldl, f.dinv);
  if (!(ratio < INFINITY)) return ratio;
  if (m > 0) {
    // Y rows: L^-1 A[i,:]^T, one warp per row of A
    const int lane = t.lane();
    for (int i = t.warp(); i < m; i += NT / 32) {
      WarpVec<KC> v;
      wv_load(v, A + (size_t)i * ld, n, lane);
      wv_lsolve(v, f.L, f.ldl, n, lane);
#pragma unroll
      for (int c = 0; c < KC; ++c) {
        const int k = c * 32 + lane;
        if (k < n) f.Y[(size_t)i * f.ldy + k] = (R)v.v[c];
      }
    }
    t.sync();
    // F = Y diag(dinv) Y^T (lower)
    for (int e = t.r; e < m * m; e += NT) {
      const int i = e / m, j = e - i * m;
      if (j > i) continue;
      double acc = 0.0;
      for (int k = 0; k < n; ++k)
        acc = fma((double)f.Y[(size_t)i * f.ldy + k] * (double)f.dinv[k], (double)f.Y[(size_t)j * f.ldy + k], acc);
      f.F[(size_t)i * f.ldf + j] = (R)acc;
    }
    t.sync();
    const double rf = ldlt<NT, R>(t, m, f.F, f.ldf, f.dfinv);
    if (!(rf < INFINITY)) return rf;
  }
  return ratio;
}

// Reduced solve [H A^T; A 0][dx; dy] = [p1; v4] with the factor, by one
// warp (the caller guards on warp 0).  p1, v4 in shared FP64; writes dx, dy.
//   u = L^-1 p1 ; dy = F^-1 (Y diag(dinv) u - v4) ; dx = L^-T diag(dinv) (u - Y^T dy)
template <int KC, class R>
QPB_NOINLINE void reduced_solve_warp(const Factor<R>& f, int n, int m, const double* p1, const double* v4, double* dx,
                                double* dy, int lane) {
  WarpVec<KC> u;
  wv_load(u, p1, n, lane);
  wv_lsolve(u, f.L, f.ldl, n, lane);
  if (m > 0) {
    WarpVec<KC> ud = u;
    wv_scale(ud, f.dinv, n, lane);
    WarpVec<KC> g;
#pragma unroll
    for (int c = 0; c < KC; ++c) g.v[c] = 0.0;
    for (int i = 0; i < m; ++i) {
      const double gi = wv_dot(ud, f.Y + (size_t)i * f.ldy, n, lane) - v4[i];
#pragma unroll
      for (int c = 0; c < KC; ++c)
        if (c == (i >> 5) && lane == (i & 31)) g.v[c] = gi;
    }
    wv_lsolve(g, f.F, f.ldf, m, lane);
    wv_scale(g, f.dfinv, m, lane);
    wv_ltsolve(g, f.F, f.ldf, m, lane);
    wv_store(g, dy, m, lane);
    for (int i = 0; i < m; ++i) {
      const double dyi = wv_get(g, i);
#pragma unroll
      for (int c = 0; c < KC; ++c) {
        const int k = c * 32 + lane;
        if (k < n) u.v[c] = fma(-(double)f.Y[(size_t)i * f.ldy + k], dyi, u.v[c]);
      }
    }
  }
  wv_scale(u, f.dinv, n, lane);
  wv_ltsolve(u, f.L, f.ldl, n, lane);
  wv_store(u, dx, n, lane);
}

}  // namespace qpb
