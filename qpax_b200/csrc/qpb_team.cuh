// qpb_team.cuh -- cooperative primitives for one "team" of threads that owns
// one QP instance: either one warp (NT == 32, several teams per CTA) or one
// whole CTA (NT == blockDim.x > 32, one team per CTA).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define QPB_DEV __device__ __forceinline__
// Large per-instance phases are real calls: one compiled copy per
// instantiation and a register budget per phase instead of per kernel.
#define QPB_NOINLINE __device__ __noinline__

namespace qpb {

constexpr unsigned kFull = 0xffffffffu;

// NaN-propagating min / max (jnp.min / jnp.max semantics).
QPB_DEV double nmax(double a, double b) { return (a > b || a != a) ? a : b; }
QPB_DEV double nmin(double a, double b) { return (a < b || a != a) ? a : b; }

template <int NT>
struct Team {
  static constexpr int kThreads = NT;
  static constexpr int kWarps = NT / 32;
  int r;        // rank within the team
  double* red;  // shared scratch, >= kWarps doubles, private to this team

  QPB_DEV int lane() const { return r & 31; }
  QPB_DEV int warp() const { return r >> 5; }
  QPB_DEV void sync() const {
    if constexpr (NT == 32) {
      __syncwarp();
    } else {
      __syncthreads();
    }
  }

  template <class Op>
  QPB_DEV double reduce(double v, Op op) const {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(kFull, v, o));
    if constexpr (NT > 32) {
      if (lane() == 0) red[warp()] = v;
      sync();
      v = red[0];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) v = op(v, red[w]);
      sync();
    }
    return v;
  }
  QPB_DEV double sum(double v) const {
    return reduce(v, [](double a, double b) { return a + b; });
  }
  QPB_DEV double max(double v) const {
    return reduce(v, [](double a, double b) { return nmax(a, b); });
  }
  QPB_DEV double min(double v) const {
    return reduce(v, [](double a, double b) { return nmin(a, b); });
  }
  // Integer OR across the team (used for flags).
  QPB_DEV int any(int v) const {
    double d = reduce((double)(v != 0), [](double a, double b) { return a > b ? a : b; });
    return d != 0.0;
  }
};

// ---------------------------------------------------------------- matvecs

// Row dots: for i in [0, rows): epi(i, M[i,:] . x).  Thread per row; the
// column walk starts at a per-row offset so that threads of a warp touch
// different shared-memory banks.
template <int NT, class T, class Epi>
QPB_DEV void rows_dot(const Team<NT>& t, int rows, int cols, const T* M, int ld, const double* x, Epi epi) {
  for (int i = t.r; i < rows; i += NT) {
    const T* row = M + (size_t)i * ld;
    double acc = 0.0;
    int j = cols ? (i % cols) : 0;
    for (int c = 0; c < cols; ++c) {
      acc = fma((double)row[j], x[j], acc);
      j = (j + 1 == cols) ? 0 : j + 1;
    }
    epi(i, acc);
  }
}

// Column dots: for j in [0, cols): epi(j, sum_i M[i][j] x[i]).  Thread per column.
template <int NT, class T, class Epi>
QPB_DEV void cols_dot(const Team<NT>& t, int rows, int cols, const T* M, int ld, const double* x, Epi epi) {
  for (int j = t.r; j < cols; j += NT) {
    double acc = 0.0;
    for (int i = 0; i < rows; ++i) acc = fma((double)M[(size_t)i * ld + j], x[i], acc);
    epi(j, acc);
  }
}

// -------------------------------------------------- LDL^T (lower, in place)

// Right-looking LDL^T of the symmetric n x n matrix whose lower triangle is in
// H (leading dimension ld).  On return the strict lower triangle holds the
// unit factor L, the diagonal holds D, and dinv[k] = 1/D[k].  Returns, to all
// threads, the pivot ratio max(D)/min(D), or +inf when a pivot is not
// strictly positive and finite (factor unusable).
template <int NT, class R>
QPB_NOINLINE double ldlt(const Team<NT>& t, int n, R* H, int ld, R* dinv) {
  for (int k = 0; k < n; ++k) {
    const R dk = H[(size_t)k * ld + k];
    const R inv = R(1) / dk;
    // trailing update with the unscaled column k: H[i][j] -= H[i][k] H[j][k] / d_k
    const int w = t.warp(), l = t.lane();
    for (int i = k + 1 + w; i < n; i += NT / 32) {
      const R hik = H[(size_t)i * ld + k] * inv;
      for (int j = k + 1 + l; j <= i; j += 32) H[(size_t)i * ld + j] -= hik * H[(size_t)j * ld + k];
    }
    t.sync();
  }
  // scale the columns to unit L, collect pivots
  double dmin = INFINITY, dmax = 0.0;
  int bad = 0;
  for (int k = t.r; k < n; k += NT) {
    const R dk = H[(size_t)k * ld + k];
    const double d = (double)dk;
    if (!(d > 0.0) || !isfinite(d)) bad = 1;
    dmin = d < dmin ? d : dmin;
    dmax = d > dmax ? d : dmax;
    dinv[k] = R(1) / dk;
  }
  t.sync();
  for (int e = t.r; e < n * n; e += NT) {
    const int i = e / n, k = e - i * n;
    if (i > k) H[(size_t)i * ld + k] *= dinv[k];
  }
  bad = t.any(bad);
  dmin = t.min(dmin);
  dmax = t.max(dmax);
  t.sync();
  if (bad || n == 0) return bad ? INFINITY : 1.0;
  return dmax / dmin;
}

// ------------------------------------------- single-warp triangular solves
// One warp solves with one right-hand side held in registers: lane l owns
// entries l, l+32, ... (up to kChunks*32 entries).

template <int kChunks>
struct WarpVec {
  double v[kChunks];
};

template <int kChunks>
QPB_DEV double wv_get(const WarpVec<kChunks>& a, int k) {
  const int owner = k & 31, chunk = k >> 5;
  double val = 0.0;
#pragma unroll
  for (int c = 0; c < kChunks; ++c)
    if (c == chunk) val = a.v[c];
  return __shfl_sync(kFull, val, owner);
}

template <int kChunks>
QPB_DEV void wv_load(WarpVec<kChunks>& a, const double* src, int n, int lane) {
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int i = c * 32 + lane;
    a.v[c] = (i < n) ? src[i] : 0.0;
  }
}

template <int kChunks>
QPB_DEV void wv_store(const WarpVec<kChunks>& a, double* dst, int n, int lane) {
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int i = c * 32 + lane;
    if (i < n) dst[i] = a.v[c];
  }
}

// a <- L^-1 a   (unit lower L, ld)
template <int kChunks, class R>
QPB_DEV void wv_lsolve(WarpVec<kChunks>& a, const R* L, int ld, int n, int lane) {
  for (int k = 0; k < n; ++k) {
    const double ak = wv_get(a, k);
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
      const int i = c * 32 + lane;
      if (i > k && i < n) a.v[c] = fma(-(double)L[(size_t)i * ld + k], ak, a.v[c]);
    }
  }
}

// a <- L^-T a   (unit lower L, ld): back substitution with rows of L^T = columns of L.
template <int kChunks, class R>
QPB_DEV void wv_ltsolve(WarpVec<kChunks>& a, const R* L, int ld, int n, int lane) {
  for (int k = n - 1; k >= 0; --k) {
    const double ak = wv_get(a, k);
#pragma unroll
    for (int c = 0; c < kChunks; ++c) {
      const int i = c * 32 + lane;
      if (i < k) a.v[c] = fma(-(double)L[(size_t)k * ld + i], ak, a.v[c]);
    }
  }
}

// a <- a .* d   (d per entry)
template <int kChunks, class R>
QPB_DEV void wv_scale(WarpVec<kChunks>& a, const R* d, int n, int lane) {
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int i = c * 32 + lane;
    if (i < n) a.v[c] *= (double)d[i];
  }
}

// Lane-parallel dot of a warp vector with a shared vector, reduced over the warp.
template <int kChunks, class R>
QPB_DEV double wv_dot(const WarpVec<kChunks>& a, const R* b, int n, int lane) {
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < kChunks; ++c) {
    const int i = c * 32 + lane;
    if (i < n) acc = fma(a.v[c], (double)b[i], acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  return acc;
}

// Copies a rows x n row-major source into dst with row stride ld (columns
// n..ld-1 zeroed), kBatch elements per thread in flight: each batch's loads
// are issued before its stores (source and destination are not known to be
// distinct, so an element-at-a-time loop would wait for every load).  With
// `sym` (rows == n) the copy is (S + S') / 2, each off-diagonal element
// formed as 0.5 * (S[i][j] + S[j][i]); rows for which zero_row(i) holds are
// written as zeros.
struct NoZeroRows {
  QPB_DEV bool operator()(int) const { return false; }
};

template <int NT, class ZeroRow = NoZeroRows>
QPB_DEV void team_copy_rows(const Team<NT>& T, double* dst, int ld, const double* src, int rows, int n, bool sym,
                            ZeroRow zero_row = ZeroRow()) {
  constexpr int kBatch = 8;
  const int total = rows * ld;
  for (int e0 = T.r; e0 < total; e0 += NT * kBatch) {
    double v[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int e = e0 + u * NT;
      double x = 0.0;
      if (e < total) {
        const int i = e / ld, j = e - i * ld;
        if (j < n && !zero_row(i)) {
          x = __ldg(src + (long)i * n + j);
          if (sym && i != j) x = 0.5 * (x + __ldg(src + (long)j * n + i));
        }
      }
      v[u] = x;
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int e = e0 + u * NT;
      if (e < total) dst[e] = v[u];
    }
  }
}

}  // namespace qpb
