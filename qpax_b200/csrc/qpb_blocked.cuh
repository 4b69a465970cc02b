// qpb_blocked.cuh -- blocked FP64 factorisation of the whole reduced KKT
// matrix and its solve, for teams of two or more warps (one CTA per QP).
//
//   K = [ H  A' ]      H = sym(Q) + G' diag(w) G   (n x n)
//       [ A  0  ]      A                           (m x n)
//
// K = L_K D_K L_K' with L_K = [L 0; M Lf], D_K = diag(D, -Df), where
// H = L D L', M = A L^-T D^-1 and F = A H^-1 A' = Lf Df Lf'.  This is the
// factorisation of qpax's reduced system (qpax/pdip.py:38-63: QR of H and
// of the Schur complement F) in one blocked LDL' pass: the first n pivots
// (H) are eliminated with their trailing updates applied to the A rows too,
// which leaves -F in the (2,2) block; that block is then factored the same
// way.  One solve with L_K, D_K, L_K' gives [dx; dy] of
// [H A'; A 0][dx; dy] = [p1; v4] (qpax/pdip.py:49-63 solve_kkt_rhs).
//
// Layout: K is N x ld FP64, lower triangle used, N = n8 + m8 (n, m padded
// to multiples of 8; pad pivots are identity, pad A rows / columns zero).
// Panels are 32 columns wide (the last of each phase may be 8, 16 or 24).
// Per panel: one warp factors the diagonal block in registers (lane r owns
// row r, shared memory broadcasts the pivot column); every thread solves rows of
// the panel below it (one row per thread); the warps update the trailing
// lower triangle with mma.m8n8k4.f64 (32 x 32 blocks, 4 x 4 fragments).
// H itself is formed with the same tensor-core tiles.
#pragma once
#include "qpb_team.cuh"

namespace qpb {

constexpr int kPanel = 32;
constexpr int kMaxDim = 256;  // n <= 256, m <= 256
constexpr int kLdStride = kPanel + 2;
constexpr int kPanelLd = kPanel + 4;  // row stride of a staged panel: 4 (mod 16)

__host__ __device__ inline int pad8(int n) { return (n + 7) & ~7; }
// Row stride of K: 4 (mod 16) doubles, so that the 8 x 4 fragment loads of a
// warp hit distinct shared-memory banks when K lives in shared memory.
__host__ __device__ inline int kkt_ld(int N) { return ((N + 15) & ~15) + 4; }

// Per-CTA shared staging of the blocked routines.
struct __align__(16) BlockedStage {
  double Ld[kPanel * kLdStride];     // unit L of the current diagonal block, zero on and above
                                     // the diagonal (row-major, 16-byte aligned rows)
  double Dd[kPanel];                 // its pivots
  double Di[kPanel];                 // and their reciprocals
  double col[kPanel];                // broadcast column of the diagonal factorisation
  double part[8 * kPanel];           // per-warp partial sums of the back substitution
  double v[2 * kMaxDim + 16];        // the right-hand side / solution of a solve
};

struct KKTView {
  double* K;
  double* dinv;
  int n, m, n8, m8, N, ld;
};

struct KKTRegion {
  __host__ __device__ static size_t bytes(int n, int m) {
    const int N = pad8(n) + pad8(m);
    return (size_t)N * kkt_ld(N) * sizeof(double) + (size_t)(N + 2) * sizeof(double) + 32;
  }
  __device__ static KKTView view(unsigned char* base, int n, int m) {
    KKTView f;
    f.n = n;
    f.m = m;
    f.n8 = pad8(n);
    f.m8 = pad8(m);
    f.N = f.n8 + f.m8;
    f.ld = kkt_ld(f.N);
    uintptr_t p = (reinterpret_cast<uintptr_t>(base) + 15) & ~uintptr_t(15);
    f.K = reinterpret_cast<double*>(p);
    f.dinv = f.K + (size_t)f.N * f.ld;
    return f;
  }
};

// D += A B on the FP64 tensor cores (no side effects beyond d0, d1, so the
// compiler may schedule fragment loads around it).
QPB_DEV void mma884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Block pair (bi >= bj) of the lower triangle of an nb x nb block grid.
QPB_DEV void tri_pair(int tau, int& bi, int& bj) {
  int r = (int)((sqrtf(8.0f * tau + 1.0f) - 1.0f) * 0.5f);
  while (r * (r + 1) / 2 > tau) --r;
  while ((r + 1) * (r + 2) / 2 <= tau) ++r;
  bi = r;
  bj = tau - r * (r + 1) / 2;
}

// Row stride (doubles) of a chunk of G staged in shared memory: 4 (mod 16),
// so the 8 x 4 fragment reads of a warp are free of bank conflicts.
__host__ __device__ inline int gstage_ld(int ldg) { return ((ldg + 15) & ~15) + 4; }
// Bytes of the two chunk buffers (rows x gstage_ld doubles of G, then rows
// weights, each).
__host__ __device__ inline size_t gstage_bytes(int ldg, int rows) {
  return 2 * (size_t)rows * (gstage_ld(ldg) + 1) * sizeof(double) + 64;
}

QPB_DEV void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
QPB_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int kPending>
QPB_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(kPending) : "memory"); }

// Lower entries of one 32 x 32 block (bi, bj) of H = Q + G' diag(w) G (Q
// symmetric) from the accumulated G' diag(w) G tiles; entries beyond n are
// identity.
QPB_DEV void store_h_block(const KKTView& f, const double* Q, int ldq, int bi, int bj, int nti, int ntj,
                           const double (&acc)[4][4][2], int g, int tg) {
  const int n = f.n;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (!(a < nti && b < ntj)) continue;
      const int i = 32 * bi + 8 * a + g;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int j = 32 * bj + 8 * b + 2 * tg + e;
        if (j > i) continue;
        double v;
        if (i < n && j < n)
          v = Q[(size_t)i * ldq + j] + acc[a][b][e];  // Q was symmetrized when loaded
        else
          v = (i == j) ? 1.0 : 0.0;
        f.K[(size_t)i * f.ld + j] = v;
      }
    }
}

// Fragments of one k-step of a block: A rows from w_k G[k, i-cols], B
// columns from G[k, j-cols]; `row` points at G[k, 0].
QPB_DEV void h_frags(double (&av)[4], double (&bv)[4], const double* row, double wk, bool in, int n, int i0, int j0,
                     int nti, int ntj, int g) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int ci = i0 + 8 * a + g, cj = j0 + 8 * a + g;
    av[a] = (in && a < nti && ci < n) ? wk * row[ci] : 0.0;
    bv[a] = (in && a < ntj && cj < n) ? row[cj] : 0.0;
  }
}
// The (up to) 16 tensor-core tiles of one k-step (lower ones only on a
// diagonal block).
QPB_DEV void h_mmas(double (&acc)[4][4][2], const double (&av)[4], const double (&bv)[4], int nti, int ntj,
                    bool diag) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
      if (a < nti && b < ntj && (!diag || b <= a)) mma884(acc[a][b][0], acc[a][b][1], av[a], bv[b]);
}
QPB_DEV void h_block_kstep(double (&acc)[4][4][2], const double* row, double wk, bool in, int n, int i0, int j0,
                           int nti, int ntj, bool diag, int g) {
  double av[4], bv[4];
  h_frags(av, bv, row, wk, in, n, i0, j0, nti, ntj, g);
  h_mmas(acc, av, bv, nti, ntj, diag);
}

// A full chunk of kRows staged rows: the next k-step's fragments load under
// this one's MMAs.
template <int kRows>
QPB_DEV void h_chunk_pipelined(double (&acc)[4][4][2], const double* buf, const double* wb, int lds, int n, int bi,
                               int bj, int nti, int ntj, int g, int tg) {
  constexpr int kSteps = kRows / 4;
  double av[4], bv[4];
  h_frags(av, bv, buf + (size_t)tg * lds, wb[tg], true, n, 32 * bi, 32 * bj, nti, ntj, g);
#pragma unroll
  for (int s = 0; s < kSteps; ++s) {
    double an[4], bn[4];
    if (s + 1 < kSteps) {
      const int r = 4 * (s + 1) + tg;
      h_frags(an, bn, buf + (size_t)r * lds, wb[r], true, n, 32 * bi, 32 * bj, nti, ntj, g);
    }
    h_mmas(acc, av, bv, nti, ntj, bi == bj);
    if (s + 1 < kSteps) {
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        av[a] = an[a];
        bv[a] = bn[a];
      }
    }
  }
}

// K <- [sym(Q) + G' diag(w) G, A'; A, 0] (lower triangle, padded).  G, A, Q
// are row-major with leading dimensions ldg, lda, ldq (ldg a multiple of 4);
// rows of G beyond p and columns beyond n read as zero.  H is computed in
// 32 x 32 blocks, one per warp.  With `gbuf` (shared memory of
// gstage_bytes(ldg, KR)), the warps take their blocks in rounds and stream G
// through two chunk buffers of KR rows (cp.async double buffering), so each
// row of G crosses from L2 once per round instead of once per block;
// without it, fragments are read from G in place (G in shared memory).
// kVariant only separates the compiled copies of the non-inlined phases per
// kernel (its register budget differs between kernels; a shared copy would
// be compiled for the smallest).
template <int NT, int kVariant = 0>
QPB_NOINLINE void form_kkt(const Team<NT>& t, const KKTView& f, int p, const double* Q, int ldq, const double* G,
                           int ldg, const double* A, int lda, const double* wv, double* gbuf, int KR) {
  constexpr int kWarps = NT / 32;
  const int n = f.n, n8 = f.n8, ld = f.ld;
  const int lane = t.lane(), g = lane >> 2, tg = lane & 3;
  const int nb = (n8 + 31) >> 5;
  const int npairs = nb * (nb + 1) / 2;
  if (gbuf == nullptr) {
    for (int tau = t.warp(); tau < npairs; tau += kWarps) {
      int bi, bj;
      tri_pair(tau, bi, bj);
      const int nti = min(4, (n8 - 32 * bi) >> 3), ntj = min(4, (n8 - 32 * bj) >> 3);
      double acc[4][4][2] = {};
      int k0 = 0;
      for (; k0 + 32 <= p; k0 += 32)  // whole 32-row groups, pipelined
        h_chunk_pipelined<32>(acc, G + (size_t)k0 * ldg, wv + k0, ldg, n, bi, bj, nti, ntj, g, tg);
      for (; k0 < p; k0 += 4) {
        const int k = k0 + tg;
        const bool in = k < p;
        h_block_kstep(acc, G + (size_t)(in ? k : 0) * ldg, in ? wv[k] : 0.0, in, n, 32 * bi, 32 * bj, nti, ntj,
                      bi == bj, g);
      }
      store_h_block(f, Q, ldq, bi, bj, nti, ntj, acc, g, tg);
    }
  } else {
    const int lds = gstage_ld(ldg);
    const int units = ldg >> 1;  // 16-byte pieces per row
    const int nch = (p + KR - 1) / KR;
    double* wbuf = gbuf + (size_t)2 * KR * lds;  // weights of the two chunks
    auto issue = [&](int ch) {
      double* dst = gbuf + (size_t)(ch & 1) * KR * lds;
      const int k0 = ch * KR, rows = min(KR, p - k0);
      for (int e = t.r; e < rows * units; e += NT) {
        const int r = e / units, u = e - r * units;
        cp_async16(dst + (size_t)r * lds + 2 * u, G + (size_t)(k0 + r) * ldg + 2 * u);
      }
      // weights in whole 16-byte pieces (k0 is even): with an odd count the
      // last piece also copies the double after w[p - 1] -- the next array
      // of the arena -- which is never read
      double* wd = wbuf + (ch & 1) * KR;
      for (int e = t.r; 2 * e < rows; e += NT) cp_async16(wd + 2 * e, wv + k0 + 2 * e);
    };
    for (int base = 0; base < npairs; base += kWarps) {
      const int tau = base + t.warp();
      const bool active = tau < npairs;
      int bi = 0, bj = 0;
      if (active) tri_pair(tau, bi, bj);
      const int nti = active ? min(4, (n8 - 32 * bi) >> 3) : 0;
      const int ntj = active ? min(4, (n8 - 32 * bj) >> 3) : 0;
      double acc[4][4][2] = {};
      if (nch > 0) issue(0);
      cp_async_commit();
      for (int ch = 0; ch < nch; ++ch) {
        if (ch + 1 < nch) issue(ch + 1);
        cp_async_commit();
        cp_async_wait<1>();  // this thread's copies of chunk ch have landed
        t.sync();            // and everyone else's
        if (active) {
          const double* buf = gbuf + (size_t)(ch & 1) * KR * lds;
          const double* wb = wbuf + (ch & 1) * KR;
          const int rows = min(KR, p - ch * KR);
          if (rows == KR && KR == 32) {
            h_chunk_pipelined<32>(acc, buf, wb, lds, n, bi, bj, nti, ntj, g, tg);
          } else if (rows == KR && KR == 16) {
            h_chunk_pipelined<16>(acc, buf, wb, lds, n, bi, bj, nti, ntj, g, tg);
          } else if (rows == KR && KR == 8) {
            h_chunk_pipelined<8>(acc, buf, wb, lds, n, bi, bj, nti, ntj, g, tg);
          } else {
            for (int kk = 0; kk < rows; kk += 4) {
              const int r = kk + tg;
              const bool in = r < rows;
              h_block_kstep(acc, buf + (size_t)(in ? r : 0) * lds, in ? wb[r] : 0.0, in, n, 32 * bi, 32 * bj,
                            nti, ntj, bi == bj, g);
            }
          }
        }
        t.sync();  // chunk ch is read before chunk ch + 2 overwrites its buffer
      }
      if (active) store_h_block(f, Q, ldq, bi, bj, nti, ntj, acc, g, tg);
    }
  }
  // A rows (and the zero (2,2) block)
  const int m = f.m, m8 = f.m8;
  const int w2 = n8 + m8;
  for (int e = t.r; e < m8 * w2; e += NT) {
    const int r = e / w2, j = e - r * w2;
    if (j > n8 + r) continue;
    double v = 0.0;
    if (j < n8) {
      if (r < m && j < n) v = A[(size_t)r * lda + j];
    }
    f.K[(size_t)(n8 + r) * ld + j] = v;
  }
}

// LDL' of the w x w diagonal block at (J0, J0) by one warp: lane r owns row r
// (entries c <= r in registers), pivot columns are broadcast through shared
// memory.  Writes the unit factor and the pivots to K, 1/d to dinv, and a
// copy to the stage.  Pivots of rows J0 + r < real_end are checked (must be
// positive and finite).
QPB_DEV void diag_factor(const KKTView& f, int J0, int w, int real_end, int sign, BlockedStage* st, int lane,
                         double& dmin, double& dmax, int& bad) {
  double* K = f.K;
  const int ld = f.ld;
  double row[kPanel];
#pragma unroll
  for (int c = 0; c < kPanel; ++c) {
    double v = (c == lane) ? 1.0 : 0.0;
    if (lane < w && c < w && c <= lane) v = K[(size_t)(J0 + lane) * ld + J0 + c];
    row[c] = v;
  }
  // Column k is broadcast through shared memory (every lane stores its entry
  // k, then reads the others): unlike a shuffle per entry, this keeps `row`
  // in registers after full unrolling.  Rows and columns beyond w are
  // identity: the steps stop at w (a multiple of 8, the same for the warp).
  double* col = st->col;
#pragma unroll
  for (int k = 0; k < kPanel; ++k) {
    if (k >= w) break;
    col[lane] = row[k];
    __syncwarp();
    // a reciprocal and a product: an FP64 division per lane is more than
    // twice as long on this chain
    const double lr = row[k] * (1.0 / col[k]);  // L[r][k] for lanes r > k
#pragma unroll
    for (int c = k + 1; c < kPanel; ++c) {
      const double vc = col[c];  // H[c][k]
      if (lane >= c) row[c] = fma(-lr, vc, row[c]);
    }
    if (lane > k) row[k] = lr;
    __syncwarp();
  }
  double d = 1.0;
#pragma unroll
  for (int c = 0; c < kPanel; ++c)
    if (c == lane) d = row[c];
  if (lane < w) {
    double* Kr = K + (size_t)(J0 + lane) * ld + J0;
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      if (c < lane) Kr[c] = row[c];
      st->Ld[lane * kLdStride + c] = (c < lane) ? row[c] : 0.0;
    }
    const double di = 1.0 / d;
    Kr[lane] = d;
    st->Dd[lane] = d;
    st->Di[lane] = di;
    f.dinv[J0 + lane] = sign > 0 ? di : -di;
    if (J0 + lane < real_end) {
      if (!(d > 0.0) || !isfinite(d)) bad = 1;
      dmin = d < dmin ? d : dmin;
      dmax = d > dmax ? d : dmax;
    }
  }
}

// Eliminate pivots [J0s, J0e) of the lower matrix K[0:N, 0:N] (rows below
// are updated too).  sign = -1 stores dinv = -1/d (the (2,2) block of K_K).
template <int NT>
QPB_DEV void ldlt_phase(const Team<NT>& t, const KKTView& f, int J0s, int J0e, int real_end, int sign,
                        BlockedStage* st, double* pbuf, size_t pcap, double& dmin, double& dmax, int& bad) {
  double* K = f.K;
  const int ld = f.ld, N = f.N;
  const int lane = t.lane(), g = lane >> 2, tg = lane & 3;
  for (int J0 = J0s; J0 < J0e; J0 += kPanel) {
    const int w = min(kPanel, J0e - J0);
    if (t.warp() == 0) diag_factor(f, J0, w, real_end, sign, st, lane, dmin, dmax, bad);
    t.sync();
    const int T0 = J0 + w;
    // With a shared-memory panel buffer large enough, the panel's L rows are
    // also written there and the trailing update reads its fragments from it.
    const bool use_p = pbuf != nullptr && (size_t)(N - T0) * kPanelLd <= pcap;
    const double* Ls = use_p ? pbuf : K + (size_t)T0 * ld + J0;  // L[T0 + r][J0 + c] at Ls[r * lls + c]
    const int lls = use_p ? kPanelLd : ld;
    // panel rows below: L[i][J] = (H[i][J] L_JJ^-T) D_J^-1, one row per thread
    for (int i = T0 + t.r; i < N; i += NT) {
      double* Ki = K + (size_t)i * ld + J0;
      double u[kPanel];
#pragma unroll
      for (int c = 0; c < kPanel; ++c) u[c] = (c < w) ? Ki[c] : 0.0;
#pragma unroll
      for (int c = 1; c < kPanel; ++c) {
        if (c < w) {
          // u[c] -= L[c][0:c] . u[0:c] in two chains, L read in pairs (L[c][c] = 0)
          const double2* Lc = reinterpret_cast<const double2*>(st->Ld + c * kLdStride);
          double s0 = u[c], s1 = 0.0;
#pragma unroll
          for (int k = 0; k < c; k += 2) {
            const double2 l2 = Lc[k >> 1];
            s0 = fma(-l2.x, u[k], s0);
            if (k + 1 < c) s1 = fma(-l2.y, u[k + 1], s1);
          }
          u[c] = s0 + s1;
        }
      }
      double* Pi = use_p ? pbuf + (size_t)(i - T0) * kPanelLd : nullptr;
#pragma unroll
      for (int c = 0; c < kPanel; ++c) {
        if (c < w) {
          const double l = u[c] * st->Di[c];
          Ki[c] = l;
          if (use_p) Pi[c] = l;
        }
      }
    }
    t.sync();
    // trailing update of the lower triangle K[T0:N, T0:N] -= L_J D_J L_J'
    const int R = N - T0;
    if (R > 0) {
      const int nb = (R + 31) >> 5;
      const int npairs = nb * (nb + 1) / 2;
      for (int tau = t.warp(); tau < npairs; tau += NT / 32) {
        int bi, bj;
        tri_pair(tau, bi, bj);
        const int i0 = T0 + 32 * bi, j0 = T0 + 32 * bj;
        const int nti = min(4, (N - i0) >> 3), ntj = min(4, (N - j0) >> 3);
        double acc[4][4][2];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            acc[a][b][0] = acc[a][b][1] = 0.0;
            if (a < nti && b < ntj && (bi != bj || b <= a)) {
              const double* c = K + (size_t)(i0 + 8 * a + g) * ld + j0 + 8 * b + 2 * tg;
              acc[a][b][0] = c[0];
              acc[a][b][1] = c[1];
            }
          }
        for (int kk = 0; kk < w; kk += 4) {
          const int k = kk + tg;
          const double dk = st->Dd[k];
          double av[4], bv[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            av[a] = (a < nti) ? -Ls[(size_t)(i0 - T0 + 8 * a + g) * lls + k] * dk : 0.0;
            bv[a] = (a < ntj) ? Ls[(size_t)(j0 - T0 + 8 * a + g) * lls + k] : 0.0;
          }
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
              if (a < nti && b < ntj && (bi != bj || b <= a)) mma884(acc[a][b][0], acc[a][b][1], av[a], bv[b]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            if (!(a < nti && b < ntj && (bi != bj || b <= a))) continue;
            const int i = i0 + 8 * a + g;
            double* c = K + (size_t)i * ld + j0 + 8 * b + 2 * tg;
            const int j = j0 + 8 * b + 2 * tg;
            if (j <= i) c[0] = acc[a][b][0];
            if (j + 1 <= i) c[1] = acc[a][b][1];
          }
      }
    }
    t.sync();
  }
}

// Factor K (already formed).  Returns the pivot ratio max(D)/min(D) of H, or
// +inf when a pivot of H or of F is not strictly positive and finite.
template <int NT, int kVariant = 0>
QPB_NOINLINE double kkt_factor(const Team<NT>& t, const KKTView& f, BlockedStage* st, double* pbuf, size_t pcap) {
  double dmin = INFINITY, dmax = 0.0;
  int bad = 0;
  ldlt_phase<NT>(t, f, 0, f.n8, f.n, 1, st, pbuf, pcap, dmin, dmax, bad);
  double fmin = INFINITY, fmax = 0.0;
  int fbad = 0;
  if (f.m8 > 0) {
    // the (2,2) block now holds -F: negate it (pad pivots -> 1)
    const int n8 = f.n8, m8 = f.m8;
    for (int e = t.r; e < m8 * m8; e += NT) {
      const int r = e / m8, c = e - r * m8;
      if (c > r) continue;
      double* x = f.K + (size_t)(n8 + r) * f.ld + n8 + c;
      *x = (r >= f.m && r == c) ? 1.0 : -*x;
    }
    t.sync();
    ldlt_phase<NT>(t, f, n8, f.N, n8 + f.m, -1, st, pbuf, pcap, fmin, fmax, fbad);
  }
  bad = t.any(bad | fbad);
  dmin = t.min(dmin);
  dmax = t.max(dmax);
  t.sync();
  if (bad) return INFINITY;
  if (f.n == 0) return 1.0;
  return dmax / dmin;
}

// v <- K^-1 v for the factored K (v: N entries in shared memory).
template <int NT, int kVariant = 0>
QPB_NOINLINE void kkt_solve(const Team<NT>& t, const KKTView& f, double* v, BlockedStage* st) {
  const double* K = f.K;
  const int ld = f.ld, N = f.N;
  const int lane = t.lane();
  // forward: L_K y = v, panel by panel (phase boundaries at n8)
  for (int J0 = 0; J0 < N;) {
    const int end = J0 < f.n8 ? f.n8 : N;
    const int w = min(kPanel, end - J0);
    if (t.warp() == 0) {
      double x = (lane < w) ? v[J0 + lane] : 0.0;
      double lrow[kPanel];
#pragma unroll
      for (int k = 0; k < kPanel; ++k) lrow[k] = (lane < w && k < lane) ? K[(size_t)(J0 + lane) * ld + J0 + k] : 0.0;
#pragma unroll
      for (int k = 0; k < kPanel; ++k) {
        if (k >= w) break;  // uniform: later steps touch no lane below w
        const double xk = __shfl_sync(kFull, x, k);
        if (k < lane) x = fma(-lrow[k], xk, x);
      }
      if (lane < w) v[J0 + lane] = x;
    }
    t.sync();
    for (int i = J0 + w + t.r; i < N; i += NT) {
      const double* Ki = K + (size_t)i * ld + J0;
      double s0 = v[i], s1 = 0.0;  // two chains: w is a multiple of 8
#pragma unroll 4
      for (int c = 0; c < w; c += 2) {
        s0 = fma(-Ki[c], v[J0 + c], s0);
        s1 = fma(-Ki[c + 1], v[J0 + c + 1], s1);
      }
      v[i] = s0 + s1;
    }
    t.sync();
    J0 += w;
  }
  for (int i = t.r; i < N; i += NT) v[i] *= f.dinv[i];
  t.sync();
  // backward: L_K' x = y, panels in reverse (phase 2, then phase 1)
  for (int ph = 1; ph >= 0; --ph) {
    const int s0 = ph ? f.n8 : 0, e0 = ph ? N : f.n8;
    if (e0 <= s0) continue;
    for (int J0 = s0 + ((e0 - s0 - 1) / kPanel) * kPanel; J0 >= s0; J0 -= kPanel) {
    const int w = min(kPanel, e0 - J0);
    const int T0 = J0 + w;
    // partial sums of column c of the rows below, one lane per column
    {
      double acc = 0.0;
      if (lane < w) {
#pragma unroll 4
        for (int i = T0 + t.warp(); i < N; i += NT / 32) acc = fma(K[(size_t)i * ld + J0 + lane], v[i], acc);
      }
      st->part[t.warp() * kPanel + lane] = acc;
    }
    t.sync();
    if (t.warp() == 0) {
      double x = 0.0;
      if (lane < w) {
        x = v[J0 + lane];
#pragma unroll
        for (int q2 = 0; q2 < NT / 32; ++q2) x -= st->part[q2 * kPanel + lane];
      }
      double lcol[kPanel];
#pragma unroll
      for (int k = 0; k < kPanel; ++k) lcol[k] = (k < w && k > lane) ? K[(size_t)(J0 + k) * ld + J0 + lane] : 0.0;
#pragma unroll
      for (int k = kPanel - 1; k >= 0; --k) {
        if (k >= w) continue;  // uniform: those steps touch no lane below w
        const double xk = __shfl_sync(kFull, x, k);
        if (k > lane) x = fma(-lcol[k], xk, x);
      }
      if (lane < w) v[J0 + lane] = x;
    }
    t.sync();
    }
  }
}

}  // namespace qpb
