"""Conditioning of the reduced KKT matrix along qpax's interior-point path
(test infrastructure: CPU, uses the oracle).

For a batch, the oracle solves to a sequence of tolerances; at each stopping
point the weights w = z/s give H = Q + G' diag(w) G, whose LDL^T pivot ratio
max(d)/min(d) and 2-norm condition number decide whether an FP32
factorisation can serve a solve: FP64 iterative refinement against an FP32
factor contracts by about cond(H) * 2^-24 per sweep, and the rule of the
mixed kernels refactors in FP64 once the pivot ratio passes 1e7.  The same
is reported at the relaxed point (kappa = 1e-3) the backward pass factors.

    python -m oracle.conditioning [--batch 256]
"""

from __future__ import annotations

import argparse

import numpy as np

from oracle import oracle


def pivot_stats(Q, G, s, z):
    ratio, cond = [], []
    for i in range(len(s)):
        H = Q[i] + G[i].T @ ((z[i] / s[i])[:, None] * G[i])
        d = np.diag(np.linalg.cholesky(H)) ** 2
        ratio.append(d.max() / d.min())
        cond.append(np.linalg.cond(H))
    return np.array(ratio), np.array(cond)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=256)
    a = ap.parse_args()
    from qpax_b200 import workloads as wl

    Q, q, A, b, G, h = wl.config2(a.batch)
    print(f"dense QP n=32 m=8 p=64, first {a.batch} instances of the seeded batch")
    print("| stop at residual | mean iterations | pivot ratio median | p90 | share > 1e7 | cond(H) median |"
          " FP64-refinement contraction (cond * 2^-24, median) |")
    print("|---|---|---|---|---|---|---|")
    for tol in (1e2, 1e1, 1e0, 1e-1, 1e-2, 1e-3, 1e-4, 1e-5, 1e-6):
        x, s, z, y, c, it = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=tol)
        r, k = pivot_stats(Q, G, s, z)
        print(f"| {tol:.0e} | {it.mean():.1f} | {np.median(r):.1e} | {np.percentile(r, 90):.1e} | "
              f"{(r > 1e7).mean():.2f} | {np.median(k):.1e} | {np.median(k) * 2.0 ** -24:.1e} |")
    x, s, z, y, c, it = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=1e-6)
    xr, sr, zr, yr, rc, rit = oracle.relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol=1e-6, target_kappa=1e-3)
    r, k = pivot_stats(Q, G, sr, zr)
    print(f"| relaxed point (kappa 1e-3) | {rit.mean():.1f} relax | {np.median(r):.1e} | {np.percentile(r, 90):.1e} |"
          f" {(r > 1e7).mean():.2f} | {np.median(k):.1e} | {np.median(k) * 2.0 ** -24:.1e} |")


if __name__ == "__main__":
    main()
