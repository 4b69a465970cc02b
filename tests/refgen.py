"""Restatements of qpax's test helpers (test infrastructure).

generate_random_qp    test/misc_test_utils.py:5-29  (same np.random draw order)
check_kkt_conditions  test/misc_test_utils.py:32-43
"""

import numpy as np


def generate_random_qp(nx, ns, ny):
    x = np.random.randn(nx)
    Q = np.random.randn(nx, nx)
    Q = Q.T @ Q
    G = np.random.randn(ns, nx)
    A = np.random.randn(ny, nx)
    s = np.abs(np.random.randn(ns))
    z = np.abs(np.random.randn(ns))
    for i in range(ns):
        if np.random.rand() < 0.5:
            s[i] = 0
        else:
            z[i] = 0
    h = G @ x + s
    b = A @ x
    y = np.random.randn(ny)
    q = -Q @ x - G.T @ z - A.T @ y
    return Q, q, A, b, G, h, x, s, z, y


def kkt_inf_norms(Q, q, A, b, G, h, x, s, z, y):
    """Per-instance inf-norms of r1..r4 (batched over a leading axis)."""
    r1 = np.einsum("bij,bj->bi", Q, x) + q + np.einsum("bij,bi->bj", A, y) + np.einsum("bij,bi->bj", G, z)
    r2 = s * z
    r3 = np.einsum("bij,bj->bi", G, x) + s - h
    r4 = np.einsum("bij,bj->bi", A, x) - b
    out = [np.abs(r).max(axis=1) if r.shape[1] else np.zeros(r.shape[0]) for r in (r1, r2, r3, r4)]
    return np.stack(out, axis=1)


def batch_random_qps(seed, count, dims):
    np.random.seed(seed)
    qps = [generate_random_qp(*dims) for _ in range(count)]
    return [np.stack([qp[k] for qp in qps]) for k in range(10)]
