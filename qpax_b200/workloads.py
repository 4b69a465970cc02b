"""Seeded synthetic QP batches for the five benchmark configurations.

All arrays are float64 numpy with a leading instance axis.  One
numpy.random.default_rng(seed) per configuration; arrays are drawn batched
in the order written below.  No dataset is involved: these are the shapes and
value distributions the configurations name.

  nnls(N)            Q = F'F, q = -F'g, G = -I, h = 0, no equalities;
                     F (10 x 5), g (10) iid N(0, 1)            (configuration 1)
  dense(B, n, m, p)  Q = M'M + 1e-3 I, q ~ N(0,1), A ~ N(0,1), b = A x0,
                     G ~ N(0,1), h = G x0 + s0, s0 ~ U(0.1, 1): strictly
                     feasible at x0 ~ N(0,1)                    (configurations 2-5)
  uneven(B)          n ~ U{4..256}, p = 2n, m ~ U{0..n//4}, dense generator
                     per instance, one seeded stream per group
                     of 256 instances                           (configuration 4)
  elastic(B)         dense(B, 64, 0, 128); in a random 30% of instances the
                     last 8 rows are overwritten by 4 pairs (g, -g) with
                     h_i + h_j = -U(0.1, 1), which no x satisfies (configuration 5)
"""

from __future__ import annotations

import numpy as np

SEEDS = {1: 1, 2: 2, 3: 3, 4: 4, 5: 5}


def nnls(N: int = 10000, seed: int = SEEDS[1], n: int = 5, rows: int = 10):
    rng = np.random.default_rng(seed)
    F = rng.standard_normal((N, rows, n))
    g = rng.standard_normal((N, rows))
    Q = np.einsum("bki,bkj->bij", F, F)
    q = -np.einsum("bki,bk->bi", F, g)
    G = np.broadcast_to(-np.eye(n), (N, n, n)).copy()
    h = np.zeros((N, n))
    A = np.zeros((N, 0, n))
    b = np.zeros((N, 0))
    return Q, q, A, b, G, h


def dense(B: int, n: int, m: int, p: int, seed: int | np.random.Generator = 0):
    rng = seed if isinstance(seed, np.random.Generator) else np.random.default_rng(seed)
    M = rng.standard_normal((B, n, n))
    Q = np.matmul(M.transpose(0, 2, 1), M) + 1e-3 * np.eye(n)
    q = rng.standard_normal((B, n))
    x0 = rng.standard_normal((B, n))
    A = rng.standard_normal((B, m, n))
    b = np.matmul(A, x0[:, :, None])[:, :, 0]
    G = rng.standard_normal((B, p, n))
    s0 = rng.uniform(0.1, 1.0, (B, p))
    h = np.matmul(G, x0[:, :, None])[:, :, 0] + s0
    return Q, q, A, b, G, h


def config2(B: int = 4096):
    return dense(B, 32, 8, 64, SEEDS[2])


def config3(B: int = 2048):
    return dense(B, 16, 4, 32, SEEDS[3])


def uneven(B: int = 16384, seed: int = SEEDS[4], n_min: int = 4, n_max: int = 256, chunk: int = 256):
    """Ragged batch: lists of per-instance (Q, q, A, b, G, h).

    Shapes come from default_rng(seed): n ~ U{n_min..n_max} for all instances,
    then m ~ U{0..n//4} per instance.  Values come from the dense generator,
    instance by instance, with one default_rng((seed, c)) per group c of
    `chunk` consecutive instances; the groups are drawn on a thread pool (the
    batch at the default size is ~9 GB of FP64 inputs)."""
    import concurrent.futures as cf
    import os

    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, size=B)
    ms = np.array([rng.integers(0, n // 4 + 1) for n in ns], dtype=np.int64)

    def group(c):
        g = np.random.default_rng((seed, c))
        out = []
        for n, m in zip(ns[c * chunk:(c + 1) * chunk], ms[c * chunk:(c + 1) * chunk]):
            inst = dense(1, int(n), int(m), int(2 * n), g)
            out.append([a[0] for a in inst])
        return out

    groups = (B + chunk - 1) // chunk
    try:  # one BLAS thread per worker: the products are small and the pool is the parallelism
        from threadpoolctl import threadpool_limits

        limit = threadpool_limits(1)
    except ImportError:
        limit = None
    try:
        with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
            parts = list(ex.map(group, range(groups)))
    finally:
        if limit is not None:
            limit.restore_original_limits()
    out = [[], [], [], [], [], []]
    for part in parts:
        for inst in part:
            for k in range(6):
                out[k].append(inst[k])
    return out


def elastic(B: int = 1024, seed: int = SEEDS[5], n: int = 64, p: int = 128, frac: float = 0.3, pairs: int = 4):
    """Returns (Q, q, G, h, infeasible_mask); the penalty of configuration 5 is 1e3."""
    rng = np.random.default_rng(seed)
    Q, q, _, _, G, h = dense(B, n, 0, p, rng)
    bad = rng.random(B) < frac
    idx = np.nonzero(bad)[0]
    g = rng.standard_normal((len(idx), pairs, n))
    hi = rng.standard_normal((len(idx), pairs))
    gap = rng.uniform(0.1, 1.0, (len(idx), pairs))
    for k in range(pairs):
        r = p - 2 * pairs + 2 * k
        G[idx, r] = g[:, k]
        G[idx, r + 1] = -g[:, k]
        h[idx, r] = hi[:, k]
        h[idx, r + 1] = -hi[:, k] - gap[:, k]
    return Q, q, G, h, bad


def loss_grad(x):
    """d/dx of ||x - 1||^2, the loss of configurations 3 and 4."""
    return 2.0 * (np.asarray(x) - 1.0)
