"""Pins the FP64 CPU oracle to qpax's own tests and golden vectors (CPU only).

Each test names the qpax test it restates.  Fixtures come from
tests/golden/qpax_pins.npz (written by tests/golden/make_golden.py from the
reference checkout).
"""

import numpy as np
import pytest

from oracle import oracle
from tests.refgen import batch_random_qps, generate_random_qp, kkt_inf_norms


def _pin(pins, prefix):
    return {k[len(prefix) + 1:]: pins[k] for k in pins.files if k.startswith(prefix + "/")}


def test_generator_restatement_matches_reference(pins):
    """tests/refgen.generate_random_qp draws exactly what test/misc_test_utils.py draws."""
    for seed in (1, 3):
        np.random.seed(seed)
        for i in range(3):
            mine = generate_random_qp(15, 10, 3)
            ref = _pin(pins, f"gen/seed{seed}/{i}")
            for k, v in zip(("Q", "q", "A", "b", "G", "h", "x", "s", "z", "y"), mine):
                np.testing.assert_array_equal(v, ref[k])


@pytest.mark.parametrize("ny", [3, 0])
def test_qp_solver_double(ny):
    """test/test_qp_solver_double.py:11-50: 1000 QPs each, tol 1e-6, conv, iters<=20, KKT<=tol.

    Seed 1 drives both halves in sequence in qpax; the ny=0 half starts from the
    state the ny=3 half left behind.
    """
    np.random.seed(1)
    first = [generate_random_qp(15, 10, 3) for _ in range(1000)]
    qps = first if ny == 3 else [generate_random_qp(15, 10, 0) for _ in range(1000)]
    Q, q, A, b, G, h = (np.stack([qp[k] for qp in qps]) for k in range(6))
    tol = 1e-6
    x, s, z, y, conv, iters = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=tol)
    assert (conv == 1).all()
    assert iters.max() <= 20
    assert kkt_inf_norms(Q, q, A, b, G, h, x, s, z, y).max() <= tol


def test_qp_solver_single_tolerance_suite():
    """test/test_qp_solver_single.py:19-58 at its tolerance (1e-2, iters<=10), in FP64."""
    Q, q, A, b, G, h, *_ = batch_random_qps(1, 1000, (15, 10, 3))
    x, s, z, y, conv, iters = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=1e-2)
    assert (conv == 1).all() and iters.max() <= 10
    assert kkt_inf_norms(Q, q, A, b, G, h, x, s, z, y).max() <= 1e-2


def _sizes(pins, name):
    d = _pin(pins, f"sizes/{name}")
    return d, (d["Q"], d["q"], d["A"], d["b"], d["G"], d["h"])


def test_no_constraints(pins):
    """test/test_constraint_sizes.py:11-27."""
    d, args = _sizes(pins, "test_no_constraints")
    x, s, z, y, conv, iters = oracle.solve_qp(*args)
    assert conv == 1 and iters == 0
    assert np.abs(d["Q"] @ x + d["q"]).max() < 1e-10


@pytest.mark.parametrize("name", ["test_eq_only", "test_QPSUT03_problem", "test_maros_meszaros"])
def test_known_answers(pins, name):
    """test/test_constraint_sizes.py:30-132 (equality-only exit, h=inf rows)."""
    d, args = _sizes(pins, name)
    x, s, z, y, conv, iters = oracle.solve_qp(*args, solver_tol=float(d["solver_tol"]))
    assert conv == 1
    assert np.abs(x - d["x_expected"]).max() < float(d["x_tol"])


def test_QPTEST(pins):
    """test/test_constraint_sizes.py:135-163: KKT <= 1e-5 with NaNs from inf rows zeroed."""
    d, (Q, q, A, b, G, h) = _sizes(pins, "test_QPTEST")
    x, s, z, y, conv, iters = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=float(d["solver_tol"]))
    with np.errstate(invalid="ignore"):
        r = np.concatenate([Q @ x + q + A.T @ y + G.T @ z, s * z, G @ x + s - h, A @ x - b])
    r = np.where(np.isnan(r), 0, r)
    assert np.abs(r).max() < 1e-5 and conv == 1


def _elastic(pins):
    P = _pin(pins, "elastic/problem_data_pos")
    I = _pin(pins, "elastic/initial_values_pos")
    return P, I


def augmented_problem(Q, q, G, h, penalty):
    """test/test_elastic_qp.py:31-47 create_elastic_problem."""
    nx, ns = len(q), len(h)
    Q2 = np.block([[Q, np.zeros((nx, ns))], [np.zeros((ns, nx)), np.zeros((ns, ns))]])
    q2 = np.concatenate((q, penalty * np.ones(ns)))
    G2 = np.block([[np.zeros((ns, nx)), -np.eye(ns)], [G, -np.eye(ns)]])
    h2 = np.concatenate((np.zeros(ns), h))
    return Q2, q2, np.zeros((0, nx + ns)), np.zeros(0), G2, h2


def test_elastic_golden_augmented(pins):
    """test/test_elastic_qp.py:58-78: augmented standard QP solve and initialize."""
    P, I = _elastic(pins)
    Q2, q2, A2, b2, G2, h2 = augmented_problem(P["Q"], P["q"], P["G"], P["h"], float(P["penalty"]))
    x, s, z, y, conv, iters = oracle.solve_qp(Q2, q2, A2, b2, G2, h2, solver_tol=1e-10)
    assert conv == 1
    assert np.linalg.norm(x - np.concatenate((P["x"], P["t"]))) < 1e-6
    assert np.linalg.norm(s - np.concatenate((P["s1"], P["s2"]))) < 1e-6
    assert np.linalg.norm(z - np.concatenate((P["z1"], P["z2"]))) < 1e-6
    xi, si, zi, yi = oracle.initialize(Q2, q2, A2, b2, G2, h2)
    assert np.linalg.norm(xi - np.concatenate((I["x"], I["t"]))) < 1e-6
    assert np.linalg.norm(si - np.concatenate((I["s1"], I["s2"]))) < 1e-6
    assert np.linalg.norm(zi - np.concatenate((I["z1"], I["z2"]))) < 1e-6


def test_elastic_golden_native(pins):
    """test/test_elastic_qp.py:80-104: initialize_elastic, solve_qp_elastic, primal x."""
    P, I = _elastic(pins)
    args = (P["Q"], P["q"], P["G"], P["h"], float(P["penalty"]))
    init = oracle.initialize_elastic(*args)
    for k, v in zip(("x", "t", "s1", "s2", "z1", "z2"), init):
        assert np.linalg.norm(v - I[k]) < 1e-6, k
    out = oracle.solve_qp_elastic(*args, solver_tol=1e-10)
    assert out[6] == 1
    for k, v in zip(("x", "t", "s1", "s2", "z1", "z2"), out[:6]):
        assert np.linalg.norm(v - P[k]) < 1e-6, k


def test_elastic_vjp_matches_augmented_vjp(pins):
    """test/test_elastic_qp.py:106-144: elastic VJP vs augmented-QP VJP within 1e-3."""
    P, _ = _elastic(pins)
    Q, q, G, h, pen = P["Q"], P["q"], P["G"], P["h"], float(P["penalty"])
    n, p = len(q), len(h)
    rng = np.random.default_rng(0)
    x_des = rng.standard_normal(n)
    x, _ = oracle.solve_qp_elastic_primal_vjp(Q, q, G, h, pen, np.zeros(n), solver_tol=1e-6, target_kappa=1e-3)
    g1 = oracle.solve_qp_elastic_primal_vjp(Q, q, G, h, pen, 2 * (x - x_des), solver_tol=1e-6, target_kappa=1e-3)[1]
    Q2, q2, A2, b2, G2, h2 = augmented_problem(Q, q, G, h, pen)
    x2, _, _, _ = oracle.solve_qp_primal_vjp(Q2, q2, A2, b2, G2, h2, np.zeros(n + p), solver_tol=1e-6)
    dl = np.concatenate((2 * (x2[:n] - x_des), np.zeros(p)))
    _, (dQ2, dq2, _, _, dG2, dh2), _, _ = oracle.solve_qp_primal_vjp(Q2, q2, A2, b2, G2, h2, dl, solver_tol=1e-6,
                                                                     target_kappa=1e-3)
    g2 = (dQ2[:n, :n], dq2[:n], dG2[p:, :n], dh2[p:])
    for a, b_ in zip(g1, g2):
        assert np.linalg.norm(a - b_) < 1e-3


def test_derivatives_vs_finite_differences():
    """test/test_qp_derivatives.py:23-52: jax.grad of ||x-1||^2 vs forward FD (step 1e-3),
    ||grad - fd|| < 0.2 ||fd|| for each of Q, q, A, b, G, h."""
    np.random.seed(3)
    Q, q, A, b, G, h, *_ = generate_random_qp(15, 10, 3)
    inputs = [Q, q, A, b, G, h]
    kappa, tol = 1e-3, 1e-5

    def loss_batch(batch_inputs):
        x = oracle.solve_qp(*batch_inputs, solver_tol=tol)[0]
        return ((x - 1.0) ** 2).sum(axis=-1)

    x0 = oracle.solve_qp(*inputs, solver_tol=tol)[0]
    _, grads, _, _ = oracle.solve_qp_primal_vjp(*inputs, 2 * (x0 - 1.0), solver_tol=tol, target_kappa=kappa)
    base = loss_batch([a[None] for a in inputs])[0]
    for i, X in enumerate(inputs):
        k = X.size
        batch = [np.repeat(a[None], k, axis=0) for a in inputs]
        pert = batch[i].reshape(k, -1)
        pert[np.arange(k), np.arange(k)] += 1e-3
        fd = ((loss_batch(batch) - base) / 1e-3).reshape(X.shape)
        assert np.linalg.norm(grads[i] - fd) < 0.2 * np.linalg.norm(fd)


def test_ragged_batch_equals_one_by_one():
    """A ragged batch gives exactly the per-instance results."""
    np.random.seed(7)
    qps = [generate_random_qp(n, 2 * n, n // 4) for n in (4, 9, 6)]
    cols = list(zip(*qps))
    out = oracle.solve_qp(*[list(c) for c in cols[:6]], solver_tol=1e-6)
    for i, qp in enumerate(qps):
        one = oracle.solve_qp(*qp[:6], solver_tol=1e-6)
        for a, b_ in zip(out, one):
            np.testing.assert_array_equal(np.asarray(a[i]), np.asarray(b_))
