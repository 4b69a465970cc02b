"""CPU checks of the benchmark inputs and of the parity report (no GPU).

The seeded generators in qpax_b200/workloads.py stand in for the five
benchmark configurations; these tests hold them to the configurations' own
wording (shapes, value distributions, feasibility, the infeasible pairs of
the elastic batch).  oracle/parity.py computes the accuracy figures that the
GPU tests and the benchmark report; here it is fed the oracle's own outputs
(every figure must be zero) and copies of them with planted mistakes (each
mistake must show in its figure).  Mistakes are planted in numpy copies of
oracle outputs, on the CPU.  oracle/conditioning.py, the analysis behind the
default precision, is held to the pivot-ratio ranges it reports.
"""

import numpy as np
import pytest

from oracle import oracle, parity
from qpax_b200 import workloads as wl


def test_nnls_configuration_shapes_and_structure():
    """Batched NNLS: Q = F'F (symmetric PSD), q = -F'g, G = -I, h = 0, no equalities."""
    Q, q, A, b, G, h = wl.nnls(64)
    assert Q.shape == (64, 5, 5) and q.shape == (64, 5) and A.shape == (64, 0, 5) and b.shape == (64, 0)
    np.testing.assert_array_equal(G, np.broadcast_to(-np.eye(5), (64, 5, 5)))
    np.testing.assert_array_equal(h, 0.0)
    np.testing.assert_allclose(Q, Q.transpose(0, 2, 1), rtol=0, atol=1e-12)
    assert np.linalg.eigvalsh(Q).min() > 0.0  # F (10 x 5) has full column rank
    rng = np.random.default_rng(wl.SEEDS[1])
    F, g = rng.standard_normal((64, 10, 5)), rng.standard_normal((64, 10))
    np.testing.assert_allclose(q, -np.einsum("bki,bk->bi", F, g), rtol=1e-13, atol=1e-13)


def test_dense_generator_draws_a_strictly_feasible_point():
    """Configuration 2's generator: M, q, x0, A, G, s0 drawn in that order;
    Q = M'M + 1e-3 I, b = A x0, h = G x0 + s0 with s0 in [0.1, 1)."""
    B, n, m, p = 16, 12, 3, 24
    Q, q, A, b, G, h = wl.dense(B, n, m, p, 7)
    rng = np.random.default_rng(7)
    M = rng.standard_normal((B, n, n))
    q_ = rng.standard_normal((B, n))
    x0 = rng.standard_normal((B, n))
    A_ = rng.standard_normal((B, m, n))
    G_ = rng.standard_normal((B, p, n))
    s0 = rng.uniform(0.1, 1.0, (B, p))
    np.testing.assert_array_equal(q, q_)
    np.testing.assert_array_equal(A, A_)
    np.testing.assert_array_equal(G, G_)
    np.testing.assert_allclose(Q, M.transpose(0, 2, 1) @ M + 1e-3 * np.eye(n), rtol=1e-14, atol=1e-12)
    np.testing.assert_allclose(b, np.einsum("bij,bj->bi", A, x0), rtol=1e-13, atol=1e-12)
    slack = h - np.einsum("bij,bj->bi", G, x0)
    assert slack.min() >= 0.1 - 1e-12 and slack.max() < 1.0 + 1e-12
    assert np.linalg.eigvalsh(Q).min() >= 1e-3 - 1e-9


def test_configurations_2_and_3_use_their_seeds_and_shapes():
    Q, q, A, b, G, h = wl.config2(8)
    assert (Q.shape, A.shape, G.shape) == ((8, 32, 32), (8, 8, 32), (8, 64, 32))
    np.testing.assert_array_equal(q, wl.dense(8, 32, 8, 64, wl.SEEDS[2])[1])
    Q, q, A, b, G, h = wl.config3(8)
    assert (Q.shape, A.shape, G.shape) == ((8, 16, 16), (8, 4, 16), (8, 32, 16))
    np.testing.assert_array_equal(G, wl.dense(8, 16, 4, 32, wl.SEEDS[3])[4])


def test_uneven_batch_shapes_and_determinism():
    """Configuration 4: n ~ U{4..256}, p = 2n, m ~ U{0..n//4}; the thread pool
    that draws groups of instances does not change what is drawn."""
    B = 96
    Q, q, A, b, G, h = wl.uneven(B, chunk=32)
    ns = np.array([v.size for v in q])
    ms = np.array([v.size for v in b])
    assert ns.min() >= 4 and ns.max() <= 256
    assert all(h[i].size == 2 * ns[i] for i in range(B))
    assert all(0 <= ms[i] <= ns[i] // 4 for i in range(B))
    assert all(Q[i].shape == (ns[i], ns[i]) and A[i].shape == (ms[i], ns[i]) and G[i].shape == (2 * ns[i], ns[i])
               for i in range(B))
    again = wl.uneven(B, chunk=32)
    for k in range(6):
        for i in (0, 31, 32, B - 1):
            np.testing.assert_array_equal(again[k][i], (Q, q, A, b, G, h)[k][i])
    # instance i of group c is the dense generator's draw from default_rng((seed, c)):
    # q, A, G are raw draws (equal bit for bit); Q, b, h are BLAS products, whose
    # rounding depends on the BLAS thread count (the generator draws on one thread)
    g1 = np.random.default_rng((wl.SEEDS[4], 1))
    for i in range(32, 35):
        inst = wl.dense(1, int(ns[i]), int(ms[i]), int(2 * ns[i]), g1)
        for k in range(6):
            if k in (1, 2, 4):
                np.testing.assert_array_equal(inst[k][0], (Q, q, A, b, G, h)[k][i])
            else:
                np.testing.assert_allclose(inst[k][0], (Q, q, A, b, G, h)[k][i], rtol=1e-13, atol=1e-12)


def test_elastic_batch_infeasible_pairs():
    """Configuration 5: a random 30 % of instances get their last 8 rows
    overwritten by 4 pairs (g, -g) with h_i + h_j = -U(0.1, 1), so g'x <= h_i
    and -g'x <= h_j cannot both hold; the other instances are the dense
    generator's strictly feasible draw."""
    B = 200
    Q, q, G, h, bad = wl.elastic(B)
    assert (Q.shape, G.shape, h.shape) == ((B, 64, 64), (B, 128, 64), (B, 128))
    assert 0.2 < bad.mean() < 0.4
    for k in range(4):
        r = 120 + 2 * k
        np.testing.assert_array_equal(G[bad, r + 1], -G[bad, r])
        gap = h[bad, r] + h[bad, r + 1]
        assert gap.max() <= -0.1 + 1e-12 and gap.min() >= -1.0 - 1e-12
    Qd, qd, _, _, Gd, hd = wl.dense(B, 64, 0, 128, np.random.default_rng(wl.SEEDS[5]))
    good = ~bad
    np.testing.assert_array_equal(G[good], Gd[good])
    np.testing.assert_array_equal(h[good], hd[good])
    np.testing.assert_array_equal(G[bad, :120], Gd[bad, :120])
    np.testing.assert_array_equal(Q, Qd)
    np.testing.assert_array_equal(q, qd)


# --- the parity report -----------------------------------------------------

TOL, KAPPA = 1e-6, 1e-3


@pytest.fixture(scope="module")
def small_batch():
    data = wl.dense(12, 8, 2, 16, 11)
    dl = wl.loss_grad(oracle.solve_qp(*data, solver_tol=TOL)[0])
    x, grads, conv, iters = oracle.solve_qp_primal_vjp(*data, dl, solver_tol=TOL, target_kappa=KAPPA)
    fw = oracle.solve_qp(*data, solver_tol=TOL)
    riters = oracle.relax_qp(*data, *fw[:4], solver_tol=TOL, target_kappa=KAPPA)[5]
    gpu = dict(x=np.array(x), s=np.array(fw[1]), z=np.array(fw[2]), y=np.array(fw[3]), conv=np.array(conv),
               iters=np.array(iters), grads=[np.array(g) for g in grads], riters=np.array(riters))
    assert (gpu["conv"] == 1).all()
    return data, dl, gpu


def _copy(gpu):
    out = {k: (np.array(v) if not isinstance(v, list) else [np.array(g) for g in v]) for k, v in gpu.items()}
    return out


def test_parity_of_the_oracle_with_itself_is_exact(small_batch):
    data, dl, gpu = small_batch
    fig, ref = parity.standard(data, TOL, KAPPA, dl, gpu)
    assert fig["instances"] == fig["compared"] == 12
    for key in ("max_err_x", "max_err_obj", "max_err_grad"):
        assert fig[key] == 0.0, key
    for key in ("conv_mismatch", "gpu_only_converged", "reference_only_converged",
                "iters_mismatch_both_converged", "relax_iters_mismatch_both_converged"):
        assert fig[key] == 0, key
    assert parity.kkt_standard(data, gpu["x"], gpu["s"], gpu["z"], gpu["y"]).max() <= TOL


def test_parity_reports_planted_mistakes(small_batch):
    data, dl, gpu = small_batch
    _, ref = parity.standard(data, TOL, KAPPA, dl, gpu)

    bad = _copy(gpu)
    bad["x"][3, 0] += 1e-3 * max(1.0, np.abs(bad["x"][3]).max())
    fig, _ = parity.standard(data, TOL, KAPPA, dl, bad, ref=ref)
    assert fig["max_err_x"] == pytest.approx(1e-3, rel=1e-6) and fig["max_err_obj"] > 0.0

    bad = _copy(gpu)
    bad["grads"][4][5] *= 1.01
    fig, _ = parity.standard(data, TOL, KAPPA, dl, bad, ref=ref)
    assert fig["max_err_grad"] > 1e-4 and fig["max_err_x"] == 0.0

    bad = _copy(gpu)
    bad["conv"][7] = 0
    bad["iters"][2] += 1
    bad["riters"][9] += 1
    fig, _ = parity.standard(data, TOL, KAPPA, dl, bad, ref=ref)
    assert fig["conv_mismatch"] == 1 and fig["reference_only_converged"] == 1 and fig["gpu_only_converged"] == 0
    assert fig["iters_mismatch_both_converged"] == 1
    assert fig["relax_iters_mismatch_both_converged"] == 1
    assert fig["compared"] == 11


def test_gpu_only_convergence_is_judged_by_its_kkt_residual(small_batch):
    """An instance the reference did not converge on but the GPU did is
    counted apart, with the KKT residual of the GPU's iterate."""
    data, dl, gpu = small_batch
    _, ref = parity.standard(data, TOL, KAPPA, dl, gpu)
    ref = dict(ref)
    ref["conv"] = np.array(ref["conv"])
    ref["conv"][4] = 0
    fig, _ = parity.standard(data, TOL, KAPPA, dl, gpu, ref=ref)
    assert fig["gpu_only_converged"] == 1 and fig["reference_only_converged"] == 0
    assert fig["gpu_only_max_kkt"] <= TOL
    bad = _copy(gpu)
    bad["x"][4] += 0.5
    fig, _ = parity.standard(data, TOL, KAPPA, dl, bad, ref=ref)
    assert fig["gpu_only_max_kkt"] > 0.1



def test_reduced_kkt_conditioning_along_the_path():
    """The measured basis of the precision choice: on the dense configuration
    the reduced KKT matrix H = Q + G' diag(z/s) G is well conditioned early
    in qpax's path and far beyond FP32 refinement (pivot ratio > 1e7, the
    refactor rule) at the 1e-6 stopping point; at the relaxed point the
    backward pass factors it is back within FP32 range."""
    from oracle.conditioning import pivot_stats

    Q, q, A, b, G, h = wl.config2(16)
    _, s0, z0, _, _, _ = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=1e0)
    r0, k0 = pivot_stats(Q, G, s0, z0)
    x, s, z, y, conv, _ = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=1e-6)
    assert (conv == 1).all()
    r6, k6 = pivot_stats(Q, G, s, z)
    _, sr, zr, _, _, _ = oracle.relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol=1e-6, target_kappa=1e-3)
    rr, _ = pivot_stats(Q, G, sr, zr)
    assert (r0 >= 1).all() and (r6 >= 1).all()
    assert np.median(r0) < 1e5 and np.median(k0) * 2.0 ** -24 < 0.1
    assert (r6 > 1e7).mean() >= 0.9 and np.median(k6) * 2.0 ** -24 > 1.0
    assert np.median(rr) < 1e7
