"""GPU parity: every entry point through the C ABI against the FP64 oracle.

Bars (written per assertion):
  x, s, z, y, t, s1, s2, z1, z2: ||gpu - oracle||_inf <= 1e-6 * max(1, ||oracle||_inf) per instance
  gradients:                     ||gpu - oracle||_inf <= 1e-5 * max(1, ||oracle||_inf) per instance and array
  converged flags, iteration counts: identical wherever the reference converges
                                 (where qpax's own method breaks down, the GPU may
                                 converge: checked by its KKT residual)
for each kernel family:
  "auto":     the default dispatch (one warp per instance in FP64 for n <= 32, m <= n_pad/4,
              one CTA per instance in FP64 above)
  "fp64-cta": one CTA per instance, FP64 factor (the plain FP64 kernel)
  "mixed":    FP32 factor + FP64 refinement + FP64 fallback (one warp per instance for
              n <= 32, m <= n_pad/4, one CTA per instance above)
"""

import numpy as np
import pytest
import torch

from oracle import oracle
from qpax_b200 import workloads as wl
from tests.refgen import batch_random_qps, kkt_inf_norms

pytestmark = pytest.mark.gpu

VARIANTS = {
    "auto": dict(precision="auto"),
    "fp64-cta": dict(precision="fp64", team_threads=128),
    "mixed": dict(precision="mixed"),
}
PRECS = list(VARIANTS)
X_TOL = 1e-6
G_TOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from qpax_b200 import _lib as L

    L.load()


def np_(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def rel_err(gpu, ref):
    g, r = np_(gpu), np.asarray(ref)
    B = r.shape[0]
    g, r = g.reshape(B, -1), r.reshape(B, -1)
    if r.shape[1] == 0:
        return np.zeros(B)
    scale = np.maximum(1.0, np.abs(r).max(axis=1))
    return np.abs(g - r).max(axis=1) / scale


def assert_close(gpu, ref, tol, what):
    e = rel_err(gpu, ref)
    bad = np.nonzero(~(e <= tol))[0]
    assert bad.size == 0, f"{what}: {bad.size} instances above {tol}, worst {np.nanmax(e):.3e} at {bad[:5]}"


def check_solve(Q, q, A, b, G, h, tol, prec, max_breakdown=0.0, **kw):
    """Every instance qpax's method solves is solved, in the same number of
    iterations, with x, s, z, y within X_TOL.  Where the FP64 reference
    itself breaks down (its QR-based solve loses accuracy at cond ~1e14+ late
    in the loop: the residual grows until the 30-iteration cap), the GPU may
    converge too -- its returned iterate must then satisfy the KKT conditions
    to 100 x tol (the flag refers to the iterate before qpax's final step);
    those trajectories are set by rounding and are not compared.  The share
    of reference breakdowns is bounded by max_breakdown."""
    import qpax_b200 as qb

    out = qb.solve_qp(Q, q, A, b, G, h, tol, **VARIANTS[prec], **kw)
    ref = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=tol)
    ok = np.atleast_1d(ref[4]) == 1
    assert (~ok).mean() <= max_breakdown, f"reference breakdowns {(~ok).sum()} of {ok.size}"
    conv = np.atleast_1d(np_(out[4]))
    np.testing.assert_array_equal(conv[ok], 1, err_msg="converged flags")
    gpu_only = (conv == 1) & ~ok
    if gpu_only.any():
        outs = [np.asarray(np_(t)).reshape(conv.size, -1) for t in out[:4]]
        kkt = kkt_inf_norms(Q, q, A, b, G, h, *outs).max(axis=1)  # batched inputs
        assert kkt[gpu_only].max() <= 100 * tol, kkt[gpu_only]
    np.testing.assert_array_equal(np.atleast_1d(np_(out[5]))[ok], np.atleast_1d(ref[5])[ok],
                                  err_msg="iteration counts")
    for k, name in enumerate("xszy"):
        assert_close(np_(out[k])[ok], np.asarray(ref[k])[ok], X_TOL, name)
    return out, ref


@pytest.mark.parametrize("prec", PRECS)
def test_nnls_configuration1(prec):
    """Batched NNLS (n=5, p=5, no equalities), solver_tol 1e-6, all six outputs."""
    check_solve(*wl.nnls(2000), 1e-6, prec, max_breakdown=0.002)


@pytest.mark.parametrize("prec", PRECS)
def test_dense_configuration2(prec):
    """n=32, m=8, p=64 at solver_tol 1e-6."""
    check_solve(*wl.dense(256, 32, 8, 64, 12), 1e-6, prec)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("ny", [3, 0])
def test_qpax_random_suite(prec, ny):
    """test/test_qp_solver_double.py:11-50 on the GPU: conv, iters <= 20, KKT <= 1e-6."""
    Q, q, A, b, G, h, *_ = batch_random_qps(1 if ny == 3 else 11, 1000, (15, 10, ny))
    out, _ = check_solve(Q, q, A, b, G, h, 1e-6, prec)
    assert (np_(out[4]) == 1).all() and np_(out[5]).max() <= 20
    kkt = kkt_inf_norms(Q, q, A, b, G, h, *[np_(t) for t in out[:4]])
    assert kkt.max() <= 1e-6


def _vjp_pair(Q, q, A, b, G, h, tol, kappa, prec):
    import qpax_b200 as qb

    x_ref = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=tol)[0]
    dl = wl.loss_grad(x_ref)
    x, grads, conv, iters = qb.solve_qp_primal_vjp(Q, q, A, b, G, h, dl, tol, kappa, **VARIANTS[prec])
    x_o, grads_o, conv_o, iters_o = oracle.solve_qp_primal_vjp(Q, q, A, b, G, h, dl, solver_tol=tol,
                                                              target_kappa=kappa)
    return (x, grads, conv, iters), (x_o, grads_o, conv_o, iters_o)


@pytest.mark.parametrize("prec", PRECS)
def test_gradients_configuration3(prec):
    """n=16, m=4, p=32: solve_qp_primal forward + backward (tol 1e-5, kappa 1e-3) vs the oracle VJP."""
    (x, grads, conv, iters), (x_o, grads_o, conv_o, iters_o) = _vjp_pair(
        *wl.dense(128, 16, 4, 32, 13), 1e-5, 1e-3, prec)
    np.testing.assert_array_equal(np_(conv), conv_o)
    assert_close(x, x_o, X_TOL, "x")
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        assert_close(g, go, G_TOL, name)


def test_gradients_vs_central_differences_of_relaxed_map():
    """The backward pass differentiates qpax's relaxed solution x_kappa(theta)
    (pdip_relaxed.py:70-103 relax_qp at target_kappa, started from the
    solve): central differences of that map with the configuration's step
    1e-6, computed on the GPU with tight tolerances (solve 1e-8, the
    tightest every perturbed copy reaches, relax 1e-11), against the GPU VJP of ||x - 1||^2, on four instances of the
    n=16, m=4, p=32 configuration.  Directions: every q entry, six h, two b
    and two A entries, a diagonal and a symmetric off-diagonal Q pair.  Bar:
    1e-5 * max(1, |grad|) (the oracle's own central differences agree to
    3e-6 here).  dG is not compared with the relaxed map: qpax's formula
    (diff_qp.py:8-17, D(lam)(dlam x' + lam dx')) is not that map's
    derivative in G (the oracle's differences disagree with it by up to 5x on
    these instances); it is held to the oracle's VJP instead
    (test_gradients_configuration3, tests/test_gpu_configs.py)."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = [np.ascontiguousarray(a[:4]) for a in wl.config3(8)]
    n = Q.shape[1]
    x0 = np_(qb.solve_qp(Q, q, A, b, G, h, 1e-5)[0])
    dl = wl.loss_grad(x0)
    _, grads, conv, _ = qb.solve_qp_primal_vjp(Q, q, A, b, G, h, dl, 1e-5, 1e-3)
    assert (np_(conv) == 1).all()
    grads = [np_(g) for g in grads]
    # (argument index in Q q A b G h, flat element indices perturbed together)
    dirs = [(1, [i]) for i in range(n)] + [(5, [r]) for r in range(6)] + [(3, [0]), (3, [1]), (2, [2]), (2, [9])] + \
           [(0, [0]), (0, [2 * n + 5, 5 * n + 2])]
    step = 1e-6
    for inst in range(4):
        batch = [np.repeat(a[inst:inst + 1], 2 * len(dirs), axis=0) for a in (Q, q, A, b, G, h)]
        for k, (ai, idx) in enumerate(dirs):
            for sgn, row in ((1.0, 2 * k), (-1.0, 2 * k + 1)):
                flat = batch[ai][row].reshape(-1)
                flat[idx] += sgn * step
        s = qb.solve_qp(*batch, 1e-8)
        assert np_(s[4]).min() == 1
        r = qb.relax_qp(*batch, *s[:4], 1e-11, 1e-3)
        assert np_(r[4]).min() == 1
        xk = np_(r[0])
        for k, (ai, idx) in enumerate(dirs):
            fd = (xk[2 * k] - xk[2 * k + 1]) @ dl[inst] / (2 * step)
            g = grads[ai][inst].reshape(-1)[idx].sum()
            assert abs(fd - g) <= 1e-5 * max(1.0, abs(g)), (inst, "QqAbGh"[ai], idx, fd, g)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("n", [48, 100, 200])
def test_larger_instances(prec, n):
    """Bins of configuration 4 (p = 2n, m = n/4): solve and gradients."""
    Q, q, A, b, G, h = wl.dense(6, n, n // 4, 2 * n, 100 + n)
    _, ref = check_solve(Q, q, A, b, G, h, 1e-6, prec, max_breakdown=0.5)
    ok = ref[4] == 1
    (_, grads, _, _), (_, grads_o, _, _) = _vjp_pair(Q, q, A, b, G, h, 1e-6, 1e-3, prec)
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        assert_close(np_(g)[ok], go[ok], G_TOL, name)


# Shapes that reach every branch of the blocked FP64 KKT factorisation
# (n > 32): n and m off multiples of 8 (partial panels, identity pads), no
# equalities (no Schur phase), a Schur complement wider than one panel, tiny p
# (the arena then stays in shared memory), the largest shapes (global arenas,
# G staged through shared memory, staged factor panels), p = 0 (qpax's
# equality-only exit).
BLOCKED_SHAPES = [(33, 0, 66), (37, 9, 20), (45, 40, 90), (70, 3, 4), (256, 64, 512), (40, 10, 0)]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", BLOCKED_SHAPES)
def test_blocked_factorisation_shapes(prec, shape):
    n, m, p = shape
    B = 3 if n > 128 else 8
    Q, q, A, b, G, h = wl.dense(B, n, m, p, 300 + n + m + p)
    _, ref = check_solve(Q, q, A, b, G, h, 1e-6, prec, max_breakdown=0.5)
    if p == 0:
        return  # qpax's relax / VJP need inequalities
    ok = ref[4] == 1
    (_, grads, _, _), (_, grads_o, _, _) = _vjp_pair(Q, q, A, b, G, h, 1e-6, 1e-3, prec)
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        assert_close(np_(g)[ok], go[ok], G_TOL, name)


def test_warp_kernel_global_arena():
    """n <= 32 with p = 200: the one-warp-per-instance kernel's arena (71 KB)
    no longer fits four to a CTA in shared memory and lives in global memory
    (grouped loads instead of asynchronous staging).  Forward with h = inf
    rows (qpax/pdip.py:166-178, :243-246) and the VJP, vs the oracle."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = wl.dense(8, 24, 4, 200, 901)
    hi = h.copy()
    hi[:, 5] = np.inf
    hi[2, 17] = np.inf
    x, s, z, y, conv, iters = (np_(t) for t in qb.solve_qp(Q, q, A, b, G, hi, 1e-6))
    ref = oracle.solve_qp(Q, q, A, b, G, hi, solver_tol=1e-6)
    np.testing.assert_array_equal(conv, ref[4])
    np.testing.assert_array_equal(iters, ref[5])
    fin = np.isfinite(hi)
    np.testing.assert_array_equal(np.isinf(s), ~fin)
    np.testing.assert_array_equal(z[~fin], 0.0)
    assert_close(x, ref[0], X_TOL, "x")
    assert_close(y, ref[3], X_TOL, "y")
    assert_close(np.where(fin, s, 0.0), np.where(fin, ref[1], 0.0), X_TOL, "s")
    assert_close(z, ref[2], X_TOL, "z")
    (xv, grads, convv, _), (x_o, grads_o, conv_o, _) = _vjp_pair(Q, q, A, b, G, h, 1e-6, 1e-3, "auto")
    np.testing.assert_array_equal(np_(convv), conv_o)
    assert_close(xv, x_o, X_TOL, "x (vjp)")
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        assert_close(g, go, G_TOL, name)


@pytest.mark.parametrize("prec", PRECS)
def test_elastic_blocked_global_arena(prec):
    """Elastic QPs large enough for the blocked factorisation from a global
    arena (n = 100, p = 150): x and the slacks vs the oracle.  With the
    penalty at 1e3 the final residual of some instances lands next to the
    tolerance, where LDL' (here) and QR (qpax) rounding can decide the last
    iteration differently: counts may differ by one; the outputs must agree."""
    import qpax_b200 as qb

    Q, q, G, h, _ = wl.elastic(6, seed=77, n=100, p=150)
    out = qb.solve_qp_elastic(Q, q, G, h, 1e3, 1e-6, **VARIANTS[prec])
    ref = oracle.solve_qp_elastic(Q, q, G, h, 1e3, solver_tol=1e-6)
    ok = ref[6] == 1
    assert ok.any()
    np.testing.assert_array_equal(np_(out[6])[ok], 1)
    assert np.abs(np_(out[7])[ok].astype(int) - ref[7][ok]).max() <= 1
    for k, name in enumerate(["x", "t", "s1", "s2"]):
        assert_close(np_(out[k])[ok], ref[k][ok], X_TOL, name)


@pytest.mark.parametrize("shape,chunks", [((32, 8, 64), 3), ((40, 0, 80), 1), ((12, 3, 24), 5)])
def test_host_buffer_pipeline(shape, chunks):
    """qpb_solve_qp_primal_vjp_host (host arrays in, host arrays out, chunked
    and overlapped) gives exactly what the device-resident calls give."""
    import qpax_b200 as qb

    n, m, p = shape
    data = wl.dense(23, n, m, p, 500 + n)
    dl = np.full((23, n), 0.1)
    x_h, g_h = qb.solve_qp_primal_vjp_host(*[torch.tensor(a).pin_memory() for a in data],
                                           torch.tensor(dl).pin_memory(), 1e-6, 1e-3, chunks=chunks)
    x_d, g_d, _, _ = qb.solve_qp_primal_vjp(*data, dl, 1e-6, 1e-3)
    np.testing.assert_array_equal(x_h.numpy(), np_(x_d))
    for a, b_, name in zip(g_h, g_d, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        np.testing.assert_array_equal(a.numpy(), np_(b_), err_msg=name)


def test_autograd_matches_vjp():
    """torch.autograd through solve_qp_primal equals the explicit VJP."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = wl.dense(16, 16, 4, 32, 21)
    ts = [torch.tensor(a, device="cuda", requires_grad=True) for a in (Q, q, A, b, G, h)]
    x = qb.solve_qp_primal(*ts, solver_tol=1e-5, target_kappa=1e-3)
    ((x - 1.0) ** 2).sum().backward()
    _, grads, _, _ = qb.solve_qp_primal_vjp(Q, q, A, b, G, h, wl.loss_grad(np_(x)), 1e-5, 1e-3)
    for t, g in zip(ts, grads):
        np.testing.assert_allclose(np_(t.grad), np_(g), rtol=0, atol=1e-12)


def test_autograd_with_host_inputs():
    """Inputs on the host (CPU float64, requires_grad) go through the GPU and
    come back with their gradients on the host, equal to the CUDA-input case
    (solve_qp_primal and solve_qp_elastic_primal)."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = wl.dense(8, 12, 3, 24, 23)
    cpu = [torch.tensor(a, requires_grad=True) for a in (Q, q, A, b, G, h)]
    dev = [torch.tensor(a, device="cuda", requires_grad=True) for a in (Q, q, A, b, G, h)]
    for ts in (cpu, dev):
        x = qb.solve_qp_primal(*ts, solver_tol=1e-6, target_kappa=1e-3)
        ((x - 1.0) ** 2).sum().backward()
    for c, d in zip(cpu, dev):
        assert c.grad is not None and c.grad.device.type == "cpu" and c.grad.dtype == torch.float64
        np.testing.assert_array_equal(c.grad.numpy(), np_(d.grad))
    Qe, qe, Ge, he, _ = wl.elastic(4, seed=3, n=10, p=20, pairs=2)
    cpu = [torch.tensor(a, requires_grad=True) for a in (Qe, qe, Ge, he)]
    x = qb.solve_qp_elastic_primal(*cpu, 50.0, solver_tol=1e-6, target_kappa=1e-3)
    x.sum().backward()
    for c in cpu:
        assert c.grad is not None and c.grad.device.type == "cpu" and c.grad.shape == c.shape


@pytest.mark.parametrize("team", [32, 128])
def test_team_sizes_agree(team):
    """Warp-per-instance and CTA-per-instance teams give the oracle's answer."""
    check_solve(*wl.dense(64, 12, 3, 24, 31), 1e-6, "mixed", team_threads=team)


def _pin(pins, prefix):
    return {k[len(prefix) + 1:]: pins[k] for k in pins.files if k.startswith(prefix + "/")}


@pytest.mark.parametrize("prec", PRECS)
def test_constraint_sizes(pins, prec):
    """test/test_constraint_sizes.py on the GPU: p = 0 exits, h = inf rows, known answers."""
    import qpax_b200 as qb

    for name in ["test_no_constraints", "test_eq_only", "test_QPSUT03_problem", "test_maros_meszaros",
                 "test_QPTEST"]:
        d = _pin(pins, f"sizes/{name}")
        args = [d[k] for k in ("Q", "q", "A", "b", "G", "h")]
        x, s, z, y, conv, iters = (np_(t) for t in qb.solve_qp(*args, float(d["solver_tol"]), **VARIANTS[prec]))
        ref = oracle.solve_qp(*args, solver_tol=float(d["solver_tol"]))
        assert int(conv) == int(ref[4]) == 1, name
        assert int(iters) == int(ref[5]), name
        assert np.abs(x - ref[0]).max() <= X_TOL * max(1, np.abs(ref[0]).max()), name
        if "x_expected" in d:
            assert np.abs(x - d["x_expected"]).max() < float(d["x_tol"]), name
        if name == "test_no_constraints":
            assert int(iters) == 0 and np.abs(d["Q"] @ x + d["q"]).max() < 1e-10
        if d["h"].size:
            np.testing.assert_array_equal(np.isinf(s), np.isinf(d["h"]))
            np.testing.assert_array_equal(z[np.isinf(d["h"])], 0.0)


@pytest.mark.parametrize("prec", PRECS)
def test_elastic_golden(pins, prec):
    """test/test_elastic_qp.py:80-104 on the GPU: initialize_elastic and solve_qp_elastic (tol 1e-10)."""
    import qpax_b200 as qb

    P, I = _pin(pins, "elastic/problem_data_pos"), _pin(pins, "elastic/initial_values_pos")
    args = (P["Q"], P["q"], P["G"], P["h"], float(P["penalty"]))
    for k, v in zip(("x", "t", "s1", "s2", "z1", "z2"), qb.initialize_elastic(*args, **VARIANTS[prec])):
        assert np.linalg.norm(np_(v) - I[k]) < 1e-6, k
    out = qb.solve_qp_elastic(*args, solver_tol=1e-10, **VARIANTS[prec])
    assert int(out[6]) == 1
    for k, v in zip(("x", "t", "s1", "s2", "z1", "z2"), out[:6]):
        assert np.linalg.norm(np_(v) - P[k]) < 1e-6, k


@pytest.mark.parametrize("prec", PRECS)
def test_elastic_configuration5(prec):
    """n=64, p=128, penalty 1e3, 30% infeasible instances: all outputs vs the oracle."""
    import qpax_b200 as qb

    Q, q, G, h, bad = wl.elastic(64)
    out = qb.solve_qp_elastic(Q, q, G, h, 1e3, 1e-6, **VARIANTS[prec])
    ref = oracle.solve_qp_elastic(Q, q, G, h, 1e3, solver_tol=1e-6)
    ok = ref[6] == 1
    assert (~ok).mean() <= 0.1
    np.testing.assert_array_equal(np_(out[6])[ok], 1)
    np.testing.assert_array_equal(np_(out[7])[ok], ref[7][ok])
    # x and the slacks, as the configuration compares them; the duals z1, z2
    # of rows with t = 0 and Gx = h are not unique and are not compared
    for k, name in enumerate(["x", "t", "s1", "s2"]):
        assert_close(np_(out[k])[ok], ref[k][ok], X_TOL, name)


@pytest.mark.parametrize("prec", PRECS)
def test_elastic_gradients(prec):
    """solve_qp_elastic_primal backward vs the oracle's restatement of qpax's elastic VJP."""
    import qpax_b200 as qb

    Q, q, G, h, _ = wl.elastic(32, seed=55, n=12, p=24, pairs=2)
    x_ref = oracle.solve_qp_elastic(Q, q, G, h, 50.0, solver_tol=1e-6)[0]
    dl = wl.loss_grad(x_ref)
    x, grads = qb.solve_qp_elastic_primal_vjp(Q, q, G, h, 50.0, dl, 1e-6, 1e-3, **VARIANTS[prec])
    x_o, grads_o = oracle.solve_qp_elastic_primal_vjp(Q, q, G, h, 50.0, dl, solver_tol=1e-6, target_kappa=1e-3)
    assert_close(x, x_o, X_TOL, "x")
    # qpax's elastic relaxation (elastic_qp.py:255-261) uses residual signs
    # that its own KKT solve does not zero when t != 0, so that loop runs to
    # its 30-iteration cap and the gradient comes from its 30th iterate; the
    # bar for this path is 1e-4 against the oracle.
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dG", "dh"]):
        assert_close(g, go, 1e-4, name)


@pytest.mark.parametrize("prec", PRECS)
def test_elastic_vjp_vs_augmented_vjp(pins, prec):
    """test/test_elastic_qp.py:106-144 on the GPU: elastic VJP vs the VJP of the
    equivalent standard QP, each gradient within 1e-3 (2-norm)."""
    import qpax_b200 as qb
    from tests.test_oracle import augmented_problem

    P = _pin(pins, "elastic/problem_data_pos")
    Q, q, G, h, pen = P["Q"], P["q"], P["G"], P["h"], float(P["penalty"])
    n, p = len(q), len(h)
    x_des = np.random.default_rng(0).standard_normal(n)
    x = np_(qb.solve_qp_elastic(Q, q, G, h, pen, 1e-6, **VARIANTS[prec])[0])
    _, g1 = qb.solve_qp_elastic_primal_vjp(Q, q, G, h, pen, 2 * (x - x_des), 1e-6, 1e-3, **VARIANTS[prec])
    Q2, q2, A2, b2, G2, h2 = augmented_problem(Q, q, G, h, pen)
    x2 = np_(qb.solve_qp(Q2, q2, A2, b2, G2, h2, 1e-6, **VARIANTS[prec])[0])
    dl = np.concatenate((2 * (x2[:n] - x_des), np.zeros(p)))
    _, (dQ2, dq2, _, _, dG2, dh2), _, _ = qb.solve_qp_primal_vjp(Q2, q2, A2, b2, G2, h2, dl, 1e-6, 1e-3,
                                                                 **VARIANTS[prec])
    g2 = (np_(dQ2)[:n, :n], np_(dq2)[:n], np_(dG2)[p:, :n], np_(dh2)[p:])
    for a, b_ in zip(g1, g2):
        assert np.linalg.norm(np_(a) - b_) < 1e-3


def test_relax_and_initialize_entry_points():
    """relax_qp and initialize as standalone calls (qpax.pdip.initialize / relax_qp)."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = wl.dense(32, 10, 2, 20, 41)
    for gi, ri in zip(qb.initialize(Q, q, A, b, G, h), oracle.initialize(Q, q, A, b, G, h)):
        assert_close(gi, ri, 1e-9, "initialize")
    x, s, z, y, _, _ = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=1e-6)
    out = qb.relax_qp(Q, q, A, b, G, h, x, s, z, y, 1e-6, 1e-3)
    ref = oracle.relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol=1e-6, target_kappa=1e-3)
    np.testing.assert_array_equal(np_(out[4]), ref[4])
    for k in range(4):
        assert_close(out[k], ref[k], X_TOL, "relax")


def test_stats_count_factorisations():
    """The optional stats output reports FP32 / FP64 factorisations per instance."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = wl.dense(64, 32, 8, 64, 51)
    stats = torch.zeros(64, 4, dtype=torch.int32, device="cuda")
    _, _, _, _, conv, iters = qb.solve_qp(Q, q, A, b, G, h, 1e-6, precision="mixed", stats=stats)
    st = np_(stats)
    total = st[:, 0] + st[:, 1]
    # one per iteration + the initial point, plus one FP64 refactor where
    # refinement against an accepted FP32 factor stalled (flag 2; the
    # instance stays on FP64 factors afterwards)
    stalled = (st[:, 3] & 2) != 0
    np.testing.assert_array_equal(total, np_(iters) + 1 + stalled)
    assert (st[:, 0] > 0).all() and (st[:, 2] > 0).all()  # FP32 factors served solves, with refinement
    stats.zero_()
    qb.solve_qp(Q, q, A, b, G, h, 1e-6, precision="fp64", stats=stats)
    assert (np_(stats)[:, 0] == 0).all()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(16, 4, 32), (32, 8, 64), (48, 12, 96)])
def test_diff_qp_entry_point(prec, shape):
    """qpb_diff_qp (qpax/diff_qp.py:20-46) as a standalone call at the
    oracle's relaxed iterate: the six gradients vs the oracle's diff_qp."""
    import qpax_b200 as qb

    n, m, p = shape
    Q, q, A, b, G, h = wl.dense(48, n, m, p, 600 + n)
    x, s, z, y, conv, _ = oracle.solve_qp(Q, q, A, b, G, h, solver_tol=1e-6)
    xr, sr, zr, yr, rconv, _ = oracle.relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol=1e-6, target_kappa=1e-3)
    assert (conv == 1).all() and (rconv == 1).all()
    dl = wl.loss_grad(xr)
    grads = qb.diff_qp(Q, q, A, b, G, h, xr, sr, zr, yr, dl, **VARIANTS[prec])
    grads_o = oracle.diff_qp(Q, q, A, b, G, h, xr, sr, zr, yr, dl)
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        assert_close(g, go, G_TOL, name)


def _elastic_solved(seed, n, p, pen):
    Q, q, G, h, _ = wl.elastic(24, seed=seed, n=n, p=p, pairs=2)
    out = oracle.solve_qp_elastic(Q, q, G, h, pen, solver_tol=1e-6)
    assert (out[6] == 1).all()
    return (Q, q, G, h), out


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(12, 24), (64, 128)])
def test_relax_qp_elastic_entry_point(prec, shape):
    """qpb_relax_qp_elastic (qpax/elastic_qp.py:319-359) from the oracle's
    elastic solution: all six relaxed variables, converged flags and
    iteration counts vs the oracle's relax_qp_elastic.  (qpax's elastic
    relaxation does not converge where t != 0 -- its residual signs,
    elastic_qp.py:255-261 -- and runs to the 30-iteration cap there, on both
    sides.)"""
    import qpax_b200 as qb

    n, p = shape
    data, out = _elastic_solved(700 + n, n, p, 50.0)
    got = qb.relax_qp_elastic(*data, 50.0, *out[:6], 1e-6, 1e-3, **VARIANTS[prec])
    ref = oracle.relax_qp_elastic(*data, 50.0, *out[:6], solver_tol=1e-6, target_kappa=1e-3)
    np.testing.assert_array_equal(np_(got[6]), ref[6])
    np.testing.assert_array_equal(np_(got[7]), ref[7])
    # Thirty iterations that never converge amplify rounding: the oracle's
    # own output moves (by ~2e-6 at n = 12, up to ~1e-2 at n = 64) when its
    # starting iterate is perturbed by 1e-15.  Each output of each instance is
    # held to 1e-6, or to ten times that self-spread (two perturbed runs)
    # where the oracle does not reproduce itself to 1e-6.
    rng = np.random.default_rng(9)
    spread = [np.zeros(len(ref[0])) for _ in range(6)]
    for _ in range(2):
        pert = [a * (1.0 + 1e-15 * rng.standard_normal(a.shape)) for a in out[:6]]
        r2 = oracle.relax_qp_elastic(*data, 50.0, *pert, solver_tol=1e-6, target_kappa=1e-3)
        for k in range(6):
            spread[k] = np.maximum(spread[k], rel_err(r2[k], ref[k]))
    for k, name in enumerate(["x", "t", "s1", "s2", "z1", "z2"]):
        e = rel_err(got[k], ref[k])
        bar = np.maximum(X_TOL, 10.0 * spread[k])
        assert (e <= bar).all(), (name, e.max(), spread[k].max())


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(12, 24), (64, 128)])
def test_diff_qp_elastic_entry_point(prec, shape):
    """qpb_diff_qp_elastic (qpax/elastic_qp.py:381-417) as a standalone call at
    the oracle's relaxed elastic iterate: dQ, dq, dG, dh vs the oracle."""
    import qpax_b200 as qb

    n, p = shape
    data, out = _elastic_solved(800 + n, n, p, 50.0)
    rel = oracle.relax_qp_elastic(*data, 50.0, *out[:6], solver_tol=1e-6, target_kappa=1e-3)
    dl = wl.loss_grad(rel[0])
    grads = qb.diff_qp_elastic(*data, *rel[:6], dl, penalty=50.0, **VARIANTS[prec])
    grads_o = oracle.diff_qp_elastic(*data, *rel[:6], dl)
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dG", "dh"]):
        assert_close(g, go, G_TOL, name)


@pytest.mark.parametrize("prec", PRECS)
def test_nonsymmetric_Q_is_read_as_its_symmetric_part(prec):
    """A non-symmetric Q: every entry point reads it as (Q + Q')/2, the matrix
    the objective 1/2 x'Qx depends on.  qpax symmetrizes in solve_qp
    (pdip.py:223) but relaxes and differentiates with the raw Q
    (diff_qp.py:66-67, 76-79) -- a deviation documented with its measured
    size; here the GPU forward must equal the oracle's on the raw Q (qpax's
    own solve) and the GPU backward the oracle's on sym(Q)."""
    import qpax_b200 as qb

    Q, q, A, b, G, h = wl.dense(32, 16, 4, 32, 71)
    K = np.random.default_rng(5).standard_normal(Q.shape)
    Qn = Q + 1e-3 * (K - K.transpose(0, 2, 1)) * np.abs(Q).mean(axis=(1, 2), keepdims=True)
    Qs = 0.5 * (Qn + Qn.transpose(0, 2, 1))
    out = qb.solve_qp(Qn, q, A, b, G, h, 1e-6, **VARIANTS[prec])
    ref = oracle.solve_qp(Qn, q, A, b, G, h, solver_tol=1e-6)
    np.testing.assert_array_equal(np_(out[4]), ref[4])
    assert_close(out[0], ref[0], X_TOL, "x (forward, raw Q)")
    dl = wl.loss_grad(ref[0])
    _, grads, _, _ = qb.solve_qp_primal_vjp(Qn, q, A, b, G, h, dl, 1e-6, 1e-3, **VARIANTS[prec])
    _, grads_o, _, _ = oracle.solve_qp_primal_vjp(Qs, q, A, b, G, h, dl, solver_tol=1e-6, target_kappa=1e-3)
    for g, go, name in zip(grads, grads_o, ["dQ", "dq", "dA", "db", "dG", "dh"]):
        assert_close(g, go, G_TOL, name)
