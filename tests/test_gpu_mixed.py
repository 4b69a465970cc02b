"""GPU: the mixed-precision one-warp path and its hand-over to the FP64 warp kernel.

For n <= 32 (m <= n_pad/4) precision="mixed" runs two launches:
  1. the mixed kernel, with an FP32 factor and FP64 refinement;
  2. the FP64 warp kernel, which resumes every instance whose FP32 factor was
     rejected (pivot ratio above 1e7, or a stalled refinement).
Each resumed instance starts from the iterate, iteration count and stage it
left in the workspace.  These tests make the hand-over happen at each stage
where it can:
  * at the initial point, when the FP32 factor of the first reduced matrix is
    rejected.  The FP64 kernel then solves the instance from scratch, so its
    outputs equal the FP64 path's bit for bit (checked against that path);
  * inside the loop.  The dense instances all hand over before they converge;
    they are checked against the oracle;
  * in the relaxation.  Started at the forward's solution, where cond(H) is
    about 1e14, the first factor is rejected.  Started at an early iterate,
    FP32 factors serve for a while and are then rejected.  Both are checked
    against the oracle.
Bars against the oracle as in test_gpu_parity: x, s, z, y within
1e-6 * max(1, |ref|), identical converged flags (and iteration counts for the
forward solve).
"""

import numpy as np
import pytest
import torch

from oracle import oracle
from qpax_b200 import workloads as wl

pytestmark = pytest.mark.gpu
X_TOL = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from qpax_b200 import _lib as L

    L.load()


def np_(t):
    return t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)


def assert_close(gpu, ref, tol, what):
    g, r = np_(gpu), np.asarray(ref)
    B = r.shape[0]
    g, r = g.reshape(B, -1), r.reshape(B, -1)
    if r.shape[1] == 0:
        return
    e = np.abs(g - r).max(axis=1) / np.maximum(1.0, np.abs(r).max(axis=1))
    assert (e <= tol).all(), f"{what}: worst {e.max():.3e}"


def scaled_variable(B, n, m, p, seed, scale=2.0 ** -13):
    """Dense QPs with variable 0 rescaled by a power of two.  x_0 = scale *
    x~_0 turns Q into D^-1 Q D^-1, and q, A, G likewise.  That multiplies
    the pivot ratio of the reduced matrix by 2^26 (6.7e7; at least 7.6e7 on
    these inputs, checked on the CPU), so the FP32 factor is rejected from
    the initial point on."""
    Q, q, A, b, G, h = wl.dense(B, n, m, p, seed)
    d = np.ones(n)
    d[0] = 1.0 / scale
    Q = Q * d[None, :, None] * d[None, None, :]
    q = q * d[None, :]
    A = A * d[None, None, :]
    G = G * d[None, None, :]
    return Q, q, A, b, G, h


@pytest.mark.parametrize("shape", [(12, 3, 24), (32, 8, 64)])
def test_hand_over_at_initial_point_equals_fp64_path(shape):
    """Outputs equal the FP64 path's bit for bit: the FP64 kernel solved
    every instance from its initial point.  (They are not held to the oracle
    here: the rescaled reduced matrices are conditioned so that LDL^T and
    qpax's QR end some instances an iteration or two apart, measured on the
    FP64 path itself; the FP64 path's parity is pinned on the unscaled
    problems in test_gpu_parity.)"""
    import qpax_b200 as qb

    n, m, p = shape
    data = scaled_variable(48, n, m, p, 71)
    stats = torch.zeros(48, 4, dtype=torch.int32, device="cuda")
    mixed = qb.solve_qp(*data, 1e-6, precision="mixed", stats=stats)
    fp64 = qb.solve_qp(*data, 1e-6, precision="fp64", team_threads=32)  # the resume launch's kernel
    st = np_(stats)
    assert (st[:, 0] == 0).all(), "an FP32 factor was accepted"
    assert ((st[:, 3] & 1) != 0).all(), "the FP32 rejection flag is missing"
    for a, b_, name in zip(mixed, fp64, ["x", "s", "z", "y", "converged", "iters"]):
        np.testing.assert_array_equal(np_(a), np_(b_), err_msg=name)


@pytest.mark.parametrize("shape", [(12, 3, 24), (32, 8, 64)])
def test_hand_over_inside_the_loop(shape):
    import qpax_b200 as qb

    n, m, p = shape
    data = wl.dense(64, n, m, p, 72)
    stats = torch.zeros(64, 4, dtype=torch.int32, device="cuda")
    out = qb.solve_qp(*data, 1e-6, precision="mixed", stats=stats)
    st = np_(stats)
    assert (st[:, 0] > 0).all() and (st[:, 1] > 0).any(), "no FP32 phase, or no hand-over"
    ref = oracle.solve_qp(*data, solver_tol=1e-6)
    np.testing.assert_array_equal(np_(out[4]), np.atleast_1d(ref[4]), err_msg="converged flags")
    np.testing.assert_array_equal(np_(out[5]), np.atleast_1d(ref[5]), err_msg="iteration counts")
    for k, name in enumerate("xszy"):
        assert_close(out[k], ref[k], X_TOL, name)


@pytest.mark.parametrize("start_tol", [1e-6, 1e-1])
def test_relaxation_hands_over(start_tol):
    """relax_qp in mixed precision from the oracle's iterate at start_tol.
    From the solution (1e-6) the first FP32 factor is rejected.  From an
    early iterate (1e-1) FP32 factors serve some steps first."""
    import qpax_b200 as qb

    data = wl.dense(64, 32, 8, 64, 73)
    x, s, z, y, _, _ = oracle.solve_qp(*data, solver_tol=start_tol)
    stats = torch.zeros(64, 4, dtype=torch.int32, device="cuda")
    out = qb.relax_qp(*data, x, s, z, y, 1e-6, 1e-3, precision="mixed", stats=stats)
    ref = oracle.relax_qp(*data, x, s, z, y, solver_tol=1e-6, target_kappa=1e-3)
    st = np_(stats)
    if start_tol == 1e-1:
        assert st[:, 0].sum() > 0, "no FP32 factor served the relaxation"
    np.testing.assert_array_equal(np_(out[4]), np.atleast_1d(ref[4]), err_msg="converged flags")
    for k, name in enumerate("xszy"):
        assert_close(out[k], ref[k], X_TOL, name)
