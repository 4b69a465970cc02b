"""Uneven batches (instances of different n, m, p in one call) against the oracle.

Bars as in test_gpu_parity.py: outputs within 1e-6 * max(1, |.|_inf), gradients
within 1e-5, identical converged flags and iteration counts on every instance
where the reference converges.  Also checks that a CUDA-graph replay of the
packed call reproduces the eager call.
"""

import numpy as np
import pytest
import torch

from oracle import oracle
from qpax_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _batch(count=48, seed=9, n_max=80):
    rng = np.random.default_rng(seed)
    ns = rng.integers(4, n_max + 1, size=count)
    data = [[], [], [], [], [], []]
    for n in ns:
        m = int(rng.integers(0, n // 4 + 1))
        inst = wl.dense(1, int(n), m, int(2 * n), rng)
        for k in range(6):
            data[k].append(inst[k][0])
    return data


def _close(gpu_list, ref_list, ok, tol, what):
    for i, (g, r) in enumerate(zip(gpu_list, ref_list)):
        if not ok[i] or np.size(r) == 0:
            continue
        g = g.detach().cpu().numpy().reshape(np.shape(r))
        err = np.abs(g - r).max() / max(1.0, np.abs(r).max())
        assert err <= tol, f"{what}[{i}] err {err:.3e}"


@pytest.mark.parametrize("precision", ["auto", "mixed"])
def test_uneven_solve_matches_oracle(precision):
    from qpax_b200.packed import solve_qp_uneven

    data = _batch()
    xs, ss, zs, ys, conv, iters = solve_qp_uneven(*data, solver_tol=1e-6, precision=precision)
    ref = oracle.solve_qp(*data, solver_tol=1e-6)
    ok = np.asarray(ref[4]) == 1
    assert ok.mean() >= 0.9
    np.testing.assert_array_equal(conv.cpu().numpy()[ok], 1)
    np.testing.assert_array_equal(iters.cpu().numpy()[ok], np.asarray(ref[5])[ok])
    for g, r, name in zip((xs, ss, zs, ys), ref[:4], "xszy"):
        _close(g, r, ok, 1e-6, name)


def test_uneven_backward_matches_oracle():
    from qpax_b200.packed import PackedPlan, pack, unpack

    data = _batch(count=32, seed=10, n_max=48)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    plan = PackedPlan(shapes)
    assert plan.num_bins >= 3
    ins = [pack(v) for v in data]
    x, s, z, y, conv, iters = plan.solve(*ins, 1e-6)
    x_ref = oracle.solve_qp(*data, solver_tol=1e-6)
    dl = [wl.loss_grad(v) for v in x_ref[0]]
    grads = plan.primal_bwd(*ins, x, s, z, y, pack(dl), 1e-6, 1e-3)
    _, grads_o, conv_o, _ = oracle.solve_qp_primal_vjp(*data, dl, solver_tol=1e-6, target_kappa=1e-3)
    ok = np.asarray(conv_o) == 1
    L = plan.lengths
    for k, name in enumerate(["dQ", "dq", "dA", "db", "dG", "dh"]):
        _close(unpack(grads[k], L[k]), grads_o[k], ok, 1e-5, name)


def _small_batch(count, seed):
    """Instances with n <= 8 (the four-per-warp lockstep kernel): n, m, p all
    vary, so the groups of one warp hold different shapes (p >= 1: packed
    batches carry inequalities)."""
    rng = np.random.default_rng(seed)
    data = [[], [], [], [], [], []]
    for i in range(count):
        n = int(rng.integers(1, 9))
        m = int(rng.integers(0, min(2, n - 1) + 1)) if n > 1 else 0
        p = int(rng.integers(1, 21))
        inst = wl.dense(1, n, m, p, rng)
        for k in range(6):
            data[k].append(inst[k][0])
    return data


def test_lockstep_groups_with_mixed_shapes():
    """37 instances with n <= 8 (the last warp partly empty), shapes varying
    within every warp: forward, then forward + backward, vs the oracle."""
    from qpax_b200.packed import PackedPlan, pack, unpack, solve_qp_uneven

    data = _small_batch(37, 21)
    xs, ss, zs, ys, conv, iters = solve_qp_uneven(*data, solver_tol=1e-6)
    ref = oracle.solve_qp(*data, solver_tol=1e-6)
    ok = np.asarray(ref[4]) == 1
    assert ok.mean() >= 0.9
    np.testing.assert_array_equal(conv.cpu().numpy()[ok], 1)
    np.testing.assert_array_equal(iters.cpu().numpy()[ok], np.asarray(ref[5])[ok])
    for g, r, name in zip((xs, ss, zs, ys), ref[:4], "xszy"):
        _close(g, r, ok, 1e-6, name)

    data = _small_batch(37, 22)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    plan = PackedPlan(shapes)
    ins = [pack(v) for v in data]
    x, s, z, y, conv, iters = plan.solve(*ins, 1e-6)
    x_ref = oracle.solve_qp(*data, solver_tol=1e-6)
    dl = [wl.loss_grad(v) for v in x_ref[0]]
    grads = plan.primal_bwd(*ins, x, s, z, y, pack(dl), 1e-6, 1e-3)
    _, grads_o, conv_o, _ = oracle.solve_qp_primal_vjp(*data, dl, solver_tol=1e-6, target_kappa=1e-3)
    ok = np.asarray(conv_o) == 1
    assert ok.mean() >= 0.9
    L = plan.lengths
    for k, name in enumerate(["dQ", "dq", "dA", "db", "dG", "dh"]):
        _close(unpack(grads[k], L[k]), grads_o[k], ok, 1e-5, name)


def test_cuda_graph_replay_matches_eager():
    from qpax_b200.packed import PackedPlan, pack

    data = _batch(count=40, seed=11, n_max=70)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    plan = PackedPlan(shapes)
    ins = [pack(v) for v in data]
    eager = plan.solve(*ins, 1e-6)
    torch.cuda.synchronize()
    outs = [torch.empty_like(t) for t in eager]
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        plan.solve(*ins, 1e-6)  # warm-up on the capture stream
    torch.cuda.current_stream().wait_stream(s)
    with torch.cuda.graph(g):
        res = plan.solve(*ins, 1e-6)
        for o, r in zip(outs, res):
            o.copy_(r)
    g.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager, outs):
        assert torch.equal(a, b)


@pytest.mark.gpu
def test_host_pipeline_matches_device_plan():
    """PackedHostPipeline (host arrays, instance groups overlapped on streams)
    gives exactly the one-plan device-resident result."""
    from qpax_b200.packed import PackedHostPipeline, PackedPlan, pack

    data = _batch(count=20, seed=13, n_max=48)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    host = [pack(v, torch.device("cpu")).pin_memory() for v in data]
    dl = torch.full((host[1].numel(),), 0.1, dtype=torch.float64).pin_memory()
    x_h, g_h = PackedHostPipeline(shapes, chunks=3).run(*host, dl, 1e-6, 1e-3)
    plan = PackedPlan(shapes)
    dev = [t.cuda() for t in host]
    out = plan.solve(*dev, 1e-6)
    grads = plan.primal_bwd(*dev, *out[:4], dl.cuda(), 1e-6, 1e-3)
    torch.testing.assert_close(x_h, out[0].cpu(), rtol=0, atol=0)
    for a, b_ in zip(g_h, grads):
        torch.testing.assert_close(a, b_.cpu(), rtol=0, atol=0)
