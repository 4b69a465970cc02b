"""Parity figures of GPU outputs against the FP64 oracle (test infrastructure).

Used by the GPU tests and by bench.py's parity report (computed outside the
timed region): the oracle is the checker here, never the thing measured.

Per-instance relative error of an array: ||gpu - ref||_inf / max(1, ||ref||_inf).
Objective: 1/2 x'Qx + q'x (elastic: plus penalty * sum(t)), relative the same way.
"""

from __future__ import annotations

import numpy as np

from oracle import oracle


def _rows(a, B):
    if isinstance(a, (list, tuple)):
        return [np.asarray(v, np.float64).reshape(-1) for v in a]
    a = np.asarray(a, np.float64).reshape(B, -1)
    return list(a)


def rel_errors(gpu, ref, B):
    """Per-instance relative inf-norm errors (uniform arrays or ragged lists)."""
    g, r = _rows(gpu, B), _rows(ref, B)
    out = np.zeros(B)
    for i in range(B):
        if r[i].size:
            out[i] = np.abs(g[i] - r[i]).max() / max(1.0, np.abs(r[i]).max())
    return out


def objective(Q, q, x, B):
    Qs, qs, xs = _rows(Q, B), _rows(q, B), _rows(x, B)
    out = np.zeros(B)
    for i in range(B):
        n = qs[i].size
        Qi = Qs[i].reshape(n, n)
        out[i] = 0.5 * xs[i] @ Qi @ xs[i] + qs[i] @ xs[i]
    return out


def _finite_max(v):
    v = np.asarray(v, np.float64)
    return float(v.max()) if v.size else 0.0


def standard(data, tol, kappa, dl, gpu_x, gpu_conv, gpu_iters, gpu_grads, ref=None):
    """Parity of a solve_qp_primal forward + backward against the oracle.

    data: (Q, q, A, b, G, h), uniform arrays or ragged lists; dl: the incoming
    gradient dl/dx both sides were given; gpu_*: numpy.  Returns (figures,
    ref) where ref is the oracle output (reusable for the same data and dl).
    """
    Q, q, A, b, G, h = data
    B = len(q) if isinstance(q, (list, tuple)) else np.asarray(q).shape[0]
    if ref is None:
        x_o, grads_o, conv_o, iters_o = oracle.solve_qp_primal_vjp(*data, dl, solver_tol=tol, target_kappa=kappa)
        ref = dict(x=x_o, grads=grads_o, conv=np.asarray(conv_o), iters=np.asarray(iters_o))
    both = (np.asarray(gpu_conv) == 1) & (ref["conv"] == 1)
    ex = rel_errors(gpu_x, ref["x"], B)
    fo, fg = objective(Q, q, ref["x"], B), objective(Q, q, gpu_x, B)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    eg = np.zeros(B)
    for g, go in zip(gpu_grads, ref["grads"]):
        eg = np.maximum(eg, rel_errors(g, go, B))
    fig = {
        "instances": int(B),
        "compared": int(both.sum()),
        "max_err_x": _finite_max(ex[both]),
        "max_err_obj": _finite_max(eo[both]),
        "max_err_grad": _finite_max(eg[both]),
        "conv_mismatch": int((np.asarray(gpu_conv) != ref["conv"]).sum()),
        "iters_mismatch": int((np.asarray(gpu_iters) != ref["iters"]).sum()),
        "reference_not_converged": int((ref["conv"] != 1).sum()),
    }
    return fig, ref


def elastic(data, penalty, tol, kappa, dl, gpu_out, gpu_grads, ref=None):
    """Parity of solve_qp_elastic_primal forward + backward: x and the slacks
    (t, s1, s2) as the elastic configuration compares them, the objective
    (with the penalty term) and the four gradients, for incoming gradient dl."""
    Q, q, G, h = data
    B = np.asarray(q).shape[0]
    if ref is None:
        out = oracle.solve_qp_elastic(Q, q, G, h, penalty, solver_tol=tol)
        _, grads_o = oracle.solve_qp_elastic_primal_vjp(Q, q, G, h, penalty, dl, solver_tol=tol, target_kappa=kappa)
        ref = dict(out=out, grads=grads_o, conv=np.asarray(out[6]), iters=np.asarray(out[7]))
    gconv = np.asarray(gpu_out[6])
    both = (gconv == 1) & (ref["conv"] == 1)
    ex = np.zeros(B)
    for k in range(4):  # x, t, s1, s2
        ex = np.maximum(ex, rel_errors(gpu_out[k], ref["out"][k], B))
    pen = np.broadcast_to(np.asarray(penalty, np.float64).reshape(-1), (B,))
    fo = objective(Q, q, ref["out"][0], B) + pen * np.asarray(ref["out"][1]).sum(axis=1)
    fg = objective(Q, q, gpu_out[0], B) + pen * np.asarray(gpu_out[1]).sum(axis=1)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    eg = np.zeros(B)
    for g, go in zip(gpu_grads, ref["grads"]):
        eg = np.maximum(eg, rel_errors(g, go, B))
    fig = {
        "instances": int(B),
        "compared": int(both.sum()),
        "max_err_x": _finite_max(ex[both]),
        "max_err_obj": _finite_max(eo[both]),
        "max_err_grad": _finite_max(eg[both]),
        "conv_mismatch": int((gconv != ref["conv"]).sum()),
        "iters_mismatch": int((np.asarray(gpu_out[7]) != ref["iters"]).sum()),
        "reference_not_converged": int((ref["conv"] != 1).sum()),
    }
    return fig, ref
