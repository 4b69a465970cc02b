"""Parity figures of GPU outputs against the FP64 oracle (test infrastructure).

Used by the GPU tests and by bench.py's parity report (computed outside the
timed region): the oracle is the checker here, never the thing measured.

Per-instance relative error of an array: ||gpu - ref||_inf / max(1, ||ref||_inf).
Objective: 1/2 x'Qx + q'x (elastic: plus penalty * sum(t)), relative the same way.

Reproducibility of the reference.  On ill-conditioned instances qpax's own
FP64 method decides its outcome by rounding: its residual reaches ~tol late
in the loop, where the reduced KKT matrix has cond ~1e14 and beyond, and
whether one more step lands below tol is a coin flip.  Run on inputs
perturbed at the rounding level (relative 1e-15, symmetric in Q), the oracle
itself then changes its converged flag or iteration count, and (in qpax's
elastic relaxation, which runs to its iteration cap) its output by up to
1e-2.  With `perturb=K`, the figures include that spread over K perturbed
runs, and the mismatch counts restricted to the instances whose reference
outcome is reproducible: same flag and iteration count in every perturbed
run, and for gradients a spread below a tenth of the gradient bar.
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


def perturb_inputs(data, eps, seed):
    """Copies of (Q, q, A, b, G, h) or (Q, q, G, h) with every entry scaled by
    (1 + eps N(0, 1)); Q's perturbation is symmetric."""
    rng = np.random.default_rng(seed)

    def one(a, sym=False):
        a = np.asarray(a, np.float64)
        e = rng.standard_normal(a.shape)
        if sym:
            e = 0.5 * (e + np.swapaxes(e, -1, -2))
        return a * (1.0 + eps * e)

    out = []
    for k, v in enumerate(data):
        if isinstance(v, (list, tuple)):
            out.append([one(a, sym=(k == 0)) for a in v])
        else:
            out.append(one(v, sym=(k == 0)))
    return out


def _spread(ref, runs, B, key):
    sp = np.zeros(B)
    for r in runs:
        if key == "grads":
            for g, go in zip(r["grads"], ref["grads"]):
                sp = np.maximum(sp, rel_errors(g, go, B))
        else:
            sp = np.maximum(sp, rel_errors(r[key], ref[key], B))
    return sp


def _figures(B, gpu_conv, gpu_iters, ex, eo, eg, ref, g_bar):
    gpu_conv, gpu_iters = np.asarray(gpu_conv), np.asarray(gpu_iters)
    both = (gpu_conv == 1) & (ref["conv"] == 1)
    fig = {
        "instances": int(B),
        "compared": int(both.sum()),
        "max_err_x": _finite_max(ex[both]),
        "max_err_obj": _finite_max(eo[both]),
        "max_err_grad": _finite_max(eg[both]),
        "conv_mismatch": int((gpu_conv != ref["conv"]).sum()),
        "iters_mismatch": int((gpu_iters != ref["iters"]).sum()),
        "reference_not_converged": int((ref["conv"] != 1).sum()),
    }
    if "stable" in ref:
        st, gst = ref["stable"], ref["grad_stable"]
        fig.update({
            "reference_outcome_not_reproducible": int((~st).sum()),
            "conv_mismatch_reproducible": int(((gpu_conv != ref["conv"]) & st).sum()),
            "iters_mismatch_reproducible": int(((gpu_iters != ref["iters"]) & st).sum()),
            "reference_grad_not_reproducible": int((both & ~gst).sum()),
            "max_err_grad_reproducible": _finite_max(eg[both & gst]),
            "reference_perturbed_runs": int(ref["perturbed_runs"]),
        })
    return fig


def forward(data, tol, gpu_x, gpu_conv, gpu_iters, perturb=2):
    """Parity of a solve_qp forward alone (figures as standard(), without
    gradients): x and the objective where both converged, converged flags and
    iteration counts where the reference outcome is reproducible."""
    Q, q, A, b, G, h = data
    B = len(q) if isinstance(q, (list, tuple)) else np.asarray(q).shape[0]

    def run(d):
        out = oracle.solve_qp(*d, solver_tol=tol)
        return dict(x=out[0], conv=np.asarray(out[4]), iters=np.asarray(out[5]))

    ref = run(data)
    runs = [run(perturb_inputs(data, 1e-15, 3000 + k)) for k in range(perturb)]
    ref["stable"] = np.all([(r["conv"] == ref["conv"]) & (r["iters"] == ref["iters"]) for r in runs], axis=0)
    ref["grad_stable"] = ref["stable"]
    ref["perturbed_runs"] = perturb
    ex = rel_errors(gpu_x, ref["x"], B)
    fo, fg = objective(Q, q, ref["x"], B), objective(Q, q, gpu_x, B)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    return _figures(B, gpu_conv, gpu_iters, ex, eo, np.zeros(B), ref, 1e-5)


def standard(data, tol, kappa, dl, gpu_x, gpu_conv, gpu_iters, gpu_grads, ref=None, perturb=0, g_bar=1e-5):
    """Parity of a solve_qp_primal forward + backward against the oracle.

    data: (Q, q, A, b, G, h), uniform arrays or ragged lists; dl: the incoming
    gradient dl/dx both sides were given; gpu_*: numpy.  Returns (figures,
    ref) where ref is the oracle output (reusable for the same data and dl).
    """
    Q, q, A, b, G, h = data
    B = len(q) if isinstance(q, (list, tuple)) else np.asarray(q).shape[0]

    def run(d):
        x, grads, conv, iters = oracle.solve_qp_primal_vjp(*d, dl, solver_tol=tol, target_kappa=kappa)
        return dict(x=x, grads=grads, conv=np.asarray(conv), iters=np.asarray(iters))

    if ref is None:
        ref = run(data)
    if perturb and "stable" not in ref:
        runs = [run(perturb_inputs(data, 1e-15, 1000 + k)) for k in range(perturb)]
        ref["stable"] = np.all([(r["conv"] == ref["conv"]) & (r["iters"] == ref["iters"]) for r in runs], axis=0)
        ref["grad_stable"] = ref["stable"] & (_spread(ref, runs, B, "grads") <= 0.1 * g_bar)
        ref["perturbed_runs"] = perturb
    ex = rel_errors(gpu_x, ref["x"], B)
    fo, fg = objective(Q, q, ref["x"], B), objective(Q, q, gpu_x, B)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    eg = np.zeros(B)
    for g, go in zip(gpu_grads, ref["grads"]):
        eg = np.maximum(eg, rel_errors(g, go, B))
    return _figures(B, gpu_conv, gpu_iters, ex, eo, eg, ref, g_bar), ref


def elastic(data, penalty, tol, kappa, dl, gpu_out, gpu_grads, ref=None, perturb=0, g_bar=1e-5):
    """Parity of solve_qp_elastic_primal forward + backward: x and the slacks
    (t, s1, s2) as the elastic configuration compares them, the objective
    (with the penalty term) and the four gradients, for incoming gradient dl."""
    Q, q, G, h = data
    B = np.asarray(q).shape[0]

    def run(d):
        out = oracle.solve_qp_elastic(*d, penalty, solver_tol=tol)
        _, grads = oracle.solve_qp_elastic_primal_vjp(*d, penalty, dl, solver_tol=tol, target_kappa=kappa)
        return dict(out=out, grads=grads, conv=np.asarray(out[6]), iters=np.asarray(out[7]))

    if ref is None:
        ref = run(data)
    if perturb and "stable" not in ref:
        runs = [run(perturb_inputs(data, 1e-15, 2000 + k)) for k in range(perturb)]
        ref["stable"] = np.all([(r["conv"] == ref["conv"]) & (r["iters"] == ref["iters"]) for r in runs], axis=0)
        ref["grad_stable"] = ref["stable"] & (_spread(ref, runs, B, "grads") <= 0.1 * g_bar)
        ref["perturbed_runs"] = perturb
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
    return _figures(B, gpu_out[6], gpu_out[7], ex, eo, eg, ref, g_bar), ref
