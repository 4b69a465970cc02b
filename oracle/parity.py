"""Parity figures of GPU outputs against the FP64 oracle (test infrastructure).

Used by the GPU tests and by bench.py's parity report (computed outside the
timed region): the oracle is the checker here, never the thing measured.

Per-instance relative error of an array: ||gpu - ref||_inf / max(1, ||ref||_inf).
Objective: 1/2 x'Qx + q'x (elastic: plus penalty * sum(t)), relative the same way.

Converged flags.  On ill-conditioned instances (n >= ~90 in the uneven
configuration, some elastic instances) qpax's QR-based reduced solve breaks
down late in the loop (cond of the reduced KKT matrix 1e14 and beyond): its
residual stalls or grows and the loop runs to its 30-iteration cap.  The
GPU's LDL^T-based solve often converges there.  The figures therefore split
flag mismatches by direction: `gpu_only_converged` instances are checked by
the KKT residual of the GPU's returned iterate (`gpu_only_max_kkt`; the flag
refers to the iterate before qpax's final step, as in qpax), and
`reference_only_converged` instances are GPU failures.

Gradients.  The backward pass differentiates the relaxed point, and the
relaxation stops at the first iterate whose residual is below tol; where that
residual lands within rounding of tol the two sides stop one iteration apart
and differentiate different points (the gradient then differs at the 1e-4
level).  Gradients are compared where the relaxation took the same number of
iterations on both sides (`relax_iters_mismatch_both_converged` counts the
others).

Reproducibility of the reference.  Where the outcome is decided by rounding,
the oracle itself changes its flag or iteration count when its inputs are
perturbed at the rounding level (relative eps, symmetric in Q); qpax's
elastic relaxation, which runs to its iteration cap, moves its output by up
to 1e-2.  With `perturb=K`, K such runs mark the instances whose reference
outcome is reproducible (same flag and iteration count in every run; for
gradients, a spread below a tenth of the gradient bar), and the `_reproducible`
counts are restricted to them.  eps is 1e-15 for FP64 arithmetic; a variant
whose solves are refined to 1e-12 is held to the spread at 1e-12.
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


def kkt_standard(data, x, s, z, y):
    """Per-instance inf-norm of qpax's residuals r1..r4 (pdip.py:93-100) at
    (x, s, z, y), with Q symmetrized as solve_qp does; rows with h = inf are
    dropped."""
    Q, q, A, b, G, h = data
    B = len(q) if isinstance(q, (list, tuple)) else np.asarray(q).shape[0]
    rows = lambda a: _rows(a, B)
    Qs, qs, As, bs, Gs, hs = (rows(v) for v in (Q, q, A, b, G, h))
    xs, ss, zs, ys = rows(x), rows(s), rows(z), rows(y)
    out = np.zeros(B)
    for i in range(B):
        n, m, p = qs[i].size, bs[i].size, hs[i].size
        Qi, Ai, Gi = Qs[i].reshape(n, n), As[i].reshape(m, n), Gs[i].reshape(p, n)
        fin = np.isfinite(hs[i])
        Gi, hi, si, zi = Gi[fin], hs[i][fin], ss[i][fin], zs[i][fin]
        r = [0.5 * (Qi + Qi.T) @ xs[i] + qs[i] + Ai.T @ ys[i] + Gi.T @ zi, si * zi, Gi @ xs[i] + si - hi,
             Ai @ xs[i] - bs[i]]
        out[i] = max((np.abs(v).max() if v.size else 0.0) for v in r)
    return out


def kkt_elastic(data, penalty, x, t, s1, s2, z1, z2):
    """Per-instance inf-norm of qpax's elastic residuals r1..r6
    (elastic_qp.py:105-110)."""
    Q, q, G, h = (np.asarray(v, np.float64) for v in data)
    B = q.shape[0]
    pen = np.broadcast_to(np.asarray(penalty, np.float64).reshape(-1), (B,))
    out = np.zeros(B)
    for i in range(B):
        r = [Q[i] @ x[i] + q[i] + G[i].T @ z2[i], -z1[i] - z2[i] + pen[i], s1[i] * z1[i], s2[i] * z2[i],
             -t[i] + s1[i], G[i] @ x[i] - t[i] + s2[i] - h[i]]
        out[i] = max(np.abs(v).max() for v in r)
    return out


def _figures(B, gpu, ref, ex, eo, eg, gpu_kkt):
    gconv, giters = np.asarray(gpu["conv"]), np.asarray(gpu["iters"])
    rconv = ref["conv"]
    both = (gconv == 1) & (rconv == 1)
    gpu_only = (gconv == 1) & (rconv != 1)
    ref_only = (gconv != 1) & (rconv == 1)
    fig = {
        "instances": int(B),
        "compared": int(both.sum()),
        "max_err_x": _finite_max(ex[both]),
        "max_err_obj": _finite_max(eo[both]),
        "max_err_grad": _finite_max(eg[both]),
        "conv_mismatch": int((gconv != rconv).sum()),
        "gpu_only_converged": int(gpu_only.sum()),
        "gpu_only_max_kkt": _finite_max(gpu_kkt[gpu_only]),
        "reference_only_converged": int(ref_only.sum()),
        "iters_mismatch_both_converged": int((both & (giters != ref["iters"])).sum()),
        "reference_not_converged": int((rconv != 1).sum()),
    }
    same_relax = np.ones(B, bool)
    if "riters" in gpu and "riters" in ref:
        same_relax = np.asarray(gpu["riters"]) == ref["riters"]
        fig["relax_iters_mismatch_both_converged"] = int((both & ~same_relax).sum())
    if "stable" in ref:
        st, gst = ref["stable"], ref["grad_stable"] & same_relax
        fig.update({
            "reference_outcome_not_reproducible": int((~st).sum()),
            "reference_only_converged_reproducible": int((ref_only & st).sum()),
            "iters_mismatch_both_converged_reproducible": int((both & st & (giters != ref["iters"])).sum()),
            "reference_grad_not_reproducible": int((both & ~gst).sum()),
            "max_err_grad_reproducible": _finite_max(eg[both & gst]),
            "reference_perturbed_runs": int(ref["perturbed_runs"]),
            "reference_perturbation": float(ref["perturbation"]),
        })
    return fig


def _stability(ref, runs, B, g_bar, eps, grads=True):
    ref["stable"] = np.all([(r["conv"] == ref["conv"]) & (r["iters"] == ref["iters"]) for r in runs], axis=0)
    ref["grad_stable"] = ref["stable"] & (_spread(ref, runs, B, "grads") <= 0.1 * g_bar) if grads else ref["stable"]
    ref["perturbed_runs"] = len(runs)
    ref["perturbation"] = eps


def forward(data, tol, gpu, perturb=2, eps=1e-15):
    """Parity of a solve_qp forward alone.  gpu: dict of numpy x, s, z, y,
    conv, iters (uniform arrays or ragged lists)."""
    Q, q, A, b, G, h = data
    B = len(q) if isinstance(q, (list, tuple)) else np.asarray(q).shape[0]

    def run(d):
        out = oracle.solve_qp(*d, solver_tol=tol)
        return dict(x=out[0], conv=np.asarray(out[4]), iters=np.asarray(out[5]))

    ref = run(data)
    if perturb:
        _stability(ref, [run(perturb_inputs(data, eps, 3000 + k)) for k in range(perturb)], B, 1e-5, eps, False)
    ex = rel_errors(gpu["x"], ref["x"], B)
    fo, fg = objective(Q, q, ref["x"], B), objective(Q, q, gpu["x"], B)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    kk = kkt_standard(data, gpu["x"], gpu["s"], gpu["z"], gpu["y"])
    return _figures(B, gpu, ref, ex, eo, np.zeros(B), kk)


def standard(data, tol, kappa, dl, gpu, ref=None, perturb=0, eps=1e-15, g_bar=1e-5):
    """Parity of a solve_qp_primal forward + backward against the oracle.

    data: (Q, q, A, b, G, h), uniform arrays or ragged lists; dl: the incoming
    gradient dl/dx both sides were given; gpu: dict of numpy x, s, z, y,
    conv, iters and grads (the six gradients).  Returns (figures, ref) where
    ref is the oracle output (reusable for the same data, dl and eps).
    """
    Q, q, A, b, G, h = data
    B = len(q) if isinstance(q, (list, tuple)) else np.asarray(q).shape[0]

    def run(d):
        x, grads, conv, iters = oracle.solve_qp_primal_vjp(*d, dl, solver_tol=tol, target_kappa=kappa)
        return dict(x=x, grads=grads, conv=np.asarray(conv), iters=np.asarray(iters))

    if ref is None:
        ref = run(data)
        fw = oracle.solve_qp(*data, solver_tol=tol)
        ref["riters"] = np.asarray(oracle.relax_qp(*data, *fw[:4], solver_tol=tol, target_kappa=kappa)[5])
    if perturb and ref.get("perturbation") != eps:
        _stability(ref, [run(perturb_inputs(data, eps, 1000 + k)) for k in range(perturb)], B, g_bar, eps)
    ex = rel_errors(gpu["x"], ref["x"], B)
    fo, fg = objective(Q, q, ref["x"], B), objective(Q, q, gpu["x"], B)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    eg = np.zeros(B)
    for g, go in zip(gpu["grads"], ref["grads"]):
        eg = np.maximum(eg, rel_errors(g, go, B))
    kk = kkt_standard(data, gpu["x"], gpu["s"], gpu["z"], gpu["y"])
    return _figures(B, gpu, ref, ex, eo, eg, kk), ref


def elastic(data, penalty, tol, kappa, dl, gpu_out, gpu_grads, ref=None, perturb=0, eps=1e-15, g_bar=1e-5):
    """Parity of solve_qp_elastic_primal forward + backward: x and the slacks
    (t, s1, s2) as the elastic configuration compares them, the objective
    (with the penalty term) and the four gradients, for incoming gradient dl.
    gpu_out: numpy (x, t, s1, s2, z1, z2, converged, iters)."""
    Q, q, G, h = data
    B = np.asarray(q).shape[0]

    def run(d):
        out = oracle.solve_qp_elastic(*d, penalty, solver_tol=tol)
        _, grads = oracle.solve_qp_elastic_primal_vjp(*d, penalty, dl, solver_tol=tol, target_kappa=kappa)
        return dict(out=out, grads=grads, conv=np.asarray(out[6]), iters=np.asarray(out[7]))

    if ref is None:
        ref = run(data)
    if perturb and ref.get("perturbation") != eps:
        _stability(ref, [run(perturb_inputs(data, eps, 2000 + k)) for k in range(perturb)], B, g_bar, eps)
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
    kk = kkt_elastic(data, penalty, *gpu_out[:6])
    gpu = {"conv": gpu_out[6], "iters": gpu_out[7]}
    return _figures(B, gpu, ref, ex, eo, eg, kk), ref


def elastic_forward(data, penalty, tol, gpu_out, perturb=2, eps=1e-15):
    """Parity of a solve_qp_elastic forward alone (x, t, s1, s2, flags)."""
    Q, q, G, h = data
    B = np.asarray(q).shape[0]

    def run(d):
        out = oracle.solve_qp_elastic(*d, penalty, solver_tol=tol)
        return dict(out=out, conv=np.asarray(out[6]), iters=np.asarray(out[7]))

    ref = run(data)
    if perturb:
        _stability(ref, [run(perturb_inputs(data, eps, 4000 + k)) for k in range(perturb)], B, 1e-5, eps, False)
    ex = np.zeros(B)
    for k in range(4):
        ex = np.maximum(ex, rel_errors(gpu_out[k], ref["out"][k], B))
    pen = np.broadcast_to(np.asarray(penalty, np.float64).reshape(-1), (B,))
    fo = objective(Q, q, ref["out"][0], B) + pen * np.asarray(ref["out"][1]).sum(axis=1)
    fg = objective(Q, q, gpu_out[0], B) + pen * np.asarray(gpu_out[1]).sum(axis=1)
    eo = np.abs(fg - fo) / np.maximum(1.0, np.abs(fo))
    kk = kkt_elastic(data, penalty, *gpu_out[:6])
    return _figures(B, {"conv": gpu_out[6], "iters": gpu_out[7]}, ref, ex, eo, np.zeros(B), kk)
