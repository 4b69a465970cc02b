"""Differentiable primal solve, mirroring qpax/diff_qp.py.

    x = solve_qp_primal(Q, q, A, b, G, h, solver_tol=1e-5, target_kappa=1e-3)

is a torch.autograd.Function: the forward runs qpb_solve_qp and keeps only
(x, s, z, y); the backward runs qpb_solve_qp_primal_bwd, which relaxes that
iterate to target_kappa (qpax/pdip_relaxed.py) and solves the adjoint KKT
system at the relaxed point (qpax/diff_qp.py:20-46), returning gradients for
Q, q, A, b, G, h -- the same custom_vjp qpax defines (:49-82).
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import as_f64, ptr
from .pdip import StdBatch, _config, _run, solve_qp


class _SolveQPPrimal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Q, q, A, b, G, h, solver_tol, target_kappa, opts):
        bt = StdBatch(Q, q, A, b, G, h)
        cfg = _config(opts)
        x, s, z, y = bt.new(bt.B, bt.n), bt.new(bt.B, bt.p), bt.new(bt.B, bt.p), bt.new(bt.B, bt.m)
        conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
        _run("qpb_solve_qp", "solve", bt, cfg, [ctypes.c_double(solver_tol)],
             [ptr(x), ptr(s), ptr(z), ptr(y), ptr(conv), ptr(iters)])
        ctx.bt = bt
        ctx.opts = opts
        ctx.tols = (solver_tol, target_kappa)
        ctx.save_for_backward(x, s, z, y)
        ctx.shapes = [t.shape for t in (Q, q, A, b, G, h)]
        return x if bt.batched else x[0]

    @staticmethod
    def backward(ctx, gx):
        bt: StdBatch = ctx.bt
        x, s, z, y = ctx.saved_tensors
        g = as_f64(gx, bt.dev).reshape(bt.B, bt.n).contiguous()
        grads = diff_qp_from_forward(bt, x, s, z, y, g, *ctx.tols, ctx.opts)
        out = [gr.reshape(shp) for gr, shp in zip(grads, ctx.shapes)]
        return (*out, None, None, None)


def diff_qp_from_forward(bt: StdBatch, x, s, z, y, gx, solver_tol, target_kappa, opts, relaxed=None):
    """qpb_solve_qp_primal_bwd: relax the forward iterate, then the adjoint solve."""
    cfg = _config(opts)
    dQ, dq, dA = bt.new(bt.B, bt.n, bt.n), bt.new(bt.B, bt.n), bt.new(bt.B, bt.m, bt.n)
    db, dG, dh = bt.new(bt.B, bt.m), bt.new(bt.B, bt.p, bt.n), bt.new(bt.B, bt.p)
    rel = relaxed or [None] * 6
    _run("qpb_solve_qp_primal_bwd", "primal_bwd", bt, cfg,
         [ptr(x), ptr(s), ptr(z), ptr(y), ptr(gx), ctypes.c_double(solver_tol), ctypes.c_double(target_kappa)],
         [ptr(dQ), ptr(dq), ptr(dA), ptr(db), ptr(dG), ptr(dh)] + [ptr(t) for t in rel])
    return dQ, dq, dA, db, dG, dh


def solve_qp_primal(Q, q, A, b, G, h, solver_tol: float = 1e-5, target_kappa: float = 1e-3, *, precision=None,
                    team_threads=None):
    """qpax/diff_qp.py:49 solve_qp_primal: returns x, differentiable in Q, q, A, b, G, h."""
    opts = dict(precision=precision, team_threads=team_threads)
    return _SolveQPPrimal.apply(*[torch.as_tensor(t) for t in (Q, q, A, b, G, h)], solver_tol, target_kappa, opts)


def diff_qp(Q, q, A, b, G, h, x, s, lam, nu, dl_dx, *, precision=None, team_threads=None):
    """qpax/diff_qp.py:20 diff_qp at a given (relaxed) iterate -> (dQ, dq, dA, db, dG, dh)."""
    bt = StdBatch(Q, q, A, b, G, h)
    cfg = _config(dict(precision=precision, team_threads=team_threads))
    its = [as_f64(t, bt.dev).reshape(bt.B, -1).contiguous() for t in (x, s, lam, nu, dl_dx)]
    dQ, dq, dA = bt.new(bt.B, bt.n, bt.n), bt.new(bt.B, bt.n), bt.new(bt.B, bt.m, bt.n)
    db, dG, dh = bt.new(bt.B, bt.m), bt.new(bt.B, bt.p, bt.n), bt.new(bt.B, bt.p)
    _run("qpb_diff_qp", "diff", bt, cfg, [ptr(t) for t in its], [ptr(dQ), ptr(dq), ptr(dA), ptr(db), ptr(dG),
                                                                 ptr(dh)])
    return bt.out(dQ, dq, dA, db, dG, dh)


_STREAMS: dict = {}


def _host_streams(dev, count):
    """Streams of the host pipeline, created once per device and reused (new
    streams per call would defeat the caching allocator's per-stream reuse)."""
    key = (dev.index, count)
    if key not in _STREAMS:
        _STREAMS[key] = [torch.cuda.Stream(device=dev) for _ in range(count)]
    return _STREAMS[key]


def solve_qp_primal_vjp_host(Q, q, A, b, G, h, dl_dx, solver_tol: float = 1e-5, target_kappa: float = 1e-3, *,
                             out=None, chunks: int = 4, streams: int = 3, precision=None):
    """solve_qp_primal_vjp for batches that live in host memory.

    Inputs are CPU tensors with a leading batch axis (pinned memory lets the
    copies overlap); the batch is cut into `chunks`, and on `streams` CUDA
    streams each chunk is copied in, solved forward and backward, and its x
    and six gradients copied back while the next chunk computes.  `out` may
    hold preallocated pinned CPU tensors (x, dQ, dq, dA, db, dG, dh).
    Returns (x, (dQ, dq, dA, db, dG, dh)) on the host; waits for completion.
    """
    dev = _lib.device()
    B = Q.shape[0]
    if out is None:
        pin = torch.cuda.is_available()
        out = [torch.empty(t.shape, dtype=torch.float64, pin_memory=pin) for t in (q, Q, q, A, b, G, h)]
    bounds = [round(i * B / chunks) for i in range(chunks + 1)]
    pool = _host_streams(dev, max(1, streams))
    main = torch.cuda.current_stream(dev)
    for s in pool:
        s.wait_stream(main)
    opts = dict(precision=precision)
    for c in range(chunks):
        lo, hi = bounds[c], bounds[c + 1]
        if hi <= lo:
            continue
        s = pool[c % len(pool)]
        with torch.cuda.stream(s):
            dev_in = [t[lo:hi].to(dev, non_blocking=True) for t in (Q, q, A, b, G, h, dl_dx)]
            x, grads, _, _ = solve_qp_primal_vjp(*dev_in[:6], dev_in[6], solver_tol, target_kappa, **opts)
            for dst, src in zip(out, (x,) + tuple(grads)):
                dst[lo:hi].copy_(src, non_blocking=True)
            for t in dev_in:
                t.record_stream(s)
    for s in pool:
        main.wait_stream(s)
    torch.cuda.synchronize(dev)
    return out[0], tuple(out[1:])


def solve_qp_primal_vjp(Q, q, A, b, G, h, dl_dx, solver_tol: float = 1e-5, target_kappa: float = 1e-3, *,
                        precision=None, team_threads=None):
    """Forward and backward of solve_qp_primal as two launches, without autograd.

    Returns (x, (dQ, dq, dA, db, dG, dh), converged, iters).
    """
    opts = dict(precision=precision, team_threads=team_threads)
    x, s, z, y, conv, iters = solve_qp(Q, q, A, b, G, h, solver_tol, **opts)
    bt = StdBatch(Q, q, A, b, G, h)
    resh = [t.reshape(bt.B, -1) for t in (x, s, z, y)]
    g = as_f64(dl_dx, bt.dev).reshape(bt.B, bt.n).contiguous()
    grads = diff_qp_from_forward(bt, *resh, g, solver_tol, target_kappa, opts)
    return x, bt.out(*grads), conv, iters
