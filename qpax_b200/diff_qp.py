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
import threading

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
        # each gradient goes back with its input's shape, device and dtype
        # (inputs may live on the host or another GPU: they are copied here)
        ctx.metas = [(t.shape, t.device, t.dtype) for t in (Q, q, A, b, G, h)]
        return x if bt.batched else x[0]

    @staticmethod
    def backward(ctx, gx):
        bt: StdBatch = ctx.bt
        x, s, z, y = ctx.saved_tensors
        g = as_f64(gx, bt.dev).reshape(bt.B, bt.n).contiguous()
        grads = diff_qp_from_forward(bt, x, s, z, y, g, *ctx.tols, ctx.opts)
        out = [gr.reshape(shp).to(device=dev, dtype=dt) for gr, (shp, dev, dt) in zip(grads, ctx.metas)]
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
    its = [_lib.rows(t, bt.dev, bt.B, w, nm) for t, w, nm in
           zip((x, s, lam, nu, dl_dx), (bt.n, bt.p, bt.p, bt.m, bt.n), ("x", "s", "lam", "nu", "dl_dx"))]
    dQ, dq, dA = bt.new(bt.B, bt.n, bt.n), bt.new(bt.B, bt.n), bt.new(bt.B, bt.m, bt.n)
    db, dG, dh = bt.new(bt.B, bt.m), bt.new(bt.B, bt.p, bt.n), bt.new(bt.B, bt.p)
    _run("qpb_diff_qp", "diff", bt, cfg, [ptr(t) for t in its], [ptr(dQ), ptr(dq), ptr(dA), ptr(db), ptr(dG),
                                                                 ptr(dh)])
    return bt.out(dQ, dq, dA, db, dG, dh)


_HOST_WS: dict = {}
_HOST_LOCK = threading.Lock()


def host_buffers(Q, q, A, b, G, h, dl_dx, out=None):
    """Checked host tensors for the host-buffer pipeline.

    Returns the seven inputs as contiguous CPU float64 tensors with a leading
    batch axis, Q (B, n, n), q (B, n), A (B, m, n), b (B, m), G (B, p, n),
    h (B, p), dl_dx (B, n), and the seven outputs x, dQ, dq, dA, db, dG, dh
    (`out`, checked, or new tensors, pinned when a device is present).  The
    pipeline copies exactly these sizes between host and device, so a buffer
    of another size or layout is refused here rather than read or written
    past its end."""
    ins = [torch.as_tensor(t, dtype=torch.float64) for t in (Q, q, A, b, G, h, dl_dx)]
    if any(t.device.type != "cpu" for t in ins):
        raise ValueError("solve_qp_primal_vjp_host takes host (CPU) tensors")
    Qh, _, Ah, _, Gh, _, _ = ins
    if Qh.dim() != 3 or Ah.dim() != 3 or Gh.dim() != 3:
        raise ValueError("solve_qp_primal_vjp_host takes batched inputs: Q (B, n, n), A (B, m, n), G (B, p, n)")
    B, n, m, p = Qh.shape[0], Qh.shape[-1], Ah.shape[-2], Gh.shape[-2]
    want = [(B, n, n), (B, n), (B, m, n), (B, m), (B, p, n), (B, p), (B, n)]
    for name, t, w in zip(("Q", "q", "A", "b", "G", "h", "dl_dx"), ins, want):
        if tuple(t.shape) != w:
            raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {w}")
    ins = [t.contiguous() for t in ins]
    oshapes = [want[1], want[0], want[1], want[2], want[3], want[4], want[5]]
    if out is None:
        pin = torch.cuda.is_available()
        out = [torch.empty(w, dtype=torch.float64, pin_memory=pin) for w in oshapes]
    else:
        out = list(out)
        if len(out) != 7:
            raise ValueError("out holds (x, dQ, dq, dA, db, dG, dh): 7 tensors")
        for name, t, w in zip(("x", "dQ", "dq", "dA", "db", "dG", "dh"), out, oshapes):
            if (not isinstance(t, torch.Tensor) or t.device.type != "cpu" or t.dtype != torch.float64
                    or tuple(t.shape) != w or not t.is_contiguous()):
                got = (f"{t.dtype} {tuple(t.shape)} on {t.device}" if isinstance(t, torch.Tensor)
                       else type(t).__name__)
                raise ValueError(f"out {name}: expected a contiguous CPU float64 tensor of shape {w}, got {got}")
    return ins, out


def _host_workspace(dev, nbytes):
    """Device workspace of the host-buffer pipeline, kept per device and grown
    on demand (allocating per call would serialize on the allocator)."""
    ws = _HOST_WS.get(dev.index)
    if ws is None or ws.numel() < nbytes + 256:
        ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
        _HOST_WS[dev.index] = ws
    return ws


def solve_qp_primal_vjp_host(Q, q, A, b, G, h, dl_dx, solver_tol: float = 1e-5, target_kappa: float = 1e-3, *,
                             out=None, chunks: int = 4, precision=None, team_threads=None):
    """solve_qp_primal_vjp for batches that live in host memory.

    Inputs are CPU float64 tensors (or arrays) with a leading batch axis;
    pinned memory lets the copies overlap the kernels.  One call of
    qpb_solve_qp_primal_vjp_host: the batch is cut into `chunks`, and each
    chunk is copied in, solved forward and backward, and its x and six
    gradients copied back while other chunks compute.  `out` may hold
    preallocated (pinned) CPU tensors (x, dQ, dq, dA, db, dG, dh).
    Returns (x, (dQ, dq, dA, db, dG, dh)) on the host; waits for completion.
    """
    dev = _lib.device()
    ins, out = host_buffers(Q, q, A, b, G, h, dl_dx, out)
    Qh, qh, Ah, bh, Gh, hh, gh = ins
    B, n, m, p = Qh.shape[0], Qh.shape[-1], Ah.shape[-2], Gh.shape[-2]
    dims = _lib.Dims(B, n, m, p)
    cfg = _config(dict(precision=precision, team_threads=team_threads))
    lib = _lib.load()
    chunks = max(1, min(int(chunks), max(B, 1)))
    need = lib.qpb_solve_qp_primal_vjp_host_workspace_size(ctypes.byref(dims), chunks, ctypes.byref(cfg))
    if need == 0:
        raise _lib.QpbError(f"unsupported problem for the host pipeline: batch={B} n={n} m={m} p={p}")
    stream = torch.cuda.current_stream(dev)
    # one cached workspace per device: calls from several threads take turns
    # (each call waits for its own completion, so the turns are short-lived)
    with _HOST_LOCK:
        wp, wb = _lib.aligned(_host_workspace(dev, need))
        _lib.call("qpb_solve_qp_primal_vjp_host", ctypes.byref(dims), *[ptr(t) for t in ins],
                  ctypes.c_double(solver_tol), ctypes.c_double(target_kappa), *[ptr(t) for t in out], None, None,
                  chunks, ctypes.byref(cfg), wp, wb, stream.cuda_stream)
        stream.synchronize()
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
