"""Elastic QP on the GPU, mirroring qpax/elastic_qp.py.

    x, t, s1, s2, z1, z2, converged, iters = solve_qp_elastic(Q, q, G, h, penalty, solver_tol=1e-3)
    x = solve_qp_elastic_primal(Q, q, G, h, penalty, solver_tol=1e-5, target_kappa=1e-3)

Gx <= h is softened with slacks t >= 0 priced at `penalty` (qpax/elastic_qp.py
:184-228); solve_qp_elastic_primal is differentiable in Q, q, G, h through a
relax + adjoint backward (qpax/elastic_qp.py:420-469).  `penalty` is a scalar
or one value per instance.  Batching and device rules as in qpax_b200.pdip.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import Dims, as_f64, ptr
from .pdip import _config


class ElasticBatch:
    def __init__(self, Q, q, G, h, penalty):
        dev = _lib.device()
        Q, q, G, h = (as_f64(t, dev) for t in (Q, q, G, h))
        self.batched = Q.dim() == 3
        if not self.batched:
            Q, q, G, h = Q[None], q[None], G[None], h[None]
        B, n, p = Q.shape[0], Q.shape[-1], G.shape[-2]
        want = {"Q": (B, n, n), "q": (B, n), "G": (B, p, n), "h": (B, p)}
        for name, t in zip("Q q G h".split(), (Q, q, G, h)):
            if tuple(t.shape) != want[name]:
                raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {want[name]}")
        pen = as_f64(penalty, dev).reshape(-1)
        pen = pen.expand(B).contiguous() if pen.numel() == 1 else pen.contiguous()
        if pen.numel() != B:
            raise ValueError(f"penalty has {pen.numel()} values for a batch of {B}")
        self.Q, self.q, self.G, self.h, self.pen = Q.contiguous(), q.contiguous(), G.contiguous(), h.contiguous(), pen
        self.B, self.n, self.p, self.dev = B, n, p, dev

    def dims(self) -> Dims:
        return Dims(self.B, self.n, 0, self.p)

    def ptrs(self):
        return [ptr(t) for t in (self.Q, self.q, self.G, self.h, self.pen)]

    def new(self, *shape, dtype=torch.float64):
        return torch.empty(*shape, dtype=dtype, device=self.dev)

    def iterate(self):
        return [self.new(self.B, self.n)] + [self.new(self.B, self.p) for _ in range(5)]

    def out(self, *ts):
        return tuple(ts) if self.batched else tuple(t[0] for t in ts)


def _arr6(ts):
    return (ctypes.c_void_p * 6)(*[ptr(t) for t in ts])


def _run(name, op, bt: ElasticBatch, cfg, mid, tune=False):
    dims = bt.dims()
    ws = _lib.workspace(op, dims, cfg, bt.dev, tune)
    wp, wb = _lib.aligned(ws)
    _lib.call(name, ctypes.byref(dims), *bt.ptrs(), *mid, ctypes.byref(cfg), wp, wb, _lib.stream_handle())


def solve_qp_elastic(Q, q, G, h, penalty, solver_tol: float = 1e-3, *, precision=None, team_threads=None,
                     stats=None):
    """qpax/elastic_qp.py:184 -> (x, t, s1, s2, z1, z2, converged, iters)."""
    bt = ElasticBatch(Q, q, G, h, penalty)
    cfg = _config(dict(precision=precision, team_threads=team_threads), stats)
    it = bt.iterate()
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    _run("qpb_solve_qp_elastic", "elastic_solve", bt, cfg,
         [ctypes.c_double(solver_tol)] + [ptr(t) for t in it] + [ptr(conv), ptr(iters)])
    return bt.out(*it, conv, iters)


def tune_solve_qp_elastic(Q, q, G, h, penalty, solver_tol: float = 1e-3, *, precision=None):
    """solve_qp_elastic with the launch shape autotuned for these dims on this
    device (qpb_tune_solve_qp_elastic); later elastic calls with these dims
    use the recorded shape.  Returns what solve_qp_elastic returns."""
    bt = ElasticBatch(Q, q, G, h, penalty)
    cfg = _config(dict(precision=precision))
    it = bt.iterate()
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    _run("qpb_tune_solve_qp_elastic", "elastic_solve", bt, cfg,
         [ctypes.c_double(solver_tol)] + [ptr(t) for t in it] + [ptr(conv), ptr(iters)], tune=True)
    return bt.out(*it, conv, iters)


def initialize_elastic(Q, q, G, h, penalty, *, precision=None, team_threads=None):
    """qpax/elastic_qp.py:27 -> (x, t, s1, s2, z1, z2)."""
    bt = ElasticBatch(Q, q, G, h, penalty)
    cfg = _config(dict(precision=precision, team_threads=team_threads))
    it = bt.iterate()
    _run("qpb_initialize_elastic", "elastic_initialize", bt, cfg, [ptr(t) for t in it])
    return bt.out(*it)


def _iter_in(bt, ts, names=("x", "t", "s1", "s2", "z1", "z2")):
    """The elastic iterate (x (n), then t, s1, s2, z1, z2 (p each)) as checked (B, width) rows."""
    widths = (bt.n,) + (bt.p,) * 5
    return [_lib.rows(t, bt.dev, bt.B, w, nm) for t, w, nm in zip(ts, widths, names)]


def relax_qp_elastic(Q, q, G, h, penalty, x, t, s1, s2, z1, z2, solver_tol: float = 1e-3,
                     target_kappa: float = 1e-3, *, precision=None, team_threads=None):
    """qpax/elastic_qp.py:319 -> (xr, tr, s1r, s2r, z1r, z2r, converged, iters)."""
    bt = ElasticBatch(Q, q, G, h, penalty)
    cfg = _config(dict(precision=precision, team_threads=team_threads))
    ins = _iter_in(bt, (x, t, s1, s2, z1, z2))
    out = bt.iterate()
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    _run("qpb_relax_qp_elastic", "elastic_relax", bt, cfg,
         [_arr6(ins), ctypes.c_double(solver_tol), ctypes.c_double(target_kappa), _arr6(out), ptr(conv),
          ptr(iters)])
    return bt.out(*out, conv, iters)


def diff_qp_elastic(Q, q, G, h, x, t, s1, s2, lam1, lam2, dl_dx, *, penalty=0.0, precision=None,
                    team_threads=None):
    """qpax/elastic_qp.py:381 diff_qp_elastic -> (dQ, dq, dG, dh)."""
    bt = ElasticBatch(Q, q, G, h, penalty)
    cfg = _config(dict(precision=precision, team_threads=team_threads))
    ins = _iter_in(bt, (x, t, s1, s2, lam1, lam2), ("x", "t", "s1", "s2", "lam1", "lam2"))
    g = as_f64(dl_dx, bt.dev).reshape(bt.B, bt.n).contiguous()
    dQ, dq, dG, dh = bt.new(bt.B, bt.n, bt.n), bt.new(bt.B, bt.n), bt.new(bt.B, bt.p, bt.n), bt.new(bt.B, bt.p)
    _run("qpb_diff_qp_elastic", "elastic_diff", bt, cfg,
         [_arr6(ins), ptr(g), ptr(dQ), ptr(dq), ptr(dG), ptr(dh)])
    return bt.out(dQ, dq, dG, dh)


def _elastic_bwd(bt: ElasticBatch, it, g, solver_tol, target_kappa, opts):
    cfg = _config(opts)
    dQ, dq, dG, dh = bt.new(bt.B, bt.n, bt.n), bt.new(bt.B, bt.n), bt.new(bt.B, bt.p, bt.n), bt.new(bt.B, bt.p)
    _run("qpb_solve_qp_elastic_primal_bwd", "elastic_primal_bwd", bt, cfg,
         [_arr6(it), ptr(g), ctypes.c_double(solver_tol), ctypes.c_double(target_kappa), ptr(dQ), ptr(dq),
          ptr(dG), ptr(dh)])
    return dQ, dq, dG, dh


class _SolveQPElasticPrimal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Q, q, G, h, penalty, solver_tol, target_kappa, opts):
        bt = ElasticBatch(Q, q, G, h, penalty)
        cfg = _config(opts)
        it = bt.iterate()
        conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
        _run("qpb_solve_qp_elastic", "elastic_solve", bt, cfg,
             [ctypes.c_double(solver_tol)] + [ptr(t) for t in it] + [ptr(conv), ptr(iters)])
        ctx.bt, ctx.opts, ctx.tols = bt, opts, (solver_tol, target_kappa)
        ctx.save_for_backward(*it)
        # each gradient goes back with its input's shape, device and dtype
        ctx.metas = [(t.shape, t.device, t.dtype) for t in (Q, q, G, h)]
        return it[0] if bt.batched else it[0][0]

    @staticmethod
    def backward(ctx, gx):
        bt = ctx.bt
        g = as_f64(gx, bt.dev).reshape(bt.B, bt.n).contiguous()
        grads = _elastic_bwd(bt, list(ctx.saved_tensors), g, *ctx.tols, ctx.opts)
        out = [gr.reshape(shp).to(device=dev, dtype=dt) for gr, (shp, dev, dt) in zip(grads, ctx.metas)]
        return (*out, None, None, None, None)


def solve_qp_elastic_primal(Q, q, G, h, penalty, solver_tol: float = 1e-5, target_kappa: float = 1e-3, *,
                            precision=None, team_threads=None):
    """qpax/elastic_qp.py:420 -> x, differentiable in Q, q, G, h (not penalty)."""
    opts = dict(precision=precision, team_threads=team_threads)
    return _SolveQPElasticPrimal.apply(*[torch.as_tensor(t) for t in (Q, q, G, h)], penalty, solver_tol,
                                       target_kappa, opts)


def solve_qp_elastic_primal_vjp(Q, q, G, h, penalty, dl_dx, solver_tol: float = 1e-5, target_kappa: float = 1e-3,
                                *, precision=None, team_threads=None):
    """Forward and backward of solve_qp_elastic_primal without autograd -> (x, (dQ, dq, dG, dh))."""
    opts = dict(precision=precision, team_threads=team_threads)
    out = solve_qp_elastic(Q, q, G, h, penalty, solver_tol, **opts)
    bt = ElasticBatch(Q, q, G, h, penalty)
    it = [t.reshape(bt.B, -1).contiguous() for t in out[:6]]
    g = as_f64(dl_dx, bt.dev).reshape(bt.B, bt.n).contiguous()
    grads = _elastic_bwd(bt, it, g, solver_tol, target_kappa, opts)
    return out[0], bt.out(*grads)
