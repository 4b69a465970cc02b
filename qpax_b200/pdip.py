"""solve_qp / initialize on the GPU, mirroring qpax/pdip.py.

    x, s, z, y, converged, iters = solve_qp(Q, q, A, b, G, h, solver_tol=1e-3)

Same argument order, defaults and return tuple as qpax.solve_qp
(qpax/pdip.py:181-251).  Arrays may carry a leading batch axis (the axis a
qpax user would jax.vmap over): Q (B, n, n), q (B, n), A (B, m, n), b (B, m),
G (B, p, n), h (B, p).  Unbatched inputs give unbatched outputs.  Inputs are
taken as float64 on the current CUDA device; outputs are CUDA tensors.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import Dims, as_f64, ptr

DEFAULTS = {"precision": "auto", "team_threads": 0, "pivot_max": 0.0, "max_sweeps": 0}


def set_defaults(**kw) -> None:
    """Set library-wide defaults for precision ('auto' | 'mixed' | 'fp64'), team_threads,
    pivot_max and max_sweeps (see include/qpb.h qpb_config)."""
    for k, v in kw.items():
        if k not in DEFAULTS:
            raise KeyError(k)
        DEFAULTS[k] = v


def _config(opts: dict, stats=None) -> _lib.Config:
    o = dict(DEFAULTS)
    o.update({k: v for k, v in opts.items() if v is not None})
    return _lib.make_config(o["precision"], o["team_threads"], o["pivot_max"], o["max_sweeps"], stats)


class StdBatch:
    """Inputs of a standard QP batch on the device, with their shapes."""

    def __init__(self, Q, q, A, b, G, h):
        dev = _lib.device()
        Q, q, A, b, G, h = (as_f64(t, dev) for t in (Q, q, A, b, G, h))
        self.batched = Q.dim() == 3
        if not self.batched:
            Q = torch.atleast_2d(Q)[None]
            n = Q.shape[-1]
            A = A.reshape(-1, n) if A.numel() else A.reshape(0, n)
            G = G.reshape(-1, n) if G.numel() else G.reshape(0, n)
            q, A, b, G, h = q.reshape(1, -1), A[None], b.reshape(1, -1), G[None], h.reshape(1, -1)
        B, n = Q.shape[0], Q.shape[-1]
        m, p = A.shape[-2], G.shape[-2]
        want = {"Q": (B, n, n), "q": (B, n), "A": (B, m, n), "b": (B, m), "G": (B, p, n), "h": (B, p)}
        for name, t in zip("Q q A b G h".split(), (Q, q, A, b, G, h)):
            if tuple(t.shape) != want[name]:
                raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {want[name]}")
        self.Q, self.q, self.A, self.b, self.G, self.h = (t.contiguous() for t in (Q, q, A, b, G, h))
        self.B, self.n, self.m, self.p = B, n, m, p
        self.dev = dev

    def dims(self) -> Dims:
        return Dims(self.B, self.n, self.m, self.p)

    def ptrs(self):
        return [ptr(t) for t in (self.Q, self.q, self.A, self.b, self.G, self.h)]

    def new(self, *shape, dtype=torch.float64):
        return torch.empty(*shape, dtype=dtype, device=self.dev)

    def out(self, *ts):
        return tuple(ts) if self.batched else tuple(t[0] for t in ts)


def _run(name: str, op: str, bt: StdBatch, cfg: _lib.Config, mid: list, tail: list, tune: bool = False) -> None:
    dims = bt.dims()
    ws = _lib.workspace(op, dims, cfg, bt.dev, tune)
    wp, wb = _lib.aligned(ws)
    _lib.call(name, ctypes.byref(dims), *bt.ptrs(), *mid, *tail, ctypes.byref(cfg), wp, wb, _lib.stream_handle())


def solve_qp(Q, q, A, b, G, h, solver_tol: float = 1e-3, *, precision=None, team_threads=None, pivot_max=None,
             max_sweeps=None, stats=None):
    """qpax/pdip.py:181 solve_qp -> (x, s, z, y, converged, iters)."""
    bt = StdBatch(Q, q, A, b, G, h)
    cfg = _config(dict(precision=precision, team_threads=team_threads, pivot_max=pivot_max, max_sweeps=max_sweeps),
                  stats)
    x, s, z, y = bt.new(bt.B, bt.n), bt.new(bt.B, bt.p), bt.new(bt.B, bt.p), bt.new(bt.B, bt.m)
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    _run("qpb_solve_qp", "solve", bt, cfg, [ctypes.c_double(solver_tol)],
         [ptr(x), ptr(s), ptr(z), ptr(y), ptr(conv), ptr(iters)])
    return bt.out(x, s, z, y, conv, iters)


def initialize(Q, q, A, b, G, h, *, precision=None, team_threads=None):
    """qpax/pdip.py:15 initialize -> (x, s, z, y) on the data as given."""
    bt = StdBatch(Q, q, A, b, G, h)
    cfg = _config(dict(precision=precision, team_threads=team_threads))
    x, s, z, y = bt.new(bt.B, bt.n), bt.new(bt.B, bt.p), bt.new(bt.B, bt.p), bt.new(bt.B, bt.m)
    _run("qpb_initialize", "initialize", bt, cfg, [], [ptr(x), ptr(s), ptr(z), ptr(y)])
    return bt.out(x, s, z, y)


def relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol: float = 1e-5, target_kappa: float = 1e-5, *,
             precision=None, team_threads=None, stats=None):
    """qpax/pdip_relaxed.py:70 relax_qp -> (xr, sr, zr, yr, converged, iters)."""
    bt = StdBatch(Q, q, A, b, G, h)
    cfg = _config(dict(precision=precision, team_threads=team_threads), stats)
    its = [_lib.rows(t, bt.dev, bt.B, w, nm) for t, w, nm in zip((x, s, z, y), (bt.n, bt.p, bt.p, bt.m), "xszy")]
    xr, sr, zr, yr = bt.new(bt.B, bt.n), bt.new(bt.B, bt.p), bt.new(bt.B, bt.p), bt.new(bt.B, bt.m)
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    _run("qpb_relax_qp", "relax", bt, cfg,
         [ptr(t) for t in its] + [ctypes.c_double(solver_tol), ctypes.c_double(target_kappa)],
         [ptr(xr), ptr(sr), ptr(zr), ptr(yr), ptr(conv), ptr(iters)])
    return bt.out(xr, sr, zr, yr, conv, iters)


def tune_solve_qp(Q, q, A, b, G, h, solver_tol: float = 1e-3, *, precision=None):
    """solve_qp with the launch shape autotuned for this (n, m, p) on this
    device (qpb_tune_solve_qp): the candidates are timed on the batch, the
    fastest is recorded, and later calls with these dims use it.  Returns what
    solve_qp returns."""
    bt = StdBatch(Q, q, A, b, G, h)
    cfg = _config(dict(precision=precision))
    x, s, z, y = bt.new(bt.B, bt.n), bt.new(bt.B, bt.p), bt.new(bt.B, bt.p), bt.new(bt.B, bt.m)
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    _run("qpb_tune_solve_qp", "solve", bt, cfg, [ctypes.c_double(solver_tol)],
         [ptr(x), ptr(s), ptr(z), ptr(y), ptr(conv), ptr(iters)], tune=True)
    return bt.out(x, s, z, y, conv, iters)
