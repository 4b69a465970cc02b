"""Uneven batches: instances of different (n, m, p) in one call.

qpax runs one jit(vmap(solve_qp)) per distinct shape (its early exits branch
on Python shapes, qpax/pdip.py:208-217).  Here a plan groups the instances by
kernel variant once; each call then launches one persistent kernel per size
bin, concurrently, from the caller's stream (capturable in a CUDA graph).

    plan = PackedPlan(shapes)                     # [(n, m, p), ...], p >= 1
    x, s, z, y, conv, iters = plan.solve(Q, q, A, b, G, h, solver_tol)   # packed 1-D tensors
    dQ, dq, dA, db, dG, dh = plan.primal_bwd(Q, ..., x, s, z, y, dl_dx, solver_tol, kappa)

Packed layout: each array is the concatenation of the per-instance row-major
arrays in instance order.  `pack` / `unpack` convert from / to lists.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

_SIGS = {
    "qpb_plan_create": ([ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.c_void_p,
                         ctypes.POINTER(_lib.Config)], ctypes.c_int),
    "qpb_plan_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "qpb_plan_workspace_size": ([ctypes.c_void_p], ctypes.c_size_t),
    "qpb_plan_num_bins": ([ctypes.c_void_p], ctypes.c_int32),
    "qpb_plan_totals": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "qpb_plan_tune_workspace_size": ([ctypes.c_void_p], ctypes.c_size_t),
    "qpb_plan_tune": ([ctypes.c_void_p] + [ctypes.c_void_p] * 6 + [ctypes.c_double] + [ctypes.c_void_p] * 6 +
                      [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p], ctypes.c_int),
    "qpb_plan_bin_info": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p], ctypes.c_int32),
    "qpb_solve_qp_packed": ([ctypes.c_void_p] + [ctypes.c_void_p] * 6 + [ctypes.c_double] + [ctypes.c_void_p] * 6 +
                            [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p], ctypes.c_int),
    "qpb_solve_qp_primal_bwd_packed": ([ctypes.c_void_p] + [ctypes.c_void_p] * 11 + [ctypes.c_double] * 2 +
                                       [ctypes.c_void_p] * 8 + [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p],
                                       ctypes.c_int),
}


def _load():
    lib = _lib.load()
    if not getattr(lib, "_qpb_packed_ready", False):
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        lib._qpb_packed_ready = True
    return lib


def sizes(shapes):
    """Per-instance lengths of (Q, q, A, b, G, h)."""
    sh = np.asarray(shapes, dtype=np.int64).reshape(-1, 3)
    n, m, p = sh[:, 0], sh[:, 1], sh[:, 2]
    return [n * n, n, m * n, m, p * n, p]


def check_packed(t, length: int, dev: torch.device, name: str, dtype=torch.float64) -> None:
    """Raise unless `t` is a contiguous `dtype` tensor of `length` elements on
    `dev`: the kernels read and write exactly the plan's packed lengths, so a
    shorter buffer would be read or written past its end on the device."""
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor, got {type(t).__name__}")
    if t.dtype != dtype or t.device != dev or t.numel() != length or not t.is_contiguous():
        what = f"{t.dtype} {tuple(t.shape)} on {t.device}" + ("" if t.is_contiguous() else ", not contiguous")
        raise ValueError(f"{name}: expected a contiguous {dtype} tensor of {length} elements on {dev}, got {what}")


def pack(arrays, device=None) -> torch.Tensor:
    """Concatenate per-instance arrays (any shapes) into one 1-D float64 tensor."""
    dev = device or _lib.device()
    parts = [torch.as_tensor(a, dtype=torch.float64).reshape(-1) for a in arrays]
    return torch.cat(parts).to(dev) if parts else torch.zeros(0, dtype=torch.float64, device=dev)


def unpack(t: torch.Tensor, lengths, shapes=None):
    """Split a packed tensor back into per-instance pieces (reshaped when shapes given)."""
    out = list(torch.split(t, [int(v) for v in lengths]))
    if shapes is not None:
        out = [o.reshape(s) for o, s in zip(out, shapes)]
    return out


class PackedPlan:
    """A plan for one uneven batch (shapes fixed at construction)."""

    def __init__(self, shapes, precision: str = "auto", team_threads: int = 0):
        self.lib = _load()
        self.dev = _lib.device()
        self.shapes = np.ascontiguousarray(np.asarray(shapes, dtype=np.int32).reshape(-1, 3))
        self.batch = int(self.shapes.shape[0])
        self.cfg = _lib.make_config(precision, team_threads)
        h = ctypes.c_void_p()
        st = self.lib.qpb_plan_create(ctypes.byref(h), self.batch, self.shapes.ctypes.data, ctypes.byref(self.cfg))
        if st != 0:
            raise _lib.QpbError(f"qpb_plan_create: {self.lib.qpb_status_string(st).decode()} (status {st})")
        self.handle = h
        tot = (ctypes.c_int64 * 6)()
        self.lib.qpb_plan_totals(self.handle, ctypes.addressof(tot))
        self.totals = [int(v) for v in tot]
        self.num_bins = int(self.lib.qpb_plan_num_bins(self.handle))
        nbytes = int(self.lib.qpb_plan_workspace_size(self.handle))
        self.workspace = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.dev)
        self.lengths = sizes(self.shapes)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            self.lib.qpb_plan_destroy(h)
            self.handle = None

    def _ws(self):
        return _lib.aligned(self.workspace)

    def new(self, k, dtype=torch.float64):
        return torch.empty(self.totals[k], dtype=dtype, device=self.dev)

    def _check_inputs(self, tensors, fields, names):
        for t, k, name in zip(tensors, fields, names):
            check_packed(t, self.totals[k], self.dev, name)

    def solve(self, Q, q, A, b, G, h, solver_tol: float = 1e-3):
        """qpb_solve_qp_packed -> packed (x, s, z, y) and per-instance (converged, iters)."""
        self._check_inputs((Q, q, A, b, G, h), range(6), "Q q A b G h".split())
        x, s, z, y = self.new(1), self.new(5), self.new(5), self.new(3)
        conv = torch.empty(self.batch, dtype=torch.int32, device=self.dev)
        iters = torch.empty(self.batch, dtype=torch.int32, device=self.dev)
        wp, wb = self._ws()
        _lib.call("qpb_solve_qp_packed", self.handle, *[_lib.ptr(t) for t in (Q, q, A, b, G, h)],
                  ctypes.c_double(solver_tol), *[_lib.ptr(t) for t in (x, s, z, y, conv, iters)], wp, wb,
                  _lib.stream_handle())
        return x, s, z, y, conv, iters

    def tune(self, Q, q, A, b, G, h, solver_tol: float = 1e-3):
        """qpb_plan_tune: time the launch shapes the kernels support for each
        size bin on this batch (forward solve on each bin's heaviest
        instances), keep the fastest per bin and record it for this device.
        Returns the packed solve outputs, like solve()."""
        self._check_inputs((Q, q, A, b, G, h), range(6), "Q q A b G h".split())
        tw = int(self.lib.qpb_plan_tune_workspace_size(self.handle))
        ws = torch.empty(tw + 256, dtype=torch.uint8, device=self.dev)
        wp, wb = _lib.aligned(ws)
        x, s, z, y = self.new(1), self.new(5), self.new(5), self.new(3)
        conv = torch.empty(self.batch, dtype=torch.int32, device=self.dev)
        iters = torch.empty(self.batch, dtype=torch.int32, device=self.dev)
        _lib.call("qpb_plan_tune", self.handle, *[_lib.ptr(t) for t in (Q, q, A, b, G, h)],
                  ctypes.c_double(solver_tol), *[_lib.ptr(t) for t in (x, s, z, y, conv, iters)], wp, wb,
                  _lib.stream_handle())
        nbytes = int(self.lib.qpb_plan_workspace_size(self.handle))
        if nbytes + 256 > self.workspace.numel():
            self.workspace = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.dev)
        return x, s, z, y, conv, iters

    def bin_info(self):
        """Per bin (launch order): dict of its instances, largest shape and launch shape."""
        out = []
        for k in range(self.num_bins):
            info = (ctypes.c_int32 * 8)()
            self.lib.qpb_plan_bin_info(self.handle, k, ctypes.addressof(info))
            v = list(info)
            out.append(dict(instances=v[0], n_max=v[1], m_max=v[2], p_max=v[3], team_threads=v[4],
                            arena="shared" if v[5] == 1 else "global", g_chunk_rows=v[6], ctas_per_sm=v[7]))
        return out

    def primal_bwd(self, Q, q, A, b, G, h, x, s, z, y, dl_dx, solver_tol: float = 1e-5,
                   target_kappa: float = 1e-3, relax_out=None):
        """qpb_solve_qp_primal_bwd_packed -> packed (dQ, dq, dA, db, dG, dh).

        relax_out: optional (converged, iters) int32 device tensors of length
        batch that receive the relaxation's per-instance outcome."""
        self._check_inputs((Q, q, A, b, G, h, x, s, z, y, dl_dx), (0, 1, 2, 3, 4, 5, 1, 5, 5, 3, 1),
                           "Q q A b G h x s z y dl_dx".split())
        rc, ri = relax_out if relax_out is not None else (None, None)
        for t, name in ((rc, "relax_out[0]"), (ri, "relax_out[1]")):
            if t is not None:
                check_packed(t, self.batch, self.dev, name, torch.int32)
        grads = [self.new(k) for k in range(6)]
        wp, wb = self._ws()
        _lib.call("qpb_solve_qp_primal_bwd_packed", self.handle,
                  *[_lib.ptr(t) for t in (Q, q, A, b, G, h, x, s, z, y, dl_dx)], ctypes.c_double(solver_tol),
                  ctypes.c_double(target_kappa), *[_lib.ptr(t) for t in grads], _lib.ptr(rc), _lib.ptr(ri),
                  wp, wb, _lib.stream_handle())
        return tuple(grads)


def solve_qp_uneven(Qs, qs, As, bs, Gs, hs, solver_tol: float = 1e-3, precision: str = "auto"):
    """solve_qp over lists of per-instance arrays of different shapes.

    Returns lists (x_i), (s_i), (z_i), (y_i) and tensors (converged, iters).
    """
    shapes = [(np.shape(Q)[0], np.shape(b)[0], np.shape(h)[0]) for Q, b, h in zip(Qs, bs, hs)]
    plan = PackedPlan(shapes, precision)
    ins = [pack(v, plan.dev) for v in (Qs, qs, As, bs, Gs, hs)]
    x, s, z, y, conv, iters = plan.solve(*ins, solver_tol)
    L = plan.lengths
    return unpack(x, L[1]), unpack(s, L[5]), unpack(z, L[5]), unpack(y, L[3]), conv, iters


class PackedHostPipeline:
    """Forward + backward of solve_qp_primal on an uneven batch held in host
    memory, with copies overlapped with the kernels.

    The instances are cut into `chunks` contiguous groups (contiguous in every
    packed array), each with its own plan and device buffers.  Streams by
    role: the groups are copied in, in order, on one stream (each at the
    link's full rate), solved forward and backward on compute streams taken
    in turn (one group's solve overlaps the previous group's tail), and their
    x and six gradients copied back on a last stream.

        pipe = PackedHostPipeline(shapes, chunks=4)
        x, grads = pipe.run(Q, q, A, b, G, h, dl_dx, solver_tol, target_kappa, out=None)

    Inputs are packed 1-D CPU float64 tensors (pinned for the copies to
    overlap); `out` may hold packed CPU tensors (x, dQ, dq, dA, db, dG, dh).
    """

    def __init__(self, shapes, chunks: int = 4, precision: str = "auto", streams: int = 4):
        sh = np.ascontiguousarray(np.asarray(shapes, dtype=np.int32).reshape(-1, 3))
        B = sh.shape[0]
        chunks = max(1, min(int(chunks), B))
        self.bounds = [B * c // chunks for c in range(chunks + 1)]
        self.lengths = sizes(sh)
        self.totals = [int(np.sum(v)) for v in self.lengths]
        # element offset of instance i in each packed field
        self.offs = [np.concatenate([[0], np.cumsum(v)]) for v in self.lengths]
        self.plans = [PackedPlan(sh[lo:hi], precision) for lo, hi in zip(self.bounds[:-1], self.bounds[1:])]
        self.dev = _lib.device()
        # copy-in, compute (streams - 2 of them, at least one), copy-out
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(max(3, streams))]
        # field of each input / output: Q q A b G h dl -> 0 1 2 3 4 5 1; x dQ dq dA db dG dh -> 1 0 1 2 3 4 5
        self.in_fields = [0, 1, 2, 3, 4, 5, 1]
        self.out_fields = [1, 0, 1, 2, 3, 4, 5]
        self.dev_in = [[torch.empty(p.totals[k], dtype=torch.float64, device=self.dev) for k in self.in_fields]
                       for p in self.plans]

    def _span(self, field, c):
        lo, hi = self.bounds[c], self.bounds[c + 1]
        return int(self.offs[field][lo]), int(self.offs[field][hi])

    def run(self, Q, q, A, b, G, h, dl_dx, solver_tol: float = 1e-5, target_kappa: float = 1e-3, out=None):
        host_in = [torch.as_tensor(t, dtype=torch.float64).reshape(-1) for t in (Q, q, A, b, G, h, dl_dx)]
        if out is None:
            pin = torch.cuda.is_available()
            out = [torch.empty(self.totals[f], dtype=torch.float64, pin_memory=pin) for f in self.out_fields]
        main = torch.cuda.current_stream(self.dev)
        for s in self.streams:
            s.wait_stream(main)
        s_in, s_out, comp = self.streams[0], self.streams[-1], self.streams[1:-1]
        for c, plan in enumerate(self.plans):
            d = self.dev_in[c]
            with torch.cuda.stream(s_in):
                for dst, src, f in zip(d, host_in, self.in_fields):
                    lo, hi = self._span(f, c)
                    dst.copy_(src[lo:hi], non_blocking=True)
            arrived = torch.cuda.Event()
            arrived.record(s_in)
            sc = comp[c % len(comp)]
            sc.wait_event(arrived)
            with torch.cuda.stream(sc):
                res = plan.solve(*d[:6], solver_tol)
                grads = plan.primal_bwd(*d[:6], *res[:4], d[6], solver_tol, target_kappa)
            solved = torch.cuda.Event()
            solved.record(sc)
            s_out.wait_event(solved)
            with torch.cuda.stream(s_out):
                for dst, src, f in zip(out, (res[0],) + tuple(grads), self.out_fields):
                    lo, hi = self._span(f, c)
                    dst[lo:hi].copy_(src, non_blocking=True)
                    src.record_stream(s_out)
                for t in res:
                    t.record_stream(s_out)
        for s in self.streams:
            main.wait_stream(s)
        torch.cuda.synchronize(self.dev)
        return out[0], tuple(out[1:])
