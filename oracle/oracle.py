"""numpy front end of the FP64 CPU oracle (oracle/qp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline / reference arm, always as the checker or the timed
CPU restatement of qpax -- never by the product path in qpax_b200/.

Each function mirrors a qpax function of the same name (kevin-tracy/qpax):
  solve_qp            qpax/pdip.py:181-251
  initialize          qpax/pdip.py:15-35
  relax_qp            qpax/pdip_relaxed.py:70-103
  diff_qp             qpax/diff_qp.py:20-46 (+ optnet_derivatives :8-17)
  solve_qp_primal_vjp qpax/diff_qp.py:61-79 (forward = solve + relax, backward = diff_qp)
  solve_qp_elastic    qpax/elastic_qp.py:184-228
  initialize_elastic  qpax/elastic_qp.py:27-47
  relax_qp_elastic    qpax/elastic_qp.py:319-359
  diff_qp_elastic     qpax/elastic_qp.py:381-417
  solve_qp_elastic_primal_vjp  qpax/elastic_qp.py:433-466

Inputs are batched with a leading instance axis (the axis qpax users vmap
over), or given as lists of per-instance arrays for ragged batches.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_qp.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "qp_oracle.c")
        ):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.oracle_num_threads.restype = ctypes.c_int
    return _lib


def num_threads() -> int:
    """OpenMP threads the oracle uses when nthreads=0."""
    return int(_load().oracle_num_threads())


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class _Batch:
    """Packs a uniform (leading batch axis) or ragged (lists) batch into the
    flat per-field arrays the C oracle reads."""

    def __init__(self, fields, shapes):
        self.shapes = np.ascontiguousarray(np.asarray(shapes, dtype=np.int32).reshape(-1, 3))
        self.B = self.shapes.shape[0]
        self.fields = fields

    @staticmethod
    def from_uniform(**arrs):
        Q = np.asarray(arrs["Q"], dtype=np.float64)
        squeeze = Q.ndim == 2
        out = {}
        for k, v in arrs.items():
            v = np.asarray(v, dtype=np.float64)
            if squeeze:
                v = v[None]
            out[k] = v
        B, n = out["Q"].shape[0], out["Q"].shape[-1]
        m = out["b"].shape[-1] if "b" in out else 0
        p = out["h"].shape[-1]
        flat = {k: np.ascontiguousarray(v.reshape(-1)) for k, v in out.items()}
        b = _Batch(flat, np.tile(np.array([n, m, p], np.int32), (B, 1)))
        b.uniform = (B, n, m, p)
        b.squeeze = squeeze
        return b

    @staticmethod
    def from_ragged(**lists):
        Qs = lists["Q"]
        shapes = []
        for i, Q in enumerate(Qs):
            n = np.asarray(Q).shape[0]
            m = np.asarray(lists["b"][i]).shape[0] if "b" in lists else 0
            p = np.asarray(lists["h"][i]).shape[0]
            shapes.append((n, m, p))
        flat = {
            k: np.ascontiguousarray(np.concatenate([np.asarray(a, np.float64).reshape(-1) for a in v]))
            if len(v)
            else np.zeros(0)
            for k, v in lists.items()
        }
        b = _Batch(flat, shapes)
        b.uniform = None
        b.squeeze = False
        return b

    def totals(self):
        n, m, p = self.shapes[:, 0].astype(np.int64), self.shapes[:, 1].astype(np.int64), self.shapes[:, 2].astype(
            np.int64
        )
        return dict(n=int(n.sum()), m=int(m.sum()), p=int(p.sum()), nn=int((n * n).sum()), mn=int((m * n).sum()),
                    pn=int((p * n).sum()))

    def unpack(self, arr, kind):
        """Split a flat output back into the caller's batch layout."""
        if self.uniform is not None:
            B, n, m, p = self.uniform
            dims = {"n": (n,), "m": (m,), "p": (p,), "nn": (n, n), "mn": (m, n), "pn": (p, n), "1": ()}[kind]
            out = arr.reshape((B,) + dims)
            return out[0] if self.squeeze else out
        sizes = {
            "n": self.shapes[:, 0],
            "m": self.shapes[:, 1],
            "p": self.shapes[:, 2],
            "nn": self.shapes[:, 0] ** 2,
            "mn": self.shapes[:, 1] * self.shapes[:, 0],
            "pn": self.shapes[:, 2] * self.shapes[:, 0],
            "1": np.ones(self.B, np.int64),
        }[kind]
        parts = np.split(arr, np.cumsum(sizes)[:-1]) if self.B > 1 else [arr]
        out = []
        for i, part in enumerate(parts):
            n, m, p = self.shapes[i]
            shp = {"nn": (n, n), "mn": (m, n), "pn": (p, n)}.get(kind)
            out.append(part.reshape(shp) if shp else (part[0] if kind == "1" else part))
        return out


def _make(ragged, **kw):
    return _Batch.from_ragged(**kw) if ragged else _Batch.from_uniform(**kw)


def _is_ragged(Q):
    return isinstance(Q, (list, tuple))


def _empty(n):
    return np.zeros(max(int(n), 0), np.float64)


def solve_qp(Q, q, A, b, G, h, solver_tol=1e-3, nthreads=0):
    """qpax/pdip.py:181 solve_qp -> (x, s, z, y, converged, iters)."""
    bt = _make(_is_ragged(Q), Q=Q, q=q, A=A, b=b, G=G, h=h)
    t = bt.totals()
    x, s, z, y = _empty(t["n"]), _empty(t["p"]), _empty(t["p"]), _empty(t["m"])
    conv = np.zeros(bt.B, np.int32)
    iters = np.zeros(bt.B, np.int32)
    f = bt.fields
    _load().oracle_solve_qp(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["A"]), _d(f["b"]), _d(f["G"]), _d(f["h"]),
        ctypes.c_double(solver_tol), _d(x), _d(s), _d(z), _d(y), _i(conv), _i(iters), nthreads,
    )
    return (bt.unpack(x, "n"), bt.unpack(s, "p"), bt.unpack(z, "p"), bt.unpack(y, "m"), bt.unpack(conv, "1"),
            bt.unpack(iters, "1"))


def initialize(Q, q, A, b, G, h, nthreads=0):
    """qpax/pdip.py:15 initialize -> (x, s, z, y), on the data as given."""
    bt = _make(_is_ragged(Q), Q=Q, q=q, A=A, b=b, G=G, h=h)
    t = bt.totals()
    x, s, z, y = _empty(t["n"]), _empty(t["p"]), _empty(t["p"]), _empty(t["m"])
    f = bt.fields
    _load().oracle_initialize(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["A"]), _d(f["b"]), _d(f["G"]), _d(f["h"]), _d(x), _d(s),
        _d(z), _d(y), nthreads,
    )
    return bt.unpack(x, "n"), bt.unpack(s, "p"), bt.unpack(z, "p"), bt.unpack(y, "m")


def relax_qp(Q, q, A, b, G, h, x, s, z, y, solver_tol=1e-5, target_kappa=1e-5, nthreads=0):
    """qpax/pdip_relaxed.py:70 relax_qp -> (xr, sr, zr, yr, converged, iters)."""
    rg = _is_ragged(Q)
    bt = _make(rg, Q=Q, q=q, A=A, b=b, G=G, h=h, x=x, s=s, z=z, y=y)
    f = bt.fields
    xr, sr, zr, yr = f["x"].copy(), f["s"].copy(), f["z"].copy(), f["y"].copy()
    conv = np.zeros(bt.B, np.int32)
    iters = np.zeros(bt.B, np.int32)
    _load().oracle_relax_qp(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["A"]), _d(f["b"]), _d(f["G"]), _d(f["h"]),
        ctypes.c_double(solver_tol), ctypes.c_double(target_kappa), _d(xr), _d(sr), _d(zr), _d(yr), _i(conv),
        _i(iters), nthreads,
    )
    return (bt.unpack(xr, "n"), bt.unpack(sr, "p"), bt.unpack(zr, "p"), bt.unpack(yr, "m"), bt.unpack(conv, "1"),
            bt.unpack(iters, "1"))


def diff_qp(Q, q, A, b, G, h, x, s, lam, nu, dl_dx, nthreads=0):
    """qpax/diff_qp.py:20 diff_qp -> (dQ, dq, dA, db, dG, dh) at the relaxed iterate."""
    bt = _make(_is_ragged(Q), Q=Q, q=q, A=A, b=b, G=G, h=h, x=x, s=s, z=lam, y=nu, g=dl_dx)
    t = bt.totals()
    f = bt.fields
    dQ, dq, dA, db, dG, dh = (_empty(t["nn"]), _empty(t["n"]), _empty(t["mn"]), _empty(t["m"]), _empty(t["pn"]),
                              _empty(t["p"]))
    _load().oracle_diff_qp(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["A"]), _d(f["G"]), _d(f["x"]), _d(f["s"]), _d(f["z"]), _d(f["y"]),
        _d(f["g"]), _d(dQ), _d(dq), _d(dA), _d(db), _d(dG), _d(dh), nthreads,
    )
    return (bt.unpack(dQ, "nn"), bt.unpack(dq, "n"), bt.unpack(dA, "mn"), bt.unpack(db, "m"), bt.unpack(dG, "pn"),
            bt.unpack(dh, "p"))


def solve_qp_primal_vjp(Q, q, A, b, G, h, dl_dx, solver_tol=1e-5, target_kappa=1e-3, nthreads=0):
    """Forward + backward of qpax/diff_qp.py:49-82 solve_qp_primal in one pass.

    Returns (x, (dQ, dq, dA, db, dG, dh), converged, iters): x is the unrelaxed
    solution, the gradients are diff_qp at relax_qp(solve_qp(...)).
    """
    bt = _make(_is_ragged(Q), Q=Q, q=q, A=A, b=b, G=G, h=h, g=dl_dx)
    t = bt.totals()
    f = bt.fields
    x = _empty(t["n"])
    dQ, dq, dA, db, dG, dh = (_empty(t["nn"]), _empty(t["n"]), _empty(t["mn"]), _empty(t["m"]), _empty(t["pn"]),
                              _empty(t["p"]))
    conv = np.zeros(bt.B, np.int32)
    iters = np.zeros(bt.B, np.int32)
    _load().oracle_solve_qp_primal_fwd_bwd(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["A"]), _d(f["b"]), _d(f["G"]), _d(f["h"]),
        ctypes.c_double(solver_tol), ctypes.c_double(target_kappa), _d(f["g"]), _d(x), _d(dQ), _d(dq), _d(dA),
        _d(db), _d(dG), _d(dh), _i(conv), _i(iters), nthreads,
    )
    grads = (bt.unpack(dQ, "nn"), bt.unpack(dq, "n"), bt.unpack(dA, "mn"), bt.unpack(db, "m"), bt.unpack(dG, "pn"),
             bt.unpack(dh, "p"))
    return bt.unpack(x, "n"), grads, bt.unpack(conv, "1"), bt.unpack(iters, "1")


def _pen(penalty, B):
    p = np.asarray(penalty, np.float64).reshape(-1)
    return np.ascontiguousarray(np.broadcast_to(p, (B,)) if p.size == 1 else p)


def _ebatch(Q, q, G, h, **extra):
    return _make(_is_ragged(Q), Q=Q, q=q, G=G, h=h, **extra)


def solve_qp_elastic(Q, q, G, h, penalty, solver_tol=1e-3, nthreads=0):
    """qpax/elastic_qp.py:184 -> (x, t, s1, s2, z1, z2, converged, iters)."""
    bt = _ebatch(Q, q, G, h)
    t = bt.totals()
    f = bt.fields
    outs = [_empty(t["n"])] + [_empty(t["p"]) for _ in range(5)]
    conv = np.zeros(bt.B, np.int32)
    iters = np.zeros(bt.B, np.int32)
    pen = _pen(penalty, bt.B)
    _load().oracle_solve_qp_elastic(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["G"]), _d(f["h"]), _d(pen), ctypes.c_double(solver_tol),
        *[_d(o) for o in outs], _i(conv), _i(iters), nthreads,
    )
    return tuple([bt.unpack(outs[0], "n")] + [bt.unpack(o, "p") for o in outs[1:]] + [bt.unpack(conv, "1"),
                                                                                     bt.unpack(iters, "1")])


def initialize_elastic(Q, q, G, h, penalty, nthreads=0):
    """qpax/elastic_qp.py:27 -> (x, t, s1, s2, z1, z2)."""
    bt = _ebatch(Q, q, G, h)
    t = bt.totals()
    f = bt.fields
    outs = [_empty(t["n"])] + [_empty(t["p"]) for _ in range(5)]
    pen = _pen(penalty, bt.B)
    _load().oracle_initialize_elastic(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["G"]), _d(f["h"]), _d(pen), *[_d(o) for o in outs],
        nthreads,
    )
    return tuple([bt.unpack(outs[0], "n")] + [bt.unpack(o, "p") for o in outs[1:]])


def relax_qp_elastic(Q, q, G, h, penalty, x, t, s1, s2, z1, z2, solver_tol=1e-3, target_kappa=1e-3, nthreads=0):
    """qpax/elastic_qp.py:319 -> (xr, tr, s1r, s2r, z1r, z2r, converged, iters)."""
    bt = _ebatch(Q, q, G, h, x=x, t=t, s1=s1, s2=s2, z1=z1, z2=z2)
    f = bt.fields
    outs = [f[k].copy() for k in ("x", "t", "s1", "s2", "z1", "z2")]
    conv = np.zeros(bt.B, np.int32)
    iters = np.zeros(bt.B, np.int32)
    pen = _pen(penalty, bt.B)
    _load().oracle_relax_qp_elastic(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["q"]), _d(f["G"]), _d(f["h"]), _d(pen), ctypes.c_double(solver_tol),
        ctypes.c_double(target_kappa), *[_d(o) for o in outs], _i(conv), _i(iters), nthreads,
    )
    return tuple([bt.unpack(outs[0], "n")] + [bt.unpack(o, "p") for o in outs[1:]] + [bt.unpack(conv, "1"),
                                                                                     bt.unpack(iters, "1")])


def diff_qp_elastic(Q, q, G, h, x, t, s1, s2, lam1, lam2, dl_dx, nthreads=0):
    """qpax/elastic_qp.py:381 -> (dQ, dq, dG, dh), cropped to the caller's blocks."""
    bt = _ebatch(Q, q, G, h, x=x, t=t, s1=s1, s2=s2, z1=lam1, z2=lam2, g=dl_dx)
    tt = bt.totals()
    f = bt.fields
    dQ, dq, dG, dh = _empty(tt["nn"]), _empty(tt["n"]), _empty(tt["pn"]), _empty(tt["p"])
    _load().oracle_diff_qp_elastic(
        bt.B, _i(bt.shapes), _d(f["Q"]), _d(f["G"]), _d(f["x"]), _d(f["t"]), _d(f["s1"]), _d(f["s2"]), _d(f["z1"]),
        _d(f["z2"]), _d(f["g"]), _d(dQ), _d(dq), _d(dG), _d(dh), nthreads,
    )
    return bt.unpack(dQ, "nn"), bt.unpack(dq, "n"), bt.unpack(dG, "pn"), bt.unpack(dh, "p")


def solve_qp_elastic_primal_vjp(Q, q, G, h, penalty, dl_dx, solver_tol=1e-5, target_kappa=1e-3, nthreads=0):
    """Forward + backward of qpax/elastic_qp.py:420-469 solve_qp_elastic_primal.

    Returns (x, (dQ, dq, dG, dh)).
    """
    x, t, s1, s2, z1, z2, _, _ = solve_qp_elastic(Q, q, G, h, penalty, solver_tol=solver_tol, nthreads=nthreads)
    xr, tr, s1r, s2r, z1r, z2r, _, _ = relax_qp_elastic(
        Q, q, G, h, penalty, x, t, s1, s2, z1, z2, solver_tol=solver_tol, target_kappa=target_kappa, nthreads=nthreads
    )
    grads = diff_qp_elastic(Q, q, G, h, xr, tr, s1r, s2r, z1r, z2r, dl_dx, nthreads=nthreads)
    return x, grads
