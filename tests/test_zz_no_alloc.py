"""qpb_solve_qp_noalloc: the solve for callers that cannot allocate device memory.

Some hosts must not call cudaMalloc while solving (a CUDA graph capture that
forbids allocation, a real-time loop that allocates only at start-up, a
plugin whose framework owns the allocator).  qpb_solve_qp_noalloc takes no
workspace: its scratch is a fixed 1 MiB array inside the library.  These
tests call it through the C ABI and check that it returns exactly what the
workspace entry point qpb_solve_qp returns, on two calls in a row (so the
second call starts from the scratch the first one left behind), and that a
problem needing more scratch than the array holds is refused.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

QPB_ERR_UNSUPPORTED = 2


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from qpax_b200 import _lib as L

    lb = L.load()
    fn = lb.qpb_solve_qp_noalloc
    fn.argtypes = ([ctypes.POINTER(L.Dims)] + [ctypes.c_void_p] * 6 + [ctypes.c_double] + [ctypes.c_void_p] * 6 +
                   [ctypes.POINTER(L.Config), ctypes.c_void_p])
    fn.restype = ctypes.c_int
    return lb


def _noalloc(lib, Q, q, A, b, G, h, tol, **cfg):
    from qpax_b200 import _lib as L
    from qpax_b200.pdip import StdBatch, _config

    bt = StdBatch(Q, q, A, b, G, h)
    c = _config(cfg)
    x, s, z, y = bt.new(bt.B, bt.n), bt.new(bt.B, bt.p), bt.new(bt.B, bt.p), bt.new(bt.B, bt.m)
    conv, iters = bt.new(bt.B, dtype=torch.int32), bt.new(bt.B, dtype=torch.int32)
    dims = bt.dims()
    st = lib.qpb_solve_qp_noalloc(ctypes.byref(dims), *bt.ptrs(), ctypes.c_double(tol),
                                  *[L.ptr(t) for t in (x, s, z, y, conv, iters)], ctypes.byref(c),
                                  L.stream_handle())
    return st, (x, s, z, y, conv, iters)


@pytest.mark.parametrize("shape,cfg", [((32, 8, 64), {}), ((12, 3, 24), {"precision": "mixed"}),
                                       ((32, 12, 64), {})])
def test_noalloc_matches_workspace_entry_point(lib, shape, cfg):
    import qpax_b200 as qb
    from qpax_b200 import workloads as wl

    n, m, p = shape
    for call, seed in enumerate((101, 202)):  # two calls in a row, different data
        data = [torch.tensor(a, device="cuda") for a in wl.dense(96, n, m, p, seed + n)]
        ref = qb.solve_qp(*data, 1e-6, **cfg)
        st, out = _noalloc(lib, *data, 1e-6, **cfg)
        torch.cuda.synchronize()
        assert st == 0, f"call {call}: status {st}"
        np.testing.assert_array_equal(out[4].cpu().numpy(), ref[4].cpu().numpy())
        np.testing.assert_array_equal(out[5].cpu().numpy(), ref[5].cpu().numpy())
        for k in range(4):
            g, r = out[k].cpu().numpy(), ref[k].cpu().numpy()
            if r.size:
                scale = np.maximum(1.0, np.abs(r).max(axis=1, keepdims=True))
                assert (np.abs(g - r) / scale).max() <= 1e-6, f"call {call}, output {k}"


def test_noalloc_global_arena_within_scratch(lib):
    """A plan whose instances live in global-memory arenas (FP64, n > 32, a
    tiny batch) that still fits the 1 MiB array: the arena offsets inside the
    array are exercised, and the outputs equal qpb_solve_qp's bit for bit, on
    two calls in a row."""
    import qpax_b200 as qb
    from qpax_b200 import _lib as L
    from qpax_b200 import workloads as wl

    B, n, m, p = 2, 48, 6, 96
    dims = L.Dims(B, n, m, p)
    need = lib.qpb_workspace_size(0, ctypes.byref(dims), None)
    assert 256 < need <= (1 << 20), need
    for call, seed in enumerate((303, 404)):
        data = [torch.tensor(a, device="cuda") for a in wl.dense(B, n, m, p, seed)]
        ref = qb.solve_qp(*data, 1e-6)
        st, out = _noalloc(lib, *data, 1e-6)
        torch.cuda.synchronize()
        assert st == 0, f"call {call}: status {st}"
        for k in range(6):
            np.testing.assert_array_equal(out[k].cpu().numpy(), ref[k].cpu().numpy(), err_msg=f"call {call}, {k}")


def test_noalloc_refuses_problems_beyond_its_scratch(lib):
    from qpax_b200 import workloads as wl

    # n = 200, p = 400: each instance needs a global arena far beyond 1 MiB
    data = [torch.tensor(a, device="cuda") for a in wl.dense(4, 200, 10, 400, 7)]
    st, _ = _noalloc(lib, *data, 1e-6)
    assert st == QPB_ERR_UNSUPPORTED
