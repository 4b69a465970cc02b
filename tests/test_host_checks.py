"""Host-side argument checks of the Python boundary (CPU only, no launch).

The C ABI takes raw pointers and sizes; the Python layer is where tensors
are turned into them.  Every buffer whose size the kernels or the copies
rely on is checked there, so a wrong length, dtype, device or layout raises
before anything runs instead of being read or written past its end.
"""

import numpy as np
import pytest
import torch

from qpax_b200.diff_qp import host_buffers
from qpax_b200.packed import check_packed

CPU = torch.device("cpu")


def test_packed_arguments_are_checked_before_any_launch():
    """PackedPlan passes raw pointers to kernels that touch exactly the plan's
    packed lengths."""
    check_packed(torch.zeros(12, dtype=torch.float64), 12, CPU, "Q")
    check_packed(torch.zeros(0, dtype=torch.float64), 0, CPU, "b")
    check_packed(torch.zeros(5, dtype=torch.int32), 5, CPU, "conv", torch.int32)
    with pytest.raises(ValueError, match="12 elements"):
        check_packed(torch.zeros(11, dtype=torch.float64), 12, CPU, "Q")
    with pytest.raises(ValueError, match="float64"):
        check_packed(torch.zeros(12, dtype=torch.float32), 12, CPU, "Q")
    with pytest.raises(ValueError, match="not contiguous"):
        check_packed(torch.zeros(24, dtype=torch.float64)[::2], 12, CPU, "Q")
    with pytest.raises(ValueError, match="on cuda"):
        check_packed(torch.zeros(12, dtype=torch.float64), 12, torch.device("cuda", 0), "Q")
    with pytest.raises(TypeError):
        check_packed(np.zeros(12), 12, CPU, "Q")


def _host_batch(B=3, n=4, m=1, p=6):
    rng = np.random.default_rng(0)
    return [rng.standard_normal(s) for s in [(B, n, n), (B, n), (B, m, n), (B, m), (B, p, n), (B, p), (B, n)]]


def test_host_pipeline_buffers_have_the_batch_shapes():
    ins, out = host_buffers(*_host_batch())
    assert [tuple(t.shape) for t in ins] == [(3, 4, 4), (3, 4), (3, 1, 4), (3, 1), (3, 6, 4), (3, 6), (3, 4)]
    assert [tuple(t.shape) for t in out] == [(3, 4), (3, 4, 4), (3, 4), (3, 1, 4), (3, 1), (3, 6, 4), (3, 6)]
    assert all(t.dtype == torch.float64 and t.is_contiguous() and t.device.type == "cpu" for t in ins + out)
    # no equalities: A (B, 0, n), b (B, 0)
    data = _host_batch(m=0)
    ins, out = host_buffers(*data)
    assert tuple(out[3].shape) == (3, 0, 4) and tuple(out[4].shape) == (3, 0)
    # caller-provided outputs are used as given
    mine = [torch.empty(t.shape, dtype=torch.float64) for t in out]
    _, out2 = host_buffers(*data, out=mine)
    assert all(a is b for a, b in zip(out2, mine))


def test_host_pipeline_refuses_mismatched_buffers():
    data = _host_batch()
    bad = list(data)
    bad[1] = data[1][:, :3]
    with pytest.raises(ValueError, match="q has shape"):
        host_buffers(*bad)
    bad = list(data)
    bad[6] = data[6][:2]
    with pytest.raises(ValueError, match="dl_dx has shape"):
        host_buffers(*bad)
    with pytest.raises(ValueError, match="batched"):
        host_buffers(*[a[0] for a in data])
    _, out = host_buffers(*data)
    for k, wrong in [(0, torch.empty(3, 5, dtype=torch.float64)),             # x one element too long
                     (1, torch.empty(3, 4, 4, dtype=torch.float32)),          # dQ in float32
                     (5, torch.empty(3, 4, 6, dtype=torch.float64).transpose(1, 2)),  # dG not contiguous
                     (6, "not a tensor")]:
        o = list(out)
        o[k] = wrong
        with pytest.raises(ValueError, match="out "):
            host_buffers(*data, out=o)
    with pytest.raises(ValueError, match="7 tensors"):
        host_buffers(*data, out=out[:6])


def test_iterates_are_checked_against_the_problem_widths():
    """relax_qp, diff_qp and their elastic forms take an iterate per instance;
    each part must hold exactly B x width values (width n, p or m)."""
    from qpax_b200._lib import rows

    t = rows(np.arange(12.0), CPU, 3, 4, "x")
    assert tuple(t.shape) == (3, 4) and t.dtype == torch.float64 and t.is_contiguous()
    assert tuple(rows(np.zeros((3, 0)), CPU, 3, 0, "y").shape) == (3, 0)
    np.testing.assert_array_equal(rows(np.arange(12.0).reshape(3, 4).T.copy().T, CPU, 3, 4, "x").numpy(),
                                  np.arange(12.0).reshape(3, 4))
    with pytest.raises(ValueError, match="expected 12 values"):
        rows(np.zeros(16), CPU, 3, 4, "x")
    with pytest.raises(ValueError, match="s has shape"):
        rows(np.zeros((3, 5)), CPU, 3, 4, "s")


def test_packed_layout_round_trip():
    """The packed layout of an uneven batch: each array is the concatenation
    of the per-instance row-major arrays in instance order; `sizes` gives
    the per-instance lengths of Q, q, A, b, G, h and `unpack` inverts `pack`."""
    from qpax_b200 import workloads as wl
    from qpax_b200.packed import pack, sizes, unpack

    data = wl.uneven(7, n_min=3, n_max=9, chunk=4)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    L = sizes(shapes)
    for k, arrays in enumerate(data):
        np.testing.assert_array_equal(L[k], [a.size for a in arrays])
        t = pack(arrays, CPU)
        assert t.dtype == torch.float64 and t.dim() == 1 and t.numel() == int(np.sum(L[k]))
        parts = unpack(t, L[k], [a.shape for a in arrays])
        for a, p in zip(arrays, parts):
            np.testing.assert_array_equal(p.numpy(), a)
    assert pack([], CPU).numel() == 0
