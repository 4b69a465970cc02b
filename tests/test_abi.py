"""The C ABI library without a GPU: it loads, exports every symbol
include/qpb.h declares, and rejects malformed calls before any CUDA work."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from qpax_b200 import _lib as L
    from qpax_b200 import build

    if not os.path.exists(L.LIB_PATH):
        build.build()
    return L.load()


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "qpb.h")).read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(qpb_\w+)\s*\(", src, flags=re.M)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 13
    for name in names:
        assert hasattr(lib, name), name


def test_version_and_status_strings(lib):
    assert lib.qpb_version() >= 100
    assert lib.qpb_status_string(0) == b"ok"
    assert b"workspace" in lib.qpb_status_string(3)


def _solve(lib, dims, cfg=None, **ptrs):
    from qpax_b200._lib import Dims

    d = ctypes.byref(dims) if isinstance(dims, Dims) else None
    p = [ptrs.get(k, 8) for k in ("Q", "q", "A", "b", "G", "h")]
    o = [ptrs.get(k, 8) for k in ("x", "s", "z", "y", "conv", "iters")]
    return lib.qpb_solve_qp(d, *p, ctypes.c_double(1e-6), *o, cfg, 256, 1 << 20, None)


def test_rejects_bad_arguments_before_launch(lib):
    from qpax_b200._lib import Config, Dims

    assert _solve(lib, None) == 1                          # null dims
    assert _solve(lib, Dims(4, 0, 0, 3)) == 1              # n < 1
    assert _solve(lib, Dims(-1, 3, 0, 3)) == 1             # negative batch
    assert _solve(lib, Dims(4, 300, 0, 3)) == 2            # n above the supported 256
    assert _solve(lib, Dims(4, 3, 0, 3), Q=None) == 1      # missing input
    assert _solve(lib, Dims(4, 3, 0, 3), x=12) == 1        # misaligned output
    bad = Config(7, 0, 0.0, 0, None)
    assert _solve(lib, Dims(4, 3, 0, 3), ctypes.byref(bad)) == 1  # unknown precision
    bad = Config(0, 64, 0.0, 0, None)
    assert _solve(lib, Dims(4, 3, 0, 3), ctypes.byref(bad)) == 1  # unsupported team size


def test_relax_without_inequalities_is_unsupported(lib):
    from qpax_b200._lib import Dims

    d = Dims(2, 3, 1, 0)
    args = [8] * 10 + [ctypes.c_double(1e-5), ctypes.c_double(1e-3)] + [8] * 6
    assert lib.qpb_relax_qp(ctypes.byref(d), *args, None, 256, 1 << 20, None) == 2
    assert lib.qpb_workspace_size(2, ctypes.byref(d), None) == 0


def test_elastic_requires_no_equalities(lib):
    from qpax_b200._lib import Dims

    d = Dims(2, 3, 1, 4)
    args = [8] * 5 + [ctypes.c_double(1e-5)] + [8] * 8
    assert lib.qpb_solve_qp_elastic(ctypes.byref(d), *args, None, 256, 1 << 20, None) == 1


def test_api_refuses_to_run_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import qpax_b200 as qb
    from qpax_b200._lib import QpbError

    with pytest.raises(QpbError):
        qb.solve_qp([[1.0]], [1.0], [[0.0]][:0], [], [[1.0]], [1.0])


def test_host_pipeline_rejects_bad_arguments(lib):
    """qpb_solve_qp_primal_vjp_host checks its arguments on the host before any
    copy or launch."""
    from qpax_b200._lib import Dims

    def call(dims, chunks=2, **over):
        names = ["Q", "q", "A", "b", "G", "h", "dl", "x", "dQ", "dq", "dA", "db", "dG", "dh"]
        ptrs = [over.get(k, 8) for k in names]
        d = ctypes.byref(dims) if dims is not None else None
        return lib.qpb_solve_qp_primal_vjp_host(d, *ptrs[:7], ctypes.c_double(1e-5), ctypes.c_double(1e-3),
                                                *ptrs[7:], None, None, chunks, None, 256, 1 << 20, None)

    assert call(None) == 1                              # null dims
    assert call(Dims(4, 3, 1, 2), chunks=0) == 1        # no chunks
    assert call(Dims(4, 3, 1, 0)) == 2                  # qpax's relax / VJP need inequalities
    assert call(Dims(4, 3, 1, 2), G=None) == 1          # missing input
    assert call(Dims(4, 3, 1, 2), dG=12) == 1           # misaligned output
    assert call(Dims(0, 3, 1, 2)) == 0                  # empty batch: nothing to do
    assert lib.qpb_solve_qp_primal_vjp_host_workspace_size(ctypes.byref(Dims(4, 3, 1, 2)), 0, None) == 0
