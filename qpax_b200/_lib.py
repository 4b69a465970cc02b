"""ctypes binding of libqpb.so (include/qpb.h) and tensor plumbing.

The library is the only compute path: if libqpb.so is missing or no CUDA
device is present, every solver entry point raises -- there is no CPU path.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqpb.so")

QPB_OK = 0
OPS = {
    "solve": 0, "initialize": 1, "relax": 2, "primal_bwd": 3, "diff": 4,
    "elastic_solve": 5, "elastic_initialize": 6, "elastic_relax": 7, "elastic_primal_bwd": 8, "elastic_diff": 9,
}
PRECISION = {"auto": 0, "mixed": 1, "fp64": 2}

_lock = threading.Lock()
_lib = None


class QpbError(RuntimeError):
    """A libqpb entry point returned a non-zero qpb_status."""


class Dims(ctypes.Structure):
    _fields_ = [("batch", ctypes.c_int32), ("n", ctypes.c_int32), ("m", ctypes.c_int32), ("p", ctypes.c_int32)]


class Config(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int32),
        ("team_threads", ctypes.c_int32),
        ("pivot_max", ctypes.c_double),
        ("max_sweeps", ctypes.c_int32),
        ("stats", ctypes.c_void_p),
    ]


# argument kinds used to declare prototypes: P = pointer, D = double
_SIGS = {
    "qpb_solve_qp": "dims P P P P P P D P P P P P P cfg P S stream",
    "qpb_initialize": "dims P P P P P P P P P P cfg P S stream",
    "qpb_relax_qp": "dims P P P P P P P P P P D D P P P P P P cfg P S stream",
    "qpb_diff_qp": "dims P P P P P P P P P P P P P P P P P cfg P S stream",
    "qpb_solve_qp_primal_bwd": "dims P P P P P P P P P P P D D P P P P P P P P P P P P cfg P S stream",
    "qpb_solve_qp_elastic": "dims P P P P P D P P P P P P P P cfg P S stream",
    "qpb_initialize_elastic": "dims P P P P P P P P P P P cfg P S stream",
    "qpb_relax_qp_elastic": "dims P P P P P A6 D D A6 P P cfg P S stream",
    "qpb_diff_qp_elastic": "dims P P P P P A6 P P P P P cfg P S stream",
    "qpb_solve_qp_elastic_primal_bwd": "dims P P P P P A6 P D D P P P P cfg P S stream",
    "qpb_tune_solve_qp": "dims P P P P P P D P P P P P P cfg P S stream",
    "qpb_tune_solve_qp_elastic": "dims P P P P P D P P P P P P P P cfg P S stream",
    "qpb_solve_qp_primal_vjp_host": "dims P P P P P P P D D P P P P P P P P P I cfg P S stream",
}
_CT = {
    "dims": ctypes.POINTER(Dims), "cfg": ctypes.POINTER(Config), "P": ctypes.c_void_p, "D": ctypes.c_double,
    "S": ctypes.c_size_t, "stream": ctypes.c_void_p, "A6": ctypes.POINTER(ctypes.c_void_p), "I": ctypes.c_int32,
}


def load() -> ctypes.CDLL:
    """Load libqpb.so, raising if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise QpbError(f"{LIB_PATH} is missing: build it with `python -m qpax_b200.build` (nvcc, sm_100a)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, sig in _SIGS.items():
                fn = getattr(lib, name)
                fn.argtypes = [_CT[k] for k in sig.split()]
                fn.restype = ctypes.c_int
            lib.qpb_workspace_size.argtypes = [ctypes.c_int32, ctypes.POINTER(Dims), ctypes.POINTER(Config)]
            lib.qpb_workspace_size.restype = ctypes.c_size_t
            lib.qpb_tune_workspace_size.argtypes = [ctypes.c_int32, ctypes.POINTER(Dims), ctypes.POINTER(Config)]
            lib.qpb_tune_workspace_size.restype = ctypes.c_size_t
            lib.qpb_solve_qp_primal_vjp_host_workspace_size.argtypes = [ctypes.POINTER(Dims), ctypes.c_int32,
                                                                        ctypes.POINTER(Config)]
            lib.qpb_solve_qp_primal_vjp_host_workspace_size.restype = ctypes.c_size_t
            lib.qpb_status_string.argtypes = [ctypes.c_int]
            lib.qpb_status_string.restype = ctypes.c_char_p
            lib.qpb_version.restype = ctypes.c_int32
            _lib = lib
    return _lib


def exported_symbols() -> list[str]:
    return ["qpb_workspace_size", "qpb_tune_workspace_size", "qpb_status_string", "qpb_version",
            "qpb_solve_qp_primal_vjp_host_workspace_size"] + list(_SIGS)


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise QpbError("qpax_b200 needs a CUDA device (B200, sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def as_f64(a, dev: torch.device) -> torch.Tensor:
    t = torch.as_tensor(a)
    if t.dtype != torch.float64 or t.device != dev:
        t = t.to(device=dev, dtype=torch.float64)
    return t.contiguous()


def rows(a, dev: torch.device, B: int, width: int, name: str) -> torch.Tensor:
    """`a` as a contiguous float64 (B, width) tensor on `dev`, refusing any
    other element count: the kernels read exactly B * width values of it."""
    t = as_f64(a, dev)
    if t.numel() != B * width:
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {B * width} values ({B} x {width})")
    return t.reshape(B, width).contiguous()


def ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr() if t.numel() else None


def make_config(precision: str = "auto", team_threads: int = 0, pivot_max: float = 0.0, max_sweeps: int = 0,
                stats: torch.Tensor | None = None) -> Config:
    if precision not in PRECISION:
        raise ValueError(f"precision must be one of {sorted(PRECISION)}")
    return Config(PRECISION[precision], team_threads, pivot_max, max_sweeps, ptr(stats))


def workspace(op: str, dims: Dims, cfg: Config, dev: torch.device, tune: bool = False) -> torch.Tensor:
    lib = load()
    size = lib.qpb_tune_workspace_size if tune else lib.qpb_workspace_size
    nbytes = size(OPS[op], ctypes.byref(dims), ctypes.byref(cfg))
    if nbytes == 0:
        raise QpbError(f"unsupported problem for {op}: batch={dims.batch} n={dims.n} m={dims.m} p={dims.p}")
    return torch.empty(int(nbytes) + 256, dtype=torch.uint8, device=dev)


def aligned(ws: torch.Tensor) -> tuple[int, int]:
    base = ws.data_ptr()
    off = (-base) % 256
    return base + off, ws.numel() - off


def call(name: str, *args) -> None:
    lib = load()
    st = getattr(lib, name)(*args)
    if st != QPB_OK:
        raise QpbError(f"{name}: {lib.qpb_status_string(st).decode()} (status {st})")


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream
