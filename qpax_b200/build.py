"""Builds libqpb.so (the CUDA library behind include/qpb.h) in-tree for sm_100a.

    python -m qpax_b200.build [--force] [--jobs N]

Each translation unit under csrc/ compiles in its own nvcc process (they are
independent), objects land in qpax_b200/_build/, and the shared library is
written to qpax_b200/libqpb.so.  Rebuilds are incremental on file times.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqpb.so")
# the benchmark's FMA-throughput helper: a library of its own, not product code
PEAK_SOURCES = ["qpb_peak.cu"]
PEAK_LIB = os.path.join(HERE, "libqpb_peak.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

SOURCES = [
    "qpb_capi.cu",
    "qpb_kern_std_f64.cu",
    "qpb_kern_std_mixed.cu",
    "qpb_kern_elastic_f64.cu",
    "qpb_kern_elastic_mixed.cu",
    "qpb_kern_warp.cu",
    "qpb_kern_warp_mixed.cu",
    "qpb_noalloc.cu",
    "qpb_plan.cu",
    "qpb_host_pipeline.cu",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libqpb.so")


def _deps_mtime() -> float:
    files = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    files += glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(f) for f in files)


def _compile(src: str, force: bool, extra: list[str]) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    if not force and os.path.exists(obj):
        if os.path.getmtime(obj) >= max(os.path.getmtime(path), _deps_mtime()):
            return obj
    cmd = [nvcc()] + FLAGS + extra + ["-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    return obj


def _link(lib: str, objs: list[str], force: bool) -> None:
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")


def build(force: bool = False, jobs: int | None = None, extra: list[str] | None = None) -> str:
    """Compile every CUDA translation unit for sm_100a and link libqpb.so (and
    the benchmark's libqpb_peak.so)."""
    os.makedirs(OBJ, exist_ok=True)
    extra = list(extra or [])
    srcs = SOURCES + PEAK_SOURCES
    jobs = jobs or min(len(srcs), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, extra), srcs))
    _link(LIB, objs[: len(SOURCES)], force)
    _link(PEAK_LIB, objs[len(SOURCES):], force)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, extra=["-Xptxas", "-v"] if a.ptxas_verbose else None))


if __name__ == "__main__":
    main()
