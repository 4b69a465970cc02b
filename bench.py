"""Benchmark: QPs/sec, forward + backward, at 1e-6 KKT residual, one B200 per rank.

Default workload (one step): the differentiable batched solve of qpax
(solve_qp_primal) over 4096 dense QPs with n = 32, m = 8, p = 64 -- the
dense-QP configuration (Q = M'M + 1e-3 I, strictly feasible h = G x0 + s0),
solver_tol 1e-6, target_kappa 1e-3, loss ||x - 1||^2:
  forward  = qpb_solve_qp            (initialize + predictor-corrector loop)
  backward = qpb_solve_qp_primal_bwd (relaxation to kappa + adjoint KKT solve
             + the six gradient outer products)
Inputs are resident in HBM; L2 is flushed (256 MB write) between steps,
outside the per-step CUDA events.  Launch shapes of the default and mixed
arms are autotuned at setup (untimed); the plain FP64 arm keeps its fixed
one-CTA-per-QP shape.  Synthetic seeded data (no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dense|nnls|small|uneven|elastic] [--batch B]
                    [--no-e2e] [--no-cpu] [--no-parity] [--no-tune] [--no-configs]
                    [--only-default] [--e2e-chunks C] [--config-steps K]

The JSON line carries the default path's `value`, the plain FP64
one-CTA-per-QP and mixed variants (`variants`, `mixed_over_plain_fp64`),
`parity` against the FP64 oracle per variant (computed after the timed
steps), `e2e` from pinned host buffers, `roofline`, `cpu_baseline`, and for
the dense workload a `configs` block with the other four configurations
(value, e2e, parity each):
  nnls     10000 non-negative least squares QPs, n = 5, G = -I, no equalities
  small    2048 dense QPs n = 16, m = 4, p = 32, solver_tol 1e-5
  uneven   16384 QPs of different sizes: n ~ U{4..256}, p = 2n,
           m ~ U{0..n/4}, one packed call (size-binned plan, CUDA graph)
  elastic  1024 elastic QPs (solve_qp_elastic_primal) n = 64, p = 128,
           penalty 1e3, 30% of them infeasible
`--workload X` runs one of them alone, with its variants.

--impl reference times the FP64 CPU restatement of qpax (oracle/) on the
host cores, on the same workload -- qpax itself (JAX) is not installable
here.  Multi-GPU: one process per GPU, each rank solves its own batch (weak
scaling, no collective on the data path); time = max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import time
from dataclasses import dataclass

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPs/sec fwd+bwd at 1e-6 KKT residual, mixed vs plain FP64 kernel, 1 B200"
KAPPA = 1e-3


@dataclass
class Spec:
    key: str
    kind: str          # "uniform" | "uneven" | "elastic"
    batch: int
    n: int
    m: int
    p: int
    tol: float
    workload: str


WORKLOADS = {
    "dense": Spec("dense", "uniform", 4096, 32, 8, 64, 1e-6,
                  "dense QP n=32 m=8 p=64, batch 4096/GPU, solve_qp_primal forward+backward, tol 1e-6, kappa 1e-3"),
    "nnls": Spec("nnls", "uniform", 10000, 5, 0, 5, 1e-6,
                 "NNLS QP n=5 (Q=F'F, F 10x5), G=-I, no equalities, batch 10000/GPU, solve_qp_primal "
                 "forward+backward, tol 1e-6, kappa 1e-3"),
    "small": Spec("small", "uniform", 2048, 16, 4, 32, 1e-5,
                  "dense QP n=16 m=4 p=32, batch 2048/GPU, solve_qp_primal forward+backward, tol 1e-5, kappa 1e-3"),
    "uneven": Spec("uneven", "uneven", 16384, 256, 64, 512, 1e-6,
                   "uneven batch of 16384 QPs/GPU, n~U{4..256}, p=2n, m~U{0..n/4}, one packed call, "
                   "solve_qp_primal forward+backward, tol 1e-6, kappa 1e-3"),
    "elastic": Spec("elastic", "elastic", 1024, 64, 0, 128, 1e-6,
                    "elastic QP n=64 p=128 penalty 1e3 (30% infeasible), batch 1024/GPU, solve_qp_elastic_primal "
                    "forward+backward, tol 1e-6, kappa 1e-3"),
}


def make_data(spec: Spec):
    """Host (numpy) inputs of the workload, seeded."""
    from qpax_b200 import workloads as wl

    if spec.key == "dense":
        return wl.config2(spec.batch)
    if spec.key == "small":
        return wl.config3(spec.batch)
    if spec.key == "nnls":
        return wl.nnls(spec.batch)
    if spec.key == "uneven":
        return wl.uneven(spec.batch)
    Q, q, G, h, _ = wl.elastic(spec.batch)
    return Q, q, G, h


def shapes_of(spec: Spec, data):
    """Per-instance (n, m, p) as int arrays."""
    if spec.kind == "uneven":
        n = np.array([len(v) for v in data[1]])
        m = np.array([len(v) for v in data[3]])
        p = np.array([len(v) for v in data[5]])
        return n, m, p
    B = spec.batch
    return np.full(B, spec.n), np.full(B, spec.m), np.full(B, spec.p)


def algorithmic_flops(n, m, p, iters_fwd, iters_relax):
    """Algorithmic FLOPs (FMA = 2, symmetric-aware) of one forward + backward
    per instance: initialize + iters_fwd predictor-corrector iterations,
    iters_relax relaxation iterations and the adjoint (one factor + one solve
    + outer products).  Elastic QPs are counted with m = 0 (their reduced
    system is the n x n matrix Q + G' diag(w) G over p rows)."""
    n, m, p = (np.asarray(v, dtype=np.float64) for v in (n, m, p))
    f_fac = p * n * (n + 1) + n ** 3 / 3 + 2 * m * n * n + m * (m + 1) * n + m ** 3 / 3
    f_sol = 4 * n * n + 2 * m * m + 4 * m * n + 4 * p * n + 6 * p
    res = 2 * n * n + 4 * m * n + 4 * p * n
    pc = res + f_fac + 2 * f_sol + 30 * (n + m + p)
    rlx = res + f_fac + f_sol + 20 * (n + m + p)
    init = f_fac + f_sol
    adj = f_fac + f_sol + 2 * n * n + 2 * m * n + 2 * p * n
    fwd = init + iters_fwd * pc
    bwd = iters_relax * rlx + adj
    return fwd, bwd


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier_max(val, world):
    from qpax_b200.shard import max_over_ranks

    return max_over_ranks(val) if world > 1 else val


def barrier(world):
    from qpax_b200.shard import barrier as _barrier

    if world > 1:
        _barrier()


# ------------------------------------------------------------- CPU (oracle)

def _oracle_chunk(spec: Spec, data, lo, hi, nthreads):
    """The oracle's forward + backward on instances [lo, hi) of the workload."""
    from oracle import oracle

    if spec.kind == "uneven":
        part = [v[lo:hi] for v in data]
        dl = [np.full(len(q), 0.1) for q in part[1]]
        oracle.solve_qp_primal_vjp(*part, dl, solver_tol=spec.tol, target_kappa=KAPPA, nthreads=nthreads)
    elif spec.kind == "elastic":
        Q, q, G, h = (a[lo:hi] for a in data)
        dl = np.full((hi - lo, spec.n), 0.1)
        oracle.solve_qp_elastic_primal_vjp(Q, q, G, h, np.full(hi - lo, 1e3), dl, solver_tol=spec.tol,
                                           target_kappa=KAPPA, nthreads=nthreads)
    else:
        part = [a[lo:hi] for a in data]
        dl = np.full((hi - lo, spec.n), 0.1)
        oracle.solve_qp_primal_vjp(*part, dl, solver_tol=spec.tol, target_kappa=KAPPA, nthreads=nthreads)


def cpu_sample(spec: Spec, data, seconds, nthreads, chunk):
    """Oracle forward + backward on consecutive chunks of the workload (wrapping
    around) until `seconds` elapse -> (QPs/s, QPs done, seconds)."""
    B = spec.batch
    done, t0, lo = 0, time.perf_counter(), 0
    while True:
        hi = min(lo + chunk, B)
        _oracle_chunk(spec, data, lo, hi, nthreads)
        done += hi - lo
        lo = 0 if hi == B else hi
        el = time.perf_counter() - t0
        if el >= seconds:
            return done / el, done, el


def cpu_baseline(spec: Spec, data):
    """The oracle (FP64 C restatement of qpax, OpenMP over instances) on all
    host threads (~12 s sample) and on one thread (~4 s sample)."""
    from oracle import oracle

    cores = oracle.num_threads()
    chunk = {"uneven": 256, "elastic": 256}.get(spec.kind, 1024)
    v, done, el = cpu_sample(spec, data, 12.0, 0, chunk)
    v1, done1, el1 = cpu_sample(spec, data, 4.0, 1, 16)
    return {"value": v, "unit": "QPs/s", "cores": cores, "kind": "port",
            "sample": f"{done} QPs of the workload in order (chunks of {chunk}), {el:.1f} s wall, forward+backward",
            "single_thread": {"value": v1, "unit": "QPs/s", "cores": 1,
                              "sample": f"{done1} QPs in order, {el1:.1f} s wall"}}


def run_reference(args, spec: Spec, world, rank):
    from oracle import oracle

    if rank != 0:
        return
    data = make_data(spec)
    B = spec.batch
    # each step is a bounded sample of the workload: the whole batch when it
    # is cheap on the host, else a fixed in-order slice of it
    per_step = {"uneven": 128, "elastic": 256}.get(spec.kind, B)
    per_step = min(per_step, B)
    step = lambda: _oracle_chunk(spec, data, 0, per_step, 0)
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    val = per_step * args.steps / el
    cores = oracle.num_threads()
    line = {
        "impl": "reference", "metric": metric_for(spec), "value": val, "unit": "QPs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_for(spec, world),
        "cpu_baseline": {"value": val, "unit": "QPs/s", "cores": cores, "kind": "port",
                         "sample": f"the first {per_step} QPs of the batch per step, {args.steps} steps"},
        "e2e": {"value": val, "unit": "QPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "qpax (JAX) is not installable offline; the timed CPU implementation is the FP64 C "
                "restatement of qpax in oracle/ (pinned to qpax's golden vectors and tests)",
    }
    print(json.dumps(line), flush=True)


def metric_for(spec: Spec):
    if spec.key == "dense":
        return METRIC
    return f"QPs/sec fwd+bwd at {spec.tol:g} KKT residual, 1 B200"


def config_for(spec: Spec, world, extra=None):
    cfg = {"workload": spec.workload, "global_batch": spec.batch * world}
    if spec.kind == "uneven":
        cfg.update({"n": "U{4..256}", "m": "U{0..n/4}", "p": "2n"})
    else:
        cfg.update({"n": spec.n, "m": spec.m, "p": spec.p})
    cfg.update(extra or {})
    return cfg


def load_traffic(spec: Spec):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
    workload's forward and backward launches, from a committed ncu summary
    ("key value" lines), when one exists."""
    name = {"dense": "traffic_dense_qp_n32_b4096.txt"}.get(spec.key)
    path = os.path.join(ROOT, "profiles", name) if name else None
    if not path or not os.path.exists(path):
        return None
    out = {"source": "profiles/" + name}
    for ln in open(path):
        parts = ln.split()
        if len(parts) == 2 and parts[0] in ("forward", "backward"):
            try:
                out[parts[0]] = float(parts[1])
            except ValueError:
                pass
    return out


# ------------------------------------------------------------- GPU arms

class UniformArm:
    """solve_qp forward + solve_qp_primal backward on a uniform batch, through
    the C ABI with preallocated outputs (one launch each)."""

    def __init__(self, spec: Spec, data, dev, opts):
        import torch

        from qpax_b200.pdip import StdBatch, _config

        self.spec, self.opts = spec, opts
        self.dev_in = [torch.tensor(a, device=dev) for a in data]
        self.bt = bt = StdBatch(*self.dev_in)
        self.cfg = _config(opts)
        B, n, m, p = spec.batch, spec.n, spec.m, spec.p
        self.x, self.s, self.z, self.y = bt.new(B, n), bt.new(B, p), bt.new(B, p), bt.new(B, m)
        self.conv, self.iters = bt.new(B, dtype=torch.int32), bt.new(B, dtype=torch.int32)
        self.rconv, self.riters = bt.new(B, dtype=torch.int32), bt.new(B, dtype=torch.int32)
        self.gx = torch.empty(B, n, dtype=torch.float64, device=dev)
        self.grads = None
        self.launches = 2
        if opts.get("tune"):  # launch shape timed and recorded for these dims (untimed setup)
            import qpax_b200 as qb

            qb.tune_solve_qp(*self.dev_in, spec.tol, precision=opts.get("precision"))

    def fwd(self):
        from qpax_b200.pdip import _run

        _run("qpb_solve_qp", "solve", self.bt, self.cfg, [ctypes.c_double(self.spec.tol)],
             [t.data_ptr() for t in (self.x, self.s, self.z, self.y, self.conv, self.iters)])

    def bwd(self):
        import torch

        from qpax_b200.diff_qp import diff_qp_from_forward

        torch.mul(self.x - 1.0, 2.0, out=self.gx)
        self.grads = diff_qp_from_forward(self.bt, self.x, self.s, self.z, self.y, self.gx, self.spec.tol, KAPPA,
                                          self.opts, relaxed=[None, None, None, None, self.rconv, self.riters])

    def counts(self):
        return self.conv.cpu().numpy(), self.iters.cpu().numpy(), self.riters.cpu().numpy()

    def parity(self, data, limit=None):
        """Figures of the last step's outputs against the oracle, given the same dl/dx."""
        from oracle import parity

        dl = self.gx.cpu().numpy()
        gpu = dict(x=self.x.cpu().numpy(), s=self.s.cpu().numpy(), z=self.z.cpu().numpy(), y=self.y.cpu().numpy(),
                   conv=self.conv.cpu().numpy(), iters=self.iters.cpu().numpy(), riters=self.riters.cpu().numpy(),
                   grads=[g.cpu().numpy() for g in self.grads])
        eps = 1e-12 if self.opts.get("precision") == "mixed" else 1e-15
        return parity.standard(data, self.spec.tol, KAPPA, dl, gpu, perturb=2, eps=eps)[0]

    def kernel_name(self, which):
        return "qpb_solve_qp (forward)" if which == "forward" else "qpb_solve_qp_primal_bwd (backward)"

    def precision_stats(self):
        """Per-instance FP32 / FP64 factorisations and FP64 refinement sweeps of
        one forward solve and one relaxation (the optional stats output of the
        C ABI), as means over the batch; untimed."""
        import torch

        import qpax_b200 as qb

        B = self.spec.batch
        out = {}
        st = torch.zeros(B, 4, dtype=torch.int32, device=self.x.device)
        x, s, z, y, _, _ = qb.solve_qp(*self.dev_in, self.spec.tol, precision=self.opts.get("precision"), stats=st)
        out["forward"] = st.double().mean(0).tolist()
        fwd_flags = st[:, 3].cpu().numpy()
        st.zero_()
        qb.relax_qp(*self.dev_in, x, s, z, y, self.spec.tol, KAPPA, precision=self.opts.get("precision"), stats=st)
        out["relaxation"] = st.double().mean(0).tolist()
        res = {k: {"fp32_factorisations": v[0], "fp64_factorisations": v[1], "refinement_sweeps": v[2]}
               for k, v in out.items()}
        res["forward"]["share_with_fp32_factor_rejected"] = float(((fwd_flags & 1) != 0).mean())
        res["note"] = "means per instance; FP64 refactor when the FP32 pivot ratio exceeds pivot_max or refinement stalls"
        return res


class ElasticArm:
    """solve_qp_elastic forward + solve_qp_elastic_primal backward."""

    def __init__(self, spec: Spec, data, dev, opts):
        import torch

        from qpax_b200.elastic_qp import ElasticBatch

        self.spec, self.opts = spec, opts
        self.dev_in = [torch.tensor(a, device=dev) for a in data]
        self.pen = torch.full((spec.batch,), 1e3, dtype=torch.float64, device=dev)
        self.bt = ElasticBatch(*self.dev_in, self.pen)
        self.gx = torch.empty(spec.batch, spec.n, dtype=torch.float64, device=dev)
        self.out = None
        self.grads = None
        self.launches = 2
        self.opts = {k: v for k, v in opts.items() if k != "tune"}
        if opts.get("tune"):
            import qpax_b200 as qb

            qb.tune_solve_qp_elastic(*self.dev_in, self.pen, spec.tol, precision=opts.get("precision"))

    def fwd(self):
        import qpax_b200 as qb

        self.out = qb.solve_qp_elastic(*self.dev_in, self.pen, self.spec.tol, **self.opts)

    def bwd(self):
        import torch

        from qpax_b200.elastic_qp import _elastic_bwd

        torch.mul(self.out[0] - 1.0, 2.0, out=self.gx)
        self.grads = _elastic_bwd(self.bt, [t.contiguous() for t in self.out[:6]], self.gx, self.spec.tol, KAPPA,
                                  self.opts)

    def counts(self):
        import qpax_b200 as qb

        conv, iters = self.out[6].cpu().numpy(), self.out[7].cpu().numpy()
        rel = qb.relax_qp_elastic(*self.dev_in, self.pen, *self.out[:6], self.spec.tol, KAPPA, **self.opts)
        return conv, iters, rel[7].cpu().numpy()

    def parity(self, data, limit=None):
        from oracle import parity

        eps = 1e-12 if self.opts.get("precision") == "mixed" else 1e-15
        return parity.elastic(tuple(data), 1e3, self.spec.tol, KAPPA, self.gx.cpu().numpy(),
                              [t.cpu().numpy() for t in self.out], [g.cpu().numpy() for g in self.grads], perturb=2,
                              eps=eps, g_bar=1e-4)[0]

    def kernel_name(self, which):
        return ("qpb_solve_qp_elastic (forward)" if which == "forward"
                else "qpb_solve_qp_elastic_primal_bwd (backward)")


class UnevenArm:
    """Packed plan: every size bin of the batch launched concurrently.  The
    forward call and the backward call (with the loss gradient between them)
    are each captured once in a CUDA graph and replayed every step."""

    def __init__(self, spec: Spec, data, dev, opts):
        import torch

        from qpax_b200.packed import PackedPlan, pack

        self.spec = spec
        n, m, p = shapes_of(spec, data)
        self.precision = opts.get("precision") or "auto"
        self.plan = PackedPlan(list(zip(n, m, p)), precision=self.precision,
                               team_threads=opts.get("team_threads") or 0)
        self.ins = [pack(v, dev) for v in data]
        if opts.get("tune"):
            self.plan.tune(*self.ins, spec.tol)
        B = spec.batch
        self.rconv = torch.empty(B, dtype=torch.int32, device=dev)
        self.riters = torch.empty(B, dtype=torch.int32, device=dev)
        self.gx = torch.empty(self.plan.totals[1], dtype=torch.float64, device=dev)
        self.launches = 2 * self.plan.num_bins
        # eager warm-up on a side stream, then capture forward and backward
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            self._fwd_eager()
            self._bwd_eager()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.g_fwd, self.g_bwd = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.g_fwd):
            self._fwd_eager()
        with torch.cuda.graph(self.g_bwd, pool=self.g_fwd.pool()):
            self._bwd_eager()
        torch.cuda.synchronize(dev)

    def _fwd_eager(self):
        self.out = self.plan.solve(*self.ins, self.spec.tol)

    def _bwd_eager(self):
        import torch

        torch.mul(self.out[0] - 1.0, 2.0, out=self.gx)
        self.grads = self.plan.primal_bwd(*self.ins, *self.out[:4], self.gx, self.spec.tol, KAPPA,
                                          relax_out=(self.rconv, self.riters))

    def fwd(self):
        self.g_fwd.replay()

    def bwd(self):
        self.g_bwd.replay()

    def release(self):
        self.g_fwd, self.g_bwd = None, None

    def counts(self):
        return self.out[4].cpu().numpy(), self.out[5].cpu().numpy(), self.riters.cpu().numpy()

    def parity(self, data, limit=512):
        """Oracle figures on the first `limit` instances (the oracle takes ~50 ms
        per large instance on one core)."""
        from oracle import parity
        from qpax_b200.packed import unpack

        k = min(limit, self.spec.batch)
        L = self.plan.lengths
        cut = lambda t, f: [v.cpu().numpy() for v in unpack(t, L[f])[:k]]
        sub = [v[:k] for v in data]
        gpu = dict(x=cut(self.out[0], 1), s=cut(self.out[1], 5), z=cut(self.out[2], 5), y=cut(self.out[3], 3),
                   conv=self.out[4][:k].cpu().numpy(), iters=self.out[5][:k].cpu().numpy(),
                   riters=self.riters[:k].cpu().numpy(), grads=[cut(self.grads[f], f) for f in range(6)])
        fig = parity.standard(sub, self.spec.tol, KAPPA, cut(self.gx, 1), gpu, perturb=2,
                              eps=1e-12 if self.precision == "mixed" else 1e-15)[0]
        fig["sample"] = f"the first {k} instances of the batch"
        return fig

    def kernel_name(self, which):
        return (f"qpb_solve_qp_packed: {self.plan.num_bins} size-bin kernels, concurrent, CUDA graph (forward)"
                if which == "forward" else
                f"qpb_solve_qp_primal_bwd_packed: {self.plan.num_bins} size-bin kernels, concurrent, CUDA graph "
                "(backward)")


ARMS = {"uniform": UniformArm, "elastic": ElasticArm, "uneven": UnevenArm}


def variants_for(spec: Spec, tune=True):
    v = {"auto": dict(precision="auto", tune=tune)}
    if spec.kind != "elastic":
        v["fp64_cta"] = dict(precision="fp64", team_threads=128)  # plain FP64, one QP per CTA
    v["mixed"] = dict(precision="mixed", tune=tune)               # FP32 factor + FP64 refinement
    return v


VARIANT_NAMES = {"auto": "default", "fp64_cta": "fp64_one_cta_per_qp", "mixed": "mixed_fp32_factor_fp64_refinement"}


def time_arm(args, arm, stream, flush, world, steps, sampler=None):
    """W warm-up steps, then `steps` timed steps (forward, backward), L2 flushed
    between steps outside the per-step events; device time, max over ranks."""
    import torch

    for _ in range(args.warmup):
        arm.fwd()
        arm.bwd()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    if sampler:
        sampler.__enter__()
    for k in range(steps):
        flush.fill_(float(k))
        evs[k][0].record(stream)
        arm.fwd()
        evs[k][1].record(stream)
        arm.bwd()
        evs[k][2].record(stream)
    torch.cuda.synchronize()
    if sampler:
        sampler.__exit__(None, None, None)
    barrier(world)
    fwd_ms = [e[0].elapsed_time(e[1]) for e in evs]
    bwd_ms = [e[1].elapsed_time(e[2]) for e in evs]
    tot = barrier_max(sum(f + b for f, b in zip(fwd_ms, bwd_ms)), world)
    return tot, float(np.mean(fwd_ms)), float(np.mean(bwd_ms))


def run_ours(args, spec: Spec, world, rank, local):
    import torch

    from qpax_b200 import _lib

    _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    data = make_data(spec)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    results = {}
    variants = variants_for(spec, tune=not args.no_tune)
    if args.only_default:
        variants = {"auto": variants["auto"]}
    arm_main = None
    for prec, opts in variants.items():
        arm = ARMS[spec.kind](spec, data, dev, opts)
        sampler = ClockSampler(local) if prec == "auto" else None
        tot, fwd_ms, bwd_ms = time_arm(args, arm, stream, flush, world, args.steps, sampler)
        conv, iters, riters = arm.counts()
        # the oracle checks (host work on rank 0 while the other ranks wait at
        # the next barrier) run in single-GPU runs only
        par = arm.parity(data) if (world == 1 and not args.no_parity) else None
        pstats = arm.precision_stats() if (prec == "mixed" and hasattr(arm, "precision_stats")) else None
        results[prec] = dict(total_ms=tot, fwd_ms=fwd_ms, bwd_ms=bwd_ms, conv=conv, iters=iters, riters=riters,
                             clocks=sampler.summary() if sampler else None, parity=par, pstats=pstats)
        if prec == "auto":
            arm_main = arm
        else:
            if hasattr(arm, "release"):
                arm.release()
            del arm

    B = spec.batch
    main_r = results["auto"]
    value = world * B * args.steps / (main_r["total_ms"] * 1e-3)
    n, m, p = shapes_of(spec, data)
    f_fwd, f_bwd = algorithmic_flops(n, m, p, main_r["iters"].astype(np.float64), main_r["riters"].astype(np.float64))
    fl = {"forward": float(f_fwd.sum()), "backward": float(f_bwd.sum())}
    dom_key = "forward" if main_r["fwd_ms"] >= main_r["bwd_ms"] else "backward"
    dom_ms = main_r["fwd_ms"] if dom_key == "forward" else main_r["bwd_ms"]
    achieved = fl[dom_key] / (dom_ms * 1e-3) / 1e12
    peaks, peak_src = load_peaks()
    simt = simt_peaks()
    traffic = load_traffic(spec)
    roof = {
        "bound": "fp64", "kernel": arm_main.kernel_name(dom_key), "achieved": achieved, "unit": "TFLOP/s",
        "peak": peaks["bf16_tflops"], "frac": achieved / peaks["bf16_tflops"],
        "peak_source": f"bf16 dense tensor peak of MEASURED_PEAKS.json ({peak_src}), the figure the benchmark "
                       "contract names; the kernel computes in FP64 (FMA pipe and FP64 tensor-core DMMA), whose "
                       "own roof is fp64_fma_peak",
        "fp64_fma_peak": simt["fp64_tflops"], "frac_of_fp64_fma_peak": achieved / simt["fp64_tflops"],
        "fp32_fma_peak": simt["fp32_tflops"], "fma_peak_source": simt["how"],
        "algorithmic_flops_per_launch": fl[dom_key], "avg_launch_ms": dom_ms,
        "traffic": (traffic or {}).get(dom_key),
        "traffic_source": (traffic or {}).get("source"),
    }
    prec_desc = {"uniform": "auto (FP64; four QPs per warp for n <= 8, one warp per QP for n <= 32, one CTA per QP "
                            "above)",
                 "elastic": "auto (FP64, one CTA per QP)",
                 "uneven": "auto (FP64; per size bin: four QPs per warp for n <= 8, one warp per QP for n <= 32, "
                           "one CTA per QP above)"}[spec.kind]
    line = {
        "metric": metric_for(spec), "value": value, "unit": "QPs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main_r["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_for(spec, world),
        "setup": {"precision": prec_desc, "parallelism": f"batch split x{world}",
                  "launch_shapes": "heuristic" if args.no_tune else "autotuned per size bin at setup (untimed)",
                  "l2": "flushed between steps (256 MB write), outside the per-step events"},
        "roofline": roof, "gpu_launches": arm_main.launches * args.steps,
        "iterations": {"forward_mean": float(main_r["iters"].mean()), "relax_mean": float(main_r["riters"].mean()),
                       "converged": float(main_r["conv"].mean())},
        "clocks": main_r["clocks"],
        "forward_ms": main_r["fwd_ms"], "backward_ms": main_r["bwd_ms"],
    }
    if len(results) > 1:
        v = {k: world * B * args.steps / (r["total_ms"] * 1e-3) for k, r in results.items()}
        line["variants"] = {VARIANT_NAMES[k]: {"value": v[k], "unit": "QPs/s", "ms_per_step": results[k]["total_ms"] /
                                               args.steps} for k in results if k != "auto"}
        plain = "fp64_cta" if "fp64_cta" in v else "auto"
        if "mixed" in v:
            line["mixed_over_plain_fp64"] = v["mixed"] / v[plain]
            if results["mixed"]["pstats"]:
                line["variants"][VARIANT_NAMES["mixed"]]["precision_stats"] = results["mixed"]["pstats"]
        line["default_over_plain_fp64"] = v["auto"] / v[plain]
    if world == 1 and not args.no_parity:
        line["parity"] = {VARIANT_NAMES[k]: r["parity"] for k, r in results.items()}
        line["parity"]["against"] = ("the FP64 oracle (C restatement of qpax) on the same inputs and the same dl/dx, "
                                     "computed after the timed steps; errors relative per instance, "
                                     "||gpu - ref||_inf / max(1, ||ref||_inf); objective 1/2 x'Qx + q'x; "
                                     "gpu_only_converged: instances where qpax's QR-based solve breaks down and the "
                                     "GPU converges (gpu_only_max_kkt: KKT residual of the GPU's returned iterate); "
                                     "'reproducible' = the oracle gives the same flag and iteration count (and a "
                                     "gradient within a tenth of the 1e-5 bar) on two runs with inputs perturbed by "
                                     "1e-15 relative (1e-12 for the mixed variant, whose solves are refined to 1e-12)")
    if not args.no_e2e:  # every rank takes part (barriers, max over ranks)
        e2e = run_e2e(args, spec, data, dev, arm_main, world)
        if rank == 0:
            line["e2e"] = e2e
    if hasattr(arm_main, "release"):
        arm_main.release()
    del arm_main
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(spec, data)
    if spec.key == "dense" and world == 1 and not args.no_configs:  # single-GPU runs
        line["configs"] = run_configs(args, world, rank, dev, stream, flush)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_configs(args, world, rank, dev, stream, flush):
    """The other four configurations on the default path, each with its own
    device-timed value, end-to-end value from host buffers and parity against
    the oracle (uneven: on its first 512 instances)."""
    import torch

    out = {}
    for key in ("nnls", "small", "uneven", "elastic"):
        spec = WORKLOADS[key]
        data = make_data(spec)
        arm = ARMS[spec.kind](spec, data, dev, dict(precision="auto", tune=not args.no_tune))
        steps = args.config_steps
        tot, fwd_ms, bwd_ms = time_arm(args, arm, stream, flush, world, steps)
        conv, iters, riters = arm.counts()
        entry = {"workload": spec.workload, "metric": metric_for(spec),
                 "launch_shapes": arm.plan.bin_info() if hasattr(arm, "plan") else None,
                 "value": world * spec.batch * steps / (tot * 1e-3), "unit": "QPs/s", "steps": steps,
                 "ms_per_step": tot / steps, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
                 "iterations": {"forward_mean": float(iters.mean()), "relax_mean": float(riters.mean()),
                                "converged": float(conv.mean())},
                 "gpu_launches": arm.launches * steps}
        if world == 1 and not args.no_parity:
            entry["parity"] = arm.parity(data)
        if not args.no_e2e:
            sub = argparse.Namespace(**vars(args))
            sub.steps = steps
            sub.e2e_chunks = E2E_CHUNKS[key]
            e2e = run_e2e(sub, spec, data, dev, arm, world)
            if rank == 0:
                entry["e2e"] = e2e
        if hasattr(arm, "release"):
            arm.release()
        del arm, data
        torch.cuda.empty_cache()
        out[key] = entry
    return out


def simt_peaks():
    """FP32 / FP64 FMA throughput of this GPU: independent FMA chains in every
    thread of a full grid (libqpb_peak.so, the benchmark's own helper library;
    the driver measures no FP64 figure)."""
    import torch

    path = os.path.join(ROOT, "qpax_b200", "libqpb_peak.so")
    if not os.path.exists(path):
        return {"fp32_tflops": 75.0, "fp64_tflops": 37.0, "how": "nominal (libqpb_peak.so not built)"}
    lib = ctypes.CDLL(path)
    fn = lib.qpb_bench_fma_peak
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_double
    out = {}
    buf = torch.zeros(1 << 20, dtype=torch.float64, device="cuda")
    for prec, key in ((0, "fp32_tflops"), (1, "fp64_tflops")):
        best = 0.0
        for _ in range(3):
            best = max(best, fn(prec, buf.data_ptr(), torch.cuda.current_stream().cuda_stream))
        out[key] = best
    out["how"] = "FMA-chain microbenchmark (libqpb_peak.so, not part of libqpb.so), best of 3, this run"
    if not (out["fp32_tflops"] > 0 and out["fp64_tflops"] > 0):
        return {"fp32_tflops": 75.0, "fp64_tflops": 37.0, "how": "nominal (microbenchmark failed)"}
    return out


# slices of the host-buffer pipelines: copies of the large workloads overlap
# best in 4-8 slices; small ones want few (each slice's launch must still fill
# the GPU)
E2E_CHUNKS = {"dense": 4, "nnls": 4, "small": 2, "uneven": 8, "elastic": 1}


def run_e2e(args, spec: Spec, data, dev, arm, world=1):
    """Same metric through the public API from pinned host buffers: H2D of the
    inputs and the incoming gradient, forward + backward, D2H of x and the
    gradients, all inside the timed region."""
    import torch

    import qpax_b200 as qb

    B = spec.batch
    if spec.kind == "uniform":
        N, M, P = spec.n, spec.m, spec.p
        host = [torch.tensor(a).pin_memory() for a in data]
        g_host = torch.full((B, N), 0.1, dtype=torch.float64).pin_memory()
        outs_host = [torch.empty((B,) + s, dtype=torch.float64).pin_memory()
                     for s in [(N,), (N, N), (N,), (M, N), (M,), (P, N), (P,)]]
        h2d = sum(t.numel() * 8 for t in host) + g_host.numel() * 8
        d2h = sum(t.numel() * 8 for t in outs_host)

        def step():
            qb.solve_qp_primal_vjp_host(*host, g_host, spec.tol, KAPPA, out=outs_host, chunks=args.e2e_chunks)

        path = (f"qpax_b200.solve_qp_primal_vjp_host -> qpb_solve_qp_primal_vjp_host (C ABI, host buffers): "
                f"pinned host tensors, {args.e2e_chunks} chunks: one copy-in stream, two compute streams taken in "
                "turn, one copy-out stream (copies overlap the solves)")
    elif spec.kind == "elastic":
        host = [torch.tensor(a).pin_memory() for a in data] + [torch.full((B,), 1e3, dtype=torch.float64).pin_memory()]
        g_host = torch.full((B, spec.n), 0.1, dtype=torch.float64).pin_memory()
        shp = [(spec.n,), (spec.n, spec.n), (spec.n,), (spec.p, spec.n), (spec.p,)]
        outs_host = [torch.empty((B,) + s, dtype=torch.float64).pin_memory() for s in shp]
        h2d = sum(t.numel() * 8 for t in host) + g_host.numel() * 8
        d2h = sum(t.numel() * 8 for t in outs_host)

        def step():
            d = [t.to(dev, non_blocking=True) for t in host + [g_host]]
            x, grads = qb.solve_qp_elastic_primal_vjp(*d[:5], d[5], spec.tol, KAPPA)
            for dst, src in zip(outs_host, (x,) + tuple(grads)):
                dst.copy_(src, non_blocking=True)

        path = "qpax_b200.solve_qp_elastic_primal_vjp (C ABI): pinned host tensors copied in and out on one stream"
    else:
        from qpax_b200.packed import PackedHostPipeline, pack

        plan = arm.plan
        n_, m_, p_ = shapes_of(spec, data)
        pipe = PackedHostPipeline(list(zip(n_, m_, p_)), chunks=args.e2e_chunks)
        host = [pack(v, torch.device("cpu")).pin_memory() for v in data]
        g_host = torch.full((plan.totals[1],), 0.1, dtype=torch.float64).pin_memory()
        outs_host = [torch.empty(plan.totals[1], dtype=torch.float64).pin_memory()] + \
                    [torch.empty(plan.totals[k], dtype=torch.float64).pin_memory() for k in range(6)]
        h2d = sum(t.numel() * 8 for t in host) + g_host.numel() * 8
        d2h = sum(t.numel() * 8 for t in outs_host)

        def step():
            pipe.run(*host, g_host, spec.tol, KAPPA, out=outs_host)

        path = (f"qpax_b200.packed.PackedHostPipeline (C ABI plans): packed pinned host tensors, {args.e2e_chunks} "
                "instance groups: one copy-in stream, two compute streams taken in turn, one copy-out stream")
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    ms = barrier_max(e0.elapsed_time(e1), world)  # every rank copies and solves its own batch
    return {"value": world * B * args.steps / (ms * 1e-3), "unit": "QPs/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "bytes_counted": "per rank (each rank copies its own batch)",
            "ms_per_step": ms / args.steps, "path": path}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="dense")
    ap.add_argument("--batch", type=int, default=0,
                    help="instances per GPU (default: the workload's own); smaller batches are for profiling")
    ap.add_argument("--only-default", action="store_true", help="time only the default (auto) path")
    ap.add_argument("--e2e-chunks", type=int, default=0,
                    help="slices of the host-buffer pipeline (0: the workload's setting, measured best)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle parity figures")
    ap.add_argument("--no-tune", action="store_true", help="heuristic launch shapes (no autotuning at setup)")
    ap.add_argument("--no-configs", action="store_true",
                    help="dense workload: skip the other four configurations' block")
    ap.add_argument("--config-steps", type=int, default=5, help="timed steps of each configuration in the block")
    args = ap.parse_args()
    spec = WORKLOADS[args.workload]
    if args.e2e_chunks <= 0:
        args.e2e_chunks = E2E_CHUNKS[spec.key]
    if args.batch > 0 and args.batch != spec.batch:
        spec = Spec(spec.key, spec.kind, args.batch, spec.n, spec.m, spec.p, spec.tol,
                    spec.workload.replace(f"{spec.batch}", f"{args.batch}", 1))
    if args.impl == "reference":
        # host-only: rank 0 times the CPU implementation, other ranks exit
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, spec, world, int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, spec, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
