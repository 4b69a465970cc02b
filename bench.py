"""Benchmark: QPs/sec, forward + backward, at 1e-6 KKT residual, one B200 per rank.

Workload (one step): the differentiable batched solve of qpax
(solve_qp_primal) over 4096 dense QPs with n = 32, m = 8, p = 64 -- the
dense-QP configuration (Q = M'M + 1e-3 I, strictly feasible h = G x0 + s0),
solver_tol 1e-6, target_kappa 1e-3, loss ||x - 1||^2:
  forward  = qpb_solve_qp            (initialize + predictor-corrector loop)
  backward = qpb_solve_qp_primal_bwd (relaxation to kappa + adjoint KKT solve
             + the six gradient outer products)
Inputs are resident in HBM; L2 is flushed (256 MB write) between steps,
outside the per-step CUDA events.  Synthetic seeded data (no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the FP64 CPU restatement of qpax (oracle/) on the
host cores, on the same workload -- qpax itself (JAX) is not installable
here.  Multi-GPU: one process per GPU, each rank solves its own batch (weak
scaling, no collective on the data path); time = max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPs/sec fwd+bwd at 1e-6 KKT residual, mixed vs plain FP64 kernel, 1 B200"
B, N, M, P = 4096, 32, 8, 64
TOL, KAPPA = 1e-6, 1e-3
WORKLOAD = "dense QP n=32 m=8 p=64, batch 4096/GPU, solve_qp_primal forward+backward, tol 1e-6, kappa 1e-3"


def algorithmic_flops(n, m, p, iters_fwd, iters_relax):
    """Algorithmic FLOPs (FMA = 2, symmetric-aware) of one forward + backward:
    initialize + iters_fwd predictor-corrector iterations, iters_relax
    relaxation iterations and the adjoint (one factor + one solve + outer products)."""
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
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier_max(val, world):
    import torch

    if world == 1:
        return val
    import torch.distributed as dist

    t = torch.tensor([val], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_baseline_sample(data, seconds=12.0, max_seconds=30.0, chunk=1024):
    """The oracle (FP64 C restatement of qpax, OpenMP over instances, all host
    threads) on repeated chunks of the same batch until `seconds` elapse."""
    from oracle import oracle

    Q, q, A, b, G, h = data
    dl = np.full((B, N), 0.1)
    done, t0 = 0, time.perf_counter()
    i = 0
    while True:
        s = slice((i * chunk) % B, (i * chunk) % B + chunk)
        oracle.solve_qp_primal_vjp(Q[s], q[s], A[s], b[s], G[s], h[s], dl[s], solver_tol=TOL, target_kappa=KAPPA)
        done += chunk
        i += 1
        el = time.perf_counter() - t0
        if el >= seconds or el >= max_seconds:
            break
    return {"value": done / el, "unit": "QPs/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{done} QPs of the workload (chunks of {chunk}), {el:.1f} s wall, forward+backward"}


def run_reference(args, world, rank):
    from oracle import oracle
    from qpax_b200 import workloads as wl

    if rank != 0:
        return
    data = wl.config2(B)
    Q, q, A, b, G, h = data
    dl = np.full((B, N), 0.1)
    step = lambda: oracle.solve_qp_primal_vjp(Q, q, A, b, G, h, dl, solver_tol=TOL, target_kappa=KAPPA)
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    val = B * args.steps / el
    cores = oracle.num_threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "QPs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD + " (all host threads)", "global_batch": B, "n": N, "m": M, "p": P},
        "cpu_baseline": {"value": val, "unit": "QPs/s", "cores": cores, "kind": "port",
                         "sample": f"the full {B}-QP batch per step, {args.steps} steps"},
        "e2e": {"value": val, "unit": "QPs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "qpax (JAX) is not installable offline; the timed CPU implementation is the FP64 C "
                "restatement of qpax in oracle/ (pinned to qpax's golden vectors and tests)",
    }
    print(json.dumps(line), flush=True)


def load_traffic():
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
    bench workload's forward and backward launches, from the committed ncu
    summary profiles/traffic_dense_qp_n32_b4096.txt ("key value" lines)."""
    path = os.path.join(ROOT, "profiles", "traffic_dense_qp_n32_b4096.txt")
    if not os.path.exists(path):
        return None
    out = {"source": "profiles/traffic_dense_qp_n32_b4096.txt"}
    for ln in open(path):
        parts = ln.split()
        if len(parts) == 2 and parts[0] in ("forward", "backward"):
            try:
                out[parts[0]] = float(parts[1])
            except ValueError:
                pass
    return out


def run_ours(args, world, rank, local):
    import torch

    import qpax_b200 as qb
    from qpax_b200 import _lib
    from qpax_b200 import workloads as wl
    from qpax_b200.diff_qp import diff_qp_from_forward
    from qpax_b200.pdip import StdBatch, _config, _run

    _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    data = wl.config2(B)
    Qd, qd, Ad, bd, Gd, hd = (torch.tensor(a, device=dev) for a in data)
    bt = StdBatch(Qd, qd, Ad, bd, Gd, hd)
    dl_host = np.full((B, N), 0.1)
    stream = torch.cuda.current_stream()

    def make_step(opts):
        cfg = _config(opts)
        x, s, z, y = bt.new(B, N), bt.new(B, P), bt.new(B, P), bt.new(B, M)
        conv, iters = bt.new(B, dtype=torch.int32), bt.new(B, dtype=torch.int32)
        rconv, riters = bt.new(B, dtype=torch.int32), bt.new(B, dtype=torch.int32)
        gx = torch.empty(B, N, dtype=torch.float64, device=dev)
        import ctypes

        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

        def fwd():
            _run("qpb_solve_qp", "solve", bt, cfg, [ctypes.c_double(TOL)],
                 [x.data_ptr(), s.data_ptr(), z.data_ptr(), y.data_ptr(), conv.data_ptr(), iters.data_ptr()])

        def bwd():
            torch.mul(x - 1.0, 2.0, out=gx)
            return diff_qp_from_forward(bt, x, s, z, y, gx, TOL, KAPPA, opts,
                                        relaxed=[None, None, None, None, rconv, riters])

        def step(timed=None):
            if timed is not None:
                timed[0].record(stream)
            fwd()
            if timed is not None:
                timed[1].record(stream)
            g = bwd()
            if timed is not None:
                timed[2].record(stream)
            return g

        return step, (x, conv, iters, rconv, riters)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    results = {}
    variants = {
        "auto": dict(precision="auto"),                       # the default path (warp kernel here)
        "fp64_cta": dict(precision="fp64", team_threads=128),  # plain FP64, one QP per CTA
        "mixed": dict(precision="mixed"),                     # FP32 factor + FP64 refinement
    }
    if args.only_default:
        variants = {"auto": variants["auto"]}
    for prec, opts in variants.items():
        step, outs = make_step(opts)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
        barrier(world)
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if prec == "auto" else None
        if sampler:
            sampler.__enter__()
        wall0 = time.perf_counter()
        for k in range(args.steps):
            flush.fill_(float(k))
            step(evs[k])
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
        if sampler:
            sampler.__exit__(None, None, None)
        barrier(world)
        fwd_ms = [e[0].elapsed_time(e[1]) for e in evs]
        bwd_ms = [e[1].elapsed_time(e[2]) for e in evs]
        tot = sum(f + b for f, b in zip(fwd_ms, bwd_ms))
        tot = barrier_max(tot, world)
        x, conv, iters, rconv, riters = outs
        results[prec] = dict(total_ms=tot, fwd_ms=float(np.mean(fwd_ms)), bwd_ms=float(np.mean(bwd_ms)),
                             wall_s=wall, conv=conv.cpu().numpy(), iters=iters.cpu().numpy(),
                             riters=riters.cpu().numpy(), rconv=rconv.cpu().numpy(),
                             clocks=sampler.summary() if sampler else None)

    main_r = results["auto"]
    value = world * B * args.steps / (main_r["total_ms"] * 1e-3)
    # roofline of the dominant launch (forward or backward kernel of the default path)
    f_fwd, f_bwd = algorithmic_flops(N, M, P, main_r["iters"].astype(np.float64),
                                     main_r["riters"].astype(np.float64))
    fl_fwd, fl_bwd = float(f_fwd.sum()), float(f_bwd.sum())
    traffic = load_traffic()
    if main_r["fwd_ms"] >= main_r["bwd_ms"]:
        dom, dom_ms, dom_fl, dom_key = "qpb_solve_qp: warp_kernel<32,8> (forward)", main_r["fwd_ms"], fl_fwd, "forward"
    else:
        dom, dom_ms, dom_fl, dom_key = "qpb_solve_qp_primal_bwd: warp_kernel<32,8> (backward)", main_r["bwd_ms"], \
            fl_bwd, "backward"
    achieved = dom_fl / (dom_ms * 1e-3) / 1e12
    peaks, peak_src = load_peaks()
    simt = simt_peaks()
    roof = {
        "bound": "tensor", "kernel": dom, "achieved": achieved, "unit": "TFLOP/s",
        "peak": peaks["bf16_tflops"], "frac": achieved / peaks["bf16_tflops"],
        "peak_source": f"bf16 dense tensor peak of MEASURED_PEAKS.json ({peak_src}); the kernel is FP64 "
                       "arithmetic, so its own roof is the FP64 FMA peak below",
        "fp64_fma_peak": simt["fp64_tflops"], "frac_of_fp64_fma_peak": achieved / simt["fp64_tflops"],
        "fp32_fma_peak": simt["fp32_tflops"], "fma_peak_source": simt["how"],
        "algorithmic_flops_per_launch": dom_fl, "avg_launch_ms": dom_ms,
        "traffic": (traffic or {}).get(dom_key),
        "traffic_source": (traffic or {}).get("source"),
    }
    line = {
        "metric": METRIC, "value": value, "unit": "QPs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main_r["total_ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "global_batch": B * world, "n": N, "m": M, "p": P,
                   "precision": "auto (FP64; one warp per QP for n <= 32)", "parallelism": f"batch split x{world}",
                   "l2": "flushed between steps (256 MB write), outside the per-step events"},
        "roofline": roof, "gpu_launches": 2 * args.steps,
        "iterations": {"forward_mean": float(main_r["iters"].mean()), "relax_mean": float(main_r["riters"].mean()),
                       "converged": float(main_r["conv"].mean())},
        "clocks": main_r["clocks"],
        "forward_ms": main_r["fwd_ms"], "backward_ms": main_r["bwd_ms"],
    }
    if "fp64_cta" in results and "mixed" in results:
        v = {k: world * B * args.steps / (r["total_ms"] * 1e-3) for k, r in results.items()}
        line["variants"] = {
            "fp64_one_cta_per_qp": {"value": v["fp64_cta"], "unit": "QPs/s",
                                    "ms_per_step": results["fp64_cta"]["total_ms"] / args.steps},
            "mixed_fp32_factor_fp64_refinement": {"value": v["mixed"], "unit": "QPs/s",
                                                  "ms_per_step": results["mixed"]["total_ms"] / args.steps},
        }
        line["mixed_over_plain_fp64"] = v["mixed"] / v["fp64_cta"]
        line["default_over_plain_fp64"] = v["auto"] / v["fp64_cta"]
        line["converged_flags_identical"] = bool(all((r["conv"] == main_r["conv"]).all() for r in results.values()))
        line["iteration_counts_identical"] = bool(all((r["iters"] == main_r["iters"]).all()
                                                      for r in results.values()))
    if rank == 0 and not args.no_e2e:
        line["e2e"] = run_e2e(args, data, dev)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_sample(data)
    if rank == 0:
        print(json.dumps(line), flush=True)


def simt_peaks():
    """FP32 / FP64 FMA throughput of this GPU, measured with a dependent-chain-free FMA loop."""
    import torch

    from qpax_b200 import _lib

    lib = _lib.load()
    fn = getattr(lib, "qpb_bench_fma_peak", None)
    if fn is None:
        return {"fp32_tflops": 75.0, "fp64_tflops": 37.0, "how": "nominal (no microbenchmark in the library)"}
    import ctypes

    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_double
    out = {}
    buf = torch.zeros(1 << 20, dtype=torch.float64, device="cuda")
    for prec, key in ((0, "fp32_tflops"), (1, "fp64_tflops")):
        best = 0.0
        for _ in range(3):
            best = max(best, fn(prec, buf.data_ptr(), torch.cuda.current_stream().cuda_stream))
        out[key] = best
    out["how"] = "qpb_bench_fma_peak, best of 3"
    if not (out["fp32_tflops"] > 0 and out["fp64_tflops"] > 0):
        return {"fp32_tflops": 75.0, "fp64_tflops": 37.0, "how": "nominal (microbenchmark failed)"}
    return out


def run_e2e(args, data, dev):
    """Same metric through the public API from pinned host buffers: H2D of the
    inputs and the incoming gradient, forward + backward, D2H of x and the six
    gradients, all inside the timed region."""
    import torch

    import qpax_b200 as qb

    host = [torch.tensor(a).pin_memory() for a in data]
    g_host = torch.full((B, N), 0.1, dtype=torch.float64).pin_memory()
    outs_host = [torch.empty((B,) + s, dtype=torch.float64).pin_memory()
                 for s in [(N,), (N, N), (N,), (M, N), (M,), (P, N), (P,)]]
    h2d = sum(t.numel() * 8 for t in host) + g_host.numel() * 8
    d2h = sum(t.numel() * 8 for t in outs_host)

    def step():
        qb.solve_qp_primal_vjp_host(*host, g_host, TOL, KAPPA, out=outs_host, chunks=args.e2e_chunks)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": B * args.steps / (ms * 1e-3), "unit": "QPs/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms / args.steps,
            "path": f"qpax_b200.solve_qp_primal_vjp_host (C ABI): pinned host tensors, {args.e2e_chunks} chunks "
                    "pipelined over 3 streams (copy in / solve + backward / copy out overlap)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--only-default", action="store_true", help="time only the default (auto) path")
    ap.add_argument("--e2e-chunks", type=int, default=4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        # host-only: rank 0 times the CPU implementation, other ranks exit
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, world, int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
