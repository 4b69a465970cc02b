"""bench.py on the CPU: the reference arm's JSON line and the clock summary.

`bench.py --impl reference` times the FP64 CPU implementation of the path
(the oracle, all host threads) on the same workload, metric and config as
the GPU arm; it needs no device, so its contract is checked here: one JSON
line with the keys the benchmark contract names, printed by rank 0 alone
when launched with several ranks.
"""

import json
import os
import socket
import subprocess
import sys

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def _json_lines(out):
    return [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]


def _check_reference_line(line, workload, world):
    spec = bench.WORKLOADS[workload]
    assert KEYS <= set(line), KEYS - set(line)
    assert line["impl"] == "reference" and line["unit"] == "QPs/s" and line["higher_is_better"] is True
    assert line["metric"] == bench.metric_for(spec)
    assert line["config"] == bench.config_for(spec, world)  # the GPU arm prints the same config
    assert line["n_gpus"] == world and line["steps"] == 1 and line["warmup"] == 3
    assert line["value"] > 0 and line["ms_per_step"] > 0 and line["vs_baseline"] is None
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "QPs/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "nnls", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_reference_line(lines[0], "nnls", 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_under_two_ranks_prints_once():
    """Launched like the multi-GPU bench (one process per rank), rank 0 alone
    runs and prints; the other rank exits 0 without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--workload", "nnls", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_reference_line(lines[0], "nnls", 2)
    assert lines[0]["config"]["global_batch"] == 2 * bench.WORKLOADS["nnls"].batch


def test_clock_summary_reads_nvidia_smi_rows():
    """Median SM clock under load, the maximum clock and the active throttle
    reasons, from `nvidia-smi --format=csv,noheader,nounits` rows."""
    cs = bench.ClockSampler(0)
    cs.lines = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.3, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1320, 1965, 1001.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "garbage line",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    s = cs.summary()
    assert s == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    cs.lines = ["0, 1200, 1965, 500, 0x8, Active, Not Active, Active, Not Active"]
    assert cs.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    cs.lines = []
    assert cs.summary()["samples"] == 0


@pytest.mark.parametrize("n,m,p", [(5, 0, 5), (32, 8, 64), (64, 0, 128)])
def test_algorithmic_flops_follow_the_factor_and_solve_counts(n, m, p):
    """One forward + backward = initialize + iters PC steps, iters_relax relax
    steps and the adjoint, each built from the factor and solve counts
    (FMA = 2, symmetric-aware)."""
    f_fac = p * n * (n + 1) + n ** 3 / 3 + 2 * m * n * n + m * (m + 1) * n + m ** 3 / 3
    f_sol = 4 * n * n + 2 * m * m + 4 * m * n + 4 * p * n + 6 * p
    fwd0, bwd0 = bench.algorithmic_flops(n, m, p, 0, 0)
    fwd1, bwd1 = bench.algorithmic_flops(n, m, p, 1, 1)
    fwd10, bwd4 = bench.algorithmic_flops(n, m, p, 10, 4)
    assert fwd0 == pytest.approx(f_fac + f_sol)
    assert bwd0 == pytest.approx(f_fac + f_sol + 2 * n * n + 2 * m * n + 2 * p * n)
    pc, rlx = fwd1 - fwd0, bwd1 - bwd0
    assert pc == pytest.approx(2 * n * n + 4 * m * n + 4 * p * n + f_fac + 2 * f_sol + 30 * (n + m + p))
    assert rlx == pytest.approx(pc - f_sol - 10 * (n + m + p))
    assert fwd10 == pytest.approx(fwd0 + 10 * pc) and bwd4 == pytest.approx(bwd0 + 4 * rlx)
