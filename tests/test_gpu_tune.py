"""The size-bin autotuner (qpb_plan_tune, qpb_tune_solve_qp_elastic).

For an uneven batch (the configuration-4 generator, n up to 128) and for the
elastic configuration's shape (n = 64, p = 128): the tuned launch shapes are
no slower than the heuristic's (device time of the forward solve, median of
five, within a 10 % allowance for run-to-run noise -- the tuner itself picks
on a two-wave sample), the tuned call's outputs still match the oracle
(the bars of tests/test_gpu_configs.py: every reproducible reference
solution is found, x within 1e-6, instances only the GPU solves have a KKT
residual below 100 x tol), and a plan created afterwards for the same shapes
starts from the recorded choice.
"""

import numpy as np
import pytest
import torch

from oracle import parity
from qpax_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _median_ms(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return float(np.median(out))


def test_packed_plan_tuning():
    from qpax_b200.packed import PackedPlan, pack, unpack

    data = wl.uneven(768, seed=44, n_max=128)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    ins = [pack(v) for v in data]
    heur = PackedPlan(shapes)
    t_heur = _median_ms(lambda: heur.solve(*ins, 1e-6))
    plan = PackedPlan(shapes)
    x, s, z, y, conv, iters = plan.tune(*ins, 1e-6)
    torch.cuda.synchronize()
    t_tuned = _median_ms(lambda: plan.solve(*ins, 1e-6))
    print("heuristic", heur.bin_info(), f"{t_heur:.3f} ms")
    print("tuned", plan.bin_info(), f"{t_tuned:.3f} ms")
    assert t_tuned <= 1.10 * t_heur, (t_tuned, t_heur)
    L = plan.lengths
    cut = lambda t, f: [v.cpu().numpy() for v in unpack(t, L[f])]
    fig = parity.forward(data, 1e-6, dict(x=cut(x, 1), s=cut(s, 5), z=cut(z, 5), y=cut(y, 3),
                                          conv=conv.cpu().numpy(), iters=iters.cpu().numpy()))
    print(fig)
    assert fig["reference_only_converged_reproducible"] == 0, fig
    assert fig["iters_mismatch_both_converged_reproducible"] == 0, fig
    assert fig["gpu_only_max_kkt"] <= 1e-4 and fig["max_err_x"] <= 1e-6, fig
    assert fig["reference_outcome_not_reproducible"] <= 0.1 * fig["instances"], fig
    res2 = plan.solve(*ins, 1e-6)
    for a, b_ in zip(res2, (x, s, z, y, conv, iters)):
        assert torch.equal(a, b_)  # the tuning call's outputs are the tuned plan's
    # a new plan for the same shapes starts from the recorded launch shapes
    again = PackedPlan(shapes)
    assert again.bin_info() == plan.bin_info()


def test_elastic_tuning():
    import qpax_b200 as qb

    Q, q, G, h, _ = wl.elastic(1024)
    dev = [torch.tensor(a, device="cuda") for a in (Q, q, G, h)]
    t_heur = _median_ms(lambda: qb.solve_qp_elastic(*dev, 1e3, 1e-6))
    out = qb.tune_solve_qp_elastic(*dev, 1e3, 1e-6)
    torch.cuda.synchronize()
    t_tuned = _median_ms(lambda: qb.solve_qp_elastic(*dev, 1e3, 1e-6))
    print(f"elastic: heuristic {t_heur:.3f} ms, tuned {t_tuned:.3f} ms")
    assert t_tuned <= 1.10 * t_heur, (t_tuned, t_heur)
    fig = parity.elastic_forward((Q, q, G, h), 1e3, 1e-6, [t.cpu().numpy() for t in out])
    print(fig)
    assert fig["reference_only_converged_reproducible"] == 0, fig
    assert fig["iters_mismatch_both_converged_reproducible"] == 0, fig
    assert fig["gpu_only_max_kkt"] <= 1e-4 and fig["max_err_x"] <= 1e-6, fig


def test_packed_plan_tuning_mixed():
    """Mixed precision: tuning a plan whose bins run the mixed one-warp
    kernel (n <= 32, two launches with hand-over records) and the mixed CTA
    kernel (n > 32).  A tuned bin may need more workspace than its heuristic
    shape; qpb_plan_tune_workspace_size covers every bin's largest
    candidate.  The outputs meet the same bars as the FP64 plan's."""
    from qpax_b200.packed import PackedPlan, pack, unpack

    data = wl.uneven(256, seed=45, n_max=96)
    shapes = [(len(q), len(b), len(h)) for q, b, h in zip(data[1], data[3], data[5])]
    ins = [pack(v) for v in data]
    plan = PackedPlan(shapes, precision="mixed")
    x, s, z, y, conv, iters = plan.tune(*ins, 1e-6)
    torch.cuda.synchronize()
    L = plan.lengths
    cut = lambda t, f: [v.cpu().numpy() for v in unpack(t, L[f])]
    fig = parity.forward(data, 1e-6, dict(x=cut(x, 1), s=cut(s, 5), z=cut(z, 5), y=cut(y, 3),
                                          conv=conv.cpu().numpy(), iters=iters.cpu().numpy()), eps=1e-12)
    print(plan.bin_info(), fig)
    assert fig["reference_only_converged_reproducible"] == 0, fig
    assert fig["iters_mismatch_both_converged_reproducible"] == 0, fig
    assert fig["gpu_only_max_kkt"] <= 1e-4 and fig["max_err_x"] <= 1e-6, fig
    res2 = plan.solve(*ins, 1e-6)
    for a, b_ in zip(res2, (x, s, z, y, conv, iters)):
        assert torch.equal(a, b_)
