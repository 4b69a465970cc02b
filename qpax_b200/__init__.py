"""qpax_b200 -- qpax's batched interior-point QP solver, on B200 CUDA kernels.

Drop-in entry points with qpax's names, argument order, defaults and return
tuples (kevin-tracy/qpax, qpax/__init__.py):

    solve_qp(Q, q, A, b, G, h, solver_tol=1e-3) -> (x, s, z, y, converged, iters)
    solve_qp_primal(Q, q, A, b, G, h, solver_tol=1e-5, target_kappa=1e-3) -> x (differentiable)
    solve_qp_elastic(Q, q, G, h, penalty, solver_tol=1e-3) -> (x, t, s1, s2, z1, z2, converged, iters)
    solve_qp_elastic_primal(Q, q, G, h, penalty, solver_tol=1e-5, target_kappa=1e-3) -> x (differentiable)

Arrays take a leading batch axis where qpax users would jax.vmap.  Compute
runs in libqpb.so (include/qpb.h); there is no CPU path.
"""

from .diff_qp import diff_qp, solve_qp_primal, solve_qp_primal_vjp, solve_qp_primal_vjp_host
from .elastic_qp import (diff_qp_elastic, initialize_elastic, relax_qp_elastic, solve_qp_elastic,
                         solve_qp_elastic_primal, solve_qp_elastic_primal_vjp, tune_solve_qp_elastic)
from .pdip import initialize, relax_qp, set_defaults, solve_qp, tune_solve_qp

__all__ = [
    "solve_qp", "solve_qp_primal", "solve_qp_elastic", "solve_qp_elastic_primal", "initialize", "relax_qp",
    "diff_qp", "solve_qp_primal_vjp", "initialize_elastic", "relax_qp_elastic", "diff_qp_elastic",
    "solve_qp_elastic_primal_vjp", "set_defaults", "tune_solve_qp", "tune_solve_qp_elastic",
]
