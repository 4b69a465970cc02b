"""Regenerates tests/golden/qpax_pins.npz from the qpax reference checkout.

Run:  python tests/golden/make_golden.py /path/to/qpax   (the reference tree)

Nothing here runs at test time: the tests read only the .npz this script
writes.  What it collects, all from the reference's own test suite:

* the elastic golden vectors `test/problem_data_pos.npz` and
  `test/initial_values_pos.npz` (used by test/test_elastic_qp.py:58-111);
* the known-answer problems of test/test_constraint_sizes.py (problem data,
  solver_tol and the expected x / tolerance of each assert), obtained by
  executing that file with numpy standing in for jax.numpy and a recorder
  standing in for qpax.solve_qp -- jax itself is not installed here;
* the first QPs drawn by test/misc_test_utils.py:generate_random_qp under
  np.random.seed(1) and seed(3), executed the same way, so the tests can pin
  their restatement of that generator.
"""

from __future__ import annotations

import ast
import os
import sys
import types

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qpax_pins.npz")


class _Stop(Exception):
    pass


def _jax_shim():
    jax = types.ModuleType("jax")
    jax.numpy = np
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.jit = lambda f, *a, **k: f
    jax.vmap = None
    jax.grad = None
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = np
    return jax


def _assert_literals(fn_node):
    """(expected array, tolerance) pairs from `assert norm(x - jnp.array([...])) < tol`."""
    out = []
    for node in ast.walk(fn_node):
        if isinstance(node, ast.Assert) and isinstance(node.test, ast.Compare):
            arr = None
            for sub in ast.walk(node.test.left):
                if (isinstance(sub, ast.Call) and isinstance(sub.func, ast.Attribute) and sub.func.attr == "array"
                        and sub.args and isinstance(sub.args[0], ast.List)):
                    arr = np.array(ast.literal_eval(sub.args[0]), dtype=np.float64)
            if arr is not None:
                tol = ast.literal_eval(node.test.comparators[0])
                out.append((arr, float(tol)))
    return out


def collect_constraint_sizes(ref):
    path = os.path.join(ref, "test", "test_constraint_sizes.py")
    src = open(path).read()
    tree = ast.parse(src)
    _jax_shim()
    calls = []

    def recorder(Q, q, A, b, G, h, solver_tol=1e-3):
        calls.append(dict(Q=Q, q=q, A=A, b=b, G=G, h=h, solver_tol=solver_tol))
        raise _Stop()

    qpax = types.ModuleType("qpax")
    qpax.solve_qp = recorder
    sys.modules["qpax"] = qpax
    ns = {"__name__": "ref_constraint_sizes"}
    exec(compile(src, path, "exec"), ns)
    pins = {}
    for fn in [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name.startswith("test_")]:
        calls.clear()
        try:
            ns[fn.name]()
        except _Stop:
            pass
        call = calls[0]
        rec = {k: np.atleast_1d(np.asarray(v, np.float64)) for k, v in call.items() if k != "solver_tol"}
        rec["Q"] = np.atleast_2d(rec["Q"])
        n = rec["Q"].shape[0]
        rec["A"] = np.asarray(call["A"], np.float64).reshape(-1, n) if np.size(call["A"]) else np.zeros((0, n))
        rec["G"] = np.asarray(call["G"], np.float64).reshape(-1, n) if np.size(call["G"]) else np.zeros((0, n))
        rec["b"] = np.asarray(call["b"], np.float64).reshape(-1)
        rec["h"] = np.asarray(call["h"], np.float64).reshape(-1)
        rec["solver_tol"] = np.float64(call["solver_tol"])
        lits = _assert_literals(fn)
        if lits:
            rec["x_expected"], tol = lits[0]
            rec["x_tol"] = np.float64(tol)
        pins[fn.name] = rec
    return pins


def collect_generator(ref, seed, count, dims):
    path = os.path.join(ref, "test", "misc_test_utils.py")
    src = open(path).read()
    _jax_shim()
    ns = {"__name__": "ref_misc_test_utils"}
    exec(compile(src, path, "exec"), ns)
    np.random.seed(seed)
    out = []
    for _ in range(count):
        out.append([np.asarray(a, np.float64) for a in ns["generate_random_qp"](*dims)])
    return out


def main(ref):
    flat = {}
    for name in ("problem_data_pos", "initial_values_pos"):
        d = np.load(os.path.join(ref, "test", name + ".npz"))
        for k in d.files:
            flat[f"elastic/{name}/{k}"] = np.asarray(d[k])
    for test, rec in collect_constraint_sizes(ref).items():
        for k, v in rec.items():
            flat[f"sizes/{test}/{k}"] = np.asarray(v)
    names = ("Q", "q", "A", "b", "G", "h", "x", "s", "z", "y")
    for seed, dims in ((1, (15, 10, 3)), (3, (15, 10, 3))):
        for i, qp in enumerate(collect_generator(ref, seed, 3, dims)):
            for k, v in zip(names, qp):
                flat[f"gen/seed{seed}/{i}/{k}"] = v
    np.savez_compressed(OUT, **flat)
    print("wrote", OUT, len(flat), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
