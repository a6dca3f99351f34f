"""Generate the committed golden fixtures of tests/golden/.

    python tests/golden/gen_golden.py

instances.npz   the seeded small OT instances (cost, source, target per case)
golden.json     per case: the exact LP optimum from scipy's HiGHS (an
                independent known answer), and the oracle's solve at tolerance
                1e-6: termination, iteration count, final objectives and the
                first evaluation records (a regression pin of the oracle).

The reference ships no tests or fixtures and cannot run here (no Julia), so
these pins are the project's own: HiGHS pins the optimum, the trajectories pin
the oracle against accidental change.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "pdot.jl_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

CASES = [
    ("uniform", 7, 5, 0),
    ("uniform", 20, 30, 1),
    ("uniform", 33, 17, 2),
    ("uniform", 64, 64, 3),
    ("uniform", 1, 9, 4),
    ("uniform", 9, 1, 5),
    ("l1_dirichlet", 16, 24, 6),
    ("gauss_mixture", 40, 30, 7),
]
TOL = 1e-6
EARLY = 16


def make_instance(kind, m, n, seed):
    from pdot import instances

    if kind == "uniform":
        return instances.uniform_sqeuclid(m, n, seed=seed)
    if kind == "l1_dirichlet":
        return instances.l1_dirichlet(m, n, seed=seed)
    if kind == "gauss_mixture":
        return instances.gauss_mixture(m, n, seed=seed)
    raise ValueError(kind)


def highs_objective(C, a, b) -> float:
    import scipy.optimize as so
    import scipy.sparse as sp

    m, n = C.shape
    rows = sp.kron(sp.eye(1, format="csr"), sp.kron(sp.csr_matrix(np.ones((1, n))), sp.eye(m)))
    cols = sp.kron(sp.eye(n), sp.csr_matrix(np.ones((1, m))))
    A = sp.vstack([rows, cols]).tocsr()
    res = so.linprog(C.ravel(order="F"), A_eq=A, b_eq=np.concatenate([a, b]), bounds=(0, None),
                     method="highs")
    assert res.status == 0, res.message
    return float(res.fun)


def record(s):
    c = s.convergence_information[0]
    return {
        "iteration_number": s.iteration_number,
        "restart_used": int(s.restart_used),
        "step_size": s.step_size,
        "primal_weight": s.primal_weight,
        "cumulative_kkt_matrix_passes": s.cumulative_kkt_matrix_passes,
        "primal_objective": c.primal_objective,
        "dual_objective": c.dual_objective,
        "l2_primal_residual": c.l2_primal_residual,
        "l2_dual_residual": c.l2_dual_residual,
    }


def main():
    import oracle
    from pdot import solve

    arrays = {}
    meta = []
    for kind, m, n, seed in CASES:
        key = f"{kind}_{m}x{n}_s{seed}"
        prob = make_instance(kind, m, n, seed)
        arrays[key + "_C"] = np.asarray(prob.cost_matrix)
        arrays[key + "_a"] = prob.source_distribution
        arrays[key + "_b"] = prob.target_distribution
        out = oracle.optimize(solve.default_parameters(TOL), prob, num_threads=1)
        fin = out.iteration_stats[-1].convergence_information[0]
        meta.append({
            "key": key, "kind": kind, "m": m, "n": n, "seed": seed, "tolerance": TOL,
            "highs_objective": highs_objective(np.asarray(prob.cost_matrix), prob.source_distribution,
                                               prob.target_distribution),
            "termination_reason": int(out.termination_reason),
            "iteration_count": out.iteration_count,
            "primal_objective": fin.primal_objective,
            "dual_objective": fin.dual_objective,
            "early": [record(s) for s in out.iteration_stats[:EARLY]],
        })
    np.savez_compressed(os.path.join(HERE, "instances.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"cases": meta}, f, indent=1)


if __name__ == "__main__":
    main()
