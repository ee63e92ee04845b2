"""Runs the oracle (CPU restatement) to convergence on the 3-D 64^3 p = 3 benchmark system and records its outer
iteration count and timing in c2_oracle_solve.json.  bench.py's CPU arm uses the count to turn its per-iteration
sample into a time to 1e-10.  Takes ~10-20 minutes on 8 cores.

    python tests/golden/make_c2_oracle_solve.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from bosss_b200 import assembly as A  # noqa: E402
from bench import SOLVER_PARAMS, TOL  # noqa: E402


def main():
    threads = O.set_threads(os.cpu_count() or 1)
    s = A.poisson_3d(64, 3, seed=0)
    vals, L = O.change_of_basis(O.Bsr.of(s))

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    bt = np.einsum("cij,cj->ci", L.reshape(-1, s.Np, s.Np), s.rhs.reshape(-1, s.Np)).reshape(-1)
    cfg = O.SolverConfig(solver=O.FGMRES_PMG, tol=TOL, top_mode=O.TERM_RELATIVE, level_keep=(20, 10, 4),
                         coarse_kind=O.COARSE_PCG, coarse_tol=SOLVER_PARAMS["CoarseTolerance"],
                         coarse_max_iter=SOLVER_PARAMS["CoarseMaxIterations"],
                         sub_reduction=SOLVER_PARAMS["SubLevelReduction"],
                         sub_max_iter=SOLVER_PARAMS["SubLevelMaxIterations"])
    ps = O.PersistentSolver(O.Bsr.of(T), cfg)
    t0 = time.perf_counter()
    r = ps.solve(bt)
    dt = time.perf_counter() - t0
    out = {"iterations": r.iterations, "converged": r.converged, "seconds": dt, "threads": threads,
           "relres_transformed": r.res / r.res0, "workload": "3-D SIP Poisson 64^3 p=3, seed 0"}
    with open(os.path.join(HERE, "c2_oracle_solve.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    main()
