"""Writes workload_fingerprints.json: sizes and norms of small seeded instances of every synthetic workload the
tests and the benchmark use (3-D SIP Poisson, 2-D Poisson, variable coefficient, XDG sphere).  The CPU test
test_workload_fingerprints recomputes them, so an accidental change of a generator shows up as a failing test.

    python tests/golden/make_workload_fingerprints.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def fingerprints():
    from bosss_b200 import assembly as A
    from bosss_b200 import xdg
    cases = {
        "poisson_3d(4,3)": A.poisson_3d(4, 3, seed=0),
        "poisson_2d_c1(n=8)": A.poisson_2d_c1(seed=0, n=8),
        "variable_coeff_3d(4,2)": A.variable_coeff_3d(4, 2, seed=0),
        "xdg_sphere(n=6,p=2)": xdg.xdg_sphere(n=6, p=2, seed=0),
    }
    out = {}
    for name, s in cases.items():
        v = np.asarray(s.values, np.float64).reshape(-1)
        out[name] = {"N": int(s.N), "nnzb": int(len(s.col_idx)), "values_l2": float(np.linalg.norm(v)),
                     "values_sum": float(v.sum()), "rhs_l2": float(np.linalg.norm(s.rhs)),
                     "rhs_sum": float(np.asarray(s.rhs).sum())}
    return out


if __name__ == "__main__":
    with open(os.path.join(HERE, "workload_fingerprints.json"), "w") as f:
        json.dump(fingerprints(), f, indent=1)
