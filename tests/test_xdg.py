"""CPU checks of the XDG (two-species cut-cell) workload generator used by the XDG parity tests and benches."""
import numpy as np
import scipy.sparse.linalg as spla

from bosss_b200 import assembly as A
from bosss_b200 import xdg


def test_uncut_domain_equals_plain_dg():
    s = xdg.xdg_sphere(n=4, p=2, centre=(5.0, 5.0, 5.0), radius=0.1, mu=(1.0, 1.0))
    assert np.all(s.nspc == 1)
    d = A.poisson_3d(4, 2)
    M1, M2 = s.to_scipy(), d.to_scipy()
    assert abs(M1 - M2).max() <= 1e-13 * abs(M2).max()


def test_cut_system_is_symmetric_positive_definite():
    s = xdg.xdg_sphere(n=6, p=1, seed=3)
    assert set(np.unique(s.nspc)) == {1, 2}
    lens = s.nspc.astype(np.int64) * s.Np
    assert s.N == lens.sum()
    M = s.to_scipy()
    assert abs(M - M.T).max() <= 1e-12 * abs(M).max()
    lo = spla.eigsh(M, k=1, which="SA", return_eigenvectors=False, tol=1e-8)[0]
    assert lo > 0.0


def test_block_layout_is_consistent():
    s = xdg.xdg_sphere(n=5, p=2, seed=4)
    lens = s.nspc.astype(np.int64) * s.Np
    rows = np.repeat(np.arange(s.nb), np.diff(s.row_ptr))
    assert len(s.values) == int((lens[rows] * lens[s.col_idx]).sum())
    for i in range(s.nb):  # sorted, unique block columns with the diagonal present
        c = s.col_idx[s.row_ptr[i]:s.row_ptr[i + 1]]
        assert np.all(np.diff(c) > 0) and i in c


def test_batch_specs_are_seeded_and_in_range():
    a, b = xdg.batch_specs(64, seed=3), xdg.batch_specs(64, seed=3)
    assert a == b and len(a) == 64
    for sp in a:
        assert sp["n"] in xdg.BATCH_EDGES and 0.15 <= sp["radius"] <= 0.35
        assert sp["mu"][0] == 1.0 and sp["mu"][1] in xdg.BATCH_JUMPS
        assert all(0.4 <= c <= 0.6 for c in sp["centre"])
    assert len({sp["n"] for sp in a}) > 1 and len({sp["mu"][1] for sp in a}) > 1


def test_xdg_matrix_text_exchange(tmp_path):
    """An XDG system (blocks of 10 and 20 rows) survives the SaveToTextFileSparse round trip bit for bit."""
    from bosss_b200 import matrixio
    s = xdg.xdg_sphere(n=4, p=2, seed=1)
    path = str(tmp_path / "xdg.txt")
    matrixio.save_text_sparse(path, s.Np, s.row_ptr, s.col_idx, s.values, s.nspc)
    M = matrixio.load_text_sparse(path)
    assert abs(M - s.to_scipy()).max() == 0.0


def test_workload_fingerprints():
    """The seeded workload generators reproduce the committed fingerprints (tests/golden/make_workload_fingerprints.py)."""
    import json
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    from make_workload_fingerprints import fingerprints
    ref = json.load(open(os.path.join(here, "workload_fingerprints.json")))
    got = fingerprints()
    assert set(got) == set(ref)
    for name, r in ref.items():
        g = got[name]
        assert g["N"] == r["N"] and g["nnzb"] == r["nnzb"], name
        for k in ("values_l2", "values_sum", "rhs_l2", "rhs_sum"):
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (name, k)
