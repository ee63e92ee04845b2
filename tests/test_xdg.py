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
