"""Sparse text export/import in BoSSS's SaveToTextFileSparse format (IMutuableMatrixEx_Extensions.cs:517-598)."""
import numpy as np

from bosss_b200 import matrixio
from helpers import random_var_bsr


def test_e16_matches_dotnet_notation():
    assert matrixio._e16(1234.5) == "1.2345000000000000E+003"
    assert matrixio._e16(-0.0009765625) == "-9.7656250000000000E-004"
    assert matrixio._e16(0.0) == "0.0000000000000000E+000"


def test_round_trip_is_exact(tmp_path):
    v = random_var_bsr(25, 4, seed=9, max_spc=2)
    path = tmp_path / "M.txt"
    nnz = matrixio.save_text_sparse(str(path), v.Np, v.row_ptr, v.col_idx, v.values, v.nspc)
    M = matrixio.load_text_sparse(str(path))
    ref = v.to_scipy()
    assert M.nnz == nnz == ref.nnz
    assert abs(M - ref).max() == 0.0                       # 17 significant digits: bit-exact
    lines = path.read_text().splitlines()
    assert lines[0] == lines[1] == str(v.N) and lines[2] == str(nnz)
    rp, ci, vals = matrixio.to_block_csr(M, v.Np, v.nspc)
    assert np.array_equal(rp, v.row_ptr) and np.array_equal(ci, v.col_idx) and np.array_equal(vals, v.values)
