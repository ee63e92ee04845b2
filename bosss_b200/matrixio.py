"""Sparse text export and import in the format of BoSSS's ``SaveToTextFileSparse``
(``src/ilPSP/layer_1.2-ilPSP/ilPSP/IMutuableMatrixEx_Extensions.cs:517-598``), so that matrices can be exchanged
with a BoSSS installation (and with the MATLAB reader documented there).

Layout: number of rows, number of columns and number of non-zero entries on the first three lines; then one
line per row: the row's non-zero count followed by ``column value`` pairs (0-based columns, values in .NET's
"E16" notation, 17 significant digits and an exponent of at least three digits), every item followed by a space.
Entries that are exactly zero are not written, as in the reference.
"""
from __future__ import annotations

import numpy as np


def _e16(v: float) -> str:
    """.NET ``ToString("E16", InvariantCulture)``: d.dddddddddddddddd E+ddd."""
    if v == 0.0:
        return "0.0000000000000000E+000"
    m, e = f"{v:.16E}".split("E")
    ei = int(e)
    return f"{m}E{'+' if ei >= 0 else '-'}{abs(ei):03d}"


def _block_lengths(Np: int, nb: int, nspc) -> np.ndarray:
    return (np.ones(nb, np.int64) if nspc is None else np.asarray(nspc, np.int64)) * int(Np)


def save_text_sparse(path: str, Np: int, row_ptr, col_idx, values, nspc=None) -> int:
    """Writes a block-CSR matrix (row-major blocks of nspc[i]*Np rows) in SaveToTextFileSparse format; returns the
    number of non-zero entries written."""
    row_ptr = np.asarray(row_ptr, np.int64)
    col_idx = np.asarray(col_idx, np.int64)
    values = np.asarray(values, np.float64).reshape(-1)
    nb = len(row_ptr) - 1
    L = _block_lengths(Np, nb, nspc)
    i0 = np.concatenate([[0], np.cumsum(L)])
    N = int(i0[-1])
    rows = [[] for _ in range(N)]
    off = 0
    for i in range(nb):
        I = int(L[i])
        for k in range(row_ptr[i], row_ptr[i + 1]):
            j = int(col_idx[k])
            J = int(L[j])
            blk = values[off:off + I * J].reshape(I, J)
            off += I * J
            for r in range(I):
                row = rows[i0[i] + r]
                for c in range(J):
                    v = blk[r, c]
                    if v != 0.0:
                        row.append((int(i0[j] + c), float(v)))
    nnz = sum(len(r) for r in rows)
    with open(path, "w", newline="\n") as f:
        f.write(f"{N}\n{N}\n{nnz}\n")
        for row in rows:
            row.sort()
            f.write(f"{len(row)} " + "".join(f"{c} {_e16(v)} " for c, v in row) + "\n")
    return nnz


def load_text_sparse(path: str):
    """Reads a SaveToTextFileSparse file into a scipy CSR matrix."""
    import scipy.sparse as sp
    with open(path) as f:
        nrows = int(f.readline())
        ncols = int(f.readline())
        f.readline()
        ri, ci, vv = [], [], []
        for r in range(nrows):
            t = f.readline().split()
            n = int(t[0])
            for q in range(n):
                ri.append(r)
                ci.append(int(t[1 + 2 * q]))
                vv.append(float(t[2 + 2 * q]))
    return sp.csr_matrix((vv, (ri, ci)), shape=(nrows, ncols))


def to_block_csr(M, Np: int, nspc=None):
    """Block-CSR arrays (row_ptr, col_idx, row-major block values) of a scipy matrix for blocks of nspc[i]*Np rows;
    a block is stored when any of its entries is non-zero, or when it is a diagonal block."""
    import scipy.sparse as sp
    M = sp.csr_matrix(M)
    N = M.shape[0]
    nb = N // int(Np) if nspc is None else len(nspc)
    L = _block_lengths(Np, nb, nspc)
    i0 = np.concatenate([[0], np.cumsum(L)])
    if i0[-1] != N:
        raise ValueError("block lengths do not add up to the matrix size")
    blk_of = np.repeat(np.arange(nb), L)
    C = M.tocoo()
    pairs = set(zip(blk_of[C.row].tolist(), blk_of[C.col].tolist())) | {(i, i) for i in range(nb)}
    pairs = sorted(pairs)
    row_ptr = np.zeros(nb + 1, np.int64)
    for i, _ in pairs:
        row_ptr[i + 1] += 1
    row_ptr = np.cumsum(row_ptr)
    col_idx = np.array([j for _, j in pairs], np.int32)
    D = M.tolil()
    vals = []
    for i, j in pairs:
        vals.append(D[i0[i]:i0[i + 1], i0[j]:i0[j + 1]].toarray().ravel())
    return row_ptr, col_idx, np.concatenate(vals) if vals else np.zeros(0)
