"""Shared helpers of the test-suite (inputs, error norms, block transforms)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from bosss_b200 import assembly as A


@dataclass
class VarBsr:
    """Block-sparse test matrix with 1 or more species per block (XDG-style uneven blocks)."""
    Np: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray
    nspc: np.ndarray
    rhs: np.ndarray

    @property
    def nb(self):
        return len(self.row_ptr) - 1

    @property
    def block_len(self):
        return self.nspc.astype(np.int64) * self.Np

    @property
    def N(self):
        return int(self.block_len.sum())

    def to_scipy(self):
        import scipy.sparse as sp
        L = self.block_len
        i0 = np.concatenate([[0], np.cumsum(L)])
        rows, cols, vals = [], [], []
        off = 0
        for i in range(self.nb):
            for k in range(self.row_ptr[i], self.row_ptr[i + 1]):
                j = self.col_idx[k]
                I, J = L[i], L[j]
                blk = self.values[off:off + I * J].reshape(I, J)
                off += I * J
                r, c = np.meshgrid(np.arange(I) + i0[i], np.arange(J) + i0[j], indexing="ij")
                rows.append(r.ravel()); cols.append(c.ravel()); vals.append(blk.ravel())
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(self.N, self.N))


def random_var_bsr(nb: int, Np: int, seed: int = 0, max_spc: int = 2, nnz_per_row: int = 5,
                   spd: bool = False, empty_rows: bool = False) -> VarBsr:
    rng = np.random.default_rng(seed)
    nspc = rng.integers(1, max_spc + 1, size=nb).astype(np.int32)
    rows = []
    for i in range(nb):
        k = min(nb, nnz_per_row)
        cols = set(rng.choice(nb, size=k - 1, replace=False).tolist()) if k > 1 else set()
        cols.add(i)
        if empty_rows and i % 7 == 3:
            cols = {i}
        rows.append(sorted(cols))
    if spd:  # symmetric pattern
        pat = [set(r) for r in rows]
        for i, r in enumerate(rows):
            for j in r:
                pat[j].add(i)
        rows = [sorted(p) for p in pat]
    row_ptr = np.zeros(nb + 1, np.int64)
    row_ptr[1:] = np.cumsum([len(r) for r in rows])
    col_idx = np.concatenate([np.asarray(r, np.int32) for r in rows])
    L = nspc.astype(np.int64) * Np
    blocks = {}
    for i, r in enumerate(rows):
        for j in r:
            blocks[(i, j)] = rng.standard_normal((L[i], L[j]))
    if spd:
        for (i, j) in list(blocks):
            if i < j:
                blocks[(j, i)] = blocks[(i, j)].T.copy()
        for i in range(nb):
            d = blocks[(i, i)]
            blocks[(i, i)] = d @ d.T + (2 * sum(np.abs(blocks[(i, j)]).sum() for j in rows[i]) + 1) * np.eye(L[i])
    values = np.concatenate([blocks[(i, j)].ravel() for i, r in enumerate(rows) for j in r])
    return VarBsr(Np=Np, row_ptr=row_ptr, col_idx=col_idx, values=values, nspc=nspc,
                  rhs=rng.standard_normal(int(L.sum())))


def l2_error(grid, p, u, exact, q=6):
    """|u_h - exact|_L2 by tensor Gauss quadrature."""
    modes = A.dg_modes(grid.D, p)
    tg, wg = A.gauss(q)
    hs = grid.cell_sizes()
    xc = grid.cell_centres()
    mesh = np.meshgrid(*([tg] * grid.D), indexing="ij")
    pts = [m.reshape(-1) for m in mesh]
    wts = np.ones(1)
    for _ in range(grid.D):
        wts = np.multiply.outer(wts, wg).reshape(-1)
    X = [xc[d][:, None] + 0.5 * hs[d][:, None] * pts[d][None, :] for d in range(grid.D)]
    basis = np.ones((grid.ncells, len(wts), len(modes)))
    jac = np.ones(grid.ncells)
    for d in range(grid.D):
        vals = np.stack([A.psi(n, pts[d]) for n in range(p + 1)], -1)
        basis = basis * (np.sqrt(2 / hs[d])[:, None, None] * vals[None, :, modes[:, d]])
        jac = jac * 0.5 * hs[d]
    uh = np.einsum("cqa,ca->cq", basis, u.reshape(grid.ncells, -1))
    return float(np.sqrt(np.sum((uh - exact(X)) ** 2 * wts[None, :] * jac[:, None])))


def apply_blocks(Lcat: np.ndarray, block_len: np.ndarray, x: np.ndarray, transpose: bool = False) -> np.ndarray:
    """y_i = L_i x_i (or L_i^T x_i) for row-major blocks concatenated in block order."""
    out = np.empty_like(x)
    lo = 0
    xo = 0
    if np.all(block_len == block_len[0]):
        n = int(block_len[0])
        Lb = Lcat.reshape(-1, n, n)
        xb = x.reshape(-1, n)
        return np.einsum("cji,cj->ci" if transpose else "cij,cj->ci", Lb, xb).reshape(-1)
    for n in block_len:
        n = int(n)
        Li = Lcat[lo:lo + n * n].reshape(n, n)
        out[xo:xo + n] = (Li.T if transpose else Li) @ x[xo:xo + n]
        lo += n * n
        xo += n
    return out


def sip_cartesian1():
    """The reference's TestCartesian1 setup (SipHardcodedControl.cs:206-245): [0,10]x[-1,1], 32x16 cells with
    y-stretch 1.01, p = 2, RHS 1, exact solution 0.5x^2 - 10x, Dirichlet at x = 0, Neumann elsewhere,
    penalty_poisson = 1.3 (SipControl.cs:76)."""
    g = A.RectilinearGrid([np.linspace(0, 10, 33), A.exponential_nodes(-1, 1, 17, 1.01)])
    s = A.assemble_sip(g, 2, penalty_base=1.3,
                       boundary=lambda d, side, x: (d == 0) & (side < 0) & np.ones_like(x[0], bool),
                       rhs_f=lambda X: -np.ones_like(X[0]))
    return g, s, (lambda X: 0.5 * X[0] ** 2 - 10 * X[0])


def greedy_colour_order(row_ptr, col_idx) -> np.ndarray:
    """Block rows ordered by the greedy colouring of the block graph in natural order (colour 0 first), the
    order the GPU block ILU(0) factors in."""
    nb = len(row_ptr) - 1
    col = np.full(nb, -1)
    for i in range(nb):
        used = {col[j] for j in col_idx[row_ptr[i]:row_ptr[i + 1]] if j != i and col[j] >= 0}
        c = 0
        while c in used:
            c += 1
        col[i] = c
    return np.concatenate([np.nonzero(col == c)[0] for c in range(col.max() + 1)]).astype(np.int32)


def dense_block_system(nb: int, Np: int, seed: int = 0) -> VarBsr:
    """Symmetric positive definite system whose block graph is complete (every block row couples to every cell)."""
    rng = np.random.default_rng(seed)
    N = nb * Np
    G = rng.standard_normal((N, N))
    M = G @ G.T + N * np.eye(N)
    row_ptr = np.arange(nb + 1, dtype=np.int64) * nb
    col_idx = np.tile(np.arange(nb, dtype=np.int32), nb)
    values = np.concatenate([M[i * Np:(i + 1) * Np, j * Np:(j + 1) * Np].ravel() for i in range(nb) for j in range(nb)])
    return VarBsr(Np=Np, row_ptr=row_ptr, col_idx=col_idx, values=values, nspc=np.ones(nb, np.int32),
                  rhs=rng.standard_normal(N))
