"""Symmetric-interior-penalty (SIP) DG Poisson assembly on rectilinear grids (workload generator).

This is the caller side of the solver path: in BoSSS the matrix handed to the linear solvers is assembled by
``BoSSS.Foundation`` from the flux forms in ``src/L3-solution/BoSSS.Solution.NSECommon/ipLaplace.cs:95-245``.
This module restates that discretisation for axis-aligned box cells, vectorised with numpy, and returns the
operator as a block-sparse (BSR) matrix with one dense Np x Np block per cell pair, in the layout that
``BlockMsrMatrix`` exposes through ``ReadBlock`` (row-major blocks, block columns sorted ascending per block row,
``src/L1-platform/BoSSS.Platform/BlockMsrMatrix.cs:315,1743``).

Conventions (all follow the reference):

* Basis: products of orthonormal Legendre polynomials on the reference box, scaled to be orthonormal on the
  physical cell; modes ordered by total degree and, within one degree, lexicographically by the exponent tuple
  (x, y[, z]) -- the order of ``OrthonormalPolynomials`` in ``src/L2-foundation/BoSSS.Foundation/Square.cs:194-250``
  and ``Cube_polynomials.cs:19-130``.  The leading Np(p') modes of a cell therefore span P_{p'}, which is what
  p-restriction (``GridAndDegRestriction``) relies on.
* Length scale: ``cj = 0.5 * (surface area + boundary area) / volume``
  (``src/L2-foundation/BoSSS.Foundation/GridData_CellData.cs:681-687``).
* Penalty: ``eta = penalty * max(cj_in, cj_out) * max(nu_in, nu_out)`` on inner faces and twice the one-sided
  value on Dirichlet faces (``ipLaplace.cs:131-143,224``).  ``penalty`` is ``penalty_base * max((p+1)(p+D)/D,
  (p+1)^2)`` in the reference; callers may instead pass the factor directly (e.g. ``(p+1)(p+2)``).
* Sign: the reference forms produce the negative Laplacian's negative, ``-a(u,v)``; this module assembles the
  symmetric positive definite ``a(u,v)`` for ``-div(nu grad u) = f``.  The solver path is indifferent to the
  sign (``SymmInv`` handles either sign of the diagonal).
* Cells are numbered lexicographically with x fastest.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional, Sequence

import numpy as np
from numpy.polynomial import legendre as npleg


# ----------------------------------------------------------------------------------------------------------------
# 1-D orthonormal Legendre helpers
# ----------------------------------------------------------------------------------------------------------------

def _legendre_coeffs(n: int) -> np.ndarray:
    c = np.zeros(n + 1)
    c[n] = math.sqrt((2 * n + 1) / 2.0)
    return c


def psi(n: int, t: np.ndarray) -> np.ndarray:
    """Orthonormal Legendre polynomial of degree n on [-1, 1]."""
    return npleg.legval(t, _legendre_coeffs(n))


def dpsi(n: int, t: np.ndarray) -> np.ndarray:
    return npleg.legval(t, npleg.legder(_legendre_coeffs(n)))


def gauss(q: int):
    return npleg.leggauss(q)


def np_of(D: int, p: int) -> int:
    """Number of modes of the total-degree space P_p in D dimensions (``PmgConfig.cs`` GetNp)."""
    if p < 0:
        return 0
    return math.comb(p + D, D)


def dg_modes(D: int, p: int) -> np.ndarray:
    """Exponent tuples of the basis, ordered by total degree then lexicographically (see module docstring)."""
    out = []
    for deg in range(p + 1):
        if D == 1:
            out.append((deg,))
        elif D == 2:
            for i in range(deg + 1):
                out.append((i, deg - i))
        elif D == 3:
            for i in range(deg + 1):
                for j in range(deg - i + 1):
                    out.append((i, j, deg - i - j))
        else:
            raise ValueError("D must be 1, 2 or 3")
    return np.asarray(out, dtype=np.int64)


def stiffness_1d(p: int) -> np.ndarray:
    """S[m, n] = int_{-1}^{1} psi_m' psi_n' dt."""
    t, w = gauss(p + 2)
    d = np.stack([dpsi(n, t) for n in range(p + 1)])
    return (d * w) @ d.T


# ----------------------------------------------------------------------------------------------------------------
# Grid
# ----------------------------------------------------------------------------------------------------------------

@dataclasses.dataclass
class RectilinearGrid:
    nodes: list  # one ascending node array per dimension

    @property
    def D(self) -> int:
        return len(self.nodes)

    @property
    def shape(self):
        return tuple(len(n) - 1 for n in self.nodes)

    @property
    def ncells(self) -> int:
        return int(np.prod(self.shape))

    def h(self, d: int) -> np.ndarray:
        return np.diff(np.asarray(self.nodes[d], dtype=np.float64))

    def cell_index_grid(self) -> np.ndarray:
        """Cell ids as an array indexed [i_{D-1}, ..., i_0] (x fastest in memory)."""
        return np.arange(self.ncells, dtype=np.int64).reshape(tuple(reversed(self.shape)))

    def cell_multi_index(self):
        ids = np.arange(self.ncells, dtype=np.int64)
        out = []
        for d in range(self.D):
            out.append(ids % self.shape[d])
            ids = ids // self.shape[d]
        return out

    def cell_sizes(self):
        mi = self.cell_multi_index()
        return [self.h(d)[mi[d]] for d in range(self.D)]

    def cell_centres(self):
        mi = self.cell_multi_index()
        out = []
        for d in range(self.D):
            n = np.asarray(self.nodes[d], dtype=np.float64)
            out.append(0.5 * (n[:-1] + n[1:])[mi[d]])
        return out

    def face_neighbours(self) -> np.ndarray:
        """[cells, 2D] neighbour ids in the order -x, +x, -y, +y, -z, +z (-1 on the boundary)."""
        mi = self.cell_multi_index()
        ids = np.arange(self.ncells, dtype=np.int64)
        out = np.full((self.ncells, 2 * self.D), -1, dtype=np.int32)
        stride = 1
        for d in range(self.D):
            lo = mi[d] > 0
            hi = mi[d] < self.shape[d] - 1
            out[lo, 2 * d] = (ids[lo] - stride).astype(np.int32)
            out[hi, 2 * d + 1] = (ids[hi] + stride).astype(np.int32)
            stride *= self.shape[d]
        return out

    def length_scale_cj(self) -> np.ndarray:
        """cj = 0.5 * (surface + boundary area) / volume, per cell (GridData_CellData.cs:681-687)."""
        hs = self.cell_sizes()
        vol = np.ones(self.ncells)
        for d in range(self.D):
            vol = vol * hs[d]
        surf = np.zeros(self.ncells)
        bnd = np.zeros(self.ncells)
        mi = self.cell_multi_index()
        for d in range(self.D):
            area = vol / hs[d]
            surf += 2 * area
            nb = (mi[d] == 0).astype(np.float64) + (mi[d] == self.shape[d] - 1).astype(np.float64)
            bnd += nb * area
        return 0.5 * (surf + bnd) / vol


def uniform_grid(D: int, n: int, lo: float = 0.0, hi: float = 1.0) -> RectilinearGrid:
    return RectilinearGrid([np.linspace(lo, hi, n + 1) for _ in range(D)])


def exponential_nodes(lo: float, hi: float, n_nodes: int, stretch: float) -> np.ndarray:
    """Geometrically stretched node distribution (cell size ratio ``stretch`` between neighbours)."""
    m = n_nodes - 1
    if stretch == 1.0:
        return np.linspace(lo, hi, n_nodes)
    r = stretch
    h0 = (hi - lo) * (r - 1.0) / (r ** m - 1.0)
    x = lo + h0 * (r ** np.arange(n_nodes) - 1.0) / (r - 1.0)
    x[-1] = hi
    return x


# ----------------------------------------------------------------------------------------------------------------
# Assembled system
# ----------------------------------------------------------------------------------------------------------------

@dataclasses.dataclass
class BsrSystem:
    """A block-sparse operator with uniform Np x Np blocks plus a right-hand side."""
    Np: int
    row_ptr: np.ndarray   # int64 [nb+1]
    col_idx: np.ndarray   # int32 [nnzb]
    values: np.ndarray    # float64 [nnzb, Np, Np], row-major blocks
    rhs: np.ndarray       # float64 [nb*Np]
    D: int = 0
    p: int = 0
    grid: Optional[RectilinearGrid] = None
    coeff: Optional[np.ndarray] = None

    @property
    def nb(self) -> int:
        return len(self.row_ptr) - 1

    @property
    def nnzb(self) -> int:
        return len(self.col_idx)

    @property
    def N(self) -> int:
        return self.nb * self.Np

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.bsr_matrix((self.values, self.col_idx.astype(np.int64), self.row_ptr),
                             shape=(self.N, self.N)).tocsr()


BoundaryKind = Callable[[int, int, np.ndarray], np.ndarray]


def _face_vectors(p: int, h: np.ndarray, side: float):
    """Traces of basis values and d/dx on the face at reference coordinate ``side`` (+1 or -1).

    Returns arrays [nf, p+1]: t[n] = sqrt(2/h) psi_n(side), d[n] = sqrt(2/h) (2/h) psi_n'(side).
    """
    tv = np.array([psi(n, np.array([side]))[0] for n in range(p + 1)])
    dv = np.array([dpsi(n, np.array([side]))[0] for n in range(p + 1)])
    s = np.sqrt(2.0 / h)[:, None]
    return s * tv[None, :], (s * (2.0 / h)[:, None]) * dv[None, :]


def _expand_1d(F: np.ndarray, modes: np.ndarray, d: int) -> np.ndarray:
    """Map per-face 1-D matrices F[nf, p+1, p+1] (direction d) to Np x Np blocks with the transverse delta."""
    a = modes[:, d]
    other = [e for e in range(modes.shape[1]) if e != d]
    mask = np.ones((len(modes), len(modes)), dtype=bool)
    for e in other:
        mask &= modes[:, e][:, None] == modes[:, e][None, :]
    return F[:, a[:, None], a[None, :]] * mask[None, :, :]


def assemble_sip(grid: RectilinearGrid, p: int, *, penalty: Optional[float] = None,
                 penalty_base: float = 1.3, coeff: Optional[np.ndarray] = None,
                 boundary: Optional[Callable] = None,
                 dirichlet_g: Optional[Callable] = None, neumann_g: Optional[Callable] = None,
                 rhs_f: Optional[Callable] = None, rhs_cellwise: Optional[np.ndarray] = None,
                 quad: Optional[int] = None) -> BsrSystem:
    """Assemble the SIP operator ``a(u, v)`` and the load vector for ``-div(nu grad u) = f``.

    ``boundary(d, side, x_face_centres) -> bool array`` says which boundary faces are Dirichlet (True) or
    Neumann (False); default: all Dirichlet.  ``coeff`` is a per-cell diffusivity nu (default 1).
    ``penalty`` overrides ``penalty_base * max((p+1)(p+D)/D, (p+1)^2)``.
    ``rhs_f(X)`` takes a list of D coordinate arrays; ``rhs_cellwise`` gives the projected load directly.
    """
    D = grid.D
    modes = dg_modes(D, p)
    Np = len(modes)
    nc = grid.ncells
    if penalty is None:
        penalty = penalty_base * max((p + 1) * (p + D) / D, (p + 1) ** 2)
    nu = np.ones(nc) if coeff is None else np.asarray(coeff, dtype=np.float64)
    uniform = all(np.allclose(grid.h(d), grid.h(d)[0], rtol=1e-13, atol=0) for d in range(D))
    if uniform and boundary is None and dirichlet_g is None and neumann_g is None:
        values, row_ptr, col_idx = _assemble_uniform(grid, p, penalty, nu)
        rhs = np.zeros((nc, Np))
        if rhs_cellwise is not None:
            rhs += rhs_cellwise
        elif rhs_f is not None:
            rhs += project_function(grid, p, rhs_f, q=quad if quad is not None else p + 2)
        return BsrSystem(Np=Np, row_ptr=row_ptr, col_idx=col_idx, values=values, rhs=rhs.reshape(-1),
                         D=D, p=p, grid=grid, coeff=None if coeff is None else nu)
    cj = grid.length_scale_cj()
    hs = grid.cell_sizes()
    mi = grid.cell_multi_index()
    shape = grid.shape
    strides = [int(np.prod(shape[:d])) for d in range(D)]

    # --- diagonal blocks: volume term
    S = stiffness_1d(p)
    diag = np.zeros((nc, Np, Np))
    for d in range(D):
        F = (nu * 4.0 / hs[d] ** 2)[:, None, None] * S[None, :, :]
        diag += _expand_1d(F, modes, d)

    off_rows, off_cols, off_vals = [], [], []
    rhs = np.zeros((nc, Np))
    q = quad if quad is not None else p + 2

    for d in range(D):
        # ---- inner faces in direction d
        has_r = mi[d] < shape[d] - 1
        L = np.nonzero(has_r)[0]
        R = L + strides[d]
        hL, hR = hs[d][L], hs[d][R]
        kL, kR = nu[L], nu[R]
        eta = penalty * np.maximum(cj[L], cj[R]) * np.maximum(kL, kR)
        tL, dL = _face_vectors(p, hL, +1.0)
        tR, dR = _face_vectors(p, hR, -1.0)
        o = lambda a, b: a[:, :, None] * b[:, None, :]   # outer[m, n] = a[m] b[n]
        FLL = -0.5 * kL[:, None, None] * (o(tL, dL) + o(dL, tL)) + eta[:, None, None] * o(tL, tL)
        FLR = -0.5 * kR[:, None, None] * o(tL, dR) + 0.5 * kL[:, None, None] * o(dL, tR) \
            - eta[:, None, None] * o(tL, tR)
        FRR = 0.5 * kR[:, None, None] * (o(tR, dR) + o(dR, tR)) + eta[:, None, None] * o(tR, tR)
        np.add.at(diag, L, _expand_1d(FLL, modes, d))
        np.add.at(diag, R, _expand_1d(FRR, modes, d))
        BLR = _expand_1d(FLR, modes, d)
        off_rows += [L, R]
        off_cols += [R, L]
        off_vals += [BLR, np.transpose(BLR, (0, 2, 1))]

        # ---- boundary faces in direction d
        for side in (-1.0, +1.0):
            K = np.nonzero(mi[d] == (0 if side < 0 else shape[d] - 1))[0]
            if len(K) == 0:
                continue
            hK = hs[d][K]
            xc = [c[K] for c in grid.cell_centres()]
            xc[d] = np.full(len(K), grid.nodes[d][0] if side < 0 else grid.nodes[d][-1])
            is_dir = np.ones(len(K), dtype=bool) if boundary is None else np.asarray(boundary(d, side, xc), bool)
            t, dv = _face_vectors(p, hK, side)
            kK = nu[K]
            etaB = 2.0 * penalty * cj[K] * kK
            sgn = -side  # +1 on the low face (normal -e_d), -1 on the high face
            o = lambda a, b: a[:, :, None] * b[:, None, :]
            FB = sgn * kK[:, None, None] * (o(t, dv) + o(dv, t)) + etaB[:, None, None] * o(t, t)
            FB = FB * is_dir[:, None, None]
            np.add.at(diag, K, _expand_1d(FB, modes, d))
            if dirichlet_g is not None or neumann_g is not None:
                rhs += _boundary_load(grid, p, modes, d, side, K, hK, t, dv, kK, etaB, is_dir,
                                      dirichlet_g, neumann_g, q)

    # ---- load vector
    if rhs_cellwise is not None:
        rhs += rhs_cellwise
    elif rhs_f is not None:
        rhs += project_function(grid, p, rhs_f, q=q)

    # ---- BSR structure: rows sorted, columns ascending within a row
    rows = np.concatenate([np.arange(nc, dtype=np.int64)] + off_rows)
    cols = np.concatenate([np.arange(nc, dtype=np.int64)] + off_cols)
    key = rows * nc + cols
    order = np.argsort(key, kind="stable")
    pos = np.empty_like(order)
    pos[order] = np.arange(len(order))
    nnzb = len(rows)
    values = np.empty((nnzb, Np, Np))
    values[pos[:nc]] = diag
    start = nc
    for blk in off_vals:
        values[pos[start:start + len(blk)]] = blk
        start += len(blk)
    row_ptr = np.zeros(nc + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=nc), out=row_ptr[1:])
    col_idx = cols[order].astype(np.int32)
    return BsrSystem(Np=Np, row_ptr=row_ptr, col_idx=col_idx, values=values, rhs=rhs.reshape(-1),
                     D=D, p=p, grid=grid, coeff=None if coeff is None else nu)


def _assemble_uniform(grid: RectilinearGrid, p: int, penalty: float, nu: np.ndarray):
    """Same operator as the general path for uniformly spaced grids with Dirichlet boundaries everywhere.

    Every block is a linear combination of a few Np x Np templates (the 1-D face/volume matrices expanded with the
    transverse delta) with per-cell / per-face coefficients (diffusivity and penalty), evaluated as one matrix
    product per block kind and written straight into a [cells, 7 slots] layout whose slots are the block columns in
    ascending order (-z, -y, -x, self, +x, +y, +z); missing neighbours are squeezed out at the end.
    """
    D = grid.D
    modes = dg_modes(D, p)
    Np = len(modes)
    shape = grid.shape                       # (n0, n1, n2): x fastest
    gshape = tuple(reversed(shape))          # array axes (z, y, x)
    nc = grid.ncells
    h = [float(grid.h(d)[0]) for d in range(D)]
    cj = grid.length_scale_cj().reshape(gshape)
    k = nu.reshape(gshape)
    S = stiffness_1d(p)
    o = lambda a, b: np.outer(a, b)
    ex = lambda F, d: _expand_1d(F[None], modes, d)[0].reshape(-1)

    # ---- diagonal templates
    tmpl = [sum(ex(4.0 / h[d] ** 2 * S, d) for d in range(D))]
    coef = [k.reshape(-1)]
    per_d = []
    for d in range(D):
        tL, dL = (v[0] for v in _face_vectors(p, np.array([h[d]]), +1.0))
        tR, dR = (v[0] for v in _face_vectors(p, np.array([h[d]]), -1.0))
        per_d.append((tL, dL, tR, dR))
        tmpl += [ex(-0.5 * (o(tL, dL) + o(dL, tL)), d), ex(o(tL, tL), d),
                 ex(0.5 * (o(tR, dR) + o(dR, tR)), d), ex(o(tR, tR), d)]
        ax = D - 1 - d                       # array axis of direction d
        n = shape[d]
        sl_lo = [slice(None)] * D
        sl_hi = [slice(None)] * D
        sl_lo[ax] = slice(0, n - 1)
        sl_hi[ax] = slice(1, n)
        sl_lo, sl_hi = tuple(sl_lo), tuple(sl_hi)
        eta_face = penalty * np.maximum(cj[sl_lo], cj[sl_hi]) * np.maximum(k[sl_lo], k[sl_hi])
        eta_b = 2.0 * penalty * cj * k
        m_plus = np.full(gshape, 2.0)
        m_plus[sl_lo] = 1.0                  # interior face towards +d
        eta_plus = eta_b.copy()
        eta_plus[sl_lo] = eta_face
        m_minus = np.full(gshape, 2.0)
        m_minus[sl_hi] = 1.0
        eta_minus = eta_b.copy()
        eta_minus[sl_hi] = eta_face
        coef += [(k * m_plus).reshape(-1), eta_plus.reshape(-1), (k * m_minus).reshape(-1), eta_minus.reshape(-1)]
    T = np.stack(tmpl)                       # [t, Np*Np]
    Cc = np.stack(coef, axis=1)              # [cells, t]

    nslot = 2 * D + 1
    full = np.zeros(gshape + (nslot, Np * Np))
    full[..., D, :] = (Cc @ T).reshape(gshape + (Np * Np,))
    exists = np.zeros(gshape + (nslot,), dtype=bool)
    exists[..., D] = True
    offsets = np.zeros(nslot, dtype=np.int64)
    for d in range(D):
        tL, dL, tR, dR = per_d[d]
        ax = D - 1 - d
        n = shape[d]
        stride = int(np.prod(shape[:d]))
        sl_lo = [slice(None)] * D
        sl_hi = [slice(None)] * D
        sl_lo[ax] = slice(0, n - 1)
        sl_hi[ax] = slice(1, n)
        sl_lo, sl_hi = tuple(sl_lo), tuple(sl_hi)
        kL, kR = k[sl_lo], k[sl_hi]
        eta = penalty * np.maximum(cj[sl_lo], cj[sl_hi]) * np.maximum(kL, kR)
        P, Q, R = (-0.5 * o(tL, dR)), (0.5 * o(dL, tR)), (-o(tL, tR))
        TLR = np.stack([ex(P, d), ex(Q, d), ex(R, d)])
        TRL = np.stack([ex(P.T, d), ex(Q.T, d), ex(R.T, d)])
        cf = np.stack([kR.reshape(-1), kL.reshape(-1), eta.reshape(-1)], axis=1)
        plus, minus = D + 1 + d, D - 1 - d
        offsets[plus], offsets[minus] = stride, -stride
        full[sl_lo + (plus,)] = (cf @ TLR).reshape(kL.shape + (Np * Np,))
        full[sl_hi + (minus,)] = (cf @ TRL).reshape(kL.shape + (Np * Np,))
        exists[sl_lo + (plus,)] = True
        exists[sl_hi + (minus,)] = True
    ex_flat = exists.reshape(nc, nslot)
    values = full.reshape(nc, nslot, Np * Np)[ex_flat].reshape(-1, Np, Np)
    row_ptr = np.zeros(nc + 1, dtype=np.int64)
    np.cumsum(ex_flat.sum(axis=1), out=row_ptr[1:])
    cols = np.arange(nc, dtype=np.int64)[:, None] + offsets[None, :]
    col_idx = cols[ex_flat].astype(np.int32)
    return values, row_ptr, col_idx


def _boundary_load(grid, p, modes, d, side, K, hK, t, dv, kK, etaB, is_dir, g_d, g_n, q):
    """Load contributions of inhomogeneous Dirichlet / Neumann data on boundary faces."""
    D = grid.D
    Np = len(modes)
    tg, wg = gauss(q)
    other = [e for e in range(D) if e != d]
    hs = grid.cell_sizes()
    xc = grid.cell_centres()
    out = np.zeros((len(K), Np))
    # tensor quadrature over the transverse directions
    grids = np.meshgrid(*([tg] * len(other)), indexing="ij") if other else []
    wts = np.ones(1)
    for _ in other:
        wts = np.multiply.outer(wts, wg).reshape(-1)
    pts = [g.reshape(-1) for g in grids]
    xface = grid.nodes[d][0] if side < 0 else grid.nodes[d][-1]
    X = [None] * D
    X[d] = np.full((len(K), len(wts)), xface)
    jac = np.ones(len(K))
    for ie, e in enumerate(other):
        he = hs[e][K]
        X[e] = xc[e][K][:, None] + 0.5 * he[:, None] * pts[ie][None, :]
        jac = jac * 0.5 * he
    # transverse basis values at the quadrature points: phi_e = sqrt(2/h_e) psi_{a_e}(t)
    trans = np.ones((len(K), len(wts), Np))
    for ie, e in enumerate(other):
        he = hs[e][K]
        vals = np.stack([psi(n, pts[ie]) for n in range(p + 1)], axis=-1)  # [nq, p+1]
        trans = trans * (np.sqrt(2.0 / he)[:, None, None] * vals[None, :, modes[:, e]])
    normal_sign = side  # outward normal = side * e_d
    if g_d is not None:
        g = np.asarray(g_d(X), dtype=np.float64) * is_dir[:, None]
        # l(v) += int ( -nu dn v g + eta v g )
        phi = trans * t[:, None, modes[:, d]]
        dnphi = normal_sign * trans * dv[:, None, modes[:, d]]
        integrand = (-kK[:, None, None] * dnphi + etaB[:, None, None] * phi) * g[:, :, None]
        out += np.einsum("kqa,q->ka", integrand, wts) * jac[:, None]
    if g_n is not None:
        g = np.asarray(g_n(X), dtype=np.float64) * (~is_dir)[:, None]
        phi = trans * t[:, None, modes[:, d]]
        out += np.einsum("kqa,q->ka", phi * g[:, :, None], wts) * jac[:, None]
    full = np.zeros((grid.ncells, Np))
    np.add.at(full, K, out)
    return full


def project_function(grid: RectilinearGrid, p: int, f: Callable, q: Optional[int] = None) -> np.ndarray:
    """L2 projection coefficients b[cell, a] = int_cell f phi_a (tensor Gauss rule, q points per direction)."""
    D = grid.D
    modes = dg_modes(D, p)
    q = q if q is not None else p + 2
    tg, wg = gauss(q)
    hs = grid.cell_sizes()
    xc = grid.cell_centres()
    grids = np.meshgrid(*([tg] * D), indexing="ij")
    pts = [g.reshape(-1) for g in grids]
    wts = np.ones(1)
    for _ in range(D):
        wts = np.multiply.outer(wts, wg).reshape(-1)
    X = [xc[d][:, None] + 0.5 * hs[d][:, None] * pts[d][None, :] for d in range(D)]
    fv = np.asarray(f(X), dtype=np.float64)
    basis = np.ones((grid.ncells, len(wts), len(modes)))
    jac = np.ones(grid.ncells)
    for d in range(D):
        vals = np.stack([psi(n, pts[d]) for n in range(p + 1)], axis=-1)
        basis = basis * (np.sqrt(2.0 / hs[d])[:, None, None] * vals[None, :, modes[:, d]])
        jac = jac * 0.5 * hs[d]
    return np.einsum("cq,cqa,q->ca", fv, basis, wts) * jac[:, None]


# ----------------------------------------------------------------------------------------------------------------
# h-levels: agglomeration of 2^D cells and exact polynomial prolongation
# ----------------------------------------------------------------------------------------------------------------

@dataclasses.dataclass
class HProlongation:
    """Prolongation from an agglomerated grid to the finer one, in the orthonormal DG basis of degree p.

    Block-sparse: row block = fine cell, column block = coarse cell (its agglomerate), each block Np x Np
    row-major; the counterpart of the prolongation operators of BoSSS's multigrid hierarchy on aggregation
    grids (MultigridOperator.cs:774,815 Restrict/Prolongate; AggregationGridBasis.cs)."""
    Np: int
    nb_fine: int
    nb_coarse: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray   # [nb_fine, Np, Np]
    coarse_grid: RectilinearGrid


def _child_projection_1d(p: int, side: int) -> np.ndarray:
    """T[j, k] = int_child psi^f_j psi^c_k with both bases orthonormal on their own interval (child = left/right half)."""
    tg, wg = gauss(p + 2)
    # fine reference coordinate t in [-1,1] -> coarse coordinate s = (t - 1)/2 (left) or (t + 1)/2 (right)
    s = 0.5 * (tg + (1.0 if side else -1.0))
    F = np.stack([psi(j, tg) for j in range(p + 1)])          # fine basis on its reference interval
    Cc = np.stack([psi(k, s) for k in range(p + 1)])          # coarse basis evaluated in the child
    # physical scaling: fine basis sqrt(2/h), coarse sqrt(2/(2h)); dx = h/2 dt  -> factor sqrt(1/2)
    return (F * wg) @ Cc.T * math.sqrt(0.5)


def h_prolongation(grid: RectilinearGrid, p: int) -> HProlongation:
    """2^D -> 1 agglomeration of a uniformly refined grid (every direction even)."""
    D = grid.D
    assert all(n % 2 == 0 for n in grid.shape), "every direction needs an even number of cells"
    modes = dg_modes(D, p)
    Np = len(modes)
    T = [_child_projection_1d(p, s) for s in (0, 1)]
    cg = RectilinearGrid([np.asarray(grid.nodes[d])[::2] for d in range(D)])
    mi = grid.cell_multi_index()
    coarse = np.zeros(grid.ncells, dtype=np.int64)
    child = np.zeros(grid.ncells, dtype=np.int64)
    stride = 1
    for d in range(D):
        coarse += (mi[d] // 2) * stride
        child += (mi[d] % 2) << d
        stride *= cg.shape[d]
    blocks = np.empty((2 ** D, Np, Np))
    for c in range(2 ** D):
        M = np.ones((Np, Np))
        for d in range(D):
            M = M * T[(c >> d) & 1][modes[:, d][:, None], modes[:, d][None, :]]
        blocks[c] = M
    return HProlongation(Np=Np, nb_fine=grid.ncells, nb_coarse=cg.ncells,
                         row_ptr=np.arange(grid.ncells + 1, dtype=np.int64), col_idx=coarse.astype(np.int32),
                         values=blocks[child], coarse_grid=cg)


def h_hierarchy(grid: RectilinearGrid, p: int, min_cells: int = 64) -> list:
    """Successive 2^D agglomerations while every direction stays even and the grid has more than min_cells."""
    out = []
    g = grid
    while all(n % 2 == 0 for n in g.shape) and g.ncells > min_cells:
        P = h_prolongation(g, p)
        out.append(P)
        g = P.coarse_grid
    return out


# ----------------------------------------------------------------------------------------------------------------
# Seeded synthetic right-hand sides and coefficients
# ----------------------------------------------------------------------------------------------------------------

@dataclasses.dataclass
class SineModes:
    """f(x) = sum_m a_m prod_d sin(pi k_{m,d} x_d); k ~ U{1..8}, a ~ N(0,1) from ``default_rng(seed)``."""
    k: np.ndarray  # [M, D] int
    a: np.ndarray  # [M]

    @staticmethod
    def seeded(seed: int, D: int, M: int = 16, kmax: int = 8) -> "SineModes":
        rng = np.random.default_rng(seed)
        k = rng.integers(1, kmax + 1, size=(M, D))
        a = rng.standard_normal(M)
        return SineModes(k=k, a=a)

    def __call__(self, X):
        out = np.zeros_like(X[0])
        for m in range(len(self.a)):
            term = np.full_like(X[0], self.a[m])
            for d in range(len(X)):
                term = term * np.sin(math.pi * self.k[m, d] * X[d])
            out += term
        return out

    def on_tensor_points(self, lo: np.ndarray, h: float, t1d: np.ndarray) -> np.ndarray:
        """f on the tensor points lo_k + (t1d + 1) h / 2 of every cell k: [cells, n1, n1, n1] (x, y, z order),
        from one sine table per direction."""
        S = [np.sin(math.pi * self.k[None, :, d, None] * (lo[:, None, None, d] + (t1d[None, None, :] + 1) * (h / 2)))
             for d in range(3)]                                                     # [cells, M, n1]
        return np.einsum("m,kmi,kmj,kml->kijl", self.a, S[0], S[1], S[2], optimize=True)

    def tables_1d(self, grid: RectilinearGrid, p: int, q: Optional[int] = None) -> np.ndarray:
        """The 1-D projections of every mode and direction, [M, D, n_d, p+1] (grids with equal extents; the
        per-cell load vector is the product over the directions summed over the modes, as in ``project``)."""
        D = grid.D
        q = q if q is not None else p + 6
        tg, wg = gauss(q)
        vals = np.stack([psi(j, tg) for j in range(p + 1)], axis=-1)  # [q, p+1]
        out = []
        for m in range(len(self.a)):
            per_d = []
            for d in range(D):
                n = np.asarray(grid.nodes[d], dtype=np.float64)
                h = np.diff(n)
                xq = 0.5 * (n[:-1] + n[1:])[:, None] + 0.5 * h[:, None] * tg[None, :]
                I = (np.sin(math.pi * self.k[m, d] * xq) * wg[None, :]) @ vals
                per_d.append(I * (0.5 * h * np.sqrt(2.0 / h))[:, None])
            out.append(per_d)
        return out

    def project_on_gpu(self, grid: RectilinearGrid, p: int, q: Optional[int] = None, out=None):
        """``project`` with the products and mode sums evaluated on the GPU (bsgpu_project_separable); returns a
        CUDA tensor [cells * Np] (or fills ``out``)."""
        import ctypes as C
        import torch
        from . import native as nat
        D = grid.D
        tabs = self.tables_1d(grid, p, q)
        flat = np.concatenate([np.ascontiguousarray(tabs[m][d]).reshape(-1)
                               for m in range(len(self.a)) for d in range(D)]) if len(self.a) else np.zeros(1)
        coef = np.ascontiguousarray(self.a, np.float64)
        Np = np_of(D, p)
        if out is None:
            out = torch.empty(grid.ncells * Np, dtype=torch.float64, device="cuda")
        shape = (C.c_int32 * D)(*grid.shape)
        nat.check(nat.lib().bsgpu_project_separable(D, shape, int(p), len(self.a), nat.ptr(coef), nat.ptr(flat),
                                                    nat.ptr(out), nat.DEVICE_POINTERS))
        return out

    def project(self, grid: RectilinearGrid, p: int, q: Optional[int] = None) -> np.ndarray:
        """Separable projection: per mode and direction a 1-D Gauss integral, combined by outer products."""
        D = grid.D
        modes = dg_modes(D, p)
        q = q if q is not None else p + 6
        tg, wg = gauss(q)
        out = np.zeros((grid.ncells, len(modes)))
        mi = grid.cell_multi_index()
        one_d = []
        for d in range(D):
            n = np.asarray(grid.nodes[d], dtype=np.float64)
            h = np.diff(n)
            xq = 0.5 * (n[:-1] + n[1:])[:, None] + 0.5 * h[:, None] * tg[None, :]
            vals = np.stack([psi(j, tg) for j in range(p + 1)], axis=-1)  # [q, p+1]
            one_d.append((xq, h, vals))
        for m in range(len(self.a)):
            term = np.full((grid.ncells, len(modes)), self.a[m])
            for d in range(D):
                xq, h, vals = one_d[d]
                I = (np.sin(math.pi * self.k[m, d] * xq) * wg[None, :]) @ vals  # [n_d, p+1]
                I = I * (0.5 * h * np.sqrt(2.0 / h))[:, None]
                term = term * I[mi[d]][:, modes[:, d]]
            out += term
        return out


def gaussian_random_field(shape: Sequence[int], spacing: float, length: float = 0.1, variance: float = 1.0,
                          seed: int = 0) -> np.ndarray:
    """Squared-exponential GRF sampled at cell centres by circulant embedding on a padded periodic grid.

    Negative eigenvalues of the embedding (if any) are clipped to zero.  Returns an array in the cell order of
    ``RectilinearGrid`` (x fastest).
    """
    rng = np.random.default_rng(seed)
    D = len(shape)
    pad = [2 * n for n in shape]
    coords = []
    for n in pad:
        i = np.arange(n)
        i = np.minimum(i, n - i)
        coords.append(i * spacing)
    mesh = np.meshgrid(*coords, indexing="ij")
    r2 = sum(m ** 2 for m in mesh)
    cov = variance * np.exp(-r2 / (2.0 * length ** 2))
    lam = np.real(np.fft.fftn(cov))
    lam = np.maximum(lam, 0.0)
    noise = rng.standard_normal(pad) + 1j * rng.standard_normal(pad)
    field = np.fft.ifftn(np.sqrt(lam) * noise) * math.sqrt(np.prod(pad))
    g = np.real(field)[tuple(slice(0, n) for n in shape)]
    # index [i0, i1, i2] -> flatten with i0 fastest
    return np.ascontiguousarray(np.transpose(g, tuple(reversed(range(D))))).reshape(-1)


# ----------------------------------------------------------------------------------------------------------------
# The benchmark systems
# ----------------------------------------------------------------------------------------------------------------

def poisson_2d_c1(seed: int = 0, n: int = 64, p: int = 2) -> BsrSystem:
    """2-D SIP Poisson, n x n quads on [0,1]^2, Dirichlet 0, penalty factor (p+1)(p+2), sine-mode RHS."""
    g = uniform_grid(2, n)
    rhs = SineModes.seeded(seed, 2).project(g, p)
    return assemble_sip(g, p, penalty=(p + 1) * (p + 2), rhs_cellwise=rhs)


def poisson_3d(n: int, p: int, seed: int = 0) -> BsrSystem:
    """3-D SIP Poisson, n^3 hexes on [0,1]^3, Dirichlet 0, penalty factor (p+1)(p+2), sine-mode RHS."""
    g = uniform_grid(3, n)
    rhs = SineModes.seeded(seed, 3).project(g, p)
    return assemble_sip(g, p, penalty=(p + 1) * (p + 2), rhs_cellwise=rhs)


def log_coeff_features(system: BsrSystem) -> np.ndarray:
    """[cells, 1 + 2D] float32: log nu of each cell and of its face neighbours (-x, +x, ...; the cell's own value
    on the boundary) -- the per-cell input of the learned stage besides the residuals."""
    nbr = system.grid.face_neighbours()
    lk = np.log(np.ones(system.nb) if system.coeff is None else np.asarray(system.coeff, np.float64))
    nb_lk = np.where(nbr >= 0, lk[np.maximum(nbr, 0)], lk[:, None])
    return np.concatenate([lk[:, None], nb_lk], axis=1).astype(np.float32)


def variable_coeff_3d(n: int, p: int, seed: int = 0, length: float = 0.1, variance: float = 1.0) -> BsrSystem:
    """3-D SIP diffusion with nu = exp(g), g a squared-exponential GRF evaluated per cell."""
    g = uniform_grid(3, n)
    field = gaussian_random_field((n, n, n), 1.0 / n, length, variance, seed=seed + 1000)
    nu = np.exp(field)
    rhs = SineModes.seeded(seed, 3).project(g, p)
    return assemble_sip(g, p, penalty=(p + 1) * (p + 2), coeff=nu, rhs_cellwise=rhs)
