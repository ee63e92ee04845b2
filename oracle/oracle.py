"""ORACLE -- test infrastructure only.

ctypes front end of the CPU restatement in ``oracle.cpp`` plus an FP64 sparse direct solve (scipy ``splu``).
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import this module; the
product library (``bosss_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PCG, FGMRES_PMG, ORTHOMG, SOFTGMRES = 0, 1, 2, 3
COARSE_DENSE, COARSE_PCG = 0, 1
SMOOTHER_BLOCKJACOBI, SMOOTHER_SCHWARZ, SMOOTHER_ILU_COLOURED, SMOOTHER_ILU_NATURAL, SMOOTHER_SCHWARZ_BLOCKS = 0, 1, 2, 3, 4
TERM_DEFAULT, TERM_RELATIVE = 0, 1


class _Bsr(C.Structure):
    _fields_ = [("nb", C.c_int64), ("Np", C.c_int32), ("nspc", C.c_void_p), ("row_ptr", C.c_void_p),
                ("col_idx", C.c_void_p), ("values", C.c_void_p)]


class _Cfg(C.Structure):
    _fields_ = [("solver", C.c_int32), ("top_mode", C.c_int32), ("tol", C.c_double), ("max_iter", C.c_int32),
                ("min_iter", C.c_int32), ("max_krylov", C.c_int32), ("n_levels", C.c_int32),
                ("level_keep", C.c_int32 * 8), ("post_sweeps", C.c_int32), ("bj_iters", C.c_int32),
                ("bj_omega", C.c_double), ("coarse_kind", C.c_int32), ("coarse_tol", C.c_double),
                ("coarse_max_iter", C.c_int32), ("sub_max_iter", C.c_int32), ("sub_reduction", C.c_double),
                ("reference_fgmres_defect", C.c_int32), ("recalc_resi_period", C.c_int32), ("smoother", C.c_int32),
                ("schwarz_parts", C.c_int32), ("schwarz_overlap", C.c_int32), ("schwarz_scaling", C.c_int32)]


class _Stats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("nested", C.c_int32), ("converged", C.c_int32),
                ("n_hist", C.c_int32), ("res0", C.c_double), ("res", C.c_double)]


def build() -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        _LIB = C.CDLL(path)
        _LIB.or_last_error.restype = C.c_char_p
    return _LIB


def _check(rc):
    if rc != 0:
        raise ArithmeticError(f"oracle error {rc}: {lib().or_last_error().decode()}")


def set_threads(n: int) -> int:
    return lib().or_set_threads(int(n))


@dataclass
class Bsr:
    """Keeps the numpy arrays alive while the C view points at them."""
    Np: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray
    nspc: np.ndarray | None = None
    _c: _Bsr = field(default=None, repr=False)

    @staticmethod
    def of(system_or_arrays, values=None) -> "Bsr":
        s = system_or_arrays
        nspc = getattr(s, "nspc", None)
        v = s.values if values is None else values
        b = Bsr(Np=int(s.Np), row_ptr=np.ascontiguousarray(s.row_ptr, np.int64),
                col_idx=np.ascontiguousarray(s.col_idx, np.int32),
                values=np.ascontiguousarray(v, np.float64).reshape(-1),
                nspc=None if nspc is None else np.ascontiguousarray(nspc, np.int32))
        b._c = _Bsr(len(b.row_ptr) - 1, b.Np, None if b.nspc is None else b.nspc.ctypes.data,
                    b.row_ptr.ctypes.data, b.col_idx.ctypes.data, b.values.ctypes.data)
        return b

    @property
    def nb(self):
        return len(self.row_ptr) - 1

    @property
    def block_len(self):
        return (np.ones(self.nb, np.int64) if self.nspc is None else self.nspc.astype(np.int64)) * self.Np

    @property
    def N(self):
        return int(self.block_len.sum())


def spmv(A: Bsr, alpha: float, x: np.ndarray, beta: float, y: np.ndarray) -> np.ndarray:
    """BlockMsrMatrix.SpMV restatement: y <- beta*y + alpha*A*x (in place)."""
    x = np.ascontiguousarray(x, np.float64)
    assert y.dtype == np.float64 and y.flags.c_contiguous
    _check(lib().or_spmv(C.byref(A._c), C.c_double(alpha), x.ctypes.data_as(C.c_void_p), C.c_double(beta),
                         y.ctypes.data_as(C.c_void_p)))
    return y


def symminv(M: np.ndarray):
    n = M.shape[0]
    Mc = np.ascontiguousarray(M, np.float64).copy()
    L = np.zeros((n, n))
    _check(lib().or_symminv(n, Mc.ctypes.data_as(C.c_void_p), L.ctypes.data_as(C.c_void_p)))
    return L


def invert(M: np.ndarray) -> np.ndarray:
    Mc = np.ascontiguousarray(M, np.float64).copy()
    _check(lib().or_invert(Mc.shape[0], Mc.ctypes.data_as(C.c_void_p)))
    return Mc


def change_of_basis(A: Bsr):
    """Returns (values of L A L^T in the same block layout, concatenated L blocks)."""
    out = np.empty_like(A.values)
    Ltot = int((A.block_len ** 2).sum())
    L = np.empty(Ltot)
    _check(lib().or_change_of_basis(C.byref(A._c), out.ctypes.data_as(C.c_void_p), L.ctypes.data_as(C.c_void_p)))
    return out, L


def restrict(A: Bsr, keep: int):
    """Sub-matrix of the leading ``keep`` modes per species, and the sub -> full index map."""
    nspc = np.ones(A.nb, np.int64) if A.nspc is None else A.nspc.astype(np.int64)
    sub_len = nspc * keep
    rows = np.repeat(np.arange(A.nb), np.diff(A.row_ptr))
    nvals = int((sub_len[rows] * sub_len[A.col_idx]).sum())
    out = np.empty(nvals)
    mp = np.empty(int(sub_len.sum()), np.int64)
    _check(lib().or_restrict(C.byref(A._c), int(keep), out.ctypes.data_as(C.c_void_p),
                             mp.ctypes.data_as(C.c_void_p)))
    return out, mp


def schwarz_rows(A: Bsr) -> np.ndarray:
    """Centre-cell rows of the inverse of every cell-plus-neighbours block, in A's block layout."""
    out = np.empty_like(A.values)
    _check(lib().or_schwarz_rows(C.byref(A._c), out.ctypes.data_as(C.c_void_p)))
    return out


def _order_ptr(order):
    if order is None:
        return None, None
    o = np.ascontiguousarray(order, np.int32)
    return o, o.ctypes.data_as(C.c_void_p)


def ilu0_factor(A: Bsr, order=None) -> np.ndarray:
    """Block ILU(0) factors (CellILU.ComputeILU) over the block rows in ``order`` (None: natural order)."""
    keep, op = _order_ptr(order)
    out = np.empty_like(A.values)
    _check(lib().or_ilu0_factor(C.byref(A._c), op, out.ctypes.data_as(C.c_void_p)))
    return out


def ilu0_solve(A: Bsr, factor: np.ndarray, b: np.ndarray, order=None) -> np.ndarray:
    keep, op = _order_ptr(order)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.N)
    f = np.ascontiguousarray(factor, np.float64)
    _check(lib().or_ilu0_solve(C.byref(A._c), op, f.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                               x.ctypes.data_as(C.c_void_p)))
    return x


def schwarz_blocks(A: Bsr, parts: int = 0, overlap: int = 1):
    """Cell lists of the multi-cell Schwarz blocks (or_schwarz_blocks): (ptr [nblocks+1], cells)."""
    lib().or_schwarz_blocks.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]
    nb, tot = C.c_int64(), C.c_int64()
    _check(lib().or_schwarz_blocks(C.byref(A._c), int(parts), int(overlap), None, None, C.byref(nb), C.byref(tot)))
    ptr = np.zeros(nb.value + 1, np.int64)
    cells = np.zeros(max(tot.value, 1), np.int32)
    _check(lib().or_schwarz_blocks(C.byref(A._c), int(parts), int(overlap), ptr.ctypes.data, cells.ctypes.data,
                                   None, None))
    return ptr, cells[:tot.value]


def block_schwarz(A: Bsr, x: np.ndarray, b: np.ndarray, parts: int = 0, overlap: int = 1, scaling: bool = False,
                  iters: int = 1) -> np.ndarray:
    """Additive Schwarz with multi-cell blocks (Schwarz.cs:56): `iters` updates of x."""
    x = np.ascontiguousarray(x, np.float64).copy()
    b = np.ascontiguousarray(b, np.float64)
    lib().or_block_schwarz.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    _check(lib().or_block_schwarz(C.byref(A._c), int(parts), int(overlap), int(bool(scaling)), int(iters),
                                  x.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p)))
    return x


def blockjacobi(A: Bsr, x: np.ndarray, b: np.ndarray, iters: int = 1, omega: float = 1.0) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64).copy()
    b = np.ascontiguousarray(b, np.float64)
    _check(lib().or_blockjacobi(C.byref(A._c), int(iters), C.c_double(omega), x.ctypes.data_as(C.c_void_p),
                                b.ctypes.data_as(C.c_void_p)))
    return x


@dataclass
class SolverConfig:
    solver: int = FGMRES_PMG
    top_mode: int = TERM_RELATIVE
    tol: float = 1e-10
    max_iter: int = 300
    min_iter: int = 1
    max_krylov: int = 30
    level_keep: tuple = (20, 10, 4)
    post_sweeps: int = 10
    bj_iters: int = 1
    bj_omega: float = 1.0
    coarse_kind: int = COARSE_PCG
    coarse_tol: float = 1e-3
    coarse_max_iter: int = 2000
    sub_max_iter: int = 100
    sub_reduction: float = 0.1
    reference_fgmres_defect: bool = False
    recalc_resi_period: int = 1
    smoother: int = SMOOTHER_BLOCKJACOBI
    schwarz_parts: int = 0
    schwarz_overlap: int = 1
    schwarz_scaling: bool = False

    def _c(self) -> _Cfg:
        c = _Cfg()
        c.solver, c.top_mode, c.tol = self.solver, self.top_mode, self.tol
        c.max_iter, c.min_iter, c.max_krylov = self.max_iter, self.min_iter, self.max_krylov
        c.n_levels = len(self.level_keep)
        for i, k in enumerate(self.level_keep):
            c.level_keep[i] = int(k)
        c.post_sweeps, c.bj_iters, c.bj_omega = self.post_sweeps, self.bj_iters, self.bj_omega
        c.coarse_kind, c.coarse_tol, c.coarse_max_iter = self.coarse_kind, self.coarse_tol, self.coarse_max_iter
        c.sub_max_iter, c.sub_reduction = self.sub_max_iter, self.sub_reduction
        c.reference_fgmres_defect = int(bool(self.reference_fgmres_defect))
        c.recalc_resi_period = int(self.recalc_resi_period)
        c.smoother = int(self.smoother)
        c.schwarz_parts, c.schwarz_overlap = int(self.schwarz_parts), int(self.schwarz_overlap)
        c.schwarz_scaling = int(bool(self.schwarz_scaling))
        return c


@dataclass
class SolveResult:
    x: np.ndarray
    iterations: int
    nested: int
    converged: bool
    res0: float
    res: float
    history: np.ndarray


def solve(A: Bsr, b: np.ndarray, cfg: SolverConfig, x0: np.ndarray | None = None) -> SolveResult:
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.N) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
    st = _Stats()
    cap = 100000
    hist = np.zeros(cap)
    cc = cfg._c()
    _check(lib().or_solve(C.byref(A._c), C.byref(cc), b.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
                          C.byref(st), hist.ctypes.data_as(C.c_void_p), cap))
    return SolveResult(x=x, iterations=st.iterations, nested=st.nested, converged=bool(st.converged),
                       res0=st.res0, res=st.res, history=hist[:min(st.n_hist, cap)].copy())


class PersistentSolver:
    """Set-up once (level matrices, block inverses), then time only the solves."""

    def __init__(self, A: Bsr, cfg: SolverConfig):
        L = lib()
        L.or_solver_create.restype = C.c_void_p
        L.or_solver_create.argtypes = [C.c_void_p, C.c_void_p]
        L.or_solver_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_solver_destroy.argtypes = [C.c_void_p]
        self.A = A
        self._cfg = cfg._c()
        self._h = L.or_solver_create(C.byref(A._c), C.byref(self._cfg))
        if not self._h:
            raise ArithmeticError(f"oracle set-up failed: {L.or_last_error().decode()}")

    def solve(self, b: np.ndarray, x0: np.ndarray | None = None) -> SolveResult:
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.A.N) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        st = _Stats()
        _check(lib().or_solver_solve(self._h, b.ctypes.data_as(C.c_void_p), x.ctypes.data_as(C.c_void_p),
                                     C.byref(st)))
        return SolveResult(x=x, iterations=st.iterations, nested=st.nested, converged=bool(st.converged),
                           res0=st.res0, res=st.res, history=np.zeros(0))

    def __del__(self):
        try:
            if self._h:
                lib().or_solver_destroy(self._h)
        except Exception:
            pass


def direct_solve(system, rhs=None, refine: int = 2) -> np.ndarray:
    """FP64 sparse direct solve (scipy SuperLU) -- the exact-solution oracle for small systems -- followed by
    ``refine`` steps of iterative refinement (x += LU^{-1}(b - A x)), which the ill-conditioned XDG systems need
    (condition numbers ~5e9 with a 1:1000 jump leave the plain LU solution ~5e-9 off)."""
    import scipy.sparse.linalg as spla
    M = system.to_scipy().tocsc()
    b = system.rhs if rhs is None else rhs
    lu = spla.splu(M)
    x = lu.solve(b)
    for _ in range(refine):
        x = x + lu.solve(b - M @ x)
    return x
