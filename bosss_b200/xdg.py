"""XDG (extended DG) SIP Poisson with a sphere level set: workload generator for the uneven-block path.

Counterpart of the reference's XDG Poisson setups (``src/L4-application/XdgPoisson3/XdgPoisson3Main.cs:162-194``,
``HardCodedControl.cs:96-140`` Ball3D; forms ``src/L3-solution/BoSSS.Solution.XNSECommon/XLaplace.cs:55-300``).
Cells cut by the level set phi(x) = |x - c| - R carry two species (A inside, B outside), each with the cell's
full polynomial space restricted to its part of the cell, so the block length is Np or 2 Np
(``XdgAggregationBasis.GetLength``, ``XdgAggregationBasis.cs:775``).  The bilinear form is SIP per species in
the volumes and on the faces (diffusivity mu_s), plus SIP coupling of the two species on the interface,
    a_G(u, v) = int_G ( -{mu du/dn}[v] - {mu dv/dn}[u] + eta_G [u][v] ),  [u] = u_A - u_B,  n from A to B,
with eta_G = penalty * cj * max(mu_A, mu_B) (the "max |mu|" SIP variant).

Simplifications of the cut-cell machinery (the solver path, not the discretisation, is what this library
accelerates): volume integrals in cut cells use a subdivision rule (sub^3 sub-boxes, Gauss points classified by
the sign of phi); face integrals touching cut cells use sub^2 sub-squares likewise; the interface integral uses a
dense Fibonacci point set on the sphere with exact normals; species parts below `frac_min` of a cell are dropped
(BoSSS agglomerates them instead); cut cells keep the length scale of uncut ones.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .assembly import (RectilinearGrid, SineModes, _expand_1d, dg_modes, dpsi, gauss, psi,
                       stiffness_1d, uniform_grid)


@dataclasses.dataclass
class XdgSystem:
    Np: int
    nspc: np.ndarray        # species per cell (1 or 2)
    species: np.ndarray     # [cells, 2] bool: species A / B present
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray      # concatenated row-major blocks
    rhs: np.ndarray
    grid: RectilinearGrid
    p: int
    centre: np.ndarray
    radius: float
    mu: tuple

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


def _basis(p, modes, t, h):
    """Values and gradients of the cell basis at reference points t [P, 3] (cell size h)."""
    s = math.sqrt(2.0 / h)
    v1 = [np.stack([psi(n, t[:, d]) for n in range(p + 1)], -1) for d in range(3)]   # [P, p+1]
    g1 = [np.stack([dpsi(n, t[:, d]) for n in range(p + 1)], -1) for d in range(3)]
    val = s ** 3 * v1[0][:, modes[:, 0]] * v1[1][:, modes[:, 1]] * v1[2][:, modes[:, 2]]
    grad = []
    for d in range(3):
        parts = [g1[e] if e == d else v1[e] for e in range(3)]
        grad.append(s ** 3 * (2.0 / h) * parts[0][:, modes[:, 0]] * parts[1][:, modes[:, 1]] * parts[2][:, modes[:, 2]])
    return val, np.stack(grad, -1)   # [P, Np], [P, Np, 3]


def _fibonacci_sphere(M, centre, R):
    i = np.arange(M) + 0.5
    phi = np.arccos(1 - 2 * i / M)
    theta = math.pi * (1 + 5 ** 0.5) * i
    n = np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], -1)
    return centre[None, :] + R * n, n, np.full(M, 4 * math.pi * R * R / M)


def xdg_sphere(n: int = 48, p: int = 2, seed: int = 0, mu=(1.0, 1000.0), radius=None, centre=None,
               sub: int = 4, frac_min: float = 0.01, penalty=None, surface_points_per_cell: int = 64,
               rhs_f=None) -> XdgSystem:
    """``rhs_f(X)`` (list of coordinate arrays) replaces the seeded sine-mode right-hand side."""
    rng = np.random.default_rng(seed)
    R = 0.3 + rng.uniform(-0.05, 0.05) if radius is None else radius
    c = rng.uniform(0.4, 0.6, size=3) if centre is None else np.asarray(centre, float)
    g = uniform_grid(3, n)
    h = 1.0 / n
    modes = dg_modes(3, p)
    Np = len(modes)
    pen = (p + 1) * (p + 2) if penalty is None else penalty
    nc = g.ncells
    mi = g.cell_multi_index()
    lo = np.stack([mi[d] * h for d in range(3)], -1)          # cell lower corners [nc, 3]
    phi = lambda X: np.linalg.norm(X - c, axis=-1) - R

    # ---- sub-cell quadrature points (reference coordinates in [-1, 1]^3)
    tq, wq = gauss(p + 1)
    sb = (np.arange(sub) + 0.5) / sub * 2 - 1                   # sub-box centres
    T = []
    for a in sb:
        for b in sb:
            for cc in sb:
                for i1, x1 in enumerate(tq):
                    for i2, x2 in enumerate(tq):
                        for i3, x3 in enumerate(tq):
                            T.append((a + x1 / sub, b + x2 / sub, cc + x3 / sub, wq[i1] * wq[i2] * wq[i3] / sub ** 3))
    T = np.asarray(T)
    tpts, tw = T[:, :3], T[:, 3]
    nq1 = len(tq)
    t1d = (sb[:, None] + tq[None, :] / sub).reshape(-1)        # the 1-D coordinates of the tensor point set
    ga, gb, gc, g1, g2, g3 = np.indices((sub, sub, sub, nq1, nq1, nq1)).reshape(6, -1)
    ixyz = ((ga * nq1 + g1) * len(t1d) + (gb * nq1 + g2)) * len(t1d) + (gc * nq1 + g3)   # point -> tensor index
    wvol = tw * (h / 2) ** 3

    # ---- classify cells: species fractions from the sub-cell points
    centres = lo + h / 2
    dmin = np.abs(phi(centres)) - math.sqrt(3) * h / 2
    maybe_cut = np.nonzero(dmin < 0)[0]
    fracA = (phi(centres) < 0).astype(float)
    cut_sign = {}
    for k0 in range(0, len(maybe_cut), 2048):
        K = maybe_cut[k0:k0 + 2048]
        X = lo[K][:, None, :] + (tpts[None, :, :] + 1) * (h / 2)
        inside = phi(X) < 0
        fracA[K] = (inside * tw[None, :]).sum(1) / tw.sum()
        for i, k in enumerate(K):
            cut_sign[k] = inside[i]
    hasA = fracA >= frac_min
    hasB = (1 - fracA) >= frac_min
    nspc = hasA.astype(np.int32) + hasB.astype(np.int32)
    cut = (nspc == 2)
    blen = nspc * Np
    spc_off = np.where(hasA, 0, -1), np.where(hasB, np.where(hasA, Np, 0), -1)   # offset of species A, B in block

    # ---- local matrices in dictionaries keyed by (row cell, col cell)
    blocks = {}

    def add(K, L, r0, c0, M):
        key = (int(K), int(L))
        B = blocks.get(key)
        if B is None:
            B = np.zeros((blen[K], blen[L]))
            blocks[key] = B
        B[r0:r0 + M.shape[0], c0:c0 + M.shape[1]] += M

    rhs = np.zeros(int(blen.sum()))
    i0 = np.concatenate([[0], np.cumsum(blen)])
    f = SineModes.seeded(seed, 3) if rhs_f is None else rhs_f

    # ---- uncut cells and faces between uncut cells: closed forms, vectorised; the rest by sub-cell rules
    mu_cell = np.where(hasA & ~cut, mu[0], mu[1])          # the single species' diffusivity of an uncut cell
    sp_cell = np.where(hasA & ~cut, 0, 1)
    S = stiffness_1d(p)
    Kvol = sum(_expand_1d((4.0 / h ** 2 * S)[None], modes, d)[0] for d in range(3))
    diagU = mu_cell[:, None, None] * Kvol[None]
    diagU[cut] = 0.0
    offU = []                                              # (rows, cols, blocks) between uncut cells
    val_q, grad_q = _basis(p, modes, tpts, h)
    GG = np.einsum("qad,qbd->qab", grad_q, grad_q).reshape(len(wvol), Np * Np)
    cut_list = np.nonzero(cut)[0]
    if len(cut_list):
        Wc = np.stack([cut_sign[k] for k in cut_list]) * wvol[None, :]         # [cut cells, q], species A
        VA = (Wc @ GG).reshape(-1, Np, Np)
        VB = ((wvol[None, :] - Wc) @ GG).reshape(-1, Np, Np)
        for i, k in enumerate(cut_list):
            add(k, k, spc_off[0][k], spc_off[0][k], mu[0] * VA[i])
            add(k, k, spc_off[1][k], spc_off[1][k], mu[1] * VB[i])
    # load vector: uncut cells by the cell rule (separable for sine modes), cut cells per species by sub-cells
    from .assembly import project_function
    full = f.project(g, p) if isinstance(f, SineModes) else project_function(g, p, f, q=p + 4)
    unc = np.nonzero(~cut)[0]
    off_u = np.where(hasA[unc], spc_off[0][unc], spc_off[1][unc])
    rhs[(i0[unc] + off_u)[:, None] + np.arange(Np)[None, :]] = full[unc]
    cut_ids = np.nonzero(cut)[0]
    for k0 in range(0, len(cut_ids), 1024):
        K = cut_ids[k0:k0 + 1024]
        X = lo[K][:, None, :] + (tpts[None, :, :] + 1) * (h / 2)
        if isinstance(f, SineModes):
            fv = f.on_tensor_points(lo[K], h, t1d).reshape(len(K), -1)[:, ixyz]
        else:
            fv = f([X[..., 0], X[..., 1], X[..., 2]])
        inside = phi(X) < 0
        for s in (0, 1):
            sel = inside if s == 0 else ~inside
            b = np.einsum("kq,qa->ka", fv * sel * wvol[None, :], val_q)
            has = hasA[K] if s == 0 else hasB[K]
            off = spc_off[s][K]
            idx = (i0[K][has] + off[has])[:, None] + np.arange(Np)[None, :]
            rhs[idx] += b[has]

    # face terms
    tf, wf = gauss(p + 1)
    sf = (np.arange(sub) + 0.5) / sub * 2 - 1
    FP = []
    for a in sf:
        for b in sf:
            for i1, x1 in enumerate(tf):
                for i2, x2 in enumerate(tf):
                    FP.append((a + x1 / sub, b + x2 / sub, wf[i1] * wf[i2] / sub ** 2))
    FP = np.asarray(FP)
    wface = FP[:, 2] * (h / 2) ** 2
    cj = g.length_scale_cj()
    o = lambda a_, b_, w_: np.einsum("q,qa,qb->ab", w_, a_, b_)
    for d in range(3):
        other = [e for e in range(3) if e != d]
        tL = np.zeros((len(FP), 3)); tR = np.zeros((len(FP), 3))
        tL[:, d] = 1.0; tR[:, d] = -1.0
        tL[:, other[0]] = tR[:, other[0]] = FP[:, 0]
        tL[:, other[1]] = tR[:, other[1]] = FP[:, 1]
        vL, gL = _basis(p, modes, tL, h)
        vR, gR = _basis(p, modes, tR, h)
        dL, dR = gL[..., d], gR[..., d]
        stride = int(np.prod(g.shape[:d]))
        TLL = (-0.5 * (o(vL, dL, wface) + o(dL, vL, wface)), o(vL, vL, wface))
        TLR = (-0.5 * o(vL, dR, wface) + 0.5 * o(dL, vR, wface), -o(vL, vR, wface))
        TRR = (0.5 * (o(vR, dR, wface) + o(dR, vR, wface)), o(vR, vR, wface))
        Ls = np.nonzero(mi[d] < g.shape[d] - 1)[0]
        Rs = Ls + stride
        eta = pen * np.maximum(cj[Ls], cj[Rs])
        uu = ~cut[Ls] & ~cut[Rs] & (sp_cell[Ls] == sp_cell[Rs])
        kL, kR, m, e = Ls[uu], Rs[uu], mu_cell[Ls[uu]], eta[uu]
        diagU[kL] += m[:, None, None] * (TLL[0][None] + e[:, None, None] * TLL[1][None])
        diagU[kR] += m[:, None, None] * (TRR[0][None] + e[:, None, None] * TRR[1][None])
        FLR = m[:, None, None] * (TLR[0][None] + e[:, None, None] * TLR[1][None])
        offU.append((kL, kR, FLR))
        offU.append((kR, kL, np.transpose(FLR, (0, 2, 1))))
        # faces that touch a cut cell: all face rules of the direction as one product per species
        kc, lc, ec = Ls[~uu], Rs[~uu], eta[~uu]
        if len(kc):
            q2 = lambda a_, b_: np.einsum("qa,qb->qab", a_, b_).reshape(len(wface), Np * Np)
            Q = np.stack([q2(vL, dL) + q2(dL, vL), q2(vL, vL), q2(vL, dR), q2(dL, vR), q2(vL, vR),
                          q2(vR, dR) + q2(dR, vR), q2(vR, vR)])                     # [7, q, Np^2]
            insF = phi(lo[kc][:, None, :] + (tL[None] + 1) * (h / 2)) < 0           # [faces, q]
            for sp in (0, 1):
                hk = hasA if sp == 0 else hasB
                ok_f = hk[kc] & hk[lc]
                Wf = wface[None, :] * (insF if sp == 0 else ~insF)
                ok_f &= Wf.any(1)
                if not ok_f.any():
                    continue
                T = np.einsum("fq,tqm->tfm", Wf[ok_f], Q).reshape(7, -1, Np, Np)
                m_ = mu[sp]
                et = ec[ok_f][:, None, None]
                FLL = -0.5 * m_ * T[0] + et * m_ * T[1]
                F = -0.5 * m_ * T[2] + 0.5 * m_ * T[3] - et * m_ * T[4]
                FRR = 0.5 * m_ * T[5] + et * m_ * T[6]
                for i, (k, l) in enumerate(zip(kc[ok_f], lc[ok_f])):
                    ok, ol = spc_off[sp][k], spc_off[sp][l]
                    add(k, k, ok, ok, FLL[i])
                    add(l, l, ol, ol, FRR[i])
                    add(k, l, ok, ol, F[i])
                    add(l, k, ol, ok, F[i].T)
        # Dirichlet boundary faces (the sphere never reaches them: uncut cells of the outer species only)
        for side in (-1.0, 1.0):
            Ks = np.nonzero(mi[d] == (0 if side < 0 else g.shape[d] - 1))[0]
            tB = np.zeros((len(FP), 3)); tB[:, d] = side
            tB[:, other[0]] = FP[:, 0]; tB[:, other[1]] = FP[:, 1]
            vB, gB = _basis(p, modes, tB, h)
            dB = gB[..., d]
            T0 = -side * (o(vB, dB, wface) + o(dB, vB, wface))
            T1 = o(vB, vB, wface)
            Ku = Ks[~cut[Ks]]
            m = mu_cell[Ku]
            diagU[Ku] += m[:, None, None] * (T0[None] + (2.0 * pen * cj[Ku])[:, None, None] * T1[None])
            for k in Ks[cut[Ks]]:   # cut boundary cells (coarse grids only)
                ins = phi(lo[k] + (tB + 1) * (h / 2)) < 0
                for sp in (0, 1):
                    ww = wface * (ins if sp == 0 else ~ins)
                    FB = mu[sp] * (-side * (o(vB, dB, ww) + o(dB, vB, ww)) + 2.0 * pen * cj[k] * o(vB, vB, ww))
                    add(k, k, spc_off[sp][k], spc_off[sp][k], FB)

    # interface terms (A inside, normal from A to B)
    Mpts = int(surface_points_per_cell * 4 * math.pi * R * R / (h * h))
    P, nrm, wg = _fibonacci_sphere(Mpts, c, R)
    cell_of = np.clip(np.floor(P / h).astype(np.int64), 0, n - 1)
    cid = cell_of[:, 0] + n * (cell_of[:, 1] + n * cell_of[:, 2])
    muA, muB = mu
    order = np.argsort(cid, kind="stable")
    cells_u, starts = np.unique(cid[order], return_index=True)
    ends = np.append(starts[1:], len(order))
    for k, a0, a1 in zip(cells_u, starts, ends):
        if not cut[k]:
            continue
        sel = order[a0:a1]
        t = (P[sel] - lo[k]) / (h / 2) - 1
        v, gr = _basis(p, modes, t, h)
        dn = np.einsum("qad,qd->qa", gr, nrm[sel])
        w = wg[sel]
        eta = pen * cj[k] * max(muA, muB)
        sig = (1.0, -1.0)
        VD = (v * w[:, None]).T @ dn
        VV = (v * w[:, None]).T @ v
        for s in (0, 1):
            for tt in (0, 1):
                ms, mt = mu[s], mu[tt]
                M = -0.5 * mt * sig[s] * VD - 0.5 * ms * sig[tt] * VD.T + eta * sig[s] * sig[tt] * VV
                add(k, k, spc_off[s][k], spc_off[tt][k], M)

    # ---- block-CSR with uneven blocks: uncut diagonal blocks (plus any sub-cell face terms of their cut
    # neighbours), uncut off-diagonal blocks, and the blocks that involve cut cells
    uncut_ids = np.nonzero(~cut)[0]
    for k in uncut_ids:
        key = (int(k), int(k))
        if key in blocks:
            blocks[key] += diagU[k]
    rows = [uncut_ids[np.array([(int(k), int(k)) not in blocks for k in uncut_ids], dtype=bool)]]
    cols = [rows[0]]
    srcs = [np.zeros(len(rows[0]), np.int64)]            # 0: diagU, 1: offU, 2: dict
    idxs = [rows[0]]
    off_vals = []
    base = 0
    for (kr, kc, V) in offU:
        rows.append(kr); cols.append(kc); srcs.append(np.ones(len(kr), np.int64))
        idxs.append(np.arange(len(kr)) + base)
        off_vals.append(V)
        base += len(kr)
    off_vals = np.concatenate(off_vals) if off_vals else np.zeros((0, Np, Np))
    dkeys = list(blocks.keys())
    rows.append(np.array([k for k, _ in dkeys], np.int64)); cols.append(np.array([l for _, l in dkeys], np.int64))
    srcs.append(np.full(len(dkeys), 2, np.int64)); idxs.append(np.arange(len(dkeys)))
    R_ = np.concatenate(rows); C_ = np.concatenate(cols); S_ = np.concatenate(srcs); I_ = np.concatenate(idxs)
    order = np.lexsort((C_, R_))
    R_, C_, S_, I_ = R_[order], C_[order], S_[order], I_[order]
    row_ptr = np.zeros(nc + 1, np.int64)
    np.add.at(row_ptr, R_ + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    col_idx = C_.astype(np.int32)
    bsz = blen[R_].astype(np.int64) * blen[C_]
    voff = np.concatenate([[0], np.cumsum(bsz)])
    values = np.empty(int(voff[-1]))
    ar = np.arange(Np * Np)
    for src, arr in ((0, diagU), (1, off_vals)):
        sel = np.nonzero(S_ == src)[0]
        if len(sel):
            values[voff[sel][:, None] + ar[None, :]] = arr[I_[sel]].reshape(len(sel), Np * Np)
    for j in np.nonzero(S_ == 2)[0]:
        values[voff[j]:voff[j + 1]] = blocks[dkeys[I_[j]]].ravel()
    species = np.stack([hasA, hasB], -1)
    return XdgSystem(Np=Np, nspc=nspc, species=species, row_ptr=row_ptr, col_idx=col_idx, values=values, rhs=rhs,
                     grid=g, p=p, centre=c, radius=R, mu=tuple(mu))


BATCH_EDGES = (16, 24, 32, 40, 48)
BATCH_JUMPS = (10.0, 100.0, 1000.0)


def batch_specs(count: int = 256, seed: int = 0, p: int = 2) -> list:
    """Seeded parameters of a batch of independent sphere problems: grid edge uniform in BATCH_EDGES, radius
    uniform in [0.15, 0.35], centre uniform in [0.4, 0.6]^3, diffusivity jump 1:J with J uniform in BATCH_JUMPS,
    and a per-problem seed of the right-hand side.  Each dict holds the keyword arguments of ``xdg_sphere``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(BATCH_EDGES))
        R = float(rng.uniform(0.15, 0.35))
        c = tuple(float(v) for v in rng.uniform(0.4, 0.6, size=3))
        J = float(rng.choice(BATCH_JUMPS))
        out.append(dict(n=n, p=p, seed=int(seed * 100003 + i), mu=(1.0, J), radius=R, centre=c))
    return out
