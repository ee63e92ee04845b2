"""CPU test of the multi-cell Schwarz blocks the library builds on the host (bsgpu_schwarz_blocks: no device work)
against the oracle's restatement (or_schwarz_blocks) and against the rules themselves: the partition covers every
cell once, blocks are connected in the block graph and at most ceil(nb / parts) cells, the overlap growth adds
exactly the face-neighbour layers (Schwarz.cs:690-735)."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200 import xdg


def _lib_blocks(s, parts, overlap):
    rp = np.ascontiguousarray(s.row_ptr, np.int64)
    ci = np.ascontiguousarray(s.col_idx, np.int32)
    nb, tot = C.c_int64(), C.c_int64()
    f = nat.lib().bsgpu_schwarz_blocks
    nat.check(f(len(rp) - 1, nat.ptr(rp), nat.ptr(ci), int(parts), int(overlap), None, None, C.byref(nb),
                C.byref(tot)))
    ptr = np.zeros(nb.value + 1, np.int64)
    cells = np.zeros(max(tot.value, 1), np.int32)
    nat.check(f(len(rp) - 1, nat.ptr(rp), nat.ptr(ci), int(parts), int(overlap), nat.ptr(ptr), nat.ptr(cells), None,
                None))
    return ptr, cells[:tot.value]


SYSTEMS = {"poisson_5x4x3": lambda: A.assemble_sip(A.RectilinearGrid(nodes=[np.linspace(0, 1, n + 1)
                                                                            for n in (5, 4, 3)]), 1),
           "xdg_sphere_6": lambda: xdg.xdg_sphere(n=6, p=1, seed=2, mu=(1.0, 10.0))}


@pytest.mark.parametrize("name", sorted(SYSTEMS))
@pytest.mark.parametrize("parts,overlap", [(0, 0), (0, 1), (7, 1), (3, 2), (1, 0), (1000, 1)])
def test_blocks_match_oracle(name, parts, overlap):
    s = SYSTEMS[name]()
    ptr, cells = _lib_blocks(s, parts, overlap)
    optr, ocells = O.schwarz_blocks(O.Bsr.of(s), parts, overlap)
    assert np.array_equal(ptr, optr) and np.array_equal(cells, ocells)


def test_partition_rules():
    s = SYSTEMS["poisson_5x4x3"]()
    nb = len(s.row_ptr) - 1
    parts = 7
    ptr, cells = _lib_blocks(s, parts, 0)
    blocks = [cells[ptr[b]:ptr[b + 1]] for b in range(len(ptr) - 1)]
    assert np.array_equal(np.sort(cells), np.arange(nb))           # every cell exactly once
    target = -(-nb // parts)
    nbr = [set(s.col_idx[s.row_ptr[c]:s.row_ptr[c + 1]]) - {c} for c in range(nb)]
    for bl in blocks:
        assert 1 <= len(bl) <= target and np.all(np.diff(bl) > 0)
        seen, todo = {bl[0]}, [bl[0]]                              # connected in the block graph
        while todo:
            c = todo.pop()
            for j in nbr[c] & set(bl.tolist()):
                if j not in seen:
                    seen.add(j)
                    todo.append(j)
        assert seen == set(bl.tolist())
    # one overlap layer: each block grows by exactly its face neighbours outside it
    ptr1, cells1 = _lib_blocks(s, parts, 1)
    for b, bl in enumerate(blocks):
        grown = set(cells1[ptr1[b]:ptr1[b + 1]].tolist())
        layer = set().union(*(nbr[c] for c in bl)) | set(bl.tolist())
        assert grown == layer


def test_rejects_bad_overlap_and_indices():
    s = SYSTEMS["poisson_5x4x3"]()
    with pytest.raises(nat.BsgpuError):
        _lib_blocks(s, 0, 3)

    class Bad:
        row_ptr = np.array([0, 1], np.int64)
        col_idx = np.array([5], np.int32)
    with pytest.raises(nat.BsgpuError):
        _lib_blocks(Bad, 0, 0)
