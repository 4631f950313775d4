"""smf's analysis output (the AnalysisKeep arrays the numeric phase reads,
solver/include/smf/analysis.hpp:25-144) rebuilt from a compact record of it:
the fill-reducing permutation and the supernode partition (first column and
parent of each supernode, numbered in postorder). Everything else that
AnalysisKeep holds for the numeric phase follows from those and the matrix:

  - the permuted lower pattern (perm_col_ptr / perm_row_idx): entry (i, j)
    of the input goes to (max, min) of its new indices, rows ascending in
    each column;
  - each front's rows (front_row_ptr / front_row_idx): the supernode's own
    columns, the rows of its original entries, and its children's
    contribution rows, ascending -- the multifrontal structure smf's
    symbolic analysis produces (symbolic_analysis.cpp), checked equal to the
    reference's own arrays by tests/test_smf_analysis.py;
  - children in descending postorder (the order smf's contribution stack
    pops them);
  - the value maps: an input without duplicates or entries above the
    diagonal is its own cleaned matrix, and every cleaned entry's permuted
    slot is found from its position in the permuted pattern.

The record of a workload is made by the reference itself
(tests/golden/make_smf_partitions.py) and loaded with `load`.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class SmfAnalysis:
    n: int
    perm: np.ndarray
    sn_start: np.ndarray
    sn_end: np.ndarray
    sn_parent: np.ndarray
    child_ptr: np.ndarray
    child_idx: np.ndarray
    front_row_ptr: np.ndarray
    front_row_idx: np.ndarray
    postorder: np.ndarray
    perm_col_ptr: np.ndarray
    perm_row_idx: np.ndarray
    clean_to_perm: np.ndarray
    orig_to_clean: np.ndarray
    clean_col_ptr: np.ndarray
    clean_row_idx: np.ndarray

    @property
    def nsn(self) -> int:
        return int(self.sn_start.size)


def from_partition(n, col_ptr, row_idx, perm, sn_first, sn_parent) -> SmfAnalysis:
    """The analysis arrays of the lower CSC (col_ptr, row_idx) under the
    ordering perm (perm[new] = old) and the supernode partition sn_first
    (nsn + 1 column boundaries, supernodes in postorder) with parents
    sn_parent (-1 at roots). The input must hold no duplicate entries and
    nothing above the diagonal."""
    col_ptr = np.asarray(col_ptr, dtype=np.int64)
    row_idx = np.asarray(row_idx, dtype=np.int64)
    perm = np.asarray(perm, dtype=np.int64)
    sn_first = np.asarray(sn_first, dtype=np.int64)
    parent = np.asarray(sn_parent, dtype=np.int64)
    nnz = int(col_ptr[-1])
    cols = np.repeat(np.arange(n), np.diff(col_ptr))
    if np.any(row_idx < cols):
        raise ValueError("entries above the diagonal: not a cleaned lower CSC")
    iperm = np.empty(n, dtype=np.int64)
    iperm[perm] = np.arange(n)
    a, b = iperm[row_idx], iperm[cols]
    pc, pr = np.minimum(a, b), np.maximum(a, b)
    order = np.lexsort((pr, pc))  # by column, then row
    key = pc[order] * n + pr[order]
    if np.any(np.diff(key) == 0):
        raise ValueError("duplicate entries: not a cleaned lower CSC")
    perm_col_ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(perm_col_ptr, pc + 1, 1)
    perm_col_ptr = np.cumsum(perm_col_ptr)
    perm_row_idx = pr[order]
    clean_to_perm = np.empty(nnz, dtype=np.int64)
    clean_to_perm[order] = np.arange(nnz)
    ns = sn_first.size - 1
    sn_start, sn_end = sn_first[:-1], sn_first[1:]
    # children in descending postorder (numbering = postorder)
    child_ptr = np.zeros(ns + 1, dtype=np.int64)
    has = parent >= 0
    np.add.at(child_ptr, parent[has] + 1, 1)
    child_ptr = np.cumsum(child_ptr)
    kids = np.nonzero(has)[0]
    kids = kids[np.lexsort((-kids, parent[kids]))]
    child_idx = kids
    # front rows, children first (postorder)
    rows = [None] * ns
    ptr = np.zeros(ns + 1, dtype=np.int64)
    for s in range(ns):
        c0, c1 = sn_start[s], sn_end[s]
        parts = [np.arange(c0, c1), perm_row_idx[perm_col_ptr[c0]:perm_col_ptr[c1]]]
        for t in range(child_ptr[s], child_ptr[s + 1]):
            c = child_idx[t]
            parts.append(rows[c][sn_end[c] - sn_start[c]:])
        rows[s] = np.unique(np.concatenate(parts))
        ptr[s + 1] = ptr[s] + rows[s].size
    i32 = lambda x: np.ascontiguousarray(x, dtype=np.int32)
    return SmfAnalysis(
        n=int(n), perm=i32(perm), sn_start=i32(sn_start), sn_end=i32(sn_end), sn_parent=i32(parent),
        child_ptr=i32(child_ptr), child_idx=i32(child_idx), front_row_ptr=i32(ptr),
        front_row_idx=i32(np.concatenate(rows)), postorder=i32(np.arange(ns)),
        perm_col_ptr=i32(perm_col_ptr), perm_row_idx=i32(perm_row_idx), clean_to_perm=i32(clean_to_perm),
        orig_to_clean=i32(np.arange(nnz)), clean_col_ptr=i32(col_ptr), clean_row_idx=i32(row_idx))


def load(path: str, n, col_ptr, row_idx) -> SmfAnalysis:
    """The analysis of a workload from its record (an .npz with perm,
    sn_first, sn_parent)."""
    z = np.load(path)
    return from_partition(n, col_ptr, row_idx, z["perm"], z["sn_first"], z["sn_parent"])


GOLDEN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")
