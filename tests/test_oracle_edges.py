"""Edge cases of the numeric phase, oracle against the reference (CPU): one-
row systems (positive, negative, zero), zero diagonals that need 2x2
pivots, rank-deficient KKTs and explicit zero columns (zero pivots in the
inertia), a forest of independent blocks, and input with duplicate entries
and entries given above the diagonal (duplicates summed, upper entries
discarded: solver/include/smf/check_matrix.hpp:19,
solver/src/workspace.cpp:129-281). Bit for bit as in test_oracle.py."""
import numpy as np
import pytest

from tests.cases import dense_lower, reference_for
from tests.test_oracle import _bitwise_same
from opt_solver_b200 import workloads as W


def _coo_lower(n, rows, cols, vals):
    """Lower CSC with duplicates and upper entries kept as given (the
    analysis cleans them)."""
    rows, cols, vals = (np.asarray(x) for x in (rows, cols, vals))
    order = np.lexsort((rows, cols))
    rows, cols, vals = rows[order], cols[order], vals[order]
    cp = np.zeros(n + 1, dtype=np.int32)
    np.add.at(cp, cols + 1, 1)
    return n, np.cumsum(cp).astype(np.int32), rows.astype(np.int32), vals.astype(np.float64)


def _rank_deficient_kkt():
    # [H A^T; A 0] with A's last row a copy of its first: one zero pivot
    rng = np.random.default_rng(5)
    m, k = 12, 5
    M = rng.standard_normal((m, m))
    H = M @ M.T + m * np.eye(m)
    A = rng.standard_normal((k, m))
    A[-1] = A[0]
    K = np.zeros((m + k, m + k))
    K[:m, :m] = H
    K[m:, :m] = A
    K[:m, m:] = A.T
    return dense_lower(K)


def _zero_column():
    # a symmetric matrix whose column 3 is structurally present but all zero
    rng = np.random.default_rng(6)
    n = 9
    M = rng.standard_normal((n, n))
    K = M + M.T + 2 * n * np.eye(n)
    K[3, :] = 0.0
    K[:, 3] = 0.0
    return dense_lower(K)


def _forest():
    # two independent Laplacians side by side: two roots in the tree
    n1, cp1, ri1, v1 = W.laplacian_2d(6)
    n2, cp2, ri2, v2 = W.laplacian_2d(5, 7)
    cp = np.concatenate([cp1, cp2[1:] + cp1[-1]]).astype(np.int32)
    ri = np.concatenate([ri1, ri2 + n1]).astype(np.int32)
    return n1 + n2, cp, ri, np.concatenate([v1, v2])


def _duplicates_and_upper():
    # a 2D Laplacian with some entries split in two and some off-diagonal
    # entries given at (col, row) instead of (row, col): the reference
    # discards the latter, so the matrix factored loses those couplings
    n, cp, ri, v = W.laplacian_2d(7)
    cols = np.repeat(np.arange(n), np.diff(cp))
    rows = ri.astype(np.int64)
    rng = np.random.default_rng(8)
    split = rng.random(v.size) < 0.3
    r2, c2 = rows[split], cols[split]
    v2 = 0.25 * v[split]
    vals = v.copy()
    vals[split] -= v2
    flip = (rng.random(v.size) < 0.3) & (rows != cols)
    rows_f = np.where(flip, cols, rows)
    cols_f = np.where(flip, rows, cols)
    return _coo_lower(n, np.concatenate([rows_f, r2]), np.concatenate([cols_f, c2]),
                      np.concatenate([vals, v2]))


EDGES = [
    ("one_pos", lambda: dense_lower([[3.0]]), False, (1, 0, 0)),
    ("one_neg", lambda: dense_lower([[-2.0]]), False, (0, 1, 0)),
    ("one_zero", lambda: dense_lower([[0.0]]), False, (0, 0, 1)),
    ("one_spd", lambda: dense_lower([[2.0]]), True, (1, 0, 0)),
    ("diag_mixed", lambda: dense_lower(np.diag([4.0, -1.0, 2.0, -3.0, 0.5])), False, (3, 2, 0)),
    ("swap_2x2", lambda: dense_lower([[0.0, 1.0], [1.0, 0.0]]), False, (1, 1, 0)),
    ("zero_diag_3x3", lambda: dense_lower([[0, 2, 0], [2, 0, 1], [0, 1, 0]]), False, None),
    ("rank_deficient_kkt", _rank_deficient_kkt, False, (12, 4, 1)),
    ("zero_column", _zero_column, False, None),
    ("forest_spd", _forest, True, (71, 0, 0)),
    ("forest_indef", _forest, False, (71, 0, 0)),
    ("duplicates_and_upper", _duplicates_and_upper, True, (49, 0, 0)),
]


@pytest.mark.parametrize("case", EDGES, ids=lambda c: c[0])
def test_edge_case_bitwise_vs_reference(case, ref_lib, oracle_lib):
    O = ref_lib
    name, build, posdef, expect = case
    n, cp, ri, v = build()
    ref = reference_for(O, posdef, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    ox = O.restated_factorize(a, O.permuted_values(a, v), posdef)
    _bitwise_same(a, fx, ox)  # inertia too, where the reference reports it (not SPD)
    if expect is not None:
        assert ox.inertia == expect
    if ox.inertia[2] == 0:
        # the residual of the matrix as the reference reads it: the entries
        # on and below the diagonal
        cols = np.repeat(np.arange(n), np.diff(cp))
        low = ri >= cols
        lcp = np.concatenate([[0], np.cumsum(np.bincount(cols[low], minlength=n))]).astype(np.int32)
        b = np.random.default_rng(2).uniform(-1, 1, n)
        x = O.restated_solve(a, ox, posdef, b)
        _, eta, om = O.residual(n, lcp, ri[low], v[low], b, x)
        assert eta <= 1e-10 and om <= 1e-12
