"""The oracle and the engine against committed golden fixtures made by the
reference smf (tests/golden/make_golden.py), and the reference's own
known-answer cases of the dense front kernel (solver/tests/test_ldlt_dense.cpp,
solver/tests/test_ldlt_aptp.cpp), so that parity is pinned without the
reference library at hand.
"""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
FILES = [f for f in FILES if not os.path.basename(f).endswith(("_smf_partition.npz", "_digest.npz"))]
FIELDS = ["perm", "sn_start", "sn_end", "sn_parent", "child_ptr", "child_idx", "front_row_ptr",
          "front_row_idx", "postorder", "perm_col_ptr", "perm_row_idx", "clean_to_perm",
          "orig_to_clean", "clean_col_ptr", "clean_row_idx"]


def _load(path):
    from oracle import oracle as O
    z = np.load(path)
    a = O.Analysis(n=int(z["n"]), matching_scale=np.zeros(0), **{k: z["an_" + k] for k in FIELDS})
    return z, a


def _check_blocks(z, a, f, p, block, rows_of, tags):
    assert np.array_equal(f, z["f"]) and np.array_equal(p, z["p"])
    for s in range(a.nsn):
        o, ff, pp = int(z["blk_off"][s]), int(z["f"][s]), int(z["p"][s])
        want = z["blocks"][o:o + ff * pp].reshape(pp, ff).T
        assert np.array_equal(block(s), want), s
        ro = int(z["row_off"][s])
        assert np.array_equal(rows_of(s), z["rows"][ro:ro + ff]), s
    if z["tags"].size:
        assert np.array_equal(tags[:z["tags"].size], z["tags"])


@pytest.mark.parametrize("path", FILES, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_golden(path, oracle_lib):
    O = oracle_lib
    z, a = _load(path)
    posdef = bool(z["posdef"])
    scale = z["scale"] if z["scale"].size else None
    ox = O.restated_factorize(a, O.permuted_values(a, z["values"], scale), posdef)
    assert ox.delayed == int(z["delayed"]) and ox.two_by_two == int(z["two_by_two"])
    assert ox.flops == float(z["flops"])
    if tuple(z["inertia"]) != (0, 0, 0):
        assert ox.inertia == tuple(int(x) for x in z["inertia"])
    _check_blocks(z, a, ox.f[:a.nsn], ox.p[:a.nsn], ox.block, ox.front_rows,
                  ox.tags if ox.tags is not None else np.zeros(0, np.int8))
    x = O.restated_solve(a, ox, posdef, z["b"], scale)
    assert np.max(np.abs(x - z["x"])) <= 1e-10 * max(1.0, np.max(np.abs(z["x"])))


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=lambda p: os.path.basename(p)[:-4])
def test_engine_matches_golden(path):
    from opt_solver_b200 import smfg
    z, a = _load(path)
    posdef = bool(z["posdef"])
    scale = z["scale"] if z["scale"].size else None
    sv = smfg.Solver(a, device=0)
    gi = sv.factor(z["values"], posdef=posdef, scale=scale)
    assert gi.delayed_pivots == int(z["delayed"]) and gi.two_by_two_pivots == int(z["two_by_two"])
    assert gi.flops == float(z["flops"])
    if tuple(z["inertia"]) != (0, 0, 0):
        assert gi.inertia == tuple(int(x) for x in z["inertia"])
    gx = sv.export()
    _check_blocks(z, a, gx.f, gx.p, gx.block, gx.front_rows,
                  gx.tags if gx.tags is not None else np.zeros(0, np.int8))
    x = sv.solve(z["b"])
    assert np.max(np.abs(x - z["x"])) <= 1e-10 * max(1.0, np.max(np.abs(z["x"])))
    sv.close()


# -- the reference's known answers of the dense front kernel ----------------

def _weak_front(d00, a21):
    """solver/tests/test_ldlt_dense.cpp:211-227's front."""
    A = np.zeros((4, 4))
    A[0, 0], A[1, 0], A[2, 0], A[3, 0] = d00, 1.0, 0.1, 0.05
    A[1, 1], A[2, 1], A[3, 1] = 1e-3, a21, 0.1
    A[2, 2], A[3, 2] = 4.0, 0.3
    A[3, 3] = -5.0
    return A + np.tril(A, -1).T


def test_kat_small_dense(oracle_lib):
    O = oracle_lib
    # LDLT.SPD2x2 / AllNegative2x2 / Indefinite3x3 (test_ldlt_dense.cpp:18-48)
    assert O.factor_front([[4, 2], [2, 3]], 2)[3][:3] == (2, 0, 0)
    assert O.factor_front([[-4, -2], [-2, -3]], 2)[3][:3] == (0, 2, 0)
    pos, neg, zero, acc = O.factor_front([[2, 1, 0], [1, 0, 1], [0, 1, 2]], 3)[3]
    assert pos + neg + zero == 3 and pos >= 1 and acc == 3


def test_kat_weak_one_by_one():
    """LdltDense.WeakOneByOneGivesWayToStableTwoByTwo (test_ldlt_dense.cpp:232-263)."""
    from oracle import oracle as O
    assert tuple(O.factor_front(_weak_front(5e-8, 0.2), 4, u=1e-8)[2][:2]) == (2, -1)
    assert O.factor_front(_weak_front(5e-8, 3e7), 4, u=1e-8)[2][0] == 1
    for u in (0.01, 1e-8):
        assert O.factor_front(_weak_front(0.05, 0.2), 4, u=u)[2][0] == 1
    assert tuple(O.factor_front(_weak_front(5e-8, 0.2), 4, u=0.01)[2][:2]) == (2, -1)


def test_kat_stalled_panels_pull_in_partners(oracle_lib):
    """LdltDense.StalledPanelsPullInPartners (test_ldlt_dense.cpp:274-347):
    constraint columns coupled only past their panel stall, pull their
    partners in and pivot as 2x2; every eligible column is accepted and the
    Schur complement of the remaining rows is the dense one."""
    O = oracle_lib
    m, nv, q, kfar = 40, 120, 40, 100
    e, f = m + nv, m + nv + q
    rng = np.random.default_rng(20261102)
    A = np.zeros((f, f))
    for c in range(m):
        for t in range(3):
            A[kfar + (c * 3 + t) % (e - kfar), c] += 1.0 + 0.5 * rng.uniform(-1, 1)
    for j in range(m, e):
        A[j, j] = 4.0 + rng.uniform(-1, 1)
        for i in range(j + 1, f):
            if rng.integers(8) == 0:
                A[i, j] = 0.3 * rng.uniform(-1, 1)
    for j in range(e, f):
        for i in range(j, f):
            A[i, j] = 2.0 if i == j else 0.1 * rng.uniform(-1, 1)
    Afull = np.tril(A) + np.tril(A, -1).T
    F, rows, tags, (pos, neg, zero, acc) = O.factor_front(Afull, e, u=0.01)
    assert acc == e and (pos, neg, zero) == (nv, m, 0)
    assert tags[0] == 2 and rows[0] == 0 and rows[1] >= kfar
    assert np.array_equal(rows[e:], np.arange(e, f))
    # Schur complement: A22 - A21 A11^-1 A12 in the original row order
    S = Afull[e:, e:] - Afull[e:, :e] @ np.linalg.solve(Afull[:e, :e], Afull[:e, e:])
    got = np.tril(F[e:, e:])
    assert np.max(np.abs(got - np.tril(S))) < 1e-10


def test_kat_saddle_point_two_by_two(oracle_lib):
    """LdltAptp.SaddlePointUsesTwoByTwo's matrix (test_ldlt_aptp.cpp:307-325)
    through the threshold kernel: all 2x2 pivots, inertia (50, 50, 0)."""
    O = oracle_lib
    nb = 50
    rng = np.random.default_rng(3)
    B = 4.0 * np.eye(nb) + rng.uniform(-0.5, 0.5, (nb, nb)) / nb
    A = np.zeros((2 * nb, 2 * nb))
    A[nb:, :nb] = B
    A[:nb, nb:] = B.T
    F, rows, tags, (pos, neg, zero, acc) = O.factor_front(A, 2 * nb)
    assert (pos, neg, zero, acc) == (nb, nb, 0, 2 * nb)
    assert np.all(tags[0::2] == 2) and np.all(tags[1::2] == -1)
