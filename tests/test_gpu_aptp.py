"""The CUDA APTP front kernel against the oracle, bit for bit.

The kernel factors every indefinite front of at least 512 rows in the
reference's deterministic mode (solver/src/ldlt_aptp.cpp:739). Here it runs
alone on dense fronts through the C ABI (smfg_aptp_front_dense) and must
reproduce the oracle's restatement, itself pinned to the reference
(tests/test_oracle_aptp.py): the lower triangle of the factored front (L, D
and the failed columns' Schur complement), the row order, the pivot tags and
the counts, on fronts with many 2x2 pivots, failed columns inside and
outside the tiles, tall trailing blocks and more than one block column.
"""
import numpy as np
import pytest

from tests.golden.make_golden import block_digest, dense_aptp_fronts
from tests.test_oracle_aptp import _oracle_dense

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(11)
    out = list(dense_aptp_fronts())
    A = rng.standard_normal((300, 300))
    out.append(("gauss_300_one_block", A + A.T, 200, 0.01))
    A = rng.standard_normal((900, 900))
    out.append(("gauss_900_300", A + A.T, 300, 0.01))
    A = rng.standard_normal((1100, 1100))
    A = A @ A.T / 1100
    A[np.diag_indices(1100)] *= -1
    out.append(("mixed_sign_1100", A, 1050, 0.01))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_aptp_dense_bitwise_vs_oracle(case, oracle_lib):
    from opt_solver_b200 import smfg
    O = oracle_lib
    name, A, ne, u = case
    F, rows, tags, res = smfg.aptp_front_dense(A, ne, u=u, small=1e-20)
    Fo, rows_o, tags_o, res_o = _oracle_dense(O, A, ne, u)
    assert res == tuple(int(x) for x in res_o)
    assert np.array_equal(rows, rows_o)
    assert np.array_equal(tags, tags_o)
    low = np.tril(np.ones(F.shape, dtype=bool))
    diff = (F != Fo) & low & ~(np.isnan(F) & np.isnan(Fo))
    assert not diff.any(), (int(diff.sum()), np.argwhere(diff)[:5])


def test_aptp_dense_matches_golden():
    """The reference's own digests of its APTP factor of the same fronts."""
    import os
    from opt_solver_b200 import smfg
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "aptp_dense_digest.npz"))
    for name, A, ne, u in dense_aptp_fronts():
        F, rows, tags, res = smfg.aptp_front_dense(A, ne, u=u, small=1e-20)
        assert np.array_equal(np.asarray(res), z[f"{name}_result"]), name
        assert np.array_equal(rows, z[f"{name}_rows"]) and np.array_equal(tags, z[f"{name}_tags"]), name
        assert block_digest(np.tril(F)) == str(z[f"{name}_sha256"]), name
