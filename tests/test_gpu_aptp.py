"""The CUDA APTP front kernel against the oracle and the reference, bit for
bit.

The kernel factors every indefinite front of at least 512 rows in the
reference's deterministic mode (solver/src/ldlt_aptp.cpp:739), the threshold
kernel then taking the columns it fails (multifrontal_serial.cpp:796-821).
Alone on dense fronts through the C ABI (smfg_aptp_front_dense) it must
reproduce the oracle's restatement, itself pinned to the reference
(tests/test_oracle_aptp.py): the lower triangle of the factored front (L, D
and the failed columns' Schur complement), the row order, the pivot tags and
the counts, on fronts with many 2x2 pivots, failed columns inside and
outside the tiles, tall trailing blocks and more than one block column. In
whole factorizations (KKT systems whose top fronts take APTP) the engine must
reproduce the reference's deterministic-mode factor front by front.
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


@pytest.mark.parametrize("grid,m,seed", [(10, 700, 6), (12, 1200, 1), (14, 2000, 2)])
def test_aptp_factor_bitwise_vs_deterministic_reference(grid, m, seed, ref_lib):
    """Whole KKT factorizations on the reference's own analysis and scaling:
    every front's realized size, rows, tags and L / D block, the inertia,
    delays, 2x2 pivots, flops and the APTP failed-column count."""
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    from tests.cases import reference_for
    from tests.test_gpu_parity import _compare_factor
    O = ref_lib
    n, cp, ri, v = W.kkt_ipm(grid, m, seed=seed)
    ref = reference_for(O, False, "auto", "auto", deterministic=True)
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    assert fx.aptp_failed > 0
    sv = smfg.Solver(a, device=0)
    gi = sv.factor(v, posdef=False, scale=fx.scale)
    assert gi.aptp_fronts == int(np.sum(fx.f >= 512))
    assert gi.aptp_failed == fx.aptp_failed
    _compare_factor(a, fx, sv.export(), gi)
    assert gi.inertia == (grid ** 3, m, 0)
    b = W.rhs(n, 1, seed=3)
    x = sv.solve(b)
    xr, _ = ref.solve(b)
    assert np.max(np.abs(x - xr)) <= 1e-9 * max(1.0, np.max(np.abs(xr)))
    sv.close()


def test_aptp_factor_matches_golden():
    """The reference's digests of its deterministic-mode factor (no reference
    library needed)."""
    import os
    from oracle import oracle as O
    from opt_solver_b200 import smfg
    from tests.test_golden import FIELDS
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "kkt_10_700_digest.npz"))
    a = O.Analysis(n=int(z["n"]), matching_scale=np.zeros(0), **{k: z["an_" + k] for k in FIELDS})
    sv = smfg.Solver(a, device=0)
    gi = sv.factor(z["values"], posdef=False, scale=z["scale"])
    gx = sv.export()
    assert gi.inertia == tuple(int(x) for x in z["inertia"])
    assert (gi.delayed_pivots, gi.two_by_two_pivots, gi.flops) == (int(z["delayed"]), int(z["two_by_two"]),
                                                                    float(z["flops"]))
    assert gi.aptp_failed == int(z["aptp_failed"])
    for s in range(a.nsn):
        assert block_digest(gx.block(s)) == str(z["block_sha256"][s]), s
    sv.close()


def test_threshold_kernel_everywhere_is_the_default_mode(ref_lib):
    """aptp_min_rows = 0: the threshold kernel on every front, bit for bit the
    reference's one-thread default mode."""
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    from tests.cases import reference_for
    from tests.test_gpu_parity import _compare_factor
    O = ref_lib
    n, cp, ri, v = W.kkt_ipm(10, 700, seed=6)
    ref = reference_for(O, False, "auto1t", "auto")
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    assert fx.aptp_failed == 0
    sv = smfg.Solver(a, device=0)
    gi = sv.factor(v, posdef=False, scale=fx.scale, aptp_min_rows=0)
    assert gi.aptp_fronts == 0
    _compare_factor(a, fx, sv.export(), gi)
    sv.close()
