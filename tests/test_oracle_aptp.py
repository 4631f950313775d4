"""The oracle's APTP kernel pinned against the reference (CPU).

Deterministic mode, the parity mode of the reference, factors every
indefinite front of at least 512 rows with a posteriori threshold pivoting
(solver/src/ldlt_aptp.cpp, as 2D tile tasks: parallel/tile_tasks.cpp:256;
dispatch multifrontal_serial.cpp:796-821, parallel/thread_plan.hpp:43-47),
then the threshold kernel on the columns it failed. The restatement in
oracle/mf_oracle.c must reproduce it bit for bit: the dense kernel alone on
fronts with many 2x2 pivots and failed columns, and whole factorizations of
KKT systems with such fronts. The committed digests pin both without the
reference library.
"""
import ctypes as C

import numpy as np
import pytest

from tests.cases import reference_for
from tests.golden.make_golden import block_digest, dense_aptp_fronts


def _oracle_dense(O, A, ne, u):
    f = A.shape[0]
    F = np.ascontiguousarray(np.tril(A).T).reshape(-1).copy()
    rows = np.arange(f, dtype=np.int32)
    tags = np.zeros(f, dtype=np.int8)
    out = np.zeros(5, dtype=np.int64)
    prm = O._MfoParams(u, 1e-20, 1e-20, 16, 96, 0, 0, 0, O.APTP_MIN_ROWS, O.APTP_NB, O.APTP_IB)
    O._oracle_lib().mfo_aptp_front(F.ctypes.data_as(C.c_void_p), f, ne, rows.ctypes.data_as(C.c_void_p),
                                   C.byref(prm), tags.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
    return F.reshape(f, f).T, rows, tags, out


def _random_fronts():
    rng = np.random.default_rng(7)
    out = list(dense_aptp_fronts())
    A = rng.standard_normal((900, 900))
    out.append(("gauss_900_300", A + A.T, 300, 0.01))      # a tall trailing block
    A = rng.standard_normal((700, 700))
    A = A @ A.T / 700
    A[np.diag_indices(700)] *= -1
    out.append(("mixed_sign_700", A, 650, 0.01))
    return out


@pytest.mark.parametrize("case", _random_fronts(), ids=lambda c: c[0])
def test_dense_aptp_bitwise_vs_reference(case, ref_lib, oracle_lib):
    from tests.golden.make_golden import dense_aptp_reference
    O = ref_lib
    name, A, ne, u = case
    F, rows, tags, res = _oracle_dense(O, A, ne, u)
    Fr, rows_r, tags_r, res_r = dense_aptp_reference(A, ne, u)
    assert np.array_equal(res, res_r)
    assert np.array_equal(rows, rows_r) and np.array_equal(tags, tags_r)
    assert np.array_equal(np.tril(F), np.tril(Fr))
    assert np.sum(tags == 2) > 0


def test_dense_aptp_matches_golden(oracle_lib):
    import os
    O = oracle_lib
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "aptp_dense_digest.npz"))
    for name, A, ne, u in dense_aptp_fronts():
        F, rows, tags, res = _oracle_dense(O, A, ne, u)
        assert np.array_equal(res, z[f"{name}_result"]), name
        assert np.array_equal(rows, z[f"{name}_rows"]) and np.array_equal(tags, z[f"{name}_tags"]), name
        assert block_digest(np.tril(F)) == str(z[f"{name}_sha256"]), name


def _factor_same(a, fx, ox):
    assert ox.status in (0, 2)
    assert (ox.delayed, ox.two_by_two, ox.flops, ox.inertia) == (fx.delayed, fx.two_by_two, fx.flops, fx.inertia)
    assert ox.aptp_failed == fx.aptp_failed > 0
    for s in range(a.nsn):
        assert ox.f[s] == fx.f[s] and ox.p[s] == fx.p[s], s
        assert np.array_equal(ox.front_rows(s), fx.front_rows(s)), s
        assert np.array_equal(ox.block(s), fx.block(s)), s
    n_t = int(np.sum(fx.p))
    assert np.array_equal(ox.tags[:n_t], fx.tags[:n_t])


@pytest.mark.parametrize("grid,m,seed", [(10, 700, 6), (12, 1200, 1)])
def test_aptp_factor_bitwise_vs_deterministic_reference(grid, m, seed, ref_lib, oracle_lib):
    from opt_solver_b200 import workloads as W
    O = ref_lib
    n, cp, ri, v = W.kkt_ipm(grid, m, seed=seed)
    ref = reference_for(O, False, "auto", "auto", deterministic=True)
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    assert np.any(fx.f >= O.APTP_MIN_ROWS)
    ox = O.restated_factorize(a, O.permuted_values(a, v, fx.scale), False)
    _factor_same(a, fx, ox)
    # the one-thread default mode (no APTP) is a different factor
    tx = O.restated_factorize(a, O.permuted_values(a, v, fx.scale), False, aptp_min_rows=0)
    assert tx.aptp_failed == 0
    assert any(not np.array_equal(tx.block(s), fx.block(s)) for s in range(a.nsn) if fx.f[s] >= 512)


def test_aptp_factor_matches_golden(oracle_lib):
    import os
    from tests.test_golden import FIELDS
    O = oracle_lib
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "kkt_10_700_digest.npz"))
    a = O.Analysis(n=int(z["n"]), matching_scale=np.zeros(0), **{k: z["an_" + k] for k in FIELDS})
    ox = O.restated_factorize(a, O.permuted_values(a, z["values"], z["scale"]), False)
    assert (ox.delayed, ox.two_by_two, ox.flops) == (int(z["delayed"]), int(z["two_by_two"]), float(z["flops"]))
    assert ox.inertia == tuple(int(x) for x in z["inertia"])
    assert ox.aptp_failed == int(z["aptp_failed"])
    assert np.array_equal(ox.f[:a.nsn], z["f"]) and np.array_equal(ox.p[:a.nsn], z["p"])
    for s in range(a.nsn):
        assert block_digest(ox.block(s)) == str(z["block_sha256"][s]), s
        ro = int(z["row_off"][s])
        assert np.array_equal(ox.front_rows(s), z["rows"][ro:ro + int(z["f"][s])]), s
    assert np.array_equal(ox.tags[:z["tags"].size], z["tags"])
