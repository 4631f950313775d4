"""The oracle pinned against the reference (CPU): the plain-C restatement of
the numeric phase (oracle/mf_oracle.c) must reproduce the reference smf
factor bit for bit on the same analysis and values, and both must meet the
reference's own accuracy bars."""
import numpy as np
import pytest

from tests.cases import cases, reference_for


def _bitwise_same(a, fx, ox):
    assert ox.status in (0, 2)
    assert ox.delayed == fx.delayed
    assert ox.two_by_two == fx.two_by_two
    assert ox.flops == fx.flops
    if fx.inertia != (0, 0, 0):
        assert ox.inertia == fx.inertia
    for s in range(a.nsn):
        assert ox.f[s] == fx.f[s] and ox.p[s] == fx.p[s], s
        assert np.array_equal(ox.front_rows(s), fx.front_rows(s)), s
        assert np.array_equal(ox.block(s), fx.block(s)), s
    if fx.tags is not None:
        n_t = int(np.sum(fx.p))
        assert np.array_equal(ox.tags[:n_t], fx.tags[:n_t])


@pytest.mark.parametrize("case", cases("small"), ids=lambda c: c[0])
def test_restatement_bitwise_vs_reference(case, ref_lib, oracle_lib):
    O = ref_lib
    name, build, posdef, ordering, scaling, expect = case
    n, cp, ri, v = build()
    ref = reference_for(O, posdef, ordering, scaling)
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    scale = fx.scale if len(fx.scale) else None
    pv = O.permuted_values(a, v, scale)
    ox = O.restated_factorize(a, pv, posdef)
    _bitwise_same(a, fx, ox)
    if expect is not None:
        assert ox.inertia == expect
    b = np.random.default_rng(1).uniform(-1, 1, n)
    x = O.restated_solve(a, ox, posdef, b, scale)
    _, eta, om = O.residual(n, cp, ri, v, b, x)
    assert eta <= 1e-10 and om <= 1e-12


def test_restatement_delays_and_2x2(ref_lib, oracle_lib):
    """A trajectory KKT: thousands of delayed columns and 2x2 pivots."""
    O = ref_lib
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.trajectory_kkt(60, np.random.default_rng(4))
    ref = reference_for(O, False, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    assert fx.delayed > 0 and fx.two_by_two > 0
    ox = O.restated_factorize(a, O.permuted_values(a, v), False)
    _bitwise_same(a, fx, ox)
    assert ox.inertia == (16 * 60 + 12, 12 * 60, 0)
