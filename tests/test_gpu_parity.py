"""GPU parity: the CUDA numeric phase against the reference smf factor on the
same analysis and values (the reference's deterministic mode, one thread).

Bar: inertia, delays, 2x2 count, flop count, every front's realized size,
stored pivots, row order, pivot tags and L / D block bit for bit; the solve's
scaled backward error at the plain path's 1e-14 (omega) and the solution
within 1e-10 relative of the reference's.
"""
import numpy as np
import pytest

from tests.cases import cases, reference_for

pytestmark = pytest.mark.gpu


def _compare_factor(a, fx, gx, gi):
    assert gi.inertia == fx.inertia or fx.inertia == (0, 0, 0)
    assert gi.delayed_pivots == fx.delayed
    assert gi.two_by_two_pivots == fx.two_by_two
    assert gi.flops == fx.flops
    bad = []
    for s in range(a.nsn):
        if gx.f[s] != fx.f[s] or gx.p[s] != fx.p[s]:
            bad.append((s, "size", int(gx.f[s]), int(fx.f[s]), int(gx.p[s]), int(fx.p[s])))
            continue
        if not np.array_equal(gx.front_rows(s), fx.front_rows(s)):
            bad.append((s, "rows"))
            continue
        A, B = gx.block(s), fx.block(s)
        if not np.array_equal(A, B):
            bad.append((s, "block", float(np.max(np.abs(A - B)))))
    assert not bad, bad[:5]
    if fx.tags is not None:
        n_t = int(np.sum(fx.p))
        assert np.array_equal(gx.tags[:n_t], fx.tags[:n_t])


@pytest.mark.parametrize("case", cases("full"), ids=lambda c: c[0])
def test_factor_bitwise_and_solve(case, ref_lib):
    O = ref_lib
    from opt_solver_b200.smfg import Solver
    from opt_solver_b200 import workloads as W

    name, build, posdef, ordering, scaling, expect = case
    n, cp, ri, v = build()
    ref = reference_for(O, posdef, ordering, scaling)
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    scale = fx.scale if len(fx.scale) else None
    sv = Solver(a)
    gi = sv.factor(v, posdef=posdef, scale=scale)
    if expect is not None:
        assert gi.inertia == expect
    gx = sv.export()
    _compare_factor(a, fx, gx, gi)
    b = W.rhs(n, 1, seed=5)
    x = sv.solve(b)
    xr, _ = ref.solve(b)
    _, eta, om = O.residual(n, cp, ri, v, b, x)
    _, eta_r, om_r = O.residual(n, cp, ri, v, b, xr)
    # the plain path's bar (1e-14) where the reference meets it; on
    # ill-conditioned KKTs no worse than the reference's own unrefined solve
    assert om <= max(1e-14, 10 * om_r), (eta, om, om_r)
    assert np.max(np.abs(x - xr)) <= 1e-9 * max(1.0, np.max(np.abs(xr)))
    # the device residual agrees with the oracle's
    _, eta_d, om_d = sv.residual(b, x)
    assert om_d <= 4 * om + 1e-18
    if om > 1e-14:  # refinement on the device reaches the plain path's bar
        xf, eta_f, om_f, steps = sv.refine(b, x, max_steps=10, omega_target=1e-14)
        _, eta2, om2 = O.residual(n, cp, ri, v, b, xf)
        assert om2 <= 1e-14, (om2, steps)


@pytest.mark.gpu
def test_multi_rhs_and_jobs(ref_lib):
    O = ref_lib
    from opt_solver_b200.smfg import Solver, SOLVE_FORWARD, SOLVE_DIAGONAL, SOLVE_BACKWARD
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.trajectory_kkt(30, np.random.default_rng(2))
    ref = reference_for(O, False, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    ref.factor(v)
    sv = Solver(a)
    sv.factor(v, posdef=False)
    B = W.rhs(n, 8, seed=3, kind="normal")
    X = sv.solve(B)
    Xr, _ = ref.solve(B)
    assert np.max(np.abs(X - Xr)) <= 1e-9 * np.max(np.abs(Xr))
    # forward, diagonal, backward in sequence equal the full solve
    y = sv.solve(B[0], job=SOLVE_FORWARD)
    y = sv.solve(y, job=SOLVE_DIAGONAL)
    y = sv.solve(y, job=SOLVE_BACKWARD)
    assert np.max(np.abs(y - X[0])) <= 1e-10 * np.max(np.abs(X[0]))


@pytest.mark.gpu
def test_multi_rhs_residual_bitwise(ref_lib):
    """The residual of several columns per pass (8, then the rest) equals
    the one-column residual column by column, bit for bit; eta and omega are
    the columns' maxima."""
    O = ref_lib
    from opt_solver_b200.smfg import Solver
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.trajectory_kkt(30, np.random.default_rng(4))
    ref = reference_for(O, False, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    sv = Solver(a)
    sv.factor(v, posdef=False)
    B = W.rhs(n, 11, seed=6, kind="normal")
    X = sv.solve(B)
    X[3] *= 1.0 + 1e-9  # columns with different backward errors
    R, eta, om = sv.residual(B, X)
    etas, oms = [], []
    for k in range(B.shape[0]):
        r1, e1, o1 = sv.residual(B[k], X[k])
        assert np.array_equal(R[k], r1), k
        etas.append(e1)
        oms.append(o1)
    assert eta == max(etas) and om == max(oms)
    _, _, om_o = O.residual(n, cp, ri, v, B[3], X[3])
    assert oms[3] <= 4 * om_o + 1e-18


@pytest.mark.gpu
def test_refactor_reuses_plan(ref_lib):
    """IpmSession-style refactors of one analysis (ipm_session.cpp:147-243)."""
    O = ref_lib
    from opt_solver_b200.smfg import Solver
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.kkt_ipm(5, 60, seed=9)
    ref = reference_for(O, False, "auto", "auto")
    a = ref.analyse(n, cp, ri, v)
    sv = Solver(a)
    rng = np.random.default_rng(0)
    for step in range(3):
        v2 = v.copy()
        diag = np.concatenate([[True] * 0])
        v2 *= 1.0 + 0.1 * rng.standard_normal(v.size)
        fx = ref.factor(v2)
        scale = fx.scale if len(fx.scale) else None
        gi = sv.factor(v2, posdef=False, scale=scale)
        _compare_factor(a, fx, sv.export(), gi)


@pytest.mark.gpu
def test_not_posdef_and_nonfinite(ref_lib):
    O = ref_lib
    from opt_solver_b200.smfg import Solver, SmfgError
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.laplacian_2d(10)
    ref = reference_for(O, True, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    sv = Solver(a)
    bad = v.copy()
    bad[cp[:-1]] = -4.0  # negative diagonal: not positive definite
    gi = sv.factor(bad, posdef=True)
    assert gi.factor_status == 1
    nanv = v.copy()
    nanv[3] = np.nan
    with pytest.raises(SmfgError):
        sv.factor(nanv, posdef=True)
    gi = sv.factor(v, posdef=True)
    assert gi.status == 0 and gi.inertia == (n, 0, 0)


@pytest.mark.parametrize("team", [2, 4, 8, 16])
def test_panel_teams_bitwise(team, oracle_lib):
    """The indefinite large-front pivoting on a team of CTAs (a thread-block
    cluster splitting the swaps and eliminations by rows) gives the one-CTA
    factor bit for bit, and both the oracle's."""
    O = oracle_lib
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.kkt_ipm(12, 800, seed=11)
    a = smfg.analyse(n, cp, ri)
    # the threshold kernel on every front (the one-thread default mode), so
    # that the team kernels take the fronts of 512 rows and more as well
    ox = O.restated_factorize(a, O.permuted_values(a, v), False, aptp_min_rows=0)
    sv = smfg.Solver(a, device=0)
    g1 = sv.factor(v, posdef=False, panel_team=1, aptp_min_rows=0)
    e1 = sv.export()
    gt = sv.factor(v, posdef=False, panel_team=team, aptp_min_rows=0)
    et = sv.export()
    assert gt.inertia == g1.inertia == ox.inertia == (12 ** 3, 800, 0)
    assert gt.delayed_pivots == g1.delayed_pivots == ox.delayed > 0
    assert np.array_equal(et.blocks, e1.blocks)
    assert np.array_equal(et.rows, e1.rows)
    for s in range(a.nsn):
        assert np.array_equal(et.block(s), ox.block(s)), s
    sv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("f,ne,k", [(3001, 1777, 16), (2048, 2048, 1), (1500, 700, 2), (4097, 333, 13)])
def test_streamed_deferred_update_bitwise(f, ne, k):
    """The streamed deferred-update kernel gives the tiled kernel's result bit
    for bit on synthetic fronts (odd and even leading dimensions, ranks 1 to
    16, square and tall trapezoids)."""
    from opt_solver_b200 import smfg
    r = smfg.kernel_bench_defer(f, ne, k, reps=1)
    assert r["mismatches"] == 0
    assert r["ms"] > 0 and r["bytes"] > 0


@pytest.mark.gpu
def test_solve_into_given_array_and_refine_in_place():
    """solve(b, out=...) and refine(..., inplace=True) give the same values
    as the copying calls (the caller's buffers, e.g. pinned host memory)."""
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.laplacian_2d(40)
    sv = smfg.Solver(smfg.analyse(n, cp, ri))
    sv.factor(v, posdef=True)
    b = W.rhs(n, 1, seed=9)
    x0 = sv.solve(b)
    out = np.empty_like(b)
    x1 = sv.solve(b, out=out)
    assert x1 is out and np.array_equal(x1, x0)
    with pytest.raises(ValueError):
        sv.solve(b, out=np.empty(n + 1))
    xr, e0, o0, s0 = sv.refine(b, x0, max_steps=3, omega_target=1e-15)
    x2 = x0.copy()
    xi, e1, o1, s1 = sv.refine(b, x2, max_steps=3, omega_target=1e-15, inplace=True)
    assert xi is x2 and np.array_equal(xi, xr) and (e0, o0, s0) == (e1, o1, s1)
    sv.close()
