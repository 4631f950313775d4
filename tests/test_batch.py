"""Configuration 4's batch: independent systems merged into one forest.

CPU: the merged analysis factors, in the oracle, to exactly the per-system
factors (blocks, rows, inertia) — the merge is a pure relabelling.
GPU: the engine factors and solves the forest; every system's inertia,
solution and backward error match its own factorization.
"""
import numpy as np
import pytest

from opt_solver_b200 import workloads as W


def _systems(count, seed=0, t_min=5, t_max=20):
    return W.trajectory_batch(count, seed=seed, t_min=t_min, t_max=t_max)


def test_merge_is_a_relabelling(oracle_lib):
    O = oracle_lib
    from opt_solver_b200 import smfg
    from opt_solver_b200.batch import merge_analyses
    mats = _systems(5, seed=3)
    ans = [smfg.analyse(n, cp, ri) for n, cp, ri, v in mats]
    merged, offs = merge_analyses(ans)
    vals = np.concatenate([m[3] for m in mats])
    mx = O.restated_factorize(merged, O.permuted_values(merged, vals), False)
    s0 = 0
    for (n, cp, ri, v), a, off in zip(mats, ans, offs):
        ox = O.restated_factorize(a, O.permuted_values(a, v), False)
        assert ox.inertia == (16 * ((n - 12) // 28) + 12, 12 * ((n - 12) // 28), 0)
        for s in range(a.nsn):
            assert mx.f[s0 + s] == ox.f[s] and mx.p[s0 + s] == ox.p[s]
            assert np.array_equal(mx.block(s0 + s), ox.block(s))
            assert np.array_equal(mx.front_rows(s0 + s), ox.front_rows(s) + off[0])
        s0 += a.nsn
    assert mx.inertia == tuple(sum(t) for t in zip(*[
        (16 * ((m[0] - 12) // 28) + 12, 12 * ((m[0] - 12) // 28), 0) for m in mats]))


@pytest.mark.gpu
def test_batch_factor_solve_per_system():
    from opt_solver_b200 import smfg
    from opt_solver_b200.batch import BatchSolver
    mats = _systems(64, seed=5, t_min=10, t_max=60)
    ans = [smfg.analyse(n, cp, ri) for n, cp, ri, v in mats]
    bs = BatchSolver(ans, device=0)
    info = bs.factor([m[3] for m in mats], posdef=False)
    stats = bs.system_stats()
    for (n, cp, ri, v), st in zip(mats, stats):
        T = (n - 12) // 28
        assert st[:3] == (16 * T + 12, 12 * T, 0)
    rhs = [W.rhs(m[0], 8, seed=i, kind="normal") for i, m in enumerate(mats)]
    X = bs.split(bs.solve(bs.stack_rhs(rhs)))
    # against each system factored on its own
    for i in (0, 17, 63):
        n, cp, ri, v = mats[i]
        sv = smfg.Solver(ans[i], device=0)
        sv.factor(v, posdef=False)
        xi = sv.solve(rhs[i])
        assert np.array_equal(X[i], xi)
        _, eta, om = sv.residual(rhs[i], X[i])
        assert om < 1e-12
        sv.close()
    bs.close()
