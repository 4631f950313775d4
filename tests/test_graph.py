"""CUDA-graph replay of the factorization (smfg_control_t.graph): the first
call captures, later calls with the same configuration replay; a replay
gives the normal path's factor bit for bit, also on new values of the same
pattern (the interior-point refactor), and falls back to the normal path
when the configuration changes."""
import numpy as np
import pytest

from opt_solver_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["spd", "kkt", "kkt_mixed"])
def test_graph_replay_bitwise(kind):
    import torch
    from opt_solver_b200 import smfg
    if kind == "spd":
        n, cp, ri, v = W.varcoef_3d(20, seed=2)
        posdef = True
    else:
        n, cp, ri, v = W.kkt_ipm(12, 800, seed=4)
        posdef = False
    prec = smfg.PREC_MIXED if kind == "kkt_mixed" else smfg.PREC_FP64
    a = smfg.analyse(n, cp, ri)
    sv = smfg.Solver(a, device=0)
    d_v = torch.from_numpy(np.ascontiguousarray(v)).cuda()
    ref = sv.factor(d_v, posdef=posdef, precision=prec)
    e_ref = sv.export()
    g1 = sv.factor(d_v, posdef=posdef, precision=prec, graph=True)   # normal + capture
    g2 = sv.factor(d_v, posdef=posdef, precision=prec, graph=True)   # replay
    e2 = sv.export()
    assert g2.inertia == ref.inertia and g2.delayed_pivots == ref.delayed_pivots
    assert np.array_equal(e2.blocks, e_ref.blocks) and np.array_equal(e2.rows, e_ref.rows)
    # new values of the same pattern (a scaled diagonal), replayed in place
    # (SPD: a larger diagonal keeps it positive definite; KKT: the primal
    # block's diagonal, Sigma, moves as in an interior-point iteration)
    rng = np.random.default_rng(1)
    v2 = v.copy()
    diag = np.asarray(ri) == np.repeat(np.arange(n), np.diff(cp))
    sel = diag & (v > 0)
    v2[sel] *= rng.uniform(1.0, 2.0, int(sel.sum()))
    d_v.copy_(torch.from_numpy(v2))
    g3 = sv.factor(d_v, posdef=posdef, precision=prec, graph=True)   # replay
    e3 = sv.export()
    r3 = sv.factor(d_v, posdef=posdef, precision=prec)               # normal path
    er = sv.export()
    assert g3.inertia == r3.inertia and g3.delayed_pivots == r3.delayed_pivots
    assert np.array_equal(e3.blocks, er.blocks)
    b = W.rhs(n, 1, seed=3)
    x = sv.solve(b)
    x, _, om, _ = sv.refine(b, x, max_steps=20, omega_target=1e-13, method=smfg.REFINE_AUTO)
    assert om < 1e-12
    sv.close()
