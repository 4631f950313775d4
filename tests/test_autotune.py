"""The autotuner (opt_solver_b200/autotune.py): buckets of the analysis,
and on the GPU a tuned team table that is no slower than the built-in rule
on the tuned matrix and gives the same factor bit for bit."""
import os

import numpy as np
import pytest

from opt_solver_b200 import workloads as W


def _kkt():
    """The 20^3 + 4,000 KKT on smf's own METIS analysis (its record)."""
    from opt_solver_b200 import smf_analysis as SA
    n, cp, ri, v = W.kkt_ipm(20, 4000, seed=0)
    a = SA.load(os.path.join(os.path.dirname(__file__), "golden", "kkt20_4000_smf_partition.npz"), n, cp, ri)
    return n, cp, ri, v, a


def test_buckets_present():
    from opt_solver_b200 import autotune
    n, cp, ri, v, a = _kkt()
    b = autotune._buckets_present(a)
    assert b == sorted(b, reverse=True) and set(b) <= {0, 1, 2, 3} and 3 in b


@pytest.mark.gpu
def test_autotune_teams():
    from opt_solver_b200 import autotune, smfg
    n, cp, ri, v, a = _kkt()
    scale = smfg.matching_scale(n, cp, ri, v)[0]
    sv = smfg.Solver(a, device=0)
    sv.factor(v, posdef=False, scale=scale)
    e0 = sv.export()
    res = autotune.tune(sv, a, v, False, scale=scale)
    print(res["panel_teams"], round(res["default_ms"], 1), "->", round(res["best_ms"], 1))
    assert all(t in (0, 1, 2, 4, 8, 16) for t in res["panel_teams"])
    assert res["best_ms"] <= res["default_ms"]
    sv.factor(v, posdef=False, scale=scale)   # with the tuned table on the plan
    e1 = sv.export()
    assert np.array_equal(e0.blocks, e1.blocks)
    sv.close()
