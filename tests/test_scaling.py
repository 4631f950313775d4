"""Symmetric max-product matching scaling (smfg_matching_scale, the
scaling smf applies with matching scaling on, solver/src/scaling_matching.cpp):
|s_i a_ij s_j| <= 1 everywhere, a unit entry in every row (the matched
ones), a perfect matching on nonsingular inputs, the same properties as
the reference's scale of a committed golden case, and, where the reference
library is built, the reference's own scale to rounding.

Row maxima: the symmetric scale s = sqrt(r c) of a matching's row and
column scalings makes the matched entries exactly 1 only on symmetric
matchings, so the test asks 1 of this matcher on these inputs and a bound
of 1/4 of the reference's scale.
"""
import os

import numpy as np
import pytest

from opt_solver_b200 import workloads as W


def _props(n, cp, ri, v, s):
    cols = np.repeat(np.arange(n), np.diff(cp))
    a = np.abs(v) * s[ri] * s[cols]
    rowmax = np.zeros(n)
    np.maximum.at(rowmax, ri, a)
    np.maximum.at(rowmax, cols, a)
    return a.max(), rowmax.min()


@pytest.mark.parametrize("gen", [lambda: W.kkt_ipm(6, 120, seed=1), lambda: W.kkt_ipm(10, 600, seed=2),
                                 lambda: W.varcoef_3d(8, seed=3),
                                 lambda: W.trajectory_kkt(20, np.random.default_rng(4))])
def test_matching_scale_properties(gen):
    from opt_solver_b200 import smfg
    n, cp, ri, v = gen()
    s, um = smfg.matching_scale(n, cp, ri, v)
    assert um == 0 and np.all(np.isfinite(s)) and np.all(s > 0)
    mx, mn = _props(n, cp, ri, v, s)
    assert mx <= 1.0 + 1e-12 and mn >= 1.0 - 1e-12


def test_matching_scale_like_reference():
    from opt_solver_b200 import smfg
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "kkt_5_60.npz"))
    n, cp, ri, v = int(z["n"]), z["col_ptr"], z["row_idx"], z["values"]
    s, um = smfg.matching_scale(n, cp, ri, v)
    assert um == 0
    # both bound the scaled entries by 1; the symmetrized scale keeps every
    # row's largest entry near 1 (exactly 1 on a symmetric matching)
    for sc in (s, z["scale"]):
        mx, mn = _props(n, cp, ri, v, sc)
        assert mx <= 1.0 + 1e-12 and mn >= 0.25


@pytest.mark.parametrize("gen", [lambda: W.kkt_ipm(6, 120, seed=1), lambda: W.kkt_ipm(10, 600, seed=2),
                                 lambda: W.varcoef_3d(8, seed=3), lambda: W.laplacian_2d(40),
                                 lambda: W.trajectory_kkt(20, np.random.default_rng(4)),
                                 lambda: W.trajectory_kkt(60, np.random.default_rng(5))],
                         ids=["kkt_6_120", "kkt_10_600", "var3d_8", "lap2d_40", "traj20", "traj60"])
def test_matching_scale_equals_reference(gen, ref_lib):
    """The same scale as the reference's own matching scaling
    (compute_matching_scale, solver/src/scaling_matching.cpp:1109) to
    rounding: the same matching and the same duals."""
    from opt_solver_b200 import smfg
    n, cp, ri, v = gen()
    s, um = smfg.matching_scale(n, cp, ri, v)
    sr, rc = ref_lib.reference_matching_scale(n, cp, ri, v)
    assert um == 0 and rc == 0
    assert np.max(np.abs(s / sr - 1.0)) <= 1e-13


def test_matching_scale_errors():
    from opt_solver_b200 import smfg
    n, cp, ri, v = W.kkt_ipm(4, 20, seed=0)
    v = v.copy()
    v[3] = np.nan
    with pytest.raises(smfg.SmfgError):
        smfg.matching_scale(n, cp, ri, v)
