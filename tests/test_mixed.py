"""The mixed-precision path: large fronts factored in outer blocks whose
trailing updates run as TF32x3 / BF16x3 split products on the tensor cores,
FP64 threshold pivoting inside the blocks, FP64 refinement against A.

Bars: inertia identical to the plain FP64 path (and to the analytic
inertia of the KKT systems), scaled backward error <= 1e-12 after
refinement, fronts outside the mixed set and its ancestors bitwise equal
to the plain path, and a mask of zeros giving the plain factor exactly.
"""
import numpy as np
import pytest

from opt_solver_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _ancestors_or_self(parent, marked):
    out = np.zeros(len(parent), dtype=bool)
    for s in np.nonzero(marked)[0]:
        t = s
        while t >= 0 and not out[t]:
            out[t] = True
            t = parent[t]
    return out


def _solve_refine(sv, b, steps=12, method=None):
    from opt_solver_b200 import smfg
    x = sv.solve(b)
    x, eta, om, it = sv.refine(b, x, max_steps=steps, omega_target=1e-13,
                               method=smfg.REFINE_AUTO if method is None else method)
    return x, om, it


@pytest.mark.parametrize("block,kind", [(256, 0), (64, 0), (512, 0), (256, 1)])
def test_mixed_spd(block, kind):
    from opt_solver_b200 import smfg
    n, cp, ri, v = W.varcoef_3d(24, seed=3)
    a = smfg.analyse(n, cp, ri)
    b = W.rhs(n, 1, seed=4)
    sv = smfg.Solver(a, device=0)
    sv.factor(v, posdef=True)
    plain = sv.export()
    xp = sv.solve(b)
    im = sv.factor(v, posdef=True, precision=smfg.PREC_MIXED, mixed_block=block, mixed_kind=kind,
                   mixed_min_front=384)
    assert im.status == 0 and im.mixed_fronts > 0 and im.reserved_d[3] > 0
    assert im.inertia == (n, 0, 0)
    mixed = sv.export()
    fsym = np.diff(a.front_row_ptr)
    is_mixed = fsym >= 384
    touched = _ancestors_or_self(a.sn_parent, is_mixed)
    for s in range(a.nsn):
        if not touched[s]:
            assert np.array_equal(mixed.block(s), plain.block(s))
        else:
            # normwise: entries of the near-null mode's last pivots lose
            # relative accuracy; refinement below is the accuracy bar
            mb, pb = mixed.block(s), plain.block(s)
            assert np.all(np.isfinite(mb))
            assert np.linalg.norm(mb - pb) <= 1e-3 * np.linalg.norm(pb)
    x, om, it = _solve_refine(sv, b, steps=30)
    assert om <= 1e-12, (om, it)
    assert np.max(np.abs(x - xp)) <= 1e-6 * np.max(np.abs(xp))
    sv.close()


def test_mixed_mask_zero_is_plain():
    from opt_solver_b200 import smfg
    n, cp, ri, v = W.varcoef_3d(20, seed=5)
    a = smfg.analyse(n, cp, ri)
    sv = smfg.Solver(a, device=0)
    sv.factor(v, posdef=True)
    plain = sv.export()
    sv.set_front_precision(np.zeros(a.nsn, dtype=np.int8))
    im = sv.factor(v, posdef=True, precision=smfg.PREC_MIXED)
    assert im.mixed_fronts == 0
    mixed = sv.export()
    assert np.array_equal(mixed.blocks, plain.blocks)
    sv.set_front_precision(None)
    sv.close()


@pytest.mark.parametrize("m,ncon,block", [(12, 800, 256), (14, 1500, 64), (16, 2000, 256)])
def test_mixed_kkt_threshold_kernel(m, ncon, block):
    """The threshold kernel's mixed path (aptp_min_rows = 0): FP64 pivoting,
    tensor-core contribution-block updates every `block` pivots."""
    from opt_solver_b200 import smfg
    n, cp, ri, v = W.kkt_ipm(m, ncon, seed=7)
    a = smfg.analyse(n, cp, ri)
    b = W.rhs(n, 1, seed=8, kind="normal")
    sv = smfg.Solver(a, device=0)
    ip = sv.factor(v, posdef=False, aptp_min_rows=0)
    assert ip.inertia == (m ** 3, ncon, 0)
    im = sv.factor(v, posdef=False, precision=smfg.PREC_MIXED, mixed_block=block, aptp_min_rows=0)
    assert im.status == 0 and im.mixed_fronts > 0
    assert im.inertia == ip.inertia
    x, om, it = _solve_refine(sv, b)
    assert om <= 1e-12, (om, it)
    sv.close()


@pytest.mark.parametrize("method", [0, 1, 2])
def test_refine_methods_plain(method):
    """Each refinement method on the plain FP64 factor of an indefinite
    KKT: the gate is met and the iterate is at least as good as the solve."""
    from opt_solver_b200 import smfg
    n, cp, ri, v = W.kkt_ipm(10, 500, seed=9)
    a = smfg.analyse(n, cp, ri)
    b = W.rhs(n, 1, seed=10, kind="normal")
    sv = smfg.Solver(a, device=0)
    sv.factor(v, posdef=False)
    x0 = sv.solve(b)
    _, _, om0 = sv.residual(b, x0)
    x, eta, om, it = sv.refine(b, x0, max_steps=10, omega_target=1e-15, method=method)
    assert om <= max(om0, 1e-15) and eta <= 1e-10
    sv.close()
