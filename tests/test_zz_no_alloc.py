"""The residual entry point that allocates nothing (smfg_residual_noalloc).

It exists for callers that must not allocate device memory once they are
running: a real-time controller that reserves all of its memory at start-up
(cudaMalloc can block and may synchronize the device), or a program whose
device memory is all committed to its own pool, where one more cudaMalloc
fails. Its scratch is a fixed array inside the library (orders up to
NOALLOC_MAX_N). These tests check it through the C ABI against the allocating
smfg_residual on two calls in a row (the shared scratch must not carry
anything from one call into the next), that a plan above the size limit is
refused, and that a plan which was never factored is refused rather than
read. This file is collected last: it must pass on its own in a fresh process
and after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solved_system(mat, posdef):
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = mat
    a = smfg.analyse(n, cp, ri)
    sv = smfg.Solver(a, device=0)
    sv.factor(v, posdef=posdef)
    b = W.rhs(n, 2, seed=11)
    x = sv.solve(b)
    return sv, b, x


@pytest.mark.parametrize("posdef", [True, False])
def test_noalloc_residual_matches_allocating_one(posdef):
    import torch
    from opt_solver_b200 import workloads as W
    mat = W.laplacian_2d(40) if posdef else W.trajectory_kkt(30, np.random.default_rng(5))
    sv, b, x = _solved_system(mat, posdef)
    # perturb x so that the residual is not at rounding level only
    x = x * (1.0 + 1e-6 * np.random.default_rng(1).standard_normal(x.shape))
    r_ref, eta_ref, om_ref = sv.residual(b, x)
    d_b = torch.from_numpy(np.ascontiguousarray(b)).cuda()
    d_x = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    for call in range(2):
        d_r = torch.full_like(d_b, float("nan"))
        eta, om = sv.residual_noalloc(d_b, d_x, d_r)
        r = d_r.cpu().numpy()
        np.testing.assert_allclose(r, r_ref, rtol=1e-12, atol=1e-300)
        assert eta == pytest.approx(eta_ref, rel=1e-12), call
        assert om == pytest.approx(om_ref, rel=1e-12), call
    sv.close()


def test_noalloc_rejects_orders_above_the_limit():
    import torch
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    side = int(np.ceil(np.sqrt(smfg.NOALLOC_MAX_N + 1)))
    n, cp, ri, v = W.laplacian_2d(side)
    assert n > smfg.NOALLOC_MAX_N
    a = smfg.analyse(n, cp, ri)
    sv = smfg.Solver(a, device=0)
    sv.factor(v, posdef=True)
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(smfg.SmfgError) as exc:
        sv.residual_noalloc(d, d)
    assert exc.value.code == 1
    assert "SMFG_NOALLOC_MAX_N" in str(exc.value)
    sv.close()


def test_residuals_refuse_a_plan_never_factored():
    import torch
    from opt_solver_b200 import smfg
    from opt_solver_b200 import workloads as W
    n, cp, ri, v = W.laplacian_2d(12)
    sv = smfg.Solver(smfg.analyse(n, cp, ri), device=0)
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    for call in (lambda: sv.residual_noalloc(d, d), lambda: sv.residual(np.ones(n), np.ones(n))):
        with pytest.raises(smfg.SmfgError) as exc:
            call()
        assert exc.value.code == smfg.SMFG_ERR_SINGULAR
    sv.factor(v, posdef=True)
    b = np.ones(n)
    x = sv.solve(b)
    eta, om = sv.residual_noalloc(torch.from_numpy(b).cuda(), torch.from_numpy(np.ascontiguousarray(x)).cuda())
    assert eta < 1e-14 and om < 1e-14
    sv.close()
