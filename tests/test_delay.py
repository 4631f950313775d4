"""Front work and the scale-on-delay rescue (opt_solver_b200/delay.py), on
the CPU: the front-work count is pinned against the reference's own
Info::front_work and delay_free_front_work on delay-heavy KKTs, and the
rescue policy runs end to end over the oracle's factorization (the engine's
bit-for-bit twin) as its backend."""
import numpy as np
import pytest

from opt_solver_b200 import delay as D
from opt_solver_b200 import workloads as W
from tests.cases import reference_for

CASES = [
    ("traj60", lambda: W.trajectory_kkt(60, np.random.default_rng(4)), "amd", "none"),
    ("traj40", lambda: W.trajectory_kkt(40, np.random.default_rng(7)), "amd", "none"),
    ("kkt_6_100", lambda: W.kkt_ipm(6, 100, seed=3), "auto", "auto"),
    ("kkt_6_100_unscaled", lambda: W.kkt_ipm(6, 100, seed=3), "amd", "none"),
]


def _delayed_out(a, f, p):
    ncol = np.asarray(a.sn_end) - np.asarray(a.sn_start)
    fsym = np.diff(np.asarray(a.front_row_ptr))
    return ncol + np.asarray(f) - fsym - np.asarray(p)


class _OracleSolver:
    """The oracle's factorization behind smfg.Solver's factor / front_stats."""

    def __init__(self, O, a):
        self.O, self.a, self.scales = O, a, []

    def factor(self, values, posdef=False, scale=None):
        self.scales.append(scale)
        self.fx = self.O.restated_factorize(self.a, self.O.permuted_values(self.a, values, scale), posdef)
        return self.fx

    def front_stats(self):
        st = np.zeros((self.a.nsn, 5), dtype=np.int64)
        st[:, 4] = _delayed_out(self.a, self.fx.f, self.fx.p)
        return st


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_front_work_like_reference(case, ref_lib, oracle_lib):
    O = ref_lib
    name, build, ordering, scaling = case
    n, cp, ri, v = build()
    ref = reference_for(O, False, ordering, scaling)
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    work, free = ref.front_work()
    assert fx.delayed > 0
    assert D.delay_free_front_work(a) == free
    assert D.front_work(a, fx.f) == work
    assert work > free
    # the engine's route: realized sizes from each front's delayed columns
    f = D.realized_front_sizes(a, _delayed_out(a, fx.f, fx.p))
    assert np.array_equal(f, fx.f)
    scale = fx.scale if len(fx.scale) else None
    ox = O.restated_factorize(a, O.permuted_values(a, v, scale), False)
    assert D.front_work(a, ox.f) == work


def test_rescue_trips_and_rescales(ref_lib, oracle_lib):
    O = ref_lib
    n, cp, ri, v = W.kkt_ipm(6, 100, seed=3)
    ref = reference_for(O, False, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    ref.factor(v)
    work_ref, free_ref = ref.front_work()
    ratio = 4.0
    assert work_ref > np.floor(ratio * free_ref)  # the reference's count trips this limit
    sv = _OracleSolver(O, a)
    fx, out = D.factor_scale_on_delay(sv, a, v, ratio=ratio)
    assert out["first_work"] == work_ref and out["limit"] == np.floor(ratio * free_ref)
    assert out["tripped"] and out["rescued"] and out["first_status"] == D.FACTOR_MAX_PIVOT_DELAYS
    assert len(sv.scales) == 2 and sv.scales[0] is None and sv.scales[1] is not None
    # the matching scaling cuts the delays' inflation; the inertia stands
    assert out["work"] < out["first_work"]
    assert fx.inertia == (216, 100, 0)
    x = O.restated_solve(a, fx, False, np.ones(n), out["scale"])
    _, eta, om = O.residual(n, cp, ri, v, np.ones(n), x)
    assert om <= 1e-12


def test_rescue_not_tripped_and_not_found(ref_lib, oracle_lib):
    O = ref_lib
    n, cp, ri, v = W.trajectory_kkt(40, np.random.default_rng(7))
    ref = reference_for(O, False, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    # under the default ratio (16) the trajectory's inflation (about 6x) passes
    sv = _OracleSolver(O, a)
    fx, out = D.factor_scale_on_delay(sv, a, v)
    assert not out["tripped"] and len(sv.scales) == 1
    assert out["work"] <= out["limit"]
    # a trip without a matching scaling keeps the first factorization
    sv = _OracleSolver(O, a)
    fx, out = D.factor_scale_on_delay(sv, a, v, ratio=1.0, rescue=lambda a_, v_: None)
    assert out["tripped"] and not out["rescued"] and len(sv.scales) == 1
    assert fx.inertia == (16 * 40 + 12, 12 * 40, 0)
    # a negative ratio disarms the limit
    sv = _OracleSolver(O, a)
    _, out = D.factor_scale_on_delay(sv, a, v, ratio=-1.0)
    assert out["limit"] == -1 and not out["tripped"]
