"""The interior-point session (opt_solver_b200/ipm.py) against the
reference's own smf::IpmSession (solver/src/ipm_session.cpp) on an IPM value
stream: barrier updates, steps whose Hessian block turns indefinite (more
negative pivots than constraints) and the inertia corrections after them.

Bar: at every step the session's decision (Ok / WrongInertia / Singular /
Error) equals the reference session's; every completed factor's inertia and
every learned expectation equal its; solutions within 1e-9 relative. The CPU
tests run the session over the oracle's factorization (the engine's bit for
bit twin, stopping after the full factor where the engine stops after the
tree level -- the decision is the same, the count only grows); the GPU tests
run it over the CUDA engine with its device-side early stop.
"""
from types import SimpleNamespace

import numpy as np
import pytest

from opt_solver_b200 import ipm as I
from opt_solver_b200 import workloads as W

STREAM = dict(m=6, n_con=100, steps=8, seed=3)
SOLVE_ANYWAY = {6}  # a step whose wrong factor the caller solves with regardless


class _OracleBackend:
    """The oracle's factorization behind smfg.Solver's factor / solve."""

    def __init__(self, O, a):
        self.O, self.a = O, a

    def factor(self, values, posdef=False, scale=None, max_negative_pivots=-1, raise_on_singular=False,
               **kw):
        O = self.O
        self.scale = scale
        self.fx = O.restated_factorize(self.a, O.permuted_values(self.a, values, scale), posdef)
        pos, neg, zero = self.fx.inertia
        st, fs = 0, 0
        if zero > 0:
            st, fs = 2, 2
        if not posdef and max_negative_pivots >= 0 and neg > max_negative_pivots:
            st, fs = 4, 4
        return SimpleNamespace(status=st, factor_status=fs, num_neg=neg, inertia=(pos, neg, zero))

    def solve(self, b):
        return self.O.restated_solve(self.a, self.fx, False, b, self.scale)

    def close(self):
        pass


def _reference_stream(O, n, cp, ri, vals, b):
    ref = O.ReferenceIpmSession()
    assert ref.analyse(n, cp, ri, vals[0], abort_on_wrong_inertia=True) == 0
    out = []
    for k, v in enumerate(vals):
        st, inert, _ = ref.factor(v)
        rec = {"status": st, "inertia": inert}
        if st == I.OK or k in SOLVE_ANYWAY:
            x, rc, inert2, learned = ref.solve(b)
            rec.update(solve_rc=rc, after=inert2, learned=learned, x=x)
        out.append(rec)
    return out


def _session_stream(sess, a, scale, vals, b):
    sess.analyse(a, posdef=False, scale=scale, ipm=I.IpmControl(learn_inertia=True, abort_on_wrong_inertia=True))
    out = []
    for k, v in enumerate(vals):
        st = sess.factor(v)
        rec = {"status": st, "inertia": sess.inertia()}
        if st == I.OK or k in SOLVE_ANYWAY:
            x, rc = sess.solve(b)
            rec.update(solve_rc=rc, after=sess.inertia(), learned=sess.expected_neg, x=x)
        out.append(rec)
    return out, sess


def _session_analysis(O, n, cp, ri, v0):
    """The analysis and scale the reference session runs on: its default
    Control (AutoSerial ordering, Auto scaling: the analysis' matching
    scale), deterministic mode, one thread."""
    ref = O.Reference(posdef=False, ordering=O.ORDER_AUTO_SERIAL, scaling=O.SCALE_AUTO,
                      deterministic=True, num_threads=1, top_tiles=True)
    a = ref.analyse(n, cp, ri, v0)
    fx = ref.factor(v0, export=False)
    return a, (fx.scale if len(fx.scale) else None)


def _check(got, want, kinds):
    for k, (g, w) in enumerate(zip(got, want)):
        assert g["status"] == w["status"], (k, kinds[k], g["status"], w["status"])
        if w["status"] != I.WRONG_INERTIA:
            assert g["inertia"] == w["inertia"], (k, g["inertia"], w["inertia"])
        else:  # both stopped past the expectation (partial counts)
            assert g["inertia"][1] > 0 and w["inertia"][1] > 0
        if "solve_rc" in w:
            assert g["solve_rc"] == w["solve_rc"] == 0
            assert g["after"] == w["after"], (k, g["after"], w["after"])
            assert g["learned"] == w["learned"], (k, g["learned"], w["learned"])
            xr = w["x"]
            assert np.max(np.abs(g["x"] - xr)) <= 1e-9 * max(1.0, np.max(np.abs(xr)))


def test_stream_decisions(ref_lib, oracle_lib):
    O = ref_lib
    n, cp, ri, vals, kinds = W.kkt_ipm_stream(**STREAM)
    b = W.rhs(n, 1, seed=2)
    want = _reference_stream(O, n, cp, ri, vals, b)
    # the stream does what it is for: aborts at the wrong steps, and the
    # solve after one completes it and learns its inertia
    sts = [r["status"] for r in want]
    assert sts == [I.WRONG_INERTIA if k == "wrong" else I.OK for k in kinds], sts
    assert want[6]["after"][1] > 100 and want[6]["learned"] == want[6]["after"][1]
    a, scale = _session_analysis(O, n, cp, ri, vals[0])
    got, sess = _session_stream(I.IpmSession(solver_factory=lambda a_, d: _OracleBackend(O, a_)), a, scale,
                                vals, b)
    _check(got, want, kinds)
    assert sess.stats.factorizations == len(vals) and sess.stats.aborted == kinds.count("wrong")


def test_no_abort_without_flag(ref_lib, oracle_lib):
    """abort_on_wrong_inertia off (the reference's default): every step runs
    to the end, Ok, with its full inertia."""
    O = ref_lib
    n, cp, ri, vals, kinds = W.kkt_ipm_stream(**STREAM)
    a, scale = _session_analysis(O, n, cp, ri, vals[0])
    sess = I.IpmSession(solver_factory=lambda a_, d: _OracleBackend(O, a_))
    sess.analyse(a, scale=scale)
    ref = O.ReferenceIpmSession()
    ref.analyse(n, cp, ri, vals[0], abort_on_wrong_inertia=False)
    b = W.rhs(n, 1, seed=4)
    for v in vals:
        st_r, in_r, _ = ref.factor(v)
        assert sess.factor(v) == st_r == I.OK
        assert sess.inertia() == in_r
        sess.solve(b)
        ref.solve(b)
    assert sess.stats.aborted == 0


def test_explicit_expectation_and_errors(ref_lib, oracle_lib):
    O = ref_lib
    n, cp, ri, vals, kinds = W.kkt_ipm_stream(**STREAM)
    a, scale = _session_analysis(O, n, cp, ri, vals[0])
    sess = I.IpmSession(solver_factory=lambda a_, d: _OracleBackend(O, a_))
    assert sess.factor(vals[0]) == I.ERROR  # no analysis yet
    sess.analyse(a, scale=scale, ipm=I.IpmControl(abort_on_wrong_inertia=True))
    ref = O.ReferenceIpmSession()
    ref.analyse(n, cp, ri, vals[0], abort_on_wrong_inertia=True)
    # an explicit expectation arms the abort before anything is learned
    for e in (99, 100):
        st_r, _, _ = ref.factor(vals[1], expected_negatives=e)
        assert sess.factor(vals[1], expected_negatives=e) == st_r
    assert st_r == I.OK
    # a solve with no factor (an aborted one is completed first; a fresh
    # session has none)
    fresh = I.IpmSession(solver_factory=lambda a_, d: _OracleBackend(O, a_))
    fresh.analyse(a, scale=scale)
    x, rc = fresh.solve(np.ones(n))
    assert x is None and rc != 0


# --------------------------------------------------------------------------
# On the GPU: the CUDA engine with its device-side early stop.

@pytest.mark.gpu
@pytest.mark.parametrize("stream", [STREAM, dict(m=10, n_con=700, steps=8, seed=6)],
                         ids=["kkt_6_100", "kkt_10_700_aptp"])
def test_gpu_stream_decisions(ref_lib, stream):
    O = ref_lib
    n, cp, ri, vals, kinds = W.kkt_ipm_stream(**stream)
    b = W.rhs(n, 1, seed=2)
    want = _reference_stream(O, n, cp, ri, vals, b)
    a, scale = _session_analysis(O, n, cp, ri, vals[0])
    got, sess = _session_stream(I.IpmSession(), a, scale, vals, b)
    _check(got, want, kinds)
    assert sess.stats.aborted == kinds.count("wrong")
    sess.close()


@pytest.mark.gpu
def test_gpu_inertia_stop_partial(ref_lib):
    """max_negative_pivots stops the level loop: partial counts past the
    limit, less work than the full factor, no solve; the next factorization
    runs in full, bit for bit the reference's."""
    O = ref_lib
    from opt_solver_b200 import smfg
    from tests.cases import reference_for
    from tests.test_gpu_parity import _compare_factor
    n, cp, ri, v = W.kkt_ipm(10, 700, seed=6)
    ref = reference_for(O, False, "auto", "auto")
    a = ref.analyse(n, cp, ri, v)
    fx = ref.factor(v)
    scale = fx.scale if len(fx.scale) else None
    sv = smfg.Solver(a)
    full = sv.factor(v, scale=scale)
    assert full.inertia == (1000, 700, 0)
    for limit in (10, 699):
        gi = sv.factor(v, scale=scale, max_negative_pivots=limit)
        assert gi.status == smfg.SMFG_ERR_WRONG_INERTIA
        assert gi.factor_status == smfg.SMFG_FACTOR_INERTIA_EXCEEDED
        assert limit < gi.num_neg <= 700 and gi.num_pos <= 1000
        if limit == 10:  # stopped low in the tree: most of the work skipped
            assert gi.flops < 0.5 * full.flops and sum(gi.inertia) < n
        with pytest.raises(smfg.SmfgError):
            sv.solve(np.ones(n))
    gi = sv.factor(v, scale=scale, max_negative_pivots=700)  # exactly the count: no stop
    assert gi.status == smfg.SMFG_OK and gi.inertia == (1000, 700, 0)
    gi = sv.factor(v, scale=scale)
    _compare_factor(a, fx, sv.export(), gi)
    sv.close()


@pytest.mark.gpu
def test_gpu_work_limit_and_rescue(ref_lib, oracle_lib):
    """The work limit stops a try on the device exactly when the reference's
    front work passes it; the scale-on-delay rescue over the engine keeps
    the same factor as over the oracle (bit for bit)."""
    O = ref_lib
    from opt_solver_b200 import smfg
    from opt_solver_b200 import delay as D
    from tests.cases import reference_for
    from tests.test_gpu_parity import _compare_factor
    n, cp, ri, v = W.kkt_ipm(6, 100, seed=3)
    ref = reference_for(O, False, "amd", "none")
    a = ref.analyse(n, cp, ri, v)
    ref.factor(v)
    work_ref, free = ref.front_work()
    sv = smfg.Solver(a)
    gi = sv.factor(v, work_limit=work_ref - 1)
    assert gi.status == smfg.SMFG_OK and gi.factor_status == smfg.SMFG_FACTOR_MAX_PIVOT_DELAYS
    with pytest.raises(smfg.SmfgError):
        sv.solve(np.ones(n))
    gi = sv.factor(v, work_limit=work_ref)
    assert gi.factor_status == smfg.SMFG_FACTOR_SUCCESS and D.engine_front_work(sv, a) == work_ref
    info, out = D.factor_scale_on_delay(sv, a, v, ratio=4.0)
    assert out["stopped_early"] and out["tripped"] and out["rescued"]
    want = O.restated_factorize(a, O.permuted_values(a, v, out["scale"]), False)
    _compare_factor(a, want, sv.export(), info)
    _, oout = D.factor_scale_on_delay(_OracleWork(O, a), a, v, ratio=4.0)
    assert oout["tripped"] and oout["rescued"] and oout["work"] == out["work"]
    # no matching scaling: the stopped try is run to the end unscaled
    info, out = D.factor_scale_on_delay(sv, a, v, ratio=1.0, rescue=lambda a_, v_: None)
    assert out["stopped_early"] and not out["rescued"]
    assert info.factor_status == smfg.SMFG_FACTOR_SUCCESS and info.inertia == (216, 100, 0)
    assert out["work"] == work_ref
    sv.close()


class _OracleWork(_OracleBackend):
    def front_stats(self):
        ncol = np.asarray(self.a.sn_end) - np.asarray(self.a.sn_start)
        fsym = np.diff(np.asarray(self.a.front_row_ptr))
        st = np.zeros((self.a.nsn, 5), dtype=np.int64)
        st[:, 4] = ncol + np.asarray(self.fx.f) - fsym - np.asarray(self.fx.p)
        return st
