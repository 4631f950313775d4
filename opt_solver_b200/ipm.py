"""An interior-point session on the GPU engine: smf's IpmSession
(solver/include/smf/ipm_session.hpp:120-273, solver/src/ipm_session.cpp),
Feature 1 -- one KKT pattern refactored many times, the analysis, plan,
scaling and device buffers kept across the refactors, the expected number of
negative pivots learned from accepted factors, and the early abort once a
factorization's negative pivots pass it.

What carries over from the reference, and where:
  - analyse(): the analysis (smf's AnalysisKeep arrays) becomes a device plan
    once; the scaling is fixed for the session (smf's matching scale of the
    analysis, or one computed from the first values) and lives on the device
    with the plan, so a refactor only moves the new values
    (ipm_session.cpp:14-145);
  - factor(values, expected_negatives): armed with an expectation (given,
    else learned) and abort_on_wrong_inertia on an indefinite matrix, the
    engine stops as soon as the negative pivots so far pass it -- after the
    tree level where that happens, skipping the rest (the reference stops at
    the front; both decide the same, since the count only grows) -- and the
    result is WRONG_INERTIA with the partial counts (ipm_session.cpp:147-243);
  - solve(b): a solve after an aborted factor first factors the same values
    in full, without a limit; a successful solve accepts the factor and, with
    learn_inertia, its negative count becomes the expectation
    (ipm_session.cpp:386-443).
Not carried over: Feature 2 (re-analysis from the realized pivot order) and
Feature 3 (the static and quasidefinite modes); the reference ships both off
(its gates failed, ipm_session.hpp:26-32).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from opt_solver_b200 import smfg

# smf::IpmFactorStatus (ipm_session.hpp:47)
OK, WRONG_INERTIA, SINGULAR, ERROR = 0, 1, 2, 3


@dataclass
class IpmControl:
    learn_inertia: bool = True
    abort_on_wrong_inertia: bool = False   # the reference's default (its gate failed)


@dataclass
class IpmStats:
    factorizations: int = 0
    accepted: int = 0
    aborted: int = 0
    fronts_skipped_levels: list = field(default_factory=list)


class IpmSession:
    """smf::IpmSession (Feature 1) on one GPU. ``analysis`` is smf's analysis
    (the AnalysisKeep arrays, e.g. opt_solver_b200.smf_analysis); ``scale``
    the session's fixed scaling (original numbering) or None.
    ``solver_factory(analysis, device)`` makes the numeric back end (default
    smfg.Solver: factor() with max_negative_pivots, solve(), close())."""

    def __init__(self, device: int = 0, solver_factory=None):
        self.device = device
        self.solver_factory = solver_factory or (lambda a, dev: smfg.Solver(a, device=dev))
        self.solver = None
        self.n = 0

    def analyse(self, analysis, posdef: bool = False, scale=None, ipm: IpmControl | None = None,
                **factor_kw):
        if self.solver is not None:
            self.solver.close()
        self.solver = self.solver_factory(analysis, self.device)
        self.n = int(analysis.n)
        self.posdef = posdef
        self.scale = None if scale is None else np.ascontiguousarray(scale, dtype=np.float64)
        self.ipm = ipm or IpmControl()
        self.factor_kw = factor_kw
        self.stats = IpmStats()
        self.expected_neg = None
        self._values = None
        self._solvable = False
        self._aborted = False
        self._pending_accept = False
        self.info = None
        return 0

    def _run(self, limit: int):
        info = self.solver.factor(self._values, posdef=self.posdef, scale=self.scale,
                                  max_negative_pivots=limit, raise_on_singular=False, **self.factor_kw)
        self.info = info
        fs = info.factor_status
        if fs == smfg.SMFG_FACTOR_INERTIA_EXCEEDED:
            self._aborted = True
            self._solvable = False
            return WRONG_INERTIA
        self._aborted = False
        if info.status == smfg.SMFG_OK and fs in (smfg.SMFG_FACTOR_SUCCESS, smfg.SMFG_FACTOR_MAX_PIVOT_DELAYS):
            self._solvable = fs == smfg.SMFG_FACTOR_SUCCESS
            self._pending_accept = self._solvable
            return OK
        if info.status == smfg.SMFG_ERR_SINGULAR and fs == smfg.SMFG_FACTOR_SINGULAR:
            self._solvable = True
            self._pending_accept = True
            return SINGULAR
        self._solvable = False
        return ERROR

    def factor(self, values, expected_negatives: int | None = None) -> int:
        """Factor new values (the analysis' input entry order). Returns OK,
        WRONG_INERTIA (stopped early: inertia() holds the partial counts),
        SINGULAR or ERROR."""
        if self.solver is None:
            return ERROR
        self._values = np.ascontiguousarray(values, dtype=np.float64)
        self._solvable = self._aborted = self._pending_accept = False
        expected = expected_negatives if expected_negatives is not None else self.expected_neg
        limit = -1
        if self.ipm.abort_on_wrong_inertia and expected is not None and expected >= 0 and not self.posdef:
            limit = int(expected)
        self.stats.factorizations += 1
        st = self._run(limit)
        if st == WRONG_INERTIA:
            self.stats.aborted += 1
        return st

    def solve(self, b):
        """Solve with the last factor (b: (n,) or (nrhs, n)); an aborted factor
        is first completed. Returns (x, rc): rc 0 on success, nonzero when
        there is no factor to solve with."""
        if self._aborted:
            self._run(-1)
        if not self._solvable:
            return None, 1
        x = self.solver.solve(b)
        if self._pending_accept:
            self.stats.accepted += 1
            self._pending_accept = False
            if self.ipm.learn_inertia and not self.posdef:
                self.expected_neg = int(self.info.num_neg)
        return x, 0

    def inertia(self):
        if self.info is None:
            return (0, 0, 0)
        if self.posdef and self.info.status == smfg.SMFG_OK:
            return (self.n, 0, 0)
        return tuple(self.info.inertia)

    def close(self):
        if self.solver is not None:
            self.solver.close()
            self.solver = None
