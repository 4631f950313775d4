"""Front work, the work limit and the scale-on-delay rescue: host policy
around the GPU factor.

The reference measures how much delayed pivots inflate a factorization by
its front work (Info::front_work): over the fronts, the fully summed columns
times the rows squared, summed as integers
(solver/src/multifrontal_serial.cpp:875). A column delayed out of a child
joins its parent as one more fully summed column and one more row, so a
front whose analysis gave it c columns and f0 rows, realized at f rows,
has c + (f - f0) fully summed columns. Without delays the sum is the
analysis' delay-free front work (delay_free_front_work,
solver/src/factor_indef.cpp:896-903).

The scale-on-delay rescue (Control::scale_on_delay_ratio, default 16,
solver/src/solve.cpp:289-560): an indefinite factorization whose front work
passes floor(ratio x delay-free work) is given up (MaxPivotDelays) and redone
with the maximum-product matching scaling of its own values; without such
a scaling (structurally singular values) the factorization runs as Auto
resolves it, to the end (solve.cpp:304-306).
The engine stops a try on the device (smfg_control_t.work_limit): after each
tree level it adds the level's front work to the count so far and skips the
rest once the count passes the limit (the reference stops after the front,
multifrontal_serial.cpp:660-671; the count only grows, so both stop exactly
when the finished count would pass). A back end without that stop is
checked on its finished factor, as the reference's task-parallel engine
does (factor_indef.cpp:834-851): the same decision, no work saved. The
reference's refinements of that policy (a kept scale reused across
refactors, the tighter next limit, the early stop on projected inflation,
the static-pivoting fallback) are not restated.
"""
from __future__ import annotations

import inspect
import math

import numpy as np

# smf::FactorStatus::MaxPivotDelays (solver/include/smf/types.hpp:234)
FACTOR_MAX_PIVOT_DELAYS = 3
# Control::scale_on_delay_ratio (solver/include/smf/control.hpp:176)
SCALE_ON_DELAY_RATIO = 16.0


def _columns_and_rows(a):
    ncol = (np.asarray(a.sn_end, dtype=np.int64) - np.asarray(a.sn_start, dtype=np.int64))
    fsym = np.diff(np.asarray(a.front_row_ptr, dtype=np.int64))
    return ncol, fsym


def delay_free_front_work(a) -> float:
    """Sum over fronts of columns x rows^2 as analysed (no delays; int64
    products and sum, exact below 9.2e18)."""
    ncol, fsym = _columns_and_rows(a)
    return float(np.sum(ncol * fsym * fsym))


def realized_front_sizes(a, delayed_out) -> np.ndarray:
    """Each front's realized rows: its analysed rows plus the columns its
    children delayed to it (delayed_out[s]: columns front s passed up)."""
    _, fsym = _columns_and_rows(a)
    f = fsym.copy()
    par = np.asarray(a.sn_parent, dtype=np.int64)
    d = np.asarray(delayed_out, dtype=np.int64)
    has = par >= 0
    np.add.at(f, par[has], d[has])
    return f


def front_work(a, f) -> float:
    """Info::front_work of a factorization whose fronts realized f rows."""
    ncol, fsym = _columns_and_rows(a)
    f = np.asarray(f, dtype=np.int64)
    elig = ncol + f - fsym
    return float(np.sum(elig * f * f))


def engine_front_work(solver, a) -> float:
    """Front work of the solver's last factorization, from its per-front
    delayed columns (smfg_front_stats)."""
    return front_work(a, realized_front_sizes(a, solver.front_stats()[:, 4]))


def cleaned_values(a, values) -> np.ndarray:
    """The caller's values on the cleaned pattern (duplicates summed in
    input order, dropped entries left out)."""
    v = np.asarray(values, dtype=np.float64)
    o2c = np.asarray(a.orig_to_clean, dtype=np.int64)
    out = np.zeros(int(np.asarray(a.clean_col_ptr)[-1]), dtype=np.float64)
    kept = o2c >= 0
    np.add.at(out, o2c[kept], v[kept])  # unbuffered: in input order
    return out


def rescue_scale(a, values):
    """The matching scaling of the values (original numbering), or None when
    the values have none (a column left unmatched)."""
    from opt_solver_b200 import smfg
    s, unmatched = smfg.matching_scale(a.n, a.clean_col_ptr, a.clean_row_idx, cleaned_values(a, values))
    if unmatched or not np.all(np.isfinite(s)) or not np.all(s > 0):
        return None
    return s


def _has_early_stop(solver) -> bool:
    try:
        return "work_limit" in inspect.signature(solver.factor).parameters
    except (TypeError, ValueError):
        return False


def factor_scale_on_delay(solver, a, values, ratio: float = SCALE_ON_DELAY_RATIO, scale=None,
                          rescue=rescue_scale, early_stop=None, **factor_kw):
    """Indefinite factor with the scale-on-delay rescue. ``solver`` has
    ``factor(values, posdef=False, scale=..., **kw)`` and ``front_stats()``
    (smfg.Solver); ``scale`` is the first try's scaling, as the caller's
    Auto resolved it. ``early_stop`` (default: when solver.factor takes
    ``work_limit``) stops the first try on the device at the limit. Returns
    (info of the kept factor, outcome) where outcome holds the delay-free
    work, the limit, each try's front work (None for a try stopped early),
    whether the limit tripped, whether the try stopped early and whether the
    rescue ran."""
    free = delay_free_front_work(a)
    limit = math.floor(ratio * free) if ratio >= 0 else -1
    if early_stop is None:
        early_stop = _has_early_stop(solver)
    stop = early_stop and limit >= 0
    kw = dict(factor_kw, work_limit=float(limit)) if stop else factor_kw
    info = solver.factor(values, posdef=False, scale=scale, **kw)
    stopped = stop and getattr(info, "factor_status", 0) == FACTOR_MAX_PIVOT_DELAYS
    work = None if stopped else engine_front_work(solver, a)
    out = {"free_work": free, "limit": limit, "first_work": work, "tripped": stopped,
           "stopped_early": stopped, "rescued": False, "work": work, "scale": scale}
    if not stopped and (limit < 0 or work <= limit):
        return info, out
    out["tripped"] = True
    out["first_status"] = FACTOR_MAX_PIVOT_DELAYS  # the try given up, as smf reports it
    s = rescue(a, values)
    if s is None:
        # no matching scaling: the factorization as Auto resolves it stands,
        # run to the end when the try stopped early
        if stopped:
            info = solver.factor(values, posdef=False, scale=scale, **factor_kw)
            out["work"] = engine_front_work(solver, a)
        return info, out
    info = solver.factor(values, posdef=False, scale=s, **factor_kw)
    out.update(rescued=True, work=engine_front_work(solver, a), scale=s)
    return info, out
