"""Autotuner of the engine's launch shapes per front-size bucket, on the
caller's own matrix (one analysis, its values), by timing factorizations on
the device.

Tuned: the team size (CTAs of a thread-block cluster) of the indefinite
large-front pivoting for each size bucket of a level's largest front
([384, 768), [768, 1536), [1536, 3072), >= 3072 rows), by coordinate
descent from the largest bucket down, and for the mixed SPD path the outer
block (pivots per tensor-core update: 128, 256, 512). Every candidate gives
the same factor (the plain path is bitwise the same for every team size);
only time is compared. The choice is set on the plan
(smfg_set_panel_teams) and returned with the timings, to be reused for the
pattern (an interior-point session tunes once).
"""
from __future__ import annotations

import numpy as np

from . import smfg

BUCKETS = ((384, 768), (768, 1536), (1536, 3072), (3072, 1 << 30))
TEAMS = (1, 2, 4, 8, 16)
BLOCKS = (128, 256, 512)


def _buckets_present(a) -> list:
    """Buckets of the levels' largest large fronts in this analysis."""
    f = np.diff(np.asarray(a.front_row_ptr))
    parent = np.asarray(a.sn_parent)
    h = np.zeros(a.nsn, dtype=np.int64)  # height above the leaves = the engine's level
    for s in range(a.nsn):  # postorder
        p = parent[s]
        if p >= 0:
            h[p] = max(h[p], h[s] + 1)
    present = set()
    for lvl in np.unique(h):
        fl = f[h == lvl]
        big = fl[fl >= BUCKETS[0][0]]
        if big.size:
            m = int(big.max())
            for b, (lo, hi) in enumerate(BUCKETS):
                if lo <= m < hi:
                    present.add(b)
    return sorted(present, reverse=True)


def _time(sv, values, reps, **kw) -> float:
    best = float("inf")
    for _ in range(reps):
        info = sv.factor(values, **kw)
        best = min(best, info.factor_ms)
    return best


def tune(sv, a, values, posdef: bool, scale=None, precision: int = smfg.PREC_FP64, reps: int = 2) -> dict:
    """Tune `sv` (a Solver on analysis `a`) on `values`; returns the choice
    and the measured factor times (ms)."""
    kw = dict(posdef=posdef, scale=scale, precision=precision)
    teams = [0, 0, 0, 0]
    sv.set_panel_teams(teams)
    base = _time(sv, values, reps, **kw)
    log = {"default": base}
    best_t = base
    if not posdef:
        for b in _buckets_present(a):
            choice = teams[b]
            for t in TEAMS:
                trial = list(teams)
                trial[b] = t
                sv.set_panel_teams(trial)
                ms = _time(sv, values, reps, **kw)
                log[f"bucket{b}_team{t}"] = ms
                if ms < best_t:
                    best_t, choice = ms, t
            teams[b] = choice
        sv.set_panel_teams(teams)
    block = 0
    if posdef and precision == smfg.PREC_MIXED:
        for blk in BLOCKS:
            ms = _time(sv, values, reps, mixed_block=blk, **kw)
            log[f"block{blk}"] = ms
            if ms < best_t:
                best_t, block = ms, blk
    return {"panel_teams": teams, "mixed_block": block, "best_ms": best_t, "default_ms": base, "trials": log}
