"""Many independent systems in one factorization (configuration 4's 1,024
trajectory KKTs).

The analyses of the systems are merged into one forest: block-diagonal
pattern, supernodes concatenated (each system's postorder numbering shifted,
so the concatenation is a postorder of the forest), children, front rows and
value maps shifted by the system's column, entry and supernode offsets. The
engine's level scheduling then factors level l of every system in the same
kernels: thousands of small fronts of uneven sizes per launch instead of one
small launch per system and level. Statuses and inertia stay per system
(the trees share nothing); the reference has no batch API (its harness loops
over systems with smf_ipm_* calls), so per-system results are what a caller
of smf would get from 1,024 separate factorizations.
"""
from __future__ import annotations

import numpy as np

from . import smfg


def merge_analyses(analyses):
    """One smfg.Analysis for the block-diagonal union of `analyses`."""
    n_off = s_off = e_off = c_off = k_off = r_off = 0
    parts = {k: [] for k in smfg._ANALYSIS_FIELDS}
    offsets = []
    for a in analyses:
        n, ns = int(a.n), int(a.nsn)
        nnz_perm = int(a.perm_col_ptr[-1])
        nnz_clean = int(a.clean_col_ptr[-1])
        offsets.append((n_off, s_off, k_off, c_off, e_off))
        parts["perm"].append(np.asarray(a.perm) + n_off)
        parts["sn_start"].append(np.asarray(a.sn_start) + n_off)
        parts["sn_end"].append(np.asarray(a.sn_end) + n_off)
        par = np.asarray(a.sn_parent).copy()
        par[par >= 0] += s_off
        parts["sn_parent"].append(par)
        cp = np.asarray(a.child_ptr)
        parts["child_ptr"].append(cp[:-1] + k_off)
        parts["child_idx"].append(np.asarray(a.child_idx) + s_off)
        frp = np.asarray(a.front_row_ptr)
        parts["front_row_ptr"].append(frp[:-1] + r_off)
        parts["front_row_idx"].append(np.asarray(a.front_row_idx) + n_off)
        parts["postorder"].append(np.asarray(a.postorder) + s_off)
        pcp = np.asarray(a.perm_col_ptr)
        parts["perm_col_ptr"].append(pcp[:-1] + c_off)
        parts["perm_row_idx"].append(np.asarray(a.perm_row_idx) + n_off)
        o2c = np.asarray(a.orig_to_clean).copy()
        o2c[o2c >= 0] += e_off
        parts["orig_to_clean"].append(o2c)
        parts["clean_to_perm"].append(np.asarray(a.clean_to_perm) + c_off)
        ccp = np.asarray(a.clean_col_ptr)
        parts["clean_col_ptr"].append(ccp[:-1] + e_off)
        parts["clean_row_idx"].append(np.asarray(a.clean_row_idx) + n_off)
        n_off += n
        s_off += ns
        k_off += int(cp[-1])
        c_off += nnz_perm
        e_off += nnz_clean
        r_off += int(frp[-1])
    arrays = {}
    for k, v in parts.items():
        arr = np.concatenate(v).astype(np.int32) if v else np.zeros(0, np.int32)
        arrays[k] = arr
    # closing entries of the pointer arrays
    arrays["child_ptr"] = np.append(arrays["child_ptr"], k_off).astype(np.int32)
    arrays["front_row_ptr"] = np.append(arrays["front_row_ptr"], len(arrays["front_row_idx"])).astype(np.int32)
    arrays["perm_col_ptr"] = np.append(arrays["perm_col_ptr"], c_off).astype(np.int32)
    arrays["clean_col_ptr"] = np.append(arrays["clean_col_ptr"], e_off).astype(np.int32)
    merged = smfg.Analysis(n_off, arrays, sum(getattr(a, "flops", 0.0) for a in analyses),
                           sum(getattr(a, "factor_entries", 0) for a in analyses))
    return merged, offsets


class BatchSolver:
    """Factor and solve many independent systems together on one GPU."""

    def __init__(self, analyses, device: int = -1):
        self.analyses = list(analyses)
        self.merged, self.offsets = merge_analyses(self.analyses)
        self.sizes = [int(a.n) for a in self.analyses]
        self.nnz_in = [int(np.asarray(a.orig_to_clean).size) for a in self.analyses]
        self.sn_counts = [int(a.nsn) for a in self.analyses]
        self.solver = smfg.Solver(self.merged, device=device)
        self.n = self.merged.n

    def close(self):
        self.solver.close()

    def factor(self, values, posdef: bool = False, **kw):
        """values: one array per system (the caller's entry order), or the
        concatenation (numpy, or a CUDA tensor already in device memory)."""
        if isinstance(values, (list, tuple)):
            values = np.concatenate([np.asarray(v, dtype=np.float64) for v in values])
        return self.solver.factor(values, posdef=posdef, **kw)

    def solve(self, b):
        """b: (nrhs, n_total) stacked right-hand sides (or a CUDA tensor)."""
        return self.solver.solve(b)

    def system_stats(self):
        """Per system: (pos, neg, zero, 2x2 pivots, delays)."""
        st = self.solver.front_stats()
        out = []
        s0 = 0
        for ns in self.sn_counts:
            blk = st[s0:s0 + ns]
            out.append(tuple(int(x) for x in blk.sum(axis=0)))
            s0 += ns
        return out

    def stack_rhs(self, rhs_list):
        """Per-system (nrhs, n_i) right-hand sides -> (nrhs, n_total)."""
        return np.ascontiguousarray(np.concatenate([np.atleast_2d(r) for r in rhs_list], axis=1))

    def split(self, x):
        """(nrhs, n_total) -> per-system (nrhs, n_i) blocks."""
        out, o = [], 0
        for n in self.sizes:
            out.append(x[..., o:o + n])
            o += n
        return out


def shard(count: int, rank: int, world: int):
    """This rank's contiguous slice [lo, hi) of `count` independent systems
    (configuration 4 on N GPUs: no data-path collective)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank / world")
    return rank * count // world, (rank + 1) * count // world


def gather_system_stats(local_stats, lo: int, count: int, world: int):
    """Every rank's per-system (pos, neg, zero, 2x2, delays) rows gathered in
    system order over torch.distributed (any backend). Returns the
    (count, 5) array on every rank; raises if the slices do not tile
    [0, count)."""
    import torch
    import torch.distributed as dist
    mine = (int(lo), [tuple(int(v) for v in r) for r in local_stats])
    if world == 1:
        parts = [mine]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, mine)
    parts.sort(key=lambda p: p[0])
    out, nxt = [], 0
    for lo_r, rows in parts:
        if lo_r != nxt:
            raise RuntimeError(f"system slices do not tile: expected {nxt}, got {lo_r}")
        out.extend(rows)
        nxt += len(rows)
    if nxt != count:
        raise RuntimeError(f"{nxt} of {count} systems gathered")
    del torch
    return np.asarray(out, dtype=np.int64).reshape(count, 5)
