"""Parity cases shared by the CPU and GPU tests: small instances of the
benchmark configurations plus the reference's own dense known-answer
matrices (solver/tests/test_ldlt_dense.cpp: SPD2x2, Indefinite3x3,
AllNegative2x2), each with the ordering / scaling the reference uses on it.
"""
from __future__ import annotations

import numpy as np

from opt_solver_b200 import workloads as W


def dense_lower(A):
    """Lower CSC of a dense symmetric matrix (explicit zeros kept)."""
    A = np.asarray(A, dtype=np.float64)
    n = A.shape[0]
    cp, ri, v = [0], [], []
    for j in range(n):
        for i in range(j, n):
            ri.append(i)
            v.append(A[i, j])
        cp.append(len(ri))
    return n, np.array(cp, dtype=np.int32), np.array(ri, dtype=np.int32), np.array(v)


# (name, builder, posdef, ordering name, scaling name, expected inertia or None)
def cases(size: str = "small"):
    out = [
        ("kat_spd2x2", lambda: dense_lower([[4, 2], [2, 3]]), True, "amd", "none", (2, 0, 0)),
        ("kat_indef3x3", lambda: dense_lower([[2, 1, 0], [1, 0, 1], [0, 1, 2]]), False, "amd", "none", (2, 1, 0)),
        ("kat_allneg2x2", lambda: dense_lower([[-4, -2], [-2, -3]]), False, "amd", "none", (0, 2, 0)),
        ("lap2d_30", lambda: W.laplacian_2d(30), True, "amd", "none", (900, 0, 0)),
        ("var3d_12", lambda: W.varcoef_3d(12, seed=1), True, "metis", "none", (1728, 0, 0)),
        ("traj_T40", lambda: W.trajectory_kkt(40, np.random.default_rng(7)), False, "amd", "none",
         (16 * 40 + 12, 12 * 40, 0)),
        ("kkt_6_100", lambda: W.kkt_ipm(6, 100, seed=3), False, "auto", "auto", (216, 100, 0)),
    ]
    if size in ("full", "large"):
        out += [
            # fronts above 384 rows: the multi-block large-front path
            ("var3d_24", lambda: W.varcoef_3d(24, seed=4), True, "metis", "none", (24 ** 3, 0, 0)),
            # large indefinite fronts with delays: a front of 977 rows takes
            # deterministic mode's APTP kernel, then the threshold kernel on
            # the 739 columns it fails
            ("kkt_10_700", lambda: W.kkt_ipm(10, 700, seed=6), False, "auto", "auto", (1000, 700, 0)),
        ]
    if size == "full":
        out += [
            ("lap2d_150", lambda: W.laplacian_2d(150), True, "amd", "none", (22500, 0, 0)),
            ("var3d_20", lambda: W.varcoef_3d(20, seed=2), True, "metis", "none", (8000, 0, 0)),
            ("traj_T200", lambda: W.trajectory_kkt(200, np.random.default_rng(11)), False, "amd", "none",
             (16 * 200 + 12, 12 * 200, 0)),
            ("kkt_8_256", lambda: W.kkt_ipm(8, 256, seed=5), False, "auto", "auto", (512, 256, 0)),
        ]
    return out


def reference_for(O, posdef, ordering, scaling, deterministic=True):
    """The reference configured as the parity oracle: deterministic mode, one
    thread (its indefinite fronts of >= 512 rows take the APTP kernel, as
    the engine's and the oracle's do by default). Ordering "auto1t":
    AutoParallel in the one-thread default mode instead, whose fronts keep
    the threshold kernel everywhere (the engine's and the oracle's
    aptp_min_rows = 0)."""
    if ordering == "auto1t":
        ordering, deterministic = "auto", False
    order = {"amd": O.ORDER_AMD, "metis": O.ORDER_METIS, "auto": O.ORDER_AUTO_PARALLEL}[ordering]
    scal = {"none": O.SCALE_NONE, "auto": O.SCALE_AUTO}[scaling]
    return O.Reference(posdef=posdef, ordering=order, scaling=scal, deterministic=deterministic,
                       num_threads=1, top_tiles=deterministic)
