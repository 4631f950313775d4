"""Golden fixtures of the numeric phase, made by the reference smf itself
(built from its sources into oracle/_ref, deterministic mode, one thread):
for each small case the analysis it produced (the AnalysisKeep arrays), the
values, the scaling it applied, its factor (per-front sizes, rows, pivot
tags, L / D blocks, inertia, delays, 2x2 pivots, flops) and its solution of
one right-hand side; for the cases with APTP fronts (deterministic mode's
kernel on indefinite fronts of >= 512 rows), digests of the factor instead
(the *_digest.npz files). The oracle and the CUDA engine are checked against
these files where the reference itself is not available. Regenerate with

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from opt_solver_b200 import workloads as W  # noqa: E402
from tests.cases import dense_lower, reference_for  # noqa: E402

ANALYSIS_FIELDS = ["perm", "sn_start", "sn_end", "sn_parent", "child_ptr", "child_idx", "front_row_ptr",
                   "front_row_idx", "postorder", "perm_col_ptr", "perm_row_idx", "clean_to_perm",
                   "orig_to_clean", "clean_col_ptr", "clean_row_idx"]


def saddle(nb=50, seed=3):
    """[[0, B^T], [B, 0]] with B = 4 I + small perturbation (the shape of the
    reference's SaddlePointUsesTwoByTwo case): inertia (nb, nb, 0), 2x2
    pivots only."""
    rng = np.random.default_rng(seed)
    B = 4.0 * np.eye(nb) + rng.uniform(-0.5, 0.5, (nb, nb)) / nb
    A = np.zeros((2 * nb, 2 * nb))
    A[nb:, :nb] = B
    A[:nb, nb:] = B.T
    return dense_lower(A)


CASES = [
    # name, builder, posdef, ordering, scaling
    ("lap2d_12", lambda: W.laplacian_2d(12), True, "amd", "none"),
    ("var3d_7", lambda: W.varcoef_3d(7, seed=9), True, "metis", "none"),
    ("traj_T12", lambda: W.trajectory_kkt(12, np.random.default_rng(5)), False, "amd", "none"),
    ("kkt_5_60", lambda: W.kkt_ipm(5, 60, seed=2), False, "auto", "auto"),
    ("saddle_50", saddle, False, "amd", "none"),
]


# Deterministic mode's APTP kernel (indefinite fronts of >= 512 rows): the
# factors are too large to store, so these fixtures keep the analysis, the
# values and a SHA-256 digest of each front's block (f x p, column-major
# float64 bytes), rows and tags.
DIGEST_CASES = [
    ("kkt_10_700", lambda: W.kkt_ipm(10, 700, seed=6), False, "auto", "auto"),
]


def block_digest(block):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(np.asarray(block, dtype=np.float64).T).tobytes()).hexdigest()


def dense_aptp_fronts():
    """Dense fronts for the APTP kernel alone: (name, A (f x f symmetric),
    eligible columns, u), seeded; many 2x2 pivots and failed columns."""
    rng = np.random.default_rng(2024)
    out = []
    A = rng.standard_normal((640, 640))
    out.append(("gauss_640", A + A.T, 560, 0.01))
    k = 300
    B = rng.standard_normal((k, 600 - k))
    S = np.zeros((600, 600))
    S[:k, k:] = B
    S[k:, :k] = B.T
    out.append(("saddle_600", S, 523, 0.01))
    T = rng.standard_normal((576, 576)) * 1e-3
    T = T + T.T
    T[np.diag_indices(576)] = rng.standard_normal(576) * 1e-6
    out.append(("tinydiag_576", T, 500, 0.1))
    return out


def dense_aptp_reference(A, ne, u):
    """The reference's APTP tile kernel on one dense front: (F, rows, tags,
    (eliminated, failed, pos, neg, zero))."""
    import ctypes as C
    f = A.shape[0]
    F = np.ascontiguousarray(np.tril(A).T).reshape(-1).copy()
    rows = np.arange(f, dtype=np.int32)
    tags = np.zeros(f, dtype=np.int8)
    out = np.zeros(5, dtype=np.int64)
    O.Reference.lib().refshim_aptp_front(F.ctypes.data_as(C.c_void_p), f, ne, rows.ctypes.data_as(C.c_void_p),
                                         C.c_double(u), C.c_double(1e-20), O.APTP_NB, O.APTP_IB, 1,
                                         tags.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
    return F.reshape(f, f).T, rows, tags, out


def main_digests():
    for name, build, posdef, ordering, scaling in DIGEST_CASES:
        n, cp, ri, v = build()
        ref = reference_for(O, posdef, ordering, scaling)
        a = ref.analyse(n, cp, ri, v)
        fx = ref.factor(v)
        out = {f"an_{k}": np.asarray(getattr(a, k), dtype=np.int32) for k in ANALYSIS_FIELDS}
        digests = [block_digest(fx.block(s)) for s in range(a.nsn)]
        out.update(
            n=np.int64(n), col_ptr=cp, row_idx=ri, values=v, posdef=np.int64(posdef),
            scale=np.asarray(fx.scale, dtype=np.float64), inertia=np.asarray(fx.inertia, dtype=np.int64),
            delayed=np.int64(fx.delayed), two_by_two=np.int64(fx.two_by_two), flops=np.float64(fx.flops),
            aptp_failed=np.int64(fx.aptp_failed), f=fx.f, p=fx.p, row_off=fx.row_off,
            rows=fx.rows[: int(np.sum(fx.f))],
            tags=np.zeros(0, np.int8) if fx.tags is None else fx.tags[: int(np.sum(fx.p))],
            block_sha256=np.array(digests))
        np.savez_compressed(os.path.join(HERE, f"{name}_digest.npz"), **out)
        print(name, "n", n, "supernodes", a.nsn, "fronts >= 512 rows", int(np.sum(fx.f >= 512)),
              "APTP failed columns", fx.aptp_failed)
    dense = {}
    for name, A, ne, u in dense_aptp_fronts():
        F, rows, tags, res = dense_aptp_reference(A, ne, u)
        dense[f"{name}_sha256"] = np.array(block_digest(np.tril(F)))
        dense[f"{name}_rows"] = rows
        dense[f"{name}_tags"] = tags
        dense[f"{name}_result"] = res
        print(name, "eliminated", res[0], "failed", res[1], "2x2", int(np.sum(tags == 2)))
    np.savez_compressed(os.path.join(HERE, "aptp_dense_digest.npz"), **dense)


def main():
    main_digests()
    for name, build, posdef, ordering, scaling in CASES:
        n, cp, ri, v = build()
        ref = reference_for(O, posdef, ordering, scaling)
        a = ref.analyse(n, cp, ri, v)
        fx = ref.factor(v)
        b = np.random.default_rng(17).uniform(-1.0, 1.0, n)
        xr, _ = ref.solve(b)
        out = {f"an_{k}": np.asarray(getattr(a, k), dtype=np.int32) for k in ANALYSIS_FIELDS}
        out.update(
            n=np.int64(n), col_ptr=cp, row_idx=ri, values=v, posdef=np.int64(posdef),
            scale=np.asarray(fx.scale, dtype=np.float64), inertia=np.asarray(fx.inertia, dtype=np.int64),
            delayed=np.int64(fx.delayed), two_by_two=np.int64(fx.two_by_two), flops=np.float64(fx.flops),
            f=fx.f, p=fx.p, blk_off=fx.blk_off, blocks=fx.blocks[: int(np.sum(fx.f.astype(np.int64) * fx.p))],
            row_off=fx.row_off, rows=fx.rows[: int(np.sum(fx.f))],
            tags=np.zeros(0, np.int8) if fx.tags is None else fx.tags[: int(np.sum(fx.p))],
            b=b, x=xr)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, "n", n, "supernodes", a.nsn, "inertia", fx.inertia, "delays", fx.delayed,
              "2x2", fx.two_by_two)


if __name__ == "__main__":
    main()
