"""Records of smf's own analysis of the benchmark workloads, made by the
reference (built from its sources in oracle/_ref): the fill-reducing
permutation and the supernode partition (first columns, parents; supernodes
in postorder). opt_solver_b200.smf_analysis rebuilds every AnalysisKeep array
the numeric phase reads from them; this script checks that the rebuilt
arrays equal the reference's before writing. Regenerate with

    python tests/golden/make_smf_partitions.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from opt_solver_b200 import smf_analysis as SA  # noqa: E402
from opt_solver_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

# name: (generator, posdef, ordering): configuration 2 (METIS), configuration
# 3 at full size and at the size the reference factors (METIS), configuration 1
# (AMD: the reference's own minimum degree, SuiteSparse AMD being absent)
CASES = {
    "spd3d64": (lambda: W.varcoef_3d(64, seed=0), True, O.ORDER_METIS),
    "kkt40_32000": (lambda: W.kkt_ipm(40, 32000, seed=0), False, O.ORDER_METIS),
    "kkt20_4000": (lambda: W.kkt_ipm(20, 4000, seed=0), False, O.ORDER_METIS),
    "lap2d150": (lambda: W.laplacian_2d(150), True, O.ORDER_AMD),
}
FIELDS = ["perm", "sn_start", "sn_end", "sn_parent", "child_ptr", "child_idx", "front_row_ptr", "front_row_idx",
          "postorder", "perm_col_ptr", "perm_row_idx", "clean_to_perm", "orig_to_clean", "clean_col_ptr",
          "clean_row_idx"]


def record(a):
    assert np.array_equal(a.postorder, np.arange(a.nsn)), "supernodes not numbered in postorder"
    assert np.array_equal(a.sn_end[:-1], a.sn_start[1:]) and a.sn_start[0] == 0 and a.sn_end[-1] == a.n
    first = np.append(a.sn_start, a.n).astype(np.int32)
    return {"perm": np.asarray(a.perm, dtype=np.int32), "sn_first": first,
            "sn_parent": np.asarray(a.sn_parent, dtype=np.int32)}


def main():
    for name, (build, posdef, ordering) in CASES.items():
        n, cp, ri, v = build()
        ref = O.Reference(posdef, ordering=ordering, scaling=O.SCALE_NONE)
        a = ref.analyse(n, cp, ri, v)
        rec = record(a)
        b = SA.from_partition(n, cp, ri, rec["perm"], rec["sn_first"], rec["sn_parent"])
        for k in FIELDS:
            assert np.array_equal(np.asarray(getattr(a, k)), getattr(b, k)), (name, k)
        np.savez_compressed(os.path.join(HERE, f"{name}_smf_partition.npz"), **rec)
        fr = np.diff(a.front_row_ptr)
        print(name, "n", n, "supernodes", a.nsn, "max front", int(fr.max()), "factor entries",
              int(np.sum(fr.astype(np.int64) * (a.sn_end - a.sn_start))))


if __name__ == "__main__":
    main()
