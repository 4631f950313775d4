"""Fill-reducing orderings of the interior-point KKT workloads from smf's own
analysis (METIS nested dissection; the reference built from its sources in
oracle/_ref). The engine takes smf's analysis output as is; these committed
permutations stand in for that analysis where the reference is not at hand
(bench.py's KKT workloads). Regenerate with

    python tests/golden/make_kkt_orderings.py

Each file holds perm[new] = old (int32) for workloads.kkt_ipm(m, n_con,
seed=0).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from opt_solver_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {"kkt40_32000": (40, 32000), "kkt20_4000": (20, 4000)}


def main():
    for name, (m, ncon) in CASES.items():
        n, cp, ri, v = W.kkt_ipm(m, ncon, seed=0)
        ref = O.Reference(False, ordering=O.ORDER_METIS, scaling=O.SCALE_NONE)
        a = ref.analyse(n, cp, ri, v)
        perm = np.asarray(a.perm, dtype=np.int32)
        assert np.array_equal(np.sort(perm), np.arange(n))
        np.savez_compressed(os.path.join(HERE, f"{name}_metis_perm.npz"), perm=perm)
        fr = np.diff(a.front_row_ptr)
        print(name, "n", n, "supernodes", a.nsn, "max front", int(fr.max()))


if __name__ == "__main__":
    main()
