"""smf's analysis rebuilt from its record (opt_solver_b200.smf_analysis):
the permutation and the supernode partition give back every AnalysisKeep
array the numeric phase reads (solver/include/smf/analysis.hpp:25-144),
equal to the reference's own; and the committed records of the benchmark
workloads rebuild into analyses of the sizes the reference reported."""
import os

import numpy as np
import pytest

from opt_solver_b200 import smf_analysis as SA
from opt_solver_b200 import workloads as W
from tests.golden.make_smf_partitions import FIELDS, record

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name,build,posdef,order", [
    ("kkt_10_700", lambda: W.kkt_ipm(10, 700, seed=6), False, "metis"),
    ("var3d_16", lambda: W.varcoef_3d(16, seed=2), True, "metis"),
    ("lap2d_40", lambda: W.laplacian_2d(40), True, "amd"),
    ("traj_T30", lambda: W.trajectory_kkt(30, np.random.default_rng(1)), False, "amd"),
])
def test_rebuilt_analysis_equals_the_reference(name, build, posdef, order, ref_lib):
    O = ref_lib
    n, cp, ri, v = build()
    ref = O.Reference(posdef, ordering={"metis": O.ORDER_METIS, "amd": O.ORDER_AMD}[order],
                      scaling=O.SCALE_NONE)
    a = ref.analyse(n, cp, ri, v)
    rec = record(a)
    b = SA.from_partition(n, cp, ri, rec["perm"], rec["sn_first"], rec["sn_parent"])
    for k in FIELDS:
        assert np.array_equal(np.asarray(getattr(a, k)), getattr(b, k)), k


@pytest.mark.parametrize("rec,build,nsn,maxf,entries", [
    ("spd3d64", lambda: W.varcoef_3d(64, seed=0), 96633, 5854, 128998326),
    ("kkt40_32000", lambda: W.kkt_ipm(40, 32000, seed=0), 33177, 32150, 978793844),
    ("kkt20_4000", lambda: W.kkt_ipm(20, 4000, seed=0), 4159, 4071, 16330416),
    ("lap2d150", lambda: W.laplacian_2d(150), 4135, 307, 842868),
])
def test_committed_records(rec, build, nsn, maxf, entries):
    """The records rebuild into the analyses the reference reported when it
    made them (supernodes, largest front, factor entries sum f * p)."""
    n, cp, ri, v = build()
    a = SA.load(os.path.join(GOLDEN, f"{rec}_smf_partition.npz"), n, cp, ri)
    fr = np.diff(a.front_row_ptr).astype(np.int64)
    assert a.nsn == nsn and int(fr.max()) == maxf
    assert int(np.sum(fr * (a.sn_end - a.sn_start))) == entries
    assert np.array_equal(np.sort(a.perm), np.arange(n))


def test_rejects_inputs_that_need_cleaning():
    n, cp, ri, v = W.laplacian_2d(4)
    perm = np.arange(n)
    first = np.array([0, n])
    parent = np.array([-1])
    bad = ri.copy()
    bad[1] = 0  # column 0 holds its diagonal twice: a duplicate
    with pytest.raises(ValueError):
        SA.from_partition(n, cp, bad, perm, first, parent)
