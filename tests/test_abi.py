"""The C ABI without a GPU: libsmfg.so loads, exports every entry point that
include/smfg.h declares, fills smf's Control defaults, rejects bad
arguments before touching a device (smf_c.h's SMF_ERR_INVALID_ARG), and its
host-side symbolic analysis (smfg_analyse*) honours the smfg_analysis_t
contract the numeric phase reads (AnalysisKeep, solver/include/smf/
analysis.hpp:25-144)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from opt_solver_b200 import smfg as S
from opt_solver_b200 import workloads as W

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "smfg.h")


def _header():
    with open(HEADER) as f:
        return f.read()


def _declared():
    src = re.sub(r"/\*.*?\*/", "", _header(), flags=re.S)
    return sorted(set(re.findall(r"SMFG_API\s+[\w\s\*]*?\b(smfg_\w+)\s*\(", src)))


def _macro(name):
    m = re.search(rf"#define\s+{name}\s+(-?\d+)", _header())
    assert m, name
    return int(m.group(1))


def test_every_declared_entry_point_is_exported():
    names = _declared()
    assert len(names) >= 30, names
    S.lib()  # builds the library when its sources are newer
    lib = C.CDLL(S.library_path())
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_defaults_and_error_strings():
    L = S.lib()
    assert L.smfg_abi_version() == _macro("SMFG_ABI_VERSION")
    c = S.Control()
    L.smfg_default_control(C.byref(c))
    assert c.abi_version == _macro("SMFG_ABI_VERSION")
    # smf's Control defaults (solver/include/smf/control.hpp:331-332, 398, 440)
    assert c.u == 0.01 and c.small_pivot == 1e-20 and c.nb == 16
    assert c.max_negative_pivots == -1 and c.posdef == 0
    assert c.precision == _macro("SMFG_PREC_FP64") and not c.scale
    # the status codes smf_c.h names keep its numbers (0..5)
    for name, code in (("SMFG_OK", 0), ("SMFG_ERR_INVALID_ARG", 1), ("SMFG_ERR_SINGULAR", 2),
                       ("SMFG_ERR_INTERNAL", 3), ("SMFG_ERR_WRONG_INERTIA", 4),
                       ("SMFG_ERR_INEXACT_INERTIA", 5)):
        assert _macro(name) == code
    for code in (0, 1, 2, 3, 4, 5, 10, 11, 12, 13, 14):
        s = L.smfg_error_string(code)
        assert s and s != b"unknown error", code
    assert L.smfg_error_string(999) == b"unknown error"


def test_bad_arguments_are_rejected_before_the_device():
    L = S.lib()
    bad = _macro("SMFG_ERR_INVALID_ARG")
    x = np.zeros(4)
    i = C.c_int()
    h = C.c_void_p()
    assert L.smfg_plan_create(None, 0, C.byref(h)) == bad
    assert L.smfg_factor(None, x.ctypes.data, None, None) == bad
    assert L.smfg_solve(None, x.ctypes.data, 1, 4, 0, None) == bad
    assert L.smfg_inertia(None, C.byref(i), C.byref(i), C.byref(i)) == bad
    assert L.smfg_residual(None, x, x, 1, None, None, None) == bad
    assert L.smfg_refine_method(None, x, x, 1, 0, 5, 0, 1e-12, None, None, None) == bad
    assert L.smfg_last_times(None, None, None, None) == bad
    assert L.smfg_set_panel_teams(None, None) == bad
    assert L.smfg_set_front_precision(None, None) == bad
    assert L.smfg_tc_update(None, 1, 1, None, 1, None, 1, 1, 0) == bad
    L.smfg_plan_destroy(None)  # a null handle is ignored
    null = C.c_void_p()
    L.smfg_plan_destroy(C.byref(null))


def _check_analysis(n, cp, ri, a):
    perm = a.perm
    assert np.array_equal(np.sort(perm), np.arange(n))
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    nsn = a.nsn
    st, en, par = a.sn_start, a.sn_end, a.sn_parent
    # supernodes tile the new numbering in postorder
    assert st[0] == 0 and en[-1] == n
    assert np.all(en > st) and np.array_equal(st[1:], en[:-1])
    assert np.all((par == -1) | (par > np.arange(nsn)))
    assert np.array_equal(np.sort(a.postorder), np.arange(nsn))
    # children lists: exactly the supernodes naming s as parent, descending
    for s in range(nsn):
        ch = a.child_idx[a.child_ptr[s]:a.child_ptr[s + 1]]
        assert np.array_equal(ch, np.sort(np.nonzero(par == s)[0])[::-1]), s
    # front rows: sorted, pivots first, rows below the pivots after them
    rows_of = []
    for s in range(nsn):
        rows = a.front_row_idx[a.front_row_ptr[s]:a.front_row_ptr[s + 1]]
        p = en[s] - st[s]
        assert np.all(np.diff(rows) > 0), s
        assert np.array_equal(rows[:p], np.arange(st[s], en[s])), s
        rows_of.append(rows)
    # the permuted lower pattern lies inside each column's front, and a
    # child's update rows inside its parent's front (extend-add closes)
    sn_of = np.repeat(np.arange(nsn), en - st)
    pcp, pri = a.perm_col_ptr, a.perm_row_idx
    for j in range(n):
        col = pri[pcp[j]:pcp[j + 1]]
        assert np.all(col >= j), j
        assert np.all(np.isin(col, rows_of[sn_of[j]])), j
    for s in range(nsn):
        if par[s] >= 0:
            upd = rows_of[s][en[s] - st[s]:]
            assert np.all(np.isin(upd, rows_of[par[s]])), s
    # value placement: every kept input entry reaches the permuted slot of
    # its (row, column) pair in the new numbering
    cols = np.repeat(np.arange(n), np.diff(cp))
    o2c = a.orig_to_clean
    assert o2c.size == ri.size
    assert np.all((o2c >= -1) & (o2c < a.clean_col_ptr[-1]))
    ccols = np.repeat(np.arange(n), np.diff(a.clean_col_ptr))
    crows = a.clean_row_idx
    pcols = np.repeat(np.arange(n), np.diff(pcp))
    slot = a.clean_to_perm
    assert np.array_equal(np.sort(slot), np.arange(pri.size))
    r_new, c_new = inv[crows], inv[ccols]
    lo, hi = np.minimum(r_new, c_new), np.maximum(r_new, c_new)
    assert np.array_equal(pcols[slot], lo) and np.array_equal(pri[slot], hi)
    kept = o2c >= 0
    ka, kb = np.minimum(ri[kept], cols[kept]), np.maximum(ri[kept], cols[kept])
    ca, cb = np.minimum(crows, ccols)[o2c[kept]], np.maximum(crows, ccols)[o2c[kept]]
    assert np.array_equal(ka, ca) and np.array_equal(kb, cb)
    assert a.flops > 0 and a.factor_entries >= n


@pytest.mark.parametrize("gen", [
    lambda: W.laplacian_2d(14, 9),
    lambda: W.varcoef_3d(6, seed=1),
    lambda: W.trajectory_kkt(12, np.random.default_rng(3)),
    lambda: W.kkt_ipm(4, 30, seed=2),
], ids=["lap2d", "var3d", "traj", "kkt"])
def test_engine_analysis_contract(gen):
    n, cp, ri, v = gen()
    for ordering in (S.ORDER_ND, S.ORDER_NATURAL):
        _check_analysis(n, cp, ri, S.analyse(n, cp, ri, ordering=ordering))
    # a caller-given ordering is kept up to the postorder of its elimination
    # tree, which changes neither the fill nor the flops: analysing again on
    # the ordering it returns gives the same counts
    perm = np.random.default_rng(7).permutation(n)
    a = S.analyse(n, cp, ri, perm=perm)
    _check_analysis(n, cp, ri, a)
    b = S.analyse(n, cp, ri, perm=a.perm)
    _check_analysis(n, cp, ri, b)
    assert (b.factor_entries, b.flops) == (a.factor_entries, a.flops)


def test_engine_analysis_rejects_a_bad_ordering():
    n, cp, ri, v = W.laplacian_2d(5, 5)
    perm = np.arange(n)
    perm[3] = perm[4]
    with pytest.raises(S.SmfgError) as e:
        S.analyse(n, cp, ri, perm=perm)
    assert e.value.code == _macro("SMFG_ERR_INVALID_ARG")


_C_CALLER = r"""
#include "smfg.h"
int main(void) {
  smfg_control_t c;
  smfg_default_control(&c);
  return (smfg_abi_version() == SMFG_ABI_VERSION && c.abi_version == SMFG_ABI_VERSION && c.nb == 16) ? 0 : 1;
}
"""


@pytest.mark.parametrize("compiler,flags", [("gcc", ["-std=c99", "-pedantic"]),
                                            ("g++", ["-std=c++17", "-x", "c++"])])
def test_header_is_plain_c_and_cpp(compiler, flags, tmp_path):
    """A C or C++ caller (smf's own code, or a plugin in C) includes the
    header warning-free and links against the library; the two calls that
    need no device run."""
    import shutil
    import subprocess
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not installed")
    S.lib()
    src = tmp_path / "caller.c"
    src.write_text(_C_CALLER)
    exe = tmp_path / f"caller_{compiler}"
    libdir = os.path.dirname(S.library_path())
    subprocess.run([compiler, *flags, "-Wall", "-Wextra", "-Werror", "-I", os.path.dirname(HEADER),
                    str(src), "-L", libdir, "-lsmfg", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                   check=True, capture_output=True)
    assert subprocess.run([str(exe)]).returncode == 0


def _planless_solver(n=8, device=0):
    """A Solver object without a device plan: enough to exercise the
    argument checks that run before the library is called."""
    sv = S.Solver.__new__(S.Solver)
    sv.n, sv.device, sv._h = n, device, None
    return sv


def test_residual_noalloc_checks_buffers_before_the_library():
    """residual_noalloc passes raw device pointers to kernels that read and
    write n * nrhs doubles: every buffer must be float64, contiguous, of
    d_b's shape and on the plan's device, else ValueError before any call."""
    import torch
    sv = _planless_solver(n=8)
    good = torch.zeros(8, dtype=torch.float64)
    cases = [
        (torch.zeros(8, dtype=torch.float32), good, None, "float64"),
        (good, torch.zeros(8, dtype=torch.float32), None, "float64"),
        (torch.zeros(2, 16, dtype=torch.float64)[:, ::2], torch.zeros(2, 8, dtype=torch.float64), None,
         "contiguous"),
        (torch.zeros(16, 2, dtype=torch.float64).t()[:, :8], torch.zeros(2, 8, dtype=torch.float64),
         None, "contiguous"),
        (good, torch.zeros(7, dtype=torch.float64), None, "shape"),
        (torch.zeros(7, dtype=torch.float64), good, None, "shape"),
        (good, good, torch.zeros(2, 8, dtype=torch.float64), "shape"),
        (good, good, None, "cuda:0"),
    ]
    for d_b, d_x, d_r, what in cases:
        with pytest.raises(ValueError, match=what):
            sv.residual_noalloc(d_b, d_x, d_r)
