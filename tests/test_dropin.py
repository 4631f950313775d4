"""The drop-in boundary end to end: smf's own C API (smf_c.h: smf_analyse,
smf_factor, smf_solve, smf_inertia) and its IPOPT plugin's MA97 interface
(smf_ma97_plugin.cpp: ma97_analyse_d, ma97_factor_d, ma97_solve_d), built
from smf's sources twice by oracle/Makefile's `dropin` target: as smf builds
them (libsmf_c_cpu.so) and with smf::Solver's factor and solve wrapped onto
the B200 engine (libsmf_c_gpu.so, opt_solver_b200/integration/
smf_gpu_hook.cpp). The caller's code is the same for both.

Bar: the GPU build's inertia, delays and 2x2 counts equal smf's own; its
solution equals the engine called directly on the same analysis bit for bit
(the same factor and solve), and smf's CPU solution within 1e-9 relative
(different solve arithmetic); the backward error is the plain path's.
"""
import ctypes as C
import os

import numpy as np
import pytest

from opt_solver_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
CPU_SO = os.path.join(REF, "libsmf_c_cpu.so")
GPU_SO = os.path.join(REF, "libsmf_c_gpu.so")


class Csc(C.Structure):
    _fields_ = [("n", C.c_int), ("col_ptr", C.c_void_p), ("row_idx", C.c_void_p), ("values", C.c_void_p)]


class Inertia(C.Structure):
    _fields_ = [("pos", C.c_int), ("neg", C.c_int), ("zero", C.c_int)]


class Ma97Control(C.Structure):
    _fields_ = [("f_arrays", C.c_int), ("action", C.c_int), ("nemin", C.c_int), ("multiplier", C.c_double),
                ("ordering", C.c_int), ("print_level", C.c_int), ("scaling", C.c_int), ("small", C.c_double),
                ("u", C.c_double), ("unit_diagnostics", C.c_int), ("unit_error", C.c_int),
                ("unit_warning", C.c_int), ("factor_min", C.c_long), ("solve_blas3", C.c_int),
                ("solve_min", C.c_int), ("solve_mf", C.c_int), ("consist_tol", C.c_double),
                ("ispare", C.c_int * 5), ("rspare", C.c_double * 10)]


class Ma97Info(C.Structure):
    _fields_ = [("flag", C.c_int), ("flag68", C.c_int), ("flag77", C.c_int), ("matrix_dup", C.c_int),
                ("matrix_rank", C.c_int), ("matrix_outrange", C.c_int), ("matrix_missing_diag", C.c_int),
                ("maxdepth", C.c_int), ("maxfront", C.c_int), ("num_delay", C.c_int), ("num_factor", C.c_long),
                ("num_flops", C.c_long), ("num_neg", C.c_int), ("num_sup", C.c_int), ("num_two", C.c_int),
                ("ordering", C.c_int), ("stat", C.c_int), ("maxsupernode", C.c_int), ("ispare", C.c_int * 4),
                ("rspare", C.c_double * 10)]


def _load(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, ROOT)} not built (make -C oracle dropin)")
    os.environ.setdefault("SMF_NUM_THREADS", "1")  # the plugin's thread count: one, as the parity mode
    L = C.CDLL(path)
    L.smf_analyse.argtypes = [C.POINTER(Csc), C.POINTER(C.c_void_p)]
    L.smf_factor.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
    L.smf_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    L.smf_inertia.argtypes = [C.c_void_p, C.POINTER(Inertia)]
    L.smf_free_analysis.argtypes = [C.POINTER(C.c_void_p)]
    L.smf_free_factor.argtypes = [C.POINTER(C.c_void_p)]
    L.ma97_default_control_d.argtypes = [C.POINTER(Ma97Control)]
    L.ma97_analyse_d.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p),
                                 C.POINTER(Ma97Control), C.POINTER(Ma97Info), C.c_void_p]
    L.ma97_factor_d.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p),
                                C.POINTER(C.c_void_p), C.POINTER(Ma97Control), C.POINTER(Ma97Info), C.c_void_p]
    L.ma97_solve_d.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                               C.POINTER(C.c_void_p), C.POINTER(Ma97Control), C.POINTER(Ma97Info)]
    L.ma97_finalise_d.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    return L


def _c_api(L, n, cp, ri, v, posdef, b):
    """smf_analyse, smf_factor, smf_inertia, smf_solve as a C caller makes them."""
    cp = np.ascontiguousarray(cp, dtype=np.int32)
    ri = np.ascontiguousarray(ri, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.float64)
    csc = Csc(n, cp.ctypes.data, ri.ctypes.data, v.ctypes.data)
    an, fa = C.c_void_p(), C.c_void_p()
    assert L.smf_analyse(C.byref(csc), C.byref(an)) == 0
    rc = L.smf_factor(an, v.ctypes.data, 0 if posdef else 1, C.byref(fa))
    assert rc == 0, rc
    inert = Inertia()
    assert L.smf_inertia(fa, C.byref(inert)) == 0
    x = np.array(b, dtype=np.float64, copy=True)
    assert L.smf_solve(an, fa, 1, x.ctypes.data, 0) == 0
    L.smf_free_factor(C.byref(fa))
    L.smf_free_analysis(C.byref(an))
    return (inert.pos, inert.neg, inert.zero), x


def _ma97(L, n, cp, ri, v, posdef, b):
    """The IPOPT plugin's MA97 calls: analyse, factor, solve, finalise."""
    cp = np.ascontiguousarray(cp, dtype=np.int32)
    ri = np.ascontiguousarray(ri, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.float64)
    ctrl, info = Ma97Control(), Ma97Info()
    L.ma97_default_control_d(C.byref(ctrl))
    ak, fk = C.c_void_p(), C.c_void_p()
    L.ma97_analyse_d(0, n, cp.ctypes.data, ri.ctypes.data, v.ctypes.data, C.byref(ak), C.byref(ctrl),
                     C.byref(info), None)
    assert info.flag >= 0, info.flag
    L.ma97_factor_d(3 if posdef else 4, cp.ctypes.data, ri.ctypes.data, v.ctypes.data, C.byref(ak), C.byref(fk),
                    C.byref(ctrl), C.byref(info), None)
    fac = dict(flag=info.flag, num_neg=info.num_neg, num_delay=info.num_delay, num_two=info.num_two,
               rank=info.matrix_rank)
    x = np.array(b, dtype=np.float64, copy=True)
    L.ma97_solve_d(0, 1, x.ctypes.data, n, C.byref(ak), C.byref(fk), C.byref(ctrl), C.byref(info))
    solve_flag = info.flag
    L.ma97_finalise_d(C.byref(ak), C.byref(fk))
    return fac, solve_flag, x


CASES = [
    ("kkt_6_100", lambda: W.kkt_ipm(6, 100, seed=3), False),
    ("traj_T40", lambda: W.trajectory_kkt(40, np.random.default_rng(7)), False),
    ("lap2d_30", lambda: W.laplacian_2d(30), True),
]


def test_dropin_libraries_export_the_interfaces():
    """Both builds load (the GPU one resolves libsmfg.so through its run
    path) and export smf's C API and the MA97 entry points."""
    for path in (CPU_SO, GPU_SO):
        L = _load(path)
        for name in ("smf_analyse", "smf_factor", "smf_solve", "smf_inertia", "ma97_analyse_d", "ma97_factor_d",
                     "ma97_solve_d", "ma97_finalise_d"):
            assert hasattr(L, name), (path, name)
    G = C.CDLL(GPU_SO)
    assert hasattr(G, "smf_gpu_hook_plans")


def test_dropin_cpu_build_solves(ref_lib):
    """The unmodified build through its C API: the harness the GPU build is
    compared with (smf's own results)."""
    O = ref_lib
    L = _load(CPU_SO)
    n, cp, ri, v = W.kkt_ipm(6, 100, seed=3)
    b = W.rhs(n, 1, seed=5)
    inert, x = _c_api(L, n, cp, ri, v, False, b)
    assert inert == (216, 100, 0)
    _, _, om = O.residual(n, cp, ri, v, b, x)
    assert om <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_dropin_c_api_on_gpu(case, ref_lib):
    O = ref_lib
    from opt_solver_b200.smfg import Solver
    name, build, posdef = case
    n, cp, ri, v = build()
    b = W.rhs(n, 1, seed=5)
    Lc, Lg = _load(CPU_SO), _load(GPU_SO)
    in_c, x_c = _c_api(Lc, n, cp, ri, v, posdef, b)
    in_g, x_g = _c_api(Lg, n, cp, ri, v, posdef, b)
    assert in_g == in_c
    assert np.max(np.abs(x_g - x_c)) <= 1e-9 * max(1.0, np.max(np.abs(x_c)))
    _, _, om = O.residual(n, cp, ri, v, b, x_g)
    _, _, om_c = O.residual(n, cp, ri, v, b, x_c)
    assert om <= max(1e-14, 10 * om_c), (om, om_c)
    # the engine called directly on smf_analyse's analysis (smf's default
    # Control: AutoSerial ordering, Auto scaling, one thread): bit for bit
    ref = O.Reference(posdef=False, ordering=O.ORDER_AUTO_SERIAL, scaling=O.SCALE_AUTO, deterministic=False,
                      num_threads=1, top_tiles=True)
    a = ref.analyse(n, cp, ri, v)
    scale = None if posdef or not len(a.matching_scale) else a.matching_scale
    sv = Solver(a)
    gi = sv.factor(v, posdef=posdef, scale=scale, aptp_min_rows=0)
    assert gi.factor_status == 0 and (posdef or gi.inertia == in_g)
    assert np.array_equal(sv.solve(b), x_g)
    sv.close()
    assert C.CDLL(GPU_SO).smf_gpu_hook_plans() >= 1


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_dropin_ma97_plugin_on_gpu(case, ref_lib):
    """IPOPT's MA97 calls into smf's plugin: the plugin's IpmSession factors
    and solves through the wrapped Solver, flags and counts as smf's own."""
    O = ref_lib
    name, build, posdef = case
    n, cp, ri, v = build()
    b = W.rhs(n, 1, seed=6)
    Lc, Lg = _load(CPU_SO), _load(GPU_SO)
    fc, sc, x_c = _ma97(Lc, n, cp, ri, v, posdef, b)
    fg, sg, x_g = _ma97(Lg, n, cp, ri, v, posdef, b)
    assert fg == fc, (fg, fc)
    assert sg == sc == 0
    assert np.max(np.abs(x_g - x_c)) <= 1e-9 * max(1.0, np.max(np.abs(x_c)))
    _, _, om = O.residual(n, cp, ri, v, b, x_g)
    _, _, om_c = O.residual(n, cp, ri, v, b, x_c)
    assert om <= max(1e-14, 10 * om_c), (om, om_c)
