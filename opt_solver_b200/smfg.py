"""Python host of the B200 numeric phase, over the C ABI of libsmfg.so
(include/smfg.h).

It mirrors smf's numeric API (solver/include/smf/solver.hpp:33-140): a
``Solver`` is created from an analysis (the AnalysisKeep arrays of
solver/include/smf/analysis.hpp:25-144), then ``factor`` / ``solve`` /
``inertia`` / ``refine`` follow ``Solver::factor``, ``Solver::solve``,
``smf_inertia`` and ``refine``. There is no CPU fallback: without the
CUDA library or a GPU every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

SMFG_OK = 0
SMFG_ERR_SINGULAR = 2
SMFG_ERR_WRONG_INERTIA = 4
# smfg_info_t.factor_status
SMFG_FACTOR_SUCCESS, SMFG_FACTOR_NOT_POSDEF, SMFG_FACTOR_SINGULAR = 0, 1, 2
SMFG_FACTOR_MAX_PIVOT_DELAYS, SMFG_FACTOR_INERTIA_EXCEEDED = 3, 4
SOLVE_FULL, SOLVE_FORWARD, SOLVE_DIAGONAL, SOLVE_BACKWARD = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1
# indefinite fronts of at least this many rows take the APTP kernel (smf's
# deterministic mode, kTopTileMinFront)
APTP_MIN_ROWS = 512
NOALLOC_MAX_N = 262144  # SMFG_NOALLOC_MAX_N

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


class SmfgError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        detail = ""
        try:
            detail = lib().smfg_last_error().decode()
        except Exception:  # noqa: BLE001
            pass
        super().__init__(f"{where}: {error_string(code)} ({code}){': ' + detail if detail else ''}")


class _Analysis(C.Structure):
    _fields_ = [("n", C.c_int), ("nsn", C.c_int)] + [
        (nm, C.c_void_p) for nm in ("perm", "sn_start", "sn_end", "sn_parent", "child_ptr",
                                    "child_idx", "front_row_ptr", "front_row_idx", "postorder",
                                    "perm_col_ptr", "perm_row_idx")] + [
        ("nnz_in", C.c_int64)] + [
        (nm, C.c_void_p) for nm in ("orig_to_clean", "clean_to_perm", "clean_col_ptr",
                                    "clean_row_idx")]


class Control(C.Structure):
    """smfg_control_t (include/smfg.h)."""
    _fields_ = [("abi_version", C.c_int), ("posdef", C.c_int), ("u", C.c_double),
                ("small_pivot", C.c_double), ("nb", C.c_int), ("blocked_min_front", C.c_int),
                ("precision", C.c_int), ("max_negative_pivots", C.c_int),
                ("scale", C.c_void_p), ("profile", C.c_int), ("mixed_block", C.c_int),
                ("mixed_kind", C.c_int), ("mixed_min_front", C.c_int), ("panel_team", C.c_int),
                ("graph", C.c_int), ("aptp_min_rows", C.c_int), ("reserved_i", C.c_int * 1),
                ("work_limit", C.c_double), ("reserved_d", C.c_double * 7)]


class Info(C.Structure):
    """smfg_info_t (include/smfg.h)."""
    _fields_ = [("status", C.c_int), ("factor_status", C.c_int), ("num_pos", C.c_int),
                ("num_neg", C.c_int), ("num_zero", C.c_int), ("delayed_pivots", C.c_int),
                ("two_by_two_pivots", C.c_int), ("max_front", C.c_int),
                ("factor_entries", C.c_int64), ("flops", C.c_double), ("max_abs", C.c_double),
                ("factor_ms", C.c_double), ("solve_ms", C.c_double), ("levels", C.c_int),
                ("kernel_launches", C.c_int), ("mixed_fronts", C.c_int),
                ("reserved_i", C.c_int * 7), ("reserved_d", C.c_double * 8)]

    @property
    def inertia(self):
        return (self.num_pos, self.num_neg, self.num_zero)

    @property
    def aptp_failed(self):
        """Columns the APTP sweeps failed (smf's Info::aptp_failed_columns)."""
        return self.reserved_i[4]

    @property
    def aptp_fronts(self):
        return self.reserved_i[5]


_lib = None


def library_path() -> str:
    return _build.LIB


def lib():
    """Load libsmfg.so (building it first when the sources are newer)."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path) or _build.needs_build():
            _build.build()
        L = C.CDLL(path)
        L.smfg_abi_version.restype = C.c_int
        L.smfg_default_control.argtypes = [C.POINTER(Control)]
        L.smfg_plan_create.argtypes = [C.POINTER(_Analysis), C.c_int, C.POINTER(C.c_void_p)]
        L.smfg_plan_create.restype = C.c_int
        L.smfg_plan_destroy.argtypes = [C.POINTER(C.c_void_p)]
        L.smfg_factor.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Control), C.POINTER(Info)]
        L.smfg_factor.restype = C.c_int
        L.smfg_factor_device.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Control), C.POINTER(Info)]
        L.smfg_factor_device.restype = C.c_int
        L.smfg_solve.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(Info)]
        L.smfg_solve.restype = C.c_int
        L.smfg_solve_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(Info)]
        L.smfg_solve_device.restype = C.c_int
        L.smfg_inertia.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]
        L.smfg_inertia.restype = C.c_int
        L.smfg_factor_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.smfg_factor_sizes.restype = C.c_int
        L.smfg_factor_export.argtypes = [C.c_void_p, _i32p, _i32p, _i64p, _f64p, _i64p, _i32p,
                                         C.c_void_p]
        L.smfg_factor_export.restype = C.c_int
        L.smfg_residual.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int, C.c_void_p,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.smfg_residual.restype = C.c_int
        L.smfg_refine.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int, C.c_int, C.c_double,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.smfg_refine.restype = C.c_int
        L.smfg_residual_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.smfg_residual_noalloc.restype = C.c_int
        L.smfg_refine_method.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_int)]
        L.smfg_refine_method.restype = C.c_int
        L.smfg_refine_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_double, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.smfg_refine_device.restype = C.c_int
        L.smfg_last_times.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]
        L.smfg_last_times.restype = C.c_int
        L.smfg_set_panel_teams.argtypes = [C.c_void_p, C.c_void_p]
        L.smfg_set_panel_teams.restype = C.c_int
        L.smfg_set_front_precision.argtypes = [C.c_void_p, C.c_void_p]
        L.smfg_set_front_precision.restype = C.c_int
        L.smfg_front_stats.argtypes = [C.c_void_p, _i32p]
        L.smfg_front_stats.restype = C.c_int
        L.smfg_error_string.argtypes = [C.c_int]
        L.smfg_error_string.restype = C.c_char_p
        L.smfg_last_error.argtypes = []
        L.smfg_last_error.restype = C.c_char_p
        L.smfg_analyse.argtypes = [C.c_int, _i32p, _i32p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
        L.smfg_analyse.restype = C.c_int
        L.smfg_analyse_ordered.argtypes = [C.c_int, _i32p, _i32p, _i32p, C.c_int,
                                           C.POINTER(C.c_void_p)]
        L.smfg_analyse_ordered.restype = C.c_int
        L.smfg_symbolic_view.argtypes = [C.c_void_p, C.POINTER(_Analysis), C.POINTER(C.c_double),
                                         C.POINTER(C.c_int64)]
        L.smfg_symbolic_view.restype = C.c_int
        L.smfg_symbolic_free.argtypes = [C.POINTER(C.c_void_p)]
        L.smfg_mlp_params.argtypes = [C.c_int, C.c_int]
        L.smfg_mlp_params.restype = C.c_int
        L.smfg_mlp_forward.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        L.smfg_mlp_forward.restype = C.c_int
        L.smfg_mlp_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                        C.c_void_p, C.c_void_p]
        L.smfg_mlp_backward.restype = C.c_int
        L.smfg_mlp_adam.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                    C.c_float, C.c_float, C.c_float, C.c_int]
        L.smfg_mlp_adam.restype = C.c_int
        L.smfg_matching_scale.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, C.POINTER(C.c_int)]
        L.smfg_matching_scale.restype = C.c_int
        L.smfg_tc_update.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_int, C.c_int, C.c_int]
        L.smfg_tc_update.restype = C.c_int
        _lib = L
    return _lib


def error_string(code: int) -> str:
    try:
        return lib().smfg_error_string(code).decode()
    except Exception:  # noqa: BLE001
        return "error"


def default_control(posdef: bool = False, u: float = 0.01, small: float = 1e-20,
                    precision: int = PREC_FP64, max_negative_pivots: int = -1) -> Control:
    c = Control()
    lib().smfg_default_control(C.byref(c))
    c.posdef = int(posdef)
    c.u = u
    c.small_pivot = small
    c.precision = precision
    c.max_negative_pivots = max_negative_pivots
    return c


@dataclass
class FrontFactor:
    """Per-front export of a factor (the FactorKeep layout)."""
    f: np.ndarray
    p: np.ndarray
    blk_off: np.ndarray
    blocks: np.ndarray
    row_off: np.ndarray
    rows: np.ndarray
    tags: np.ndarray | None

    def block(self, s: int) -> np.ndarray:
        f, p = int(self.f[s]), int(self.p[s])
        o = int(self.blk_off[s])
        return self.blocks[o:o + f * p].reshape(p, f).T

    def front_rows(self, s: int) -> np.ndarray:
        o = int(self.row_off[s])
        return self.rows[o:o + int(self.f[s])]


_ANALYSIS_FIELDS = ("perm", "sn_start", "sn_end", "sn_parent", "child_ptr", "child_idx",
                    "front_row_ptr", "front_row_idx", "postorder", "perm_col_ptr",
                    "perm_row_idx", "orig_to_clean", "clean_to_perm", "clean_col_ptr",
                    "clean_row_idx")

ORDER_ND, ORDER_NATURAL, ORDER_ND_FINE = 0, 1, 2


class Analysis:
    """AnalysisKeep arrays (numpy int32) with smf's conventions; from
    ``analyse`` below or from smf's own analyse."""

    def __init__(self, n, arrays, flops=0.0, factor_entries=0):
        self.n = int(n)
        for k, v in arrays.items():
            setattr(self, k, v)
        self.flops = flops
        self.factor_entries = factor_entries

    @property
    def nsn(self) -> int:
        return int(self.sn_start.size)


def analyse(n, col_ptr, row_idx, ordering: int = ORDER_ND, nemin: int = 8,
            perm=None) -> Analysis:
    """Symbolic analysis of a lower CSC pattern (smfg_analyse: the engine's
    own nested-dissection analysis, host code). perm (perm[new] = old): a
    caller-given fill-reducing ordering instead (smfg_analyse_ordered)."""
    L = lib()
    cp = np.ascontiguousarray(col_ptr, dtype=np.int32)
    ri = np.ascontiguousarray(row_idx, dtype=np.int32)
    h = C.c_void_p()
    if perm is not None:
        pm = np.ascontiguousarray(perm, dtype=np.int32)
        rc = L.smfg_analyse_ordered(int(n), cp, ri, pm, nemin, C.byref(h))
    else:
        rc = L.smfg_analyse(int(n), cp, ri, ordering, nemin, C.byref(h))
    if rc != SMFG_OK:
        raise SmfgError(rc, "smfg_analyse")
    try:
        ca = _Analysis()
        fl = C.c_double()
        fe = C.c_int64()
        L.smfg_symbolic_view(h, C.byref(ca), C.byref(fl), C.byref(fe))
        nsn = ca.nsn
        nslots = None
        sizes = {
            "perm": n, "sn_start": nsn, "sn_end": nsn, "sn_parent": nsn, "child_ptr": nsn + 1,
            "front_row_ptr": nsn + 1, "postorder": nsn, "perm_col_ptr": n + 1,
            "clean_col_ptr": n + 1, "orig_to_clean": ca.nnz_in,
        }
        arrays = {}

        def grab(name, count):
            ptr = getattr(ca, name)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(count,)).copy()

        for k, cnt in sizes.items():
            arrays[k] = grab(k, cnt)
        nslots = int(arrays["child_ptr"][-1])
        arrays["child_idx"] = grab("child_idx", max(nslots, 0)) if nslots else np.zeros(0, np.int32)
        arrays["front_row_idx"] = grab("front_row_idx", int(arrays["front_row_ptr"][-1]))
        cnnz = int(arrays["clean_col_ptr"][-1])
        arrays["perm_row_idx"] = grab("perm_row_idx", int(arrays["perm_col_ptr"][-1]))
        arrays["clean_row_idx"] = grab("clean_row_idx", cnnz)
        arrays["clean_to_perm"] = grab("clean_to_perm", cnnz)
        return Analysis(n, arrays, fl.value, fe.value)
    finally:
        L.smfg_symbolic_free(C.byref(h))


def matching_scale(n, col_ptr, row_idx, values):
    """smfg_matching_scale: symmetric max-product matching scaling (n
    doubles, original numbering) and the count of unmatched columns."""
    s = np.zeros(n, dtype=np.float64)
    um = C.c_int()
    rc = lib().smfg_matching_scale(int(n), np.ascontiguousarray(col_ptr, dtype=np.int32),
                                   np.ascontiguousarray(row_idx, dtype=np.int32),
                                   np.ascontiguousarray(values, dtype=np.float64), s, C.byref(um))
    if rc != SMFG_OK:
        raise SmfgError(rc, "smfg_matching_scale")
    return s, um.value


TC_TF32X3, TC_BF16X3 = 0, 1
REFINE_CLASSICAL, REFINE_FGMRES, REFINE_AUTO = 0, 1, 2


def aptp_front_dense(A, ne: int, u: float = 0.01, small: float = 1e-20, device: int = 0):
    """smfg_aptp_front_dense: the APTP front kernel on one dense symmetric
    front A (f x f, lower triangle used, first ne columns eligible) on the
    GPU. Returns (F (f x f, lower part meaningful), rows, tags, (eliminated,
    failed, positive, negative, zero))."""
    import torch
    A = np.asarray(A, dtype=np.float64)
    f = A.shape[0]
    if A.shape != (f, f) or not 0 < ne <= f:
        raise ValueError("A must be square with 0 < ne <= f")
    dev = torch.device("cuda", device)
    # column-major storage: the transpose's rows are A's columns
    dF = torch.from_numpy(np.ascontiguousarray(np.tril(A).T)).to(dev)
    drows = torch.arange(f, dtype=torch.int32, device=dev)
    dtags = torch.zeros(f, dtype=torch.int8, device=dev)
    out = np.zeros(5, dtype=np.int64)
    L = lib()
    L.smfg_aptp_front_dense.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                        C.c_double, C.c_void_p]
    torch.cuda.synchronize(dev)
    with torch.cuda.device(dev):
        rc = L.smfg_aptp_front_dense(C.c_void_p(dF.data_ptr()), f, int(ne), C.c_void_p(drows.data_ptr()),
                                     C.c_void_p(dtags.data_ptr()), float(u), float(small), out.ctypes.data)
    if rc != SMFG_OK:
        raise SmfgError(rc, "smfg_aptp_front_dense")
    F = dF.cpu().numpy().T
    return F, drows.cpu().numpy(), dtags.cpu().numpy(), tuple(int(x) for x in out)


def kernel_bench_defer(f: int = 8000, ne: int = 4000, k: int = 16, reps: int = 5) -> dict:
    """smfg_kernel_bench_defer: the streamed deferred-update kernel on one
    synthetic front (f rows, ne eligible columns, k pending pivots): best
    device ms, algorithmic bytes, GB/s, and entries differing bitwise from
    the tiled kernel (0 expected)."""
    L = lib()
    L.smfg_kernel_bench_defer.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
    ms, by, mm = C.c_double(), C.c_double(), C.c_longlong()
    rc = L.smfg_kernel_bench_defer(f, ne, k, reps, C.byref(ms), C.byref(by), C.byref(mm))
    if rc != SMFG_OK:
        raise SmfgError(rc, "smfg_kernel_bench_defer")
    return {"ms": ms.value, "bytes": by.value, "gbs": by.value / (ms.value * 1e6), "mismatches": mm.value}


def tc_update(C_t, L_t, W_t, kind: int = TC_TF32X3):
    """smfg_tc_update on CUDA float64 tensors given TRANSPOSED (row-major
    (k, n) / (n, n) tensors are the column-major n x k / n x n matrices):
    lower(C) -= L W^T with tensor-core split products, in place."""
    n = C_t.shape[0]
    k = L_t.shape[0]
    for t in (C_t, L_t, W_t):
        if not (t.is_cuda and t.dtype.is_floating_point and t.element_size() == 8 and t.is_contiguous()):
            raise ValueError("CUDA float64 contiguous tensors expected")
    if C_t.shape != (n, n) or L_t.shape != (k, n) or W_t.shape != (k, n):
        raise ValueError("shapes: C (n, n), L and W (k, n)")
    rc = lib().smfg_tc_update(C_t.data_ptr(), n, n, L_t.data_ptr(), n, W_t.data_ptr(), n, k, kind)
    if rc != SMFG_OK:
        raise SmfgError(rc, "smfg_tc_update")


class Solver:
    """The numeric phase on one GPU for one analysis (smf::Solver's factor /
    solve / inertia / refine; AnalysisKeep arrays from any object with the
    attributes n, perm, sn_start, sn_end, sn_parent, child_ptr, child_idx,
    front_row_ptr, front_row_idx, postorder, perm_col_ptr, perm_row_idx,
    orig_to_clean, clean_to_perm, clean_col_ptr, clean_row_idx)."""

    def __init__(self, analysis, device: int = -1):
        L = lib()
        self._arrays = {k: np.ascontiguousarray(getattr(analysis, k), dtype=np.int32)
                        for k in _ANALYSIS_FIELDS}
        self.n = int(analysis.n)
        self.nsn = int(self._arrays["sn_start"].size)
        self.nnz_in = int(self._arrays["orig_to_clean"].size)
        a = self._arrays
        ca = _Analysis(self.n, self.nsn, *[a[k].ctypes.data for k in _ANALYSIS_FIELDS[:11]],
                       self.nnz_in, *[a[k].ctypes.data for k in _ANALYSIS_FIELDS[11:]])
        h = C.c_void_p()
        rc = L.smfg_plan_create(C.byref(ca), device, C.byref(h))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_plan_create")
        self._h = h
        if device < 0:  # the plan took the current device
            import torch
            device = torch.cuda.current_device()
        self.device = int(device)
        self.posdef = False
        self.info = Info()
        self._scale = None

    def close(self):
        if getattr(self, "_h", None):
            lib().smfg_plan_destroy(C.byref(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    # -- factor ------------------------------------------------------------
    def set_front_precision(self, mask=None):
        """Per-front choice for mixed factorizations (smfg_set_front_precision):
        mask[s] = 1 lets supernode s use tensor-core updates; None: all may."""
        if mask is None:
            rc = lib().smfg_set_front_precision(self._h, None)
        else:
            m = np.ascontiguousarray(mask, dtype=np.int8)
            if m.size != self.nsn:
                raise ValueError(f"expected {self.nsn} entries")
            rc = lib().smfg_set_front_precision(self._h, m.ctypes.data)
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_set_front_precision")

    def set_panel_teams(self, teams=None):
        """smfg_set_panel_teams: CTAs per front-size bucket (4 ints of 0, 1, 2, 4,
        8, 16; 0 = rule)."""
        if teams is None:
            rc = lib().smfg_set_panel_teams(self._h, None)
        else:
            t = np.ascontiguousarray(teams, dtype=np.int32)
            if t.size != 4:
                raise ValueError("four buckets")
            rc = lib().smfg_set_panel_teams(self._h, t.ctypes.data)
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_set_panel_teams")

    def factor(self, values, posdef: bool = False, u: float = 0.01, small: float = 1e-20,
               scale=None, precision: int = PREC_FP64, max_negative_pivots: int = -1,
               raise_on_singular: bool = False, mixed_block: int = 0, mixed_kind: int = 0,
               mixed_min_front: int = 0, panel_team: int = 0, graph: bool = False,
               aptp_min_rows: int = APTP_MIN_ROWS, work_limit: float = -1.0) -> Info:
        """Factor new values (the caller's entry order). ``values`` is a
        numpy array, or any object with ``data_ptr()`` (a CUDA tensor) for
        values already in device memory. precision=PREC_MIXED: tensor-core
        trailing updates on large fronts (mixed_block pivots per update,
        mixed_kind TC_TF32X3 / TC_BF16X3, fronts of mixed_min_front rows or
        more; 0 = the library's defaults). aptp_min_rows: indefinite fronts of
        at least this many rows take the APTP kernel (smf's deterministic
        mode, the default 512); 0 = the threshold kernel everywhere (smf's
        one-thread default mode). max_negative_pivots >= 0 on an indefinite
        matrix: the factorization stops after the tree level where the
        negative pivots pass it (factor_status SMFG_FACTOR_INERTIA_EXCEEDED,
        partial counts, returned rather than raised). work_limit >= 0: it
        stops once the realized work (sum over factored fronts of pivots x
        rows^2) passes it (factor_status SMFG_FACTOR_MAX_PIVOT_DELAYS)."""
        c = default_control(posdef, u, small, precision, max_negative_pivots)
        c.aptp_min_rows = int(aptp_min_rows)
        c.work_limit = float(work_limit)
        c.mixed_block = mixed_block
        c.mixed_kind = mixed_kind
        c.mixed_min_front = mixed_min_front
        c.panel_team = panel_team
        c.graph = int(graph)
        if scale is not None and len(scale):
            self._scale = np.ascontiguousarray(scale, dtype=np.float64)
            c.scale = self._scale.ctypes.data
        else:
            self._scale = None
        info = Info()
        if hasattr(values, "data_ptr"):
            rc = lib().smfg_factor_device(self._h, C.c_void_p(values.data_ptr()), C.byref(c),
                                          C.byref(info))
        else:
            v = np.ascontiguousarray(values, dtype=np.float64)
            if v.size != self.nnz_in:
                raise ValueError(f"expected {self.nnz_in} values, got {v.size}")
            rc = lib().smfg_factor(self._h, v.ctypes.data, C.byref(c), C.byref(info))
        self.posdef = posdef
        self.info = info
        if rc == SMFG_ERR_WRONG_INERTIA and max_negative_pivots >= 0:
            return info
        if rc not in (SMFG_OK, SMFG_ERR_SINGULAR) or (rc == SMFG_ERR_SINGULAR and raise_on_singular):
            raise SmfgError(rc, "smfg_factor")
        return info

    def profile_factor(self, values, posdef: bool = False, precision: int = PREC_FP64,
                       scale=None, **mixed) -> dict:
        """One factorization with CUDA events around every launch of the
        large-front update kernels: FP64 GEMMs and tensor-core passes (split
        + product), their device times, launch counts and algorithmic flops
        (2 per multiply-add of the updates)."""
        c = default_control(posdef, 0.01, 1e-20, precision)
        c.profile = 1
        c.mixed_block = mixed.get("mixed_block", 0)
        c.mixed_kind = mixed.get("mixed_kind", 0)
        c.mixed_min_front = mixed.get("mixed_min_front", 0)
        if scale is not None and len(scale):
            self._scale = np.ascontiguousarray(scale, dtype=np.float64)
            c.scale = self._scale.ctypes.data
        info = Info()
        if hasattr(values, "data_ptr"):
            rc = lib().smfg_factor_device(self._h, C.c_void_p(values.data_ptr()), C.byref(c),
                                          C.byref(info))
        else:
            v = np.ascontiguousarray(values, dtype=np.float64)
            rc = lib().smfg_factor(self._h, v.ctypes.data, C.byref(c), C.byref(info))
        if rc not in (SMFG_OK, SMFG_ERR_SINGULAR):
            raise SmfgError(rc, "smfg_factor")
        self.info = info
        return {"gemm_ms": info.reserved_d[0], "gemm_flops": info.reserved_d[1],
                "gemm_launches": info.reserved_i[0], "arena_bytes": info.reserved_d[2],
                "tc_ms": info.reserved_d[4], "tc_flops": info.reserved_d[3],
                "tc_passes": info.reserved_i[1], "panel_ms": info.reserved_d[5],
                "schur_ms": info.reserved_d[7], "defer_bytes": info.reserved_d[6],
                "defer_updates": info.reserved_i[2], "defer_small": info.reserved_i[3],
                "factor_ms": info.factor_ms}

    # -- solve -------------------------------------------------------------
    def solve(self, b, job: int = SOLVE_FULL, out=None):
        """x = A^-1 b. b: (n,) or (nrhs, n) numpy array (returned as a new
        array, or in `out`, a C-contiguous float64 array of b's shape, e.g. a
        view of pinned host memory), or a CUDA tensor solved in place
        (returned)."""
        info = Info()
        if hasattr(b, "data_ptr"):
            nrhs = 1 if b.dim() == 1 else int(b.shape[0])
            rc = lib().smfg_solve_device(self._h, C.c_void_p(b.data_ptr()), nrhs, self.n, job,
                                         C.byref(info))
            if rc != SMFG_OK:
                raise SmfgError(rc, "smfg_solve_device")
            self.info.solve_ms = info.solve_ms
            return b
        if out is not None:
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape != np.shape(b):
                raise ValueError("out: a C-contiguous float64 array of b's shape")
            if out is not b:
                np.copyto(out, b)
            x = out
        else:
            x = np.array(b, dtype=np.float64, copy=True, order="C")
        nrhs = 1 if x.ndim == 1 else x.shape[0]
        rc = lib().smfg_solve(self._h, x.ctypes.data, nrhs, self.n, job, C.byref(info))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_solve")
        self.info.solve_ms = info.solve_ms
        self.last_solve_launches = info.kernel_launches
        return x

    def inertia(self):
        p, n, z = C.c_int(), C.c_int(), C.c_int()
        rc = lib().smfg_inertia(self._h, C.byref(p), C.byref(n), C.byref(z))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_inertia")
        return (p.value, n.value, z.value)

    def front_stats(self) -> np.ndarray:
        """(nsn, 5): positive, negative, zero, 2x2 pivots, delayed columns."""
        st = np.zeros(5 * self.nsn, dtype=np.int32)
        rc = lib().smfg_front_stats(self._h, st)
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_front_stats")
        return st.reshape(self.nsn, 5)

    def factor_sizes(self):
        """(stored factor entries sum f * p, realized front rows sum f) of
        the last factorization (smfg_factor_sizes)."""
        be, re_ = C.c_int64(), C.c_int64()
        rc = lib().smfg_factor_sizes(self._h, C.byref(be), C.byref(re_))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_factor_sizes")
        return int(be.value), int(re_.value)

    def export(self) -> FrontFactor:
        be, re_ = C.c_int64(), C.c_int64()
        lib().smfg_factor_sizes(self._h, C.byref(be), C.byref(re_))
        ns = self.nsn
        f = np.zeros(ns, dtype=np.int32)
        p = np.zeros(ns, dtype=np.int32)
        bo = np.zeros(ns, dtype=np.int64)
        ro = np.zeros(ns, dtype=np.int64)
        blocks = np.zeros(max(1, be.value), dtype=np.float64)
        rows = np.zeros(max(1, re_.value), dtype=np.int32)
        tags = None if self.posdef else np.zeros(max(1, self.n), dtype=np.int8)
        rc = lib().smfg_factor_export(self._h, f, p, bo, blocks, ro, rows,
                                      None if tags is None else tags.ctypes.data)
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_factor_export")
        return FrontFactor(f, p, bo, blocks, ro, rows, tags)

    def residual(self, b, x):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        nrhs = 1 if b.ndim == 1 else b.shape[0]
        r = np.zeros_like(b)
        eta, om = C.c_double(), C.c_double()
        rc = lib().smfg_residual(self._h, b.reshape(-1), x.reshape(-1), nrhs, r.ctypes.data,
                                 C.byref(eta), C.byref(om))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_residual")
        return r, eta.value, om.value

    def residual_noalloc(self, d_b, d_x, d_r=None):
        """smfg_residual_noalloc: the residual of device buffers (float64
        CUDA tensors on the plan's device, contiguous, shape (n,) or (nrhs,
        n)) computed in the library's fixed scratch array, allocating
        nothing. For callers that must not allocate device memory while
        they run, such as a real-time controller that reserves everything up
        front, or a program whose device memory is all committed to its own
        pool. Returns (eta_inf, omega); r is written to d_r when given. The
        plan's order must not exceed NOALLOC_MAX_N, and calls that overlap
        on the GPU race on the shared scratch. The buffers are checked here
        before the library is called: a wrong dtype, layout, size or device
        would make the kernels read or write past them."""
        tensors = [("d_b", d_b), ("d_x", d_x)] + ([("d_r", d_r)] if d_r is not None else [])
        shape = tuple(d_b.shape)
        if len(shape) not in (1, 2) or shape[-1] != self.n:
            raise ValueError(f"d_b must have shape (n,) or (nrhs, n) with n = {self.n}, got {shape}")
        for name, t in tensors:
            if str(t.dtype) != "torch.float64":
                raise ValueError(f"{name} must be float64, got {t.dtype}")
        for name, t in tensors:
            if tuple(t.shape) != shape:
                raise ValueError(f"{name} has shape {tuple(t.shape)}, d_b has {shape}")
        for name, t in tensors:
            if not t.is_contiguous():
                raise ValueError(f"{name} must be contiguous")
        for name, t in tensors:
            if t.device.type != "cuda" or t.device.index != self.device:
                raise ValueError(f"{name} must be on cuda:{self.device}, got {t.device}")
        nrhs = 1 if len(shape) == 1 else shape[0]
        if nrhs < 1:
            raise ValueError("no right-hand side given")
        eta, om = C.c_double(), C.c_double()
        rc = lib().smfg_residual_noalloc(self._h, C.c_void_p(d_b.data_ptr()), C.c_void_p(d_x.data_ptr()),
                                         None if d_r is None else C.c_void_p(d_r.data_ptr()), nrhs,
                                         C.byref(eta), C.byref(om))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_residual_noalloc")
        return eta.value, om.value

    def refine(self, b, x, max_steps: int = 10, omega_target: float = 1e-8,
               method: int = REFINE_CLASSICAL, restart: int = 20, inplace: bool = False):
        """Iterative refinement of x for b (smfg_refine_method): classical,
        FGMRES or auto; returns (x, eta_inf, omega, solves used). inplace:
        x (a C-contiguous float64 array) is refined in place, not copied."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        if inplace:
            if x.dtype != np.float64 or not x.flags.c_contiguous:
                raise ValueError("inplace: x must be a C-contiguous float64 array")
        else:
            x = np.array(x, dtype=np.float64, copy=True, order="C")
        nrhs = 1 if b.ndim == 1 else b.shape[0]
        eta, om, st = C.c_double(), C.c_double(), C.c_int()
        rc = lib().smfg_refine_method(self._h, b.reshape(-1), x.reshape(-1), nrhs, method, max_steps,
                                      restart, omega_target, C.byref(eta), C.byref(om), C.byref(st))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_refine_method")
        return x, eta.value, om.value, st.value

    def last_times(self):
        """(factor_ms, solve_ms, refine_ms) of the last calls, device time."""
        f, s_, r = C.c_double(), C.c_double(), C.c_double()
        lib().smfg_last_times(self._h, C.byref(f), C.byref(s_), C.byref(r))
        return f.value, s_.value, r.value

    def refine_device(self, d_b, d_x, nrhs: int = 1, max_steps: int = 10,
                      omega_target: float = 1e-8, method: int = REFINE_AUTO, restart: int = 20):
        """smfg_refine_device on CUDA tensors (n x nrhs, leading dimension
        n); d_x refined in place. Returns (eta_inf, omega, solves used)."""
        eta, om, st = C.c_double(), C.c_double(), C.c_int()
        rc = lib().smfg_refine_device(self._h, C.c_void_p(d_b.data_ptr()), C.c_void_p(d_x.data_ptr()), nrhs,
                                      method, max_steps, restart, omega_target, C.byref(eta),
                                      C.byref(om), C.byref(st))
        if rc != SMFG_OK:
            raise SmfgError(rc, "smfg_refine_device")
        return eta.value, om.value, st.value
