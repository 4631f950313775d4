"""Test infrastructure (the oracle): ctypes bindings to the two CPU checkers.

* ``Reference`` drives the reference smf solver compiled from its own sources
  (oracle/_ref/libsmfref.so, built by oracle/Makefile): its symbolic analysis
  (whose AnalysisKeep arrays the CUDA engine consumes as is), its numeric
  factor / solve / refinement, and per-front exports of its FactorKeep.
* ``restated_factorize`` runs the plain-C restatement (mf_oracle.c) of the
  reference numeric phase on the same analysis.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module; the product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libsmfref.so")
ORACLE_SO = os.path.join(HERE, "_build", "libmforacle.so")

# smf enums (solver/include/smf/types.hpp)
ORDER_AUTO_SERIAL, ORDER_AUTO_PARALLEL, ORDER_AMD, ORDER_METIS, ORDER_USER, ORDER_MATCHING = range(6)
SCALE_NONE, SCALE_EQUIL, SCALE_MATCHING, SCALE_USER, SCALE_AUTO = range(5)
POSDEF_KERNEL_LDLT, POSDEF_KERNEL_LAPACK = 0, 1

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def oracle_available() -> bool:
    return os.path.exists(ORACLE_SO)


@dataclass
class Analysis:
    """The AnalysisKeep arrays the numeric phase consumes
    (solver/include/smf/analysis.hpp:25-144), all 0-based int32."""
    n: int
    perm: np.ndarray            # perm[new] = old
    sn_start: np.ndarray
    sn_end: np.ndarray
    sn_parent: np.ndarray
    child_ptr: np.ndarray
    child_idx: np.ndarray       # descending postorder
    front_row_ptr: np.ndarray
    front_row_idx: np.ndarray   # sorted, first width() are the pivots
    postorder: np.ndarray
    perm_col_ptr: np.ndarray    # permuted lower pattern
    perm_row_idx: np.ndarray
    clean_to_perm: np.ndarray   # cleaned entry -> permuted slot
    orig_to_clean: np.ndarray   # input entry -> cleaned slot (-1 dropped)
    clean_col_ptr: np.ndarray
    clean_row_idx: np.ndarray
    matching_scale: np.ndarray  # empty when the analysis computed none

    @property
    def nsn(self) -> int:
        return int(self.sn_start.size)


@dataclass
class FactorExport:
    status: int
    inertia: tuple
    delayed: int
    two_by_two: int
    max_front: int
    flops: float
    factor_ms: float
    f: np.ndarray
    p: np.ndarray
    blk_off: np.ndarray
    blocks: np.ndarray
    row_off: np.ndarray
    rows: np.ndarray
    tags: np.ndarray | None
    scale: np.ndarray
    aptp_failed: int = 0  # columns the APTP kernel failed (Info::aptp_failed_columns)

    def block(self, s: int) -> np.ndarray:
        f, p = int(self.f[s]), int(self.p[s])
        o = int(self.blk_off[s])
        return self.blocks[o:o + f * p].reshape(p, f).T  # f x p column-major view

    def front_rows(self, s: int) -> np.ndarray:
        o = int(self.row_off[s])
        return self.rows[o:o + int(self.f[s])]


class Reference:
    """The reference smf solver (oracle/_ref/libsmfref.so)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not ref_available():
                raise RuntimeError(f"reference library not built: {REF_SO}")
            lib = C.CDLL(REF_SO)
            lib.refshim_create.restype = C.c_void_p
            lib.refshim_free.argtypes = [C.c_void_p]
            lib.refshim_set_control.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                                C.c_int]
            lib.refshim_analyse.argtypes = [C.c_void_p, C.c_int, _i32p, _i32p, C.c_void_p, C.c_void_p]
            lib.refshim_analyse.restype = C.c_int
            lib.refshim_analysis_sizes.argtypes = [C.c_void_p, _i64p]
            lib.refshim_analysis_export.argtypes = [C.c_void_p] + [_i32p] * 15 + [C.c_void_p]
            lib.refshim_analyse_ms.argtypes = [C.c_void_p]
            lib.refshim_analyse_ms.restype = C.c_double
            lib.refshim_factor.argtypes = [C.c_void_p, _f64p, _i64p, _f64p]
            lib.refshim_factor.restype = C.c_int
            lib.refshim_factor_sizes.argtypes = [C.c_void_p, _i64p]
            lib.refshim_factor_export.argtypes = [C.c_void_p, _i32p, _i32p, _i64p, _f64p, _i64p,
                                                  _i32p, C.c_void_p, C.c_void_p]
            lib.refshim_factor_export.restype = C.c_int
            lib.refshim_solve.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, C.c_int, C.c_void_p]
            lib.refshim_solve.restype = C.c_int
            lib.refshim_refine.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int, _f64p, _i32p]
            lib.refshim_refine.restype = C.c_int
            lib.refshim_front_work.argtypes = [C.c_void_p, _f64p]
            lib.refshim_aptp_failed.argtypes = [C.c_void_p]
            lib.refshim_aptp_failed.restype = C.c_int64
            lib.refshim_matching_scale.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p]
            lib.refshim_matching_scale.restype = C.c_int
            lib.refshim_ipm_create.restype = C.c_void_p
            lib.refshim_ipm_free.argtypes = [C.c_void_p]
            lib.refshim_ipm_analyse.argtypes = [C.c_void_p, C.c_int, _i32p, _i32p, _f64p, C.c_int]
            lib.refshim_ipm_analyse.restype = C.c_int
            lib.refshim_ipm_factor.argtypes = [C.c_void_p, _f64p, C.c_int64, C.c_int, _i64p]
            lib.refshim_ipm_solve.argtypes = [C.c_void_p, _f64p, C.c_int, _i64p]
            lib.refshim_ipm_solve.restype = C.c_int
            cls._lib = lib
        return cls._lib

    def __init__(self, posdef: bool, ordering: int = ORDER_AMD, deterministic: bool = True,
                 num_threads: int = 1, u: float = 0.01, small: float = 1e-20,
                 scaling: int = SCALE_AUTO, nemin: int = 0,
                 posdef_kernel: int = POSDEF_KERNEL_LDLT, top_tiles: bool = True):
        self.L = self.lib()
        self.h = self.L.refshim_create()
        self.posdef = posdef
        self.L.refshim_set_control(self.h, ordering, nemin, int(deterministic), num_threads, u,
                                   small, scaling, int(posdef), posdef_kernel, int(top_tiles))
        self.n = 0
        self.nnz = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.refshim_free(self.h)
            self.h = None

    def analyse(self, n, col_ptr, row_idx, values=None, user_perm=None) -> Analysis:
        col_ptr = np.ascontiguousarray(col_ptr, dtype=np.int32)
        row_idx = np.ascontiguousarray(row_idx, dtype=np.int32)
        vals = None if values is None else np.ascontiguousarray(values, dtype=np.float64)
        up = None if user_perm is None else np.ascontiguousarray(user_perm, dtype=np.int32)
        self._keep = (vals, up)
        rc = self.L.refshim_analyse(self.h, int(n), col_ptr, row_idx,
                                    None if vals is None else vals.ctypes.data,
                                    None if up is None else up.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"reference analyse failed: {rc}")
        sz = np.zeros(12, dtype=np.int64)
        self.L.refshim_analysis_sizes(self.h, sz)
        n, ns, nch, nfr, _pnnz, nin, nms, cnnz = (int(x) for x in sz[:8])
        self.n = n
        self.nnz = int(col_ptr[-1])
        z = lambda k: np.zeros(k, dtype=np.int32)
        a = Analysis(n=n, perm=z(n), sn_start=z(ns), sn_end=z(ns), sn_parent=z(ns),
                     child_ptr=z(ns + 1), child_idx=z(nch), front_row_ptr=z(ns + 1),
                     front_row_idx=z(nfr), postorder=z(ns), perm_col_ptr=z(n + 1),
                     perm_row_idx=z(cnnz), clean_to_perm=z(cnnz),
                     orig_to_clean=z(nin if nin else cnnz), clean_col_ptr=z(n + 1),
                     clean_row_idx=z(cnnz), matching_scale=np.zeros(nms, dtype=np.float64))
        self.L.refshim_analysis_export(self.h, a.perm, a.sn_start, a.sn_end, a.sn_parent,
                                       a.child_ptr, a.child_idx, a.front_row_ptr, a.front_row_idx,
                                       a.postorder, a.perm_col_ptr, a.perm_row_idx,
                                       a.clean_to_perm, a.orig_to_clean, a.clean_col_ptr,
                                       a.clean_row_idx,
                                       a.matching_scale.ctypes.data if nms else None)
        self.analyse_ms = self.L.refshim_analyse_ms(self.h)
        return a

    def factor(self, values, export: bool = True) -> FactorExport:
        """Factor; with export, copy the FactorKeep out per front (needs the
        serial engine's step layout: deterministic mode or one thread)."""
        vals = np.ascontiguousarray(values, dtype=np.float64)
        st = np.zeros(10, dtype=np.int64)
        fm = np.zeros(2, dtype=np.float64)
        self.L.refshim_factor(self.h, vals, st, fm)
        if not export:
            z = np.zeros(0, dtype=np.int32)
            return FactorExport(status=int(st[0]), inertia=(int(st[1]), int(st[2]), int(st[3])),
                                delayed=int(st[4]), two_by_two=int(st[5]), max_front=int(st[6]),
                                flops=float(fm[0]), factor_ms=float(fm[1]), f=z, p=z, blk_off=z,
                                blocks=np.zeros(0), row_off=z, rows=z, tags=None, scale=np.zeros(0))
        fs = np.zeros(6, dtype=np.int64)
        self.L.refshim_factor_sizes(self.h, fs)
        nsteps, fext, rows_total, _nd, _pd, nscale = (int(x) for x in fs)
        ns = nsteps
        f = np.zeros(ns, dtype=np.int32)
        p = np.zeros(ns, dtype=np.int32)
        bo = np.zeros(ns, dtype=np.int64)
        ro = np.zeros(ns, dtype=np.int64)
        blocks = np.zeros(max(fext, 1), dtype=np.float64)
        rows = np.zeros(max(rows_total, 1), dtype=np.int32)
        tags = None if self.posdef else np.zeros(max(self.n, 1), dtype=np.int8)
        scale = np.zeros(nscale, dtype=np.float64)
        if st[0] in (0, 2):
            rc = self.L.refshim_factor_export(self.h, f, p, bo, blocks, ro, rows,
                                              None if tags is None else tags.ctypes.data,
                                              scale.ctypes.data if nscale else None)
            if rc != 0:
                raise RuntimeError(f"reference factor export failed: {rc}")
        return FactorExport(status=int(st[0]), inertia=(int(st[1]), int(st[2]), int(st[3])),
                            delayed=int(st[4]), two_by_two=int(st[5]), max_front=int(st[6]),
                            flops=float(fm[0]), factor_ms=float(fm[1]), f=f, p=p, blk_off=bo,
                            blocks=blocks, row_off=ro, rows=rows, tags=tags, scale=scale,
                            aptp_failed=int(self.L.refshim_aptp_failed(self.h)))

    def front_work(self):
        """(the last factorization's Info::front_work, the analysis'
        delay_free_front_work)."""
        out = np.zeros(2, dtype=np.float64)
        self.L.refshim_front_work(self.h, out)
        return float(out[0]), float(out[1])

    def solve(self, b, job: int = 0):
        """Full solve; b of shape (n,) or (nrhs, n). Returns (x, ms)."""
        x = np.array(b, dtype=np.float64, copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[0]
        ms = C.c_double(0.0)
        rc = self.L.refshim_solve(self.h, x.reshape(-1), nrhs, self.n, job, C.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference solve failed: {rc}")
        return x, ms.value

    def refine(self, b, x):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.array(x, dtype=np.float64, copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[0]
        res = np.zeros(2, dtype=np.float64)
        it = np.zeros(2, dtype=np.int32)
        self.L.refshim_refine(self.h, b.reshape(-1), x.reshape(-1), nrhs, res, it)
        return x, float(res[0]), float(res[1]), int(it[0])


class ReferenceIpmSession:
    """The reference's smf::IpmSession (solver/src/ipm_session.cpp) in its
    default Control (AutoSerial ordering, Auto scaling), deterministic mode,
    one thread, indefinite: analyse once, then factor / solve a stream of
    values. factor() returns (IpmFactorStatus 0 Ok / 1 WrongInertia /
    2 Singular / 3 Error, inertia, delayed pivots); solve() returns (x, rc,
    inertia afterwards, learned expectation or None)."""

    def __init__(self):
        self.L = Reference.lib()
        self.h = self.L.refshim_ipm_create()
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.refshim_ipm_free(self.h)
            self.h = None

    def analyse(self, n, col_ptr, row_idx, values, abort_on_wrong_inertia: bool = True) -> int:
        self.n = int(n)
        self.nnz = int(col_ptr[-1])
        return self.L.refshim_ipm_analyse(self.h, self.n, np.ascontiguousarray(col_ptr, dtype=np.int32),
                                          np.ascontiguousarray(row_idx, dtype=np.int32),
                                          np.ascontiguousarray(values, dtype=np.float64),
                                          int(abort_on_wrong_inertia))

    def factor(self, values, expected_negatives=None):
        out = np.zeros(5, dtype=np.int64)
        v = np.ascontiguousarray(values, dtype=np.float64)
        self.L.refshim_ipm_factor(self.h, v, v.size, -1 if expected_negatives is None else int(expected_negatives),
                                  out)
        return int(out[0]), (int(out[1]), int(out[2]), int(out[3])), int(out[4])

    def solve(self, b):
        x = np.array(b, dtype=np.float64, copy=True)
        out = np.zeros(4, dtype=np.int64)
        rc = self.L.refshim_ipm_solve(self.h, x, self.n, out)
        return x, rc, (int(out[0]), int(out[1]), int(out[2])), (None if out[3] < 0 else int(out[3]))


# --------------------------------------------------------------------------
# The C restatement (mf_oracle.c)

class _MfoAnalysis(C.Structure):
    _fields_ = [("n", C.c_int), ("nsn", C.c_int)] + [
        (nm, C.c_void_p) for nm in ("sn_start", "sn_end", "sn_parent", "child_ptr", "child_idx",
                                    "front_row_ptr", "front_row_idx", "postorder", "pcp", "pri")]


class _MfoParams(C.Structure):
    _fields_ = [("u", C.c_double), ("eff_small", C.c_double), ("small_pivot", C.c_double),
                ("nb", C.c_int), ("blocked_min_front", C.c_int), ("posdef", C.c_int),
                ("mixed_min_front", C.c_int), ("mixed_bits", C.c_int),
                ("aptp_min_rows", C.c_int), ("aptp_nb", C.c_int), ("aptp_ib", C.c_int)]


class _MfoFactor(C.Structure):
    _fields_ = [("f_out", C.c_void_p), ("p_out", C.c_void_p), ("blk_off", C.c_void_p),
                ("row_off", C.c_void_p), ("blocks", C.c_void_p), ("blk_cap", C.c_int64),
                ("rows", C.c_void_p), ("row_cap", C.c_int64), ("tags", C.c_void_p),
                ("pos", C.c_int64), ("neg", C.c_int64), ("zero", C.c_int64),
                ("delayed", C.c_int64), ("two_by_two", C.c_int64), ("max_front", C.c_int64),
                ("aptp_failed", C.c_int64), ("flops", C.c_double), ("status", C.c_int)]


_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        if not oracle_available():
            raise RuntimeError(f"oracle restatement not built: {ORACLE_SO}")
        _olib = C.CDLL(ORACLE_SO)
        _olib.mfo_factorize.argtypes = [C.c_void_p, _f64p, C.c_void_p, C.c_void_p]
        _olib.mfo_factorize.restype = C.c_int
        _olib.mfo_solve_permuted.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _f64p]
        _olib.mfo_residual.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _olib.mfo_factor_front.argtypes = [_f64p, C.c_int, C.c_int, _i32p, C.c_void_p,
                                           np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS"), _i64p]
    return _olib


# Deterministic mode's APTP kernel: indefinite fronts of at least 512 rows
# (kTopTileMinFront, parallel/thread_plan.hpp:43), outer block 256
# (Control::top_tile_nb, control.hpp:638), inner block 32 (Control::aptp_ib).
APTP_MIN_ROWS, APTP_NB, APTP_IB = 512, 256, 32


def factor_front(A, ne: int, u: float = 0.01, small: float = 1e-20, nb: int = 16,
                 blocked_min_front: int = 96, posdef: bool = False):
    """One dense front (f x f symmetric, lower triangle used, first ne columns
    eligible) through the restated front kernel: (F, rows, tags, (pos, neg,
    zero, accepted))."""
    F = np.array(A, dtype=np.float64, order="F")
    f = F.shape[0]
    flat = np.ascontiguousarray(F.T.reshape(-1))  # column-major storage
    rows = np.arange(f, dtype=np.int32)
    tags = np.zeros(f, dtype=np.int8)
    out = np.zeros(4, dtype=np.int64)
    m = float(np.max(np.abs(F))) if F.size else 0.0
    eff = small * m if 0.0 < m < small else small
    prm = _MfoParams(u, eff, small, nb, blocked_min_front, int(posdef), 0, 0, 0, APTP_NB, APTP_IB)
    _oracle_lib().mfo_factor_front(flat, f, ne, rows, C.byref(prm), tags, out)
    return flat.reshape(f, f).T, rows, tags, tuple(int(x) for x in out)


def permuted_values(a: Analysis, values, scale=None):
    """Input values -> the permuted lower pattern (duplicates summed in input
    order, then S A S), as map_values_to_permuted and factor_indef's scaling
    pass place them (solver/src/workspace.cpp:129-281,
    solver/src/factor_indef.cpp:513-559)."""
    values = np.asarray(values, dtype=np.float64)
    cnnz = a.clean_row_idx.size
    clean = np.zeros(cnnz, dtype=np.float64)
    for k in range(values.size):  # input order (duplicates summed in order)
        c = a.orig_to_clean[k]
        if c >= 0:
            clean[c] += values[k]
    if scale is not None and len(scale):
        cols = np.repeat(np.arange(a.n), np.diff(a.clean_col_ptr))
        clean = clean * (scale[a.clean_row_idx] * scale[cols])
    pv = np.zeros(a.perm_row_idx.size, dtype=np.float64)
    pv[a.clean_to_perm] = clean
    return pv


def eff_small_of(pv, small=1e-20):
    m = float(np.max(np.abs(pv))) if pv.size else 0.0
    return small * m if (0.0 < m < small) else small


def restated_factorize(a: Analysis, pv, posdef: bool, u: float = 0.01, small: float = 1e-20,
                       nb: int = 16, blocked_min_front: int = 96, mixed_min_front: int = 0,
                       mixed_bits: int = 0, aptp_min_rows: int = APTP_MIN_ROWS):
    """Run mf_oracle.c on analysis `a` and permuted values `pv`: the
    reference's deterministic mode (APTP on indefinite fronts of at least
    aptp_min_rows rows; 0 = threshold pivoting everywhere, the reference's
    one-thread default mode). mixed_*: emulate the engine's split-product
    updates on fronts of at least mixed_min_front rows (mixed_bits 8: BF16x3,
    11: TF32x3)."""
    lib = _oracle_lib()
    keep = [np.ascontiguousarray(x, dtype=np.int32) for x in (
        a.sn_start, a.sn_end, a.sn_parent, a.child_ptr, a.child_idx, a.front_row_ptr,
        a.front_row_idx, a.postorder, a.perm_col_ptr, a.perm_row_idx)]
    ca = _MfoAnalysis(a.n, a.nsn, *[x.ctypes.data for x in keep])
    prm = _MfoParams(u, eff_small_of(pv, small), small, nb, blocked_min_front, int(posdef),
                     int(mixed_min_front), int(mixed_bits), int(aptp_min_rows), APTP_NB, APTP_IB)
    ns = a.nsn
    fsz = np.diff(a.front_row_ptr).astype(np.int64)
    # capacity: front rows grow with delays; allow generous room
    blk_cap = int(np.sum(fsz * fsz)) * 4 + 1024 + int(a.n) * int(a.n if a.n < 4000 else 4000)
    row_cap = int(np.sum(fsz)) * 4 + a.n * 4 + 1024
    f = np.zeros(ns, dtype=np.int32)
    p = np.zeros(ns, dtype=np.int32)
    bo = np.zeros(ns, dtype=np.int64)
    ro = np.zeros(ns, dtype=np.int64)
    blocks = np.zeros(blk_cap, dtype=np.float64)
    rows = np.zeros(row_cap, dtype=np.int32)
    tags = np.zeros(row_cap, dtype=np.int8)
    out = _MfoFactor(f.ctypes.data, p.ctypes.data, bo.ctypes.data, ro.ctypes.data,
                     blocks.ctypes.data, blk_cap, rows.ctypes.data, row_cap, tags.ctypes.data)
    pv = np.ascontiguousarray(pv, dtype=np.float64)
    lib.mfo_factorize(C.byref(ca), pv, C.byref(prm), C.byref(out))
    fx = FactorExport(status=out.status, inertia=(out.pos, out.neg, out.zero), delayed=out.delayed,
                      two_by_two=out.two_by_two, max_front=out.max_front, flops=out.flops,
                      factor_ms=0.0, f=f, p=p, blk_off=bo, blocks=blocks, row_off=ro, rows=rows,
                      tags=None if posdef else tags, scale=np.zeros(0), aptp_failed=out.aptp_failed)
    fx._c = (ca, keep, out)  # keep alive for solves
    return fx


def restated_solve(a: Analysis, fx: FactorExport, posdef: bool, b, scale=None):
    """Full solve through the restated factor: x = P S (L D L^T)^-1 S P^T b."""
    lib = _oracle_lib()
    ca, _keep, out = fx._c
    b = np.asarray(b, dtype=np.float64)
    s = np.ones(a.n) if scale is None or not len(scale) else np.asarray(scale)
    w = np.ascontiguousarray(b[a.perm] * s[a.perm])
    lib.mfo_solve_permuted(C.byref(ca), C.byref(out), int(posdef), w)
    x = np.empty(a.n)
    x[a.perm] = w * s[a.perm]
    return x


def reference_matching_scale(n, col_ptr, row_idx, values):
    """The reference's matching scaling (compute_matching_scale) of a lower
    CSC matrix: (scale, ErrorCode)."""
    s = np.zeros(n, dtype=np.float64)
    rc = Reference.lib().refshim_matching_scale(
        int(n), np.ascontiguousarray(col_ptr, dtype=np.int32), np.ascontiguousarray(row_idx, dtype=np.int32),
        np.ascontiguousarray(values, dtype=np.float64), s)
    return s, int(rc)


def residual(n, col_ptr, row_idx, values, b, x):
    """(r, eta_inf, omega) with long-double accumulation."""
    lib = _oracle_lib()
    r = np.zeros(n)
    eta = C.c_double()
    om = C.c_double()
    lib.mfo_residual(int(n), np.ascontiguousarray(col_ptr, dtype=np.int32),
                     np.ascontiguousarray(row_idx, dtype=np.int32),
                     np.ascontiguousarray(values, dtype=np.float64),
                     np.ascontiguousarray(b, dtype=np.float64),
                     np.ascontiguousarray(x, dtype=np.float64), r, C.byref(eta), C.byref(om))
    return r, eta.value, om.value
