"""The learned per-front precision selector of the mixed-precision path.

For every large front (the fronts the tensor-core path may take) a small MLP
reads per-supernode features and predicts whether that front's
reduced-precision updates keep the factorization's pivoting unchanged: the
front and its parent produce the same pivot counts (positive, negative,
zero, 2x2) and the same delayed columns as the plain FP64 path. The
network is trained on outcomes the solver itself produces on synthetic
matrices (plain FP64 factor vs mixed factors with random front masks; the
plain path is the judge), with the engine's own forward / backward / Adam
kernels (smfg_mlp_*). At factorization time the fronts it rejects stay in
FP64, and any front it misjudged (a changed inertia, changed counts of the
front or its parent against the last plain factorization) is refactored in
FP64 (``factor_checked``).

Features (per supernode, from the analysis, the scaled values and the last
factorization's per-front counts):
  0 log2 f        symbolic front rows
  1 log2 p        eliminated columns (supernode width)
  2 log2 (1 + q)  contribution-block rows, q = f - p
  3 p / f
  4 log2 (1 + delayed columns the children passed up)
  5 2x2 share of the children's pivots
  6 height of the front in the tree / height of the tree
  7 log10 max over its columns of (largest off-diagonal / |diagonal|) of
    the scaled input matrix (the assembled block's diagonal dominance)
  8 positive definite path (1) or not (0)
  9 log2 (1 + delayed columns the front itself passed up)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import smfg

N_FEATURES = 10
LARGE_MIN = 384  # the engine's large-front class (kLargeMin)


def _tree_height(parent):
    n = len(parent)
    h = np.zeros(n, dtype=np.int64)
    for s in range(n):  # postorder: children before parents
        p = parent[s]
        if p >= 0:
            h[p] = max(h[p], h[s] + 1)
    return h


def _diag_ratio(a, values, scale):
    """log10 of the largest |off-diagonal| / |diagonal| over each
    supernode's columns, in the permuted (scaled) lower pattern."""
    values = np.asarray(values, dtype=np.float64)
    cnnz = a.clean_row_idx.size
    clean = np.zeros(cnnz)
    oc = np.asarray(a.orig_to_clean)
    ok = oc >= 0
    np.add.at(clean, oc[ok], values[ok])
    if scale is not None and len(scale):
        cols = np.repeat(np.arange(a.n), np.diff(a.clean_col_ptr))
        clean = clean * scale[a.clean_row_idx] * scale[cols]
    pv = np.zeros(a.perm_row_idx.size)
    pv[a.clean_to_perm] = clean
    cp = np.asarray(a.perm_col_ptr, dtype=np.int64)
    ri = np.asarray(a.perm_row_idx)
    colj = np.repeat(np.arange(a.n), np.diff(cp))
    absv = np.abs(pv)
    diag = np.zeros(a.n)
    isd = ri == colj
    diag[colj[isd]] = absv[isd]
    off = np.zeros(a.n)
    np.maximum.at(off, colj[~isd], absv[~isd])
    np.maximum.at(off, ri[~isd], absv[~isd])
    ratio = np.log10((off + 1e-300) / (diag + 1e-300))
    ratio = np.clip(ratio, -20, 20)
    out = np.full(a.nsn, -20.0)
    starts, ends = np.asarray(a.sn_start), np.asarray(a.sn_end)
    for s in range(a.nsn):
        out[s] = ratio[starts[s]:ends[s]].max()
    return out


def front_features(a, values, posdef: bool, stats=None, scale=None) -> np.ndarray:
    """(nsn, N_FEATURES) float32. stats: the last factorization's
    Solver.front_stats() (nsn x 5), or None (zeros)."""
    ns = a.nsn
    f = np.diff(np.asarray(a.front_row_ptr)).astype(np.float64)
    p = (np.asarray(a.sn_end) - np.asarray(a.sn_start)).astype(np.float64)
    q = f - p
    parent = np.asarray(a.sn_parent)
    h = _tree_height(parent)
    H = max(1, int(h.max()))
    X = np.zeros((ns, N_FEATURES), dtype=np.float64)
    X[:, 0] = np.log2(f)
    X[:, 1] = np.log2(p)
    X[:, 2] = np.log2(1.0 + q)
    X[:, 3] = p / f
    if stats is not None:
        st = np.asarray(stats, dtype=np.float64)
        din = np.zeros(ns)
        piv = np.zeros(ns)
        two = np.zeros(ns)
        for s in range(ns):
            t = parent[s]
            if t >= 0:
                din[t] += st[s, 4]
                piv[t] += st[s, 0] + st[s, 1]
                two[t] += 2 * st[s, 3]
        X[:, 4] = np.log2(1.0 + din)
        X[:, 5] = np.where(piv > 0, two / np.maximum(piv, 1), 0.0)
        X[:, 9] = np.log2(1.0 + st[:, 4])
    X[:, 6] = h / H
    X[:, 7] = _diag_ratio(a, values, scale) / 10.0
    X[:, 8] = 1.0 if posdef else 0.0
    return X.astype(np.float32)


def candidates(a) -> np.ndarray:
    """The fronts the mixed path may take (the large-front class)."""
    return np.diff(np.asarray(a.front_row_ptr)) >= LARGE_MIN


def outcome_labels(a, stats_plain, stats_mixed, mask) -> np.ndarray:
    """1 where a mixed front left its own and its parent's pivot counts
    (positive, negative, zero, 2x2, delayed) as the plain path's, else 0;
    -1 for fronts that were not mixed."""
    parent = np.asarray(a.sn_parent)
    same = np.all(np.asarray(stats_plain) == np.asarray(stats_mixed), axis=1)
    lab = np.full(a.nsn, -1, dtype=np.int64)
    for s in np.nonzero(mask)[0]:
        ok = same[s] and (parent[s] < 0 or same[parent[s]])
        lab[s] = 1 if ok else 0
    return lab


class Selector:
    """The MLP on the GPU (parameters, Adam moments: CUDA float32 tensors),
    trained and evaluated by smfg_mlp_forward / _backward / _adam."""

    def __init__(self, d: int = N_FEATURES, h: int = 16, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.d, self.h = d, h
        self.dev = torch.device("cuda", device)
        self.np = int(smfg.lib().smfg_mlp_params(d, h))
        g = torch.Generator().manual_seed(seed)
        W1 = torch.randn(h, d, generator=g) * (2.0 / d) ** 0.5
        w2 = torch.randn(h, generator=g) * (1.0 / h) ** 0.5
        P = torch.cat([W1.reshape(-1), torch.zeros(h), w2, torch.zeros(1)])
        self.P = P.float().to(self.dev).contiguous()
        self.M = torch.zeros_like(self.P)
        self.V = torch.zeros_like(self.P)
        self.step = 0
        self.mu = torch.zeros(d)
        self.sd = torch.ones(d)
        self.threshold = 0.5

    # feature standardization (fitted on the training set)
    def _x(self, X):
        t = self.torch
        Xt = t.as_tensor(np.asarray(X, dtype=np.float32))
        return ((Xt - self.mu) / self.sd).float().to(self.dev).contiguous()

    def predict(self, X) -> np.ndarray:
        X = np.asarray(X, dtype=np.float32)
        if X.shape[0] == 0:
            return np.zeros(0, dtype=np.float32)
        Xd = self._x(X)
        out = self.torch.empty(X.shape[0], dtype=self.torch.float32, device=self.dev)
        L = smfg.lib()
        rc = L.smfg_mlp_forward(C.c_void_p(Xd.data_ptr()), X.shape[0], self.d, C.c_void_p(self.P.data_ptr()),
                                self.h, C.c_void_p(out.data_ptr()))
        if rc != smfg.SMFG_OK:
            raise smfg.SmfgError(rc, "smfg_mlp_forward")
        return out.cpu().numpy()

    def grad(self, Xd, yd, wd):
        """(gradient tensor, loss) on standardized device inputs."""
        t = self.torch
        n = int(Xd.shape[0])
        nb = (n + 127) // 128
        scratch = t.empty(nb * (self.np + 1), dtype=t.float32, device=self.dev)
        g = t.empty(self.np + 1, dtype=t.float32, device=self.dev)
        rc = smfg.lib().smfg_mlp_backward(C.c_void_p(Xd.data_ptr()), C.c_void_p(yd.data_ptr()),
                                          C.c_void_p(wd.data_ptr()) if wd is not None else None, n, self.d,
                                          C.c_void_p(self.P.data_ptr()), self.h, C.c_void_p(scratch.data_ptr()),
                                          C.c_void_p(g.data_ptr()))
        if rc != smfg.SMFG_OK:
            raise smfg.SmfgError(rc, "smfg_mlp_backward")
        return g[:self.np], float(g[self.np].item())

    def fit(self, X, y, epochs: int = 300, lr: float = 0.02, balance: bool = True) -> list:
        """Full-batch Adam on weighted BCE (classes balanced); returns the
        loss per epoch."""
        t = self.torch
        X = np.asarray(X, dtype=np.float32)
        y = np.asarray(y, dtype=np.float32)
        self.mu = t.as_tensor(X.mean(axis=0))
        self.sd = t.as_tensor(X.std(axis=0) + 1e-6)
        Xd = self._x(X)
        yd = t.as_tensor(y).to(self.dev).contiguous()
        w = np.ones_like(y)
        if balance and 0 < y.sum() < len(y):
            pos = y.mean()
            w = np.where(y > 0.5, 0.5 / pos, 0.5 / (1.0 - pos)).astype(np.float32)
        wd = t.as_tensor(w).to(self.dev).contiguous()
        hist = []
        L = smfg.lib()
        for _ in range(epochs):
            g, loss = self.grad(Xd, yd, wd)
            self.step += 1
            rc = L.smfg_mlp_adam(C.c_void_p(self.P.data_ptr()), C.c_void_p(g.data_ptr()),
                                 C.c_void_p(self.M.data_ptr()), C.c_void_p(self.V.data_ptr()), self.np, lr, 0.9,
                                 0.999, 1e-8, self.step)
            if rc != smfg.SMFG_OK:
                raise smfg.SmfgError(rc, "smfg_mlp_adam")
            hist.append(loss)
        return hist

    def mask(self, a, X) -> np.ndarray:
        """int8 mask for Solver.set_front_precision: the large fronts the
        network accepts."""
        m = np.zeros(a.nsn, dtype=np.int8)
        cand = candidates(a)
        if cand.any():
            p = self.predict(X[cand])
            m[np.nonzero(cand)[0][p >= self.threshold]] = 1
        return m


def factor_checked(sv, a, values, posdef, mask, stats_plain, expected_inertia=None, scale=None, **kw):
    """A mixed factorization with the selector's mask, judged against the
    last plain factorization's per-front counts: fronts whose own or
    parent's counts changed (or all mixed fronts, when the inertia is not
    the expected one) are set to FP64 and the matrix is refactored.
    Returns (info, mask used last, misjudged fronts); info.total_ms holds
    the device time of all factorizations of the call."""
    parent = np.asarray(a.sn_parent)
    sv.set_front_precision(mask)
    info = sv.factor(values, posdef=posdef, precision=smfg.PREC_MIXED, scale=scale, **kw)
    total_ms = info.factor_ms
    st = sv.front_stats()
    bad = np.zeros(a.nsn, dtype=bool)
    if stats_plain is not None:
        diff = ~np.all(st == stats_plain, axis=1)
        for s in np.nonzero(mask)[0]:
            if diff[s] or (parent[s] >= 0 and diff[parent[s]]):
                bad[s] = True
    if expected_inertia is not None and tuple(info.inertia) != tuple(expected_inertia):
        bad |= mask.astype(bool)
    nbad = int(bad.sum())
    if nbad:
        mask = mask.copy()
        mask[bad] = 0
        sv.set_front_precision(mask)
        info = sv.factor(values, posdef=posdef, precision=smfg.PREC_MIXED, scale=scale, **kw)
        total_ms += info.factor_ms
    info.total_ms = total_ms
    return info, mask, nbad


def collect_outcomes(problems, runs: int = 4, share: float = 0.6, seed: int = 0, device: int = 0):
    """Training data from the solver itself: for each (n, col_ptr, row_idx,
    values, posdef) problem, a plain FP64 factorization (the judge) and
    `runs` mixed factorizations with random masks over the large fronts
    (TF32x3 and BF16x3 alternating); features of every mixed front with
    its outcome label. Returns (X, y, problem index per row)."""
    rng = np.random.default_rng(seed)
    Xs, ys, gs = [], [], []
    for g, (n, cp, ri, v, posdef) in enumerate(problems):
        a = smfg.analyse(n, cp, ri)
        scale = None if posdef else smfg.matching_scale(n, cp, ri, v)[0]
        sv = smfg.Solver(a, device=device)
        sv.factor(v, posdef=posdef, scale=scale)
        stp = sv.front_stats()
        X = front_features(a, v, posdef, stp, scale)
        cand = candidates(a)
        for r in range(runs):
            mask = (cand & (rng.random(a.nsn) < share)).astype(np.int8)
            if not mask.any():
                continue
            sv.set_front_precision(mask)
            sv.factor(v, posdef=posdef, scale=scale, precision=smfg.PREC_MIXED, mixed_kind=r % 2)
            lab = outcome_labels(a, stp, sv.front_stats(), mask)
            sel = lab >= 0
            Xs.append(X[sel])
            ys.append(lab[sel].astype(np.float32))
            gs.append(np.full(int(sel.sum()), g))
        sv.close()
    if not Xs:
        return np.zeros((0, N_FEATURES), np.float32), np.zeros(0, np.float32), np.zeros(0, np.int64)
    return np.concatenate(Xs), np.concatenate(ys), np.concatenate(gs)


def save(sel: "Selector", path: str):
    np.savez(path, P=sel.P.cpu().numpy(), mu=sel.mu.numpy(), sd=sel.sd.numpy(), d=sel.d, h=sel.h,
             threshold=sel.threshold)


def load(path: str, device: int = 0) -> "Selector":
    z = np.load(path)
    sel = Selector(int(z["d"]), int(z["h"]), device=device)
    t = sel.torch
    sel.P = t.as_tensor(z["P"]).float().to(sel.dev).contiguous()
    sel.mu = t.as_tensor(z["mu"])
    sel.sd = t.as_tensor(z["sd"])
    sel.threshold = float(z["threshold"])
    return sel


def training_problems(count: int = 36, seed: int = 0):
    """The synthetic training families: interior-point KKTs of several sizes,
    constraint counts and barrier ranges, and SPD variable-coefficient grids
    (workloads.py's generators)."""
    from . import workloads as W
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        if i % 4 == 3:
            out.append(W.varcoef_3d(int(rng.integers(16, 25)), seed=1000 + i) + (True,))
        else:
            m = int(rng.integers(10, 17))
            ncon = int(rng.integers(m ** 3 // 4, m ** 3 // 2))
            lo = float(rng.uniform(-10, -4))
            out.append(W.kkt_ipm(m, ncon, seed=2000 + i, sigma_range=(lo, -lo)) + (False,))
    return out


def main(argv=None):
    """python -m opt_solver_b200.selector OUT.npz: train the selector on the
    solver's outcomes over the synthetic families and save it."""
    import sys
    argv = sys.argv[1:] if argv is None else argv
    out = argv[0] if argv else "selector.npz"
    X, y, _ = collect_outcomes(training_problems(), runs=4, seed=1)
    sel = Selector(N_FEATURES, 16, seed=0)
    hist = sel.fit(X, y, epochs=500, lr=0.02)
    p = sel.predict(X)
    acc = float(np.mean((p >= sel.threshold) == (y > 0.5)))
    print(f"samples {len(y)}, positive share {y.mean():.3f}, loss {hist[0]:.4f} -> {hist[-1]:.4f}, "
          f"training accuracy {acc:.3f}")
    save(sel, out)


if __name__ == "__main__":
    main()
