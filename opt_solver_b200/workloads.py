"""Seeded synthetic matrices with the shapes of the benchmark configurations.

All matrices are returned as lower-triangular CSC (``col_ptr``, ``row_idx``,
``values``; int32 / float64 numpy arrays, rows sorted within each column),
the input format of smf's ``smf_csc_t`` (solver/include/smf/smf_c.h:143-159).
The data is synthetic: no public matrix collection is read.
"""
from __future__ import annotations

import numpy as np


def _csc_from_coo(n, rows, cols, vals):
    """Lower CSC from (row >= col) triplets, duplicates summed, rows sorted."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    lo = np.maximum(rows, cols)
    hi = np.minimum(rows, cols)
    key = hi * n + lo
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order]
    uniq, first = np.unique(key, return_index=True)
    summed = np.add.reduceat(vals, first) if len(vals) else vals
    c = (uniq // n).astype(np.int64)
    r = (uniq % n).astype(np.int32)
    col_ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(col_ptr, c + 1, 1)
    col_ptr = np.cumsum(col_ptr).astype(np.int32)
    return col_ptr, r, summed.astype(np.float64)


def laplacian_2d(nx: int, ny: int | None = None):
    """5-point Laplacian on an nx x ny grid with Dirichlet boundary: diagonal
    4, off-diagonals -1 (configuration 1 at 150 x 150, n = 22,500)."""
    ny = nx if ny is None else ny
    n = nx * ny
    idx = np.arange(n).reshape(ny, nx)
    r = [idx.ravel()]
    c = [idx.ravel()]
    v = [np.full(n, 4.0)]
    r.append(idx[:, 1:].ravel()); c.append(idx[:, :-1].ravel()); v.append(np.full(ny * (nx - 1), -1.0))
    r.append(idx[1:, :].ravel()); c.append(idx[:-1, :].ravel()); v.append(np.full((ny - 1) * nx, -1.0))
    return (n,) + _csc_from_coo(n, np.concatenate(r), np.concatenate(c), np.concatenate(v))


def _grid3d_edges(m: int):
    idx = np.arange(m ** 3).reshape(m, m, m)
    a = [idx[:, :, 1:].ravel(), idx[:, 1:, :].ravel(), idx[1:, :, :].ravel()]
    b = [idx[:, :, :-1].ravel(), idx[:, :-1, :].ravel(), idx[:-1, :, :].ravel()]
    return np.concatenate(a), np.concatenate(b)


def varcoef_3d(m: int, seed: int = 0):
    """SPD variable-coefficient 7-point operator on an m^3 grid: edge
    conductivities log-uniform in [1e-3, 1e3] from the seed, diagonal = sum of
    incident conductivities + 1e-6 (configuration 2 at m = 64)."""
    rng = np.random.default_rng(seed)
    n = m ** 3
    ea, eb = _grid3d_edges(m)
    cond = 10.0 ** rng.uniform(-3.0, 3.0, size=ea.size)
    diag = np.full(n, 1e-6)
    np.add.at(diag, ea, cond)
    np.add.at(diag, eb, cond)
    rows = np.concatenate([np.arange(n), ea])
    cols = np.concatenate([np.arange(n), eb])
    vals = np.concatenate([diag, -cond])
    return (n,) + _csc_from_coo(n, rows, cols, vals)


def kkt_ipm(m: int, n_con: int, seed: int = 0, delta: float = 1e-8,
            sigma_range=(-8.0, 8.0), sigma_scale: float = 1.0):
    """Indefinite interior-point KKT [H + Sigma, J^T; J, -delta I]: H the
    7-point Laplacian on m^3 (diagonal 6, off-diagonals -1), Sigma diagonal
    log-uniform in 10^sigma_range, J with n_con rows of 4 distinct random
    columns and N(0, 1) values (configuration 3 at m = 40, n_con = 32,000;
    expected inertia (m^3)+ / n_con-)."""
    rng = np.random.default_rng(seed)
    nh = m ** 3
    n = nh + n_con
    ea, eb = _grid3d_edges(m)
    sigma = sigma_scale * 10.0 ** rng.uniform(sigma_range[0], sigma_range[1], size=nh)
    jcols = np.stack([rng.choice(nh, size=4, replace=False) for _ in range(n_con)]) if n_con else np.zeros((0, 4), dtype=np.int64)
    jvals = rng.standard_normal(size=(n_con, 4))
    rows = [np.arange(nh), ea, nh + np.repeat(np.arange(n_con), 4), nh + np.arange(n_con)]
    cols = [np.arange(nh), eb, jcols.ravel(), nh + np.arange(n_con)]
    vals = [6.0 + sigma, np.full(ea.size, -1.0), jvals.ravel(), np.full(n_con, -delta)]
    return (n,) + _csc_from_coo(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def kkt_ipm_stream(m: int, n_con: int, steps: int = 8, seed: int = 0, wrong=(3, 6),
                   n_neg: int = 12, shift: float = 60.0, reg: float = 100.0):
    """An interior-point method's value stream on one kkt_ipm pattern: step 0
    the base values; every later step a barrier update (each Sigma entry
    times 10^U(-0.5, 0.5)); at the steps in ``wrong`` the Hessian block made
    indefinite (``n_neg`` diagonal entries set to -``shift``: more
    negative pivots than the n_con constraints give), and the step after each
    the method's inertia correction (the same values plus ``reg`` on the
    Hessian diagonal). Returns (n, col_ptr, row_idx, [values per step],
    [kind per step]) with kind "base", "barrier", "wrong" or "corrected"."""
    n, cp, ri, v0 = kkt_ipm(m, n_con, seed=seed)
    nh = m ** 3
    rng = np.random.default_rng(seed + 1000)
    hdiag = cp[:nh].astype(np.int64)       # rows sorted: a column's diagonal comes first
    sigma = v0[hdiag] - 6.0
    neg_rows = rng.choice(nh, size=min(n_neg, nh), replace=False)
    vals, kinds = [v0.copy()], ["base"]
    prev = v0
    for k in range(1, steps):
        if kinds[-1] == "wrong":
            v = prev.copy()
            v[hdiag] += reg
            kinds.append("corrected")
        else:
            v = v0.copy()
            v[hdiag] = 6.0 + sigma * 10.0 ** rng.uniform(-0.5, 0.5, size=nh)
            if k in wrong:
                v[hdiag[neg_rows]] = -shift
                kinds.append("wrong")
            else:
                kinds.append("barrier")
        vals.append(v)
        prev = v
    return n, cp, ri, vals, kinds


def trajectory_kkt(T: int, rng: np.random.Generator, nx: int = 12, nu: int = 4, eq_reg: float = 1e-9):
    """One trajectory-optimisation KKT system (configuration 4): stages
    [x_k, u_k, lambda_{k+1}] for k < T, then x_T; stage Hessians Q = G G^T +
    1e-6 I with G of (nx+nu) x 2(nx+nu) N(0, 1) entries (Wishart); dynamics
    x_{k+1} = A x_k + B u_k with A = I + 0.01 N(0, 1), B ~ N(0, 0.1^2);
    -eq_reg on the multipliers' diagonal. n = 28 T + 12 at nx = 12, nu = 4;
    inertia (16 T + 12, 12 T, 0)."""
    nz = nx + nu
    stride = nz + nx
    n = stride * T + nx
    A = np.eye(nx) + 0.01 * rng.standard_normal((nx, nx))
    B = 0.1 * rng.standard_normal((nx, nu))
    rows, cols, vals = [], [], []
    for k in range(T + 1):
        base = k * stride
        dim = nz if k < T else nx
        G = rng.standard_normal((dim, 2 * dim))
        Q = G @ G.T + 1e-6 * np.eye(dim)
        ii, jj = np.tril_indices(dim)
        rows.append(base + ii); cols.append(base + jj); vals.append(Q[ii, jj])
        if k < T:
            lam = base + nz
            nxt = base + stride
            # lambda rows: A x_k + B u_k - x_{k+1}
            li, lj = np.meshgrid(np.arange(nx), np.arange(nx), indexing="ij")
            rows.append(lam + li.ravel()); cols.append(base + lj.ravel()); vals.append(A.ravel())
            bi, bj = np.meshgrid(np.arange(nx), np.arange(nu), indexing="ij")
            rows.append(lam + bi.ravel()); cols.append(base + nx + bj.ravel()); vals.append(B.ravel())
            rows.append(nxt + np.arange(nx)); cols.append(lam + np.arange(nx)); vals.append(-np.ones(nx))
            rows.append(lam + np.arange(nx)); cols.append(lam + np.arange(nx)); vals.append(np.full(nx, -eq_reg))
    return (n,) + _csc_from_coo(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def trajectory_batch(count: int, seed: int = 0, t_min: int = 10, t_max: int = 200):
    """Configuration 4: `count` independent trajectory KKT systems with
    horizons uniform in {t_min..t_max}."""
    rng = np.random.default_rng(seed)
    horizons = rng.integers(t_min, t_max + 1, size=count)
    return [trajectory_kkt(int(T), rng) for T in horizons]


def rhs(n: int, nrhs: int = 1, seed: int = 0, kind: str = "uniform"):
    rng = np.random.default_rng(seed)
    if kind == "normal":
        b = rng.standard_normal((nrhs, n))
    else:
        b = rng.uniform(-1.0, 1.0, size=(nrhs, n))
    # nrhs > 1: shape (nrhs, n), i.e. the column-major n x nrhs block with
    # leading dimension n that smf's solve takes.
    return b if nrhs > 1 else b[0].copy()


def sigma_stream(n_sigma: int, count: int = 60, seed: int = 0, mu0: float = 1e-1, mu1: float = 1e-10,
                 sigma_range=(-8.0, 8.0)):
    """The barrier diagonals of an interior-point refactor stream
    (configuration 5): Sigma_k = Sigma_0 mu_k / mu_0 with mu geometric from
    mu0 to mu1 over `count` steps and per-entry multiplicative noise
    log-uniform in [0.5, 2]; Sigma_0 log-uniform in 10^sigma_range. Returns
    a (count, n_sigma) array."""
    rng = np.random.default_rng(seed)
    sigma0 = 10.0 ** rng.uniform(sigma_range[0], sigma_range[1], size=n_sigma)
    mus = np.geomspace(mu0, mu1, count)
    out = np.empty((count, n_sigma))
    for k in range(count):
        noise = 10.0 ** rng.uniform(np.log10(0.5), np.log10(2.0), size=n_sigma)
        out[k] = sigma0 * (mus[k] / mu0) * noise
    return out


def diagonal_slots(n, col_ptr, row_idx):
    """Positions of the diagonal entries in a lower CSC (one per column)."""
    cp = np.asarray(col_ptr, dtype=np.int64)
    ri = np.asarray(row_idx)
    cols = np.repeat(np.arange(n), np.diff(cp))
    pos = np.nonzero(ri == cols)[0]
    out = np.full(n, -1, dtype=np.int64)
    out[cols[pos]] = pos
    return out
