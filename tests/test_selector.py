"""The learned per-front precision selector: its network's CUDA forward /
backward / Adam kernels against the FP64 NumPy oracle (oracle/mlp.py, itself
checked by finite differences), the features, the outcome labels, and what
the trained network gains: on held-out KKT systems, mixed factorizations
with the network's mask misjudge fewer fronts (fronts the plain-path judge
sends back to FP64) than mixing every large front."""
import numpy as np
import pytest

from opt_solver_b200 import workloads as W


def test_oracle_gradient_finite_differences():
    from oracle import mlp
    rng = np.random.default_rng(0)
    d, h, n = 6, 5, 40
    P = rng.normal(size=h * d + 2 * h + 1)
    X = rng.normal(size=(n, d))
    y = (rng.random(n) < 0.4).astype(float)
    w = rng.uniform(0.5, 2.0, n)
    loss, g = mlp.loss_and_grad(P, X, y, w, d, h)
    eps = 1e-6
    for i in range(P.size):
        e = np.zeros_like(P)
        e[i] = eps
        fd = (mlp.loss_and_grad(P + e, X, y, w, d, h)[0] - mlp.loss_and_grad(P - e, X, y, w, d, h)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), i


def test_features_and_labels():
    from opt_solver_b200 import selector as S
    from opt_solver_b200 import smfg
    n, cp, ri, v = W.kkt_ipm(8, 300, seed=1)
    a = smfg.analyse(n, cp, ri)
    st = np.zeros((a.nsn, 5), dtype=np.int32)
    st[:, 4] = 1
    X = S.front_features(a, v, False, st)
    assert X.shape == (a.nsn, S.N_FEATURES) and np.all(np.isfinite(X))
    assert np.all(X[:, 8] == 0.0) and np.all((X[:, 6] >= 0) & (X[:, 6] <= 1))
    # labels: a mixed front is good iff it and its parent kept their counts
    parent = np.asarray(a.sn_parent)
    s = int(np.nonzero(parent >= 0)[0][0])
    mask = np.zeros(a.nsn, np.int8)
    mask[s] = 1
    st2 = st.copy()
    assert S.outcome_labels(a, st, st2, mask)[s] == 1
    st2[parent[s], 4] += 1
    lab = S.outcome_labels(a, st, st2, mask)
    assert lab[s] == 0 and np.all(lab[np.arange(a.nsn) != s] == -1)


@pytest.mark.gpu
def test_mlp_kernels_against_oracle():
    import torch
    from opt_solver_b200 import selector as S
    from oracle import mlp
    rng = np.random.default_rng(1)
    d, h, n = 10, 16, 700
    sel = S.Selector(d, h, seed=3)
    P = sel.P.cpu().numpy().astype(np.float64)
    X = rng.normal(size=(n, d)).astype(np.float32)
    y = (rng.random(n) < 0.3).astype(np.float32)
    w = rng.uniform(0.5, 2.0, n).astype(np.float32)
    # the kernels see standardized inputs: identity standardization
    sel.mu = torch.zeros(d)
    sel.sd = torch.ones(d)
    p = sel.predict(X)
    pr, _, _ = mlp.forward(P, X.astype(np.float64), d, h)
    assert np.max(np.abs(p - pr)) <= 2e-6
    dev = sel.dev
    g, loss = sel.grad(torch.as_tensor(X).to(dev), torch.as_tensor(y).to(dev), torch.as_tensor(w).to(dev))
    lr_, gr = mlp.loss_and_grad(P, X, y, w, d, h)
    g = g.cpu().numpy()
    assert abs(loss - lr_) <= 1e-5 * max(1.0, abs(lr_))
    assert np.max(np.abs(g - gr)) <= 1e-5 * max(1.0, np.max(np.abs(gr)))
    # deterministic: the same gradient twice
    g2, _ = sel.grad(torch.as_tensor(X).to(dev), torch.as_tensor(y).to(dev), torch.as_tensor(w).to(dev))
    assert np.array_equal(g, g2.cpu().numpy())


def _kkt_problems(seeds):
    return [W.kkt_ipm(12 + s % 4, 900 + 300 * (s % 3), seed=s) + (False,) for s in seeds]


@pytest.mark.gpu
def test_selector_learns_and_gains():
    from opt_solver_b200 import selector as S
    from opt_solver_b200 import smfg
    X, y, g = S.collect_outcomes(_kkt_problems(range(0, 24)), runs=4, seed=7)
    assert 0 < y.mean() < 1
    sel = S.Selector(S.N_FEATURES, 16, seed=0)
    hist = sel.fit(X, y, epochs=400, lr=0.02)
    assert hist[-1] < 0.9 * hist[0]
    bad_all = bad_sel = accepted = candidates = 0
    for s in range(100, 108):  # held-out systems
        n, cp, ri, v, posdef = _kkt_problems([s])[0]
        a = smfg.analyse(n, cp, ri)
        scale = smfg.matching_scale(n, cp, ri, v)[0]
        sv = smfg.Solver(a, device=0)
        ip = sv.factor(v, posdef=False, scale=scale)
        stp = sv.front_stats()
        cand = S.candidates(a).astype(np.int8)
        Xf = S.front_features(a, v, False, stp, scale)
        m = sel.mask(a, Xf)
        i1, _, b1 = S.factor_checked(sv, a, v, False, cand, stp, ip.inertia, scale)
        i2, _, b2 = S.factor_checked(sv, a, v, False, m, stp, ip.inertia, scale)
        assert i1.inertia == i2.inertia == ip.inertia
        bad_all += b1
        bad_sel += b2
        accepted += int(m.sum())
        candidates += int(cand.sum())
        sv.close()
    print(f"misjudged fronts: all large fronts mixed {bad_all}, selector {bad_sel}; "
          f"selector kept {accepted} of {candidates} large fronts mixed")
    assert accepted > 0
    assert bad_sel < bad_all
