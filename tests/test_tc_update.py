"""The tensor-core split-product rank-k update (smfg_tc_update): the kernel
of the mixed-precision path's trailing updates, lower(C) -= L W^T.

Checked against the FP64 product (torch) with the split method's error
bound, against a plain FP32 product (TF32x3 must be at least as accurate),
and the strict upper triangle must be left untouched.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

CASES = [(300, 16, 0), (1000, 256, 0), (777, 100, 1), (128, 64, 0), (129, 65, 1), (2000, 33, 0),
         (513, 300, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,kind", CASES)
def test_tc_update_against_fp64(n, k, kind):
    from opt_solver_b200 import smfg
    g = torch.Generator().manual_seed(1000 * n + k)
    Lt = torch.randn(k, n, dtype=torch.float64, generator=g)
    # W = L D with D of mixed signs and magnitudes, as in an LDL^T front
    d = torch.exp(torch.randn(k, 1, dtype=torch.float64, generator=g)) * torch.sign(
        torch.randn(k, 1, dtype=torch.float64, generator=g))
    Wt = Lt * d
    Ct = torch.randn(n, n, dtype=torch.float64, generator=g) * 10
    dev = torch.device("cuda", 0)
    Ct_d, Lt_d, Wt_d = Ct.to(dev), Lt.to(dev), Wt.to(dev)
    smfg.tc_update(Ct_d, Lt_d, Wt_d, kind)
    got = Ct_d.cpu().T.numpy()          # column-major C
    C0 = Ct.T.numpy()
    L = Lt.T.numpy()
    W = Wt.T.numpy()
    exact = C0 - L @ W.T
    absprod = np.abs(L) @ np.abs(W).T
    low = np.tril(np.ones((n, n), dtype=bool))
    # upper triangle untouched, bit for bit
    assert np.array_equal(got[~low], C0[~low])
    err = np.abs(got - exact)[low]
    scale = absprod[low] + 1e-300
    # split error ~3 * 2^-22 (TF32) / 3 * 2^-17 (BF16) per product, plus
    # FP32 accumulation over 3k products
    unit = 2.0 ** -22 if kind == 0 else 2.0 ** -17
    bound = 4 * unit + 3 * k * 2.0 ** -24
    assert np.max(err / scale) <= bound, (np.max(err / scale), bound)
    if kind == 0:
        torch.backends.cuda.matmul.allow_tf32 = False
        p32 = (Lt_d.float().T @ Wt_d.float()).double().cpu().numpy()
        err32 = np.abs((C0 - p32) - exact)[low]
        # the tensor cores' FP32 accumulation truncates; the split products
        # stay within a small factor of a plain FP32 FMA product
        print(f"n={n} k={k}: max err TF32x3 {np.max(err):.3e}, FP32 {np.max(err32):.3e}, "
              f"mean {np.mean(err):.3e} / {np.mean(err32):.3e}")
        assert np.max(err) <= 8 * np.max(err32) + 1e-300
