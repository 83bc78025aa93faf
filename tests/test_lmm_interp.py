"""The node design of the interpolated LMM scan (csrc/lmm.cu, lmm_lr_prepare
and lr_coef_kernel), restated in numpy: 5 or 11 equal intervals of ln(delta)
over the genes' range (the fewer that keeps each within 3), 12
Chebyshev-Lobatto nodes each (neighbours share their end node), and each
gene's Lagrange weights on its interval.

Pinned here: over the whole REML search range of delta (1e-8 to 1e6) and
eigenvalues from 0 to 50, the interpolated weights w_i = 1 / (1 + delta
lambda_i) are within 2^-22 relative of the exact ones (the precision to
which the FP16 hi/lo pair of the direct form holds w itself), and within
1e-9 over a range of delta of 1e4; the nodes fit one gene-side tile (128);
and the weights' absolute sums (the Lebesgue function, which bounds how
rounding in the node values can grow) stay below 5. The GPU tests
(test_gpu_lmm.py, test_gpu_fullsize.py) check the scan itself against the
oracle."""
import numpy as np

SPAN, NODES = 3.0, 12


def nodes(lo, hi):
    if hi - lo < 1e-6:
        lo, hi = lo - 0.5, hi + 0.5
    nint = 5 if int(np.ceil((hi - lo) / SPAN)) <= 5 else 11
    h = (hi - lo) / nint
    na = np.empty(nint * (NODES - 1) + 1)
    for q in range(nint):
        for i in range(NODES):
            na[q * (NODES - 1) + i] = lo + h * (q + 0.5 * (1.0 - np.cos(np.pi * i / (NODES - 1))))
    return na, lo, h, nint


def weights(a, na, lo, h, nint):
    q = min(max(int(np.floor((a - lo) / h)), 0), nint - 1)
    base = q * (NODES - 1)
    x = na[base:base + NODES]
    lw = np.array([np.prod([(a - x[i]) / (x[j] - x[i]) for i in range(NODES) if i != j]) for j in range(NODES)])
    return base, lw


def _worst(lam, delta):
    a = np.log(delta)
    na, lo, h, nint = nodes(a.min(), a.max())
    assert na.size <= 128
    assert np.all(np.diff(na) > 0)
    wn = 1.0 / (1.0 + np.outer(lam, np.exp(na)))
    worst, leb = 0.0, 0.0
    for ag, d in zip(a, delta):
        base, lw = weights(ag, na, lo, h, nint)
        w = 1.0 / (1.0 + d * lam)
        wi = wn[:, base:base + NODES] @ lw
        worst = max(worst, float(np.max(np.abs(wi - w) / w)))
        leb = max(leb, float(np.abs(lw).sum()))
    assert leb < 5.0, leb
    return worst


def test_interpolated_weights_over_the_search_range():
    rng = np.random.default_rng(3)
    lam = np.concatenate([[0.0, 1e-12, 1e-6], rng.uniform(0, 50, 400), np.exp(rng.uniform(-12, 3, 100))])
    delta = np.concatenate([[1e-8, 1e6], np.exp(rng.uniform(np.log(1e-8), np.log(1e6), 600))])
    assert _worst(lam, delta) < 2.0 ** -22
    narrow = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), 600))
    assert _worst(lam, narrow) < 1e-9


def test_narrow_and_single_delta_ranges():
    for a0, a1 in ((0.3, 0.3), (-2.0, -1.9), (1.0, 4.0), (1.0, 4.0001)):
        na, lo, h, nint = nodes(a0, a1)
        assert h <= SPAN + 1e-12 and na[0] <= a0 and na[-1] >= a1 - 1e-12
        for ag in np.linspace(a0, a1, 7):
            base, lw = weights(ag, na, lo, h, nint)
            assert abs(lw.sum() - 1.0) < 1e-12                # interpolation reproduces constants
            assert 0 <= base and base + NODES <= na.size
