"""Rounding of the interpolated LMM scan against the direct form, emulated in
numpy (csrc/lmm.cu: LmmNodeEpi, lr_split_kernel, lr_coef_kernel and the scan
epilogue's S = gg - a' A00^-1 a).

Both forms are emulated with the device's number formats: each operand split
into an FP16 hi/lo pair under a power-of-two scale (a row's largest entry in
[2^10, 2^11)), products hi*hi + hi*lo + lo*hi summed in FP32. The direct
form contracts Gt^2 and Gt against the genes' weights over all n samples;
the interpolated form first forms the node genes' gg and a_0 that way, then
scales each node column by a power of two, splits it again, and contracts it
with the genes' Lagrange weights (over each column scale, under a per-gene
power of two). On genes whose REML deltas span the search range, the
interpolated form's largest relative error in gg and in S stays within twice
the direct form's, and both stay below 2e-5 (the screening tolerance of the
GPU tests is stated in t, T_ERRS[0] = 2e-6, about half the relative error of
S for t near the candidate threshold)."""
import numpy as np

from test_lmm_interp import NODES, nodes, weights


def _split(x, axis):
    m = np.abs(x).max(axis=axis, keepdims=True)
    m[m == 0] = 1.0
    sc = 2.0 ** (10 - np.floor(np.log2(m)))
    y = x * sc
    hi = y.astype(np.float16).astype(np.float64)
    lo = (y - hi).astype(np.float16).astype(np.float64)
    return hi, lo, sc


def _mm3(A, B):
    """A [s, k] (rows split) times B [k, g] (columns split), FP32 sums."""
    ah, al, sa = _split(A, 1)
    bh, bl, sb = _split(B, 0)
    f = np.float32
    acc = ah.astype(f) @ bh.astype(f) + ah.astype(f) @ bl.astype(f) + al.astype(f) @ bh.astype(f)
    return acc.astype(np.float64) / sa / sb


def _colscale(P):
    m = np.abs(P).max(0)
    out = np.zeros_like(m)
    nz = m > 0
    out[nz] = 2.0 ** (14 - np.floor(np.log2(m[nz])))
    return out


def test_interpolated_rounding_matches_the_direct_form():
    rng = np.random.default_rng(7)
    n, m, G = 400, 600, 240
    # a GRM with family structure: 40 families of 5 plus unrelated samples
    fam = np.repeat(np.arange(40), 5)
    Z = rng.standard_normal((n, 3000))
    Z[:200] += 1.5 * rng.standard_normal((40, 3000))[fam]
    Z = (Z - Z.mean(0)) / Z.std(0)
    lam, Q = np.linalg.eigh(Z @ Z.T / Z.shape[1])
    lam = np.clip(lam, 0, None)
    maf = rng.uniform(0.02, 0.5, m)
    D = rng.binomial(2, maf[:, None], (m, n)).astype(np.float64)
    Gt = (D - D.mean(1, keepdims=True)) @ Q                    # rotated SNPs [m, n]
    X0 = Q.T @ np.ones(n)                                        # rotated intercept
    delta = np.exp(rng.uniform(np.log(1e-8), np.log(1e6), G))
    W = 1.0 / (1.0 + np.outer(lam, delta))
    gg, a0, A00 = (Gt ** 2) @ W, Gt @ (X0[:, None] * W), (X0 ** 2) @ W
    S = gg - a0 ** 2 / A00

    # direct form
    gg_d, a0_d = _mm3(Gt ** 2, W), _mm3(Gt, X0[:, None] * W)
    # interpolated form: node genes, column scales, Lagrange weights
    a = np.log(delta)
    na, lo, h, nint = nodes(a.min(), a.max())
    Wn = 1.0 / (1.0 + np.outer(lam, np.exp(na)))
    Pg, Pa = _mm3(Gt ** 2, Wn), _mm3(Gt, X0[:, None] * Wn)
    L = np.zeros((na.size, G))
    for g in range(G):
        base, lw = weights(a[g], na, lo, h, nint)
        L[base:base + NODES, g] = lw
    sg, sa = _colscale(Pg), _colscale(Pa)
    inv = lambda s: np.where(s > 0, 1.0 / np.where(s > 0, s, 1.0), 0.0)   # noqa: E731
    gg_l = _mm3(Pg * sg, L * inv(sg)[:, None])
    a0_l = _mm3(Pa * sa, L * inv(sa)[:, None])

    def worst(g_, a_):
        return float(np.max(np.abs(g_ - gg) / gg)), float(np.max(np.abs(g_ - a_ ** 2 / A00 - S) / S))

    gd, sd = worst(gg_d, a0_d)
    gl, sl = worst(gg_l, a0_l)
    assert gl <= 2 * gd + 1e-7 and sl <= 2 * sd + 1e-7, (gd, sd, gl, sl)
    assert max(gd, sd, gl, sl) < 2e-5, (gd, sd, gl, sl)
