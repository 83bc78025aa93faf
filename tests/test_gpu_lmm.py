"""GPU parity: GRM, eigenbasis, batched REML and the trans/gw LMM scan through
the C ABI against the numpy oracle."""
import numpy as np
import pytest

import oracle_scan
import restate as R
from gpu_util import T_ERRS, acat_p_from, check_scan as _check_scan, log10_diff

pytestmark = pytest.mark.gpu


def _case(seed=7, n=256, m=2000, G=96, ncov=0, miss=0.02, fam=(10, 6, 196)):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=2, chrom_len=4_000_000, miss_rate=miss, maf_lo=0.02,
                             family=fam)
    Y, C, _ = synth.make_pheno_lmm(seed + 1, g, G, ncov, n_trans=30, beta_sd=0.5)
    X = np.column_stack([np.ones(n), C]) if ncov else np.ones((n, 1))
    return g, synth.pack_bed_rows(g.codes), Y, X


@pytest.mark.parametrize("miss_hand", [1, 0])
def test_grm_matches_oracle(miss_hand):
    from eqtl_b200 import capi
    g, rows, _, _ = _case(seed=3, m=1500)
    n = g.codes.shape[1]
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n), miss_hand, 0.8, 0.0)
        K, N, mu = c.grm()
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute" if miss_hand else "filter", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, Nr, mr = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    assert mu == mr
    assert np.array_equal(N, Nr)                       # integer counts bit-exact
    np.testing.assert_allclose(K, Kr, rtol=0, atol=2e-6 * np.abs(Kr).max())
    np.testing.assert_allclose(np.diag(K), np.diag(Kr), rtol=2e-6)


def test_basis_eigenvalues():
    from eqtl_b200 import capi
    g, rows, _, _ = _case(seed=4, m=800)
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        lam, Q = c.lmm_basis(Kr)
    lr, Qr = np.linalg.eigh(Kr)
    lr = np.maximum(lr, 0)                             # make_lmm_basis clips at 0
    np.testing.assert_allclose(lam, lr, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(Q.T @ Q, np.eye(n), atol=1e-10)
    # sign-invariant: the clipped reconstruction Q diag(lambda) Q'
    np.testing.assert_allclose((Q * lam) @ Q.T, (Qr * lr) @ Qr.T, atol=1e-9)


@pytest.mark.parametrize("ncov,prec", [(0, 0), (1, 0), (0, 2), (2, 0), (5, 0), (20, 0), (0, 1), (1, 1), (5, 1)])
def test_trans_lmm_matches_oracle(ncov, prec):
    """ncov 0-1: three or four accumulators in one TMEM group; ncov 2, 5 and
    20 (p = 3, 6, 21): orthonormalised covariate accumulators in groups of
    four; p > 3 also takes the batched REML, and p = 21 its larger scratch
    instance. prec 0: split FP16 (the exact dosage slice for NUM and a_k
    where p <= 2); 1: split BF16 on both sides; 2: the FP32 CUDA-core
    comparator."""
    from eqtl_b200 import capi
    g, rows, Y, X = _case(ncov=ncov)
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    with capi.Context(0, precision=prec) as c:
        c.load_bed(rows, n, np.arange(n))
        c.set_basis(Q, lam)
        res = c.scan_trans_lmm(Y, X, pthr=1e-3)
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-3)
    ora, pairs_ref = _at_device_delta(res[3], ora, pairs_ref, dec.dosage[k], Y, X, Q, lam)
    _check_scan(res[:3], ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[1 if prec == 1 else 0], rel=1e-6)


@pytest.mark.parametrize("ncov", [0, 1])
def test_trans_lmm_interpolated_matches_oracle(ncov, monkeypatch):
    """gg and a_k interpolated between node deltas (EQTL_LMM_FORM=lr; the
    default from 256 genes on) on genes whose REML deltas span the search
    range: pure noise (delta at its lower end), mostly polygenic, and the
    rest. The direct form of the same scan agrees with the oracle too."""
    from eqtl_b200 import capi
    # n = 250 < k_pad = 256 leaves the padding column the exact operand needs
    g, rows, Y, X = _case(ncov=ncov, G=96, n=250, fam=(10, 6, 190))
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    rng = np.random.default_rng(11)
    Y = Y.copy()
    Y[:, :8] = rng.standard_normal((n, 8))
    Y[:, 8:16] = (Q * np.sqrt(lam)) @ rng.standard_normal((n, 8)) + 1e-3 * rng.standard_normal((n, 8))
    res = {}
    for form in ("lr", "direct"):
        monkeypatch.setenv("EQTL_LMM_FORM", form)
        with capi.Context(0) as c:
            c.load_bed(rows, n, np.arange(n))
            c.set_basis(Q, lam)
            res[form] = c.scan_trans_lmm(Y, X, pthr=1e-3)
            assert (c.lmm_form()[0] > 0) == (form == "lr")
    d = res["lr"][3]
    assert np.array_equal(d, res["direct"][3])            # REML does not depend on the form
    assert d.min() < 1e-4 and d.max() > 1e2, (d.min(), d.max())
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-3)
    ora, pairs_ref = _at_device_delta(d, ora, pairs_ref, dec.dosage[k], Y, X, Q, lam)
    for form in ("lr", "direct"):
        _check_scan(res[form][:3], ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)


@pytest.mark.parametrize("G", [1, 2])
def test_trans_lmm_interpolated_narrow_delta_range(G, monkeypatch):
    """A narrow range of deltas takes the smaller node layout: 5 intervals,
    56 nodes, K = 64 columns per accumulator (one gene: the degenerate range,
    widened by 1/2 on each side)."""
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=29, ncov=1, G=4, n=250, fam=(10, 6, 190))
    Y = Y[:, :G].copy()
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    monkeypatch.setenv("EQTL_LMM_FORM", "lr")
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        c.set_basis(Q, lam)
        res = c.scan_trans_lmm(Y, X, pthr=1e-2)
        nodes, cols = c.lmm_form()
    assert nodes > 0 and cols == (64 if nodes <= 64 else 128)
    if G == 1:
        assert (nodes, cols) == (56, 64)
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-2)
    ora, pairs_ref = _at_device_delta(res[3], ora, pairs_ref, dec.dosage[k], Y, X, Q, lam, pthr=1e-2)
    _check_scan(res[:3], ora, pairs_ref, 1e-2, n - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)


@pytest.mark.parametrize("form", ["lr", "direct"])
def test_trans_lmm_excludes_cis_windows(form, monkeypatch):
    """The trans scope: each gene's cis window excluded (genes without a
    location test every SNP). Windows of 0.8 Mb on 4 Mb chromosomes leave
    16-SNP chunks clear of a gene's window (the chunk-level shortcut) and
    chunks that straddle it (the per-pair test), in both forms of gg and a_k."""
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=23, ncov=1, G=96, n=250, fam=(10, 6, 190))
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    chrom_id = {c: i for i, c in enumerate(sorted(set(g.chrom)))}
    schrom = np.array([chrom_id[g.chrom[s]] for s in k], np.int32)
    spos = g.pos[k]
    rng = np.random.default_rng(2)
    G = Y.shape[1]
    gchrom = rng.integers(-1, 2, G).astype(np.int32)        # -1 = gene without location
    center = rng.integers(1, 4_000_000, G)
    glo, ghi = np.maximum(center - 400_000, 1), center + 400_000
    monkeypatch.setenv("EQTL_LMM_FORM", form)
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        c.set_basis(Q, lam)
        res = c.scan_trans_lmm(Y, X, pthr=1e-3, windows=(gchrom, glo, ghi, schrom, spos, True))
        assert (c.lmm_form()[0] > 0) == (form == "lr")
    excl = oracle_scan.windows_mask(schrom, spos, gchrom, glo, ghi)
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-3, excl=excl)
    ora, pairs_ref = _at_device_delta(res[3], ora, pairs_ref, dec.dosage[k], Y, X, Q, lam, excl=excl)
    _check_scan(res[:3], ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)


def _at_device_delta(d_dev, ora, pairs_ref, G, Y, X, Q, lam, pthr=1e-3, excl=None):
    """REML delta: wherever the device's delta differs from the oracle's, it
    must be an optimum of the same objective (-loglik within 1e-6 of the
    oracle's), and the statistics are then checked at the device's delta.
    The objective is flat at its optimum, so two FP64 runs of the same
    schedule stop at slightly different deltas (at the edge of the search,
    grid best 1e-5, the Newton polish differences with h = 1e-9 and follows
    FP64 rounding); with many covariates beta moves ~1e-5 across that flat
    part."""
    d_ora = ora["delta"]
    flat = d_dev != d_ora
    if not flat.any():
        return ora, pairs_ref
    df = Y.shape[0] - X.shape[1]
    Xt = Q.T @ X
    for j in np.nonzero(flat)[0]:
        yt = Q.T @ Y[:, j]
        f_dev, f_ora = R.reml_negll(d_dev[j], yt, Xt, lam, df), R.reml_negll(d_ora[j], yt, Xt, lam, df)
        assert abs(f_dev - f_ora) <= 1e-6 * abs(f_ora), (j, d_dev[j], d_ora[j], f_dev, f_ora)
    return oracle_scan.trans_lmm(G, Y, X, Q, lam, pthr, excl=excl, deltas=np.where(flat, d_dev, np.nan))


@pytest.mark.parametrize("ncov", [0, 3])
def test_cis_lmm_matches_oracle(ncov):
    """Scope 2 (cis) on the LMM paths: one TMEM group (p = 1, banded tiles of
    128 SNPs) and grouped accumulators (p = 4, banded tiles of 64 SNPs).
    beta / t within 1e-6 like the trans scans: genes whose REML delta sits at
    the top of the search (~3e5) weight K's null space ~1e5 times the rest,
    and S = gg - a'A00^-1 a cancels there, which the FP64 refinement meets by
    solving with the Cholesky factor of A00 as the reference solves with its
    LDLT factors."""
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=19, ncov=ncov)
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    chrom_id = {c: i for i, c in enumerate(sorted(set(g.chrom)))}
    schrom = np.array([chrom_id[g.chrom[s]] for s in k], np.int32)
    spos = g.pos[k]
    rng = np.random.default_rng(2)
    G = Y.shape[1]
    gchrom = rng.integers(0, 2, G).astype(np.int32)
    center = rng.integers(1, 4_000_000, G)
    glo, ghi = np.maximum(center - 500_000, 1), center + 500_000
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        c.set_basis(Q, lam)
        res = c.scan_trans_lmm(Y, X, pthr=1e-2, windows=(gchrom, glo, ghi, schrom, spos, 2))
    inwin = oracle_scan.windows_mask(schrom, spos, gchrom, glo, ghi)
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-2, excl=~inwin)
    ora, pairs_ref = _at_device_delta(res[3], ora, pairs_ref, dec.dosage[k], Y, X, Q, lam, 1e-2, ~inwin)
    assert np.array_equal(res[0]["n_tested"], ora["n_tested"])
    _check_scan(res[:3], ora, pairs_ref, 1e-2, n - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)


def test_trans_lmm_device_basis_statistics():
    """With the device's own eigenbasis (cuSOLVER signs) every statistic still
    matches: only permutations depend on eigenvector signs."""
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=17, G=64)
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        c.lmm_basis()                         # device GRM + cuSOLVER
        res = c.scan_trans_lmm(Y, X, pthr=1e-3)
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-3)
    np.testing.assert_allclose(res[3], ora["delta"], rtol=1e-4)
    _check_scan(res[:3], ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)
