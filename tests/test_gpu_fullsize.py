"""Parity at the benchmark shapes' full size (trans/gw LMM: n = 2,000,
m = 500,000 SNPs, 10,000 genes, the bench's synthetic workload; trans/gw LM:
n = 1,000, m = 1,000,000, 20,000 genes, 10 covariates), through properties
that do not depend on size, since the oracle cannot run 5e9 or 2e10 tests:

- every gene is tested on the same set of SNPs (gw scope: all SNPs that pass
  the subset gate), no more than the kept SNPs;
- every reported pair has p <= the threshold, and each gene's best p is no
  larger than that of any of its reported pairs;
- the scan's printed statistics equal an independent FP64 test of the same
  pairs through eqtl_test_pairs (which fits the null model again);
- for 200 reported and 200 random (gene, SNP) pairs the statistics match
  the oracle's FP64 restatement at the device's REML delta and eigenbasis
  (beta within 1e-6 relative, log10 p within 1e-6);
- for 20 genes (the 10 with the most reported pairs and 10 at random) the
  oracle tests every kept SNP in FP64 (at the device's delta and basis for
  the LMM): the number of tests, the set of pairs at p <= the threshold
  (identical except pairs within 1e-6 in log10 of it), the best SNP
  (identical or a near-tie) and acat_p (within 1e-3 in log10 plus the
  gene's sensitivity to the stated screening error of t).

A GRM at the GRM benchmark's shape (n = 2,000 with the family structure,
m = 200,000 SNPs) is checked against the oracle's FP64 GRM: N counts
bit-exact, K within 5e-6 of its largest entry. K's large positive sums (its
diagonal and related pairs) carry the drift of the tensor cores' FP32
accumulation over one K range of 512 SNPs (about 3e-6 relative); the
ranges meet in FP64."""
import argparse
import os
import sys

import numpy as np
import pytest

import restate as R
from gpu_util import T_ERR, acat_p_from, log10_diff

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

CHUNK = 25_000  # kept SNPs the oracle holds at once


def pick_genes(genes, pairs, rng, k=10):
    """The k genes with the most reported pairs and k others at random."""
    cnt = np.bincount(pairs["gene"], minlength=len(genes))
    top = np.argsort(-cnt, kind="stable")[:k]
    rest = np.setdiff1d(np.arange(len(genes)), top)
    return np.concatenate([top, rng.choice(rest, size=k, replace=False)]).astype(np.int64)


def check_gene_sets(sel, stats_of_chunk, rows_kept, n, genes, pairs, pthr, df):
    """Every kept SNP against the genes `sel` in FP64: stats_of_chunk(dosage
    rows [c, n]) -> dict of [c, len(sel)] arrays (the oracle's statistics)."""
    G = len(sel)
    acc = [R.AcatAcc() for _ in range(G)]
    tested = np.zeros(G, np.int64)
    best_p = np.full(G, 2.0)
    best_s = np.full(G, -1, np.int64)
    ora_pairs = [dict() for _ in range(G)]
    p_of = [dict() for _ in range(G)]   # oracle p of the device's pairs and best SNPs
    dev_pairs = [dict() for _ in range(G)]
    pos = {int(g): j for j, g in enumerate(sel)}
    for q in pairs:
        j = pos.get(int(q["gene"]))
        if j is not None:
            dev_pairs[j][int(q["snp"])] = float(q["p"])
    dev_best = genes["best_snp"][sel]
    for c0 in range(0, rows_kept.shape[0], CHUNK):
        dec = R.decode_bed_rows(rows_kept[c0:c0 + CHUNK], n, np.arange(n), "impute", 0.8, 0.0)
        _, ok = R.subset_maf(dec.dosage)
        st = stats_of_chunk(dec.dosage)
        for j in range(G):
            pv, tv = st["p"][ok, j], st["stat"][ok, j]
            idx = np.nonzero(ok)[0] + c0
            tested[j] += pv.size
            acc[j].add_many(pv)
            acc[j].add_sensitivity(pv, tv, df)
            if pv.size:
                i = int(np.argmin(pv))             # first minimum (strict < in the reference)
                if pv[i] < best_p[j]:
                    best_p[j], best_s[j] = pv[i], idx[i]
            for i in np.nonzero(pv <= pthr)[0]:
                ora_pairs[j][int(idx[i])] = float(pv[i])
            for s in list(dev_pairs[j]) + [int(dev_best[j])]:
                if c0 <= s < c0 + CHUNK and ok[s - c0]:
                    p_of[j][s] = float(st["p"][s - c0, j])
    ap = acat_p_from(genes[sel])
    for j, g in enumerate(sel):
        assert genes["n_tested"][g] == tested[j], (g, genes["n_tested"][g], tested[j])
        for s in set(ora_pairs[j]) ^ set(dev_pairs[j]):
            pv = ora_pairs[j].get(s, dev_pairs[j].get(s))
            assert abs(np.log10(pv) - np.log10(pthr)) < 1e-6, (g, s, pv)
        for s in set(ora_pairs[j]) & set(dev_pairs[j]):
            assert log10_diff(ora_pairs[j][s], dev_pairs[j][s]) < 1e-6, (g, s)
        if dev_best[j] != best_s[j]:                # a near-tie
            assert log10_diff(p_of[j][int(dev_best[j])], best_p[j]) < 1e-4, (g, dev_best[j], best_s[j])
        tol = 1e-3 + 3 * acc[j].log10_sensitivity() * T_ERR
        assert log10_diff(ap[j], acc[j].p()) <= tol, (g, ap[j], acc[j].p(), tol)


@pytest.mark.gpu
def test_trans_lmm_full_size_properties():
    import bench
    from eqtl_b200 import capi
    args = argparse.Namespace(n=2000, m=500_000, genes=10_000, family=(50, 10, 1500))
    rows, Y, X, _ = bench.workload(args)
    n, G = Y.shape
    pthr = 1e-5
    with capi.Context(0) as c:
        keep, _, _ = c.load_bed(rows, n, np.arange(n, dtype=np.int32))
        lam, Q = c.lmm_basis(outputs=True)
        c.pheno_load(Y, X)
        genes, pairs, _, delta = c.scan_trans_lmm(None, None, pthr=pthr)
        kept_rows = np.nonzero(keep)[0]
        # the same test set for every gene, within the kept SNPs
        nt = genes["n_tested"]
        assert np.all(nt == nt[0]) and 0 < nt[0] <= kept_rows.size
        # reported pairs and best SNPs
        assert pairs.size > 0 and np.all(pairs["p"] <= pthr)
        best_p = genes["best_p"]
        pg = {}
        for q in pairs:
            pg[int(q["gene"])] = min(pg.get(int(q["gene"]), 1.0), float(q["p"]))
        for g, pmin in pg.items():
            assert best_p[g] <= pmin * (1 + 1e-12), (g, best_p[g], pmin)
        # an independent FP64 test of a sample of the reported pairs
        rng = np.random.default_rng(5)
        sel = rng.choice(pairs.size, size=min(2000, pairs.size), replace=False)
        again, d2 = c.test_pairs("lmm", Y, X, pairs["gene"][sel], pairs["snp"][sel])
        np.testing.assert_array_equal(d2, delta)
        for f in ("beta", "se", "t"):
            np.testing.assert_allclose(again[f], pairs[f][sel], rtol=1e-10, atol=0)
        np.testing.assert_allclose(np.log10(again["p"]), np.log10(pairs["p"][sel]), rtol=0, atol=1e-10)
        # the oracle on reported and random pairs, at the device's delta and basis
        rep = pairs[rng.choice(pairs.size, size=min(200, pairs.size), replace=False)]
        rg = rng.integers(0, G, 200)
        rs = rng.integers(0, nt[0], 200)
        cols = np.concatenate([rep["gene"], rg]).astype(np.int64)
        snps = np.concatenate([rep["snp"], rs]).astype(np.int64)
        dev, _ = c.test_pairs("lmm", Y, X, cols, snps)
    dec = R.decode_bed_rows(rows[kept_rows[snps]], n, np.arange(n), "impute", 0.8, 0.0)
    for k in range(cols.size):
        j = int(cols[k])
        prep = R.prep_lmm(Y[:, j], X, Q, lam, delta=delta[j])
        st = R.test_lmm_many(prep, dec.dosage[k:k + 1])
        assert abs(dev["beta"][k] - st["beta"][0]) <= 1e-6 * abs(st["beta"][0]) + 1e-12, (k, dev[k], st["beta"][0])
        assert abs(np.log10(dev["p"][k]) - np.log10(st["p"][0])) <= 1e-6, (k, dev["p"][k], st["p"][0])
    # every kept SNP against 20 genes in FP64, at the device's delta and basis
    sel = pick_genes(genes, pairs, rng)
    preps = [R.prep_lmm(Y[:, int(j)], X, Q, lam, delta=delta[int(j)]) for j in sel]
    check_gene_sets(sel, lambda D: R.lmm_stats_gtil_genes(preps, D @ Q), rows[kept_rows], n, genes, pairs, pthr,
                    n - X.shape[1] - 1)


@pytest.mark.gpu
def test_trans_lm_full_size_properties():
    """The trans/gw LM at its benchmark shape: n = 1,000, m = 1,000,000 SNPs,
    20,000 genes with Y ~ N(0, 1), intercept + 10 covariates (2e10 tests)."""
    from eqtl_b200 import capi, synth
    n, m, G = 1000, 1_000_000, 20_000
    rows, _, _ = synth.make_bed_rows_chunked(20261203, n, m, maf_lo=0.01, maf_hi=0.5, miss_rate=0.01)
    rng = np.random.default_rng(20261204)
    Y = rng.standard_normal((n, G))
    X = np.column_stack([np.ones(n), rng.standard_normal((n, 10))])
    pthr = 1e-5
    with capi.Context(0) as c:
        keep, _, _ = c.load_bed(rows, n, np.arange(n, dtype=np.int32))
        c.pheno_load(Y, X)
        genes, pairs, _ = c.scan_trans_lm(None, None, pthr=pthr)
        kept_rows = np.nonzero(keep)[0]
        nt = genes["n_tested"]
        assert np.all(nt == nt[0]) and 0 < nt[0] <= kept_rows.size
        assert pairs.size > 0 and np.all(pairs["p"] <= pthr)
        # about pthr of the tests under the null
        assert 0.5 * pthr * nt.sum() < pairs.size < 1.5 * pthr * nt.sum()
        rng = np.random.default_rng(6)
        sel = rng.choice(pairs.size, size=min(2000, pairs.size), replace=False)
        again, _ = c.test_pairs("lm", Y, X, pairs["gene"][sel], pairs["snp"][sel])
        for f in ("beta", "se", "t"):
            np.testing.assert_allclose(again[f], pairs[f][sel], rtol=1e-12, atol=0)
        rep = pairs[rng.choice(pairs.size, size=200, replace=False)]
        cols = np.concatenate([rep["gene"], rng.integers(0, G, 200)]).astype(np.int64)
        snps = np.concatenate([rep["snp"], rng.integers(0, nt[0], 200)]).astype(np.int64)
        dev, _ = c.test_pairs("lm", Y, X, cols, snps)
    dec = R.decode_bed_rows(rows[kept_rows[snps]], n, np.arange(n), "impute", 0.8, 0.0)
    for k in range(cols.size):
        st = R.test_lm_many(R.prep_lm(Y[:, int(cols[k])], X), dec.dosage[k:k + 1])
        assert abs(dev["beta"][k] - st["beta"][0]) <= 1e-9 * abs(st["beta"][0]) + 1e-13, (k, dev[k], st["beta"][0])
        assert abs(np.log10(dev["p"][k]) - np.log10(st["p"][0])) <= 1e-8, (k, dev["p"][k], st["p"][0])
    # every kept SNP against 20 genes in FP64
    sel = pick_genes(genes, pairs, rng)
    preps = [R.prep_lm(Y[:, int(j)], X) for j in sel]
    Ys = np.column_stack([pr.y_s for pr in preps])
    yty = np.array([pr.yty for pr in preps])
    XtX_inv = preps[0].XtX_inv

    def lm_chunk(D):  # test_lm_many's arithmetic for all selected genes at once
        g_s = D - ((D @ X) @ XtX_inv.T) @ X.T
        gtg = np.einsum("ij,ij->i", g_s, g_s)
        return R.lm_stats(gtg[:, None], g_s @ Ys, yty[None, :], n, X.shape[1])

    check_gene_sets(sel, lm_chunk, rows[kept_rows], n, genes, pairs, pthr, n - X.shape[1] - 1)


@pytest.mark.gpu
def test_grm_full_size():
    """The GRM at n = 2,000 (50 families of 10 siblings + 1,500 unrelated),
    m = 200,000 SNPs, 1% missing calls, against the oracle's FP64 GRM."""
    from eqtl_b200 import capi, synth
    n, m = 2000, 200_000
    rows, _, _ = synth.make_bed_rows_chunked(20261202, n, m, family=(50, 10, 1500), maf_lo=0.01, maf_hi=0.5,
                                             miss_rate=0.01)
    with capi.Context(0) as c:
        keep, _, _ = c.load_bed(rows, n, np.arange(n, dtype=np.int32))
        K, N, m_used = c.grm()
    dec = R.decode_bed_rows(rows[np.nonzero(keep)[0]], n, np.arange(n), "impute", 0.8, 0.0)
    Kr, Nr, mr = R.compute_grm(dec.dosage, dec.codes < 0)
    assert m_used == mr
    np.testing.assert_array_equal(N, Nr)
    np.testing.assert_allclose(K, Kr, rtol=0, atol=5e-6 * np.abs(Kr).max())
