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
  (beta within 1e-6 relative, log10 p within 1e-6)."""
import argparse
import os
import sys

import numpy as np
import pytest

import restate as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


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
