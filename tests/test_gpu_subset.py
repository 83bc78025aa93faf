"""Per-gene sample subsets (eqtl_geno_subset): scans over a subset of the
analysis samples, with the SNPs imputed and filtered over every analysis
sample as the reference does before it subsets a SNP to a gene's keep set
(src/scan_trans_lm.cpp:121-151, src/scan_trans_lmm.cpp:192-228), against the
oracle given the same subset of the full-set dosages; and the full view back."""
import numpy as np
import pytest

import oracle_scan
import restate as R
from gpu_util import T_ERRS, check_scan

pytestmark = pytest.mark.gpu


def _case(seed=31, n=240, m=1500, G=60, ncov=2):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=3, chrom_len=3_000_000, miss_rate=0.03, maf_lo=0.01)
    Y, C = synth.make_pheno_lm(seed + 1, g, G, ncov, cis_effects=False, n_trans=30, beta_sd=0.4)
    X = np.column_stack([np.ones(n), C])
    return g, synth.pack_bed_rows(g.codes), Y, X


def _subset(n, frac=0.8, seed=5):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, int(frac * n), replace=False)).astype(np.int32)


def test_lm_on_a_subset_and_back():
    from eqtl_b200 import capi
    g, rows, Y, X = _case()
    n = g.codes.shape[1]
    S = _subset(n)
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    Gk = dec.dosage[dec.keep]                      # imputed over every analysis sample
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        full0 = c.scan_trans_lm(Y, X, pthr=1e-3)
        c.geno_subset(S)
        res = c.scan_trans_lm(Y[S], X[S], pthr=1e-3)
        c.geno_subset(None)
        full1 = c.scan_trans_lm(Y, X, pthr=1e-3)
    ora, pairs_ref = oracle_scan.trans_lm(Gk[:, S], Y[S], X[S], 1e-3)
    check_scan(res, ora, pairs_ref, 1e-3, S.size - X.shape[1] - 1, t_err=T_ERRS[0])
    # the full view again gives the first scan's results
    assert np.array_equal(full0[0], full1[0]) and np.array_equal(full0[1], full1[1])


def test_lmm_on_a_subset_with_its_sliced_grm():
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=41, ncov=1)
    n = g.codes.shape[1]
    S = _subset(n, 0.75, seed=9)
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, _, _ = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Ks = Kr[np.ix_(S, S)]                          # build_gene_ready's slice of the full GRM
    Q, lam = R.make_lmm_basis(Ks)
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        c.geno_subset(S)
        c.set_basis(Q, lam)
        res = c.scan_trans_lmm(Y[S], X[S], pthr=1e-3)
    Gs = dec.dosage[k][:, S]
    # the oracle at the device's REML deltas (the REML itself is checked
    # against the oracle's optimum in test_gpu_lmm.py)
    ora, pairs_ref = oracle_scan.trans_lmm(Gs, Y[S], X[S], Q, lam, 1e-3, deltas=res[3])
    check_scan(res[:3], ora, pairs_ref, 1e-3, S.size - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)


def test_subset_refusals():
    from eqtl_b200 import capi
    g, rows, Y, X = _case(m=300, G=5)
    n = g.codes.shape[1]
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        with pytest.raises(capi.EqtlError):
            c.geno_subset(np.array([5, 3], np.int32))        # not increasing
        with pytest.raises(capi.EqtlError):
            c.geno_subset(np.array([0, n], np.int32))        # out of range
        c.geno_subset(_subset(n))
        with pytest.raises(capi.EqtlError):
            c.grm()                                          # the GRM covers every sample
        c.geno_subset(None)
        c.grm()
