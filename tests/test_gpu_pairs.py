"""GPU parity of eqtl_test_pairs (the FP64 pair tests behind the gene-level
permutations) against the oracle's per-column prep and tests: LM with a
fresh residualisation per column, LMM with a fresh REML fit per column."""
import numpy as np
import pytest

import restate as R
from gpu_util import log10_diff

pytestmark = pytest.mark.gpu


def _case(seed, n=160, m=400, G=12, ncov=2):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=2, chrom_len=2_000_000, miss_rate=0.02, maf_lo=0.02,
                             family=(6, 5, n - 30))
    Y, C = synth.make_pheno_lm(seed + 1, g, G, ncov, cis_effects=False, n_trans=6, beta_sd=0.5)
    X = np.column_stack([np.ones(n), C])
    return g, synth.pack_bed_rows(g.codes), Y, X


def _pairs(G, m, k, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, G, k).astype(np.int32), rng.integers(0, m, k).astype(np.int64)


@pytest.mark.parametrize("model", ["lm", "lmm"])
def test_test_pairs_matches_oracle(model):
    from eqtl_b200 import capi
    g, rows, Y, X = _case(31)
    n = g.codes.shape[1]
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Gd = dec.dosage[k]
    cols, snps = _pairs(Y.shape[1], k.size, 600, 5)
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        if model == "lmm":
            Kr, _, _ = R.compute_grm(Gd, dec.codes[k] < 0)
            Q, lam = R.make_lmm_basis(Kr)
            c.set_basis(Q, lam)
        out, delta = c.test_pairs(model, Y, X, cols, snps)
    _, ok = R.subset_maf(Gd)
    for j in range(Y.shape[1]):
        sel = np.nonzero(cols == j)[0]
        if sel.size == 0:
            continue
        if model == "lm":
            st = R.test_lm_many(R.prep_lm(Y[:, j], X), Gd[snps[sel]])
            rel = 1e-9
        else:
            prep = R.prep_lmm(Y[:, j], X, Q, lam)
            assert abs(delta[j] - prep.delta) <= 1e-5 * abs(prep.delta)
            if delta[j] != prep.delta:
                # the REML objective is flat at its optimum: both deltas must
                # reach the same minimum, and the statistics are compared at
                # the device's delta (beta moves ~1e-6 across that flat part)
                yt, Xt, df = Q.T @ Y[:, j], Q.T @ X, n - X.shape[1]
                f_dev = R.reml_negll(delta[j], yt, Xt, lam, df)
                f_ora = R.reml_negll(prep.delta, yt, Xt, lam, df)
                assert abs(f_dev - f_ora) <= 1e-9 * abs(f_ora), (j, delta[j], prep.delta, f_dev, f_ora)
                prep = R.prep_lmm(Y[:, j], X, Q, lam, delta=delta[j])
            st = R.test_lmm_many(prep, Gd[snps[sel]])
            rel = 1e-6
        gate = ok[snps[sel]]
        got = out[sel]
        assert np.all(np.isnan(got["p"][~gate]))
        assert np.all(log10_diff(got["p"][gate], st["p"][gate]) < max(1e-8, 100 * rel))
        np.testing.assert_allclose(got["beta"][gate], st["beta"][gate], rtol=rel, atol=1e-12)
        np.testing.assert_allclose(got["t"][gate], st["stat"][gate], rtol=10 * rel, atol=1e-10)
