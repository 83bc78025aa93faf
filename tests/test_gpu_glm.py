"""GPU parity: the NB-GLM scan (eqtl_scan_glm: null fit per gene, score test
per pair, src/model_glm.cpp:13-132) through the C ABI against the numpy
oracle, for one covariate column, two, and the grouped scan (p > 2), with
trans-window exclusion; and its refusal of non-count phenotypes."""
import numpy as np
import pytest

import oracle_scan
import restate as R
from gpu_util import T_ERR, check_scan as _check_scan

pytestmark = pytest.mark.gpu


def _case(seed=31, n=300, m=2500, G=80, ncov=1):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=3, chrom_len=3_000_000, miss_rate=0.02, maf_lo=0.02)
    Y, C = synth.make_pheno_counts(seed + 1, g, G, ncov, n_trans=25, beta_sd=0.4)
    X = np.column_stack([np.ones(n), C])
    return g, synth.pack_bed_rows(g.codes), Y, X


@pytest.mark.parametrize("ncov", [0, 1, 3])
def test_glm_matches_oracle(ncov):
    """p = 1 and 2: one TMEM group with the explicit (X'WX)^-1; p = 4: the
    grouped scan with orthonormalised covariate accumulators."""
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=31 + ncov, ncov=ncov)
    n = g.codes.shape[1]
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        genes, pairs, cands, phi, conv = c.scan_glm(Y, X, pthr=1e-3)
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    ora, pairs_ref = oracle_scan.glm(dec.dosage[dec.keep], Y, X, 1e-3)
    assert np.array_equal(conv, ora["converged"])
    np.testing.assert_allclose(phi, ora["phi"], rtol=1e-6)
    _check_scan((genes, pairs, cands), ora, pairs_ref, 1e-3, None, t_err=T_ERR, rel=1e-6)


def test_glm_trans_windows():
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=41, G=60, ncov=2)
    n = g.codes.shape[1]
    with capi.Context(0) as c:
        keep, _, _ = c.load_bed(rows, n, np.arange(n))
        kidx = np.nonzero(keep)[0]
        chrom_id = {ch: i for i, ch in enumerate(sorted(set(g.chrom)))}
        schrom = np.array([chrom_id[g.chrom[s]] for s in kidx], np.int32)
        spos = g.pos[kidx]
        rng = np.random.default_rng(2)
        G = Y.shape[1]
        gchrom = rng.integers(-1, 3, G).astype(np.int32)
        center = rng.integers(1, 3_000_000, G)
        glo, ghi = np.maximum(center - 300_000, 1), center + 300_000
        genes, pairs, cands, phi, conv = c.scan_glm(Y, X, pthr=1e-3, windows=(gchrom, glo, ghi, schrom, spos, True))
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    excl = oracle_scan.windows_mask(schrom, spos, gchrom, glo, ghi)
    ora, pairs_ref = oracle_scan.glm(dec.dosage[kidx], Y, X, 1e-3, excl=excl)
    _check_scan((genes, pairs, cands), ora, pairs_ref, 1e-3, None, t_err=T_ERR, rel=1e-6)


def test_glm_refuses_non_counts():
    from eqtl_b200 import capi
    g, rows, Y, X = _case(seed=51, G=8, m=400)
    n = g.codes.shape[1]
    Y = Y.copy()
    Y[3, 5] = 2.5
    with capi.Context(0) as c:
        c.load_bed(rows, n, np.arange(n))
        with pytest.raises(capi.EqtlError, match="non-negative integer counts"):
            c.scan_glm(Y, X, pthr=1e-3)
