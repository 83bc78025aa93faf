"""GPU parity for dosage rows (eqtl_geno_load_dosage: a VCF's FORMAT/DS
values, src/vcf_session.cpp:193-258): integer dosages give what the same
calls as .bed rows give, and continuous dosages match the oracle through the
decode, the GRM and the LM and LMM scans."""
import numpy as np
import pytest

import oracle_scan
import restate as R
from gpu_util import T_ERRS, check_scan as _check_scan
from test_gpu_lmm import _at_device_delta

pytestmark = pytest.mark.gpu


def _ds_from(codes, seed, sd=0.15, extra_miss=0.01):
    """Imputed-style dosages near the calls: clip(call + N(0, sd), 0, 2) in
    FP32, NaN where the call is missing and at a further `extra_miss` of the
    entries."""
    rng = np.random.default_rng(seed)
    ds = np.clip(codes + rng.normal(0.0, sd, codes.shape), 0.0, 2.0)
    ds[(codes < 0) | (rng.random(codes.shape) < extra_miss)] = np.nan
    return ds.astype(np.float32)


def _lm_case(seed=5, n=300, m=3000, G=150, ncov=3):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=3, chrom_len=3_000_000, miss_rate=0.02, maf_lo=0.01)
    Y, C = synth.make_pheno_lm(seed + 1, g, G, ncov, cis_effects=False, n_trans=40, beta_sd=0.4)
    return g, synth.pack_bed_rows(g.codes), Y, np.column_stack([np.ones(n), C])


def _lmm_case(seed=7, n=256, m=2000, G=96, ncov=2):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=2, chrom_len=4_000_000, miss_rate=0.02, maf_lo=0.02,
                             family=(10, 6, 196))
    Y, C, _ = synth.make_pheno_lmm(seed + 1, g, G, ncov, n_trans=30, beta_sd=0.5)
    return g, Y, np.column_stack([np.ones(n), C])


def test_integer_dosages_equal_bed_rows():
    """The same calls as FP32 dosage rows and as .bed rows: the decode is
    bit-identical (integer sums), and so are the scan's tested sets and best
    SNPs; statistics agree to FP64 summation order."""
    from eqtl_b200 import capi
    g, rows, Y, X = _lm_case(seed=13)
    n = g.codes.shape[1]
    sel = np.random.default_rng(3).permutation(n)[:220]
    ds = np.where(g.codes < 0, np.nan, g.codes).astype(np.float32)
    with capi.Context(0) as c:
        out = []
        for load in ("bed", "dosage", "bed"):
            if load == "bed":
                kp, af, nm = c.load_bed(rows, n, sel, 1, 0.05, 0.02)
            else:
                kp, af, nm = c.load_dosage(ds, sel, 1, 0.05, 0.02)
            dos = c.dosage(0, c.n_kept)
            genes, pairs, _ = c.scan_trans_lm(Y[sel], X[sel], pthr=1e-3)
            K, N, mu = c.grm()
            out.append((kp, af, nm, dos, genes, pairs, K, N, mu))
    for o in out[1:]:
        for a, b in zip(out[0][:4], o[:4]):
            assert np.array_equal(a, b)
        gb, gd = out[0][4], o[4]
        assert np.array_equal(gb["n_tested"], gd["n_tested"]) and np.array_equal(gb["best_snp"], gd["best_snp"])
        np.testing.assert_allclose(gd["best_p"], gb["best_p"], rtol=1e-12)
        pb, pd = out[0][5], o[5]
        assert np.array_equal(pb["snp"], pd["snp"]) and np.array_equal(pb["gene"], pd["gene"])
        for f in ("beta", "se", "t", "p"):
            np.testing.assert_allclose(pd[f], pb[f], rtol=1e-12)
        assert np.array_equal(out[0][7], o[7]) and out[0][8] == o[8]
        np.testing.assert_allclose(o[6], out[0][6], rtol=0, atol=1e-12 * np.abs(out[0][6]).max())


@pytest.mark.parametrize("prec", [0, 1])
def test_continuous_dosage_lm_matches_oracle(prec):
    from eqtl_b200 import capi
    g, _, Y, X = _lm_case()
    n = g.codes.shape[1]
    ds = _ds_from(g.codes, 21)
    with capi.Context(0, precision=prec) as c:
        keep, af, nm = c.load_dosage(ds, np.arange(n))
        got = c.dosage(0, c.n_kept)
        res = c.scan_trans_lm(Y, X, pthr=1e-3)
    dec = R.decode_dosage_rows(ds, np.arange(n), "impute", 0.8, 0.0)
    assert np.array_equal(keep, dec.keep) and np.array_equal(nm, dec.n_miss)
    np.testing.assert_allclose(af, dec.af, rtol=1e-14)
    np.testing.assert_allclose(got, dec.dosage[dec.keep], rtol=1e-14)
    ora, pairs_ref = oracle_scan.trans_lm(dec.dosage[dec.keep], Y, X, 1e-3)
    _check_scan(res, ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[prec])


def test_continuous_dosage_grm_and_lmm_match_oracle():
    from eqtl_b200 import capi
    g, Y, X = _lmm_case()
    n = g.codes.shape[1]
    ds = _ds_from(g.codes, 22)
    dec = R.decode_dosage_rows(ds, np.arange(n), "impute", 0.8, 0.0)
    k = np.nonzero(dec.keep)[0]
    Kr, Nr, mr = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    Q, lam = R.make_lmm_basis(Kr)
    with capi.Context(0) as c:
        c.load_dosage(ds, np.arange(n))
        K, N, mu = c.grm()
        c.set_basis(Q, lam)
        res = c.scan_trans_lmm(Y, X, pthr=1e-3)
    assert mu == mr and np.array_equal(N, Nr)
    np.testing.assert_allclose(K, Kr, rtol=0, atol=2e-6 * np.abs(Kr).max())
    ora, pairs_ref = oracle_scan.trans_lmm(dec.dosage[k], Y, X, Q, lam, 1e-3)
    ora, pairs_ref = _at_device_delta(res[3], ora, pairs_ref, dec.dosage[k], Y, X, Q, lam)
    _check_scan(res[:3], ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[0], rel=1e-6)
