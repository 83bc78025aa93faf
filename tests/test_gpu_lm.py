"""GPU parity: bed decode and the trans/gw LM scan through the C ABI against
the numpy oracle (oracle/restate.py)."""
import numpy as np
import pytest

import oracle_scan
import restate as R
from gpu_util import T_ERR, T_ERRS, acat_p_from, check_scan as _check_scan, log10_diff

pytestmark = pytest.mark.gpu


def _case(seed=5, n=300, m=3000, G=150, ncov=3, miss=0.02):
    from eqtl_b200 import synth
    g = synth.make_genotypes(seed, n=n, m=m, n_chrom=3, chrom_len=3_000_000, miss_rate=miss, maf_lo=0.01)
    Y, C = synth.make_pheno_lm(seed + 1, g, G, ncov, cis_effects=False, n_trans=40, beta_sd=0.4)
    X = np.column_stack([np.ones(n), C])
    rows = synth.pack_bed_rows(g.codes)
    return g, rows, Y, X


@pytest.fixture(scope="module")
def ctx():
    from eqtl_b200 import capi
    with capi.Context(0) as c:
        yield c


@pytest.mark.parametrize("miss_hand,max_miss,maf", [(1, 0.8, 0.0), (1, 0.01, 0.05), (0, 0.8, 0.0)])
def test_decode_bit_exact(ctx, miss_hand, max_miss, maf):
    g, rows, _, _ = _case(seed=11, n=257, m=700)
    n = g.codes.shape[1]
    perm = np.random.default_rng(3).permutation(n)[:200]     # analysis subset, shuffled order
    keep, af, nm = ctx.load_bed(rows, n, perm, miss_hand, max_miss, maf)
    dec = R.decode_bed_rows(rows, n, perm, "impute" if miss_hand == 1 else "filter", max_miss, maf)
    assert np.array_equal(keep, dec.keep)
    assert np.array_equal(nm, dec.n_miss)
    assert np.array_equal(af, dec.af)                       # bit-exact FP64
    k = np.nonzero(dec.keep)[0]
    got = ctx.dosage(0, k.size)
    assert np.array_equal(got, dec.dosage[k])               # bit-exact incl. imputed means


@pytest.mark.parametrize("prec", [0, 1])
def test_trans_lm_gw_matches_oracle(prec):
    from eqtl_b200 import capi
    g, rows, Y, X = _case()
    n = g.codes.shape[1]
    with capi.Context(0, precision=prec) as c:
        keep, _, _ = c.load_bed(rows, n, np.arange(n))
        res = c.scan_trans_lm(Y, X, pthr=1e-3)
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    Gd = dec.dosage[dec.keep]
    ora, pairs_ref = oracle_scan.trans_lm(Gd, Y, X, 1e-3)
    _check_scan(res, ora, pairs_ref, 1e-3, n - X.shape[1] - 1, t_err=T_ERRS[prec])


def test_trans_lm_excludes_cis_windows(ctx):
    g, rows, Y, X = _case(seed=21, G=130)
    n = g.codes.shape[1]
    keep, _, _ = ctx.load_bed(rows, n, np.arange(n))
    kidx = np.nonzero(keep)[0]
    chrom_id = {c: i for i, c in enumerate(sorted(set(g.chrom)))}
    schrom = np.array([chrom_id[g.chrom[s]] for s in kidx], np.int32)
    spos = g.pos[kidx]
    rng = np.random.default_rng(0)
    G = Y.shape[1]
    gchrom = rng.integers(-1, 3, G).astype(np.int32)        # -1 = gene without location
    center = rng.integers(1, 3_000_000, G)
    glo, ghi = np.maximum(center - 400_000, 1), center + 400_000
    res = ctx.scan_trans_lm(Y, X, pthr=1e-3, windows=(gchrom, glo, ghi, schrom, spos, True))
    excl = oracle_scan.windows_mask(schrom, spos, gchrom, glo, ghi)
    ora, pairs_ref = oracle_scan.trans_lm(g_dos := R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8,
                                                                      0.0).dosage[kidx], Y, X, 1e-3, excl=excl)
    _check_scan(res, ora, pairs_ref, 1e-3, n - X.shape[1] - 1)


@pytest.mark.parametrize("shuffle_snps", [False, True])
def test_cis_scope_matches_oracle(ctx, shuffle_snps):
    """Scope 2 (cis): only each gene's window. SNPs in position order take the
    banded tile list; a shuffled SNP order takes the masked full grid."""
    g, rows, Y, X = _case(seed=23, G=140)
    n = g.codes.shape[1]
    order = np.random.default_rng(4).permutation(rows.shape[0]) if shuffle_snps else np.arange(rows.shape[0])
    rows_o = rows[order]
    keep, _, _ = ctx.load_bed(rows_o, n, np.arange(n))
    kidx = np.nonzero(keep)[0]
    chrom_id = {c: i for i, c in enumerate(sorted(set(g.chrom)))}
    schrom = np.array([chrom_id[g.chrom[order[s]]] for s in kidx], np.int32)
    spos = g.pos[order[kidx]]
    rng = np.random.default_rng(1)
    G = Y.shape[1]
    gchrom = rng.integers(-1, 3, G).astype(np.int32)
    center = np.sort(rng.integers(1, 3_000_000, G))
    glo, ghi = np.maximum(center - 300_000, 1), center + 300_000
    res = ctx.scan_trans_lm(Y, X, pthr=1e-2, windows=(gchrom, glo, ghi, schrom, spos, 2))
    inwin = oracle_scan.windows_mask(schrom, spos, gchrom, glo, ghi)
    dos = R.decode_bed_rows(rows_o, n, np.arange(n), "impute", 0.8, 0.0).dosage[kidx]
    ora, pairs_ref = oracle_scan.trans_lm(dos, Y, X, 1e-2, excl=~inwin)
    assert np.array_equal(res[0]["n_tested"], ora["n_tested"])
    _check_scan(res, ora, pairs_ref, 1e-2, n - X.shape[1] - 1)


def test_trans_lm_stage2_candidates(ctx):
    g, rows, Y, X = _case(seed=31, G=64)
    n = g.codes.shape[1]
    ctx.load_bed(rows, n, np.arange(n))
    genes, pairs, cands = ctx.scan_trans_lm(Y, X, pthr=1e-6, perm_thr=1e-2)
    dec = R.decode_bed_rows(rows, n, np.arange(n), "impute", 0.8, 0.0)
    ora, _ = oracle_scan.trans_lm(dec.dosage[dec.keep], Y, X, 1e-6)
    P = ora["stats"]["p"]
    want = {(s, gg) for s, gg in zip(*np.nonzero(P < 1e-2))}
    got = {(int(q["snp"]), int(q["gene"])) for q in cands}
    for k in want ^ got:
        assert abs(np.log10(P[k]) + 2) < 1e-6, k
    # sorted by gene, then p
    gs = cands["gene"]
    assert np.all(np.diff(gs) >= 0)
