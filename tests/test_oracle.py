"""Pins the numpy restatement (oracle/) against outputs of the reference
program itself (tests/golden/, made by tests/golden/make_golden.py)."""
import json
import math
import os

import numpy as np
import pytest

import driver
import restate as R
import refargs
import tsvcmp

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = [c for c in sorted(os.listdir(GOLD)) if os.path.isdir(os.path.join(GOLD, c))]


def _runs():
    out = []
    for c in CASES:
        man = json.load(open(os.path.join(GOLD, c, "manifest.json")))
        for tag, r in man["runs"].items():
            if r["argv"][0] != "fission":  # the fission subcommand has its own tests
                out.append((c, tag, r["argv"]))
    return out


def _models_scopes(opt):
    sc = ["gw"] if not opt.gff else {"cis": ["cis"], "trans": ["trans"], "gw": ["gw"],
                                      "all": ["cis", "trans"]}[opt.mode]
    return [(m, s) for m in opt.out_models for s in sc]


@pytest.mark.parametrize("case,tag,argv", [r for r in _runs() if "--make-grm" not in r[2]])
def test_scan_matches_reference(case, tag, argv):
    d = os.path.join(GOLD, case)
    opt = refargs.options_from_argv(argv, d)
    sc = driver.Scanner(opt)
    res = sc.run()
    tol = tsvcmp.Tol(log10p=1e-5, beta_rel=1e-6)
    errs = []
    for (model, scope), (pairs, tops, region) in res.items():
        pre = os.path.join(d, f"ref_{tag}.{model}.{scope}")
        pthr = opt.pval_cis if scope == "cis" else opt.pval_trans
        _, rp = tsvcmp.read_tsv(pre + ".pairs.tsv")
        _, rt = tsvcmp.read_tsv(pre + ".top.tsv")
        _, rr = tsvcmp.read_tsv(pre + ".region.tsv")
        errs += [f"{model}.{scope} pairs: {e}" for e in tsvcmp.compare_pairs(rp, pairs, tol, pthr)]
        errs += [f"{model}.{scope} top: {e}" for e in tsvcmp.compare_pairs(rt, tops, tol, pthr)]
        errs += [f"{model}.{scope} region: {e}" for e in tsvcmp.compare_region(rr, region, tol, acat_sens=sc.sens,
                                                                                   t_err=1e-7)]
    assert not errs, "\n".join(errs[:40])


@pytest.mark.parametrize("case,tag,argv", [r for r in _runs() if "--make-grm" in r[2]])
def test_grm_matches_reference(case, tag, argv):
    d = os.path.join(GOLD, case)
    opt = refargs.options_from_argv(argv, d)
    rows, n_file, fam, bim = R.read_bed(opt.bfile)
    dec = R.decode_bed_rows(rows, n_file, list(range(n_file)), opt.miss_hand, opt.max_miss, opt.maf)
    k = np.nonzero(dec.keep)[0]
    K, N, m = R.compute_grm(dec.dosage[k], dec.codes[k] < 0)
    n = n_file
    ref_bin = np.fromfile(os.path.join(d, f"ref_{tag}.grm.bin"), dtype=np.float32)
    ref_N = np.fromfile(os.path.join(d, f"ref_{tag}.grm.N.bin"), dtype=np.float32)
    assert ref_bin.size == n * (n + 1) // 2
    # integer denominators are bit-exact
    assert np.array_equal(ref_N, N.astype(np.float32))
    got = R.grm_lower_f32(K)
    np.testing.assert_allclose(got, ref_bin, rtol=1e-6, atol=1e-7)
    ids = [ln.split()[1] for ln in open(os.path.join(d, f"ref_{tag}.grm.id"))]
    assert ids == fam


def test_p_from_t_known_values():
    # t = 0 -> p = 1; symmetric; df large approaches the normal tail
    assert R.p_from_t(np.array([0.0]), 10)[0] == 1.0
    a = R.p_from_t(np.array([2.5, -2.5]), 30)
    assert a[0] == a[1]
    # independent implementation: scipy's regularised incomplete beta
    from scipy.special import betainc
    for t, df in [(3.0, 1e6), (0.1, 5), (7.5, 998), (40.0, 1998), (1e-7, 118)]:
        want = betainc(0.5 * df, 0.5, df / (df + t * t))
        assert abs(R.p_from_t(np.array([t]), df)[0] / want - 1) < 1e-9
    # non-finite t -> 1
    assert R.p_from_t(np.array([np.inf]), 10)[0] == 1.0


def test_shuffle_matches_reference_perm_file():
    # shuffle_indices is exercised end to end by the perm golden run (p_emp
    # only matches when every permutation matches); this checks invariants.
    idx = R.shuffle_indices(101, R.perm_seed(7, 3, "G00001"))
    assert sorted(idx) == list(range(101))
    assert idx != list(range(101))


def test_dosage_decode_restates_bed_decode():
    """decode_dosage_rows on integer dosages (NaN = missing) is the .bed
    decode of the same calls: keep flags, af, counts and imputed dosages."""
    from eqtl_b200 import synth
    g = synth.make_genotypes(31, n=97, m=400, n_chrom=2, chrom_len=1_000_000, miss_rate=0.05, maf_lo=0.005)
    rows = synth.pack_bed_rows(g.codes)
    ds = np.where(g.codes < 0, np.nan, g.codes).astype(np.float32)
    sel = np.random.default_rng(1).permutation(97)[:80]
    for hand, mm, maf in (("impute", 0.8, 0.0), ("impute", 0.03, 0.05), ("filter", 0.8, 0.0)):
        a = R.decode_bed_rows(rows, 97, sel, hand, mm, maf)
        b = R.decode_dosage_rows(ds, sel, hand, mm, maf)
        assert np.array_equal(a.keep, b.keep) and np.array_equal(a.n_miss, b.n_miss)
        assert np.array_equal(a.af, b.af)
        assert np.array_equal(a.dosage, b.dosage, equal_nan=True)
        assert np.array_equal(a.codes < 0, b.codes < 0)


def test_vcf_dosage_reader_restates_gt_reader(tmp_path):
    """Without an ID "DS" in the header read_vcf_dosage gives read_vcf_gt's
    records; with FORMAT/DS it reads the DS values as FP32 numbers."""
    from eqtl_b200 import synth
    rng = np.random.default_rng(2)
    d = rng.binomial(2, 0.3, (6, 10)).astype(np.int8)
    d[0, 3] = -1
    p = str(tmp_path / "a.vcf")
    synth.write_vcf(p, [f"s{i}" for i in range(10)], ["1"] * 6, list(range(1, 7)), [""] * 6, ["A"] * 6, ["C"] * 6, d)
    s1, r1, _ = R.read_vcf_gt(p)
    s2, r2, _ = R.read_vcf_dosage(p)
    assert s1 == s2 and len(r1) == len(r2)
    for a, b in zip(r1, r2):
        assert a[:5] == b[:5] and not b[7]
        assert np.array_equal(np.where(a[5] < 0, np.nan, a[5]), b[5], equal_nan=True)
    ds = rng.uniform(0, 2, (6, 10))
    ds[2, 4] = np.nan
    q = str(tmp_path / "b.vcf")
    synth.write_vcf(q, [f"s{i}" for i in range(10)], ["1"] * 6, list(range(1, 7)), [""] * 6, ["A"] * 6, ["C"] * 6, d,
                    ds=ds)
    _, r3, _ = R.read_vcf_dosage(q)
    got = np.stack([r[5] for r in r3])
    assert all(r[7] for r in r3)
    assert np.array_equal(got, ds.astype(np.float32).astype(np.float64), equal_nan=True)


def _read_matrix(path):
    rows = [ln.rstrip("\n").split("\t") for ln in open(path)]
    return rows[0][1:], [r[0] for r in rows[1:]], np.array([[float(v) for v in r[1:]] for r in rows[1:]])


@pytest.mark.parametrize("tag", ["counts", "cont", "covar"])
def test_peer_matches_reference(tag):
    """The PEER restatement from the reference's own starting values and its
    thinned Y1 (tests/golden/fission) gives the reference's factors to the
    6 significant digits the factors file carries."""
    if not os.path.exists(os.path.join(os.path.dirname(GOLD), "..", "oracle", "_ref", "stdnormal")):
        pytest.skip("oracle/_ref/stdnormal not built (make -C oracle)")
    d = os.path.join(GOLD, "fission")
    argv = json.load(open(os.path.join(d, "manifest.json")))["runs"][tag]["argv"]
    opt = dict(zip(argv[1::2], argv[2::2])) if len(argv) % 2 == 1 else {}
    k = int(opt["--peer-factors"])
    seed = int(opt.get("--seed", 42)) + 1
    genes, samples, Y1 = _read_matrix(os.path.join(d, f"ref_{tag}.Y1.tsv"))
    _, fs, F = _read_matrix(os.path.join(d, f"ref_{tag}.factors.tsv"))
    assert fs == samples
    Yp = Y1
    if "-c" in opt:
        Yp = R.fission_residualize(Y1, driver.load_covar(os.path.join(d, opt["-c"]), samples))
    X0, W0 = R.peer_start(seed, Y1.shape[0], Y1.shape[1], k)
    X, _ = R.peer_factors(Yp, k, int(opt.get("--fission-max-iter", 1000)), float(opt.get("--fission-tol", 1e-3)),
                          X0, W0)
    np.testing.assert_allclose(X, F, rtol=1e-5, atol=1e-5 * np.abs(F).max())
