"""The eqtl host program (eqtl_b200/bin/eqtl) against outputs of the reference
program itself (tests/golden/): the same command lines, every pairs / top /
region file and the GCTA GRM files. Each command line runs twice: on the
golden PLINK files (-b) and on the same genotypes as a VCF (-v; the
reference's own VCF reader needs htslib, absent here, so the golden outputs
of the .bed runs are the reference for both).

Tolerances: LM pairs carry the FP64 refinement (log10 p within 1e-5, beta
within 1e-6 relative); LMM adds the REML optimiser difference (1e-4 and
1e-5). ACAT p uses the condition-aware bound of the parity tests (1e-3 plus
3 |dlog10 acat / dt| times the screening error of t, from the oracle).
Permutation p_emp is exact for the LM (same seeded shuffles, FP64 tests);
for the LMM the permuted phenotypes live in the eigenbasis, whose eigenvector
signs differ between Eigen and cuSOLVER, so p_emp / p_beta agree in
distribution only and are checked for presence."""
import json
import os
import subprocess

import numpy as np
import pytest

import driver
import restate as R
import refargs
import tsvcmp
from gpu_util import T_ERR

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIN = os.path.join(os.path.dirname(GOLD), "..", "eqtl_b200", "bin", "eqtl")


def _runs():
    out = []
    for c in sorted(os.listdir(GOLD)):
        if not os.path.isdir(os.path.join(GOLD, c)):
            continue
        man = json.load(open(os.path.join(GOLD, c, "manifest.json")))
        for tag, r in man["runs"].items():
            if r["argv"][0] != "fission":  # the fission subcommand has its own tests
                out.append((c, tag, r["argv"]))
    return out


def bed_to_vcf(prefix: str, out_path: str, ds: bool = False) -> None:
    """The same genotypes as a gzip-compressed VCF: ALT = A1 (the counted
    allele), REF = A2, IDs and positions from the .bim. With `ds` every record
    also carries FORMAT/DS with the same dosages ("." where the call is
    missing), which the program then reads instead of GT. The index next to
    it (needed by cis scans) holds no sequences: records are read in file
    order."""
    from eqtl_b200 import synth
    rows, n_file, fam, bim = R.read_bed(prefix)
    i = np.arange(n_file)
    codes = (rows[:, i // 4] >> (2 * (i % 4))) & 3
    dosage = np.array([2, -1, 1, 0], np.int8)[codes]
    dsv = np.where(dosage < 0, np.nan, dosage.astype(np.float64)) if ds else None
    synth.write_vcf(out_path, fam, [b[0] for b in bim], [b[3] for b in bim], [b[1] for b in bim],
                    [b[5] for b in bim], [b[4] for b in bim], dosage, ds=dsv)
    synth.write_tabix_header(out_path)


def _run(argv, case_dir, out_prefix, src="bed", tmp=None):
    a = list(argv)
    a[a.index("-o") + 1] = out_prefix
    if src in ("vcf", "vcf_ds"):  # the same genotypes through -v (GT, or DS)
        vcf = os.path.join(str(tmp), "geno.vcf.gz" if src == "vcf" else "geno_ds.vcf.gz")
        if not os.path.exists(vcf):
            bed_to_vcf(os.path.join(case_dir, a[a.index("-b") + 1]), vcf, ds=src == "vcf_ds")
        k = a.index("-b")
        a[k:k + 2] = ["-v", vcf]
    r = subprocess.run([os.path.abspath(BIN)] + a, cwd=case_dir, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.gpu
@pytest.mark.parametrize("src", ["bed", "vcf", "vcf_ds"])
@pytest.mark.parametrize("case,tag,argv", [r for r in _runs() if "--make-grm" in r[2]])
def test_cli_make_grm(case, tag, argv, src, tmp_path):
    d = os.path.join(GOLD, case)
    out = str(tmp_path / "out")
    _run(argv, d, out, src, tmp_path)
    ref = os.path.join(d, f"ref_{tag}")
    assert open(out + ".grm.id").read() == open(ref + ".grm.id").read()
    N, Nr = (np.fromfile(p + ".grm.N.bin", dtype=np.float32) for p in (out, ref))
    assert np.array_equal(N, Nr)
    K, Kr = (np.fromfile(p + ".grm.bin", dtype=np.float32) for p in (out, ref))
    np.testing.assert_allclose(K, Kr, rtol=0, atol=2e-6 * np.abs(Kr).max())


@pytest.mark.gpu
@pytest.mark.parametrize("src", ["bed", "vcf", "vcf_ds"])
@pytest.mark.parametrize("case,tag,argv", [r for r in _runs() if "--make-grm" not in r[2]])
def test_cli_scan_matches_reference(case, tag, argv, src, tmp_path):
    d = os.path.join(GOLD, case)
    out = str(tmp_path / "out")
    _run(argv, d, out, src, tmp_path)
    opt = refargs.options_from_argv(argv, d)
    ora = driver.Scanner(opt)
    ora.run()                                    # per-gene ACAT sensitivities
    scopes = ["gw"] if not opt.gff else {"cis": ["cis"], "trans": ["trans"], "gw": ["gw"],
                                         "all": ["cis", "trans"]}[opt.mode]
    errs = []
    for model in opt.out_models:
        tol = tsvcmp.Tol(log10p=1e-5, beta_rel=1e-6) if model == "lm" else tsvcmp.Tol(log10p=1e-4, beta_rel=1e-5)
        for scope in scopes:
            ref, got = os.path.join(d, f"ref_{tag}.{model}.{scope}"), f"{out}.{model}.{scope}"
            pthr = opt.pval_cis if scope == "cis" else opt.pval_trans
            for kind in ("pairs", "top"):
                hr, rr = tsvcmp.read_tsv(f"{ref}.{kind}.tsv")
                hg, gg = tsvcmp.read_tsv(f"{got}.{kind}.tsv")
                assert hr == hg
                errs += [f"{model}.{scope} {kind}: {e}" for e in tsvcmp.compare_pairs(rr, gg, tol, pthr)]
            hr, rr = tsvcmp.read_tsv(f"{ref}.region.tsv")
            hg, gg = tsvcmp.read_tsv(f"{got}.region.tsv")
            assert hr == hg
            exact_perm = model == "lm"
            errs += [f"{model}.{scope} region: {e}" for e in
                     tsvcmp.compare_region(rr, gg, tsvcmp.Tol(log10p=1e-3), check_perm=exact_perm,
                                           acat_sens=ora.sens, t_err=T_ERR)]
            if not exact_perm:
                R = {r[0]: r for r in rr}
                for g in gg:
                    if g[0] in R and R[g[0]][7] != "NA":
                        assert g[7] != "NA", (model, scope, g[0])
            # the gene order of each file is the reference's
            assert [r[0] for r in rr] == [g[0] for g in gg], (model, scope)
    assert not errs, "\n".join(errs[:40])


def test_cli_help_and_refusals():
    """Host-only behaviour of the command line (no GPU needed)."""
    exe = os.path.abspath(BIN)
    if not os.path.exists(exe):
        pytest.skip("eqtl_b200/bin/eqtl not built")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--pval-cis" in r.stdout
    r = subprocess.run([exe, "-v", "x.vcf.gz", "-e", "p.tsv"], capture_output=True, text=True)
    assert r.returncode == 1 and "VCF" in r.stderr
    r = subprocess.run([exe, "-b", "geno"], capture_output=True, text=True)
    assert r.returncode == 1 and "missing -e/--pheno" in r.stderr
    r = subprocess.run([exe, "-b", "geno", "-e", "p.tsv", "--model", "glmm"], capture_output=True, text=True)
    assert r.returncode == 1 and "glmm" in r.stderr
    r = subprocess.run([exe, "-b", "geno", "-e", "p.tsv", "--model", "lm,glm", "--pheno-norm", "int"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "--pheno-norm int is incompatible with count model glm" in r.stderr
    r = subprocess.run([exe, "-b", "geno", "-e", "p.tsv", "--maf", "0.7"], capture_output=True, text=True)
    assert r.returncode == 1 and "--maf must be in [0,0.5]" in r.stderr
